// One persistent launch over a batch that mixes PSF models and ROI sizes.
//
// The batch is split into buckets of one (model, ROI size) each. Every warp walks the buckets
// in order; inside a bucket its G-lane groups take ROIs one at a time from the bucket's counter
// (gauss_fit_range with `claim`), so all groups of a warp run the same model code, refill
// without waiting for each other, and the warp moves on only when the bucket's ROIs are all
// taken. The handler of a bucket is its model and CPL = ceil(R / G) columns per lane; G = 4
// covers ROI sizes up to 16 pixels. Buckets of 7 to 10 pixels run 2 lanes of 4 or 5 columns
// per ROI instead (the per-bucket launches' default for these sizes, so that both forms give the
// same results): the two 2-lane groups of a 4-lane slot split its shared memory in halves. A
// batch runs as two such launches, the LM pass over every bucket and then the Fisher/CRLB pass at
// the fitted parameters, each with single-pass handlers (see FitPass).
#pragma once
#include "fit_common.cuh"
#include "gauss_fit.cuh"
#include "models.cuh"

namespace pb200 {

struct MixedTask {
    ModelDesc d;
    FitArgs a;      // a.n = bucket size; a.fisher = this bucket's scratch rows
    int handler;    // model * 8 + (CPL - 1) for 4 lanes per ROI, model * 8 + 4 + (CPL - 4) for 2 lanes
};

__host__ __device__ constexpr int mixed_handler(int model, int lanes, int cpl) {
    return model * 8 + (lanes == 2 ? 4 + cpl - 4 : cpl - 1);
}

// One (model, CPL) handler: inlined into the kernel's switch, or compiled as its own function
// (register-allocated on its own) when NOINL is set.
template <class M, int G, int CPL, int PASS>
__device__ __forceinline__ void mixed_handler_inl(const MixedTask* __restrict__ T, int* claim, int chunk, float* spix,
                                                  int lane, unsigned mask) {
    gauss_fit_range<M, G, CPL, PASS>(T->d, T->a, 0, T->a.n, chunk, spix, lane, mask, claim);
}
template <class M, int G, int CPL, int PASS>
__device__ __noinline__ void mixed_handler_call(const MixedTask* __restrict__ T, int* claim, int chunk, float* spix,
                                                int lane, unsigned mask) {
    gauss_fit_range<M, G, CPL, PASS>(T->d, T->a, 0, T->a.n, chunk, spix, lane, mask, claim);
}

// Kernel variants: (THREADS, MINB) launch bounds fix the register budget; NOINL picks the
// handler form. Variant 0: 128 threads, 3 blocks/SM, inlined; 1: 256 threads, 2 blocks/SM,
// separate handlers; 2: 128 threads, 4 blocks/SM, separate handlers.
// counters[b] counts the ROIs of bucket b already taken (zeroed before each launch); a group
// takes `chunk` consecutive ROIs per claim.
template <int G, int THREADS, int MINB, bool NOINL, int PASS>
__global__ void __launch_bounds__(THREADS, MINB) mixed_fit_kernel(const MixedTask* __restrict__ tasks, int ntasks,
                                                                  int* __restrict__ counters, int chunk,
                                                                  int strideFloats) {
    extern __shared__ __align__(16) float sm[];
    const int lane = threadIdx.x & (G - 1);
    const int gib = threadIdx.x / G;
    const unsigned mask = group_mask<G>();
    const unsigned mask2 = group_mask<2>();
    float* spix = sm + gib * strideFloats;
    for (int b = 0; b < ntasks; b++) {
        // skip a bucket whose ROIs are all taken without touching its code
        int taken = 0;
        if ((threadIdx.x & 31) == 0) taken = *(volatile int*)(counters + b);
        taken = __shfl_sync(0xffffffffu, taken, 0);
        const MixedTask& T = tasks[b];
        if (taken >= T.a.n) continue;
        int* claim = counters + b;
#define PB_MIXED_CASE(MID, CPLV)                                                                         \
    case mixed_handler(MID, G, CPLV):                                                                    \
        if (NOINL) mixed_handler_call<GaussModel<MID>, G, CPLV, PASS>(&T, claim, chunk, spix, lane, mask); \
        else mixed_handler_inl<GaussModel<MID>, G, CPLV, PASS>(&T, claim, chunk, spix, lane, mask);        \
        break;
#define PB_MIXED_CASE2(MID, CPLV)                                                                         \
    case mixed_handler(MID, 2, CPLV):                                                                     \
        if constexpr (G == 4) {                                                                           \
            float* half = spix + (lane >> 1) * (strideFloats >> 1);                                       \
            if (NOINL) mixed_handler_call<GaussModel<MID>, 2, CPLV, PASS>(&T, claim, chunk, half, lane & 1, mask2); \
            else mixed_handler_inl<GaussModel<MID>, 2, CPLV, PASS>(&T, claim, chunk, half, lane & 1, mask2);        \
        }                                                                                                 \
        break;
#define PB_MIXED_MODEL(MID) PB_MIXED_CASE(MID, 1) PB_MIXED_CASE(MID, 2) PB_MIXED_CASE(MID, 3) PB_MIXED_CASE(MID, 4) \
    PB_MIXED_CASE2(MID, 4) PB_MIXED_CASE2(MID, 5)
        switch (T.handler) {
            PB_MIXED_MODEL(MODEL_XYIBG)
            PB_MIXED_MODEL(MODEL_XYIBG_CONSTSIGMA)
            PB_MIXED_MODEL(MODEL_XYIBG_SIGMA)
            PB_MIXED_MODEL(MODEL_XYIBG_SIGMAXY)
            PB_MIXED_MODEL(MODEL_XYZIBG)
        default:
            break;
        }
#undef PB_MIXED_MODEL
#undef PB_MIXED_CASE
#undef PB_MIXED_CASE2
        __syncwarp();
    }
}

}  // namespace pb200
