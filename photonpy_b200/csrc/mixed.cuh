// One persistent launch over a batch that mixes PSF models and ROI sizes.
//
// The batch is split into buckets of one (model, ROI size) each, and every bucket into tiles
// of `tileRois` ROIs. Warps claim tiles from a global counter (one atomicAdd per tile, lane
// 0, broadcast with a shuffle); the G-lane groups of the warp then fit that tile's ROIs with
// per-group refill (gauss_fit_range), so all groups of a warp run the same model code and
// only wait for each other at tile boundaries. The handler of a bucket is its model and
// CPL = ceil(R / G) columns per lane; G = 4 covers ROI sizes up to 16 pixels.
#pragma once
#include "fit_common.cuh"
#include "gauss_fit.cuh"
#include "models.cuh"

namespace pb200 {

struct MixedTask {
    ModelDesc d;
    FitArgs a;      // a.n = bucket size; a.fisher = this bucket's scratch rows
    int tileBegin;  // first global tile of this bucket (buckets are stored in tile order)
    int handler;    // model * 4 + (CPL - 1)
};

// One (model, CPL) handler: inlined into the kernel's switch, or compiled as its own function
// (register-allocated on its own) when NOINL is set.
template <class M, int G, int CPL>
__device__ __forceinline__ void mixed_handler_inl(const MixedTask* __restrict__ T, int roi0, int end, float* spix,
                                                  int lane, unsigned mask) {
    gauss_fit_range<M, G, CPL>(T->d, T->a, roi0, end, 32 / G, spix, lane, mask);
}
template <class M, int G, int CPL>
__device__ __noinline__ void mixed_handler_call(const MixedTask* __restrict__ T, int roi0, int end, float* spix,
                                                int lane, unsigned mask) {
    gauss_fit_range<M, G, CPL>(T->d, T->a, roi0, end, 32 / G, spix, lane, mask);
}

// Kernel variants: (THREADS, MINB) launch bounds fix the register budget; NOINL picks the
// handler form. Variant 0: 128 threads, 3 blocks/SM, inlined; 1: 256 threads, 2 blocks/SM,
// separate handlers; 2: 128 threads, 4 blocks/SM, separate handlers.
template <int G, int THREADS, int MINB, bool NOINL>
__global__ void __launch_bounds__(THREADS, MINB) mixed_fit_kernel(const MixedTask* __restrict__ tasks, int ntasks,
                                                        int totalTiles, int tileRois, int* __restrict__ tileCounter,
                                                        int strideFloats) {
    extern __shared__ __align__(16) float sm[];
    constexpr int GPW = 32 / G;
    const int lane = threadIdx.x & (G - 1);
    const int gib = threadIdx.x / G;
    const int giw = (threadIdx.x & 31) / G;
    const unsigned mask = group_mask<G>();
    float* spix = sm + gib * strideFloats;
    while (true) {
        int t = 0;
        if ((threadIdx.x & 31) == 0) t = atomicAdd(tileCounter, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= totalTiles) break;
        int b = 0;
        while (b + 1 < ntasks && tasks[b + 1].tileBegin <= t) b++;
        const MixedTask& T = tasks[b];
        const int start = (t - T.tileBegin) * tileRois;
        const int end = min(start + tileRois, T.a.n);
        const int roi0 = start + giw;
#define PB_MIXED_CASE(MID, CPLV)                                                                          \
    case MID * 4 + CPLV - 1:                                                                              \
        if (NOINL) mixed_handler_call<GaussModel<MID>, G, CPLV>(&T, roi0, end, spix, lane, mask);         \
        else mixed_handler_inl<GaussModel<MID>, G, CPLV>(&T, roi0, end, spix, lane, mask);                \
        break;
#define PB_MIXED_MODEL(MID) PB_MIXED_CASE(MID, 1) PB_MIXED_CASE(MID, 2) PB_MIXED_CASE(MID, 3) PB_MIXED_CASE(MID, 4)
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
        __syncwarp();
    }
}

}  // namespace pb200
