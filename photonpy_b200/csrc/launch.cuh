// Kernel launchers: one persistent launch per (model, lanes per ROI, columns per lane).
// The grid is sized to the SM count times the resident blocks per SM; groups stride over the
// batch. Each model's launchers are instantiated in its own translation unit (k_*.cu).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

#include "fit_common.cuh"
#include "fit_kernels.cuh"
#include "adjoint.cuh"
#include "gauss_fit.cuh"
#include "models.cuh"

namespace pb200 {

using FitLaunch = void (*)(const ModelDesc&, FitArgs, int threads, cudaStream_t);
// LM launch over ROIs still arriving (gauss_fit_stream_kernel): FitArgs with a.claim set, the ready flags
using StreamLaunch = void (*)(const ModelDesc&, FitArgs, int* flags, int threads, cudaStream_t);
using AdjointLaunch = void (*)(const ModelDesc&, AdjointArgs, cudaStream_t);
using EvalLaunch = void (*)(const ModelDesc&, const float*, const float*, float*, float*, int, int threads,
                            cudaStream_t);

constexpr int kMaxSmemPerBlock = 200 * 1024;

int num_sms();        // estimator.cu
void count_launch();  // estimator.cu

inline void check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Zeroes the ROI counter of an LM launch (FitArgs::claim) on the launch's stream.
inline void reset_claim(int* claim, cudaStream_t s) {
    const cudaError_t e = cudaMemsetAsync(claim, 0, sizeof(int), s);
    if (e != cudaSuccess) throw std::runtime_error(std::string("ROI counter reset: ") + cudaGetErrorString(e));
}

// Opt the kernel in to more than 48 KB of dynamic shared memory. Set on every launch: the
// attribute is per kernel and per device, and the call costs about a microsecond.
template <class KernelT>
inline void set_smem_attr(KernelT kern, size_t smem) {
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) throw std::runtime_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    }
}

// Threads per block a group kernel launches with: the requested count, halved while the block's
// shared memory (threads / G groups of strideFloats floats) exceeds kMaxSmemPerBlock.
inline int launched_threads(int threads, int G, int strideFloats) {
    while ((size_t)(threads / G) * strideFloats * sizeof(float) > (size_t)kMaxSmemPerBlock && threads > 32)
        threads /= 2;
    return threads;
}

// Launch a persistent group kernel: `strideFloats` of shared memory per group of G lanes.
template <class KernelT, class... Extra>
inline void launch_groups(KernelT kern, int G, int threads, int strideFloats, int n, const ModelDesc& d, FitArgs a,
                          cudaStream_t s, Extra... extra) {
    threads = launched_threads(threads, G, strideFloats);
    const int gpb = threads / G;
    const size_t smem = (size_t)gpb * strideFloats * sizeof(float);
    if (smem > (size_t)kMaxSmemPerBlock || gpb < 1) throw std::runtime_error("ROI too large for shared memory");
    set_smem_attr(kern, smem);
    int perSM = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kern, threads, smem) != cudaSuccess || perSM < 1)
        throw std::runtime_error("fit kernel: occupancy query failed");
    const long long needed = ((long long)n + gpb - 1) / gpb;
    const long long cap = (long long)num_sms() * perSM;
    const int grid = (int)(needed < cap ? needed : cap);
    a.smemStride = strideFloats;
    kern<<<grid, threads, smem, s>>>(d, a, extra...);
    check_launch("fit kernel launch");
    count_launch();
}

// Arguments of the LM launch (no Fisher outputs) and of the Fisher launch at the fitted
// parameters (FIT_CRLB_ONLY, parameters read from the LM launch's output).
inline FitArgs lm_pass_args(const FitArgs& a) {
    FitArgs lm = a;
    lm.crlb = nullptr;
    lm.fisher = nullptr;
    lm.glrt = nullptr;
    lm.glrtMeanRoi = nullptr;
    lm.chisq = nullptr;
    return lm;
}
inline FitArgs fisher_pass_args(const FitArgs& a) {
    FitArgs fi = a;
    fi.flags |= FIT_CRLB_ONLY;
    fi.initial = a.params;
    fi.params = nullptr;
    fi.iterations = nullptr;
    fi.trace = nullptr;
    fi.traceLen = 0;
    fi.diag = nullptr;
    fi.claim = nullptr;
    return fi;
}

// Split into single-pass launches as in launch_fit_gauss.
template <class M, int G>
void launch_fit_generic(const ModelDesc& d, FitArgs a, int threads, cudaStream_t s) {
    if (a.n <= 0) return;
    const int stride = group_smem_floats<M>(d.roisize);
    if (a.flags & FIT_CRLB_ONLY) {
        launch_groups(fit_kernel<M, G, PASS_FISHER>, G, threads, stride, a.n, d, a, s);
        return;
    }
    if (a.claim && !model_is_spline(M::kId)) reset_claim(a.claim, s);
    launch_groups(fit_kernel<M, G, PASS_LM>, G, threads, stride, a.n, d, lm_pass_args(a), s);
    if (a.crlb || a.glrt) launch_groups(fit_kernel<M, G, PASS_FISHER>, G, threads, stride, a.n, d, fisher_pass_args(a), s);
}

// Worst shared-memory bank conflict (threads per bank) of one warp of the column-blocked
// kernel's pixel pass with group stride S: the sample reads (lane l of group g reads row y at
// g*S + R*y + CPL*l + q, one float per column, or one float4 per row when CPL == 4 and R % 4
// == 0, served 8 threads at a time), plus the y-term float4 read (one address per group,
// broadcast to its lanes).
inline int gauss_stride_conflicts(int S, int npix4, int R, int G, int CPL) {
    const bool vec = CPL == 4 && (R & 3) == 0;
    int worst = 1;
    for (int y = 0; y < R; y++) {
        for (int q = 0; q < (vec ? 1 : CPL); q++) {
            for (int ph = 0; ph < (vec ? 4 : 1); ph++) {
                int count[32] = {0};
                const int t0 = vec ? ph * 8 : 0, t1 = vec ? t0 + 8 : 32;
                for (int t = t0; t < t1; t++) {
                    const int g = t / G, l = t % G, c = CPL * l + q;
                    if (c >= R) continue;
                    const int addr = g * S + R * y + c;
                    for (int w = 0; w < (vec ? 4 : 1); w++) worst = std::max(worst, ++count[(addr + w) & 31]);
                }
            }
        }
    }
    int ytab = 1;
    for (int ph = 0; ph < 4; ph++) {
        int count[32] = {0};
        for (int g = ph * 8 / G; g <= (ph * 8 + 7) / G; g++)
            for (int w = 0; w < 4; w++) ytab = std::max(ytab, ++count[(g * S + npix4 + w) & 31]);
    }
    return worst + ytab;
}

// Group stride of the single-model column-blocked launches: of base, base + 4, ... up to
// round_up(base, 32) + 16 floats (base = gauss_group_base_floats; the upper end keeps a block's
// shared memory, and so the block size that fits, no larger than with a fixed 16-mod-32 stride),
// the smallest with the fewest bank conflicts in the pixel pass. With the 16-mod-32 stride every
// second group of a warp read the same banks: 8-way conflicts on the sample reads of 2-lane
// groups, 4-way with 4 lanes of 3 columns.
template <int K>
int gauss_group_stride(int R, int G, int CPL) {
    static std::mutex mtx;
    static std::map<long long, int> cache;
    const long long key = ((long long)R << 16) | (G << 8) | CPL;
    std::lock_guard<std::mutex> lock(mtx);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    const int base = gauss_group_base_floats<K>(R), npix4 = round_up(R * R, 4);
    int best = base, bestCost = 1 << 30;
    const int last = round_up(base, 32) + 16;
    for (int S = base; S <= last; S += 4) {
        const int c = gauss_stride_conflicts(S, npix4, R, G, CPL);
        if (c < bestCost) {
            bestCost = c;
            best = S;
        }
    }
    cache[key] = best;
    return best;
}

// LM launch, then (when CRLB or GLRT values are requested) the Fisher launch at the fitted
// parameters, each with its single-pass kernel instance.
template <class M, int G, int CPL>
void launch_fit_gauss(const ModelDesc& d, FitArgs a, int threads, cudaStream_t s) {
    if (a.n <= 0) return;
    const int stride = gauss_group_stride<M::K>(d.roisize, G, CPL);
    if (a.flags & FIT_CRLB_ONLY) {
        launch_groups(gauss_fit_kernel<M, G, CPL, PASS_FISHER>, G, threads, stride, a.n, d, a, s);
        return;
    }
    if (a.claim) reset_claim(a.claim, s);
    launch_groups(gauss_fit_kernel<M, G, CPL, PASS_LM>, G, threads, stride, a.n, d, lm_pass_args(a), s);
    if (a.crlb || a.glrt)
        launch_groups(gauss_fit_kernel<M, G, CPL, PASS_FISHER>, G, threads, stride, a.n, d, fisher_pass_args(a), s);
}

template <class M, int G>
void launch_eval(const ModelDesc& d, const float* params, const float* consts, float* ev, float* deriv, int n,
                 int threads, cudaStream_t s) {
    if (n <= 0) return;
    auto kern = eval_kernel<M, G>;
    const int stride = round_up(M::table_floats(d.roisize), 32) + 8;
    const int gpb = threads / G;
    const size_t smem = (size_t)gpb * stride * sizeof(float);
    set_smem_attr(kern, smem);
    int perSM = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kern, threads, smem) != cudaSuccess || perSM < 1)
        throw std::runtime_error("eval kernel: occupancy query failed");
    const long long needed = ((long long)n + gpb - 1) / gpb;
    const long long cap = (long long)num_sms() * perSM * 4;
    const int grid = (int)(needed < cap ? needed : cap);
    kern<<<grid, threads, smem, s>>>(d, params, consts, ev, deriv, n, stride);
    check_launch("eval kernel launch");
    count_launch();
}

template <class M, int G>
void launch_adjoint(const ModelDesc& d, AdjointArgs a, cudaStream_t s) {
    if (a.n <= 0) return;
    auto kern = adjoint_kernel<M, G>;
    const int threads = 256;
    a.smemStride = adjoint_group_floats<M>(d.roisize);
    const int gpb = threads / G;
    const size_t smem = (size_t)gpb * a.smemStride * sizeof(float);
    set_smem_attr(kern, smem);
    int perSM = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kern, threads, smem) != cudaSuccess || perSM < 1)
        throw std::runtime_error("adjoint kernel: occupancy query failed");
    const long long needed = ((long long)a.n + gpb - 1) / gpb;
    const long long cap = (long long)num_sms() * perSM;
    const int grid = (int)(needed < cap ? needed : cap);
    kern<<<grid, threads, smem, s>>>(d, a);
    check_launch("adjoint kernel launch");
    count_launch();
}

// Columns per lane the column-blocked kernel is built for: up to 5 with 2 lanes per ROI (ROIs
// up to 10 pixels wide, 16 per warp), 4 with 4..16 lanes, 2 with 32.
inline int gauss_max_cpl(int G) { return G == 32 ? 2 : (G == 2 ? 5 : 4); }

// Gaussian models: column-blocked kernel with CPL = ceil(R / G) (1..gauss_max_cpl(G)).
template <class M>
FitLaunch gauss_fit_table(int G, int CPL) {
#define PB_CASE(g)                                    \
    case g:                                           \
        switch (CPL) {                                \
        case 1: return launch_fit_gauss<M, g, 1>;     \
        case 2: return launch_fit_gauss<M, g, 2>;     \
        case 3: return launch_fit_gauss<M, g, 3>;     \
        default: return launch_fit_gauss<M, g, 4>;    \
        }
    switch (G) {
    case 2:
        switch (CPL) {
        case 1: return launch_fit_gauss<M, 2, 1>;
        case 2: return launch_fit_gauss<M, 2, 2>;
        case 3: return launch_fit_gauss<M, 2, 3>;
        case 4: return launch_fit_gauss<M, 2, 4>;
        default: return launch_fit_gauss<M, 2, 5>;
        }
        PB_CASE(4)
        PB_CASE(8)
        PB_CASE(16)
    default:
        return CPL <= 1 ? launch_fit_gauss<M, 32, 1> : launch_fit_gauss<M, 32, 2>;
    }
#undef PB_CASE
}

template <class M, int G, int CPL>
void launch_fit_gauss_stream(const ModelDesc& d, FitArgs a, int* flags, int threads, cudaStream_t s) {
    if (a.n <= 0 || !a.claim) return;
    const int stride = gauss_group_stride<M::K>(d.roisize, G, CPL);
    reset_claim(a.claim, s);
    launch_groups(gauss_fit_stream_kernel<M, G, CPL>, G, threads, stride, a.n, d, lm_pass_args(a), s, flags);
}

// Streamed LM launchers of the 2- and 4-lane shapes (the default configurations up to 16 px);
// null for the others, whose host calls use the slot pipeline.
template <class M>
StreamLaunch gauss_stream_table(int G, int CPL) {
    if (G == 2) {
        switch (CPL) {
        case 1: return launch_fit_gauss_stream<M, 2, 1>;
        case 2: return launch_fit_gauss_stream<M, 2, 2>;
        case 3: return launch_fit_gauss_stream<M, 2, 3>;
        case 4: return launch_fit_gauss_stream<M, 2, 4>;
        default: return launch_fit_gauss_stream<M, 2, 5>;
        }
    }
    if (G == 4) {
        switch (CPL) {
        case 1: return launch_fit_gauss_stream<M, 4, 1>;
        case 2: return launch_fit_gauss_stream<M, 4, 2>;
        case 3: return launch_fit_gauss_stream<M, 4, 3>;
        default: return launch_fit_gauss_stream<M, 4, 4>;
        }
    }
    return nullptr;
}

template <class M>
FitLaunch generic_fit_table(int G) {
    switch (G) {
    case 2:  // the per-pixel table kernel starts at 4 lanes per ROI
    case 4: return launch_fit_generic<M, 4>;
    case 8: return launch_fit_generic<M, 8>;
    case 16: return launch_fit_generic<M, 16>;
    default: return launch_fit_generic<M, 32>;
    }
}

// Spline launchers: the reference-form instance (one voxel per pixel, OVS = false) unless the
// description carries a finer calibration (spline_q != 1), which runs the OVS instance.
template <int MODE, int G>
void launch_fit_spline(const ModelDesc& d, FitArgs a, int threads, cudaStream_t s) {
    if (d.spline_q == 1.0f) launch_fit_generic<SplineModelT<MODE, false>, G>(d, a, threads, s);
    else launch_fit_generic<SplineModelT<MODE, true>, G>(d, a, threads, s);
}
template <int MODE>
FitLaunch spline_fit_table(int G) {
    switch (G) {
    case 2:
    case 4: return launch_fit_spline<MODE, 4>;
    case 8: return launch_fit_spline<MODE, 8>;
    case 16: return launch_fit_spline<MODE, 16>;
    default: return launch_fit_spline<MODE, 32>;
    }
}
template <int MODE, int G>
void launch_eval_spline(const ModelDesc& d, const float* params, const float* consts, float* ev, float* deriv, int n,
                        int threads, cudaStream_t s) {
    if (d.spline_q == 1.0f) launch_eval<SplineModelT<MODE, false>, G>(d, params, consts, ev, deriv, n, threads, s);
    else launch_eval<SplineModelT<MODE, true>, G>(d, params, consts, ev, deriv, n, threads, s);
}
template <int MODE>
EvalLaunch spline_eval_table(int G) {
    switch (G) {
    case 8: return launch_eval_spline<MODE, 8>;
    case 16: return launch_eval_spline<MODE, 16>;
    default: return launch_eval_spline<MODE, 32>;
    }
}

template <class M>
EvalLaunch eval_table(int G) {
    switch (G) {
    case 8: return launch_eval<M, 8>;
    case 16: return launch_eval<M, 16>;
    default: return launch_eval<M, 32>;
    }
}

// FP64 CRLB from the packed Fisher scratch rows (one thread per ROI).
inline void launch_crlb(int K, const float* fisher, float* crlb, float* chisq, int n, cudaStream_t s,
                        bool absDiag = false) {
    if (n <= 0) return;
    const int threads = 128;
    const int grid = (n + threads - 1) / threads < 65535 * 4 ? (n + threads - 1) / threads : 65535 * 4;
    if (absDiag) {
        if (K != 2) throw std::runtime_error("crlb: |diag| form is provided for 2 parameters only");
        crlb_kernel<2, true><<<grid, threads, 0, s>>>(fisher, crlb, chisq, n);
        check_launch("crlb kernel launch");
        count_launch();
        return;
    }
    switch (K) {
    case 4: crlb_kernel<4><<<grid, threads, 0, s>>>(fisher, crlb, chisq, n); break;
    case 5: crlb_kernel<5><<<grid, threads, 0, s>>>(fisher, crlb, chisq, n); break;
    case 6: crlb_kernel<6><<<grid, threads, 0, s>>>(fisher, crlb, chisq, n); break;
    case 7: crlb_kernel<7><<<grid, threads, 0, s>>>(fisher, crlb, chisq, n); break;
    case 8: crlb_kernel<8><<<grid, threads, 0, s>>>(fisher, crlb, chisq, n); break;
    default: throw std::runtime_error("crlb: unsupported number of parameters");
    }
    check_launch("crlb kernel launch");
    count_launch();
}

inline int fisher_row_floats(int K) { return K * (K + 1) / 2 + 1; }

// Mixed-model persistent kernel (k_mixed.cu).
struct MixedTask;
int mixed_lanes();
void launch_mixed(const MixedTask* d_tasks, int ntasks, int totalClaims, int chunk, int* d_counters,
                  int strideFloats, int variant, bool fisherPass, cudaStream_t s);

// Per-model entry points (k_*.cu). `variant` 0 = column-blocked Gaussian kernel,
// 1 = generic table kernel (the only one for the spline).
FitLaunch fit_launcher_for(int model, int G, int CPL, int variant);
EvalLaunch eval_launcher_for(int model, int G);

#define PB_DECLARE_MODEL_LAUNCHERS(name)                               \
    FitLaunch fit_launcher_##name(int G, int CPL, int variant);        \
    StreamLaunch stream_launcher_##name(int G, int CPL);               \
    EvalLaunch eval_launcher_##name(int G);                            \
    AdjointLaunch adjoint_launcher_##name();
PB_DECLARE_MODEL_LAUNCHERS(xyibg)
PB_DECLARE_MODEL_LAUNCHERS(constsigma)
PB_DECLARE_MODEL_LAUNCHERS(sigma)
PB_DECLARE_MODEL_LAUNCHERS(sigmaxy)
PB_DECLARE_MODEL_LAUNCHERS(astig)
PB_DECLARE_MODEL_LAUNCHERS(spline)
#undef PB_DECLARE_MODEL_LAUNCHERS
FitLaunch fit_launcher_tilted(int G, int CPL, int variant);
FitLaunch fit_launcher_tilted_sxy(int G, int CPL, int variant);
FitLaunch fit_launcher_intensity_bg(int G);
FitLaunch fit_launcher_spline_tilted(int G);
FitLaunch fit_launcher_spline_bgimage(int G);
EvalLaunch eval_launcher_spline_tilted(int G);
EvalLaunch eval_launcher_spline_bgimage(int G);
EvalLaunch eval_launcher_tilted(int G);
EvalLaunch eval_launcher_tilted_sxy(int G);

}  // namespace pb200
