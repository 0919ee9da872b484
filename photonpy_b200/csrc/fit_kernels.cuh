// Batched Levenberg-Marquardt Poisson-MLE fit, Fisher/CRLB and model-evaluation kernels.
//
// Work decomposition (sm_100a): a group of G lanes (G = 4, 8, 16 or 32; several groups
// per warp for small ROIs) owns one ROI at a time. The ROI's pixels are staged in shared
// memory with coalesced loads, the separable per-iteration table is built cooperatively,
// each lane accumulates the Poisson gradient/Hessian terms of its pixels in registers and
// a register butterfly (shfl.xor inside the group) reduces them. Every lane of the group
// then runs the tiny damped K x K Cholesky solve redundantly, so the decision to stop is
// identical on all lanes without a broadcast.
//
// The loop is flat: one trip = one LM iteration (or the Fisher pass) for every group of
// the warp, and a group whose ROI has finished loads its next ROI at the top of the next
// trip. Groups never wait for their warp-mates' ROIs to converge.
//
// Reference semantics kept (Estimators/Estimation.h:104-134, 194-251):
//  * sample clamped at 1e-6, mu clamped at 1e-6, x_f2 = (x*invmu)*invmu, beta -= (1 - x*invmu)*J;
//  * damping lambda>0: alpha_kk += lambda * sum_j alpha_jk^2; lambda<0: alpha_kk -= lambda;
//  * Cholesky fails (LM stops) only on an exactly-zero pivot (SolveMatrix.h:107-125);
//  * theta += step, model CheckLimits, stop when i > 0 and every |delta_k| <= StopLimit(k);
//  * iterations = i + 1 (maxIterations + 1 when the cap is hit); trace[i] = theta at the
//    start of iteration i for i < traceBufLen.
// Changes by design: pixel sums are reduced in a tree instead of sequentially; a Cholesky
// pivot that loses more than 6 decimal digits (0 < v < 1e-6 * a_kk, or v < 0) is re-solved in
// FP64; the Fisher matrix is accumulated in FP32 and inverted in FP64 (LUP with partial
// pivoting and the reference's 1e-9 tolerance, Estimation.h:63-102, SolveMatrix.h:411-452).
#pragma once
#include <type_traits>

#include "fit_common.cuh"
#include "models.cuh"

namespace pb200 {

// Models whose per-spot constants are a whole image (read per pixel, not held in registers).
template <class M, class = void>
struct pixel_consts_trait : std::false_type {};
template <class M>
struct pixel_consts_trait<M, std::void_t<decltype(M::kPixelConsts)>> : std::integral_constant<bool, M::kPixelConsts> {};
template <class M>
__host__ __device__ constexpr bool model_has_pixel_consts() {
    return pixel_consts_trait<M>::value;
}

// Models that evaluate several pixels per call (M::kPixelBlock, M::pixel_block<PB>).
template <class M, class = void>
struct pixel_block_trait : std::integral_constant<int, 1> {};
template <class M>
struct pixel_block_trait<M, std::void_t<decltype(M::kPixelBlock)>> : std::integral_constant<int, M::kPixelBlock> {};

// Shared-memory scratch a group needs besides its pixels: the model table, or the FP64
// Fisher/LM work area (2*K*K doubles + K doubles), whichever is larger.
template <class M>
__host__ __device__ constexpr int group_scratch_floats(int R) {
    return M::table_floats(R) > (4 * M::K * M::K + 2 * M::K + 4) ? M::table_floats(R)
                                                                   : (4 * M::K * M::K + 2 * M::K + 4);
}

template <class M>
__host__ __device__ constexpr int group_smem_floats(int R) {
    return round_up(round_up(R * R, 4) + group_scratch_floats<M>(R), 32) + 8;
}

template <class M, int G, int PASS>
__global__ void __launch_bounds__(256) fit_kernel(const ModelDesc d, const FitArgs a) {
    constexpr int K = M::K;
    constexpr int NA = K * (K + 1) / 2;
    constexpr int NACC = NA + K + 1;
    constexpr int NC = model_num_consts(M::kId);
    enum { MODE_LM = 0, MODE_FISHER = 1, MODE_SKIP = 2, MODE_LOAD = 3, MODE_IDLE = 4 };
    extern __shared__ __align__(16) float sm[];

    const int lane = threadIdx.x & (G - 1);
    const int gib = threadIdx.x / G;
    const int gpb = blockDim.x / G;
    const unsigned mask = group_mask<G>();
    const int R = d.roisize;
    const int npix = R * R;
    float* spix = sm + gib * a.smemStride;
    float* tab = spix + round_up(npix, 4);  // model table, or FP64 work area after a reduction
    const int gstride = gridDim.x * gpb;
    const int dx = G % R, dy = G / R;
    const int x0 = lane % R, y0 = lane / R;
    constexpr bool kLM = PASS != PASS_FISHER, kFisher = PASS != PASS_LM;
    const bool fisherOnly = PASS == PASS_FISHER || (PASS == PASS_BOTH && (a.flags & FIT_CRLB_ONLY) != 0);
    const bool wantFisher = kFisher && (a.crlb || a.glrt);
    const bool haveSmp = a.smp != nullptr;
    const bool glrt = a.glrt != nullptr;  // needs samples (checked by the host)
    const bool vec4 = ((npix & 3) == 0) && ((reinterpret_cast<uintptr_t>(a.smp) & 15) == 0);

    // LM launches with a counter take one ROI per claim (see gauss_fit_kernel). Not the spline
    // models: with 16 lanes per ROI a warp holds two ROIs, whose iteration counts spread little
    // (a fixed assignment keeps 99% of the lanes busy), and the counter's register made the
    // LM instance spill (4.83 against 5.25 M ROIs/s for 13x13 ROIs).
    constexpr bool kClaims = PASS == PASS_LM && !model_is_spline(M::kId);
    int roi = blockIdx.x * gpb + gib;
    if constexpr (kClaims) {
        if (a.claim) roi = group_claim<G>(a.claim, 1, lane, mask);
    }
    float th[K];
    float cs[NC > 0 ? NC : 1];
    int it = 0;
    int mode = MODE_LOAD;
    bool rescuedAny = false;

    while (true) {
        if (mode == MODE_LOAD && roi >= a.n) mode = MODE_IDLE;
        if (mode == MODE_LOAD) {
            // ---- load the next ROI into shared memory and set the start parameters ----
            __syncwarp(mask);  // previous ROI's readers are done with spix/tab
            const float* src = haveSmp ? a.smp + (size_t)roi * npix : nullptr;
            if (haveSmp) {
                if (vec4) {
                    const float4* s4 = reinterpret_cast<const float4*>(src);
                    float4* d4 = reinterpret_cast<float4*>(spix);
                    for (int i = lane; i < (npix >> 2); i += G) d4[i] = __ldcs(s4 + i);
                } else {
                    for (int i = lane; i < npix; i += G) spix[i] = __ldcs(src + i);
                }
            }
#pragma unroll
            for (int c = 0; c < NC; c++) cs[c] = a.consts[(size_t)roi * NC + c];
            if (a.initial) {
#pragma unroll
                for (int k = 0; k < K; k++) th[k] = a.initial[(size_t)roi * K + k];
            } else {
                __syncwarp(mask);
                // centre of mass (Estimation.h:336-352); exact for integer-valued samples
                float sx = 0.0f, sy = 0.0f, s = 0.0f;
                int x = x0, y = y0;
                for (int p = lane; p < npix; p += G) {
                    const float v = spix[p];
                    sx += (float)x * v;
                    sy += (float)y * v;
                    s += v;
                    x += dx;
                    y += dy;
                    if (x >= R) { x -= R; y++; }
                }
                sx = group_sum<G>(sx, mask);
                sy = group_sum<G>(sy, mask);
                s = group_sum<G>(s, mask);
                M::initial(d, __fdiv_rn(sx, s), __fdiv_rn(sy, s), s, th);
            }
            it = 0;
            rescuedAny = false;
            if (fisherOnly) mode = MODE_FISHER;
            else if (a.maxIter <= 0) mode = wantFisher ? MODE_FISHER : MODE_SKIP;  // start value, iterations = 1
            else mode = MODE_LM;
        }
        // The groups of a warp leave together (an idle group waits for its warp-mates), so every
        // lane passes this point once per trip and the warp reconverges before the pixel pass.
        if (__all_sync(0xffffffffu, mode == MODE_IDLE)) break;
        __syncwarp();

        if (mode == MODE_LM || mode == MODE_FISHER) {
            if (mode == MODE_LM && a.trace && lane == 0 && it < a.traceLen) {
#pragma unroll
                for (int k = 0; k < K; k++) a.trace[((size_t)roi * a.traceLen + it) * K + k] = th[k];
            }
            // ---- per-iteration table, then the pixel pass ----
            M m;
            m.begin(d, th, cs);
            if constexpr (model_has_pixel_consts<M>()) m.img = a.consts + (size_t)roi * npix;
            __syncwarp(mask);
            m.build_table(d, tab, lane, G);
            __syncwarp(mask);

            float acc[NACC];
#pragma unroll
            for (int q = 0; q < NACC; q++) acc[q] = 0.0f;
            const bool lm = kLM && (!kFisher || mode == MODE_LM);
            // one pixel's terms; a lane visits its pixels lane, lane + G, ... in this order
            auto accumulate = [&](float mu, const float (&J)[K], float s) {
                float w;
                if (lm) {
                    // ComputeLevMarAlphaBeta (Estimation.h:109-128)
                    const float sv = s < 1e-6f ? 1e-6f : s;
                    const float muc = mu > 1e-6f ? mu : 1e-6f;
                    const float invmu = PB200_LM_IEEE_RCP ? __frcp_rn(muc) : rcp_nr(muc);
                    const float t = __fmul_rn(sv, invmu);
                    w = __fmul_rn(t, invmu);
                    const float bf = __fsub_rn(1.0f, t);
#pragma unroll
                    for (int k = 0; k < K; k++) acc[NA + k] -= bf * J[k];
                } else {
                    // ComputeChiSquareAndCRLB (Estimation.h:76-95)
                    const float mu8 = fmaxf(1e-8f, mu);
                    w = rcp_nr(mu8);
                    if (haveSmp) {
                        const float e = s - mu8;
                        acc[NACC - 1] += __fdiv_rn(e * e, mu8);
                    }
                }
                int q = 0;
#pragma unroll
                for (int i = 0; i < K; i++) {
                    const float wi = J[i] * w;
#pragma unroll
                    for (int j = i; j < K; j++) acc[q++] += wi * J[j];
                }
            };
            constexpr int PB = pixel_block_trait<M>::value;
            if constexpr (PB > 1) {
                for (int p0 = lane; p0 < npix; p0 += G * PB) {
                    int xs[PB], ys[PB];
#pragma unroll
                    for (int t = 0; t < PB; t++) {
                        const int p = p0 + G * t;
                        ys[t] = p / R;
                        xs[t] = p - ys[t] * R;
                    }
                    float mus[PB], Js[PB][K];
                    m.template pixel_block<PB>(d, tab, xs, ys, mus, Js);
#pragma unroll
                    for (int t = 0; t < PB; t++) {
                        const int p = p0 + G * t;
                        if (p < npix) accumulate(mus[t], Js[t], haveSmp ? spix[p] : 0.0f);
                    }
                }
            } else {
                int x = x0, y = y0;
                for (int p = lane; p < npix; p += G) {
                    float mu, J[K];
                    m.pixel(d, tab, x, y, mu, J);
                    accumulate(mu, J, haveSmp ? spix[p] : 0.0f);
                    x += dx;
                    y += dy;
                    if (x >= R) { x -= R; y++; }
                }
            }
#pragma unroll
            for (int q = 0; q < NACC; q++) acc[q] = group_sum<G>(acc[q], mask);

            if (lm) {
                float step[K], dk[K];
                int rc = lm_solve<K, NACC>(acc, a.lambda, step, dk);
                if (rc == 2) {
                    rc = lm_rescue<K, NACC>(acc, dk, step, tab, lane, mask) ? 1 : 0;
                    if (rc) rescuedAny = true;
                }
                bool done;
                if (rc == 0) {
                    done = true;  // the reference breaks out with iterations = i + 1
                } else {
                    float last[K];
#pragma unroll
                    for (int k = 0; k < K; k++) {
                        last[k] = th[k];
                        th[k] = th[k] + step[k];
                    }
                    M::check_limits(d, th);
                    bool small = true;
#pragma unroll
                    for (int k = 0; k < K; k++)
                        if (fabsf(last[k] - th[k]) > M::stop_limit(k)) small = false;
                    done = (it > 0 && small);
                    if (!done) {
                        it++;
                        if (it >= a.maxIter) {
                            done = true;
                            it = a.maxIter;  // iterations = maxIterations + 1
                        }
                    }
                }
                if (!done) continue;
                if (wantFisher) {
                    mode = MODE_FISHER;
                    continue;
                }
            } else {
                // ---- Fisher pass: deferred FP64 inverse (crlb_kernel), or on lane 0 ----
                if (glrt) {
                    // likelihood-ratio terms at the final parameters (GLRT_PSF.cu:112-124), in a
                    // pass of their own so that the LM pixel loop stays free of them
                    float on = 0.0f, sd = 0.0f, sr = 0.0f;
                    int gx = x0, gy = y0;
                    for (int p = lane; p < npix; p += G) {
                        float mu, J[K];
                        m.pixel(d, tab, gx, gy, mu, J);
                        const float s = spix[p];
                        const float mu8 = fmaxf(mu, 1e-8f), d8 = fmaxf(s, 1e-8f);
                        on += d8 * logf(mu8) - mu8;
                        sd += d8;
                        sr += s;
                        gx += dx;
                        gy += dy;
                        if (gx >= R) { gx -= R; gy++; }
                    }
                    glrt_store(group_sum<G>(on, mask), group_sum<G>(sd, mask), group_sum<G>(sr, mask), a, roi, npix,
                               lane);
                }
                if (a.fisher) fisher_store<K, NACC, G>(acc, a.fisher + (size_t)roi * (NA + 1), lane);
                else if (a.crlb) fisher_finish<K, NACC>(acc, tab, lane, mask, a.crlb + (size_t)roi * K,
                                                        a.chisq ? a.chisq + roi : nullptr);
            }
        }
        if (mode == MODE_IDLE) continue;
        // ---- ROI finished: write results, move to the next ROI ----
        if (lane == 0 && !fisherOnly) {
#pragma unroll
            for (int k = 0; k < K; k++) a.params[(size_t)roi * K + k] = th[k];
            if (a.iterations) a.iterations[roi] = it + 1;
            if (a.diag) a.diag[roi] = rescuedAny ? 1 : 0;
        }
        if constexpr (kClaims) roi = a.claim ? group_claim<G>(a.claim, 1, lane, mask) : roi + gstride;
        else roi += gstride;
        mode = MODE_LOAD;
    }
}

// ExpectedValue / Derivatives (Estimation.h:159-181; layouts ev[n][H][W], deriv[n][K][H][W]).
template <class M, int G>
__global__ void __launch_bounds__(256) eval_kernel(const ModelDesc d, const float* __restrict__ params,
                                                   const float* __restrict__ consts, float* __restrict__ ev,
                                                   float* __restrict__ deriv, int n, int smemStride) {
    constexpr int K = M::K;
    constexpr int NC = model_num_consts(M::kId);
    extern __shared__ __align__(16) float sm[];
    const int lane = threadIdx.x & (G - 1);
    const int gib = threadIdx.x / G;
    const int gpb = blockDim.x / G;
    const unsigned mask = group_mask<G>();
    const int R = d.roisize, npix = R * R;
    float* tab = sm + gib * smemStride;
    for (int roi = blockIdx.x * gpb + gib; roi < n; roi += gridDim.x * gpb) {
        float th[K], cs[NC > 0 ? NC : 1];
#pragma unroll
        for (int k = 0; k < K; k++) th[k] = params[(size_t)roi * K + k];
#pragma unroll
        for (int c = 0; c < NC; c++) cs[c] = consts[(size_t)roi * NC + c];
        M m;
        m.begin(d, th, cs);
        if constexpr (model_has_pixel_consts<M>()) m.img = consts + (size_t)roi * npix;
        __syncwarp(mask);
        m.build_table(d, tab, lane, G);
        __syncwarp(mask);
        for (int p = lane; p < npix; p += G) {
            float mu, J[K];
            m.pixel(d, tab, p % R, p / R, mu, J);
            if (ev) __stcs(ev + (size_t)roi * npix + p, mu);
            if (deriv) {
#pragma unroll
                for (int k = 0; k < K; k++) __stcs(deriv + ((size_t)roi * K + k) * npix + p, J[k]);
            }
        }
    }
}

}  // namespace pb200
