// Column-blocked LM fit kernel for the separable Gaussian PSF models.
//
// A group of G lanes owns one ROI at a time (several groups per warp). Lane l owns the CPL
// consecutive columns l*CPL .. l*CPL+CPL-1: it computes their x-terms (pixel-integrated
// Gaussian, its x/sigma derivatives) into registers, computes the y-terms of the rows with
// the same indices into shared memory, and then walks all R rows, reading one y-term
// (broadcast inside the group) and CPL samples per row. The Hessian/gradient partial sums
// stay in registers and are reduced with shfl.xor inside the group; every lane then runs
// the damped K x K solve redundantly, so all lanes of a group take the same decisions.
//
// The loop is flat: one trip = one LM iteration (or the Fisher pass) of every group in the
// warp; a group whose ROI has finished loads the next one at the top of the next trip, so
// groups never wait for their warp-mates to converge. The LM launches take ROIs one at a time
// from a per-launch counter (FitArgs::claim); the Fisher launches assign them statically:
// group g processes ROIs g, g + total_groups, ...
//
// Semantics follow photonpy's LevMarOptimize (Estimators/Estimation.h:104-134, 194-251);
// see fit_common.cuh for the solve and models.cuh for the per-pixel arithmetic.
#pragma once
#include "fit_common.cuh"
#include "models.cuh"

namespace pb200 {

// Shared-memory floats of one group: pixels, then max(y-terms, FP64 re-solve scratch,
// Fisher scratch when the pixel area cannot hold it). The launches space the groups by a
// stride of at least this many floats chosen against bank conflicts (gauss_group_stride).
template <int K>
__host__ __device__ constexpr int gauss_group_base_floats(int R) {
    return round_up(round_up(R * R, 4) + cmax(cmax(4 * R, rescue_floats(K)),
                                              (round_up(R * R, 4) >= 4 * K * K) ? 0 : 4 * K * K),
                    4);
}


// ---------------------------------------------------------------------------------------
// Separable accumulation of the Poisson Hessian and gradient.
//
// Every Gaussian model's Jacobian is J = C v over the "virtual" columns
//   v = [X.z Y.x, X.x Y.z, X.x Y.x, 1, X.w Y.x, X.x Y.w]
// of x-terms X (the pixel's column) and y-terms Y (its row); V = 4 for the fixed-sigma
// models, 6 otherwise, and C is a 0/1 selection for XYIBg and SigmaXY, a sum of the two sigma
// columns (times I) for one free sigma, and a dsigma/dz combination of them for astig. Each
// sum_p w v_i v_j is (product of y-factors) * sum over the row's columns of w * (product of
// x-factors); per pixel only the distinct x-factor products are accumulated (10, or 6), and
// the y-factors are applied once per row. Per pixel that is about 31 FP32 operations for
// SigmaXY instead of the 44 of a per-pixel Jacobian outer product; the sums are the same
// terms in another order.
// ---------------------------------------------------------------------------------------
__host__ __device__ constexpr int gauss_virtual_cols(int mid) {
    return (mid == MODEL_XYIBG || mid == MODEL_XYIBG_CONSTSIGMA) ? 4 : 6;
}

// T (per row): sum over columns of w times the distinct x-factor products, in the order
//   V = 6: zz, zx, z, zw, xx, x, xw, 1, w, ww       V = 4: zz, zx, z, xx, x, 1
template <int V>
__device__ __forceinline__ void row_add_w(float (&T)[V == 6 ? 10 : 6], float w, const float4& X) {
    const float wz = w * X.z, wx = w * X.x;
    T[0] += wz * X.z;
    T[1] += wz * X.x;
    T[2] += wz;
    if constexpr (V == 6) {
        const float ww = w * X.w;
        T[3] += wz * X.w;
        T[4] += wx * X.x;
        T[5] += wx;
        T[6] += wx * X.w;
        T[7] += w;
        T[8] += ww;
        T[9] += ww * X.w;
    } else {
        T[3] += wx * X.x;
        T[4] += wx;
        T[5] += w;
    }
}

// U (per row): sum over columns of bf = 1 - x/mu times the distinct x-factors z, x, 1 (, w).
template <int V>
__device__ __forceinline__ void row_add_b(float (&U)[V == 6 ? 4 : 3], float bf, const float4& X) {
    U[0] += bf * X.z;
    U[1] += bf * X.x;
    U[2] += bf;
    if constexpr (V == 6) U[3 % (V == 6 ? 4 : 3)] += bf * X.w;
}

// Applies one row's y-factors. av = [alpha_v packed upper (V(V+1)/2) | beta_v (V) | chi^2].
template <int V>
__device__ __forceinline__ void row_finish(float* av, const float (&T)[V == 6 ? 10 : 6],
                                           const float (&U)[V == 6 ? 4 : 3], const float4& Y) {
    const float xx = Y.x * Y.x, xz = Y.x * Y.z, zz = Y.z * Y.z;
    if constexpr (V == 6) {
        const float xw = Y.x * Y.w, zw = Y.z * Y.w, ww = Y.w * Y.w;
        av[0] += xx * T[0];
        av[1] += xz * T[1];
        av[2] += xx * T[1];
        av[3] += Y.x * T[2];
        av[4] += xx * T[3];
        av[5] += xw * T[1];
        av[6] += zz * T[4];
        av[7] += xz * T[4];
        av[8] += Y.z * T[5];
        av[9] += xz * T[6];
        av[10] += zw * T[4];
        av[11] += xx * T[4];
        av[12] += Y.x * T[5];
        av[13] += xx * T[6];
        av[14] += xw * T[4];
        av[15] += T[7];
        av[16] += Y.x * T[8];
        av[17] += Y.w * T[5];
        av[18] += xx * T[9];
        av[19] += xw * T[6];
        av[20] += ww * T[4];
        av[21] -= Y.x * U[0];
        av[22] -= Y.z * U[1];
        av[23] -= Y.x * U[1];
        av[24] -= U[2];
        av[25] -= Y.x * U[3 % (V == 6 ? 4 : 3)];
        av[26] -= Y.w * U[1];
    } else {
        av[0] += xx * T[0];
        av[1] += xz * T[1];
        av[2] += xx * T[1];
        av[3] += Y.x * T[2];
        av[4] += zz * T[3];
        av[5] += xz * T[3];
        av[6] += Y.z * T[4];
        av[7] += xx * T[3];
        av[8] += Y.x * T[4];
        av[9] += T[5];
        av[10] -= Y.x * U[0];
        av[11] -= Y.z * U[1];
        av[12] -= Y.x * U[1];
        av[13] -= U[2];
    }
}

// Model Hessian/gradient (acc = [alpha packed | beta | chi^2], K parameters) from the
// virtual ones: alpha = C alpha_v C^T, beta = C beta_v.
template <class M, int NV, int NACC>
__device__ __forceinline__ void map_virtual(const float (&av)[NV], float (&acc)[NACC], const M& m) {
    constexpr int MID = M::kId;
    constexpr int K = M::K;
    constexpr int V = gauss_virtual_cols(MID);
    constexpr int NAV = V * (V + 1) / 2;
    constexpr int NA = K * (K + 1) / 2;
    if constexpr (MID == MODEL_XYIBG || MID == MODEL_XYIBG_CONSTSIGMA || MID == MODEL_XYIBG_SIGMAXY) {
#pragma unroll
        for (int q = 0; q < NACC; q++) acc[q] = av[q];
    } else {
        // model column k is virtual column src(k), or (for k == kc) c4 v4 + c5 v5
        constexpr int kc = (MID == MODEL_XYZIBG) ? 2 : 4;
        float c4, c5;
        if constexpr (MID == MODEL_XYZIBG) {
            c4 = m.tI * m.dsxz;
            c5 = m.tI * m.dsyz;
        } else {
            c4 = m.tI;
            c5 = m.tI;
        }
        auto src = [](int k) constexpr -> int {
            return (MID == MODEL_XYZIBG) ? (k < 2 ? k : k - 1) : k;  // astig: x, y, (z), I, bg
        };
#pragma unroll
        for (int i = 0; i < K; i++) {
#pragma unroll
            for (int j = i; j < K; j++) {
                const int q = upk(i, j, K);
                if (i != kc && j != kc) {
                    acc[q] = av[upk(src(i), src(j), V)];
                } else if (i == kc && j == kc) {
                    acc[q] = c4 * c4 * av[upk(4, 4, V)] + 2.0f * c4 * c5 * av[upk(4, 5, V)] +
                             c5 * c5 * av[upk(5, 5, V)];
                } else {
                    const int o = (i == kc) ? src(j) : src(i);
                    acc[q] = c4 * av[upk(o, 4, V)] + c5 * av[upk(o, 5, V)];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < K; k++)
            acc[NA + k] = (k == kc) ? c4 * av[NAV + 4] + c5 * av[NAV + 5] : av[NAV + src(k)];
        acc[NACC - 1] = av[NV - 1];
    }
}

// Fit the ROIs roi, roi + roiStep, ... < roiEnd of one (model, ROI size) with one group of G
// lanes (`lane`, `mask`) and its shared-memory area `spix` (gauss_group_base_floats floats). With
// `claim` set, the group instead takes its ROIs, the first included, from that counter, roiStep
// consecutive ROIs per atomicAdd of the group's first lane, so groups refill from a shared pool
// until it runs out. STREAM: the ROIs are still arriving (streamFlags, see wait_stream_ready);
// a group waits for each claimed ROI and reads its samples from L2.
template <class M, int G, int CPL, int PASS = PASS_BOTH, bool STREAM = false>
__device__ __forceinline__ void gauss_fit_range(const ModelDesc& d, const FitArgs& a, int roi, const int roiEnd,
                                                const int roiStep, float* spix, const int lane, const unsigned mask,
                                                int* claim = nullptr, int* streamFlags = nullptr) {
    int claimEnd = 0;
    auto claim_next = [&]() -> int {
        int r = 0;
        if (lane == 0) {
            r = atomicAdd(claim, roiStep);
            if constexpr (STREAM) {
                // a group that gives up waiting ends; the host reads the error flag
                if (r < roiEnd && !wait_stream_ready(streamFlags, min(r + roiStep, roiEnd) - 1)) r = roiEnd;
            }
        }
        r = __shfl_sync(mask, r, 0, G);
        claimEnd = r + roiStep;
        return r;
    };
    if (claim) roi = claim_next();
    constexpr int K = M::K;
    constexpr int NA = K * (K + 1) / 2;
    constexpr int NACC = NA + K + 1;
    constexpr int NC = model_num_consts(M::kId);
    enum { MODE_LM = 0, MODE_FISHER = 1, MODE_SKIP = 2, MODE_LOAD = 3, MODE_IDLE = 4 };
    const int R = d.roisize;
    const int npix = R * R;
    const int npix4 = round_up(npix, 4);
    float* aux = spix + npix4;  // y-terms (R float4), or the FP64 re-solve scratch
    float4* ytab = reinterpret_cast<float4*>(aux);
    float* fisherScratch = (npix4 >= 4 * K * K) ? spix : aux;
    const int c0 = lane * CPL;
    constexpr bool kLM = PASS != PASS_FISHER, kFisher = PASS != PASS_LM;
    const bool fisherOnly = PASS == PASS_FISHER || (PASS == PASS_BOTH && (a.flags & FIT_CRLB_ONLY) != 0);
    const bool wantFisher = kFisher && (a.crlb || a.glrt);
    const bool haveSmp = a.smp != nullptr;
    const bool glrt = a.glrt != nullptr;  // needs samples (checked by the host)
    const bool vec4 = ((npix & 3) == 0) && ((reinterpret_cast<uintptr_t>(a.smp) & 15) == 0);
    const bool rowVec4 = (CPL == 4) && ((R & 3) == 0) && (c0 + 4 <= R);

    float th[K];
    float cs[NC > 0 ? NC : 1];
    int it = 0;
    int mode = MODE_LOAD;
    bool rescuedAny = false;

    while (true) {
        if (mode == MODE_LOAD && roi >= roiEnd) mode = MODE_IDLE;
        if (mode == MODE_LOAD) {
            __syncwarp(mask);  // the previous ROI's readers are done with spix/aux
            if (haveSmp) {
                const float* src = a.smp + (size_t)roi * npix;
                if (vec4) {
                    const float4* s4 = reinterpret_cast<const float4*>(src);
                    float4* d4 = reinterpret_cast<float4*>(spix);
                    for (int i = lane; i < (npix >> 2); i += G) d4[i] = STREAM ? __ldcg(s4 + i) : __ldcs(s4 + i);
                } else {
                    for (int i = lane; i < npix; i += G) spix[i] = STREAM ? __ldcg(src + i) : __ldcs(src + i);
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
                for (int y = 0; y < R; y++) {
#pragma unroll
                    for (int q = 0; q < CPL; q++) {
                        const int x = c0 + q;
                        if (x < R) {
                            const float v = spix[y * R + x];
                            sx += (float)x * v;
                            sy += (float)y * v;
                            s += v;
                        }
                    }
                }
                sx = group_sum<G>(sx, mask);
                sy = group_sum<G>(sy, mask);
                s = group_sum<G>(s, mask);
                M::initial(d, __fdiv_rn(sx, s), __fdiv_rn(sy, s), s, th);
            }
            it = 0;
            rescuedAny = false;
            if (fisherOnly) mode = MODE_FISHER;
            else if (a.maxIter <= 0) mode = wantFisher ? MODE_FISHER : MODE_SKIP;
            else mode = MODE_LM;
        }
        // The groups of a warp leave together: a group without ROIs idles until its warp-mates
        // are done. So every lane of the warp passes this point once per trip, and the warp is
        // reconverged here before the pixel pass (groups that loaded a ROI this trip would
        // otherwise run the pass apart from the others).
        if (__all_sync(0xffffffffu, mode == MODE_IDLE)) break;
        __syncwarp();

        if (mode == MODE_LM || mode == MODE_FISHER) {
            if (mode == MODE_LM && a.trace && lane == 0 && it < a.traceLen) {
#pragma unroll
                for (int k = 0; k < K; k++) a.trace[((size_t)roi * a.traceLen + it) * K + k] = th[k];
            }
            M m;
            m.template begin_group<G>(d, th, cs, lane, mask);
            float4 X[CPL], Yown[CPL];
            m.template term_block<CPL>(c0, m.tx, m.cx1, m.cx2, m.sigx, m.gax, X);
            m.template term_block<CPL>(c0, m.ty, m.cy1, m.cy2, m.sigy, m.gay, Yown);
            __syncwarp(mask);  // previous readers of ytab / scratch are done
#pragma unroll
            for (int q = 0; q < CPL; q++)
                if (c0 + q < R) ytab[c0 + q] = Yown[q];
            __syncwarp(mask);

            constexpr int V = gauss_virtual_cols(M::kId);
            constexpr int NV = V * (V + 1) / 2 + V + 1;
            constexpr int NT = (V == 6) ? 10 : 6;
            constexpr int NU = (V == 6) ? 4 : 3;
            float av[NV];
#pragma unroll
            for (int q = 0; q < NV; q++) av[q] = 0.0f;
            const bool lm = kLM && (!kFisher || mode == MODE_LM);
            if (c0 < R) {
                for (int y = 0; y < R; y++) {
                    const float4 Y = ytab[y];
                    float sv[CPL];
                    if (!haveSmp) {
#pragma unroll
                        for (int q = 0; q < CPL; q++) sv[q] = 0.0f;
                    } else if (rowVec4) {
                        const float4 s4 = *reinterpret_cast<const float4*>(spix + y * R + c0);
                        sv[0] = s4.x;
                        sv[1 % CPL] = s4.y;
                        sv[2 % CPL] = s4.z;
                        sv[3 % CPL] = s4.w;
                    } else {
#pragma unroll
                        for (int q = 0; q < CPL; q++) sv[q] = (c0 + q < R) ? spix[y * R + c0 + q] : 0.0f;
                    }
                    float T[NT], U[NU];
#pragma unroll
                    for (int q = 0; q < NT; q++) T[q] = 0.0f;
#pragma unroll
                    for (int q = 0; q < NU; q++) U[q] = 0.0f;
#pragma unroll
                    for (int q = 0; q < CPL; q++) {
                        if (CPL > 1 && c0 + q >= R) continue;
                        const float mu = fmaf(X[q].y, Y.x, m.tbg);  // tbg + (tI*DeltaX)*DeltaY
                        const float s = sv[q];
                        float w;
                        if (lm) {
                            // ComputeLevMarAlphaBeta (Estimation.h:109-128); a NaN sample counts as 1e-6
                            const float sval = fmaxf(s, 1e-6f);
                            const float muc = fmaxf(mu, 1e-6f);
                            const float invmu = lm_rcp(muc);
                            const float t = __fmul_rn(sval, invmu);
                            w = __fmul_rn(t, invmu);
                            row_add_b<V>(U, __fsub_rn(1.0f, t), X[q]);
                        } else {
                            // ComputeChiSquareAndCRLB (Estimation.h:76-95)
                            const float mu8 = fmaxf(1e-8f, mu);
                            w = rcp_nr(mu8);
                            if (haveSmp) {
                                const float e = s - mu8;
                                av[NV - 1] += __fdiv_rn(e * e, mu8);
                            }
                        }
                        row_add_w<V>(T, w, X[q]);
                    }
                    row_finish<V>(av, T, U, Y);
                }
            }
#pragma unroll
            for (int q = 0; q < NV; q++) av[q] = group_sum<G>(av[q], mask);
            float acc[NACC];
            map_virtual<M>(av, acc, m);

            if (lm) {
                float step[K], dk[K];
                int rc = lm_solve<K, NACC>(acc, a.lambda, step, dk);
                if (rc == 2) {
                    rc = lm_rescue<K, NACC>(acc, dk, step, aux, lane, mask) ? 1 : 0;
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
                if (glrt) {
                    // likelihood-ratio terms at the final parameters (GLRT_PSF.cu:112-124), in a
                    // pass of their own so that the LM pixel loop stays free of them
                    float on = 0.0f, sd = 0.0f, sr = 0.0f;
                    if (c0 < R) {
                        for (int y = 0; y < R; y++) {
                            const float4 Y = ytab[y];
#pragma unroll
                            for (int q = 0; q < CPL; q++) {
                                if (c0 + q >= R) continue;
                                float mu, J[K];
                                m.pixel_xy(X[q], Y, mu, J);
                                const float s = spix[y * R + c0 + q];
                                const float mu8 = fmaxf(mu, 1e-8f), d8 = fmaxf(s, 1e-8f);
                                on += d8 * logf(mu8) - mu8;
                                sd += d8;
                                sr += s;
                            }
                        }
                    }
                    glrt_store(group_sum<G>(on, mask), group_sum<G>(sd, mask), group_sum<G>(sr, mask), a, roi, npix,
                               lane);
                }
                if (a.fisher) fisher_store<K, NACC, G>(acc, a.fisher + (size_t)roi * (NA + 1), lane);
                else if (a.crlb) fisher_finish<K, NACC>(acc, fisherScratch, lane, mask, a.crlb + (size_t)roi * K,
                                                        a.chisq ? a.chisq + roi : nullptr);
            }
        }
        if (mode == MODE_IDLE) continue;
        if (lane == 0 && !fisherOnly) {
#pragma unroll
            for (int k = 0; k < K; k++) a.params[(size_t)roi * K + k] = th[k];
            if (a.iterations) a.iterations[roi] = it + 1;
            if (a.diag) a.diag[roi] = rescuedAny ? 1 : 0;
        }
        roi = claim ? (roi + 1 < claimEnd ? roi + 1 : claim_next()) : roi + roiStep;
        mode = MODE_LOAD;
    }
}


// Standalone launch: every group of the grid strides over the whole batch.
template <class M, int G, int CPL, int PASS>
__global__ void __launch_bounds__(256) gauss_fit_kernel(const ModelDesc d, const FitArgs a) {
    extern __shared__ __align__(16) float sm[];
    const int lane = threadIdx.x & (G - 1);
    const int gib = threadIdx.x / G;
    const int gpb = blockDim.x / G;
    // LM launches with a counter: one ROI per claim, so groups (and the warps and blocks they
    // share) run out of work within one ROI of each other instead of after a fixed list whose
    // iteration counts differ. The Fisher pass costs the same for every ROI and keeps the fixed
    // assignment.
    int* claim = PASS == PASS_LM ? a.claim : nullptr;
    gauss_fit_range<M, G, CPL, PASS>(d, a, claim ? 0 : blockIdx.x * gpb + gib, a.n, claim ? 1 : gridDim.x * gpb,
                                     sm + gib * a.smemStride, lane, group_mask<G>(), claim);
}

// LM launch over ROIs that a copy engine is still bringing in (host calls, see host_fit_streamed
// in estimator.cu): flags[1 + b] is set once ROI block b has arrived, flags[0] reports a wait
// that ran out. Groups take ROIs from the counter a.claim as in gauss_fit_kernel.
template <class M, int G, int CPL>
__global__ void __launch_bounds__(256) gauss_fit_stream_kernel(const ModelDesc d, const FitArgs a, int* flags) {
    extern __shared__ __align__(16) float sm[];
    const int lane = threadIdx.x & (G - 1);
    const int gib = threadIdx.x / G;
    gauss_fit_range<M, G, CPL, PASS_LM, true>(d, a, 0, a.n, 1, sm + gib * a.smemStride, lane, group_mask<G>(), a.claim,
                                              flags);
}

}  // namespace pb200
