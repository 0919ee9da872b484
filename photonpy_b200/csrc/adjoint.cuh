// Adjoint of the summed Poisson negative log-likelihood (new functionality; photonpy has no
// gradient with respect to its calibration).
//
//   NLL_n = sum_p [ mu_p - x_p log(max(mu_p, 1e-6)) ]          (constant terms dropped)
//   dNLL_n/dmu_p = r_p = 1 - x_p / max(mu_p, 1e-6)
//
// Per spot: dtheta_k = g_n sum_p r_p dmu_p/dtheta_k (true derivatives: for the free-sigma
// models the reference's Jacobian column, sigma * dmu/dsigma, is divided by sigma).
// Calibration (summed over spots, g_n = upstream gradient of spot n):
//   XYIBg        d/dsigma_x, d/dsigma_y  via dDelta/dsigma of the pixel-integrated Gaussian
//   XYZIBg       d/d(s0, gamma, d, A, B) for x and y: dmu/dsigma (the reference's G21 terms,
//                GaussianPSFModels.h:715-742) times dsigma/dcoefficient of
//                sigma = s0 sqrt(1 + t^2/d^2 + A t^3/d^2 + B t^4/d^4), t = z - gamma
//   CSpline      d/dcoef[k][j][i][m] = sum g_n r_p I delta_f[m] over the pixels that read voxel
//                (k, j, i) (zero where the PSF value is clamped at 0), scattered with 16-byte
//                vector atomics; optionally also the diagonal of the Fisher information with
//                respect to the coefficients, sum g_n I^2 delta_f[m]^2 / mu_p (the Gauss-Newton
//                curvature a calibration step divides by)
// Nothing per pixel is stored: mu and its derivatives are recomputed from the model table.
#pragma once
#include "fit_common.cuh"
#include "models.cuh"

namespace pb200 {

struct AdjointArgs {
    const float* smp;      // [n][npix]
    const float* params;   // [n][K]
    const float* consts;   // [n][numconst] or null
    const float* gradOut;  // [n] upstream gradient of each spot's NLL, or null (= 1)
    float* nll;            // [n] or null
    float* dparams;        // [n][K] or null
    float* dcalib;         // XYIBg [2], XYZIBg [10], CSpline [Nz*Ny*Nx*64], or null; accumulated into
    float* curv;           // CSpline only: [Nz*Ny*Nx*64] Fisher diagonal of the coefficients, or null;
                           // accumulated into
    int n;
    int smemStride;        // floats per group (model table + extra sigma-derivative table)
};

template <class M>
__host__ __device__ constexpr int adjoint_group_floats(int R) {
    return round_up(M::table_floats(R) + 2 * R, 32) + 8;
}

template <class M, int G>
__global__ void __launch_bounds__(256) adjoint_kernel(const ModelDesc d, const AdjointArgs a) {
    constexpr int K = M::K;
    constexpr int NC = model_num_consts(M::kId);
    constexpr int MID = M::kId;
    constexpr bool kSigmaCal = (MID == MODEL_XYIBG);
    constexpr bool kAstig = (MID == MODEL_XYZIBG);
    constexpr bool kSpline = (MID == MODEL_CSPLINE);
    constexpr int NCAL = kSigmaCal ? 2 : (kAstig ? 10 : 0);
    extern __shared__ __align__(16) float sm[];
    __shared__ float blockCal[10];
    const int lane = threadIdx.x & (G - 1);
    const int gib = threadIdx.x / G;
    const int gpb = blockDim.x / G;
    const unsigned mask = group_mask<G>();
    const int R = d.roisize, npix = R * R;
    float* tab = sm + gib * a.smemStride;
    float* dsig = tab + M::table_floats(R);  // [2R]: dDelta/dsigma per column, then per row (XYIBg)
    if (threadIdx.x < 10) blockCal[threadIdx.x] = 0.0f;
    __syncthreads();

    for (int roi = blockIdx.x * gpb + gib; roi < a.n; roi += gridDim.x * gpb) {
        float th[K], cs[NC > 0 ? NC : 1];
#pragma unroll
        for (int k = 0; k < K; k++) th[k] = a.params[(size_t)roi * K + k];
#pragma unroll
        for (int c = 0; c < NC; c++) cs[c] = a.consts[(size_t)roi * NC + c];
        M m;
        m.begin(d, th, cs);
        __syncwarp(mask);
        m.build_table(d, tab, lane, G);
        if constexpr (kSigmaCal) {
            // dDelta/dsigma = (e1 exp(-e1^2) - e0 exp(-e0^2)) / (sqrt(pi) sigma), e = (c - t -+ 0.5)/(sqrt(2) sigma)
            for (int i = lane; i < 2 * R; i += G) {
                const bool isx = i < R;
                const int c = isx ? i : i - R;
                const float t = isx ? th[0] : th[1];
                const float s = isx ? d.sigma[0] : d.sigma[1];
                const float k1 = 1.0f / (sqrtf(2.0f) * s);
                const float e0 = ((float)c - t + 0.5f) * k1, e1 = ((float)c - t - 0.5f) * k1;
                dsig[i] = (e1 * expf(-e1 * e1) - e0 * expf(-e0 * e0)) * (0.5641895835477563f / s);
            }
        }
        __syncwarp(mask);
        float acc[K], cal[2] = {0.0f, 0.0f}, nll = 0.0f;
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] = 0.0f;
        const float g = a.gradOut ? a.gradOut[roi] : 1.0f;
        const float* smp = a.smp + (size_t)roi * npix;
        for (int p = lane; p < npix; p += G) {
            const int x = p % R, y = p / R;
            float mu, J[K];
            m.pixel(d, tab, x, y, mu, J);
            const float xs = smp[p];
            const float muc = fmaxf(mu, 1e-6f);
            const float r = 1.0f - xs / muc;
            nll += mu - xs * logf(muc);
#pragma unroll
            for (int k = 0; k < K; k++) acc[k] += r * J[k];
            if constexpr (kSigmaCal) {
                const float4 X = reinterpret_cast<const float4*>(tab)[x];
                const float4 Y = reinterpret_cast<const float4*>(tab)[R + y];
                cal[0] += r * th[2] * Y.x * dsig[x];
                cal[1] += r * th[2] * X.x * dsig[R + y];
            } else if constexpr (kAstig) {
                const float4 X = reinterpret_cast<const float4*>(tab)[x];
                const float4 Y = reinterpret_cast<const float4*>(tab)[R + y];
                cal[0] += r * Y.y * X.w;  // (tI DeltaY) G21x = dmu/dsigma_x
                cal[1] += r * X.y * Y.w;  // (tI DeltaX) G21y = dmu/dsigma_y
            } else if constexpr (kSpline) {
                if ((a.dcalib || a.curv) && J[3] > 0.0f) {  // J[3] is the PSF value, clamped at 0 by the model
                    const size_t off = m.coef_offset(x, y);
                    const float4* df = reinterpret_cast<const float4*>(tab);
                    if (a.dcalib) {
                        const float w = g * r * th[3];
                        float4* dst = reinterpret_cast<float4*>(a.dcalib + off);
#pragma unroll 4
                        for (int q = 0; q < 16; q++) {
                            const float4 f = df[q];
                            atomicAdd(dst + q, make_float4(w * f.x, w * f.y, w * f.z, w * f.w));
                        }
                    }
                    if (a.curv) {
                        const float w2 = g * th[3] * th[3] / muc;
                        float4* dst = reinterpret_cast<float4*>(a.curv + off);
#pragma unroll 4
                        for (int q = 0; q < 16; q++) {
                            const float4 f = df[q];
                            atomicAdd(dst + q, make_float4(w2 * f.x * f.x, w2 * f.y * f.y, w2 * f.z * f.z, w2 * f.w * f.w));
                        }
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] = group_sum<G>(acc[k], mask);
        nll = group_sum<G>(nll, mask);
        cal[0] = group_sum<G>(cal[0], mask);
        cal[1] = group_sum<G>(cal[1], mask);
        if (lane == 0) {
            if (MID == MODEL_XYIBG_SIGMA) acc[4 % K] /= th[4 % K];
            if (MID == MODEL_XYIBG_SIGMAXY) {
                acc[4 % K] /= th[4 % K];
                acc[5 % K] /= th[5 % K];
            }
            if (a.dparams) {
#pragma unroll
                for (int k = 0; k < K; k++) a.dparams[(size_t)roi * K + k] = g * acc[k];
            }
            if (a.nll) a.nll[roi] = nll;
            if (a.dcalib && kSigmaCal) {
                atomicAdd(&blockCal[0], g * cal[0]);
                atomicAdd(&blockCal[1], g * cal[1]);
            }
            if (a.dcalib && kAstig) {
                // dsigma/d(s0, gamma, d, A, B) at this spot's z, for x then y
#pragma unroll
                for (int ax = 0; ax < 2; ax++) {
                    const float* c = ax == 0 ? d.astig_x : d.astig_y;
                    const float s0 = c[0], dd = c[2], A = c[3], B = c[4];
                    const float t = th[2] - c[1];
                    const float d2 = dd * dd, d3 = d2 * dd, d4 = d2 * d2, d5 = d4 * dd;
                    const float t2 = t * t, t3 = t2 * t, t4 = t2 * t2;
                    const float q = 1.0f + t2 / d2 + A * t3 / d2 + B * t4 / d4;
                    const float sq = sqrtf(q);
                    const float h = s0 / (2.0f * sq);
                    const float dqdt = 2.0f * t / d2 + 3.0f * A * t2 / d2 + 4.0f * B * t3 / d4;
                    const float dqdd = -2.0f * t2 / d3 - 2.0f * A * t3 / d3 - 4.0f * B * t4 / d5;
                    const float ds[5] = {sq, -h * dqdt, h * dqdd, h * t3 / d2, h * t4 / d4};
                    const float gs = g * cal[ax];
#pragma unroll
                    for (int j = 0; j < 5; j++) atomicAdd(&blockCal[ax * 5 + j], gs * ds[j]);
                }
            }
        }
    }
    if (NCAL > 0) {
        __syncthreads();
        if (a.dcalib && threadIdx.x < NCAL) atomicAdd(&a.dcalib[threadIdx.x], blockCal[threadIdx.x]);
    }
}

}  // namespace pb200
