// Device-side PSF models for the batched Poisson-MLE estimator.
//
// Each model follows the per-pixel arithmetic of photonpy's models, operation by
// operation, with explicit round-to-nearest intrinsics so nvcc does not fuse the
// reference's separate multiplies and adds:
//   Gauss2D XYIBg / ConstSigma   Estimators/Gaussian/GaussianPSFModels.h:35-227
//   Gauss2D XYIBgSigma           Estimators/Gaussian/GaussianPSFModels.h:308-387
//   Gauss2D XYIBgSigmaXY         Estimators/Gaussian/GaussianPSFModels.h:391-471
//   Gauss2D XYZIBg (astigmatic)  Estimators/Gaussian/GaussianPSFModels.h:636-751
//   CSpline XYZIBg (flat bg)     Estimators/CSpline/CubicSplinePSFModels.h:14-154
//   CSpline XYZITiltedBg         Estimators/CSpline/CubicSplinePSFModels.h:157-298
//   CSpline XYZIBgImage          Estimators/CSpline/CubicSplinePSFModels.h:300-443
//   Gauss2D XYITiltedBg          Estimators/Gaussian/GaussianPSFModels.h:228-304
//   Gauss2D XYITiltedBgSigmaXY   Estimators/Gaussian/GaussianPSFModels.h:474-558
//   IntensityBgModel             Estimators/Gaussian/GaussianPSFModels.h:562-615
//
// B200 layout: the reference recomputes erf/exp for every pixel although they depend
// only on the column (x) or the row (y). Here a group of lanes first builds a small
// per-ROI-iteration table in shared memory (2R entries of 4 floats for the Gaussians,
// the 4x64 power-basis vectors for the spline), then each lane evaluates its pixels
// from the table. Table values are bit-identical to what the reference computes per
// pixel, so the per-pixel mu and Jacobian keep the reference's rounding (up to the
// last-ulp differences between CUDA's and glibc's erff/expf).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pb200 {

enum ModelId : int {
    MODEL_XYIBG = 0,
    MODEL_XYIBG_CONSTSIGMA = 1,
    MODEL_XYIBG_SIGMA = 2,
    MODEL_XYIBG_SIGMAXY = 3,
    MODEL_XYZIBG = 4,
    MODEL_CSPLINE = 5,
    MODEL_XYITILTEDBG = 6,
    MODEL_XYITILTEDBG_SIGMAXY = 7,
    MODEL_INTENSITYBG = 8,  // intensity and background at a known position and sigma
    MODEL_CSPLINE_TILTED = 9,
    MODEL_CSPLINE_BGIMAGE = 10,
    MODEL_COUNT = 11
};

__host__ __device__ constexpr bool model_is_spline(int m) {
    return m == MODEL_CSPLINE || m == MODEL_CSPLINE_TILTED || m == MODEL_CSPLINE_BGIMAGE;
}

// Plain-old-data description of one estimator instance, passed by value to kernels.
struct ModelDesc {
    int model;
    int roisize;
    float sigma[2];       // fixed sigma (XYIBg) or initial sigma(s) (Sigma / SigmaXY)
    float astig_x[5];     // s0, gamma, d, A, B  (B = 0 reproduces the reference's 4-term form)
    float astig_y[5];
    float minz, maxz;     // astig z clamp
    int spline_shape[3];  // Nz, Ny, Nx of the coefficient grid
    float spline_zmin, spline_zmax;
    const float* coefs;   // device, [Nz][Ny][Nx][64]
    // spline voxels per ROI pixel along x and y: 1 for photonpy's spline (one voxel per pixel); 2
    // for a calibration sampled at 0.5 px (extension; the reference has no xy scale)
    float spline_q;
    // device, the same coefficients q-major: float4 q (coefficients 4q..4q+3) of voxel v at
    // coefsQ[q * Nz*Ny*Nx + v], so that lanes reading neighbouring voxels read neighbouring
    // addresses (the fit kernels' copy; null when the caller supplies coefs directly)
    const float4* coefsQ;
    // fixed-sigma XYIBg: 1/(sqrt(2 pi) sigma_x), 1/(sqrt(2) sigma_x), then the same for y, computed
    // once per estimator with the reference's float operations (model_desc_fixed_sigma; all 0 when
    // not computed); the other models compute their scales per ROI and iteration
    float fixed_c[4];
};


__host__ __device__ constexpr int model_num_params(int m) {
    return (m == MODEL_XYIBG || m == MODEL_XYIBG_CONSTSIGMA)            ? 4
           : (m == MODEL_XYIBG_SIGMAXY || m == MODEL_XYITILTEDBG)       ? 6
           : (m == MODEL_XYITILTEDBG_SIGMAXY)                           ? 8
           : (m == MODEL_INTENSITYBG)                                   ? 2
           : (m == MODEL_CSPLINE_TILTED)                                ? 7
                                                                        : 5;
}
__host__ __device__ constexpr int model_num_consts(int m) {
    return (m == MODEL_XYIBG_CONSTSIGMA || m == MODEL_XYITILTEDBG) ? 2 : (m == MODEL_INTENSITYBG ? 3 : 0);
}

// MATH_PI in the reference is the float literal 3.141592653589793f (MathUtils.h:95).
#define PB_PI 3.141592653589793f
// sqrt(2 pi), sqrt(2) and 1/sqrt(pi) as the reference's float arithmetic produces them (IEEE
// square root and division of float operands, MATH_PI being the float literal above). Every set-up
// starts from these instead of recomputing them per ROI and iteration; PB200_CheckModelConstants
// compares them with the device's own __fsqrt_rn / __fdiv_rn results.
constexpr float kSqrt2Pi = 0x1.40d932p+1f;
constexpr float kSqrt2 = 0x1.6a09e6p+0f;
constexpr float kInvSqrtPi = 0x1.20dd74p-1f;

// Host side: the fixed-sigma scales of an XYIBg description from its sigma pair (IEEE float
// multiply and divide, as MUL/DIV on the device). Call whenever sigma changes.
inline void model_desc_fixed_sigma(ModelDesc& d) {
    d.fixed_c[0] = 1.0f / (kSqrt2Pi * d.sigma[0]);
    d.fixed_c[1] = 1.0f / (kSqrt2 * d.sigma[0]);
    d.fixed_c[2] = 1.0f / (kSqrt2Pi * d.sigma[1]);
    d.fixed_c[3] = 1.0f / (kSqrt2 * d.sigma[1]);
}
#define MUL(a, b) __fmul_rn((a), (b))
#define ADD(a, b) __fadd_rn((a), (b))
#define SUB(a, b) __fsub_rn((a), (b))
#define DIV(a, b) __fdiv_rn((a), (b))

// clamp(f,a,b) = fmaxf(a, fminf(f, b)), CudaMath.h:1152-1155 (NaN maps to b).
__device__ __forceinline__ float pb_clamp(float f, float a, float b) { return fmaxf(a, fminf(f, b)); }

// Gauss2D_Border = 1.5f; upper x/y limit = (R - 1.5f) - 1 (GaussianPSFModels.h:55-56).
__device__ __forceinline__ float gauss_xy_max(int R) { return SUB(SUB((float)R, 1.5f), 1.0f); }

// IEEE quotients q[i] = num[i] / den[i] of N divisions by the G lanes of a group (mask: the
// group's lanes) in ceil(N / G) rounds: in round r lane j divides pair r G + j, then every lane
// receives the round's quotients by shuffles. All lanes must pass the same N pairs.
template <int N, int G>
__device__ __forceinline__ void group_div(const float (&num)[N], const float (&den)[N], float (&q)[N], int lane,
                                          unsigned mask) {
#pragma unroll
    for (int r = 0; r < (N + G - 1) / G; r++) {
        float a = 1.0f, b = 1.0f;
#pragma unroll
        for (int j = 0; j < G && r * G + j < N; j++)
            if (lane == j) {
                a = num[r * G + j];
                b = den[r * G + j];
            }
        const float t = __fdiv_rn(a, b);
#pragma unroll
        for (int j = 0; j < G && r * G + j < N; j++) q[r * G + j] = __shfl_sync(mask, t, j, G);
    }
}

// ---------------------------------------------------------------------------------------
// Gaussian models: table = x-terms [R][4] then y-terms [R][4].
// ---------------------------------------------------------------------------------------
template <int MID>
struct GaussModel {
    static constexpr int K = model_num_params(MID);
    static constexpr int kId = MID;
    static __host__ __device__ constexpr int table_floats(int R) { return 8 * R; }

    // per ROI-iteration scalars
    float tx, ty, tI, tbg;
    float cx1, cx2, cy1, cy2;  // OneOverSqrt2SigmaX, OneOverSqrt2PiSigmaX, ... (Y)
    float invSqrtPi;
    float sigx, sigy;          // astig: sigma_x(z), sigma_y(z)
    float dsxz, dsyz;          // astig: dsigma/dz
    float gax, gay;            // astig: 1 / (sqrt(2 pi) sigma^2) of the G21 terms, x and y

    __device__ __forceinline__ void begin(const ModelDesc& d, const float* th, const float* consts) {
        tx = th[0];
        ty = th[1];
        const float s2pi = kSqrt2Pi;
        const float s2 = kSqrt2;
        if (MID == MODEL_XYZIBG) {
            tI = th[3];
            tbg = th[4];
            const float tz = th[2];
            const float s0x = d.astig_x[0], gx = d.astig_x[1], dx = d.astig_x[2], Ax = d.astig_x[3], Bx = d.astig_x[4];
            const float s0y = d.astig_y[0], gy = d.astig_y[1], dy = d.astig_y[2], Ay = d.astig_y[3], By = d.astig_y[4];
            const float dy2 = MUL(dy, dy), dx2 = MUL(dx, dx);
            const float dy4 = MUL(dy2, dy2), dx4 = MUL(dx2, dx2);
            const float tzx = SUB(tz, gx), tzx2 = MUL(tzx, tzx), tzx3 = MUL(tzx2, tzx), tzx4 = MUL(tzx2, tzx2);
            const float tzy = SUB(tz, gy), tzy2 = MUL(tzy, tzy), tzy3 = MUL(tzy2, tzy), tzy4 = MUL(tzy2, tzy2);
            // 1 + tz^2/d^2 + A tz^3/d^2 (+ B tz^4/d^4, which adds exactly 0 when B == 0)
            const float qx = ADD(ADD(ADD(1.0f, DIV(tzx2, dx2)), DIV(MUL(Ax, tzx3), dx2)), DIV(MUL(Bx, tzx4), dx4));
            const float qy = ADD(ADD(ADD(1.0f, DIV(tzy2, dy2)), DIV(MUL(Ay, tzy3), dy2)), DIV(MUL(By, tzy4), dy4));
            const float sqx = __fsqrt_rn(qx), sqy = __fsqrt_rn(qy);
            sigx = MUL(s0x, sqx);
            sigy = MUL(s0y, sqy);
            cx2 = DIV(1.0f, MUL(s2pi, sigx));
            cx1 = DIV(1.0f, MUL(s2, sigx));
            cy2 = DIV(1.0f, MUL(s2pi, sigy));
            cy1 = DIV(1.0f, MUL(s2, sigy));
            // s0 * (2 tz/d^2 + A*3*tz^2/d^2 + B*4*tz^3/d^4) / (2 sqrt(q))
            const float nx = ADD(ADD(DIV(MUL(2.0f, tzx), dx2), DIV(MUL(MUL(Ax, 3.0f), tzx2), dx2)),
                                 DIV(MUL(MUL(Bx, 4.0f), tzx3), dx4));
            const float ny = ADD(ADD(DIV(MUL(2.0f, tzy), dy2), DIV(MUL(MUL(Ay, 3.0f), tzy2), dy2)),
                                 DIV(MUL(MUL(By, 4.0f), tzy3), dy4));
            dsxz = DIV(MUL(s0x, nx), MUL(2.0f, sqx));
            dsyz = DIV(MUL(s0y, ny), MUL(2.0f, sqy));
            gax = DIV(1.0f, MUL(MUL(s2pi, sigx), sigx));
            gay = DIV(1.0f, MUL(MUL(s2pi, sigy), sigy));
        } else {
            tI = th[2];
            tbg = th[3];
            float sx, sy;
            if (MID == MODEL_XYIBG) { sx = d.sigma[0]; sy = d.sigma[1]; }
            else if (MID == MODEL_XYIBG_CONSTSIGMA) { sx = consts[0]; sy = consts[1]; }
            else if (MID == MODEL_XYIBG_SIGMA) { sx = th[4]; sy = th[4]; }
            else { sx = th[4]; sy = th[5]; }
            invSqrtPi = kInvSqrtPi;
            if (MID == MODEL_XYIBG && d.fixed_c[0] > 0.0f) {
                cx2 = d.fixed_c[0];
                cx1 = d.fixed_c[1];
                cy2 = d.fixed_c[2];
                cy1 = d.fixed_c[3];
            } else {
                cx2 = DIV(1.0f, MUL(s2pi, sx));
                cy2 = DIV(1.0f, MUL(s2pi, sy));
                cx1 = DIV(1.0f, MUL(s2, sx));
                cy1 = DIV(1.0f, MUL(s2, sy));
            }
            sigx = sx;
            sigy = sy;
            gax = gay = 0.0f;
        }
    }

    // begin() for the G lanes of a group, which all hold the same theta: the same floats. For the
    // astigmatic model the 14-18 IEEE divisions of sigma(z), its z derivative and the erf/exp
    // scales are shared out across the lanes (one division per lane per round, quotients exchanged
    // by shuffles within the group) instead of every lane dividing every pair: 1M 12x12 ROIs
    // 10.58 -> 9.07 ms on a B200, results unchanged bit for bit. With B == 0 the quartic terms,
    // which would add exactly +0, are left out, which is photonpy's 4-coefficient expression
    // itself. The other models have 5 divisions per set-up; sharing them did not pay (XYIBg 10x10
    // with 2 lanes per ROI: 3.01 -> 3.19 ms), so they run begin().
    template <int G>
    __device__ __forceinline__ void begin_group(const ModelDesc& d, const float* th, const float* consts, int lane,
                                                unsigned mask) {
        tx = th[0];
        ty = th[1];
        const float s2pi = kSqrt2Pi;
        const float s2 = kSqrt2;
        if (MID == MODEL_XYZIBG) {
            tI = th[3];
            tbg = th[4];
            const float tz = th[2];
            const float s0x = d.astig_x[0], gx = d.astig_x[1], dx = d.astig_x[2], Ax = d.astig_x[3], Bx = d.astig_x[4];
            const float s0y = d.astig_y[0], gy = d.astig_y[1], dy = d.astig_y[2], Ay = d.astig_y[3], By = d.astig_y[4];
            const float dy2 = MUL(dy, dy), dx2 = MUL(dx, dx);
            const float dy4 = MUL(dy2, dy2), dx4 = MUL(dx2, dx2);
            const float tzx = SUB(tz, gx), tzx2 = MUL(tzx, tzx), tzx3 = MUL(tzx2, tzx), tzx4 = MUL(tzx2, tzx2);
            const float tzy = SUB(tz, gy), tzy2 = MUL(tzy, tzy), tzy3 = MUL(tzy2, tzy), tzy4 = MUL(tzy2, tzy2);
            const float num[8] = {tzx2, MUL(Ax, tzx3), MUL(2.0f, tzx), MUL(MUL(Ax, 3.0f), tzx2),
                                  tzy2, MUL(Ay, tzy3), MUL(2.0f, tzy), MUL(MUL(Ay, 3.0f), tzy2)};
            const float den[8] = {dx2, dx2, dx2, dx2, dy2, dy2, dy2, dy2};
            float q1[8];
            group_div<8, G>(num, den, q1, lane, mask);
            float qx = ADD(ADD(1.0f, q1[0]), q1[1]);
            float qy = ADD(ADD(1.0f, q1[4]), q1[5]);
            float nx = ADD(q1[2], q1[3]);
            float ny = ADD(q1[6], q1[7]);
            if (Bx != 0.0f || By != 0.0f) {  // the quartic extension
                const float numB[4] = {MUL(Bx, tzx4), MUL(MUL(Bx, 4.0f), tzx3), MUL(By, tzy4), MUL(MUL(By, 4.0f), tzy3)};
                const float denB[4] = {dx4, dx4, dy4, dy4};
                float qB[4];
                group_div<4, G>(numB, denB, qB, lane, mask);
                qx = ADD(qx, qB[0]);
                nx = ADD(nx, qB[1]);
                qy = ADD(qy, qB[2]);
                ny = ADD(ny, qB[3]);
            }
            const float sqx = __fsqrt_rn(qx), sqy = __fsqrt_rn(qy);
            sigx = MUL(s0x, sqx);
            sigy = MUL(s0y, sqy);
            const float num2[8] = {1.0f, 1.0f, 1.0f, 1.0f, MUL(s0x, nx), MUL(s0y, ny), 1.0f, 1.0f};
            const float den2[8] = {MUL(s2pi, sigx), MUL(s2, sigx), MUL(s2pi, sigy), MUL(s2, sigy), MUL(2.0f, sqx),
                                   MUL(2.0f, sqy), MUL(MUL(s2pi, sigx), sigx), MUL(MUL(s2pi, sigy), sigy)};
            float q2[8];
            group_div<8, G>(num2, den2, q2, lane, mask);
            cx2 = q2[0];
            cx1 = q2[1];
            cy2 = q2[2];
            cy1 = q2[3];
            dsxz = q2[4];
            dsyz = q2[5];
            gax = q2[6];
            gay = q2[7];
        } else {
            begin(d, th, consts);
        }
    }

    // One 1D term for coordinate c (pixel index) along an axis with centre t.
    // Output slots: [0]=Delta, [1]=tI*Delta, [2]=tI*dE, [3]=model-specific.
    __device__ __forceinline__ void term(int c, float t, float c1, float c2, float sig, bool isx, float4* out) const {
        const float d0 = SUB((float)c, t);
        const float e0 = MUL(ADD(d0, 0.5f), c1);
        const float e1 = MUL(SUB(d0, 0.5f), c1);
        const float delta = SUB(MUL(0.5f, erff(e0)), MUL(0.5f, erff(e1)));
        const float ex1 = expf(MUL(-e1, e1));
        const float ex0 = expf(MUL(-e0, e0));
        const float dE = MUL(c2, SUB(ex1, ex0));
        float4 r;
        r.x = delta;
        r.y = MUL(tI, delta);
        if (MID == MODEL_XYIBG || MID == MODEL_XYIBG_CONSTSIGMA) {
            r.z = MUL(tI, dE);
            r.w = 0.0f;
        } else if (MID == MODEL_XYIBG_SIGMA || MID == MODEL_XYIBG_SIGMAXY) {
            const float dDs = MUL(SUB(MUL(ex1, e1), MUL(ex0, e0)), invSqrtPi);
            r.z = MUL(tI, dE);
            r.w = (MID == MODEL_XYIBG_SIGMAXY) ? MUL(tI, dDs) : dDs;
        } else {
            // G21 = 1/(sqrt(2 pi) s s) * ((c-t-.5) exp(-(c-t-.5)^2/(2 s s)) - (c-t+.5) exp(-(c-t+.5)^2/(2 s s)))
            const float m = SUB(d0, 0.5f), p = ADD(d0, 0.5f);
            const float ss2 = MUL(MUL(2.0f, sig), sig);
            const float a = DIV(1.0f, MUL(MUL(kSqrt2Pi, sig), sig));
            const float g = MUL(a, SUB(MUL(m, expf(DIV(MUL(-m, m), ss2))), MUL(p, expf(DIV(MUL(-p, p), ss2)))));
            r.z = MUL(tI, dE);
            r.w = g;
        }
        (void)isx;
        *out = r;
    }

    // The 1D terms of N consecutive coordinates c0..c0+N-1 along one axis. erf and exp are
    // evaluated once per pixel edge: the upper edge of pixel c, ((c - t) + 0.5) * c1, and the
    // lower edge of pixel c+1, ((c+1 - t) - 0.5) * c1, are the same float whenever the two
    // rounded subtractions agree, and only then is the edge value reused. Every term is
    // therefore bit-identical to term() above.
    template <int N>
    __device__ __forceinline__ void term_block(int c0, float t, float c1, float c2, float sig, float ga,
                                               float4 (&out)[N]) const {
        float m[N + 1], E[N + 1], ef[N + 1], ex[N + 1], gx[N + 1];
        float ss2 = 0.0f;
        if (MID == MODEL_XYZIBG) ss2 = MUL(MUL(2.0f, sig), sig);
#pragma unroll
        for (int k = 0; k <= N; k++) {
            m[k] = SUB(SUB((float)(c0 + k), t), 0.5f);
            E[k] = MUL(m[k], c1);
            ef[k] = erff(E[k]);
            ex[k] = expf(MUL(-E[k], E[k]));
            if (MID == MODEL_XYZIBG) gx[k] = expf(DIV(MUL(-m[k], m[k]), ss2));
        }
#pragma unroll
        for (int q = 0; q < N; q++) {
            const float p = ADD(SUB((float)(c0 + q), t), 0.5f);
            float e0, erf0, exp0, g0 = 0.0f;
            if (p == m[q + 1]) {
                e0 = E[q + 1];
                erf0 = ef[q + 1];
                exp0 = ex[q + 1];
                if (MID == MODEL_XYZIBG) g0 = gx[q + 1];
            } else {
                e0 = MUL(p, c1);
                erf0 = erff(e0);
                exp0 = expf(MUL(-e0, e0));
                if (MID == MODEL_XYZIBG) g0 = expf(DIV(MUL(-p, p), ss2));
            }
            const float e1 = E[q], erf1 = ef[q], exp1 = ex[q];
            const float delta = SUB(MUL(0.5f, erf0), MUL(0.5f, erf1));
            const float dE = MUL(c2, SUB(exp1, exp0));
            float4 r;
            r.x = delta;
            r.y = MUL(tI, delta);
            r.z = MUL(tI, dE);
            if (MID == MODEL_XYIBG || MID == MODEL_XYIBG_CONSTSIGMA) {
                r.w = 0.0f;
            } else if (MID == MODEL_XYIBG_SIGMA || MID == MODEL_XYIBG_SIGMAXY) {
                const float dDs = MUL(SUB(MUL(exp1, e1), MUL(exp0, e0)), invSqrtPi);
                r.w = (MID == MODEL_XYIBG_SIGMAXY) ? MUL(tI, dDs) : dDs;
            } else {
                r.w = MUL(ga, SUB(MUL(m[q], gx[q]), MUL(p, g0)));
            }
            out[q] = r;
        }
    }

    // mu and Jacobian of one pixel from its x-term X and y-term Y (see pixel()).
    __device__ __forceinline__ void pixel_xy(const float4& X, const float4& Y, float& mu, float (&J)[K]) const {
        mu = fmaf(X.y, Y.x, tbg);  // tbg + (tI*DeltaX)*DeltaY, one rounding
        const float dmx = MUL(X.z, Y.x);
        const float dmy = MUL(Y.z, X.x);
        const float dI = MUL(X.x, Y.x);
        if (MID == MODEL_XYZIBG) {
            J[0] = dmx;
            J[1] = dmy;
            J[2] = ADD(MUL(MUL(Y.y, X.w), dsxz), MUL(MUL(X.y, Y.w), dsyz));
            J[3] = dI;
            J[4 % K] = 1.0f;
        } else {
            J[0] = dmx;
            J[1] = dmy;
            J[2] = dI;
            J[3] = 1.0f;
            if (MID == MODEL_XYIBG_SIGMA) {
                J[4 % K] = MUL(tI, ADD(MUL(X.w, Y.x), MUL(Y.w, X.x)));
            } else if (MID == MODEL_XYIBG_SIGMAXY) {
                J[4 % K] = MUL(X.w, Y.x);
                J[5 % K] = MUL(Y.w, X.x);
            }
        }
    }

    __device__ __forceinline__ void build_table(const ModelDesc& d, float* tab, int lane, int G) const {
        const int R = d.roisize;
        float4* t4 = reinterpret_cast<float4*>(tab);
        for (int i = lane; i < 2 * R; i += G) {
            if (i < R) term(i, tx, cx1, cx2, sigx, true, &t4[i]);
            else term(i - R, ty, cy1, cy2, sigy, false, &t4[i]);
        }
    }

    // mu and Jacobian for pixel (x, y) from the table.
    __device__ __forceinline__ void pixel(const ModelDesc& d, const float* tab, int x, int y, float& mu,
                                          float (&J)[K]) const {
        const float4 X = reinterpret_cast<const float4*>(tab)[x];
        const float4 Y = reinterpret_cast<const float4*>(tab)[d.roisize + y];
        // mu = tbg + (tI*DeltaX)*DeltaY
        mu = ADD(tbg, MUL(X.y, Y.x));
        const float dmx = MUL(X.z, Y.x);  // (tI*dEx)*DeltaY
        const float dmy = MUL(Y.z, X.x);  // (tI*dEy)*DeltaX
        const float dI = MUL(X.x, Y.x);
        if (MID == MODEL_XYZIBG) {
            // dmu/dz = ((tI*DeltaY)*G21x)*dsx/dz + ((tI*DeltaX)*G21y)*dsy/dz
            const float dMsx = MUL(Y.y, X.w);
            const float dMsy = MUL(X.y, Y.w);
            J[0] = dmx;
            J[1] = dmy;
            J[2] = ADD(MUL(dMsx, dsxz), MUL(dMsy, dsyz));
            J[3] = dI;
            J[4] = 1.0f;
        } else {
            J[0] = dmx;
            J[1] = dmy;
            J[2] = dI;
            J[3] = 1.0f;
            if (MID == MODEL_XYIBG_SIGMA) {
                // tI * (dDeltaX_dsigma*DeltaY + dDeltaY_dsigma*DeltaX)
                J[4 % K] = MUL(tI, ADD(MUL(X.w, Y.x), MUL(Y.w, X.x)));
            } else if (MID == MODEL_XYIBG_SIGMAXY) {
                J[4 % K] = MUL(X.w, Y.x);
                J[5 % K] = MUL(Y.w, X.x);
            }
        }
    }

    // CheckLimits (GaussianPSFModels.h:54-61, 327-337, 410-419, 654-661)
    __device__ __forceinline__ static void check_limits(const ModelDesc& d, float (&t)[K]) {
        const int R = d.roisize;
        const float hi = gauss_xy_max(R);
        t[0] = pb_clamp(t[0], 1.5f, hi);
        t[1] = pb_clamp(t[1], 1.5f, hi);
        if (MID == MODEL_XYIBG || MID == MODEL_XYIBG_CONSTSIGMA) {
            if (t[2] < 25.0f) t[2] = 25.0f;
            if (t[3] < 0.0f) t[3] = 0.0f;
        } else if (MID == MODEL_XYIBG_SIGMA) {
            if (t[2] < 10.0f) t[2] = 10.0f;
            if (t[3] < 0.0f) t[3] = 0.0f;
            if (t[4 % K] < 1.0f) t[4 % K] = 1.0f;
            const float smax = MUL((float)R, 0.5f);
            if (t[4 % K] > smax) t[4 % K] = smax;
        } else if (MID == MODEL_XYIBG_SIGMAXY) {
            if (t[2] < 10.0f) t[2] = 10.0f;
            if (t[3] < 0.0f) t[3] = 0.0f;
            const float smax = MUL((float)R, 0.5f);
            t[4 % K] = pb_clamp(t[4 % K], 1.0f, smax);
            t[5 % K] = pb_clamp(t[5 % K], 1.0f, smax);
        } else {
            t[2] = pb_clamp(t[2], d.minz, d.maxz);
            t[3] = fmaxf(t[3], 10.0f);
            t[4 % K] = fmaxf(t[4 % K], 0.0f);
        }
    }

    __device__ __forceinline__ static float stop_limit(int k) {
        if (MID == MODEL_XYIBG || MID == MODEL_XYIBG_CONSTSIGMA) return k == 2 ? 1e-1f : 1e-5f;
        if (MID == MODEL_XYIBG_SIGMA) return k == 2 ? 1e-1f : (k == 3 ? 1e-4f : 1e-5f);
        if (MID == MODEL_XYIBG_SIGMAXY) return k == 2 ? 1e-1f : (k == 3 ? 1e-4f : 1e-5f);
        return k == 2 ? 1e-1f : 1e-4f;  // astig {x,y,z,I,bg} = {1e-4,1e-4,1e-1,1e-4,1e-4}
    }

    // Initial value from the centre of mass (GaussianPSFModels.h:147-151, 382-386, 466-470, 664-674)
    __device__ __forceinline__ static void initial(const ModelDesc& d, float comx, float comy, float sum,
                                                   float (&t)[K]) {
        t[0] = comx;
        t[1] = comy;
        if (MID == MODEL_XYIBG || MID == MODEL_XYIBG_CONSTSIGMA) {
            t[2] = MUL(sum, 0.7f);
            t[3] = 0.0f;
        } else if (MID == MODEL_XYIBG_SIGMA) {
            t[2] = sum;
            t[3] = 0.0f;
            t[4 % K] = d.sigma[0];
        } else if (MID == MODEL_XYIBG_SIGMAXY) {
            t[2] = sum;
            t[3] = 0.0f;
            t[4 % K] = d.sigma[0];
            t[5 % K] = d.sigma[1];
        } else {
            t[2] = 0.0f;
            t[3] = sum;
            t[4 % K] = 0.01f;
        }
    }
};

// ---------------------------------------------------------------------------------------
// Gaussian spot on a tilted background plane (generic table kernel only).
//   XYITiltedBg          theta = (x, y, I, bg, bgx, bgy), sigma_x/sigma_y from the spot's two
//                        constants; mu = ((bg + bgx (x - W/2)) + bgy (y - H/2)) + I DeltaX DeltaY
//   XYITiltedBgSigmaXY   theta = (x, y, I, bg, bgx, bgy, sx, sy); the reference keeps the tilt
//                        columns x - W/2, y - H/2 in the Jacobian but leaves the tilt out of mu
//                        (GaussianPSFModels.h:542 vs 549), reproduced here
// Table: x-terms [R] then y-terms [R] of float4 (Delta, I*Delta, I*dE, I*dDelta/dsigma).
// ---------------------------------------------------------------------------------------
template <int MID>
struct TiltedGaussModel {
    static constexpr int K = model_num_params(MID);
    static constexpr int kId = MID;
    static constexpr bool kFreeSigma = (MID == MODEL_XYITILTEDBG_SIGMAXY);
    static __host__ __device__ constexpr int table_floats(int R) { return 8 * R; }

    float tx, ty, tI, tbg, bgx, bgy;
    float cx1, cx2, cy1, cy2, invSqrtPi, half;

    __device__ __forceinline__ void begin(const ModelDesc& d, const float* th, const float* consts) {
        tx = th[0];
        ty = th[1];
        tI = th[2];
        tbg = th[3];
        bgx = th[4];
        bgy = th[5];
        const float sx = kFreeSigma ? th[6 % K] : consts[0];
        const float sy = kFreeSigma ? th[7 % K] : consts[1];
        const float s2pi = kSqrt2Pi, s2 = kSqrt2;
        invSqrtPi = kInvSqrtPi;
        cx2 = DIV(1.0f, MUL(s2pi, sx));
        cy2 = DIV(1.0f, MUL(s2pi, sy));
        cx1 = DIV(1.0f, MUL(s2, sx));
        cy1 = DIV(1.0f, MUL(s2, sy));
        half = MUL((float)d.roisize, 0.5f);
    }

    __device__ __forceinline__ void term(int c, float t, float c1, float c2, float4* out) const {
        const float d0 = SUB((float)c, t);
        const float e0 = MUL(ADD(d0, 0.5f), c1);
        const float e1 = MUL(SUB(d0, 0.5f), c1);
        const float delta = SUB(MUL(0.5f, erff(e0)), MUL(0.5f, erff(e1)));
        const float ex1 = expf(MUL(-e1, e1));
        const float ex0 = expf(MUL(-e0, e0));
        float4 r;
        r.x = delta;
        r.y = MUL(tI, delta);
        r.z = MUL(tI, MUL(c2, SUB(ex1, ex0)));
        r.w = kFreeSigma ? MUL(tI, MUL(SUB(MUL(ex1, e1), MUL(ex0, e0)), invSqrtPi)) : 0.0f;
        *out = r;
    }

    __device__ __forceinline__ void build_table(const ModelDesc& d, float* tab, int lane, int G) const {
        const int R = d.roisize;
        float4* t4 = reinterpret_cast<float4*>(tab);
        for (int i = lane; i < 2 * R; i += G) {
            if (i < R) term(i, tx, cx1, cx2, &t4[i]);
            else term(i - R, ty, cy1, cy2, &t4[i]);
        }
    }

    __device__ __forceinline__ void pixel(const ModelDesc& d, const float* tab, int x, int y, float& mu,
                                          float (&J)[K]) const {
        const float4 X = reinterpret_cast<const float4*>(tab)[x];
        const float4 Y = reinterpret_cast<const float4*>(tab)[d.roisize + y];
        const float px = SUB((float)x, half), py = SUB((float)y, half);
        if (kFreeSigma) mu = ADD(tbg, MUL(X.y, Y.x));
        else mu = ADD(ADD(ADD(tbg, MUL(bgx, px)), MUL(bgy, py)), MUL(X.y, Y.x));
        J[0] = MUL(X.z, Y.x);  // (I dEx) DeltaY
        J[1] = MUL(Y.z, X.x);  // (I dEy) DeltaX
        J[2] = MUL(X.x, Y.x);
        J[3] = 1.0f;
        J[4] = px;
        J[5] = py;
        if (kFreeSigma) {
            J[6 % K] = MUL(X.w, Y.x);
            J[7 % K] = MUL(Y.w, X.x);
        }
    }

    // CheckLimits (GaussianPSFModels.h:251-258, 495-505)
    __device__ __forceinline__ static void check_limits(const ModelDesc& d, float (&t)[K]) {
        const int R = d.roisize;
        const float hi = gauss_xy_max(R);
        t[0] = pb_clamp(t[0], 1.5f, hi);
        t[1] = pb_clamp(t[1], 1.5f, hi);
        if (t[2] < (kFreeSigma ? 10.0f : 25.0f)) t[2] = kFreeSigma ? 10.0f : 25.0f;
        if (t[3] < 0.0f) t[3] = 0.0f;
        if (kFreeSigma) {
            const float smax = MUL((float)R, 0.5f);
            t[6 % K] = pb_clamp(t[6 % K], 1.0f, smax);
            t[7 % K] = pb_clamp(t[7 % K], 1.0f, smax);
        }
    }

    // StopLimit (GaussianPSFModels.h:242-246, 486-490)
    __device__ __forceinline__ static float stop_limit(int k) {
        if (k == 2) return 1e-1f;
        if (kFreeSigma && k >= 3 && k <= 5) return 1e-4f;
        return 1e-5f;
    }

    // Initial value (GaussianPSFModels.h:299-303, 553-557)
    __device__ __forceinline__ static void initial(const ModelDesc& d, float comx, float comy, float sum,
                                                   float (&t)[K]) {
        t[0] = comx;
        t[1] = comy;
        t[2] = kFreeSigma ? sum : MUL(sum, 0.7f);
        t[3] = 0.0f;
        t[4] = 0.0f;
        t[5] = 0.0f;
        if (kFreeSigma) {
            t[6 % K] = d.sigma[0];
            t[7 % K] = d.sigma[1];
        }
    }
};

// ---------------------------------------------------------------------------------------
// Intensity and background of a spot at a known position and width (the model behind
// Gauss2D_EstimateIntensityBg, GaussianPSF.cu:216-240): theta = (I, bg), constants =
// (x, y, sigma), mu = I * DeltaX DeltaY + bg. Table: DeltaX [R] then DeltaY [R].
// ---------------------------------------------------------------------------------------
struct IntensityBgModel {
    static constexpr int K = 2;
    static constexpr int kId = MODEL_INTENSITYBG;
    static __host__ __device__ constexpr int table_floats(int R) { return 2 * R; }

    float tI, tbg, tx, ty, c1;

    __device__ __forceinline__ void begin(const ModelDesc&, const float* th, const float* consts) {
        tI = th[0];
        tbg = th[1];
        tx = consts[0];
        ty = consts[1];
        c1 = DIV(1.0f, MUL(kSqrt2, consts[2]));
    }

    __device__ __forceinline__ void build_table(const ModelDesc& d, float* tab, int lane, int G) const {
        const int R = d.roisize;
        for (int i = lane; i < 2 * R; i += G) {
            const bool isx = i < R;
            const float d0 = SUB((float)(isx ? i : i - R), isx ? tx : ty);
            const float e0 = MUL(ADD(d0, 0.5f), c1);
            const float e1 = MUL(SUB(d0, 0.5f), c1);
            tab[i] = SUB(MUL(0.5f, erff(e0)), MUL(0.5f, erff(e1)));
        }
    }

    __device__ __forceinline__ void pixel(const ModelDesc& d, const float* tab, int x, int y, float& mu,
                                          float (&J)[K]) const {
        const float psf = MUL(tab[x], tab[d.roisize + y]);  // DeltaX * DeltaY
        mu = ADD(MUL(tI, psf), tbg);
        J[0] = psf;
        J[1] = 1.0f;
    }

    // CheckLimits / StopLimit (GaussianPSFModels.h:587-599)
    __device__ __forceinline__ static void check_limits(const ModelDesc&, float (&t)[K]) {
        if (t[0] < 1e-5f) t[0] = 1e-5f;
        if (t[1] < 1e-8f) t[1] = 1e-8f;
    }
    __device__ __forceinline__ static float stop_limit(int k) { return k == 0 ? 1e-2f : 1e-4f; }

    // Every spot starts at (I, bg) = (1, 0) (GaussianPSF.cu:226).
    __device__ __forceinline__ static void initial(const ModelDesc&, float, float, float, float (&t)[K]) {
        t[0] = 1.0f;
        t[1] = 0.0f;
    }
};

// ---------------------------------------------------------------------------------------
// Cubic spline: table = delta_f, delta_dxf, delta_dyf, delta_dzf [4][64]. OVS: the calibration is
// sampled finer than a pixel (ModelDesc::spline_q voxels per pixel, the oversampled extension);
// without it the voxel scale is 1 at compile time, photonpy's model exactly. MODE 0 flat
// background, 1 tilted background (theta += bgx, bgy; mu += bgx (x - W/2) + bgy (y - W/2)),
// 2 background image (mu = I psf + bg * image; the image is the spot's R*R constants, read
// per pixel through `img`; this mode centres tx, ty differently, CubicSplinePSFModels.h:371-374).
// ---------------------------------------------------------------------------------------
template <int MODE, bool OVS = false>
struct SplineModelT {
    static constexpr int K = (MODE == 1) ? 7 : 5;
    static constexpr int kId = (MODE == 0) ? MODEL_CSPLINE : (MODE == 1 ? MODEL_CSPLINE_TILTED : MODEL_CSPLINE_BGIMAGE);
    static constexpr bool kPixelConsts = (MODE == 2);
    static constexpr int kPixelBlock = 4;  // pixels per pixel_block() call
    static __host__ __device__ constexpr int table_floats(int) { return 256; }

    float tx, ty, tI, tbg, du;
    float vq;  // voxels per ROI pixel (1: the reference's model)

    // pixel index c in spline-grid units before the centre offset: vq c (c itself without OVS)
    __device__ __forceinline__ float gridc(int c) const { return OVS ? MUL((float)c, vq) : (float)c; }
    float spx, spy, spz;
    float bgx, bgy, halfw;
    const float* img;  // MODE 2: this spot's background image [R][R]
    int k;  // z slice
    int Nx, Ny;

    __device__ __forceinline__ void begin(const ModelDesc& d, const float* th, const float*) {
        const int Nz = d.spline_shape[0];
        Ny = d.spline_shape[1];
        Nx = d.spline_shape[2];
        du = DIV(SUB(d.spline_zmax, d.spline_zmin), (float)Nz);
        vq = OVS ? d.spline_q : 1.0f;
        if (MODE == 2) {
            const float w = (float)d.roisize;
            tx = ADD(ADD(SUB(th[0], DIV(w, 2.0f)), DIV(ADD(SUB(w, (float)Nx), 1.0f), 2.0f)), 0.5f);
            ty = ADD(ADD(SUB(th[1], DIV(w, 2.0f)), DIV(ADD(SUB(w, (float)Ny), 1.0f), 2.0f)), 0.5f);
        } else {
            // grid coordinate of pixel x: vq x - tx (vq = 1: x - (theta_x - Nx/2), the reference)
            tx = SUB(OVS ? MUL(th[0], vq) : th[0], MUL((float)Nx, 0.5f));
            ty = SUB(OVS ? MUL(th[1], vq) : th[1], MUL((float)Ny, 0.5f));
        }
        tI = th[3];
        tbg = th[4];
        bgx = (MODE == 1) ? th[5 % K] : 0.0f;
        bgy = (MODE == 1) ? th[6 % K] : 0.0f;
        halfw = MUL((float)d.roisize, 0.5f);
        img = nullptr;
        // sub-voxel offset: the reference truncates toward zero (CubicSplinePSFModels.h:89-91),
        // which is its fractional part wherever the model is valid (Nx/2 >= max x); the
        // oversampled extension takes the fractional part (floor) everywhere
        float sx = -tx;
        spx = SUB(sx, OVS ? floorf(sx) : (float)(int)sx);
        float sy = -ty;
        spy = SUB(sy, OVS ? floorf(sy) : (float)(int)sy);
        float sz = DIV(SUB(th[2], d.spline_zmin), du);
        int kk = (int)sz;
        kk = max(0, min(kk, Nz - 1));
        k = kk;
        spz = pb_clamp(SUB(sz, (float)kk), 0.0f, 1.0f);
    }

    // Power-basis tables (CubicSplinePSFModels.h:101-118): entry idx = m*16 + n*4 + o,
    // xyz = (spx^o * spy^n) * spz^m built by repeated multiplication as in the reference.
    __device__ __forceinline__ void build_table(const ModelDesc&, float* tab, int lane, int G) const {
        for (int idx = lane; idx < 64; idx += G) {
            const int m = idx >> 4, n = (idx >> 2) & 3, o = idx & 3;
            float xxx = 1.0f, yyy = 1.0f, zzz = 1.0f;
            for (int q = 0; q < o; q++) xxx = MUL(xxx, spx);
            for (int q = 0; q < n; q++) yyy = MUL(yyy, spy);
            for (int q = 0; q < m; q++) zzz = MUL(zzz, spz);
            const float xyz = MUL(MUL(xxx, yyy), zzz);
            tab[idx] = xyz;
            // delta_dxf[m,n,o+1] = (o+1)*xyz(m,n,o); entries with o == 0 stay 0
            float xo = 1.0f;
            for (int q = 0; q < o - 1; q++) xo = MUL(xo, spx);
            tab[64 + idx] = (o > 0) ? MUL((float)o, MUL(MUL(xo, yyy), zzz)) : 0.0f;
            float yn = 1.0f;
            for (int q = 0; q < n - 1; q++) yn = MUL(yn, spy);
            tab[128 + idx] = (n > 0) ? MUL((float)n, MUL(MUL(xxx, yn), zzz)) : 0.0f;
            float zm = 1.0f;
            for (int q = 0; q < m - 1; q++) zm = MUL(zm, spz);
            tab[192 + idx] = (m > 0) ? MUL((float)m, MUL(MUL(xxx, yyy), zm)) : 0.0f;
        }
    }

    __device__ __forceinline__ void pixel(const ModelDesc& d, const float* tab, int x, int y, float& mu,
                                          float (&J)[K]) const {
        const float yy = SUB(gridc(y), ty);
        const int j = max(0, min((int)yy, Ny - 1));
        const float xx = SUB(gridc(x), tx);
        const int i = max(0, min((int)xx, Nx - 1));
        const float4* c4 = reinterpret_cast<const float4*>(d.coefs + 64 * ((size_t)k * Nx * Ny + (size_t)j * Nx + i));
        const float4* f4 = reinterpret_cast<const float4*>(tab);
        float psf = 0.0f, dx = 0.0f, dy = 0.0f, dz = 0.0f;
#pragma unroll 4
        for (int q = 0; q < 16; q++) {
            const float4 c = __ldg(c4 + q);
            const float4 a = f4[q], b = f4[16 + q], e = f4[32 + q], g = f4[48 + q];
            psf = ADD(ADD(ADD(ADD(psf, MUL(a.x, c.x)), MUL(a.y, c.y)), MUL(a.z, c.z)), MUL(a.w, c.w));
            dx = ADD(ADD(ADD(ADD(dx, MUL(b.x, c.x)), MUL(b.y, c.y)), MUL(b.z, c.z)), MUL(b.w, c.w));
            dy = ADD(ADD(ADD(ADD(dy, MUL(e.x, c.x)), MUL(e.y, c.y)), MUL(e.z, c.z)), MUL(e.w, c.w));
            dz = ADD(ADD(ADD(ADD(dz, MUL(g.x, c.x)), MUL(g.y, c.y)), MUL(g.z, c.z)), MUL(g.w, c.w));
        }
        dx = MUL(dx, OVS ? -MUL(tI, vq) : -tI);
        dy = MUL(dy, OVS ? -MUL(tI, vq) : -tI);
        dz = MUL(dz, DIV(tI, du));
        if (psf < 0.0f) psf = 0.0f;
        J[0] = dx;
        J[1] = dy;
        J[2] = dz;
        J[3] = psf;
        if (MODE == 1) {
            const float px = SUB((float)x, halfw), py = SUB((float)y, halfw);
            mu = ADD(ADD(ADD(MUL(tI, psf), tbg), MUL(bgx, px)), MUL(bgy, py));
            J[4] = 1.0f;
            J[5 % K] = px;
            J[6 % K] = py;
        } else if (MODE == 2) {
            const float bg = __ldg(img + y * d.roisize + x);
            mu = ADD(MUL(tI, psf), MUL(tbg, bg));
            J[4] = bg;
        } else {
            mu = ADD(MUL(tI, psf), tbg);
            J[4] = 1.0f;
        }
    }

    // pixel() for PB pixels at once: each 16-byte read of the shared power-basis tables serves
    // all PB pixels (the tables, not the coefficients, are the bulk of the shared-memory
    // traffic). Every pixel's sums are formed in the same order as in pixel(). Pixels with
    // y >= roisize (past the ROI) get defined, unused values.
    template <int PB>
    __device__ __forceinline__ void pixel_block(const ModelDesc& d, const float* tab, const int (&x)[PB],
                                                const int (&y)[PB], float (&mu)[PB], float (&J)[PB][K]) const {
        const float4* cp[PB];
        float psf[PB], ddx[PB], ddy[PB], ddz[PB];
        const size_t nvox = (size_t)d.spline_shape[0] * Ny * Nx;
        const bool qmajor = d.coefsQ != nullptr;
        const size_t qstride = qmajor ? nvox : 1;
#pragma unroll
        for (int t = 0; t < PB; t++) {
            const int j = max(0, min((int)SUB(gridc(y[t]), ty), Ny - 1));
            const int i = max(0, min((int)SUB(gridc(x[t]), tx), Nx - 1));
            const size_t v = (size_t)k * Nx * Ny + (size_t)j * Nx + i;
            cp[t] = qmajor ? d.coefsQ + v : reinterpret_cast<const float4*>(d.coefs) + 16 * v;
            psf[t] = ddx[t] = ddy[t] = ddz[t] = 0.0f;
        }
        const float4* f4 = reinterpret_cast<const float4*>(tab);
#pragma unroll 2
        for (int q = 0; q < 16; q++) {
            const float4 a = f4[q], b = f4[16 + q], e = f4[32 + q], g = f4[48 + q];
#pragma unroll
            for (int t = 0; t < PB; t++) {
                const float4 c = __ldg(cp[t] + q * qstride);
                psf[t] = ADD(ADD(ADD(ADD(psf[t], MUL(a.x, c.x)), MUL(a.y, c.y)), MUL(a.z, c.z)), MUL(a.w, c.w));
                ddx[t] = ADD(ADD(ADD(ADD(ddx[t], MUL(b.x, c.x)), MUL(b.y, c.y)), MUL(b.z, c.z)), MUL(b.w, c.w));
                ddy[t] = ADD(ADD(ADD(ADD(ddy[t], MUL(e.x, c.x)), MUL(e.y, c.y)), MUL(e.z, c.z)), MUL(e.w, c.w));
                ddz[t] = ADD(ADD(ADD(ADD(ddz[t], MUL(g.x, c.x)), MUL(g.y, c.y)), MUL(g.z, c.z)), MUL(g.w, c.w));
            }
        }
        const float zs = DIV(tI, du);
        const float xs = OVS ? -MUL(tI, vq) : -tI;
#pragma unroll
        for (int t = 0; t < PB; t++) {
            float p = psf[t];
            if (p < 0.0f) p = 0.0f;
            J[t][0] = MUL(ddx[t], xs);
            J[t][1] = MUL(ddy[t], xs);
            J[t][2] = MUL(ddz[t], zs);
            J[t][3] = p;
            if (MODE == 1) {
                const float px = SUB((float)x[t], halfw), py = SUB((float)y[t], halfw);
                mu[t] = ADD(ADD(ADD(MUL(tI, p), tbg), MUL(bgx, px)), MUL(bgy, py));
                J[t][4] = 1.0f;
                J[t][5 % K] = px;
                J[t][6 % K] = py;
            } else if (MODE == 2) {
                const float bg = y[t] < d.roisize ? __ldg(img + y[t] * d.roisize + x[t]) : 0.0f;
                mu[t] = ADD(MUL(tI, p), MUL(tbg, bg));
                J[t][4] = bg;
            } else {
                mu[t] = ADD(MUL(tI, p), tbg);
                J[t][4] = 1.0f;
            }
        }
    }

    // Offset of the 64 coefficients pixel (x, y) reads (same voxel choice as pixel()).
    __device__ __forceinline__ size_t coef_offset(int x, int y) const {
        const int j = max(0, min((int)SUB(gridc(y), ty), Ny - 1));
        const int i = max(0, min((int)SUB(gridc(x), tx), Nx - 1));
        return 64 * ((size_t)k * Nx * Ny + (size_t)j * Nx + i);
    }

    // CheckLimits (CubicSplinePSFModels.h:44-50, 185-191, 330-336): bgx, bgy are not clamped
    __device__ __forceinline__ static void check_limits(const ModelDesc& d, float (&t)[K]) {
        const float hi = SUB(SUB((float)d.roisize, 1.0f), 1.5f);
        t[0] = pb_clamp(t[0], 1.5f, hi);
        t[1] = pb_clamp(t[1], 1.5f, hi);
        t[2] = pb_clamp(t[2], ADD(d.spline_zmin, 1e-3f), SUB(d.spline_zmax, 1e-3f));
        t[3] = fmaxf(t[3], 10.0f);
        t[4] = fmaxf(t[4], 0.0f);
    }

    __device__ __forceinline__ static float stop_limit(int k) { return k == 2 ? 1e-7f : 1e-4f; }

    __device__ __forceinline__ static void initial(const ModelDesc&, float comx, float comy, float sum,
                                                   float (&t)[K]) {
        t[0] = comx;
        t[1] = comy;
        t[2] = 0.0f;
        t[3] = sum;
        t[4] = 0.0f;
        if (MODE == 1) {
            t[5 % K] = 0.0f;
            t[6 % K] = 0.0f;
        }
    }
};
using SplineModel = SplineModelT<0>;

}  // namespace pb200
