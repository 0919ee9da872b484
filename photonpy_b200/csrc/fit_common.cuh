// Shared pieces of the fit kernels: launch arguments, lane-group helpers, the damped K x K
// LM solve (packed triangles, registers only) and the FP64 paths run by one lane on shared
// memory (LM re-solve of a weak pivot, Fisher-matrix inverse).
//
// Reference semantics (Estimators/Estimation.h:194-251, SolveMatrix.h:107-163, 411-452):
//  * damping lambda > 0: a_kk += lambda * sum_j a_jk^2 (scale invariant); lambda < 0: a_kk -= lambda;
//  * the Cholesky factorization fails (LM stops) only on an exactly-zero pivot;
//  * Fisher inverse by LUP with partial pivoting and tolerance 1e-9 (failure -> +Inf CRLB).
// By design: a pivot that lost more than six decimal digits (v <= 1e-6 * a_kk, including
// v < 0) is re-solved in FP64; the Fisher matrix is inverted in FP64 instead of FP32.
//
// Arithmetic of the LM step, chosen at compile time:
//   PB200_LM_IEEE_RCP  1: the per-pixel weight uses the IEEE reciprocal 1/mu, as
//                         Estimation.h:116-117 does; 0: the approximate reciprocal (1 ulp).
//   PB200_LM_IEEE_CHOL 1: the damped Cholesky solve takes square roots and divides with the
//                         reference's operation order and no contraction (SolveMatrix.h:107-163,
//                         Estimation.h:213-223); 0: pivots applied through rsqrt products.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef PB200_LM_IEEE_RCP
#define PB200_LM_IEEE_RCP 0
#endif
#ifndef PB200_LM_IEEE_CHOL
#define PB200_LM_IEEE_CHOL 0
#endif

namespace pb200 {

enum FitFlags : int {
    FIT_CRLB_ONLY = 1,  // skip LM: params come from `initial`, compute Fisher/CRLB/chi^2 only
};

// Which passes a kernel instance contains: both (the mixed-batch kernel), the LM fit only, or
// the Fisher/CRLB (+ GLRT) pass only. The standalone launches use the single-pass instances:
// without the other pass's code and registers they run faster (the host issues the LM launch,
// then the Fisher launch at the fitted parameters).
enum FitPass { PASS_BOTH = 0, PASS_LM = 1, PASS_FISHER = 2 };

struct FitArgs {
    const float* smp;      // [n][npix] (may be null with FIT_CRLB_ONLY: no chi-square)
    const float* consts;   // [n][numconst] or null
    const float* initial;  // [n][K] or null (centre-of-mass start)
    float* params;         // [n][K]
    int* iterations;       // [n] or null
    float* trace;          // [n][traceLen][K] or null
    int traceLen;
    float* crlb;           // [n][K] or null (no Fisher pass)
    float* chisq;          // [n] or null
    int* diag;             // [n] or null: 1 when an FP64 re-solve happened for the spot
    float* fisher;         // [n][K(K+1)/2 + 1] scratch: packed FP32 Fisher matrix + chi-square, inverted
                           // afterwards by crlb_kernel; null = invert in the fit kernel (lane 0)
    float* glrt;           // [n][3] or null: {ll_on, ll_off, mean} of the likelihood-ratio test
    const float* glrtMeanRoi;  // null: each spot's own mean; else every spot's mean comes from these npix
                               // samples (the reference's behaviour, see glrt_store)
    int n;
    int maxIter;
    float lambda;
    int smemStride;        // floats of shared memory per group
    int flags;
    int* claim;            // null: group g fits ROIs g, g + groups, ...; else (LM launches) a counter, zeroed
                           // by the launcher, from which each group takes its next ROI when it is done
};

__host__ __device__ constexpr int round_up(int a, int b) { return (a + b - 1) / b * b; }
__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

// Packed upper-triangle index (i <= j) of a symmetric K x K matrix, row-major.
// Written without recursion so that, inside fully unrolled loops, it folds to a constant and
// the packed arrays it indexes stay in registers.
__host__ __device__ __forceinline__ constexpr int upk(int i, int j, int K) {
    return (i <= j) ? (i * K - (i * (i - 1)) / 2 + (j - i)) : (j * K - (j * (j - 1)) / 2 + (i - j));
}
// Packed lower-triangle index (j <= i).
__host__ __device__ __forceinline__ constexpr int lok(int i, int j) { return i * (i + 1) / 2 + j; }

// Floats of shared memory for the FP64 LM re-solve (doubles first: D packed, y; then floats).
__host__ __device__ constexpr int rescue_floats(int K) { return 3 * (K * (K + 1) / 2) + 5 * K + 1; }

template <int G>
__device__ __forceinline__ unsigned group_mask() {
    if (G == 32) return 0xffffffffu;
    const unsigned lane = threadIdx.x & 31;
    return ((1u << (G & 31)) - 1u) << (lane & ~(unsigned)(G - 1));
}

template <int G>
__device__ __forceinline__ float group_sum(float v, unsigned mask) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
}

// Streamed input of a fit launch that starts before all of its ROIs have arrived: a copy engine
// writes the ROIs of block b (1 << kStreamBlockShift ROIs), then sets flags[1 + b]; flags[0] is
// the error flag. Waits for the block of `roi` with acquire loads and growing sleeps; gives up
// after about 1-2 s of polling (2^20 polls; a chunk's copy takes milliseconds), or at once when
// another group already has, sets the error flag and returns false.
constexpr int kStreamBlockShift = 10;
__device__ __forceinline__ bool wait_stream_ready(int* flags, int roi) {
    const int* f = flags + 1 + (roi >> kStreamBlockShift);
    unsigned ns = 32;
    for (int i = 0; i < (1 << 20); i++) {
        int v, err;
        asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(f) : "memory");
        if (v) return true;
        asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(err) : "l"(flags) : "memory");
        if (err) return false;
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
    }
    atomicExch(flags, 1);
    return false;
}

// First of `count` ROIs taken from a launch's counter by a group of G lanes (lane 0 takes them).
template <int G>
__device__ __forceinline__ int group_claim(int* counter, int count, int lane, unsigned mask) {
    int r = 0;
    if (lane == 0) r = atomicAdd(counter, count);
    return __shfl_sync(mask, r, 0, G);
}

// 1/x for x >= 1e-8 (never denormal): approximate reciprocal + one Newton step, no branch.
__device__ __forceinline__ float rcp_nr(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    const float e = fmaf(-x, r, 1.0f);
    return fmaf(r, e, r);
}

// 1/x with the approximate reciprocal alone (within 1 ulp), for the per-pixel LM weights.
__device__ __forceinline__ float rcp_fast(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// 1/mu of the per-pixel LM weight (x >= 1e-6).
__device__ __forceinline__ float lm_rcp(float x) {
#if PB200_LM_IEEE_RCP
    return __frcp_rn(x);
#else
    return rcp_fast(x);
#endif
}

// Damped LM step with the reference's arithmetic: damping (Estimation.h:213-223), Cholesky
// (SolveMatrix.h:107-125) and the two triangular solves (SolveMatrix.h:145-163), each sum
// formed left to right with separately rounded products, square roots and quotients IEEE
// rounded. Same return codes as lm_solve below.
template <int K, int NACC>
__device__ __forceinline__ int lm_solve_ieee(const float (&acc)[NACC], float lambda, float (&step)[K], float (&dk)[K]) {
    constexpr int NA = K * (K + 1) / 2;
    float A[K][K];
    {
        int q = 0;
#pragma unroll
        for (int i = 0; i < K; i++)
#pragma unroll
            for (int j = i; j < K; j++) {
                A[i][j] = acc[q];
                A[j][i] = acc[q];
                q++;
            }
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
        float s = 0.0f;
#pragma unroll
        for (int j = 0; j < K; j++) s = __fadd_rn(s, __fmul_rn(A[j][k], A[j][k]));
        dk[k] = (lambda < 0.0f) ? __fsub_rn(A[k][k], lambda) : __fadd_rn(A[k][k], __fmul_rn(s, lambda));
    }
    float L[K][K];
    int status = 1;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        float sum = 0.0f;
#pragma unroll
        for (int p = 0; p < k; ++p) sum = __fadd_rn(sum, __fmul_rn(L[k][p], L[k][p]));
        const float v = __fsub_rn(dk[k], sum);
        if (v == 0.0f) status = 0;
        else if (!(v > 1e-6f * dk[k]) && status == 1) status = 2;  // also catches v < 0 and NaN
        L[k][k] = __fsqrt_rn(v);
#pragma unroll
        for (int i = k + 1; i < K; ++i) {
            float s2 = 0.0f;
#pragma unroll
            for (int p = 0; p < k; ++p) s2 = __fadd_rn(s2, __fmul_rn(L[i][p], L[k][p]));
            L[i][k] = __fdiv_rn(__fsub_rn(A[i][k], s2), L[k][k]);
        }
    }
    float y[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        float sum = 0.0f;
#pragma unroll
        for (int k = 0; k < i; ++k) sum = __fadd_rn(sum, __fmul_rn(L[i][k], y[k]));
        y[i] = __fdiv_rn(__fsub_rn(acc[NA + i], sum), L[i][i]);
    }
#pragma unroll
    for (int i = K - 1; i >= 0; --i) {
        float sum = 0.0f;
#pragma unroll
        for (int k = i + 1; k < K; ++k) sum = __fadd_rn(sum, __fmul_rn(L[k][i], step[k]));
        step[i] = __fdiv_rn(__fsub_rn(y[i], sum), L[i][i]);
    }
    return status;
}

// Damped LM step in registers. acc = [alpha upper packed (NA) | beta (K) | extra].
// Returns 1 on success, 0 on an exactly-zero pivot (reference failure), 2 when a pivot is
// weak and the step must be re-solved in FP64. (Two-dimensional arrays and running packed
// indices keep every access compile-time after unrolling, so nothing lands in local memory.)
template <int K, int NACC>
__device__ __forceinline__ int lm_solve(const float (&acc)[NACC], float lambda, float (&step)[K], float (&dk)[K]) {
#if PB200_LM_IEEE_CHOL
    return lm_solve_ieee<K, NACC>(acc, lambda, step, dk);
#endif
    constexpr int NA = K * (K + 1) / 2;
    float A[K][K];
    {
        int q = 0;
#pragma unroll
        for (int i = 0; i < K; i++)
#pragma unroll
            for (int j = i; j < K; j++) {
                A[i][j] = acc[q];
                A[j][i] = acc[q];
                q++;
            }
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
        float s = 0.0f;
#pragma unroll
        for (int j = 0; j < K; j++) s += A[j][k] * A[j][k];
        dk[k] = (lambda < 0.0f) ? A[k][k] - lambda : A[k][k] + s * lambda;
    }
    float L[K][K], Linv[K];
    int status = 1;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        float sum = 0.0f;
#pragma unroll
        for (int p = 0; p < k; ++p) sum += L[k][p] * L[k][p];
        const float v = dk[k] - sum;
        if (v == 0.0f) status = 0;
        else if (!(v > 1e-6f * dk[k]) && status == 1) status = 2;  // also catches v < 0 and NaN
        const float inv = rsqrtf(v);
        L[k][k] = v * inv;
        Linv[k] = inv;
#pragma unroll
        for (int i = k + 1; i < K; ++i) {
            float s2 = 0.0f;
#pragma unroll
            for (int p = 0; p < k; ++p) s2 += L[i][p] * L[k][p];
            L[i][k] = (A[i][k] - s2) * inv;
        }
    }
    float y[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
        float sum = 0.0f;
#pragma unroll
        for (int k = 0; k < i; ++k) sum += L[i][k] * y[k];
        y[i] = (acc[NA + i] - sum) * Linv[i];
    }
#pragma unroll
    for (int i = K - 1; i >= 0; --i) {
        float sum = 0.0f;
#pragma unroll
        for (int k = i + 1; k < K; ++k) sum += L[k][i] * step[k];
        step[i] = (y[i] - sum) * Linv[i];
    }
    return status;
}

// FP64 Cholesky solve by one lane. A: packed upper (float, NA), b: K, dk: damped diagonal.
// Scratch: D packed lower (double, NA), y (double, K). Writes x (float, K). Returns false when a
// pivot is zero or negative: the FP32 Hessian is then not positive definite even in FP64 (its
// accumulation rounding exceeds what is left of the pivot), and the fit stops at its current
// parameters, as the reference's fit does on a zero pivot, instead of taking a NaN step.
static __device__ __noinline__ bool lm_solve_fp64_lane(int K, const float* A, const float* b, const float* dk, double* D,
                                               double* y, float* x) {
    for (int k = 0; k < K; ++k) {
        double sum = 0.0;
        for (int p = 0; p < k; ++p) sum += D[lok(k, p)] * D[lok(k, p)];
        const double v = (double)dk[k] - sum;
        if (!(v > 0.0)) return false;
        D[lok(k, k)] = sqrt(v);
        for (int i = k + 1; i < K; ++i) {
            double s2 = 0.0;
            for (int p = 0; p < k; ++p) s2 += D[lok(i, p)] * D[lok(k, p)];
            D[lok(i, k)] = ((double)A[upk(i, k, K)] - s2) / D[lok(k, k)];
        }
    }
    for (int i = 0; i < K; ++i) {
        double sum = 0.0;
        for (int k = 0; k < i; ++k) sum += D[lok(i, k)] * y[k];
        y[i] = ((double)b[i] - sum) / D[lok(i, i)];
    }
    for (int i = K - 1; i >= 0; --i) {
        double sum = 0.0;
        for (int k = i + 1; k < K; ++k) sum += D[lok(k, i)] * y[k];
        y[i] = (y[i] - sum) / D[lok(i, i)];  // y[k>i] already hold the solution
    }
    for (int i = 0; i < K; ++i) x[i] = (float)y[i];
    return true;
}

// FP64 LUP inverse with the reference's 1e-9 tolerance (SolveMatrix.h:219-318, 344-392), one
// lane on shared memory: A[K*K] is overwritten, IA[K*K] receives the inverse.
static __device__ __noinline__ bool invert_fp64_lane(int K, double* A, double* IA) {
    int P[8];
    for (int i = 0; i <= K; i++) P[i] = i;
    for (int i = 0; i < K; i++) {
        double maxA = 0.0;
        int imax = i;
        for (int k = i; k < K; k++) {
            const double v = fabs(A[k * K + i]);
            if (v > maxA) { maxA = v; imax = k; }
        }
        if (maxA < (double)1e-9f) return false;
        if (imax != i) {
            const int tp = P[i]; P[i] = P[imax]; P[imax] = tp;
            for (int j = 0; j < K; j++) {
                const double t = A[i * K + j]; A[i * K + j] = A[imax * K + j]; A[imax * K + j] = t;
            }
            P[K]++;
        }
        for (int j = i + 1; j < K; j++) {
            A[j * K + i] /= A[i * K + i];
            for (int k = i + 1; k < K; k++) A[j * K + k] -= A[j * K + i] * A[i * K + k];
        }
    }
    for (int j = 0; j < K; j++) {
        for (int i = 0; i < K; i++) {
            double v = (P[i] == j) ? 1.0 : 0.0;
            for (int k = 0; k < i; k++) v -= A[i * K + k] * IA[k * K + j];
            IA[i * K + j] = v;
        }
        for (int i = K - 1; i >= 0; i--) {
            double v = IA[i * K + j];
            for (int k = i + 1; k < K; k++) v -= A[i * K + k] * IA[k * K + j];
            IA[i * K + j] = v / A[i * K + i];
        }
    }
    return true;
}

// Group-wide FP64 re-solve: lane 0 solves on `scratch` (>= rescue_floats(K) floats, 8-byte
// aligned), every lane receives the step. Returns false on a zero pivot.
template <int K, int NACC>
__device__ __forceinline__ bool lm_rescue(const float (&acc)[NACC], const float (&dk)[K], float (&step)[K],
                                          float* scratch, int lane, unsigned mask) {
    constexpr int NA = K * (K + 1) / 2;
    double* D = reinterpret_cast<double*>(scratch);
    double* yv = D + NA;
    float* A = reinterpret_cast<float*>(yv + K);
    float* b = A + NA;
    float* dd = b + K;
    float* xs = dd + K;
    float* flag = xs + K;
    __syncwarp(mask);
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NA; q++) A[q] = acc[q];
#pragma unroll
        for (int q = 0; q < K; q++) {
            b[q] = acc[NA + q];
            dd[q] = dk[q];
        }
        flag[0] = lm_solve_fp64_lane(K, A, b, dd, D, yv, xs) ? 1.0f : 0.0f;
    }
    __syncwarp(mask);
    const bool ok = flag[0] != 0.0f;
#pragma unroll
    for (int q = 0; q < K; q++) step[q] = xs[q];
    __syncwarp(mask);
    return ok;
}

// Likelihood-ratio test against a background-only model (GLRT_PSF.cu:104-131), evaluated
// after the Fisher pass at the final parameters. With d = max(x, 1e-8), mu8 = max(mu, 1e-8):
//   ll_on  = sum_p d log(mu8) - mu8     (summed over the pixels by the caller: llOn)
//   mean   = sum_p x / npix              (sumRaw; exact for integer counts in any order)
//   ll_off = sum_p d log(mean) - mean = log(mean) sum_p d - npix mean   (sumD = sum_p d)
// The reference computes `mean` from the first ROI of each call for every spot (its loop
// variable shadows the spot index, GLRT_PSF.cu:107-109); a non-null a.glrtMeanRoi reproduces
// that, summing those samples sequentially as the reference does. By default each spot uses
// its own mean.
__device__ __forceinline__ void glrt_store(float llOn, float sumD, float sumRaw, const FitArgs& a, int roi, int npix,
                                           int lane) {
    if (lane != 0) return;
    float mean = sumRaw;
    if (a.glrtMeanRoi) {
        mean = 0.0f;
        for (int i = 0; i < npix; i++) mean += a.glrtMeanRoi[i];
    }
    mean = __fdiv_rn(mean, (float)npix);
    float* o = a.glrt + (size_t)roi * 3;
    o[0] = llOn;
    o[1] = sumD * logf(mean) - (float)npix * mean;
    o[2] = mean;
}

// Fisher pass epilogue, deferred form: the group's lanes store the packed FP32 Fisher matrix
// and the chi-square of ROI `roi` into the scratch row; crlb_kernel inverts it later.
template <int K, int NACC, int G>
__device__ __forceinline__ void fisher_store(const float (&acc)[NACC], float* row, int lane) {
    constexpr int NA = K * (K + 1) / 2;
#pragma unroll
    for (int q = 0; q < NA; q++)
        if ((q % G) == lane) row[q] = acc[q];
    if (lane == ((NA) % G)) row[NA] = acc[NACC - 1];
}

// One thread per ROI: FP64 LUP inverse of the packed Fisher matrix (reference algorithm and
// 1e-9 tolerance, SolveMatrix.h:219-318, 344-392), CRLB = sqrt(diag) (+Inf when singular, as
// Estimation.h:101 via InvertMatrix), chi-square copied out. ABS: sqrt(|diag|), as
// ComputeCRLB (Estimation.h:318-333) does for the intensity/background fit.
template <int K, bool ABS = false>
__global__ void __launch_bounds__(128) crlb_kernel(const float* __restrict__ fisher, float* __restrict__ crlb,
                                                   float* __restrict__ chisq, int n) {
    constexpr int NA = K * (K + 1) / 2;
    for (int roi = blockIdx.x * blockDim.x + threadIdx.x; roi < n; roi += gridDim.x * blockDim.x) {
        const float* row = fisher + (size_t)roi * (NA + 1);
        double A[K][K];
        {
            int q = 0;
#pragma unroll
            for (int i = 0; i < K; i++)
#pragma unroll
                for (int j = i; j < K; j++) {
                    const double v = (double)row[q++];
                    A[i][j] = v;
                    A[j][i] = v;
                }
        }
        int P[K];
#pragma unroll
        for (int i = 0; i < K; i++) P[i] = i;
        bool ok = true;
#pragma unroll
        for (int i = 0; i < K; i++) {
            double maxA = 0.0;
            int imax = i;
#pragma unroll
            for (int k = i; k < K; k++) {
                const double v = fabs(A[k][i]);
                if (v > maxA) { maxA = v; imax = k; }
            }
            if (maxA < (double)1e-9f) ok = false;
            // row swap i <-> imax with compile-time indices only
#pragma unroll
            for (int r = i + 1; r < K; r++) {
                if (r == imax) {
                    const int tp = P[i]; P[i] = P[r]; P[r] = tp;
#pragma unroll
                    for (int j = 0; j < K; j++) {
                        const double t = A[i][j]; A[i][j] = A[r][j]; A[r][j] = t;
                    }
                }
            }
#pragma unroll
            for (int j = i + 1; j < K; j++) {
                A[j][i] /= A[i][i];
#pragma unroll
                for (int k = i + 1; k < K; k++) A[j][k] -= A[j][i] * A[i][k];
            }
        }
        // column j of the inverse: forward (unit lower) then backward substitution; keep the diagonal
        float* out = crlb + (size_t)roi * K;
#pragma unroll
        for (int j = 0; j < K; j++) {
            double x[K];
#pragma unroll
            for (int i = 0; i < K; i++) {
                double v = (P[i] == j) ? 1.0 : 0.0;
#pragma unroll
                for (int k = 0; k < i; k++) v -= A[i][k] * x[k];
                x[i] = v;
            }
#pragma unroll
            for (int i = K - 1; i >= 0; i--) {
                double v = x[i];
#pragma unroll
                for (int k = i + 1; k < K; k++) v -= A[i][k] * x[k];
                x[i] = v / A[i][i];
            }
            out[j] = ok ? (float)sqrt(ABS ? fabs(x[j]) : x[j]) : __int_as_float(0x7f800000);
        }
        if (chisq) chisq[roi] = row[NA];
    }
}

// Fisher pass epilogue, in-kernel form: FP64 inverse on lane 0, CRLB = sqrt(diag), chi-square.
template <int K, int NACC>
__device__ __forceinline__ void fisher_finish(const float (&acc)[NACC], float* scratch, int lane, unsigned mask,
                                              float* crlb, float* chisq) {
    __syncwarp(mask);
    if (lane == 0) {
        double* F = reinterpret_cast<double*>(scratch);
        double* IF = F + K * K;
        int q = 0;
#pragma unroll
        for (int i = 0; i < K; i++)
#pragma unroll
            for (int j = i; j < K; j++) {
                F[i * K + j] = (double)acc[q];
                F[j * K + i] = (double)acc[q];
                q++;
            }
        const bool ok = invert_fp64_lane(K, F, IF);
        for (int k = 0; k < K; k++) crlb[k] = ok ? (float)sqrt(IF[k * (K + 1)]) : __int_as_float(0x7f800000);
        if (chisq) *chisq = acc[NACC - 1];
    }
    __syncwarp(mask);
}

}  // namespace pb200
