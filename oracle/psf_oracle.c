/* CPU oracle for the batched Poisson-MLE PSF estimator.
 *
 * TEST INFRASTRUCTURE ONLY. This file is a plain-C restatement of photonpy's
 * estimator arithmetic (cpp/SMLMLib/Estimators/Estimation.h, SolveMatrix.h,
 * Estimators/Gaussian/GaussianPSFModels.h, Estimators/CSpline/CubicSplinePSFModels.h,
 * Estimators/CSpline/CubicSplinePSF.cu). It exists so that tests/, the smoke
 * check and bench.py's CPU-baseline leg can check the CUDA product against the
 * reference's algorithm. The product (photonpy_b200) never links or calls it.
 *
 * Parity pin: tests/test_oracle.py checks the FP32 build of this file against
 * golden vectors produced by the reference's own C++ CPU estimator
 * (tests/golden/make_golden.py, built by oracle/build_ref.sh).
 *
 * Build: gcc -O2 -fPIC -shared -ffp-contract=off (no FMA contraction, like the
 * reference's host -O3 build on x86-64 without -march=native).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define PSO_MAXK 8

enum {
    PSO_XYIBG = 0,            /* Gauss2D_Model_XYIBg            (GaussianPSFModels.h:35-152)  */
    PSO_XYIBG_CONSTSIGMA = 1, /* Gauss2D_Model_XYIBgConstSigma  (GaussianPSFModels.h:156-227) */
    PSO_XYIBG_SIGMA = 2,      /* Gauss2D_Model_XYIBgSigma       (GaussianPSFModels.h:308-387) */
    PSO_XYIBG_SIGMAXY = 3,    /* Gauss2D_Model_XYIBgSigmaXY     (GaussianPSFModels.h:391-471) */
    PSO_XYZIBG = 4,           /* Gauss2D_Model_XYZIBg (astig)   (GaussianPSFModels.h:636-751) */
    PSO_CSPLINE = 5,          /* CSpline_Model_XYZIBg           (CubicSplinePSFModels.h:14-154) */
    PSO_XYITILTEDBG = 6,      /* Gauss2D_Model_XYITiltedBg      (GaussianPSFModels.h:228-304) */
    PSO_XYITILTEDBG_SIGMAXY = 7, /* Gauss2D_Model_XYITiltedBgSigmaXY (GaussianPSFModels.h:474-558) */
    PSO_INTENSITYBG = 8,      /* IntensityBgModel (GaussianPSFModels.h:562-615): theta = (I, bg),
                                 constants = (x, y, sigma), mu = I * DeltaX DeltaY + bg */
    PSO_CSPLINE_TILTED = 9,   /* CSpline_Model_XYZITiltedBg     (CubicSplinePSFModels.h:157-298) */
    PSO_CSPLINE_BGIMAGE = 10  /* CSpline_Model_XYZIBgImage      (CubicSplinePSFModels.h:300-443) */
};

typedef struct {
    int model;
    int roisize;
    float sigma[2];         /* fixed sigma (XYIBg) or initial sigma(s) (Sigma, SigmaXY)        */
    float astig_x[5];       /* s0, gamma, d, A, B   (B = 0 is the reference's 4-term form)    */
    float astig_y[5];
    float minz, maxz;
    int spline_shape[3];    /* coefficient grid (z, y, x)                                      */
    float spline_zmin, spline_zmax;
    const float* coefs;     /* [Nz][Ny][Nx][64]                                                */
    float spline_q;         /* spline voxels per ROI pixel in x and y (0 or 1: photonpy's      */
                            /* one voxel per pixel; 2: a calibration sampled at 0.5 px)        */
} pso_model_t;

int pso_num_params(int model)
{
    switch (model) {
    case PSO_XYIBG: case PSO_XYIBG_CONSTSIGMA: return 4;
    case PSO_XYIBG_SIGMAXY: case PSO_XYITILTEDBG: return 6;
    case PSO_XYITILTEDBG_SIGMAXY: return 8;
    case PSO_INTENSITYBG: return 2;
    case PSO_CSPLINE_TILTED: return 7;
    default: return 5;
    }
}

int pso_num_constants(int model)
{
    if (model == PSO_INTENSITYBG) return 3;
    return (model == PSO_XYIBG_CONSTSIGMA || model == PSO_XYITILTEDBG) ? 2 : 0;
}

/* Constants per spot of a model instance: the background-image spline takes a whole image. */
int pso_model_constants(const pso_model_t* m)
{
    if (m->model == PSO_CSPLINE_BGIMAGE) return m->roisize * m->roisize;
    return pso_num_constants(m->model);
}

int pso_sizeof_model(void) { return (int)sizeof(pso_model_t); }

/* ---- FP32: the reference's arithmetic ---- */
#define REAL float
#define SUFFIX _f32
#define ERF erff
#define EXP expf
#define SQRT sqrtf
#define FMAX fmaxf
#define FMIN fminf
#define FABS fabsf
#include "psf_oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef ERF
#undef EXP
#undef SQRT
#undef FMAX
#undef FMIN
#undef FABS

/* ---- FP64 oracle ---- */
#define REAL double
#define SUFFIX _f64
#define ERF erf
#define EXP exp
#define SQRT sqrt
#define FMAX fmax
#define FMIN fmin
#define FABS fabs
#include "psf_oracle_impl.h"

/* CSpline_Compute (CubicSplinePSF.cu:151-204): per output voxel, the 4x4x4 neighbourhood
 * (clamped at the border) is solved against the 64x64 power-basis matrix with a double
 * LUP decomposition. Output shape = shape - 3 + 2*border, 64 coefficients per voxel,
 * coefficient index = zpow*16 + ypow*4 + xpow. */
int pso_spline_compute(const int* shape, const float* data, float* coefs, int border)
{
    static double A[64 * 64];
    int P[65];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            for (int k = 0; k < 4; k++)
                for (int l = 0; l < 4; l++)
                    for (int m = 0; m < 4; m++)
                        for (int n = 0; n < 4; n++)
                            A[64 * (i * 16 + j * 4 + k) + (l * 16 + m * 4 + n)] =
                                (double)(powf((float)(i - 1.0), (float)l) * powf((float)(j - 1.0), (float)m) *
                                         powf((float)(k - 1.0), (float)n));
    const int N = 64;
    for (int i = 0; i <= N; i++) P[i] = i;
    for (int i = 0; i < N; i++) {
        double maxA = 0, absA;
        int imax = i;
        for (int k = i; k < N; k++)
            if ((absA = fabs(A[k * N + i])) > maxA) { maxA = absA; imax = k; }
        if (maxA < (double)1e-10f) return -1;
        if (imax != i) {
            int j = P[i]; P[i] = P[imax]; P[imax] = j;
            for (int jj = 0; jj < N; jj++) {
                double t = A[i * N + jj]; A[i * N + jj] = A[imax * N + jj]; A[imax * N + jj] = t;
            }
            P[N]++;
        }
        for (int j = i + 1; j < N; j++) {
            A[j * N + i] /= A[i * N + i];
            for (int k = i + 1; k < N; k++) A[j * N + k] -= A[j * N + i] * A[i * N + k];
        }
    }
    const int o0 = shape[0] - 3 + border * 2, o1 = shape[1] - 3 + border * 2, o2 = shape[2] - 3 + border * 2;
    for (int i = 0; i < o0; i++)
        for (int j = 0; j < o1; j++)
            for (int k = 0; k < o2; k++) {
                double b[64], x[64];
                for (int m = 0; m < 4; m++)
                    for (int n = 0; n < 4; n++)
                        for (int o = 0; o < 4; o++) {
                            int z = i + m - border, y = j + n - border, xx = k + o - border;
                            z = z < 0 ? 0 : (z > shape[0] - 1 ? shape[0] - 1 : z);
                            y = y < 0 ? 0 : (y > shape[1] - 1 ? shape[1] - 1 : y);
                            xx = xx < 0 ? 0 : (xx > shape[2] - 1 ? shape[2] - 1 : xx);
                            b[m * 16 + n * 4 + o] = data[(size_t)shape[1] * shape[2] * z + (size_t)shape[2] * y + xx];
                        }
                for (int r = 0; r < N; r++) {
                    x[r] = b[P[r]];
                    for (int q = 0; q < r; q++) x[r] -= A[r * N + q] * x[q];
                }
                for (int r = N - 1; r >= 0; r--) {
                    for (int q = r + 1; q < N; q++) x[r] -= A[r * N + q] * x[q];
                    x[r] = x[r] / A[r * N + r];
                }
                float* dst = coefs + 64 * ((size_t)o1 * o2 * i + (size_t)o2 * j + k);
                for (int a = 0; a < 64; a++) dst[a] = (float)x[a];
            }
    return 0;
}

/* Likelihood-ratio test of GLRT_PSF::Estimate (GLRT_PSF.cu:96-131), after the fit: per spot
 * out[3] = {ll_on, ll_off, mean}, with mu = the model's expected value at params[spot]
 * clamped at 1e-8, d = max(sample, 1e-8), mean = (sequential float sum of the mean source)
 * / npix, ll_on = sum d log(mu) - mu, ll_off = sum d log(mean) - mean, both summed pixel by
 * pixel in row-major order as the reference does. mean_roi == NULL: each spot's own samples
 * are the mean source; otherwise every spot uses mean_roi (npix floats), which is what the
 * reference computes (its mean loop reads the first ROI of the call, GLRT_PSF.cu:107-108). */
int pso_glrt_f32(const pso_model_t* m, int n, const float* params, const float* samples, const float* constants,
                 const float* mean_roi, float* out)
{
    const int K = pso_num_params(m->model), npix = m->roisize * m->roisize, nc = pso_model_constants(m);
    float* ev = (float*)malloc(sizeof(float) * npix);
    for (int s = 0; s < n; s++) {
        const float* smp = samples + (size_t)s * npix;
        pso_derivatives_f32(m, 1, params + (size_t)s * K, nc ? constants + (size_t)s * nc : NULL, NULL, ev);
        const float* src = mean_roi ? mean_roi : smp;
        float mean = 0.0f;
        for (int p = 0; p < npix; p++) mean += src[p];
        mean /= (float)npix;
        float ll_on = 0.0f, ll_off = 0.0f;
        for (int p = 0; p < npix; p++) {
            const float mu = fmaxf(ev[p], 1e-8f);
            const float d = fmaxf(smp[p], 1e-8f);
            ll_on += d * logf(mu) - mu;
            ll_off += d * logf(mean) - mean;
        }
        out[(size_t)s * 3 + 0] = ll_on;
        out[(size_t)s * 3 + 1] = ll_off;
        out[(size_t)s * 3 + 2] = mean;
    }
    free(ev);
    return 0;
}

/* ---- Spot detection (SpotDetection/SpotDetector.cu:49-84, 101-151; ImageFilters.h:6-105) ----
 * Box filter with windows clipped at the image border: X pass then Y pass, each a sequential
 * float sum over [c - win/2, c - win/2 + win) divided by the number of pixels in the window. */
static void sd_box(const float* in, float* tmp, float* out, int w, int h, int win)
{
    const int back = -win / 2, forw = back + win;
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            int xs = x + back; if (xs < 0) xs = 0;
            int xe = x + forw; if (xe > w) xe = w;
            float sum = 0.0f;
            for (int i = xs; i < xe; i++) sum += in[(size_t)y * w + i];
            tmp[(size_t)y * w + x] = sum / (float)(xe - xs);
        }
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            int ys = y + back; if (ys < 0) ys = 0;
            int ye = y + forw; if (ye > h) ye = h;
            float sum = 0.0f;
            for (int i = ys; i < ye; i++) sum += tmp[(size_t)i * w + x];
            out[(size_t)y * w + x] = sum / (float)(ye - ys);
        }
}

/* Maximum filter (ComparisonFilter2DStack with depth 1 and thrust::maximum: a < b ? b : a). */
static void sd_max(const float* in, float* tmp, float* out, int w, int h, int win)
{
    const int back = -win / 2, forw = back + win;
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            int xs = x + back; if (xs < 0) xs = 0;
            int xe = x + forw; if (xe > w) xe = w;
            float v = in[(size_t)y * w + xs];
            for (int i = xs + 1; i < xe; i++) { float b = in[(size_t)y * w + i]; v = v < b ? b : v; }
            tmp[(size_t)y * w + x] = v;
        }
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            int ys = y + back; if (ys < 0) ys = 0;
            int ye = y + forw; if (ye > h) ye = h;
            float v = tmp[(size_t)ys * w + x];
            for (int i = ys + 1; i < ye; i++) { float b = tmp[(size_t)i * w + x]; v = v < b ? b : v; }
            out[(size_t)y * w + x] = v;
        }
}

/* Detection of one frame: detection image D = box(src - bg, u1) - box(src - bg, u2); a pixel is
 * a spot when D equals its max-filtered value, lies more than roisize/2 from the left/top border
 * and its ROI ends before the last row/column, and min_i < D < max_i. Spots in row-major pixel
 * order; the first max_spots are written (index y*w + x, score D). Returns the number found. */
int pso_detect_spots(const float* frame, const float* bg, int w, int h, int u1, int u2, int mf, int roisize,
                     float min_i, float max_i, int max_spots, int* idx, float* score)
{
    const size_t n = (size_t)w * h;
    float* src = (float*)malloc(sizeof(float) * n);
    float* tmp = (float*)malloc(sizeof(float) * n);
    float* f1 = (float*)malloc(sizeof(float) * n);
    float* f2 = (float*)malloc(sizeof(float) * n);
    float* mx = (float*)malloc(sizeof(float) * n);
    for (size_t p = 0; p < n; p++) src[p] = bg ? frame[p] - bg[p] : frame[p];
    sd_box(src, tmp, f1, w, h, u1);
    sd_box(src, tmp, f2, w, h, u2);
    for (size_t p = 0; p < n; p++) f1[p] = f1[p] - f2[p];
    sd_max(f1, tmp, mx, w, h, mf);
    int found = 0;
    const int half = roisize / 2, rest = roisize - roisize / 2;
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const float a = f1[(size_t)y * w + x], b = mx[(size_t)y * w + x];
            const int isMax = a == b && x > half && y > half && x + rest < w - 1 && y + rest < h - 1;
            if (isMax && b > min_i && b < max_i) {
                if (found < max_spots) {
                    idx[found] = y * w + x;
                    score[found] = b;
                }
                found++;
            }
        }
    free(src); free(tmp); free(f1); free(f2); free(mx);
    return found;
}

/* ROIs of SpotDetector_ProcessFrame: corner = (y, x) - roisize/2, pixels clamped to the frame. */
void pso_cut_rois(const float* frame, int w, int h, const int* idx, int n, int roisize, int* corner_yx, float* rois)
{
    for (int i = 0; i < n; i++) {
        const int cy = idx[i] / w - roisize / 2, cx = idx[i] % w - roisize / 2;
        corner_yx[2 * i] = cy;
        corner_yx[2 * i + 1] = cx;
        for (int y = 0; y < roisize; y++)
            for (int x = 0; x < roisize; x++) {
                int fy = cy + y, fx = cx + x;
                if (fx < 0) fx = 0;
                if (fy < 0) fy = 0;
                if (fx >= w) fx = w - 1;
                if (fy >= h) fy = h - 1;
                rois[((size_t)i * roisize + y) * roisize + x] = frame[(size_t)fy * w + fx];
            }
    }
}
