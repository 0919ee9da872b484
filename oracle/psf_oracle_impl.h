/* Type-generic body of the CPU oracle. Included twice by psf_oracle.c:
 * once with REAL=float (the reference's own arithmetic, same operation order,
 * compiled without FMA contraction) and once with REAL=double (the FP64 oracle
 * used to state every result's error).
 *
 * TEST INFRASTRUCTURE ONLY: the product never links or calls this code.
 *
 * Reference anchors (paths inside photonpy's cpp/SMLMLib):
 *   LevMarOptimize            Estimators/Estimation.h:194-251
 *   ComputeLevMarAlphaBeta    Estimators/Estimation.h:104-134
 *   ComputeChiSquareAndCRLB   Estimators/Estimation.h:63-102
 *   ComputeCOM                Estimators/Estimation.h:336-352
 *   Cholesky / SolveCholesky  SolveMatrix.h:107-125, 145-163
 *   LUPDecompose / LUPInvert  SolveMatrix.h:267-318, 344-367; InvertMatrix 411-452
 *   Gaussian models           Estimators/Gaussian/GaussianPSFModels.h:35-471, 636-751
 *   Cubic spline model        Estimators/CSpline/CubicSplinePSFModels.h:14-154
 *   Tilted-background models  Estimators/Gaussian/GaussianPSFModels.h:228-304, 474-558
 *   Intensity/background fit  Estimators/Gaussian/GaussianPSFModels.h:562-615 (IntensityBgModel),
 *                             Estimators/Gaussian/GaussianPSF.cu:216-240, Estimation.h:318-333
 */

#define FN(name) CAT(name, SUFFIX)
#define CAT(a, b) CAT_(a, b)
#define CAT_(a, b) a##b

/* clamp(f,a,b) = fmax(a, fmin(f, b)) exactly as CudaMath.h:1152-1155 */
static inline REAL FN(o_clamp)(REAL f, REAL a, REAL b) { return FMAX(a, FMIN(f, b)); }
/* largest integer <= f, in the REAL type */
static inline REAL FN(o_floor)(REAL f) { REAL t = (REAL)(long long)f; return t > f ? t - 1 : t; }

/* Per-pixel model values: mu[p] and jac[k*npix + p], row-major pixels. */
static void FN(model_eval)(const pso_model_t* m, const REAL* theta, const float* consts,
                           REAL* mu, REAL* jac)
{
    const int H = m->roisize, W = m->roisize, npix = H * W;
    const REAL PI_ = (REAL)3.141592653589793f; /* MATH_PI is a float literal (MathUtils.h:95) */
    switch (m->model) {
    case PSO_XYIBG:
    case PSO_XYIBG_CONSTSIGMA: {
        REAL sx, sy;
        if (m->model == PSO_XYIBG) { sx = m->sigma[0]; sy = m->sigma[1]; }
        else { sx = consts[0]; sy = consts[1]; }
        const REAL OneOverSqrt2PiSigmaX = (REAL)1 / (SQRT(2 * PI_) * sx);
        const REAL OneOverSqrt2SigmaX = (REAL)1 / (SQRT((REAL)2) * sx);
        const REAL OneOverSqrt2PiSigmaY = (REAL)1 / (SQRT(2 * PI_) * sy);
        const REAL OneOverSqrt2SigmaY = (REAL)1 / (SQRT((REAL)2) * sy);
        REAL tx = theta[0], ty = theta[1], tI = theta[2], tbg = theta[3];
        for (int y = 0; y < H; y++) {
            REAL Yexp0 = ((REAL)y - ty + (REAL)0.5) * OneOverSqrt2SigmaY;
            REAL Yexp1 = ((REAL)y - ty - (REAL)0.5) * OneOverSqrt2SigmaY;
            REAL DeltaY = (REAL)0.5 * ERF(Yexp0) - (REAL)0.5 * ERF(Yexp1);
            REAL dEy = OneOverSqrt2PiSigmaY * (EXP(-Yexp1 * Yexp1) - EXP(-Yexp0 * Yexp0));
            for (int x = 0; x < W; x++) {
                REAL Xexp0 = ((REAL)x - tx + (REAL)0.5) * OneOverSqrt2SigmaX;
                REAL Xexp1 = ((REAL)x - tx - (REAL)0.5) * OneOverSqrt2SigmaX;
                REAL DeltaX = (REAL)0.5 * ERF(Xexp0) - (REAL)0.5 * ERF(Xexp1);
                REAL dEx = OneOverSqrt2PiSigmaX * (EXP(-Xexp1 * Xexp1) - EXP(-Xexp0 * Xexp0));
                int p = y * W + x;
                mu[p] = tbg + tI * DeltaX * DeltaY;
                jac[0 * npix + p] = tI * dEx * DeltaY;
                jac[1 * npix + p] = tI * dEy * DeltaX;
                jac[2 * npix + p] = DeltaX * DeltaY;
                jac[3 * npix + p] = 1;
            }
        }
        break;
    }
    case PSO_XYIBG_SIGMA:
    case PSO_XYIBG_SIGMAXY: {
        const int sxy = m->model == PSO_XYIBG_SIGMAXY;
        REAL tx = theta[0], ty = theta[1], tI = theta[2], tbg = theta[3];
        REAL tsx = theta[4], tsy = sxy ? theta[5] : theta[4];
        const REAL invSqrtPi = (REAL)1 / SQRT(PI_);
        const REAL OneOverSqrt2PiSigmaX = (REAL)1 / (SQRT(2 * PI_) * tsx);
        const REAL OneOverSqrt2PiSigmaY = (REAL)1 / (SQRT(2 * PI_) * tsy);
        const REAL OneOverSqrt2SigmaX = (REAL)1 / (SQRT((REAL)2) * tsx);
        const REAL OneOverSqrt2SigmaY = (REAL)1 / (SQRT((REAL)2) * tsy);
        for (int y = 0; y < H; y++) {
            REAL Yexp0 = ((REAL)y - ty + (REAL)0.5) * OneOverSqrt2SigmaY;
            REAL Yexp1 = ((REAL)y - ty - (REAL)0.5) * OneOverSqrt2SigmaY;
            REAL DeltaY = (REAL)0.5 * ERF(Yexp0) - (REAL)0.5 * ERF(Yexp1);
            REAL expY1 = EXP(-Yexp1 * Yexp1), expY0 = EXP(-Yexp0 * Yexp0);
            REAL dEy = OneOverSqrt2PiSigmaY * (expY1 - expY0);
            REAL dDeltaY_dsigma = (expY1 * Yexp1 - expY0 * Yexp0) * invSqrtPi;
            for (int x = 0; x < W; x++) {
                REAL Xexp0 = ((REAL)x - tx + (REAL)0.5) * OneOverSqrt2SigmaX;
                REAL Xexp1 = ((REAL)x - tx - (REAL)0.5) * OneOverSqrt2SigmaX;
                REAL DeltaX = (REAL)0.5 * ERF(Xexp0) - (REAL)0.5 * ERF(Xexp1);
                REAL expX1 = EXP(-Xexp1 * Xexp1), expX0 = EXP(-Xexp0 * Xexp0);
                REAL dEx = OneOverSqrt2PiSigmaX * (expX1 - expX0);
                REAL dDeltaX_dsigma = (expX1 * Xexp1 - expX0 * Xexp0) * invSqrtPi;
                int p = y * W + x;
                mu[p] = tbg + tI * DeltaX * DeltaY;
                jac[0 * npix + p] = tI * dEx * DeltaY;
                jac[1 * npix + p] = tI * dEy * DeltaX;
                jac[2 * npix + p] = DeltaX * DeltaY;
                jac[3 * npix + p] = 1;
                if (sxy) {
                    jac[4 * npix + p] = tI * dDeltaX_dsigma * DeltaY;
                    jac[5 * npix + p] = tI * dDeltaY_dsigma * DeltaX;
                } else {
                    jac[4 * npix + p] = tI * (dDeltaX_dsigma * DeltaY + dDeltaY_dsigma * DeltaX);
                }
            }
        }
        break;
    }
    case PSO_XYZIBG: {
        REAL tx = theta[0], ty = theta[1], tz = theta[2], tI = theta[3], tbg = theta[4];
        REAL s0_x = m->astig_x[0], gamma_x = m->astig_x[1], d_x = m->astig_x[2], A_x = m->astig_x[3], B_x = m->astig_x[4];
        REAL s0_y = m->astig_y[0], gamma_y = m->astig_y[1], d_y = m->astig_y[2], A_y = m->astig_y[3], B_y = m->astig_y[4];
        REAL d_y2 = d_y * d_y, d_x2 = d_x * d_x;
        REAL d_y4 = d_y2 * d_y2, d_x4 = d_x2 * d_x2;
        const REAL tzx = tz - gamma_x, tzx2 = tzx * tzx, tzx3 = tzx2 * tzx, tzx4 = tzx2 * tzx2;
        const REAL tzy = tz - gamma_y, tzy2 = tzy * tzy, tzy3 = tzy2 * tzy, tzy4 = tzy2 * tzy2;
        /* The reference's 4-coefficient form; the B term adds exactly +0 when B == 0. */
        const REAL qx = (REAL)1 + tzx2 / d_x2 + A_x * tzx3 / d_x2 + B_x * tzx4 / d_x4;
        const REAL qy = (REAL)1 + tzy2 / d_y2 + A_y * tzy3 / d_y2 + B_y * tzy4 / d_y4;
        const REAL sigma_x = s0_x * SQRT(qx);
        const REAL sigma_y = s0_y * SQRT(qy);
        const REAL OneOverSqrt2PiSigma_x = (REAL)1 / (SQRT(2 * PI_) * sigma_x);
        const REAL OneOverSqrt2Sigma_x = (REAL)1 / (SQRT((REAL)2) * sigma_x);
        const REAL OneOverSqrt2PiSigma_y = (REAL)1 / (SQRT(2 * PI_) * sigma_y);
        const REAL OneOverSqrt2Sigma_y = (REAL)1 / (SQRT((REAL)2) * sigma_y);
        const REAL dSigmaXThetaZ = s0_x * (2 * tzx / d_x2 + A_x * 3 * tzx2 / d_x2 + B_x * 4 * tzx3 / d_x4) /
                                   (2 * SQRT(qx));
        const REAL dSigmaYThetaZ = s0_y * (2 * tzy / d_y2 + A_y * 3 * tzy2 / d_y2 + B_y * 4 * tzy3 / d_y4) /
                                   (2 * SQRT(qy));
        for (int y = 0; y < H; y++) {
            REAL Yexp0 = ((REAL)y - ty + (REAL)0.5) * OneOverSqrt2Sigma_y;
            REAL Yexp1 = ((REAL)y - ty - (REAL)0.5) * OneOverSqrt2Sigma_y;
            REAL DeltaY = (REAL)0.5 * ERF(Yexp0) - (REAL)0.5 * ERF(Yexp1);
            REAL dEy = OneOverSqrt2PiSigma_y * (EXP(-Yexp1 * Yexp1) - EXP(-Yexp0 * Yexp0));
            REAL ym = (REAL)y - ty - (REAL)0.5, yp = (REAL)y - ty + (REAL)0.5;
            REAL G21y = (REAL)1 / (SQRT((REAL)2 * PI_) * sigma_y * sigma_y) *
                        (ym * EXP(-ym * ym / ((REAL)2 * sigma_y * sigma_y)) -
                         yp * EXP(-yp * yp / ((REAL)2 * sigma_y * sigma_y)));
            for (int x = 0; x < W; x++) {
                REAL Xexp0 = ((REAL)x - tx + (REAL)0.5) * OneOverSqrt2Sigma_x;
                REAL Xexp1 = ((REAL)x - tx - (REAL)0.5) * OneOverSqrt2Sigma_x;
                REAL DeltaX = (REAL)0.5 * ERF(Xexp0) - (REAL)0.5 * ERF(Xexp1);
                REAL dEx = OneOverSqrt2PiSigma_x * (EXP(-Xexp1 * Xexp1) - EXP(-Xexp0 * Xexp0));
                REAL xm = (REAL)x - tx - (REAL)0.5, xp = (REAL)x - tx + (REAL)0.5;
                REAL G21x = (REAL)1 / (SQRT((REAL)2 * PI_) * sigma_x * sigma_x) *
                            (xm * EXP(-xm * xm / ((REAL)2 * sigma_x * sigma_x)) -
                             xp * EXP(-xp * xp / ((REAL)2 * sigma_x * sigma_x)));
                int p = y * W + x;
                mu[p] = tbg + tI * DeltaX * DeltaY;
                jac[0 * npix + p] = tI * dEx * DeltaY;
                jac[1 * npix + p] = tI * dEy * DeltaX;
                REAL dMuSigmaX = tI * DeltaY * G21x;
                REAL dMuSigmaY = tI * DeltaX * G21y;
                jac[2 * npix + p] = dMuSigmaX * dSigmaXThetaZ + dMuSigmaY * dSigmaYThetaZ;
                jac[3 * npix + p] = DeltaX * DeltaY;
                jac[4 * npix + p] = 1;
            }
        }
        break;
    }
    case PSO_XYITILTEDBG:
    case PSO_XYITILTEDBG_SIGMAXY: {
        /* mu = bg + bgx (x - W/2) + bgy (y - H/2) + I DeltaX DeltaY for XYITiltedBg (sigma from the
         * spot's constants). XYITiltedBgSigmaXY has the tilt in its Jacobian but, as in the
         * reference (GaussianPSFModels.h:542 vs 549), not in mu. */
        const int free = m->model == PSO_XYITILTEDBG_SIGMAXY;
        REAL tx = theta[0], ty = theta[1], tI = theta[2], tbg = theta[3], bgx = theta[4], bgy = theta[5];
        REAL tsx = free ? theta[6] : (REAL)consts[0];
        REAL tsy = free ? theta[7] : (REAL)consts[1];
        const REAL halfw = (REAL)((float)W * 0.5f), halfh = (REAL)((float)H * 0.5f);
        const REAL invSqrtPi = (REAL)1 / SQRT(PI_);
        const REAL OneOverSqrt2PiSigmaX = (REAL)1 / (SQRT(2 * PI_) * tsx);
        const REAL OneOverSqrt2SigmaX = (REAL)1 / (SQRT((REAL)2) * tsx);
        const REAL OneOverSqrt2PiSigmaY = (REAL)1 / (SQRT(2 * PI_) * tsy);
        const REAL OneOverSqrt2SigmaY = (REAL)1 / (SQRT((REAL)2) * tsy);
        for (int y = 0; y < H; y++) {
            REAL Yexp0 = ((REAL)y - ty + (REAL)0.5) * OneOverSqrt2SigmaY;
            REAL Yexp1 = ((REAL)y - ty - (REAL)0.5) * OneOverSqrt2SigmaY;
            REAL DeltaY = (REAL)0.5 * ERF(Yexp0) - (REAL)0.5 * ERF(Yexp1);
            REAL expY1 = EXP(-Yexp1 * Yexp1), expY0 = EXP(-Yexp0 * Yexp0);
            REAL dEy = OneOverSqrt2PiSigmaY * (expY1 - expY0);
            REAL dDeltaY_dsigma = (expY1 * Yexp1 - expY0 * Yexp0) * invSqrtPi;
            for (int x = 0; x < W; x++) {
                REAL Xexp0 = ((REAL)x - tx + (REAL)0.5) * OneOverSqrt2SigmaX;
                REAL Xexp1 = ((REAL)x - tx - (REAL)0.5) * OneOverSqrt2SigmaX;
                REAL DeltaX = (REAL)0.5 * ERF(Xexp0) - (REAL)0.5 * ERF(Xexp1);
                REAL expX1 = EXP(-Xexp1 * Xexp1), expX0 = EXP(-Xexp0 * Xexp0);
                REAL dEx = OneOverSqrt2PiSigmaX * (expX1 - expX0);
                REAL dDeltaX_dsigma = (expX1 * Xexp1 - expX0 * Xexp0) * invSqrtPi;
                int p = y * W + x;
                if (free) mu[p] = tbg + tI * DeltaX * DeltaY;
                else mu[p] = tbg + bgx * ((REAL)x - halfw) + bgy * ((REAL)y - halfh) + tI * DeltaX * DeltaY;
                jac[0 * npix + p] = tI * dEx * DeltaY;
                jac[1 * npix + p] = tI * dEy * DeltaX;
                jac[2 * npix + p] = DeltaX * DeltaY;
                jac[3 * npix + p] = 1;
                jac[4 * npix + p] = (REAL)x - halfw;
                jac[5 * npix + p] = (REAL)y - halfh;
                if (free) {
                    jac[6 * npix + p] = tI * dDeltaX_dsigma * DeltaY;
                    jac[7 * npix + p] = tI * dDeltaY_dsigma * DeltaX;
                }
            }
        }
        break;
    }
    case PSO_INTENSITYBG: {
        /* psf = DeltaX DeltaY at the fixed position (constants x, y) and sigma (constant 2),
         * precomputed once per spot in the reference (ComputeGaussianPSF); mu = I psf + bg */
        const REAL cx = (REAL)1 / (SQRT((REAL)2) * (REAL)consts[2]);
        const REAL tx = (REAL)consts[0], ty = (REAL)consts[1];
        for (int y = 0; y < H; y++) {
            REAL Yexp0 = ((REAL)y - ty + (REAL)0.5) * cx;
            REAL Yexp1 = ((REAL)y - ty - (REAL)0.5) * cx;
            REAL DeltaY = (REAL)0.5 * ERF(Yexp0) - (REAL)0.5 * ERF(Yexp1);
            for (int x = 0; x < W; x++) {
                REAL Xexp0 = ((REAL)x - tx + (REAL)0.5) * cx;
                REAL Xexp1 = ((REAL)x - tx - (REAL)0.5) * cx;
                REAL DeltaX = (REAL)0.5 * ERF(Xexp0) - (REAL)0.5 * ERF(Xexp1);
                const REAL psf = DeltaX * DeltaY;
                int p = y * W + x;
                mu[p] = theta[0] * psf + theta[1];
                jac[0 * npix + p] = psf;
                jac[1 * npix + p] = 1;
            }
        }
        break;
    }
    case PSO_CSPLINE:
    case PSO_CSPLINE_TILTED:
    case PSO_CSPLINE_BGIMAGE: {
        /* flat background (CubicSplinePSFModels.h:14-154), tilted background (:157-298:
         * mu += bgx (x - W/2) + bgy (y - W/2)) and background image (:300-443: mu = I psf + bg *
         * image, the image being the spot's constants, with its own centring of tx, ty) */
        const int Nz = m->spline_shape[0], Ny = m->spline_shape[1], Nx = m->spline_shape[2];
        const float du_f = (m->spline_zmax - m->spline_zmin) / (float)Nz;
        const REAL du = (REAL)du_f;
        REAL tx = theta[0], ty = theta[1], tz = theta[2], tI = theta[3], tbg = theta[4];
        /* voxels per ROI pixel: 1 reproduces the reference; the oversampled extension scales the
         * grid coordinate of pixel x to q x - tx and the x/y derivatives by q */
        const REAL q = m->spline_q > 0 ? (REAL)m->spline_q : (REAL)1;
        if (m->model == PSO_CSPLINE_BGIMAGE) {
            const float wf = (float)W;
            tx = tx - (REAL)(wf / 2.0f) + (REAL)((wf - (float)Nx + 1) / 2.0f);
            ty = ty - (REAL)(wf / 2.0f) + (REAL)((wf - (float)Ny + 1) / 2.0f);
            tx += (REAL)0.5f;
            ty += (REAL)0.5f;
        } else {
            tx = tx * q - (REAL)(Nx * 0.5f);
            ty = ty * q - (REAL)(Ny * 0.5f);
        }
        const REAL halfw = (REAL)((float)W * 0.5f);
        REAL df[64], dxf[64], dyf[64], dzf[64];
        for (int i = 0; i < 64; i++) df[i] = dxf[i] = dyf[i] = dzf[i] = 0;
        REAL spx = -tx; spx -= q == 1 ? (REAL)(int)spx : FN(o_floor)(spx);
        REAL spy = -ty; spy -= q == 1 ? (REAL)(int)spy : FN(o_floor)(spy);
        REAL spz = (tz - (REAL)m->spline_zmin) / du;
        int k = (int)spz; if (k < 0) k = 0; if (k > Nz - 1) k = Nz - 1;
        spz = FN(o_clamp)(spz - (REAL)k, 0, 1);
        REAL zzz = 1;
        for (int mm = 0; mm <= 3; mm++) {
            REAL yyy = 1;
            for (int n = 0; n <= 3; n++) {
                REAL xxx = 1;
                for (int o = 0; o <= 3; o++) {
                    const REAL xyz = xxx * yyy * zzz;
                    df[mm * 16 + n * 4 + o] = xyz;
                    if (o < 3) dxf[mm * 16 + n * 4 + o + 1] = ((REAL)o + 1) * xyz;
                    if (n < 3) dyf[mm * 16 + (n + 1) * 4 + o] = ((REAL)n + 1) * xyz;
                    if (mm < 3) dzf[(mm + 1) * 16 + n * 4 + o] = ((REAL)mm + 1) * xyz;
                    xxx *= spx;
                }
                yyy *= spy;
            }
            zzz *= spz;
        }
        for (int y = 0; y < H; y++) {
            REAL yy = (REAL)y * q - ty;
            int j = (int)yy; if (j < 0) j = 0; if (j > Ny - 1) j = Ny - 1;
            for (int x = 0; x < W; x++) {
                REAL xx = (REAL)x * q - tx;
                int i = (int)xx; if (i < 0) i = 0; if (i > Nx - 1) i = Nx - 1;
                REAL psf = 0, dx = 0, dy = 0, dz = 0;
                const float* c = m->coefs + 64 * ((size_t)k * Nx * Ny + (size_t)j * Nx + i);
                for (int idx = 0; idx < 64; idx++) {
                    REAL coef = (REAL)c[idx];
                    psf += df[idx] * coef;
                    dx += dxf[idx] * coef;
                    dy += dyf[idx] * coef;
                    dz += dzf[idx] * coef;
                }
                dx *= -(tI * q);
                dy *= -(tI * q);
                dz *= tI / du;
                if (psf < 0) psf = 0;
                int p = y * W + x;
                if (m->model == PSO_CSPLINE_TILTED) {
                    mu[p] = tI * psf + tbg + theta[5] * ((REAL)x - halfw) + theta[6] * ((REAL)y - halfw);
                    jac[5 * npix + p] = (REAL)x - halfw;
                    jac[6 * npix + p] = (REAL)y - halfw;
                } else if (m->model == PSO_CSPLINE_BGIMAGE) {
                    mu[p] = tI * psf + tbg * (REAL)consts[p];
                } else {
                    mu[p] = tI * psf + tbg;
                }
                jac[0 * npix + p] = dx;
                jac[1 * npix + p] = dy;
                jac[2 * npix + p] = dz;
                jac[3 * npix + p] = psf;
                jac[4 * npix + p] = m->model == PSO_CSPLINE_BGIMAGE ? (REAL)consts[p] : 1;
            }
        }
        break;
    }
    }
}

static void FN(check_limits)(const pso_model_t* m, REAL* t)
{
    const int R = m->roisize;
    switch (m->model) {
    case PSO_XYIBG:
    case PSO_XYIBG_CONSTSIGMA:
        t[0] = FN(o_clamp)(t[0], (REAL)1.5f, (REAL)((float)R - 1.5f - 1));
        t[1] = FN(o_clamp)(t[1], (REAL)1.5f, (REAL)((float)R - 1.5f - 1));
        if (t[2] < 25) t[2] = 25;
        if (t[3] < 0) t[3] = 0;
        break;
    case PSO_XYIBG_SIGMA:
        t[0] = FN(o_clamp)(t[0], (REAL)1.5f, (REAL)((float)R - 1.5f - 1));
        t[1] = FN(o_clamp)(t[1], (REAL)1.5f, (REAL)((float)R - 1.5f - 1));
        if (t[2] < 10) t[2] = 10;
        if (t[3] < 0) t[3] = 0;
        if (t[4] < 1) t[4] = 1;
        if (t[4] > (REAL)(R * 0.5f)) t[4] = (REAL)(R * 0.5f);
        break;
    case PSO_XYIBG_SIGMAXY:
        t[0] = FN(o_clamp)(t[0], (REAL)1.5f, (REAL)((float)R - 1.5f - 1));
        t[1] = FN(o_clamp)(t[1], (REAL)1.5f, (REAL)((float)R - 1.5f - 1));
        if (t[2] < 10) t[2] = 10;
        if (t[3] < 0) t[3] = 0;
        t[4] = FN(o_clamp)(t[4], 1, (REAL)(R * 0.5f));
        t[5] = FN(o_clamp)(t[5], 1, (REAL)(R * 0.5f));
        break;
    case PSO_XYZIBG:
        t[0] = FN(o_clamp)(t[0], (REAL)1.5f, (REAL)((float)R - 1.5f - 1));
        t[1] = FN(o_clamp)(t[1], (REAL)1.5f, (REAL)((float)R - 1.5f - 1));
        t[2] = FN(o_clamp)(t[2], (REAL)m->minz, (REAL)m->maxz);
        t[3] = FMAX(t[3], 10);
        t[4] = FMAX(t[4], 0);
        break;
    case PSO_XYITILTEDBG:
        t[0] = FN(o_clamp)(t[0], (REAL)1.5f, (REAL)((float)R - 1.5f - 1));
        t[1] = FN(o_clamp)(t[1], (REAL)1.5f, (REAL)((float)R - 1.5f - 1));
        if (t[2] < 25) t[2] = 25;
        if (t[3] < 0) t[3] = 0;
        break;
    case PSO_XYITILTEDBG_SIGMAXY:
        t[0] = FN(o_clamp)(t[0], (REAL)1.5f, (REAL)((float)R - 1.5f - 1));
        t[1] = FN(o_clamp)(t[1], (REAL)1.5f, (REAL)((float)R - 1.5f - 1));
        if (t[2] < 10) t[2] = 10;
        if (t[3] < 0) t[3] = 0;
        t[6] = FN(o_clamp)(t[6], 1, (REAL)(R * 0.5f));
        t[7] = FN(o_clamp)(t[7], 1, (REAL)(R * 0.5f));
        break;
    case PSO_INTENSITYBG:
        if (t[0] < (REAL)1e-5f) t[0] = (REAL)1e-5f;
        if (t[1] < (REAL)1e-8f) t[1] = (REAL)1e-8f;
        break;
    case PSO_CSPLINE:
    case PSO_CSPLINE_TILTED:
    case PSO_CSPLINE_BGIMAGE:
        t[0] = FN(o_clamp)(t[0], (REAL)1.5f, (REAL)((float)R - 1.0f - 1.5f));
        t[1] = FN(o_clamp)(t[1], (REAL)1.5f, (REAL)((float)R - 1.0f - 1.5f));
        t[2] = FN(o_clamp)(t[2], (REAL)(m->spline_zmin + 1e-3f), (REAL)(m->spline_zmax - 1e-3f));
        t[3] = FMAX(t[3], 10);
        t[4] = FMAX(t[4], 0);
        break;
    }
}

static void FN(initial_estimate)(const pso_model_t* m, const float* smp, REAL* t)
{
    const int R = m->roisize;
    REAL sumX = 0, sumY = 0, sum = 0;
    for (int y = 0; y < R; y++)
        for (int x = 0; x < R; x++) {
            REAL v = (REAL)smp[y * R + x];
            sumX += (REAL)x * v;
            sumY += (REAL)y * v;
            sum += v;
        }
    REAL comx = sumX / sum, comy = sumY / sum;
    switch (m->model) {
    case PSO_XYIBG:
    case PSO_XYIBG_CONSTSIGMA:
        t[0] = comx; t[1] = comy; t[2] = sum * (REAL)0.7f; t[3] = 0; break;
    case PSO_XYIBG_SIGMA:
        t[0] = comx; t[1] = comy; t[2] = sum; t[3] = 0; t[4] = m->sigma[0]; break;
    case PSO_XYIBG_SIGMAXY:
        t[0] = comx; t[1] = comy; t[2] = sum; t[3] = 0; t[4] = m->sigma[0]; t[5] = m->sigma[1]; break;
    case PSO_XYZIBG:
        t[0] = comx; t[1] = comy; t[2] = 0; t[3] = sum; t[4] = (REAL)0.01f; break;
    case PSO_CSPLINE:
    case PSO_CSPLINE_BGIMAGE:
        t[0] = comx; t[1] = comy; t[2] = 0; t[3] = sum; t[4] = 0; break;
    case PSO_CSPLINE_TILTED:
        t[0] = comx; t[1] = comy; t[2] = 0; t[3] = sum; t[4] = 0; t[5] = 0; t[6] = 0; break;
    case PSO_XYITILTEDBG:
        t[0] = comx; t[1] = comy; t[2] = sum * (REAL)0.7f; t[3] = 0; t[4] = 0; t[5] = 0; break;
    case PSO_INTENSITYBG:
        t[0] = 1; t[1] = 0; break;  /* GaussianPSF.cu:226 starts every spot at (1, 0) */
    case PSO_XYITILTEDBG_SIGMAXY:
        t[0] = comx; t[1] = comy; t[2] = sum; t[3] = 0; t[4] = 0; t[5] = 0;
        t[6] = m->sigma[0]; t[7] = m->sigma[1]; break;
    }
}

static const float* FN(stop_limits)(int model)
{
    static const float g4[] = {1e-5f, 1e-5f, 1e-1f, 1e-5f};
    static const float g5[] = {1e-5f, 1e-5f, 1e-1f, 1e-4f, 1e-5f};
    static const float g6[] = {1e-5f, 1e-5f, 1e-1f, 1e-4f, 1e-5f, 1e-5f};
    static const float a5[] = {1e-4f, 1e-4f, 1e-1f, 1e-4f, 1e-4f};
    static const float s5[] = {1e-4f, 1e-4f, 1e-7f, 1e-4f, 1e-4f};
    static const float t6[] = {1e-5f, 1e-5f, 1e-1f, 1e-5f, 1e-5f, 1e-5f};
    static const float t8[] = {1e-5f, 1e-5f, 1e-1f, 1e-4f, 1e-4f, 1e-4f, 1e-5f, 1e-5f};
    static const float ib[] = {1e-2f, 1e-4f};
    static const float s7[] = {1e-4f, 1e-4f, 1e-7f, 1e-4f, 1e-4f, 1e-4f, 1e-4f};
    switch (model) {
    case PSO_XYIBG: case PSO_XYIBG_CONSTSIGMA: return g4;
    case PSO_XYIBG_SIGMA: return g5;
    case PSO_XYIBG_SIGMAXY: return g6;
    case PSO_XYZIBG: return a5;
    case PSO_XYITILTEDBG: return t6;
    case PSO_XYITILTEDBG_SIGMAXY: return t8;
    case PSO_INTENSITYBG: return ib;
    case PSO_CSPLINE_TILTED: return s7;
    default: return s5;
    }
}

/* Lower Cholesky; fails only on an exactly-zero pivot (SolveMatrix.h:107-125). */
static int FN(cholesky)(int d, const REAL* S, REAL* D)
{
    for (int k = 0; k < d; ++k) {
        REAL sum = 0;
        for (int p = 0; p < k; ++p) sum += D[k * d + p] * D[k * d + p];
        REAL v = S[k * d + k] - sum;
        if (v == 0) return 0;
        D[k * d + k] = SQRT(v);
        for (int i = k + 1; i < d; ++i) {
            REAL s2 = 0;
            for (int p = 0; p < k; ++p) s2 += D[i * d + p] * D[k * d + p];
            REAL q = D[k * d + k];
            if (q == 0) return 0;
            D[i * d + k] = (S[i * d + k] - s2) / q;
        }
    }
    return 1;
}

static int FN(solve_cholesky)(int d, const REAL* LU, const REAL* b, REAL* x)
{
    REAL y[PSO_MAXK];
    for (int i = 0; i < d; ++i) {
        REAL sum = 0;
        for (int k = 0; k < i; ++k) sum += LU[i * d + k] * y[k];
        REAL v = LU[i * d + i];
        if (v == 0) return 0;
        y[i] = (b[i] - sum) / v;
    }
    for (int i = d - 1; i >= 0; --i) {
        REAL sum = 0;
        for (int k = i + 1; k < d; ++k) sum += LU[k * d + i] * x[k];
        x[i] = (y[i] - sum) / LU[i * d + i];
    }
    return 1;
}

/* InvertMatrix via LUPDecompose + LUPInvert, tol 1e-9 (SolveMatrix.h:411-452). */
static int FN(invert)(int N, const REAL* Ain, REAL* IA)
{
    REAL A[PSO_MAXK * PSO_MAXK];
    int P[PSO_MAXK + 1];
    for (int i = 0; i < N * N; i++) A[i] = Ain[i];
    for (int i = 0; i <= N; i++) P[i] = i;
    const REAL tol = (REAL)1e-9f;
    for (int i = 0; i < N; i++) {
        REAL maxA = 0, absA;
        int imax = i;
        for (int k = i; k < N; k++)
            if ((absA = FABS(A[k * N + i])) > maxA) { maxA = absA; imax = k; }
        if (maxA < tol) return 0;
        if (imax != i) {
            int j = P[i]; P[i] = P[imax]; P[imax] = j;
            for (int jj = 0; jj < N; jj++) {
                REAL tmp = A[i * N + jj]; A[i * N + jj] = A[imax * N + jj]; A[imax * N + jj] = tmp;
            }
            P[N]++;
        }
        for (int j = i + 1; j < N; j++) {
            A[j * N + i] /= A[i * N + i];
            for (int k = i + 1; k < N; k++) A[j * N + k] -= A[j * N + i] * A[i * N + k];
        }
    }
    for (int j = 0; j < N; j++) {
        for (int i = 0; i < N; i++) {
            IA[i * N + j] = (P[i] == j) ? 1 : 0;
            for (int k = 0; k < i; k++) IA[i * N + j] -= A[i * N + k] * IA[k * N + j];
        }
        for (int i = N - 1; i >= 0; i--) {
            for (int k = i + 1; k < N; k++) IA[i * N + j] -= A[i * N + k] * IA[k * N + j];
            IA[i * N + j] = IA[i * N + j] / A[i * N + i];
        }
    }
    return 1;
}

/* One spot of LevMarOptimize (Estimation.h:194-251). Returns the iteration count (i+1). */
static int FN(levmar_spot)(const pso_model_t* m, const float* smp, const float* consts, REAL* theta,
                           int maxIterations, REAL lambdaStep, REAL* trace, int traceBufLen,
                           REAL* mu, REAL* jac)
{
    const int K = pso_num_params(m->model), npix = m->roisize * m->roisize;
    const float* stop = FN(stop_limits)(m->model);
    int i;
    for (i = 0; i < maxIterations; i++) {
        if (i < traceBufLen)
            for (int k = 0; k < K; k++) trace[i * K + k] = theta[k];
        REAL alpha[PSO_MAXK * PSO_MAXK], beta[PSO_MAXK], step[PSO_MAXK], LU[PSO_MAXK * PSO_MAXK];
        for (int q = 0; q < K * K; q++) { alpha[q] = 0; LU[q] = 0; }
        for (int q = 0; q < K; q++) beta[q] = 0;
        FN(model_eval)(m, theta, consts, mu, jac);
        for (int p = 0; p < npix; p++) {
            REAL sampleValue = (REAL)smp[p];
            REAL mup = mu[p];
            if (sampleValue < (REAL)1e-6f) sampleValue = (REAL)1e-6f;
            REAL mu_c = mup > (REAL)1e-6f ? mup : (REAL)1e-6f;
            REAL invmu = (REAL)1 / mu_c;
            REAL x_f2 = sampleValue * invmu * invmu;
            for (int a = 0; a < K; a++)
                for (int b = a; b < K; b++)
                    alpha[K * a + b] += jac[a * npix + p] * jac[b * npix + p] * x_f2;
            REAL beta_factor = 1 - sampleValue * invmu;
            for (int a = 0; a < K; a++) beta[a] -= beta_factor * jac[a * npix + p];
        }
        for (int a = 1; a < K; a++)
            for (int b = 0; b < a; b++) alpha[K * a + b] = alpha[K * b + a];
        for (int k = 0; k < K; k++) {
            if (lambdaStep < 0) alpha[k * K + k] -= lambdaStep;
            else {
                REAL s = 0;
                for (int j = 0; j < K; j++) s += alpha[j * K + k] * alpha[j * K + k];
                alpha[k * K + k] += s * lambdaStep;
            }
        }
        if (!FN(cholesky)(K, alpha, LU)) break;
        if (!FN(solve_cholesky)(K, LU, beta, step)) break;
        REAL last[PSO_MAXK];
        for (int k = 0; k < K; k++) { last[k] = theta[k]; theta[k] += step[k]; }
        FN(check_limits)(m, theta);
        int small = 1;
        for (int k = 0; k < K; k++)
            if (FABS(last[k] - theta[k]) > (REAL)stop[k]) { small = 0; break; }
        if (i > 0 && small) break;
    }
    return i + 1;
}

typedef struct {
    const pso_model_t* m;
    int n;
    const float* samples;
    const float* constants;
    const float* initial;
    float* params;
    int* iterations;
    float* trace;
    int traceBufLen;
    int maxIterations;
    double lambda;
    int next;               /* shared work counter */
    pthread_mutex_t* lock;
} FN(fit_job_t);

static void* FN(fit_worker)(void* arg)
{
    FN(fit_job_t)* job = (FN(fit_job_t)*)arg;
    const pso_model_t* m = job->m;
    const int K = pso_num_params(m->model), npix = m->roisize * m->roisize, nc = pso_model_constants(m);
    REAL* mu = (REAL*)malloc(sizeof(REAL) * npix);
    REAL* jac = (REAL*)malloc(sizeof(REAL) * npix * K);
    REAL* tr = job->traceBufLen > 0 ? (REAL*)malloc(sizeof(REAL) * K * job->traceBufLen) : NULL;
    for (;;) {
        pthread_mutex_lock(job->lock);
        int start = job->next;
        job->next += 64;
        pthread_mutex_unlock(job->lock);
        if (start >= job->n) break;
        int end = start + 64 < job->n ? start + 64 : job->n;
        for (int s = start; s < end; s++) {
            REAL theta[PSO_MAXK];
            const float* smp = job->samples + (size_t)s * npix;
            const float* cs = nc ? job->constants + (size_t)s * nc : NULL;
            if (job->initial) for (int k = 0; k < K; k++) theta[k] = (REAL)job->initial[(size_t)s * K + k];
            else FN(initial_estimate)(m, smp, theta);
            int it = FN(levmar_spot)(m, smp, cs, theta, job->maxIterations, (REAL)job->lambda, tr,
                                     job->traceBufLen, mu, jac);
            for (int k = 0; k < K; k++) job->params[(size_t)s * K + k] = (float)theta[k];
            if (job->iterations) job->iterations[s] = it;
            if (job->trace) {
                int nt = it < job->traceBufLen ? it : job->traceBufLen;
                for (int q = 0; q < nt * K; q++) job->trace[(size_t)s * job->traceBufLen * K + q] = (float)tr[q];
            }
        }
    }
    free(mu); free(jac); free(tr);
    return NULL;
}

int FN(pso_fit)(const pso_model_t* m, int n, const float* samples, const float* constants,
                const float* initial, int maxIterations, double lambda, float* params, int* iterations,
                float* trace, int traceBufLen, int nthreads)
{
    if (n <= 0) return 0;
    pthread_mutex_t lock = PTHREAD_MUTEX_INITIALIZER;
    FN(fit_job_t) job = {m, n, samples, constants, initial, params, iterations, trace, traceBufLen,
                         maxIterations, lambda, 0, &lock};
    if (nthreads < 1) nthreads = 1;
    pthread_t th[256];
    if (nthreads > 256) nthreads = 256;
    for (int t = 0; t < nthreads; t++) pthread_create(&th[t], NULL, FN(fit_worker), &job);
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    return 0;
}

/* ExpectedValue / Derivatives (Estimation.h:159-181): ev[n][npix], deriv[n][K][npix]. */
int FN(pso_derivatives)(const pso_model_t* m, int n, const float* params, const float* constants,
                        float* deriv, float* ev)
{
    const int K = pso_num_params(m->model), npix = m->roisize * m->roisize, nc = pso_model_constants(m);
    REAL* mu = (REAL*)malloc(sizeof(REAL) * npix);
    REAL* jac = (REAL*)malloc(sizeof(REAL) * npix * K);
    for (int s = 0; s < n; s++) {
        REAL theta[PSO_MAXK];
        for (int k = 0; k < K; k++) theta[k] = (REAL)params[(size_t)s * K + k];
        FN(model_eval)(m, theta, nc ? constants + (size_t)s * nc : NULL, mu, jac);
        for (int p = 0; p < npix; p++) {
            if (ev) ev[(size_t)s * npix + p] = (float)mu[p];
            if (deriv)
                for (int k = 0; k < K; k++) deriv[((size_t)s * K + k) * npix + p] = (float)jac[k * npix + p];
        }
    }
    free(mu); free(jac);
    return 0;
}

/* ComputeChiSquareAndCRLB (Estimation.h:63-102): Fisher with mu >= 1e-8, chisq when a sample
 * is given, LUP inverse (Inf on failure), sqrt of the diagonal. fisher_out is optional [n][K][K]. */
int FN(pso_crlb)(const pso_model_t* m, int n, const float* params, const float* samples,
                 const float* constants, float* crlb, float* chisq, double* fisher_out)
{
    const int K = pso_num_params(m->model), npix = m->roisize * m->roisize, nc = pso_model_constants(m);
    REAL* mu = (REAL*)malloc(sizeof(REAL) * npix);
    REAL* jac = (REAL*)malloc(sizeof(REAL) * npix * K);
    for (int s = 0; s < n; s++) {
        REAL theta[PSO_MAXK], fi[PSO_MAXK * PSO_MAXK], inv[PSO_MAXK * PSO_MAXK];
        for (int k = 0; k < K; k++) theta[k] = (REAL)params[(size_t)s * K + k];
        FN(model_eval)(m, theta, nc ? constants + (size_t)s * nc : NULL, mu, jac);
        for (int q = 0; q < K * K; q++) fi[q] = 0;
        REAL cs = 0;
        for (int p = 0; p < npix; p++) {
            REAL mup = FMAX((REAL)1e-8f, mu[p]);
            if (samples) {
                REAL e = (REAL)samples[(size_t)s * npix + p] - mup;
                cs += e * e / mup;
            }
            REAL inv_mu_c = (REAL)1 / mup;
            for (int a = 0; a < K; a++)
                for (int b = a; b < K; b++) fi[K * a + b] += jac[a * npix + p] * jac[b * npix + p] * inv_mu_c;
        }
        for (int a = 1; a < K; a++)
            for (int b = 0; b < a; b++) fi[K * a + b] = fi[K * b + a];
        if (fisher_out)
            for (int q = 0; q < K * K; q++) fisher_out[(size_t)s * K * K + q] = (double)fi[q];
        int ok = FN(invert)(K, fi, inv);
        for (int k = 0; k < K; k++)
            /* ComputeCRLB (Estimation.h:318-333), used by the intensity/background fit, takes
             * fabs of the diagonal; ComputeChiSquareAndCRLB does not */
            crlb[(size_t)s * K + k] = ok ? (float)SQRT(m->model == PSO_INTENSITYBG ? FABS(inv[k * (K + 1)])
                                                                                  : inv[k * (K + 1)])
                                         : INFINITY;
        if (chisq) chisq[s] = (float)cs;
    }
    free(mu); free(jac);
    return 0;
}

#undef FN
#undef CAT
#undef CAT_
