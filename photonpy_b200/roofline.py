"""Algorithmic work counts for the roofline figures.

One localization = LM fit (centre-of-mass start + Levenberg-Marquardt) + one Fisher/CRLB
pass, as photonpy's EstimationQueue runs them (EstimationQueue.cpp:285-289).

FLOPs (FMA = 2, add/mul = 1; erf/exp are counted as transcendental ops, not FLOPs):
  per pixel and executed LM iteration:
      3 (mu) + J_model + 5 (weights) + K + K(K+1) (Hessian upper triangle) + 2K (gradient)
      with J_model = 5 (XYIBg), 8 (Sigma), 9 (SigmaXY), 10 (astig), 4*2*64 = 512 (spline)
  per ROI and executed iteration: 2*(K^3/3 + 2K^2) for the damped Cholesky solve
  per pixel, once (Fisher pass): K(K+1) + 4 (chi-square)
The number of executed iterations of a spot is min(iterations, maxIterations), where
iterations is the reference's count (i+1 at the stop, maxIterations+1 when capped).

HBM algorithmic bytes per ROI: 4*H*W (+4*numconst) in, 4*(2K+1) + 4 out
(params, CRLB, chi-square, iteration count).
"""
from __future__ import annotations

import numpy as np

K_OF = {"XYIBg": 4, "XYIBgConstSigma": 4, "XYIBgSigma": 5, "XYIBgSigmaXY": 6, "XYZIBg": 5, "CSpline": 5}
JAC_FLOPS = {"XYIBg": 5, "XYIBgConstSigma": 5, "XYIBgSigma": 8, "XYIBgSigmaXY": 9, "XYZIBg": 10, "CSpline": 512}
TRANSC_PER_TERM = {"XYIBg": 4, "XYIBgConstSigma": 4, "XYIBgSigma": 4, "XYIBgSigmaXY": 4, "XYZIBg": 6, "CSpline": 0}


def flops_per_pixel_iteration(kind: str) -> int:
    K = K_OF[kind]
    return 3 + JAC_FLOPS[kind] + 5 + K + K * (K + 1) + 2 * K


def flops_per_solve(kind: str) -> float:
    K = K_OF[kind]
    return 2.0 * (K ** 3 / 3.0 + 2 * K * K)


def localization_flops(kind: str, R: int, iterations, max_iterations: int = 50) -> float:
    """Total algorithmic FLOPs of fitting + CRLB for spots with the given iteration counts."""
    it = np.minimum(np.asarray(iterations, dtype=np.int64), max_iterations).astype(np.float64)
    npix = R * R
    K = K_OF[kind]
    per_it = npix * flops_per_pixel_iteration(kind) + flops_per_solve(kind)
    fisher = npix * (K * (K + 1) + 4)
    return float(per_it * it.sum() + fisher * it.size)


def lm_flops(kind: str, R: int, iterations, max_iterations: int = 50) -> float:
    """The LM launch's share of localization_flops (everything but the Fisher pass)."""
    it = np.minimum(np.asarray(iterations, dtype=np.int64), max_iterations).astype(np.float64)
    return float((R * R * flops_per_pixel_iteration(kind) + flops_per_solve(kind)) * it.sum())


def transcendental_ops(kind: str, R: int, iterations, max_iterations: int = 50) -> float:
    """erf/exp evaluations (separable form: 2R 1D terms per iteration)."""
    it = np.minimum(np.asarray(iterations, dtype=np.int64), max_iterations).astype(np.float64)
    return float(2 * R * TRANSC_PER_TERM[kind] * (it.sum() + it.size))


def hbm_bytes_per_roi(kind: str, R: int, numconst: int = 0) -> int:
    K = K_OF[kind]
    return 4 * R * R + 4 * numconst + 4 * (2 * K + 1) + 4
