"""Generalized likelihood-ratio test to detect spots vs background — counterpart of
photonpy/cpp/glrt.py over GLRT_CreatePSF.

``CreateEstimator(psf, ctx)`` returns an Estimator whose ``Estimate`` also fills
``diag[:, 0:3] = (ll_on, ll_off, mean)``: the Poisson log-likelihood of the fitted PSF model,
of a flat background-only model, and the ROI mean that model uses. ``ComputeLogPFA(diag)``
turns them into log false-positive probabilities. Each spot uses its own ROI mean; the
reference uses the first ROI of every call for all spots, which
``SetReferenceMean(est, True)`` reproduces.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from .context import Context
from .estimator import Estimator
from .lib import check_error


def CreateEstimator(psf, ctx: Context):
    """photonpy/cpp/glrt.py:12-23"""
    _GLRT_CreatePSF = ctx.smlm.lib.GLRT_CreatePSF
    _GLRT_CreatePSF.argtypes = [ct.c_void_p, ct.c_void_p]
    _GLRT_CreatePSF.restype = ct.c_void_p
    inst = _GLRT_CreatePSF(psf.inst, ctx.inst if ctx else None)
    est = Estimator(ctx, inst, getattr(psf, "calib", None))
    return est


def SetReferenceMean(est, on=True):
    """Select the reference's background mean (first ROI of each call) instead of each spot's own."""
    f = est.ctx.smlm.lib.PB200_SetGLRTReferenceMean
    f.argtypes = [ct.c_void_p, ct.c_int]
    f.restype = ct.c_int
    if f(est.inst, 1 if on else 0) != 0:
        check_error("SetGLRTReferenceMean")


def ComputeLogPFA(diag):
    """photonpy/cpp/glrt.py:25-36: Tg = 2 (ll_on - ll_off) clamped at 0, log P_fa = 2 log Phi(-sqrt(Tg))."""
    from scipy.stats import norm
    ll_on = diag[:, 0]
    ll_off = diag[:, 1]
    Tg = 2 * (ll_on - ll_off)
    Tg = np.maximum(0, Tg)
    return 2 * norm.logcdf(-np.sqrt(Tg))
