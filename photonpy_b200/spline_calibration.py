"""Gradient-descent re-calibration of a cubic-spline PSF (extension; photonpy has no gradient with
respect to its spline coefficients).

Given ROIs of emitters whose parameters are known (beads at known positions and z, or spots
localized with the current calibration), the coefficients c of the spline estimator's PSF are
refined by gradient descent on the summed Poisson negative log-likelihood of the ROIs,

    NLL(c) = sum_n sum_p mu_p(c) - x_p log(max(mu_p(c), 1e-6)),

with the hand-written adjoint kernel (PB200_SplineCoefGradient): one pass over the ROIs gives the
NLL and its gradient g with respect to every coefficient (and the diagonal D of the Fisher
information with respect to the coefficients). A step moves along -g, so only coefficient
combinations the data constrain change (g lies in the span of the model's coefficient
derivatives); the step length comes from a line search: mu is linear in c wherever the PSF is
not clamped at 0, so NLL(c - a g) is convex in a, and a parabola through NLL(c), its slope
-|g|^2 and one trial point (a = 1 / max D, a step the curvature along any single coefficient
allows) gives the minimiser. The step is accepted when it lowers the NLL by at least 1e-4 of the
predicted decrease, else halved.
"""
from __future__ import annotations

import ctypes as ct

import torch

from .lib import check_error, load_library


def _bind(L):
    vp = ct.c_void_p
    L.PB200_SplineCoefGradient.argtypes = [vp, ct.c_int, vp, vp, vp, vp, vp, vp, vp]
    L.PB200_SplineCoefGradient.restype = ct.c_int
    return L


def _p(t):
    return None if t is None else ct.c_void_p(t.data_ptr())


def spline_nll_grad(est, samples, params, coefs, want_grad=True):
    """(total NLL as a float, gradient [coefs.shape] or None, Fisher diagonal or None) of the ROIs
    `samples` [n, R, R] with spot parameters `params` [n, 5] under coefficients `coefs`; all CUDA
    float32 tensors."""
    L = _bind(load_library())
    n = samples.shape[0]
    nll = torch.empty(n, device=samples.device, dtype=torch.float32)
    grad = torch.zeros_like(coefs) if want_grad else None
    diag = torch.zeros_like(coefs) if want_grad else None
    s = torch.cuda.current_stream(samples.device).cuda_stream
    rc = L.PB200_SplineCoefGradient(est.inst, n, _p(samples), _p(params), _p(coefs), _p(nll), _p(grad), _p(diag),
                                    ct.c_void_p(s))
    if rc != 0:
        check_error("SplineCoefGradient")
    return float(nll.double().sum().item()), grad, diag


def recalibrate(est, samples, params, coefs0, steps=20, max_halvings=30, callback=None):
    """Refine the spline coefficients of `est` (a flat-background spline estimator) from `coefs0`
    by `steps` gradient-descent steps on the summed NLL of `samples` at the known spot
    parameters `params`. Returns dict(coefs, nll: the NLL before the first and after every step,
    step_sizes: the accepted step length of every step, 0 where no decrease was found).
    `callback(step, coefs, nll)` is called after every step."""
    samples = samples.contiguous()
    params = params.contiguous()
    c = coefs0.detach().clone().contiguous()
    f, g, d = spline_nll_grad(est, samples, params, c)
    history, alphas = [f], []
    for k in range(steps):
        gg = float((g.double() ** 2).sum().item())
        accepted, alpha = False, 0.0
        if gg > 0:
            a_trial = 1.0 / max(float(d.max().item()), 1e-30)
            f_trial, _, _ = spline_nll_grad(est, samples, params, (c - a_trial * g).contiguous(), want_grad=False)
            curv = 2.0 * (f_trial - f + a_trial * gg) / (a_trial * a_trial)  # NLL'' along -g
            alpha = gg / curv if curv > 0 else a_trial
            for _ in range(max_halvings):
                trial = (c - alpha * g).contiguous()
                f_new, _, _ = spline_nll_grad(est, samples, params, trial, want_grad=False)
                if f_new <= f - 1e-4 * alpha * gg:
                    accepted = True
                    break
                alpha *= 0.5
        if accepted:
            c = trial
            f, g, d = spline_nll_grad(est, samples, params, c)
        alphas.append(alpha if accepted else 0.0)
        history.append(f)
        if callback is not None:
            callback(k, c, f)
    return dict(coefs=c, nll=history, step_sizes=alphas)
