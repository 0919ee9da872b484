"""PyTorch autograd boundary of the hand-written adjoint kernel (PB200_PoissonNLLAdjoint).

``poisson_nll(est, theta, samples, calib=None)`` returns the per-spot Poisson negative
log-likelihood  NLL_n = sum_p mu_p - x_p log(max(mu_p, 1e-6))  of the estimator's PSF model and
is differentiable with respect to

* ``theta``  [n, K] per-spot parameters (true derivatives, including sigma of the free-sigma
  models), and
* ``calib``  the PSF calibration: XYIBg (sigma_x, sigma_y) [2]; astigmatic XYZIBg
  (s0, gamma, d, A, B) for x and y [2, 5]; cubic spline coefficients [Nz, Ny, Nx, 64].

Forward and backward are CUDA kernels that recompute mu and its derivatives per pixel (no
per-pixel derivative stack is stored). Everything stays on the device except the small
XYIBg/astig calibration vectors, which are read to the host to parameterise the kernel.
"""
from __future__ import annotations

import ctypes as ct

import torch

from .lib import check_error, load_library

_MODEL_XYIBG, _MODEL_XYZIBG, _MODEL_CSPLINE = 0, 4, 5


def _bind(L):
    vp = ct.c_void_p
    L.PB200_PoissonNLLAdjoint.argtypes = [vp, ct.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.PB200_PoissonNLLAdjoint.restype = ct.c_int
    return L


def _p(t):
    return None if t is None else ct.c_void_p(t.data_ptr())


def model_id(est) -> int:
    L = load_library()
    r = ct.c_int()
    return int(L.PB200_ModelInfo(est.inst, ct.byref(r)))


def _call(est, samples, theta, constants, calib, grad_out, nll, dtheta, dcalib):
    L = _bind(load_library())
    mid = model_id(est)
    host_calib = None
    coefs = None
    if calib is not None:
        if mid == _MODEL_CSPLINE:
            coefs = calib.detach().contiguous()
        elif mid in (_MODEL_XYIBG, _MODEL_XYZIBG):
            vals = calib.detach().reshape(-1).to("cpu", torch.float32)
            host_calib = (ct.c_float * vals.numel())(*vals.tolist())
    s = torch.cuda.current_stream(samples.device).cuda_stream
    rc = L.PB200_PoissonNLLAdjoint(est.inst, samples.shape[0], _p(samples), _p(theta), _p(constants), host_calib,
                                   _p(coefs), _p(grad_out), _p(nll), _p(dtheta), _p(dcalib), ct.c_void_p(s))
    if rc != 0:
        check_error("PoissonNLLAdjoint")


class PoissonNLL(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, calib, samples, est, constants):
        theta_c = theta.detach().contiguous().float()
        nll = torch.empty(samples.shape[0], device=samples.device, dtype=torch.float32)
        _call(est, samples, theta_c, constants, calib, None, nll, None, None)
        ctx.est = est
        ctx.save_for_backward(theta_c, calib if calib is not None else torch.empty(0), samples,
                              constants if constants is not None else torch.empty(0))
        ctx.has_calib = calib is not None
        ctx.has_consts = constants is not None
        return nll

    @staticmethod
    def backward(ctx, grad_nll):
        theta, calib, samples, constants = ctx.saved_tensors
        calib = calib if ctx.has_calib else None
        constants = constants if ctx.has_consts else None
        g = grad_nll.detach().contiguous().float()
        dtheta = torch.empty_like(theta) if ctx.needs_input_grad[0] else None
        dcalib = None
        if ctx.has_calib and ctx.needs_input_grad[1]:
            dcalib = torch.zeros(calib.numel(), device=samples.device, dtype=torch.float32)
        _call(ctx.est, samples, theta, constants, calib, g, None, dtheta, dcalib)
        if dcalib is not None:
            dcalib = dcalib.reshape(calib.shape).to(calib.device)
        return dtheta, dcalib, None, None, None


def poisson_nll(est, theta, samples, calib=None, constants=None):
    """Per-spot Poisson NLL of `samples` [n, R, R] (CUDA float32) under `est` at `theta` [n, K];
    differentiable with respect to theta and calib (see module docstring)."""
    assert samples.is_cuda and samples.dtype == torch.float32 and samples.is_contiguous()
    return PoissonNLL.apply(theta, calib, samples, est, constants)
