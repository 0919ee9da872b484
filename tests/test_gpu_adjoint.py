"""Adjoint kernel of the summed Poisson NLL (PB200_PoissonNLLAdjoint / photonpy_b200.autograd).

Gradients with respect to per-spot parameters and the PSF calibration are checked against
central finite differences of an FP64 NLL (relative error <= 1e-3) and, for x/y/I/bg, against
the reference's own Derivatives output (golden vectors): dNLL/dtheta = sum_p (1 - x/mu) dmu/dtheta.
Points are displaced from the optimum so that the gradients are not dominated by rounding.
"""
import math

import numpy as np
import pytest

from conftest import load_golden
from photonpy_b200 import synth

pytestmark = pytest.mark.gpu


def _nll64(ev, smp):
    mu = np.maximum(ev, 1e-6)
    return np.sum(mu - smp * np.log(mu), axis=(-1, -2))


def _gauss_ev64(R, th, sx, sy):
    n = len(th)
    return synth.gauss2d_ev(R, th[:, 0], th[:, 1], th[:, 2], th[:, 3], np.full(n, sx), np.full(n, sy))


def _astig_ev64(R, th, cx, cy):
    sx = synth.astig_sigma(th[:, 2], *cx)
    sy = synth.astig_sigma(th[:, 2], *cy)
    return synth.gauss2d_ev(R, th[:, 0], th[:, 1], th[:, 3], th[:, 4], sx, sy)


def _spline_ev64(coefs, zr, R, th):
    coefs = coefs.astype(np.float64)
    Nz, Ny, Nx = coefs.shape[:3]
    du = (zr[1] - zr[0]) / Nz
    out = np.zeros((len(th), R, R))
    for s, t in enumerate(th.astype(np.float64)):
        tx, ty = t[0] - Nx * 0.5, t[1] - Ny * 0.5
        spx = -tx - int(-tx)
        spy = -ty - int(-ty)
        sz = (t[2] - zr[0]) / du
        k = min(max(int(sz), 0), Nz - 1)
        spz = min(max(sz - k, 0.0), 1.0)
        df = np.array([spx ** o * spy ** n * spz ** m for m in range(4) for n in range(4) for o in range(4)])
        for y in range(R):
            j = min(max(int(y - ty), 0), Ny - 1)
            for x in range(R):
                i = min(max(int(x - tx), 0), Nx - 1)
                psf = max(coefs[k, j, i] @ df, 0.0)
                out[s, y, x] = t[3] * psf + t[4]
    return out


def _rel(a, b):
    return np.linalg.norm(a - b, axis=-1) / np.maximum(np.linalg.norm(b, axis=-1), 1e-12)


@pytest.fixture(scope="module")
def torch_mod():
    import torch
    return torch


def _grads(est, smp, th, torch_mod, calib=None):
    from photonpy_b200.autograd import poisson_nll
    torch = torch_mod
    x = torch.from_numpy(np.ascontiguousarray(smp, np.float32)).cuda()
    t = torch.tensor(th, dtype=torch.float32, device="cuda", requires_grad=True)
    c = None
    if calib is not None:
        c = torch.tensor(calib, dtype=torch.float32, device="cuda" if calib.ndim == 4 else "cpu", requires_grad=True)
    nll = poisson_nll(est, t, x, calib=c)
    nll.sum().backward()
    return nll.detach().cpu().numpy(), t.grad.cpu().numpy(), (None if c is None else c.grad.cpu().numpy())


def test_xyibg_theta_and_sigma_gradients(ctx, torch_mod):
    import photonpy_b200 as pb
    d = synth.xyibg(48, seed=21)
    th = d["truth"].astype(np.float64).copy()
    th[:, 0] += 0.3
    th[:, 1] -= 0.2
    th[:, 2] *= 1.2
    th[:, 3] *= 0.8
    sig = np.array([1.6, 1.4])
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(d["R"], tuple(sig), True)
    nll, gth, gcal = _grads(est, d["samples"], th, torch_mod, calib=sig.astype(np.float32))
    R = d["R"]
    nll64 = _nll64(_gauss_ev64(R, th, sig[0], sig[1]), d["samples"].astype(np.float64))
    assert np.allclose(nll, nll64, rtol=1e-5)
    fd = np.zeros_like(th)
    for k in range(4):
        h = 1e-4 * max(1.0, np.abs(th[:, k]).mean())
        tp, tm = th.copy(), th.copy()
        tp[:, k] += h
        tm[:, k] -= h
        fd[:, k] = (_nll64(_gauss_ev64(R, tp, sig[0], sig[1]), d["samples"]) -
                    _nll64(_gauss_ev64(R, tm, sig[0], sig[1]), d["samples"])) / (2 * h)
    assert np.max(_rel(gth, fd)) < 1e-3
    fdc = np.zeros(2)
    for k in range(2):
        sp, sm = sig.copy(), sig.copy()
        sp[k] += 1e-5
        sm[k] -= 1e-5
        fdc[k] = (np.sum(_nll64(_gauss_ev64(R, th, *sp), d["samples"])) -
                  np.sum(_nll64(_gauss_ev64(R, th, *sm), d["samples"]))) / 2e-5
    assert np.linalg.norm(gcal - fdc) / np.linalg.norm(fdc) < 1e-3
    est.Destroy()


def test_sigmaxy_theta_gradient_uses_true_sigma_derivative(ctx, torch_mod):
    import photonpy_b200 as pb
    d = synth.sigmaxy(32, seed=22)
    th = d["truth"].astype(np.float64).copy()
    th[:, 0] += 0.25
    th[:, 4] *= 1.15
    th[:, 5] *= 0.9
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBgSigmaXY(d["R"], 1.7, True)
    _, gth, _ = _grads(est, d["samples"], th, torch_mod)
    R = d["R"]

    def nll(t):
        return _nll64(synth.gauss2d_ev(R, t[:, 0], t[:, 1], t[:, 2], t[:, 3], t[:, 4], t[:, 5]), d["samples"])
    fd = np.zeros_like(th)
    for k in range(6):
        h = 1e-4 * max(1.0, np.abs(th[:, k]).mean())
        tp, tm = th.copy(), th.copy()
        tp[:, k] += h
        tm[:, k] -= h
        fd[:, k] = (nll(tp) - nll(tm)) / (2 * h)
    assert np.max(_rel(gth, fd)) < 1e-3
    est.Destroy()


def test_astig_calibration_gradient_with_quartic_term(ctx, torch_mod):
    import photonpy_b200 as pb
    d = synth.astig(40, seed=23, B=0.05)
    cx, cy = d["astig"]
    th = d["truth"].astype(np.float64).copy()
    th[:, 2] += 60.0
    th[:, 0] += 0.2
    calib = pb.Gauss3D_CalibrationB(cx, cy, d["zrange"])
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYZIBg(d["R"], calib, True)
    cal = np.array([cx, cy], np.float64)
    nll, gth, gcal = _grads(est, d["samples"], th, torch_mod, calib=cal.astype(np.float32))
    R = d["R"]
    nll64 = _nll64(_astig_ev64(R, th, cal[0], cal[1]), d["samples"])
    assert np.allclose(nll, nll64, rtol=1e-5)
    fd = np.zeros_like(th)
    for k in range(5):
        h = 1e-3 * max(1.0, np.abs(th[:, k]).mean())
        tp, tm = th.copy(), th.copy()
        tp[:, k] += h
        tm[:, k] -= h
        fd[:, k] = (_nll64(_astig_ev64(R, tp, cal[0], cal[1]), d["samples"]) -
                    _nll64(_astig_ev64(R, tm, cal[0], cal[1]), d["samples"])) / (2 * h)
    assert np.max(_rel(gth, fd)) < 1e-3
    fdc = np.zeros((2, 5))
    for a in range(2):
        for j in range(5):
            h = 1e-4 * max(abs(cal[a, j]), 1e-2)
            cp, cm = cal.copy(), cal.copy()
            cp[a, j] += h
            cm[a, j] -= h
            fdc[a, j] = (np.sum(_nll64(_astig_ev64(R, th, cp[0], cp[1]), d["samples"])) -
                         np.sum(_nll64(_astig_ev64(R, th, cm[0], cm[1]), d["samples"]))) / (2 * h)
    # compare each coefficient's gradient relative to the largest gradient of the same axis
    for a in range(2):
        scale = np.abs(fdc[a]).max()
        assert np.abs(gcal[a] - fdc[a]).max() / scale < 1e-3, (gcal, fdc)
    est.Destroy()


def test_spline_coefficient_gradient(ctx, torch_mod):
    import photonpy_b200 as pb
    g = load_golden("spline_r13")
    sm = pb.CSplineMethods(ctx)
    coefs = sm.ComputeSplineCoeff(g["zstack"], border=1)
    zr = tuple(float(v) for v in g["spline_zrange"])
    calib = pb.CSplineCalibration(zr[0], zr[1], coefs)
    est = sm.CreatePSF_XYZIBg(int(g["roisize"]), calib, sm.FlatBg, True)
    th = g["truth"][:6].astype(np.float64).copy()
    th[:, 0] += 0.2
    th[:, 3] *= 1.1
    smp = g["samples"][:6]
    nll, gth, gcoef = _grads(est, smp, th, torch_mod, calib=coefs)
    R = int(g["roisize"])
    assert np.allclose(nll, _nll64(_spline_ev64(coefs, zr, R, th), smp), rtol=1e-5)
    # finite differences on the coefficients with the largest gradients
    flat = np.argsort(-np.abs(gcoef.reshape(-1)))[:8]
    for f in flat:
        h = 1e-4 * max(abs(coefs.reshape(-1)[f]), 1e-3)
        cp, cm = coefs.astype(np.float64).copy(), coefs.astype(np.float64).copy()
        cp.reshape(-1)[f] += h
        cm.reshape(-1)[f] -= h
        fd = (np.sum(_nll64(_spline_ev64(cp, zr, R, th), smp)) - np.sum(_nll64(_spline_ev64(cm, zr, R, th), smp))) / (2 * h)
        assert abs(gcoef.reshape(-1)[f] - fd) / abs(fd) < 1e-3
    est.Destroy()


def test_theta_gradient_matches_reference_derivatives(ctx, torch_mod):
    """dNLL/dtheta from the adjoint equals sum_p (1 - x/mu) J with J and mu from the reference's
    Derivatives (golden) for x, y, I, bg."""
    from helpers import cuda_estimator
    for name in ["xyibg_r10", "astig_r12"]:
        gld = load_golden(name)
        est = cuda_estimator(name, gld, ctx)
        n = len(gld["ev"])
        th = gld["truth"][:n].astype(np.float64)
        smp = gld["samples"][:n].astype(np.float64)
        _, gth, _ = _grads(est, gld["samples"][:n], th, torch_mod)
        mu = np.maximum(gld["ev"].astype(np.float64), 1e-6)
        r = 1 - smp / mu
        ref = np.einsum("nkyx,nyx->nk", gld["deriv"].astype(np.float64), r)
        assert np.max(_rel(gth, ref)) < 1e-3, name
        est.Destroy()
