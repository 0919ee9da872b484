"""Cubic-spline PSF sampled at 0.5 px (the 26x26x41 calibration of the spline workload) and its
gradient-descent re-calibration.

photonpy's spline has one voxel per ROI pixel (CubicSplinePSFModels.h:79-96,120-141); the
oversampled form (CSpline_CreatePSF_Oversampled) is an extension, so the FP64 oracle with the same
voxel scale is the checker. With a step of 1 px it equals photonpy's form bit for bit. The
z-stack is the astigmatic model with the quartic term (s0 1.3 px, c 150 nm, d 400 nm, A 0.1,
B 0.05) on 26x26 points 0.5 px apart and 41 z planes 20 nm apart, each plane normalised.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STEP = 0.5


def _calibration(pb, ctx):
    from photonpy_b200 import synth
    zstack, zr = synth.astig_zstack(shape_xy=26, nz=41, zrange_um=(-0.4, 0.4), B=0.05, step_px=STEP)
    sm = pb.CSplineMethods(ctx)
    coefs = sm.ComputeSplineCoeff(zstack, border=1)
    return sm, zstack, zr, coefs


def test_unit_step_equals_reference_form(ctx):
    import photonpy_b200 as pb
    from conftest import load_golden
    from photonpy_b200.cspline import CSplinePSF
    g = load_golden("spline_r13")
    sm = pb.CSplineMethods(ctx)
    coefs = sm.ComputeSplineCoeff(g["zstack"], border=1)
    zr = g["spline_zrange"]
    calib = pb.CSplineCalibration(float(zr[0]), float(zr[1]), coefs)
    a = sm.CreatePSF_XYZIBg(int(g["roisize"]), calib, sm.FlatBg, True)
    b = CSplinePSF(ctx, sm._CSpline_CreatePSF_Oversampled(int(g["roisize"]), calib, None, sm.FlatBg, 1.0, True,
                                                          ctx.inst), calib)
    pa, _, _, ia = a.Estimate(g["samples"], return_iterations=True)
    pb_, _, _, ib = b.Estimate(g["samples"], return_iterations=True)
    assert np.array_equal(pa, pb_) and np.array_equal(ia, ib)
    assert np.array_equal(a.CRLBAndChiSquare(pa, g["samples"])[0], b.CRLBAndChiSquare(pa, g["samples"])[0])
    da, ea = a.Derivatives(g["truth"][:8])
    db, eb = b.Derivatives(g["truth"][:8])
    assert np.array_equal(da, db) and np.array_equal(ea, eb)
    a.Destroy()
    b.Destroy()


def test_half_pixel_spline_matches_fp64_oracle(ctx):
    import photonpy_b200 as pb
    from oracle import oracle as O
    from photonpy_b200 import synth
    sm, zstack, zr, coefs = _calibration(pb, ctx)
    assert np.array_equal(coefs, O.spline_compute(zstack, border=1))
    synth.use_torch(None, 0)
    d = synth.spline(1500, seed=41, B=0.05)
    calib = pb.CSplineCalibration(zr[0], zr[1], coefs)
    est = sm.CreatePSF_XYZIBg(d["R"], calib, sm.FlatBg, True, xyStep=STEP)
    m = O.Model(O.CSPLINE, d["R"], coefs=coefs, spline_zrange=zr, spline_xy_step=STEP)
    # model values and derivatives at the truth: float32 evaluation against the FP64 oracle
    deriv, ev = est.Derivatives(d["truth"][:32])
    d64, ev64 = m.derivatives(d["truth"][:32], fp64=True)
    assert np.max(np.abs(ev - ev64) / (np.abs(ev64) + 1.0)) < 1e-5
    scale = np.abs(d64).max(axis=(2, 3), keepdims=True) + 1e-20
    assert np.max(np.abs(deriv - d64) / scale) < 1e-4
    params, _, _, its = est.Estimate(d["samples"], return_iterations=True)
    p64, it64 = m.fit(d["samples"], fp64=True, iterations=200, lambda_=1e-18)
    # the z stop limit of photonpy's spline (1e-7 um) lets a fifth of the FP32 fits run to the cap
    conv = (its <= 50) & (it64 <= 200)
    assert conv.mean() > 0.7
    dxy = np.abs(params[conv, :2] - p64[conv, :2]).max(axis=1)
    dz = np.abs(params[conv, 2] - p64[conv, 2])
    rel = np.abs(params[conv, 3:] - p64[conv, 3:]) / np.maximum(np.abs(p64[conv, 3:]), 1e-6)
    print("xy", np.quantile(dxy, [.5, .99, 1]), "z um", np.quantile(dz, [.5, .99, 1]), "I/bg", np.quantile(rel, .99))
    assert np.mean(dxy <= 1e-3) >= 0.99
    assert np.mean(dz <= 1e-3) >= 0.99  # 1 nm, z in micrometres
    assert np.mean(np.all(rel <= 1e-4, axis=1)) >= 0.97
    # the 2x oversampled spline describes the analytic PSF the ROIs are drawn from: fits recover
    # the truth to well within a pixel
    assert np.median(np.abs(params[conv, :2] - d["truth"][conv, :2])) < 0.1
    crlb = est.CRLBAndChiSquare(params, d["samples"])[0]
    crlb64, _ = m.crlb(params, d["samples"], fp64=True)
    ok = np.all(np.isfinite(crlb64), axis=1)
    assert np.quantile((np.abs(crlb - crlb64) / crlb64)[ok].max(axis=1), 0.99) < 1e-4
    est.Destroy()


def _recalibration_problem(pb, ctx, n, seed, noise_free):
    """Spots with known parameters (workload distributions), ROIs drawn from the 0.5 px spline model
    itself (Poisson, or the expected values themselves), and coefficients with 5% multiplicative
    Gaussian noise per coefficient."""
    import torch
    sm, zstack, zr, coefs = _calibration(pb, ctx)
    calib = pb.CSplineCalibration(zr[0], zr[1], coefs)
    est = sm.CreatePSF_XYZIBg(13, calib, sm.FlatBg, True, xyStep=STEP)
    est._calib = calib
    rng = np.random.default_rng(seed)
    theta = np.stack([rng.uniform(5, 7, n), rng.uniform(5, 7, n), rng.uniform(-0.38, 0.38, n),
                      np.exp(rng.uniform(np.log(500), np.log(1e4), n)), rng.uniform(2, 15, n)], 1).astype(np.float32)
    ev = est.ExpectedValue(theta)
    samples = ev if noise_free else rng.poisson(ev).astype(np.float32)
    c_true = torch.from_numpy(coefs).cuda()
    noise = torch.from_numpy(rng.standard_normal(coefs.shape).astype(np.float32)).cuda()
    return est, torch.from_numpy(samples).cuda(), torch.from_numpy(theta).cuda(), c_true, c_true * (1 + 0.05 * noise)


def test_recalibration_lowers_nll_and_coefficient_error(ctx):
    """20 gradient-descent steps from coefficients with 5% Gaussian noise, on the expected values of
    20,000 spots of the spline model itself (so the unperturbed coefficients minimise the NLL):
    every step lowers the summed NLL and the distance to the unperturbed coefficients (a step along
    -g with an exact line search shortens the error of a convex quadratic; coefficients no pixel
    reads keep their noise)."""
    import torch
    import photonpy_b200 as pb
    from photonpy_b200.spline_calibration import recalibrate
    est, samples, theta, c_true, c0 = _recalibration_problem(pb, ctx, 20000, 44, noise_free=True)
    errs = []
    out = recalibrate(est, samples, theta, c0, steps=20,
                      callback=lambda k, c, f: errs.append(float(torch.linalg.vector_norm(c - c_true).item())))
    err0 = float(torch.linalg.vector_norm(c0 - c_true).item())
    nll = out["nll"]
    print("nll", [round(v - nll[-1], 1) for v in nll], "err", [round(e / err0, 4) for e in errs],
          "steps", out["step_sizes"])
    assert len(nll) == 21 and len(errs) == 20
    assert all(b < a for a, b in zip(nll, nll[1:]))
    e = [err0] + errs
    assert all(b < a for a, b in zip(e, e[1:]))
    est.Destroy()


def test_recalibration_from_poisson_rois(ctx):
    """The same from 500,000 Poisson ROIs (the spline workload's size): every step lowers the NLL,
    and the coefficient error weighted by the Fisher information of the data (the PSF error where
    pixels constrain it) falls by a fifth within the first steps and stays below its start; with
    1.6 million coefficients the later steps also fit the photon noise (measured on a B200: 0.89,
    0.84, ... 0.79 at step 8, then back up to 0.83 at step 20)."""
    import torch
    import photonpy_b200 as pb
    from photonpy_b200.spline_calibration import recalibrate, spline_nll_grad
    est, samples, theta, c_true, c0 = _recalibration_problem(pb, ctx, 500000, 45, noise_free=False)
    _, _, fisher = spline_nll_grad(est, samples, theta, c_true)
    werr = (lambda c: float(torch.sqrt((fisher.double() * (c - c_true).double() ** 2).sum()).item()))
    errs = []
    out = recalibrate(est, samples, theta, c0, steps=20, callback=lambda k, c, f: errs.append(werr(c)))
    nll = out["nll"]
    print("nll", [round(v - nll[-1], 1) for v in nll], "weighted err", [round(e / werr(c0), 4) for e in errs])
    assert all(b < a for a, b in zip(nll, nll[1:]))
    assert min(errs) < 0.82 * werr(c0)
    assert errs[-1] < 0.9 * werr(c0)
    est.Destroy()
