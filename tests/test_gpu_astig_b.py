"""Astigmatic 3D Gaussian with the quartic term (B = 0.05): fit and CRLB against the FP64 oracle.

photonpy's model has sigma(z) = s0 sqrt(1 + tz^2/d^2 + A tz^3/d^2) (GaussianPSFModels.h:698-702);
the workload this library is benchmarked on adds B tz^4/d^4 (Gauss2D_CreatePSF_XYZIBgB,
Gauss3D_CalibrationB). The reference cannot express it, so the FP64 oracle (the same model and LM
in double precision, iterated to its own convergence) is the checker. With B = 0 the extension
is bit-identical to photonpy's 4-coefficient form.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _astig_b(n, seed, B):
    from photonpy_b200 import synth
    synth.use_torch(None, 0)
    return synth.astig(n, seed=seed, B=B)


def _estimator(pb, ctx, d):
    cx, cy = d["astig"]
    return pb.GaussianPSFMethods(ctx).CreatePSF_XYZIBg(d["R"], pb.Gauss3D_CalibrationB(cx, cy, d["zrange"]), True)


def _oracle(d):
    from oracle import oracle as O
    cx, cy = d["astig"]
    return O.Model(O.XYZIBG, d["R"], astig_x=list(cx), astig_y=list(cy), zrange=tuple(d["zrange"]))


def test_quartic_astig_fit_matches_fp64_oracle(ctx):
    import photonpy_b200 as pb
    d = _astig_b(2000, 31, 0.05)
    est = _estimator(pb, ctx, d)
    params, _, _, its = est.Estimate(d["samples"], return_iterations=True)
    est.Destroy()
    m = _oracle(d)
    p64, it64 = m.fit(d["samples"], fp64=True, iterations=200, lambda_=1e-18)
    conv = (its <= 50) & (it64 <= 200)
    assert conv.mean() > 0.95
    dxy = np.abs(params[conv, :2] - p64[conv, :2]).max(axis=1)
    dz = np.abs(params[conv, 2] - p64[conv, 2])
    rel = np.abs(params[conv, 3:] - p64[conv, 3:]) / np.abs(p64[conv, 3:])
    print("xy", np.quantile(dxy, [.5, .99, 1]), "z nm", np.quantile(dz, [.5, .99, 1]), "I/bg", np.quantile(rel, [.5, .99]))
    assert np.mean(dxy <= 1e-3) >= 0.99
    assert np.mean(dz <= 1.0) >= 0.99
    assert np.mean(np.all(rel <= 1e-4, axis=1)) >= 0.97


def test_quartic_astig_crlb_matches_fp64_oracle(ctx):
    import photonpy_b200 as pb
    d = _astig_b(500, 32, 0.05)
    est = _estimator(pb, ctx, d)
    crlb, chisq = est.CRLBAndChiSquare(d["truth"], d["samples"])
    m = _oracle(d)
    crlb64, chisq64 = m.crlb(d["truth"], d["samples"], fp64=True)
    rel = np.abs(crlb - crlb64) / crlb64
    assert np.quantile(rel.max(axis=1), 0.99) < 1e-4, np.quantile(rel, [.5, .99, 1])
    assert np.quantile(np.abs(chisq - chisq64) / chisq64, 0.99) < 1e-4
    # B changes the model: the same spots under the B = 0 form have measurably different bounds
    d0 = dict(d)
    cx, cy = d["astig"]
    d0["astig"] = (list(cx[:4]) + [0.0], list(cy[:4]) + [0.0])
    crlb0, _ = _oracle(d0).crlb(d["truth"], d["samples"], fp64=True)
    assert np.median(np.abs(crlb0[:, 2] - crlb64[:, 2]) / crlb64[:, 2]) > 1e-3
    est.Destroy()


def test_quartic_astig_with_zero_b_equals_reference_form(ctx):
    """Gauss3D_CalibrationB with B = 0 fits exactly like photonpy's Gauss3D_Calibration."""
    import photonpy_b200 as pb
    d = _astig_b(400, 33, 0.0)
    cx, cy = d["astig"]
    e4 = pb.GaussianPSFMethods(ctx).CreatePSF_XYZIBg(d["R"], pb.Gauss3D_Calibration(cx[:4], cy[:4], d["zrange"]), True)
    e5 = _estimator(pb, ctx, d)
    p4, _, _, i4 = e4.Estimate(d["samples"], return_iterations=True)
    p5, _, _, i5 = e5.Estimate(d["samples"], return_iterations=True)
    assert np.array_equal(p4, p5) and np.array_equal(i4, i5)
    assert np.array_equal(e4.CRLBAndChiSquare(p4, d["samples"])[0], e5.CRLBAndChiSquare(p5, d["samples"])[0])
    e4.Destroy()
    e5.Destroy()
