"""Likelihood-ratio test estimator (GLRT_CreatePSF, photonpy_b200.glrt).

Checks, on the GPU: the GLRT estimator fits exactly like its model estimator; its three
diagnostics equal the oracle's restatement of GLRT_PSF.cu:96-131 evaluated at the same
parameters (mean bit-exact for integer counts, log-likelihoods within 2e-5 relative, a
float32 summation-order tolerance over <= 256 pixels); the reference-mean mode reproduces the
reference's first-ROI mean bit-exactly; diagnostics travel through the estimation queue; and,
when the reference's own CUDA build is present, the reference GLRT's outputs match the
oracle at the reference's own fitted parameters (pins the restatement). The detection test
follows photonpy/tests/glrt_psf.py (9x9 ROIs, sigma 1.5, I = 50, bg = 5).
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref_lib
from photonpy_b200 import synth

pytestmark = pytest.mark.gpu

RTOL = 2e-5


def _close(a, b, rtol=RTOL, scale=None):
    """Equal NaN positions, elsewhere |a - b| <= rtol * max(|b|, scale, 1). `scale` is the sum of
    the magnitudes of the summed terms: a log-likelihood that cancels (a poor fit, ll ~ -3e4 from
    terms of 1e5) carries the rounding of its terms, not of its value."""
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), (np.flatnonzero(na != nb)[:5], a[na != nb][:5], b[na != nb][:5])
    ref = np.maximum(np.abs(b), 1.0)
    if scale is not None:
        ref = np.maximum(ref, 0.1 * scale)
    ok = np.abs(a[~na] - b[~nb]) <= rtol * ref[~nb]
    assert ok.all(), (np.flatnonzero(~ok)[:5], a[~na][~ok][:5], b[~nb][~ok][:5])
    return True


def _ll_scale(om, params, smp):
    """sum_p |d log mu| + mu, the magnitude of the terms of ll_on (float64)."""
    mu = np.maximum(om.expected_value(params).astype(np.float64), 1e-8)
    d = np.maximum(smp.astype(np.float64), 1e-8)
    return np.sum(np.abs(d * np.log(mu)) + mu, axis=(1, 2))


@pytest.mark.parametrize("kind", ["xyibg", "sigmaxy", "astig"])
def test_glrt_matches_oracle_and_model_fit(ctx, kind):
    import photonpy_b200 as pb
    from photonpy_b200 import glrt
    g = pb.GaussianPSFMethods(ctx)
    if kind == "xyibg":
        d = synth.xyibg(3000, seed=41)
        est = g.CreatePSF_XYIBg(d["R"], d["sigma"], True)
        om = O.Model(O.XYIBG, d["R"], sigma=d["sigma"])
    elif kind == "sigmaxy":
        d = synth.sigmaxy(2000, seed=42)
        est = g.CreatePSF_XYIBgSigmaXY(d["R"], d["sigma"], True)
        om = O.Model(O.XYIBG_SIGMAXY, d["R"], sigma=d["sigma"])
    else:
        d = synth.astig(2000, seed=43)
        cx, cy = d["astig"]
        est = g.CreatePSF_XYZIBg(d["R"], pb.Gauss3D_Calibration(list(cx[:4]), list(cy[:4]), list(d["zrange"])), True)
        om = O.Model(O.XYZIBG, d["R"], astig_x=cx, astig_y=cy, zrange=tuple(d["zrange"]))
    ge = glrt.CreateEstimator(est, ctx)
    assert ge.NumDiag() == 3 and ge.NumParams() == est.NumParams()
    smp = d["samples"]
    p0, _, _, it0 = est.Estimate(smp, return_iterations=True)
    p1, diag, _, it1 = ge.Estimate(smp, return_iterations=True)
    assert np.array_equal(p0, p1) and np.array_equal(it0, it1)
    want = om.glrt(p1, smp)
    assert np.array_equal(diag[:, 2], want[:, 2])  # integer counts: exact in any order
    assert _close(diag[:, 1], want[:, 1])
    # ll_on: spots whose fitted background went to its 1e-6 floor have mu in the PSF tails set by
    # the cancellation 0.5 (erf(a) - erf(b)) with erf ~ 1, where erff implementations differ by
    # many relative ulps (the reference's CPU and GPU builds differ there too); compare the
    # spots with min(mu) >= 1e-3 and require them to be the large majority.
    ok = om.expected_value(p1).reshape(len(p1), -1).min(axis=1) >= 1e-3
    assert ok.mean() > 0.95
    assert _close(diag[ok, 0], want[ok, 0], scale=_ll_scale(om, p1[ok], smp[ok]))
    lp = glrt.ComputeLogPFA(diag)
    assert lp.shape == (len(smp),) and np.all(lp <= 0)
    ge.Destroy()
    est.Destroy()


def test_glrt_reference_mean_mode(ctx):
    import photonpy_b200 as pb
    from photonpy_b200 import glrt
    d = synth.xyibg(1000, seed=44)
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(d["R"], d["sigma"], True)
    ge = glrt.CreateEstimator(est, ctx)
    glrt.SetReferenceMean(ge, True)
    smp = d["samples"]
    p, diag, _ = ge.Estimate(smp)
    om = O.Model(O.XYIBG, d["R"], sigma=d["sigma"])
    want = om.glrt(p, smp, mean_roi=smp[0])
    assert np.all(diag[:, 2] == want[0, 2])
    assert np.array_equal(diag[:, 2], want[:, 2])
    assert _close(diag[:, 1], want[:, 1]) and _close(diag[:, 0], want[:, 0])
    ge.Destroy()
    est.Destroy()


def test_glrt_detects_spots_like_reference_test(ctx):
    """photonpy/tests/glrt_psf.py: 9x9, sigma 1.5, theta = (4.5, 4.5, 50, 5). The dim spot is
    detected (median P_fa 1.5e-7 with the oracle); background-only ROIs, where the fit latches on
    to noise, give a median P_fa of 5.8e-3 (oracle, same seeds)."""
    import photonpy_b200 as pb
    from photonpy_b200 import glrt
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(9, 1.5, True)
    ge = glrt.CreateEstimator(est, ctx)
    rng = np.random.default_rng(45)
    theta = np.repeat([[4.5, 4.5, 50.0, 5.0]], 5000, 0)
    smp = rng.poisson(est.ExpectedValue(theta)).astype(np.float32)
    _, diag, _ = ge.Estimate(smp)
    pfa_spot = np.exp(glrt.ComputeLogPFA(diag))
    bg = rng.poisson(np.full((5000, 9, 9), 5.0)).astype(np.float32)
    _, diag_bg, _ = ge.Estimate(bg)
    pfa_bg = np.exp(glrt.ComputeLogPFA(diag_bg))
    assert np.median(pfa_spot) < 1e-5 and np.mean(pfa_spot) < 0.05
    assert np.median(pfa_bg) > 1e-3
    assert np.mean(pfa_spot) < 0.2 * np.mean(pfa_bg)
    ge.Destroy()
    est.Destroy()


def test_glrt_through_queue(ctx):
    import photonpy_b200 as pb
    from photonpy_b200 import glrt
    d = synth.xyibg(5000, seed=46)
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(d["R"], d["sigma"], True)
    ge = glrt.CreateEstimator(est, ctx)
    p, diag, _ = ge.Estimate(d["samples"])
    with pb.EstimQueue(ge, batchSize=300, numStreams=2) as q:
        q.Schedule(d["samples"], ids=np.arange(5000, dtype=np.int32))
        q.WaitUntilDone()
        r = q.GetResults()
    r.SortByID(isUnique=True)
    assert np.array_equal(r.estim, p)
    assert np.array_equal(r.diagnostics, diag)
    ge.Destroy()
    est.Destroy()


@pytest.mark.skipif(not ref_lib.available(), reason="reference build absent")
def test_reference_glrt_pins_oracle():
    """The reference's GLRT (its CUDA build) against the oracle at the reference's own fitted
    parameters, with the reference's first-ROI mean: pins the restatement of GLRT_PSF.cu."""
    L = ref_lib.lib()
    if not hasattr(L, "GLRT_CreatePSF"):
        pytest.skip("reference build without GLRT_PSF.cu")
    d = synth.xyibg(2000, seed=47)
    model = ref_lib.RefEstimator("XYIBg", d["R"], cuda=True, sigma=d["sigma"])
    rg = ref_lib.RefGLRT(model)
    p, diag = rg.estimate(d["samples"])
    om = O.Model(O.XYIBG, d["R"], sigma=d["sigma"])
    want = om.glrt(p, d["samples"], mean_roi=d["samples"][0])
    assert np.array_equal(diag[:, 2], want[:, 2])
    assert _close(diag[:, 0], want[:, 0]) and _close(diag[:, 1], want[:, 1])
    model.close()
