"""The CPU oracle against the reference's own golden vectors (no GPU needed).

tests/golden/*.npz hold what photonpy's C++ CPU estimator returned for seeded inputs
(tests/golden/make_golden.py). The FP32 oracle restates that arithmetic in C and must
reproduce it bit for bit; the FP64 oracle must agree within FP32 noise.
"""
import numpy as np
import pytest

from conftest import GOLDEN_SETS, load_golden
from helpers import coefs_sha, oracle_model
from oracle import oracle as O


@pytest.mark.parametrize("name", GOLDEN_SETS)
def test_oracle_fit_bit_exact(name):
    g = load_golden(name)
    m = oracle_model(name, g)
    c = g.get("constants")
    p, it, tr = m.fit(g["samples"], constants=c, trace_len=50)
    assert np.array_equal(p, g["params"])
    assert np.array_equal(it, g["iterations"])
    assert np.array_equal(tr[: len(g["trace"])], g["trace"])


@pytest.mark.parametrize("name", GOLDEN_SETS)
def test_oracle_crlb_chisq_bit_exact(name):
    g = load_golden(name)
    m = oracle_model(name, g)
    c = g.get("constants")
    crlb, chisq = m.crlb(g["params"], g["samples"], constants=c)
    assert np.array_equal(crlb, g["crlb"])
    assert np.array_equal(chisq, g["chisq"])
    crlb_t, _ = m.crlb(g["truth"], None, constants=c)
    assert np.array_equal(crlb_t, g["crlb_truth"])


@pytest.mark.parametrize("name", GOLDEN_SETS)
def test_oracle_derivatives_bit_exact(name):
    g = load_golden(name)
    m = oracle_model(name, g)
    c = g.get("constants")
    n = len(g["ev"])
    d, ev = m.derivatives(g["truth"][:n], constants=None if c is None else c[:n])
    assert np.array_equal(ev, g["ev"])
    assert np.array_equal(d, g["deriv"])


def test_oracle_spline_coefficients_bit_exact():
    g = load_golden("spline_r13")
    coefs = O.spline_compute(g["zstack"], border=1)
    assert tuple(coefs.shape) == tuple(g["coefs_shape"])
    assert coefs_sha(coefs) == bytes(g["coefs_sha256"]).decode() if isinstance(g["coefs_sha256"].item(), bytes) \
        else str(g["coefs_sha256"])
    assert np.array_equal(coefs.reshape(-1)[g["coefs_pick"]], g["coefs_pick_values"])


@pytest.mark.parametrize("name", ["xyibg_r10", "sigmaxy_r16", "astig_r12"])
def test_fp64_oracle_close_to_fp32(name):
    """The FP64 oracle converges to the same optimum within FP32 noise on converged spots."""
    g = load_golden(name)
    m = oracle_model(name, g)
    p64, it64 = m.fit(g["samples"], fp64=True, iterations=200)
    conv = (g["iterations"] <= 50) & (it64 <= 200)
    d = np.abs(p64[conv, :2] - g["params"][conv, :2])
    # a few spots settle in different local optima (FP64 takes other LM paths); the bulk agrees
    assert np.quantile(d, 0.95) < 1e-3


def test_oracle_derivative_matches_finite_difference():
    """Analytic Jacobian vs central differences of the FP64 model (psf_g2d_sigma.py:9-17)."""
    for name in GOLDEN_SETS:
        g = load_golden(name)
        m = oracle_model(name, g)
        c = g.get("constants")
        th = g["truth"][:8].astype(np.float64)
        cc = None if c is None else c[:8]
        d, _ = m.derivatives(th, constants=cc, fp64=True)
        K = th.shape[1]
        for k in range(K):
            h = 1e-2 * max(1.0, float(np.abs(th[:, k]).mean()))  # EV comes back as float32
            if name.startswith("spline") and k < 3:
                # the spline is only piecewise smooth across voxel faces: keep the stencil small
                h = 1e-3 if k < 2 else 1e-4
            tp, tm = th.copy(), th.copy()
            tp[:, k] += h
            tm[:, k] -= h
            num = (m.expected_value(tp, cc, fp64=True).astype(np.float64) -
                   m.expected_value(tm, cc, fp64=True).astype(np.float64)) / (2 * h)
            if name.startswith("sigma") and k >= 4:
                # photonpy's free-sigma Jacobian column is sigma * dmu/dsigma (the 1/sigma of the
                # erf-argument chain rule is absent, GaussianPSFModels.h:359,368,444,453)
                num = num * th[:, k][:, None, None]
            if name.startswith("tiltedsxy") and k in (4, 5):
                # XYITiltedBgSigmaXY keeps the tilt columns in its Jacobian but leaves the tilt out of
                # mu (GaussianPSFModels.h:542 vs 549): the columns are x - W/2 and y - H/2, mu ignores them
                R = int(g["roisize"])
                pix = np.arange(R) - R * 0.5
                want = np.broadcast_to(pix[None, None, :] if k == 4 else pix[None, :, None], d[:, k].shape)
                assert np.array_equal(d[:, k], want) and np.all(num == 0), (name, k)
                continue
            if name.startswith("tiltedsxy") and k >= 6:
                num = num * th[:, k][:, None, None]  # the same sigma * dmu/dsigma columns
            scale = np.abs(d[:, k]).max() + 1e-12
            assert np.abs(num - d[:, k]).max() / scale < 5e-3, (name, k)


def test_glrt_restatement_matches_float64_formula():
    """pso_glrt_f32 (GLRT_PSF.cu:96-131) against the same formula in float64 numpy."""
    from photonpy_b200 import synth
    d = synth.xyibg(50, seed=9)
    m = O.Model(O.XYIBG, d["R"], sigma=d["sigma"])
    p, _ = m.fit(d["samples"])
    got = m.glrt(p, d["samples"])
    ev = m.expected_value(p).astype(np.float64)
    s = d["samples"].astype(np.float64)
    mu, dd = np.maximum(ev, 1e-8), np.maximum(s, 1e-8)
    mean = s.mean(axis=(1, 2))
    assert np.array_equal(got[:, 2], mean.astype(np.float32))
    assert np.allclose(got[:, 0], np.sum(dd * np.log(mu) - mu, axis=(1, 2)), rtol=1e-5)
    ll_off = np.sum(dd * np.log(mean)[:, None, None] - mean[:, None, None], axis=(1, 2))
    assert np.allclose(got[:, 1], ll_off, rtol=1e-5)
    # the reference's mean source: first ROI for every spot
    ref = m.glrt(p, d["samples"], mean_roi=d["samples"][0])
    assert np.all(ref[:, 2] == got[0, 2])


def _intensity_bg_inputs(g):
    n = len(g["samples"])
    flat = g["sigma"].reshape(-1)  # the reference reads sigma[i] of the flat [n][2] array
    consts = np.stack([g["xy"][:, 0], g["xy"][:, 1], flat[:n]], 1).astype(np.float32)
    return consts, np.tile(np.float32([1.0, 0.0]), (n, 1))


def test_oracle_intensity_bg_bit_exact():
    """Gauss2D_EstimateIntensityBg (GaussianPSF.cu:216-240) restated: fit and CRLB equal the
    reference's CPU output bit for bit, including its flat indexing of sigma."""
    g = load_golden("intensitybg_r9")
    consts, init = _intensity_bg_inputs(g)
    m = O.Model(O.INTENSITYBG, int(g["roisize"]))
    p, _ = m.fit(g["samples"], constants=consts, initial=init, iterations=int(g["max_iterations"]), lambda_=1e-15)
    assert np.array_equal(p, g["ibg"])
    crlb, _ = m.crlb(p, None, constants=consts)
    assert np.array_equal(crlb, g["ibg_crlb"])


def test_oracle_spot_detection_finds_planted_spots():
    """The detection restatement (SpotDetector.cu:49-84) finds well-separated bright spots, in
    row-major order, honours the border rule and the maxSpots cap."""
    from photonpy_b200 import synth
    d = synth.frames(1, h=96, w=128, spots_per_frame=12, seed=3, I=(2000, 4000), margin=10)
    fr = d["frames"][0]
    found, idx, score, corner, rois = O.detect_spots(fr, 5, 10, 7, 9, 7.0)
    assert np.all(np.diff(idx) > 0)
    ys, xs = idx // 128, idx % 128
    tx, ty = d["truth"][:, 1], d["truth"][:, 2]
    dist = np.hypot(xs[:, None] - tx[None], ys[:, None] - ty[None]).min(axis=0)
    assert np.mean(dist < 1.5) > 0.8
    assert np.all((xs > 4) & (ys > 4) & (xs + 5 < 127) & (ys + 5 < 95))
    assert np.array_equal(corner, np.stack([ys - 4, xs - 4], 1))
    assert np.array_equal(rois[0], fr[corner[0, 0]:corner[0, 0] + 9, corner[0, 1]:corner[0, 1] + 9])
    f2, idx2, _, _, _ = O.detect_spots(fr, 5, 10, 7, 9, 7.0, max_spots=3)
    assert f2 == found and np.array_equal(idx2, idx[:3])
