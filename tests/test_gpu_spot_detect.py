"""Spot detection and ROI extraction on the GPU (SpotDetector_ProcessFrame, ExtractROIs,
PB200_DetectSpotsDevice, photonpy_b200.spotdetect).

The detection restatement in the oracle is pinned bit for bit against the reference's own CUDA
detector (oracle/_ref, run on this GPU); the CUDA path is then compared bit for bit with the
oracle: same spots in the same order, same scores, corners and ROI pixels. Cases: frames whose
sizes are not multiples of the 32-pixel tile, spots at the borders, a background image, an
intensity window, the maxSpots cap, several frames per launch, filter sizes outside the
register-strip instantiations (the generic kernel). The end-to-end check fits the detected ROIs
and compares positions with the planted spots. The exact count division the box filters use is
compared with IEEE division for every float.
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref_lib
from photonpy_b200 import synth

pytestmark = pytest.mark.gpu

CASES = [
    dict(h=96, w=128, sigma=1.5, roisize=9, min_i=7.0, max_i=np.inf, bg=False, cap=1000, seed=1),
    dict(h=77, w=131, sigma=1.3, roisize=8, min_i=5.0, max_i=40.0, bg=True, cap=1000, seed=2),
    dict(h=200, w=45, sigma=2.0, roisize=11, min_i=3.0, max_i=np.inf, bg=False, cap=7, seed=3),
]


def _frame(c):
    d = synth.frames(1, h=c["h"], w=c["w"], spots_per_frame=25, seed=c["seed"], sigma=c["sigma"], margin=0)
    fr = d["frames"][0]
    bg = None
    if c["bg"]:
        rng = np.random.default_rng(c["seed"] + 100)
        bg = rng.uniform(2.0, 6.0, size=fr.shape).astype(np.float32)
    return fr, bg


def _sizes(sigma):
    u1 = int(sigma * 2 + 2)
    return u1, 2 * u1, int(sigma * 5)


@pytest.mark.skipif(not ref_lib.available(), reason="reference build absent")
@pytest.mark.parametrize("c", CASES)
def test_reference_detector_pins_oracle(c):
    if not hasattr(ref_lib.lib(), "SpotDetector_ProcessFrame"):
        pytest.skip("reference build without the spot detector")
    fr, bg = _frame(c)
    u1, u2, mf = _sizes(c["sigma"])
    n, sc, sz, corner, rois = ref_lib.process_frame(fr, u1, u2, mf, c["roisize"], c["min_i"], c["max_i"], bg,
                                                    max_spots=c["cap"])
    found, idx, score, ocorner, orois = O.detect_spots(fr, u1, u2, mf, c["roisize"], c["min_i"], c["max_i"], bg,
                                                       max_spots=c["cap"])
    assert n == min(found, c["cap"]) and n > 0
    assert np.array_equal(sc, score)
    assert np.array_equal(corner, ocorner)
    assert np.array_equal(rois, orois)
    assert np.all(sz == 0)


@pytest.mark.parametrize("c", CASES)
def test_process_frame_equals_oracle(ctx, c):
    from photonpy_b200 import spotdetect
    fr, bg = _frame(c)
    sd = spotdetect.SpotDetector(c["sigma"], c["roisize"], c["min_i"], c["max_i"], bg)
    rois, corner, scores, spotz = spotdetect.SpotDetectionMethods(ctx).ProcessFrame(fr, sd, c["roisize"], c["cap"])
    u1, u2, mf = _sizes(c["sigma"])
    found, idx, oscore, ocorner, orois = O.detect_spots(fr, u1, u2, mf, c["roisize"], c["min_i"], c["max_i"], bg,
                                                        max_spots=c["cap"])
    assert len(scores) == min(found, c["cap"]) > 0
    assert np.array_equal(scores, oscore)
    assert np.array_equal(corner, ocorner)
    assert np.array_equal(rois, orois)
    assert np.all(spotz == 0)


@pytest.mark.parametrize("sizes", [(5, 9, 7), (3, 7, 4), (10, 20, 20), (1, 3, 1), (6, 12, 3)])
def test_process_frame_filter_sizes(ctx, sizes):
    """Box/maximum filter sizes set directly: (5, 9) and (3, 7) are not u2 = 2 u1 and (10, 20) is
    above the instantiations, so these run the generic kernel; (1, 3, 1) makes every pixel a
    local maximum; (6, 12, 3) is a register-strip kernel with a small maximum filter."""
    from photonpy_b200 import spotdetect
    u1, u2, mf = sizes
    d = synth.frames(1, h=70, w=90, spots_per_frame=12, seed=20 + u1, margin=0)
    fr = d["frames"][0]
    sd = spotdetect.SpotDetector(1.5, 7, 2.0)
    sd.uniformFilter1Size, sd.uniformFilter2Size, sd.maxFilterSize = u1, u2, mf
    rois, corner, scores, _ = spotdetect.SpotDetectionMethods(ctx).ProcessFrame(fr, sd, 7, 5000)
    found, idx, oscore, ocorner, orois = O.detect_spots(fr, u1, u2, mf, 7, 2.0, max_spots=5000)
    assert len(scores) == min(found, 5000) > 0
    assert np.array_equal(scores, oscore)
    assert np.array_equal(corner, ocorner)
    assert np.array_equal(rois, orois)


def test_process_frame_nan_and_inf_pixels(ctx):
    """NaN and infinite pixels: tiles whose detection image holds NaN take the left-to-right
    maximum fold (where NaN is not skipped like a number); results equal the oracle's."""
    from photonpy_b200 import spotdetect
    d = synth.frames(1, h=96, w=100, spots_per_frame=20, seed=31, margin=0)
    fr = d["frames"][0].copy()
    fr[10, 10] = np.nan
    fr[50, 70] = np.inf
    fr[80, 5] = -np.inf
    fr[40, 40] = np.nan
    fr[41, 44] = np.inf
    sd = spotdetect.SpotDetector(1.5, 9, 7.0)
    rois, corner, scores, _ = spotdetect.SpotDetectionMethods(ctx).ProcessFrame(fr, sd, 9, 1000)
    u1, u2, mf = _sizes(1.5)
    found, idx, oscore, ocorner, orois = O.detect_spots(fr, u1, u2, mf, 9, 7.0, max_spots=1000)
    assert len(scores) == min(found, 1000) > 0
    assert np.array_equal(scores, oscore, equal_nan=True)
    assert np.array_equal(corner, ocorner)
    assert np.array_equal(rois, orois, equal_nan=True)


def test_count_division_exhaustive(ctx):
    """The box filters' sum / count (rounded reciprocal, one FMA correction) equals IEEE division
    bit for bit for all 2^32 floats and every count 1..32."""
    import ctypes
    lib = ctx.smlm.lib
    bad = (ctypes.c_ulonglong * 32)()
    last = (ctypes.c_uint * 32)()
    assert lib.PB200_CheckCountDivision(32, bad, last) == 0
    assert list(bad) == [0] * 32, [(k + 1, bad[k], hex(last[k])) for k in range(32) if bad[k]]


def test_detect_device_batch_equals_oracle(ctx):
    import torch
    from photonpy_b200 import spotdetect
    d = synth.frames(6, h=150, w=170, spots_per_frame=30, seed=11)
    sd = spotdetect.SpotDetector(1.5, 9, 7.0)
    cap = 25  # below the count of some frames: the cap applies per frame
    rois, corner, fidx, scores, found = spotdetect.SpotDetectionMethods(ctx).DetectDevice(
        torch.from_numpy(d["frames"]).cuda(), sd, 9, cap)
    rois, corner, fidx, scores, found = (t.cpu().numpy() for t in (rois, corner, fidx, scores, found))
    u1, u2, mf = _sizes(1.5)
    for f in range(6):
        nf, idx, osc, ocor, orois = O.detect_spots(d["frames"][f], u1, u2, mf, 9, 7.0, max_spots=cap)
        sel = fidx == f
        assert found[f] == nf
        assert sel.sum() == min(nf, cap)
        assert np.array_equal(scores[sel], osc)
        assert np.array_equal(corner[sel], ocor)
        assert np.array_equal(rois[sel], orois)


def test_extract_rois_matches_reference_semantics(ctx):
    """ExtractROIs (SpotDetector.cu:155-178): y/x clamped; slice z of each box comes from frame z
    of the stack (the reference ignores the corner's z when reading)."""
    from photonpy_b200 import spotdetect
    rng = np.random.default_rng(5)
    frames = rng.normal(size=(4, 40, 50)).astype(np.float32)
    corners = np.array([[0, -3, -2], [1, 35, 47], [2, 10, 20], [3, -5, 45]], np.int32)
    rois = spotdetect.SpotDetectionMethods(ctx).ExtractROIs(frames, (2, 7, 6), corners)
    want = np.zeros_like(rois)
    for i, (z0, y0, x0) in enumerate(corners):
        for z in range(2):
            for y in range(7):
                for x in range(6):
                    want[i, z, y, x] = frames[z, min(max(y0 + y, 0), 39), min(max(x0 + x, 0), 49)]
    assert np.array_equal(rois, want)
    if ref_lib.available() and hasattr(ref_lib.lib(), "ExtractROIs"):
        import ctypes as ct
        out = np.zeros_like(rois)
        ref_lib.lib().ExtractROIs(frames.ctypes.data, 50, 40, 4, 6, 7, 2, corners.ctypes.data, 4, out.ctypes.data)
        assert np.array_equal(rois, out)
        del ct


def test_localize_frames_end_to_end(ctx):
    """Frames -> detection -> fused fit on the GPU: detected spots land within 0.3 px of the
    planted ones (isolated spots, I >= 1000)."""
    import torch
    import photonpy_b200 as pb
    from photonpy_b200 import spotdetect
    d = synth.frames(8, h=128, w=128, spots_per_frame=15, seed=12, I=(1000, 3000), margin=8)
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(9, 1.5, True)
    sd = spotdetect.SpotDetector(1.5, 9, 7.0)
    r = spotdetect.localize_frames(torch.from_numpy(d["frames"]).cuda(), sd, est, 9)
    p = r["params"].cpu().numpy()
    fr = r["frame"].cpu().numpy()
    t = d["truth"]
    hits = 0
    for f in range(8):
        tf = t[t[:, 0] == f]
        pf = p[fr == f]
        dd = np.hypot(pf[:, None, 0] - tf[None, :, 1], pf[:, None, 1] - tf[None, :, 2])
        hits += int(np.sum(dd.min(axis=0) < 0.3))
    assert hits >= 0.8 * len(t)
    est.Destroy()
