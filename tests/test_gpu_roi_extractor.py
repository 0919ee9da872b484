"""ROI extractor on the GPU (ROIExtractor_Create + ImgProc_AddFrameU16 + ROIExtractor_Get*):
boxes of predefined ROIs cut from a stream of 16-bit frames.

The oracle restates the extractor (calibrated frames, one box per frame of each ROI, records in
order of last frame, start frame, request order); the reference's own extractor (oracle/_ref)
pins it on ROIs inside the frame, records and boxes bit for bit and in the same order. The CUDA
extractor must give the oracle's records and boxes, in order, also for boxes that cross the
frame border (clamped here; the reference reads outside the frame there)."""
import time

import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref_lib

pytestmark = pytest.mark.gpu


def _movie(n, h, w, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(90, 400, size=(n, h, w)).astype(np.uint16)


def _rois(n, h, w, roisize, nframes_max, inside, seed, nmovie):
    rng = np.random.default_rng(seed)
    r = np.zeros(n, O.ROI_TYPE)
    if inside:
        r["cornerpos"][:, 0] = rng.integers(0, w - roisize + 1, n)
        r["cornerpos"][:, 1] = rng.integers(0, h - roisize + 1, n)
    else:
        r["cornerpos"][:, 0] = rng.integers(-roisize, w, n)
        r["cornerpos"][:, 1] = rng.integers(-roisize, h, n)
    r["startframe"] = rng.integers(0, nmovie, n)
    r["numframes"] = rng.integers(1, nframes_max + 1, n)
    return r


def _run(ctx, frames, rois, roiframes, roisize, calib=None):
    from photonpy_b200.image_proc import ROIExtractor
    q = ROIExtractor(frames.shape[1:], rois, roiframes, roisize, calib, ctx)
    for f in frames:
        q.PushFrameU16(f)
    t0 = time.time()
    while not q.IsIdle():
        assert time.time() - t0 < 60
        time.sleep(0.005)
    assert q.NumFinishedFrames() == len(frames)
    out = q.GetResults(q.GetResultCount())
    q.Destroy()
    return out


@pytest.mark.parametrize("roiframes,nfmax,calib", [(1, 1, None), (2, 3, "gain_offset"), (3, 3, None)])
def test_extractor_equals_oracle(ctx, roiframes, nfmax, calib):
    from photonpy_b200.calib import GainOffset_Calib
    frames = _movie(23, 70, 90, seed=roiframes)
    rois = _rois(400, 70, 90, 9, nfmax, inside=False, seed=nfmax, nmovie=25)
    rois["numframes"][::37] = 0  # complete at their start frame with no box
    cal = GainOffset_Calib(0.5, 100.0, ctx) if calib else None
    r, b = _run(ctx, frames, rois, roiframes, 9, cal)
    orr, ob = O.extract_rois(frames, rois, roiframes, 9, ("gain_offset", 0.5, 100.0) if calib else None)
    assert len(r) == len(orr) > 0
    assert np.array_equal(r, orr)
    assert np.array_equal(b, ob)


@pytest.mark.skipif(not ref_lib.available(), reason="reference build absent")
def test_reference_extractor_pins_oracle():
    if not hasattr(ref_lib.lib(), "ROIExtractor_Create"):
        pytest.skip("reference build without the ROI extractor")
    frames = _movie(12, 64, 80, seed=7)
    rois = _rois(150, 64, 80, 7, 3, inside=True, seed=8, nmovie=12)
    r, b = ref_lib.roi_extractor(frames, rois, 3, 7)
    orr, ob = O.extract_rois(frames, rois, 3, 7)
    assert len(r) == len(orr) > 0
    assert np.array_equal(r, orr)
    assert np.array_equal(b, ob)


def test_extract_rois_iterator(ctx):
    from photonpy_b200 import process_movie as pm
    frames = _movie(10, 48, 60, seed=3)
    rng = np.random.default_rng(4)
    pos = np.stack([rng.integers(0, 50, 200), rng.integers(0, 40, 200)], axis=1)
    fr = rng.integers(0, 10, 200)
    got_r, got_b = [], []
    for r, b in pm.extract_rois_iterator(iter(frames), pos, fr, None, 7, ctx, 20):
        got_r.append(r)
        got_b.append(b)
    r, b = np.concatenate(got_r), np.concatenate(got_b)
    rois = np.zeros(200, O.ROI_TYPE)
    rois["cornerpos"] = pos
    rois["startframe"] = fr
    rois["numframes"] = 1
    orr, ob = O.extract_rois(frames, rois, 1, 7)
    assert np.array_equal(r, orr) and np.array_equal(b, ob)
