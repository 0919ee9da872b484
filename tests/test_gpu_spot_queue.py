"""Spot-extraction queue on the GPU (SpotExtractionQueue_Create + ImgProc_* + RQ_*), calibrated
ProcessFrame, and the movie -> ROI file -> localizations path of process_movie.

The oracle restates the queue (calibration in float32, sums left to right, the detection
restatement pinned to the reference's detector, ROI stacks of the calibrated frames); the
reference's own queue (oracle/_ref, its CUDA detector) pins it. The CUDA queue must give the
same records and ROI pixels bit for bit. Records are compared after ordering by (id, y, x): the
reference detects on several threads, so its order across frames is not fixed, and RQ_Pop
hands back a batch newest first."""
import time

import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref_lib
from photonpy_b200 import synth

pytestmark = pytest.mark.gpu


def _sizes(sigma):
    u1 = int(sigma * 2 + 2)
    return u1, 2 * u1, int(sigma * 5)


def _movie(n, h, w, seed, gain=None, offset=None, spots=25):
    d = synth.frames(n, h=h, w=w, spots_per_frame=spots, seed=seed, margin=0)
    counts = d["frames"]
    if gain is None:
        return counts.astype(np.uint16), d
    raw = np.clip(np.round(counts / gain + offset), 0, 65535)
    return raw.astype(np.uint16), d


def _sorted(info, rois):
    order = np.lexsort((info["x"], info["y"], info["id"]))
    return info[order], rois[order]


def _run_queue(ctx, frames, sd, roisize, sumframes, calib=None):
    from photonpy_b200 import spotdetect
    sm = spotdetect.SpotDetectionMethods(ctx)
    q, rq = sm.CreateQueue(frames.shape[1:], [roisize, roisize], sd, calib=calib, sumframes=sumframes)
    for f in frames:
        q.PushFrameU16(f)
    t0 = time.time()
    while q.NumFinishedFrames() < len(frames) // sumframes or not q.IsIdle():
        assert time.time() - t0 < 60
        time.sleep(0.005)
    info, rois = rq.Fetch()
    q.Destroy()
    rq.Destroy()
    return info, rois.reshape(len(info), sumframes, roisize, roisize)


CASES = [
    dict(sf=1, calib=None, h=96, w=130, sigma=1.5, roisize=9, n=9),
    dict(sf=2, calib="gain_offset", h=80, w=77, sigma=1.3, roisize=8, n=7),
    dict(sf=3, calib="image", h=64, w=100, sigma=2.0, roisize=11, n=9),
]


@pytest.mark.parametrize("c", CASES)
def test_queue_equals_oracle(ctx, c):
    from photonpy_b200 import spotdetect
    from photonpy_b200.calib import GainOffset_Calib, GainOffsetImage_Calib
    rng = np.random.default_rng(7)
    gain = offset = None
    calib = ocal = None
    if c["calib"] == "gain_offset":
        gain, offset = 0.5, 100.0
        calib = GainOffset_Calib(gain, offset, ctx)
        ocal = ("gain_offset", gain, offset)
    frames, _ = _movie(c["n"], c["h"], c["w"], seed=c["sf"] * 11, gain=gain if gain else None,
                       offset=offset if offset else 0)
    if c["calib"] == "image":
        g = rng.uniform(0.8, 1.2, (c["h"], c["w"])).astype(np.float32)
        o = rng.uniform(0.0, 3.0, (c["h"], c["w"])).astype(np.float32)
        calib = GainOffsetImage_Calib(g, o, ctx)
        ocal = ("image", g, o)
    sd = spotdetect.SpotDetector(c["sigma"], c["roisize"], 6.0)
    info, rois = _run_queue(ctx, frames, sd, c["roisize"], c["sf"], calib)
    u1, u2, mf = _sizes(c["sigma"])
    oinfo, orois = O.spot_extraction_queue(frames, u1, u2, mf, c["roisize"], 6.0, sumframes=c["sf"], calib=ocal)
    assert len(info) == len(oinfo) > 0
    info, rois = _sorted(info, rois)
    oinfo, orois = _sorted(oinfo, orois)
    assert np.array_equal(info, oinfo)
    assert np.array_equal(rois, orois)


@pytest.mark.skipif(not ref_lib.available(), reason="reference build absent")
@pytest.mark.parametrize("sf,go", [(1, None), (2, (0.5, 100.0))])
def test_reference_queue_pins_oracle(sf, go):
    if not hasattr(ref_lib.lib(), "SpotExtractionQueue_Create"):
        pytest.skip("reference build without the frame queue")
    frames, _ = _movie(6, 72, 90, seed=40 + sf, gain=go[0] if go else None, offset=go[1] if go else 0)
    u1, u2, mf = _sizes(1.5)
    info, rois = ref_lib.spot_queue(frames, u1, u2, mf, 9, 6.0, sumframes=sf, gain_offset=go)
    ocal = ("gain_offset", go[0], go[1]) if go else None
    oinfo, orois = O.spot_extraction_queue(frames, u1, u2, mf, 9, 6.0, sumframes=sf, calib=ocal)
    assert len(info) == len(oinfo) > 0
    info, rois = _sorted(info, rois)
    oinfo, orois = _sorted(oinfo, orois)
    assert np.array_equal(info, oinfo)
    assert np.array_equal(rois, orois)


def test_queue_frames_with_many_spots(ctx):
    """More spots in a frame than the detector's first output capacity (256): the batch runs
    again with room for all of them, as the reference keeps every spot."""
    from photonpy_b200 import spotdetect
    frames, _ = _movie(3, 96, 96, seed=5, spots=40)
    sd = spotdetect.SpotDetector(1.5, 5, -1e30)
    sd.uniformFilter1Size, sd.uniformFilter2Size, sd.maxFilterSize = 1, 3, 1  # nearly every pixel
    info, rois = _run_queue(ctx, frames, sd, 5, 1)
    oinfo, orois = O.spot_extraction_queue(frames, 1, 3, 1, 5, -1e30, sumframes=1)
    assert len(oinfo) > 3 * 256
    info, rois = _sorted(info, rois)
    oinfo, orois = _sorted(oinfo, orois)
    assert np.array_equal(info, oinfo)
    assert np.array_equal(rois, orois)


def test_process_frame_with_calibration(ctx):
    """SpotDetector.cu:104-141: detection on the calibrated frame, ROIs from the frame as given."""
    from photonpy_b200 import spotdetect
    from photonpy_b200.calib import GainOffset_Calib
    frames, _ = _movie(1, 90, 110, seed=9, gain=0.5, offset=100.0)
    raw = frames[0].astype(np.float32)
    sd = spotdetect.SpotDetector(1.5, 9, 6.0)
    rois, corner, scores, _ = spotdetect.SpotDetectionMethods(ctx).ProcessFrame(raw, sd, 9, 500,
                                                                                calib=GainOffset_Calib(0.5, 100.0, ctx))
    cal = O.camera_calibrate(raw, "gain_offset", 0.5, 100.0)
    found, idx, oscore, ocorner, _ = O.detect_spots(cal, *_sizes(1.5), 9, 6.0, max_spots=500)
    assert len(scores) == found > 0
    assert np.array_equal(scores, oscore) and np.array_equal(corner, ocorner)
    want = np.stack([raw[np.clip(np.arange(cy, cy + 9), 0, 89)][:, np.clip(np.arange(cx, cx + 9), 0, 109)]
                     for cy, cx in ocorner])
    assert np.array_equal(rois, want)


def test_float_frames_rejected(ctx):
    from photonpy_b200 import spotdetect
    from photonpy_b200.lib import last_error
    sd = spotdetect.SpotDetector(1.5, 9, 6.0)
    q, rq = spotdetect.SpotDetectionMethods(ctx).CreateQueue((32, 32), [9, 9], sd)
    q.PushFrameF32(np.zeros((32, 32), np.float32))
    assert "16-bit" in last_error()
    assert q.IsIdle() and len(rq) == 0
    q.Destroy()
    from photonpy_b200 import lib
    lib.clear_error()


def test_detect_spots_file_and_localize(ctx, tmp_path):
    """process_movie: frames -> ROI file (photonpy's format) -> EstimQueue fit; the file holds the
    oracle's ROIs, and the fitted positions land on the planted spots."""
    import photonpy_b200 as pb
    from photonpy_b200 import process_movie as pm
    from photonpy_b200 import spotdetect
    d = synth.frames(12, h=128, w=128, spots_per_frame=12, seed=13, I=(1500, 3000), margin=8)
    frames = d["frames"].astype(np.uint16)
    sd = spotdetect.SpotDetector(1.5, 9, 6.0)
    fn = str(tmp_path / "movie.rois")
    nrois, nframes = pm.detect_spots(sd, None, iter(frames), 1, fn, 20, ctx)
    assert nframes == 12
    info, px = pm.load_rois(fn)
    assert len(info) == nrois
    oinfo, orois = O.spot_extraction_queue(frames, *_sizes(1.5), 9, 6.0, sumframes=1)
    a_i, a_p = _sorted(info, px.reshape(-1, 1, 9, 9))
    b_i, b_p = _sorted(oinfo, orois)
    assert np.array_equal(a_i, b_i) and np.array_equal(a_p, b_p)
    psf = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(9, 1.5, True)
    r = pm.localize_rois(fn, psf)
    assert len(r.estim) == nrois and np.array_equal(r.ids, info["id"])
    x = r.estim[:, 0] + info["x"]
    y = r.estim[:, 1] + info["y"]
    t = d["truth"]
    hits = 0
    for f in range(12):
        tf = t[t[:, 0] == f]
        sel = info["id"] == f
        dd = np.hypot(x[sel][:, None] - tf[None, :, 1], y[sel][:, None] - tf[None, :, 2])
        hits += int(np.sum(dd.min(axis=0) < 0.3))
    assert hits >= 0.8 * len(t)
    psf.Destroy()
