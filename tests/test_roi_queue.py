"""ROI queue (RQ_*), camera-calibration objects and the ROI file format on the host (no GPU).

RQ_* and the calibration factories are host code, so the library is exercised here without a
GPU; where the reference library is built (oracle/_ref) its RQ_* run side by side and must give
the same records in the same order: the `count` oldest ROIs, newest first, and nothing at all
when fewer than `count` are queued (ROIQueue.cpp:33-52)."""
import ctypes as ct

import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref_lib

INFO = np.dtype([("id", "<i4"), ("score", "<f4"), ("x", "<i4"), ("y", "<i4"), ("z", "<i4")])


def _rq_ops(L, shape):
    vp = ct.c_void_p
    L.RQ_Create.argtypes = [vp, vp]
    L.RQ_Create.restype = vp
    L.RQ_Push.argtypes = [vp, ct.c_int, vp, vp]
    L.RQ_Pop.argtypes = [vp, ct.c_int, vp, vp]
    L.RQ_Length.argtypes = [vp]
    L.RQ_Length.restype = ct.c_int
    L.RQ_SmpShape.argtypes = [vp, vp]
    L.RQ_Delete.argtypes = [vp]
    s = np.array(shape, np.int32)
    q = L.RQ_Create(s.ctypes.data, None)
    assert q
    return q


def _script(L):
    rng = np.random.default_rng(3)
    shape = (2, 3, 4)
    q = _rq_ops(L, shape)
    smp = int(np.prod(shape))
    out = []
    pushed = 0
    for batch in (5, 1, 7):
        info = np.zeros(batch, INFO)
        info["id"] = np.arange(pushed, pushed + batch)
        info["score"] = rng.uniform(size=batch)
        info["x"], info["y"], info["z"] = 10 + info["id"], 20 + info["id"], 0
        data = rng.normal(size=(batch, smp)).astype(np.float32)
        L.RQ_Push(q, batch, info.ctypes.data, data.ctypes.data)
        pushed += batch
    out.append(L.RQ_Length(q))
    for cnt in (4, 20, 8):  # 20 > length: nothing written
        info = np.zeros(cnt, INFO)
        data = np.zeros((cnt, smp), np.float32)
        L.RQ_Pop(q, cnt, info.ctypes.data, data.ctypes.data)
        out.append((info.copy(), data.copy(), L.RQ_Length(q)))
    sh = np.zeros(3, np.int32)
    L.RQ_SmpShape(q, sh.ctypes.data)
    L.RQ_Delete(q)
    return out, sh


def test_roi_queue_semantics():
    from photonpy_b200.lib import load_library
    out, sh = _script(load_library())
    assert out[0] == 13
    info, data, left = out[1]
    assert list(info["id"]) == [3, 2, 1, 0] and left == 9  # oldest four, newest first
    info, data, left = out[2]
    assert not any(info.tobytes()) and not data.any() and left == 9
    info, data, left = out[3]
    assert list(info["id"]) == [11, 10, 9, 8, 7, 6, 5, 4] and left == 1
    assert list(sh) == [2, 3, 4]


@pytest.mark.skipif(not ref_lib.available(), reason="reference build absent")
def test_roi_queue_equals_reference():
    from photonpy_b200.lib import load_library
    ours, sh = _script(load_library())
    ref, rsh = _script(ref_lib.lib())
    assert ours[0] == ref[0]
    for a, b in zip(ours[1:], ref[1:]):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    assert np.array_equal(sh, rsh)


def test_calibration_objects_and_context_ownership():
    import photonpy_b200 as pb
    from photonpy_b200.calib import GainOffset_Calib, GainOffsetImage_Calib, sCMOS_Calib
    from photonpy_b200.roi_queue import ROIQueue
    with pb.Context() as ctx:
        a = GainOffset_Calib(0.5, 100.0, ctx)
        b = GainOffsetImage_Calib(np.ones((8, 9)), np.zeros((8, 9)), ctx)
        c = sCMOS_Calib(ctx, np.zeros((8, 9)), np.ones((8, 9)), np.ones((8, 9)))
        q = ROIQueue([1, 7, 7], ctx)
        q.Push(np.ones((3, 7, 7)), id=np.arange(3))
        assert a.inst and b.inst and c.inst and len(q) == 3
        info, data = q.Fetch()
        assert list(info["id"]) == [2, 1, 0] and data.shape == (3, 7, 7)
    # the context destroyed the calibrations and the queue


def test_oracle_calibration_arithmetic():
    raw = np.array([[0, 99, 100, 101, 65535]], np.uint16)
    v = O.camera_calibrate(raw, "gain_offset", 0.5, 100.0)
    assert v.dtype == np.float32
    assert list(v[0]) == [0.0, 0.0, 0.0, 0.5, np.float32((65535.0 - 100.0) * 0.5)]
    s = O.camera_calibrate(raw, "scmos", np.full(raw.shape, 2.0), np.full(raw.shape, 100.0))
    assert list(s[0][:3]) == [-200.0, -2.0, 0.0]


def test_rois_file_format_roundtrip(tmp_path):
    """photonpy's ROI file: pairs of numpy.save arrays; maxrois cuts inside a batch."""
    from photonpy_b200 import process_movie as pm
    fn = str(tmp_path / "r.rois")
    batches = []
    with open(fn, "wb") as f:
        for b, n in enumerate((4, 3, 5)):
            info = np.zeros(n, INFO)
            info["id"] = b
            px = np.full((n, 5, 5), b, np.float32)
            np.save(f, info, allow_pickle=False)
            np.save(f, px, allow_pickle=False)
            batches.append((info, px))
    info, px = pm.load_rois(fn)
    assert len(info) == 12 and px.shape == (12, 5, 5)
    info, px = pm.load_rois(fn, maxrois=6)
    assert len(info) == 6 and list(info["id"]) == [0, 0, 0, 0, 1, 1]
    assert [len(i) for i, _ in pm.load_rois_iterator(fn, maxrois=7)] == [4, 3]
