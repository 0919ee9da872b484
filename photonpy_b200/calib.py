"""Camera calibration objects — counterpart of photonpy/cpp/calib.py.

Each object is owned by its context (destroyed with it) and is passed as ``calib`` to
``SpotDetectionMethods.ProcessFrame`` and ``SpotDetectionMethods.CreateQueue``. The transforms
(CameraCalibration.cu:19-57): gain/offset ``max(0, (x - offset) * gain)``, per pixel the same
with images, sCMOS ``(x - offset) * gain`` per pixel (see the integration notes for how this
differs from photonpy's sCMOS transform).
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import numpy.ctypeslib as ctl

from .lib import check_error


class sCMOS_Calib:
    def __init__(self, ctx, offset, gain, variance):
        fn = ctx.lib.sCMOS_Calib_Create
        fn.argtypes = [ct.c_int32, ct.c_int32, ctl.ndpointer(np.float32, flags="aligned, c_contiguous"),
                       ctl.ndpointer(np.float32, flags="aligned, c_contiguous"),
                       ctl.ndpointer(np.float32, flags="aligned, c_contiguous"), ct.c_void_p]
        fn.restype = ct.c_void_p
        offset = np.ascontiguousarray(offset, dtype=np.float32)
        gain = np.ascontiguousarray(gain, dtype=np.float32)
        variance = np.ascontiguousarray(variance, dtype=np.float32)
        assert len(offset.shape) == 2
        assert np.array_equal(offset.shape, gain.shape)
        assert np.array_equal(offset.shape, variance.shape)
        self.inst = fn(offset.shape[1], offset.shape[0], offset, gain, variance, ctx.inst)
        if not self.inst:
            check_error("sCMOS_Calib_Create")


class GainOffset_Calib:
    """Constant global gain/offset."""

    def __init__(self, gain, offset, ctx):
        fn = ctx.lib.GainOffsetCalib_Create
        fn.argtypes = [ct.c_float, ct.c_float, ct.c_void_p]
        fn.restype = ct.c_void_p
        self.inst = fn(gain, offset, ctx.inst)
        if not self.inst:
            check_error("GainOffsetCalib_Create")


class GainOffsetImage_Calib:
    """Gain/offset given per pixel as images."""

    def __init__(self, gain, offset, ctx):
        fn = ctx.lib.GainOffsetImageCalib_Create
        fn.argtypes = [ct.c_int32, ct.c_int32, ctl.ndpointer(np.float32, flags="aligned, c_contiguous"),
                       ctl.ndpointer(np.float32, flags="aligned, c_contiguous"), ct.c_void_p]
        fn.restype = ct.c_void_p
        gain = np.ascontiguousarray(gain, dtype=np.float32)
        offset = np.ascontiguousarray(offset, dtype=np.float32)
        assert np.array_equal(gain.shape, offset.shape)
        self.inst = fn(gain.shape[1], gain.shape[0], gain, offset, ctx.inst)
        if not self.inst:
            check_error("GainOffsetImageCalib_Create")
