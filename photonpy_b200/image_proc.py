"""Frame processors — counterpart of photonpy/cpp/image_proc.py (ImgProc_* of
ImageProcessor.cpp:12-51).

``ImageProcessor`` wraps the instance ``SpotDetectionMethods.CreateQueue`` returns (the
spot-extraction queue): frames go in with ``PushFrameU16``; ``NumFinishedFrames`` counts the
(summed) frames done and ``IsIdle`` tells when every pushed frame has been processed.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import numpy.ctypeslib as ctl

from .context import Context
from .lib import check_error


class ImageProcessor:
    def __init__(self, imgshape, inst, ctx: Context):
        self.frameCounter = 0
        self.ctx = ctx
        vp = ct.c_void_p
        lib = ctx.lib
        self._ImgProc_NumFinishedFrames = lib.ImgProc_NumFinishedFrames
        self._ImgProc_NumFinishedFrames.argtypes = [vp]
        self._ImgProc_AddFrameU16 = lib.ImgProc_AddFrameU16
        self._ImgProc_AddFrameU16.argtypes = [vp, ctl.ndpointer(np.uint16, flags="aligned, c_contiguous")]
        self._ImgProc_AddFrameF32 = lib.ImgProc_AddFrameF32
        self._ImgProc_AddFrameF32.argtypes = [vp, ctl.ndpointer(np.float32, flags="aligned, c_contiguous")]
        self._ImgProc_ReadFrame = lib.ImgProc_ReadFrame
        self._ImgProc_ReadFrame.argtypes = [vp, ctl.ndpointer(np.float32, flags="aligned, c_contiguous"),
                                            ctl.ndpointer(np.float32, flags="aligned, c_contiguous")]
        self._ImgProc_GetQueueLength = lib.ImgProc_GetQueueLength
        self._ImgProc_GetQueueLength.argtypes = [vp]
        self._ImgProc_IsIdle = lib.ImgProc_IsIdle
        self._ImgProc_IsIdle.argtypes = [vp]
        self._ImgProc_IsIdle.restype = ct.c_bool
        self._ImgProc_Destroy = lib.ImgProc_Destroy
        self._ImgProc_Destroy.argtypes = [vp]
        self.imgshape = imgshape
        self.inst = inst

    def PushFrameU16(self, img):
        assert np.array_equal(img.shape, self.imgshape)
        self._ImgProc_AddFrameU16(self.inst, np.ascontiguousarray(img, dtype=np.uint16))

    def PushFrameF32(self, img):
        assert np.array_equal(img.shape, self.imgshape)
        self._ImgProc_AddFrameF32(self.inst, np.ascontiguousarray(img, dtype=np.float32))

    def GetQueueLength(self):
        return self._ImgProc_GetQueueLength(self.inst)

    def NumFinishedFrames(self):
        return self._ImgProc_NumFinishedFrames(self.inst)

    def ReadResultFrame(self):
        filtered = np.empty(self.imgshape, dtype=np.float32)
        img = np.empty(self.imgshape, dtype=np.float32)
        num = self._ImgProc_ReadFrame(self.inst, img, filtered)
        if num > 0:
            return img, filtered
        return None

    def IsIdle(self):
        return self._ImgProc_IsIdle(self.inst)

    def Destroy(self):
        """Stops the processor (frames not yet processed are dropped); the reference leaves
        this to the context."""
        if self.inst:
            self._ImgProc_Destroy(self.inst)
            self.inst = None


def check_instance(inst, what):
    if not inst:
        check_error(what)
    return inst
