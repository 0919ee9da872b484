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


class ROIExtractor(ImageProcessor):
    """photonpy/cpp/image_proc.py ROIExtractor: boxes of predefined ROIs cut from a stream of
    16-bit frames. rois: ROIType records (cornerpos = (x, y), startframe, numframes)."""

    ROIType = np.dtype([("cornerpos", "<i4", 2), ("startframe", "<i4"), ("numframes", "<i4")])

    def __init__(self, imgshape, rois, roiframes, roisize, calib, ctx: Context):
        lib = ctx.lib
        create = lib.ROIExtractor_Create
        create.argtypes = [ct.c_int32, ct.c_int32, ctl.ndpointer(ROIExtractor.ROIType, flags="aligned, c_contiguous"),
                           ct.c_int32, ct.c_int32, ct.c_int32, ct.c_void_p, ct.c_void_p]
        create.restype = ct.c_void_p
        self._GetResultCount = lib.ROIExtractor_GetResultCount
        self._GetResultCount.argtypes = [ct.c_void_p]
        self._GetResultCount.restype = ct.c_int32
        self._GetResults = lib.ROIExtractor_GetResults
        self._GetResults.argtypes = [ct.c_void_p, ct.c_int32,
                                     ctl.ndpointer(ROIExtractor.ROIType, flags="aligned, c_contiguous"),
                                     ctl.ndpointer(np.float32, flags="aligned, c_contiguous")]
        self._GetResults.restype = ct.c_int32
        rois = np.ascontiguousarray(rois, dtype=ROIExtractor.ROIType)
        inst = create(imgshape[1], imgshape[0], rois, len(rois), roiframes, roisize,
                      calib.inst if calib else None, ctx.inst)
        check_instance(inst, "ROIExtractor_Create")
        self.roiframes = roiframes
        self.roisize = roisize
        super().__init__(imgshape, inst, ctx)

    def GetResultCount(self):
        return self._GetResultCount(self.inst)

    def GetResults(self, numrois):
        rois = np.zeros(numrois, dtype=ROIExtractor.ROIType)
        framedata = np.zeros((numrois, self.roiframes, self.roisize, self.roisize), dtype=np.float32)
        count = self._GetResults(self.inst, numrois, rois, framedata)
        return rois[:count], framedata[:count]


def check_instance(inst, what):
    if not inst:
        check_error(what)
    return inst
