"""Spot detection and ROI extraction — counterpart of photonpy/cpp/spotdetect.py.

``SpotDetector`` is the same ctypes structure (filter sizes derived from the PSF sigma as
photonpy does), ``SpotDetectionMethods.ProcessFrame`` / ``ExtractROIs`` call the C ABI with the
reference's signatures, and ``SpotDetectionMethods.DetectDevice`` runs the detector on a batch
of frames already on the GPU (torch tensors) and returns ROIs on the GPU, ready for
``Estimator.EstimateDevice``. ``localize_frames`` chains the two: frames in, localizations out,
with nothing but the frames crossing PCIe.

``CreateQueue`` builds photonpy's spot-extraction queue (16-bit frames in, ROIs of summed
frames out through a ``ROIQueue``), run in GPU batches. Not provided: the PSF-correlation
detector.
"""
from __future__ import annotations

import ctypes

import numpy as np
import numpy.ctypeslib as ctl

from .lib import check_error


class SpotDetectorNativeFactory:
    def __init__(self, inst, destructor):
        self.inst = inst
        self.destructor = destructor

    def __enter__(self):
        return self

    def __exit__(self, *args):
        self.destructor(self.inst)


class SpotDetector(ctypes.Structure):
    """photonpy/cpp/spotdetect.py:26-69. detectionImage = uniform1 - uniform2; spots where
    max(detectionImage, maxFilterSize) == detectionImage."""
    _fields_ = [
        ("uniformFilter1Size", ctypes.c_int32),
        ("uniformFilter2Size", ctypes.c_int32),
        ("maxFilterSize", ctypes.c_int32),
        ("roisize", ctypes.c_int32),
        ("minIntensity", ctypes.c_float),
        ("maxIntensity", ctypes.c_float),
        ("backgroundImagePtr", ctypes.c_void_p),
    ]

    def __init__(self, psfSigma, roisize, minIntensity=7, maxIntensity=np.inf, backgroundImage=None):
        psfSigma = np.mean(psfSigma)
        self.uniformFilter1Size = int(psfSigma * 2 + 2)
        self.uniformFilter2Size = self.uniformFilter1Size * 2
        self.maxFilterSize = int(psfSigma * 5)
        self.roisize = roisize
        self.minIntensity = minIntensity
        self.maxIntensity = maxIntensity
        self.backgroundImage_ = None
        if backgroundImage is not None:
            self.backgroundImage_ = np.ascontiguousarray(backgroundImage, dtype=np.float32)
            self.backgroundImagePtr = self.backgroundImage_.ctypes.data
        else:
            self.backgroundImagePtr = 0

    def print(self):
        print("Spot detector config: \n" +
              f"uniform filter 1: {self.uniformFilter1Size}\n"
              f"uniform filter 2: {self.uniformFilter2Size}\n"
              f"maxfilter: {self.maxFilterSize}\n"
              f"min intensity: {self.minIntensity}\n"
              f"max intensity: {self.maxIntensity}\n")

    def CreateNativeFactory(self, ctx):
        m = SpotDetectionMethods(ctx)
        inst = m._SpotDetector_Configure(self)
        if not inst:
            check_error("SpotDetector_Configure")
        return SpotDetectorNativeFactory(inst, m._SpotDetector_DestroyFactory)

    def _key(self):
        return (self.uniformFilter1Size, self.uniformFilter2Size, self.maxFilterSize, self.roisize,
                float(self.minIntensity), float(self.maxIntensity), self.backgroundImagePtr or 0)

    def _cached_factory(self, methods):
        """Native factory kept with this detector for repeated device calls (its device scratch
        then stays allocated); rebuilt when a field changes."""
        key = self._key()
        cached = self.__dict__.get("_native")
        if cached is not None and cached[0] == key:
            return cached[1]
        self._release_native()
        inst = methods._SpotDetector_Configure(self)
        if not inst:
            check_error("SpotDetector_Configure")
        self._native = (key, inst, methods._SpotDetector_DestroyFactory)
        return inst

    def _release_native(self):
        cached = self.__dict__.pop("_native", None)
        if cached is not None:
            cached[2](cached[1])

    def __del__(self):
        try:
            self._release_native()
        except Exception:
            pass


class SpotDetectionMethods:
    def __init__(self, ctx):
        self.ctx = ctx
        lib = ctx.smlm.lib
        vp = ctypes.c_void_p
        self._SpotDetector_Configure = lib.SpotDetector_Configure
        self._SpotDetector_Configure.argtypes = [ctypes.POINTER(SpotDetector)]
        self._SpotDetector_Configure.restype = vp
        self._SpotDetector_DestroyFactory = lib.SpotDetector_DestroyFactory
        self._SpotDetector_DestroyFactory.argtypes = [vp]
        self._SpotDetector_ProcessFrame = lib.SpotDetector_ProcessFrame
        self._SpotDetector_ProcessFrame.argtypes = [
            ctl.ndpointer(np.float32, flags="aligned, c_contiguous"),  # frame
            ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,  # width, height, roisize, maxspots
            ctl.ndpointer(np.float32, flags="aligned, c_contiguous"),  # spot scores
            ctl.ndpointer(np.int32, flags="aligned, c_contiguous"),  # spot z
            ctl.ndpointer(np.int32, flags="aligned, c_contiguous"),  # corner positions
            ctl.ndpointer(np.float32, flags="aligned, c_contiguous"),  # rois
            vp, vp]
        self._SpotDetector_ProcessFrame.restype = ctypes.c_int32
        self._ExtractROIs = lib.ExtractROIs
        self._ExtractROIs.argtypes = [
            ctl.ndpointer(np.float32, flags="aligned, c_contiguous"),
            ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
            ctl.ndpointer(np.int32, flags="aligned, c_contiguous"), ctypes.c_int32,
            ctl.ndpointer(np.float32, flags="aligned, c_contiguous")]
        self._SpotExtractionQueue_Create = lib.SpotExtractionQueue_Create
        self._SpotExtractionQueue_Create.argtypes = [ctypes.c_int32, ctypes.c_int32, vp, vp, vp, ctypes.c_int32,
                                                     ctypes.c_int32, vp]
        self._SpotExtractionQueue_Create.restype = vp
        self._DetectDevice = lib.PB200_DetectSpotsDevice
        self._DetectDevice.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, vp, vp, vp, vp, vp]
        self._DetectDevice.restype = ctypes.c_int

    def ExtractROIs(self, frames, roishape, cornerPosZYX):
        """photonpy/cpp/spotdetect.py:209-222."""
        assert len(frames.shape) == 3
        assert cornerPosZYX.shape[1] == 3
        numspots = len(cornerPosZYX)
        cornerPosZYX = np.ascontiguousarray(cornerPosZYX, dtype=np.int32)
        frames = np.ascontiguousarray(frames, dtype=np.float32)
        rois = np.zeros((numspots, *roishape), dtype=np.float32)
        self._ExtractROIs(frames, frames.shape[2], frames.shape[1], frames.shape[0], roishape[2], roishape[1],
                          roishape[0], cornerPosZYX, numspots, rois)
        check_error("ExtractROIs")
        return rois

    def CreateQueue(self, imgshape, roishape, spotDetectorType, calib=None, sumframes=1, numThreads=3, ctx=None):
        """photonpy/cpp/spotdetect.py:178-203: a spot-detection queue. Returns (input_queue,
        output_queue): an ImageProcessor taking 16-bit frames and the ROIQueue of
        [sumframes, *roishape] ROIs it fills."""
        from .image_proc import ImageProcessor
        from .roi_queue import ROIQueue
        if ctx is None:
            ctx = self.ctx
        rq = ROIQueue([sumframes, *roishape], ctx)
        with spotDetectorType.CreateNativeFactory(self.ctx) as sdf:
            inst = self._SpotExtractionQueue_Create(imgshape[1], imgshape[0], rq.inst, sdf.inst,
                                                    calib.inst if calib else None, numThreads, sumframes,
                                                    ctx.inst if ctx else None)
        if not inst:
            check_error("SpotExtractionQueue_Create")
        return ImageProcessor(imgshape, inst, self.ctx), rq

    def ProcessFrame(self, image, spotDetector, roisize, maxSpotsPerFrame, calib=None):
        """photonpy/cpp/spotdetect.py:224-245: returns (rois, cornerYX, scores, spotz). With a
        camera calibration the detector sees the calibrated frame; the ROIs hold the frame as
        given."""
        assert len(image.shape) == 2
        h, w = image.shape
        image = np.ascontiguousarray(image, dtype=np.float32)
        scores = np.zeros(maxSpotsPerFrame, dtype=np.float32)
        rois = np.zeros((maxSpotsPerFrame, roisize, roisize), dtype=np.float32)
        cornerYX = np.zeros((maxSpotsPerFrame, 2), dtype=np.int32)
        spotz = np.zeros(maxSpotsPerFrame, dtype=np.int32)
        with spotDetector.CreateNativeFactory(self.ctx) as sdf:
            numspots = self._SpotDetector_ProcessFrame(image, w, h, roisize, maxSpotsPerFrame, scores, spotz, cornerYX,
                                                       rois, sdf.inst, calib.inst if calib else None)
        check_error("SpotDetector_ProcessFrame")
        return rois[:numspots], cornerYX[:numspots], scores[:numspots], spotz[:numspots]

    def DetectDevice(self, frames, spotDetector, roisize, maxSpotsPerFrame, background=None, stream=None):
        """Detect spots in a batch of frames on the GPU. frames: torch float32 CUDA tensor
        [n, h, w] (or [h, w]). Returns torch tensors on the device:
        (rois [m, roisize, roisize], cornerYX [m, 2], frame index [m], scores [m], found [n]),
        spots in frame order, then row-major pixel order within a frame; at most
        maxSpotsPerFrame per frame."""
        import torch
        if frames.dim() == 2:
            frames = frames[None]
        assert frames.is_cuda and frames.dtype == torch.float32
        frames = frames.contiguous()
        n, h, w = frames.shape
        dev = frames.device
        K = int(maxSpotsPerFrame)
        found = torch.empty(n, dtype=torch.int32, device=dev)
        corner = torch.empty((n, K, 2), dtype=torch.int32, device=dev)
        scores = torch.empty((n, K), dtype=torch.float32, device=dev)
        rois = torch.empty((n, K, roisize, roisize), dtype=torch.float32, device=dev)
        bg = None
        if background is None:
            background = spotDetector.backgroundImage_
        if background is not None:
            bg = torch.as_tensor(background, dtype=torch.float32, device=dev).contiguous()
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        inst = spotDetector._cached_factory(self)
        rc = self._DetectDevice(inst, frames.data_ptr(), None if bg is None else bg.data_ptr(), n, w, h,
                                int(roisize), K, found.data_ptr(), corner.data_ptr(), scores.data_ptr(),
                                rois.data_ptr(), ctypes.c_void_p(s.cuda_stream))
        if rc != 0:
            check_error("DetectSpotsDevice")
        counts = torch.clamp(found, max=K)
        keep = torch.arange(K, device=dev)[None, :] < counts[:, None].to(torch.int64)
        frame_idx = torch.arange(n, device=dev)[:, None].expand(n, K)
        return rois[keep], corner[keep], frame_idx[keep], scores[keep], found


def localize_frames(frames, spotDetector, estimator, roisize, maxSpotsPerFrame=1000, background=None):
    """Frames (torch CUDA [n, h, w]) -> spot detection -> fused fit + CRLB on the GPU.
    Returns a dict of torch tensors: params [m, K] in frame pixel coordinates (x, y shifted
    by the ROI corner), crlb, iterations, chisq, frame [m], score [m]."""
    import torch
    sm = SpotDetectionMethods(estimator.ctx)
    rois, corner, frame_idx, scores, _ = sm.DetectDevice(frames, spotDetector, roisize, maxSpotsPerFrame,
                                                         background=background)
    out = estimator.EstimateDevice(rois.contiguous(), with_crlb=True)
    params = out["params"].clone()
    params[:, 0] += corner[:, 1].to(torch.float32)
    params[:, 1] += corner[:, 0].to(torch.float32)
    return dict(params=params, crlb=out["crlb"], iterations=out["iterations"], chisq=out["chisq"],
                frame=frame_idx, score=scores, roi_params=out["params"])
