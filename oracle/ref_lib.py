"""Minimal ctypes binding of the reference photonpy library built by oracle/build_ref.sh.

TEST INFRASTRUCTURE ONLY: used to generate golden vectors, by parity tests when the
reference build is present, and by bench.py's reference (CPU baseline) arm. It calls
the reference's unmodified C ABI (cpp/SMLMLib/Estimators/Estimator.h:157-171,
Estimators/Gaussian/GaussianPSF.h:35-41, Estimators/CSpline/CubicSplinePSF.h:33-40) the
same way photonpy/cpp/estimator.py does; all arithmetic happens inside the reference.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libphotonpy_ref.so")

_lib = None


def available() -> bool:
    return os.path.exists(REF_LIB)


class Gauss3DCalib(ct.Structure):
    _fields_ = [("x", ct.c_float * 4), ("y", ct.c_float * 4), ("zrange", ct.c_float * 2)]


class CSplineCalib(ct.Structure):
    _fields_ = [("shape", ct.c_int32 * 3), ("z_min", ct.c_float), ("z_max", ct.c_float), ("coefs", ct.c_void_p)]


class Props(ct.Structure):
    _fields_ = [("numParams", ct.c_int), ("sampleCount", ct.c_int), ("numDiag", ct.c_int), ("numConst", ct.c_int),
                ("sampleIndexDims", ct.c_int)]


class LMParams(ct.Structure):
    _fields_ = [("iterations", ct.c_int32), ("lambda_", ct.c_float), ("factor", ct.c_float)]


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{REF_LIB} not built (run oracle/build_ref.sh)")
        L = ct.CDLL(REF_LIB)
        vp = ct.c_void_p
        L.Context_Create.restype = vp
        L.Context_Destroy.argtypes = [vp]
        for name, args in [
            ("Gauss2D_CreatePSF_XYIBg", [ct.c_int, ct.c_float, ct.c_float, ct.c_bool, vp]),
            ("Gauss2D_CreatePSF_XYIBgConstSigma", [ct.c_int, ct.c_bool, vp]),
            ("Gauss2D_CreatePSF_XYIBgSigma", [ct.c_int, ct.c_float, ct.c_bool, vp]),
            ("Gauss2D_CreatePSF_XYIBgSigmaXY", [ct.c_int, ct.c_float, ct.c_float, ct.c_bool, vp]),
            ("Gauss2D_CreatePSF_XYZIBg", [ct.c_int, ct.POINTER(Gauss3DCalib), ct.c_bool, vp]),
            ("CSpline_CreatePSF", [ct.c_int, ct.POINTER(CSplineCalib), vp, ct.c_int, ct.c_bool, vp]),
            ("Gauss2D_CreatePSF_XYITiltedBg", [ct.c_int, ct.c_bool, vp]),
            ("Gauss2D_CreatePSF_XYITiltedBgSigmaXY", [ct.c_int, ct.c_float, ct.c_float, ct.c_bool, vp]),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = vp
        L.Estimator_Delete.argtypes = [vp]
        L.Estimator_GetProperties.argtypes = [vp, ct.POINTER(Props)]
        L.Estimator_SetLMParams.argtypes = [vp, ct.POINTER(LMParams)]
        L.Estimator_Estimate.argtypes = [vp, ct.c_int, vp, vp, vp, vp, vp, vp, vp, vp, ct.c_int]
        L.Estimator_ChiSquareAndCRLB.argtypes = [vp, vp, vp, vp, vp, ct.c_int, vp, vp]
        L.Estimator_ComputeDerivatives.argtypes = [vp, ct.c_int, vp, vp, vp, vp, vp]
        L.Estimator_ComputeExpectedValue.argtypes = [vp, ct.c_int, vp, vp, vp, vp]
        L.CSpline_Compute.argtypes = [vp, vp, vp, ct.c_int]
        L.Gauss2D_EstimateIntensityBg.argtypes = [vp, vp, vp, ct.c_int, vp, vp, vp, ct.c_int, ct.c_int, ct.c_bool]
        L.Gauss2D_EstimateIntensityBg.restype = None
        if hasattr(L, "GLRT_CreatePSF"):
            L.GLRT_CreatePSF.argtypes = [vp, vp]
            L.GLRT_CreatePSF.restype = vp
        if hasattr(L, "SpotDetector_Configure"):
            L.SpotDetector_Configure.argtypes = [ct.POINTER(SpotDetectorConfig)]
            L.SpotDetector_Configure.restype = vp
            L.SpotDetector_DestroyFactory.argtypes = [vp]
            L.SpotDetector_ProcessFrame.argtypes = [vp, ct.c_int, ct.c_int, ct.c_int, ct.c_int, vp, vp, vp, vp, vp, vp]
            L.SpotDetector_ProcessFrame.restype = ct.c_int
            L.ExtractROIs.argtypes = [vp, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int, vp, ct.c_int, vp]
        if hasattr(L, "EstimQueue_Create"):
            L.EstimQueue_Create.argtypes = [vp, ct.c_int, ct.c_int, ct.c_bool, ct.c_int, vp]
            L.EstimQueue_Create.restype = vp
            L.EstimQueue_Delete.argtypes = [vp]
            L.EstimQueue_Schedule.argtypes = [vp, ct.c_int, vp, vp, vp, vp, vp]
            L.EstimQueue_Flush.argtypes = [vp]
            L.EstimQueue_IsIdle.argtypes = [vp]
            L.EstimQueue_IsIdle.restype = ct.c_bool
            L.EstimQueue_GetResultCount.argtypes = [vp]
            L.EstimQueue_GetResultCount.restype = ct.c_int
            L.EstimQueue_GetResults.argtypes = [vp, ct.c_int, vp, vp, vp, vp, vp, vp]
            L.EstimQueue_GetResults.restype = ct.c_int
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


class SpotDetectorConfig(ct.Structure):
    """SpotDetectorConfig (SpotDetection/SpotDetector.h:39-62), as photonpy/cpp/spotdetect.py lays it out."""
    _fields_ = [("uniformFilter1Size", ct.c_int32), ("uniformFilter2Size", ct.c_int32), ("maxFilterSize", ct.c_int32),
                ("roisize", ct.c_int32), ("minIntensity", ct.c_float), ("maxIntensity", ct.c_float),
                ("backgroundImagePtr", ct.c_void_p)]


def process_frame(frame, u1, u2, maxfilter, roisize, min_intensity, max_intensity=np.inf, background=None,
                  max_spots=10000):
    """The reference's SpotDetector_ProcessFrame (its CUDA detector; needs a GPU): returns
    (count, scores, spotz, corner [n, 2] (y, x), rois [n, roisize, roisize])."""
    L = lib()
    frame = np.ascontiguousarray(frame, dtype=np.float32)
    h, w = frame.shape
    cfg = SpotDetectorConfig(int(u1), int(u2), int(maxfilter), int(roisize), float(min_intensity),
                             float(max_intensity), None)
    bg = None
    if background is not None:
        bg = np.ascontiguousarray(background, dtype=np.float32)
        cfg.backgroundImagePtr = bg.ctypes.data
    sdf = L.SpotDetector_Configure(ct.byref(cfg))
    scores = np.zeros(max_spots, np.float32)
    spotz = np.zeros(max_spots, np.int32)
    corner = np.zeros((max_spots, 2), np.int32)
    rois = np.zeros((max_spots, roisize, roisize), np.float32)
    n = L.SpotDetector_ProcessFrame(_p(frame), w, h, int(roisize), int(max_spots), _p(scores), _p(spotz), _p(corner),
                                    _p(rois), sdf, None)
    L.SpotDetector_DestroyFactory(sdf)
    return n, scores[:n], spotz[:n], corner[:n], rois[:n]


class RefEstimator:
    """One reference estimator instance (host pointers; cuda selects the reference's GPU kernels)."""

    def __init__(self, kind: str, roisize: int, cuda: bool = False, sigma=(1.5, 1.5), astig=None, zrange=(-1, 1),
                 coefs=None, spline_zrange=(0, 1), spline_mode=0):
        L = lib()
        self.ctx = L.Context_Create()
        self.roisize = roisize
        if kind == "XYIBg":
            inst = L.Gauss2D_CreatePSF_XYIBg(roisize, sigma[0], sigma[1], cuda, self.ctx)
        elif kind == "XYIBgConstSigma":
            inst = L.Gauss2D_CreatePSF_XYIBgConstSigma(roisize, cuda, self.ctx)
        elif kind == "XYIBgSigma":
            inst = L.Gauss2D_CreatePSF_XYIBgSigma(roisize, sigma[0], cuda, self.ctx)
        elif kind == "XYIBgSigmaXY":
            inst = L.Gauss2D_CreatePSF_XYIBgSigmaXY(roisize, sigma[0], sigma[1], cuda, self.ctx)
        elif kind == "XYITiltedBg":
            inst = L.Gauss2D_CreatePSF_XYITiltedBg(roisize, cuda, self.ctx)
        elif kind == "XYITiltedBgSigmaXY":
            inst = L.Gauss2D_CreatePSF_XYITiltedBgSigmaXY(roisize, sigma[0], sigma[1], cuda, self.ctx)
        elif kind == "XYZIBg":
            c = Gauss3DCalib()
            for i in range(4):
                c.x[i] = astig[0][i]
                c.y[i] = astig[1][i]
            c.zrange[0], c.zrange[1] = zrange
            inst = L.Gauss2D_CreatePSF_XYZIBg(roisize, ct.byref(c), cuda, self.ctx)
        elif kind == "CSpline":
            self._coefs = np.ascontiguousarray(coefs, dtype=np.float32)
            c = CSplineCalib()
            c.shape[0], c.shape[1], c.shape[2] = self._coefs.shape[:3]
            c.z_min, c.z_max = spline_zrange
            c.coefs = self._coefs.ctypes.data
            inst = L.CSpline_CreatePSF(roisize, ct.byref(c), None, int(spline_mode), cuda, self.ctx)
        else:
            raise ValueError(kind)
        if not inst:
            raise RuntimeError(f"reference failed to create {kind}")
        self.inst = inst
        p = Props()
        L.Estimator_GetProperties(inst, ct.byref(p))
        self.K, self.numconst, self.numdiag = p.numParams, p.numConst, p.numDiag
        self.set_lm(50, 1e-18)

    def set_lm(self, iterations, lambda_):
        lmp = LMParams()
        lmp.iterations, lmp.lambda_, lmp.factor = iterations, lambda_, 0
        self.iterations = iterations
        lib().Estimator_SetLMParams(self.inst, ct.byref(lmp))

    def estimate(self, samples, constants=None, initial=None, trace_len=None):
        L = lib()
        samples = np.ascontiguousarray(samples, dtype=np.float32)
        n = samples.shape[0]
        tl = self.iterations if trace_len is None else trace_len
        params = np.zeros((n, self.K), np.float32)
        its = np.zeros(n, np.int32)
        diag = np.zeros((n, max(self.numdiag, 1)), np.float32)
        trace = np.zeros((n, max(tl, 1), self.K), np.float32)
        const = np.ascontiguousarray(constants if constants is not None else np.zeros((n, self.numconst)),
                                     dtype=np.float32)
        roipos = np.zeros((n, 2), np.int32)
        init = None if initial is None else np.ascontiguousarray(initial, dtype=np.float32)
        L.Estimator_Estimate(self.inst, n, _p(samples), _p(const), _p(roipos), _p(init), _p(params), _p(diag),
                             _p(its), _p(trace), tl)
        return params, its, trace

    def crlb_chisq(self, params, samples=None, constants=None):
        L = lib()
        params = np.ascontiguousarray(params, dtype=np.float32)
        n = params.shape[0]
        crlb = np.zeros((n, self.K), np.float32)
        chisq = np.zeros(n, np.float32)
        const = np.ascontiguousarray(constants if constants is not None else np.zeros((n, self.numconst)),
                                     dtype=np.float32)
        roipos = np.zeros((n, 2), np.int32)
        smp = None if samples is None else np.ascontiguousarray(samples, dtype=np.float32)
        L.Estimator_ChiSquareAndCRLB(self.inst, _p(params), _p(smp), _p(const), _p(roipos), n, _p(crlb),
                                     _p(chisq))
        return crlb, chisq

    def derivatives(self, params, constants=None):
        L = lib()
        params = np.ascontiguousarray(params, dtype=np.float32)
        n = params.shape[0]
        R = self.roisize
        ev = np.zeros((n, R, R), np.float32)
        deriv = np.zeros((n, self.K, R, R), np.float32)
        const = np.ascontiguousarray(constants if constants is not None else np.zeros((n, self.numconst)),
                                     dtype=np.float32)
        roipos = np.zeros((n, 2), np.int32)
        L.Estimator_ComputeDerivatives(self.inst, n, _p(params), _p(const), _p(roipos), _p(deriv), _p(ev))
        return deriv, ev

    def close(self):
        if self.inst:
            lib().Estimator_Delete(self.inst)
            self.inst = None
        if self.ctx:
            lib().Context_Destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefGLRT:
    """The reference's GLRT estimator (GLRT_CreatePSF, GLRT_PSF.cu:156) wrapping a CUDA RefEstimator."""

    def __init__(self, model: RefEstimator):
        self.model = model
        self.inst = lib().GLRT_CreatePSF(model.inst, model.ctx)
        if not self.inst:
            raise RuntimeError("reference GLRT_CreatePSF failed")
        self.K = model.K
        lmp = LMParams()
        lmp.iterations, lmp.lambda_, lmp.factor = model.iterations, 1e-18, 0
        lib().Estimator_SetLMParams(self.inst, ct.byref(lmp))

    def estimate(self, samples):
        """-> params [n][K], diag [n][3] = (ll_on, ll_off, mean)."""
        L = lib()
        samples = np.ascontiguousarray(samples, dtype=np.float32)
        n = samples.shape[0]
        params = np.zeros((n, self.K), np.float32)
        diag = np.zeros((n, 3), np.float32)
        its = np.zeros(n, np.int32)
        const = np.zeros((n, max(self.model.numconst, 1)), np.float32)
        roipos = np.zeros((n, 2), np.int32)
        trace = np.zeros((n, 1, self.K), np.float32)
        L.Estimator_Estimate(self.inst, n, _p(samples), _p(const), _p(roipos), None, _p(params), _p(diag), _p(its),
                             _p(trace), 1)
        return params, diag


EstimResultDType = np.dtype([("id", "<i4"), ("chisq", "<f4"), ("iterations", "<i4")])


class RefQueue:
    """The reference's EstimationQueue (EstimationQueue.cpp:317-420) over a CUDA RefEstimator."""

    def __init__(self, model: RefEstimator, batchSize=1024, maxQueueLen=5, numStreams=-1):
        self.model = model
        self.inst = lib().EstimQueue_Create(model.inst, batchSize, maxQueueLen, False, numStreams, None)
        if not self.inst:
            raise RuntimeError("reference EstimQueue_Create failed")

    def schedule(self, samples, ids):
        samples = np.ascontiguousarray(samples, dtype=np.float32)
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        n = samples.shape[0]
        const = np.zeros((n, max(self.model.numconst, 1)), np.float32)
        roipos = np.zeros((n, 2), np.int32)
        lib().EstimQueue_Schedule(self.inst, n, _p(ids), _p(samples), None, _p(const), _p(roipos))

    def wait(self, sleep=0.001):
        import time
        lib().EstimQueue_Flush(self.inst)
        while not lib().EstimQueue_IsIdle(self.inst):
            time.sleep(sleep)

    def results(self):
        """-> (estim [n][K], crlb [n][K], ids, chisq, iterations), whole batches in the queue's order."""
        L = lib()
        n = L.EstimQueue_GetResultCount(self.inst)
        K = self.model.K
        estim = np.zeros((n, K), np.float32)
        crlb = np.zeros((n, K), np.float32)
        roipos = np.zeros((n, 2), np.int32)
        res = np.zeros(n, EstimResultDType)
        got = L.EstimQueue_GetResults(self.inst, n, _p(estim), None, _p(crlb), _p(roipos), None, _p(res))
        return estim[:got], crlb[:got], res["id"][:got], res["chisq"][:got], res["iterations"][:got]

    def close(self):
        if self.inst:
            lib().EstimQueue_Delete(self.inst)
            self.inst = None


def estimate_intensity_bg(images, xy, sigma, max_iterations=100):
    """The reference's Gauss2D_EstimateIntensityBg (GaussianPSF.cu:216-240) on the CPU:
    images [n][w][w], xy [n][2], sigma as passed by photonpy's EstimateIBg ([n][2] floats, of
    which the reference reads the flat element i for spot i). Returns (IBg [n][2], crlb [n][2])."""
    L = lib()
    images = np.ascontiguousarray(images, dtype=np.float32)
    n, w = images.shape[0], images.shape[1]
    xy = np.ascontiguousarray(xy, dtype=np.float32)
    sigma = np.ascontiguousarray(sigma, dtype=np.float32)
    roipos = np.zeros((n, 2), np.int32)
    ibg = np.zeros((n, 2), np.float32)
    crlb = np.zeros((n, 2), np.float32)
    L.Gauss2D_EstimateIntensityBg(_p(images), _p(ibg), _p(crlb), n, _p(xy), _p(roipos), _p(sigma), w,
                                  int(max_iterations), False)
    return ibg, crlb


def spline_compute(data, border=0):
    L = lib()
    data = np.ascontiguousarray(data, dtype=np.float32)
    shape = np.ascontiguousarray(data.shape, dtype=np.int32)
    out = np.zeros((*(np.array(data.shape) - 3 + 2 * border), 64), np.float32)
    L.CSpline_Compute(_p(shape), _p(data), _p(out), int(border))
    return out


ROIInfoDType = np.dtype([("id", "<i4"), ("score", "<f4"), ("x", "<i4"), ("y", "<i4"), ("z", "<i4")])


def spot_queue(frames_u16, u1, u2, maxfilter, det_roisize, min_intensity, max_intensity=np.inf, sumframes=1,
               roisize=None, gain_offset=None, timeout=120.0):
    """The reference's spot-extraction queue (SpotExtractionQueue_Create, ImgFilterQueue.cu:346;
    its CUDA detector, so it needs a GPU): pushes the 16-bit frames, waits for the summed frames
    (bounded), pops every ROI. gain_offset: None or (gain, offset) for GainOffsetCalib_Create.
    Returns (info, rois [n, sumframes, roisize, roisize]) in the order RQ_Pop gives them."""
    import time
    L = lib()
    vp = ct.c_void_p
    frames = np.ascontiguousarray(frames_u16, dtype=np.uint16)
    n, h, w = frames.shape
    rs = int(roisize or det_roisize)
    L.RQ_Create.argtypes = [vp, vp]
    L.RQ_Create.restype = vp
    L.RQ_Length.argtypes = [vp]
    L.RQ_Length.restype = ct.c_int
    L.RQ_Pop.argtypes = [vp, ct.c_int, vp, vp]
    L.SpotExtractionQueue_Create.argtypes = [ct.c_int, ct.c_int, vp, vp, vp, ct.c_int, ct.c_int, vp]
    L.SpotExtractionQueue_Create.restype = vp
    L.ImgProc_AddFrameU16.argtypes = [vp, vp]
    L.ImgProc_NumFinishedFrames.argtypes = [vp]
    L.ImgProc_NumFinishedFrames.restype = ct.c_int
    L.GainOffsetCalib_Create.argtypes = [ct.c_float, ct.c_float, vp]
    L.GainOffsetCalib_Create.restype = vp
    L.ImgProc_Destroy.argtypes = [vp]
    ctx = L.Context_Create()
    q = None
    try:
        shape = np.array([sumframes, rs, rs], np.int32)
        rq = L.RQ_Create(shape.ctypes.data, ctx)
        cfg = SpotDetectorConfig(int(u1), int(u2), int(maxfilter), int(det_roisize), float(min_intensity),
                                 float(max_intensity), None)
        sdf = L.SpotDetector_Configure(ct.byref(cfg))
        calib = None
        if gain_offset is not None:
            calib = L.GainOffsetCalib_Create(float(gain_offset[0]), float(gain_offset[1]), ctx)
        q = L.SpotExtractionQueue_Create(w, h, rq, sdf, calib, 2, sumframes, ctx)
        L.SpotDetector_DestroyFactory(sdf)
        for f in range(n):
            L.ImgProc_AddFrameU16(q, frames[f].ctypes.data)
        t0 = time.time()
        while L.ImgProc_NumFinishedFrames(q) < n // sumframes:
            if time.time() - t0 > timeout:
                raise TimeoutError("reference spot-extraction queue did not finish")
            time.sleep(0.01)
        time.sleep(0.05)
        cnt = L.RQ_Length(rq)
        info = np.zeros(cnt, ROIInfoDType)
        rois = np.zeros((cnt, sumframes, rs, rs), np.float32)
        if cnt:
            L.RQ_Pop(rq, cnt, info.ctypes.data, rois.ctypes.data)
        return info, rois
    finally:
        if q:
            L.ImgProc_Destroy(q)  # the queue before the ROI queue it fills
        L.Context_Destroy(ctx)


ROI_TYPE = np.dtype([("cornerpos", "<i4", 2), ("startframe", "<i4"), ("numframes", "<i4")])


def roi_extractor(frames_u16, rois, roiframes, roisize, gain_offset=None, timeout=120.0):
    """The reference's ROI extractor (ROIExtractor_Create, ImageProcessor.cpp:221; needs a GPU):
    pushes the 16-bit frames, waits (bounded) until it is idle, and takes every record in the
    order ROIExtractor_GetResults gives them. ROIs must lie inside the frame (the reference
    reads outside it otherwise)."""
    import time
    L = lib()
    vp = ct.c_void_p
    frames = np.ascontiguousarray(frames_u16, dtype=np.uint16)
    n, h, w = frames.shape
    rois = np.ascontiguousarray(rois, dtype=ROI_TYPE)
    L.ROIExtractor_Create.argtypes = [ct.c_int, ct.c_int, vp, ct.c_int, ct.c_int, ct.c_int, vp, vp]
    L.ROIExtractor_Create.restype = vp
    L.ROIExtractor_GetResultCount.argtypes = [vp]
    L.ROIExtractor_GetResultCount.restype = ct.c_int
    L.ROIExtractor_GetResults.argtypes = [vp, ct.c_int, vp, vp]
    L.ROIExtractor_GetResults.restype = ct.c_int
    L.ImgProc_AddFrameU16.argtypes = [vp, vp]
    L.ImgProc_IsIdle.argtypes = [vp]
    L.ImgProc_IsIdle.restype = ct.c_bool
    L.ImgProc_Destroy.argtypes = [vp]
    L.GainOffsetCalib_Create.argtypes = [ct.c_float, ct.c_float, vp]
    L.GainOffsetCalib_Create.restype = vp
    ctx = L.Context_Create()
    q = None
    try:
        calib = None
        if gain_offset is not None:
            calib = L.GainOffsetCalib_Create(float(gain_offset[0]), float(gain_offset[1]), ctx)
        q = L.ROIExtractor_Create(w, h, rois.ctypes.data, len(rois), int(roiframes), int(roisize), calib, ctx)
        for f in range(n):
            L.ImgProc_AddFrameU16(q, frames[f].ctypes.data)
        t0 = time.time()
        time.sleep(0.05)
        while not L.ImgProc_IsIdle(q):
            if time.time() - t0 > timeout:
                raise TimeoutError("reference ROI extractor did not finish")
            time.sleep(0.01)
        time.sleep(0.05)
        cnt = L.ROIExtractor_GetResultCount(q)
        out_r = np.zeros(cnt, ROI_TYPE)
        out_b = np.zeros((cnt, roiframes, roisize, roisize), np.float32)
        if cnt:
            got = L.ROIExtractor_GetResults(q, cnt, out_r.ctypes.data, out_b.ctypes.data)
            out_r, out_b = out_r[:got], out_b[:got]
        return out_r, out_b
    finally:
        if q:
            L.ImgProc_Destroy(q)
        L.Context_Destroy(ctx)
