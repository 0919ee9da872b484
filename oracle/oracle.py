"""ctypes front end of the CPU oracle (psf_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of bench.py, never by the photonpy_b200 package.

The FP32 functions restate photonpy's CPU estimator arithmetic
(cpp/SMLMLib/Estimators/Estimation.h:63-251, SolveMatrix.h:84-452,
Estimators/Gaussian/GaussianPSFModels.h, Estimators/CSpline/CubicSplinePSFModels.h);
the FP64 functions are the same algorithm in double precision and serve as the
"true MLE" yardstick. Parity of the FP32 build with the reference's own C++ CPU
estimator is pinned by tests/test_oracle.py against tests/golden/*.npz.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "liboracle.so")
SOURCES = [os.path.join(HERE, "psf_oracle.c"), os.path.join(HERE, "psf_oracle_impl.h")]

XYIBG, XYIBG_CONSTSIGMA, XYIBG_SIGMA, XYIBG_SIGMAXY, XYZIBG, CSPLINE, XYITILTEDBG, XYITILTEDBG_SIGMAXY, \
    INTENSITYBG, CSPLINE_TILTED, CSPLINE_BGIMAGE = range(11)
NUM_PARAMS = {XYIBG: 4, XYIBG_CONSTSIGMA: 4, XYIBG_SIGMA: 5, XYIBG_SIGMAXY: 6, XYZIBG: 5, CSPLINE: 5, XYITILTEDBG: 6,
              XYITILTEDBG_SIGMAXY: 8, INTENSITYBG: 2, CSPLINE_TILTED: 7, CSPLINE_BGIMAGE: 5}


class PsoModel(ct.Structure):
    _fields_ = [
        ("model", ct.c_int32),
        ("roisize", ct.c_int32),
        ("sigma", ct.c_float * 2),
        ("astig_x", ct.c_float * 5),
        ("astig_y", ct.c_float * 5),
        ("minz", ct.c_float),
        ("maxz", ct.c_float),
        ("spline_shape", ct.c_int32 * 3),
        ("spline_zmin", ct.c_float),
        ("spline_zmax", ct.c_float),
        ("coefs", ct.c_void_p),
        ("spline_q", ct.c_float),
    ]


_lock = threading.Lock()
_lib = None


def build(force: bool = False) -> str:
    """Compile psf_oracle.c with gcc (no FMA contraction, no fast-math)."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    newest = max(os.path.getmtime(s) for s in SOURCES)
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= newest:
        return LIB_PATH
    tmp = LIB_PATH + f".tmp{os.getpid()}"
    cmd = ["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-std=gnu11",
           "-o", tmp, SOURCES[0], "-lm", "-lpthread"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            path = build()
            L = ct.CDLL(path)
            fp = ct.POINTER(ct.c_float)
            ip = ct.POINTER(ct.c_int32)
            dp = ct.POINTER(ct.c_double)
            for sfx in ("_f32", "_f64"):
                f = getattr(L, "pso_fit" + sfx)
                f.argtypes = [ct.POINTER(PsoModel), ct.c_int, fp, fp, fp, ct.c_int, ct.c_double, fp, ip, fp,
                              ct.c_int, ct.c_int]
                f = getattr(L, "pso_derivatives" + sfx)
                f.argtypes = [ct.POINTER(PsoModel), ct.c_int, fp, fp, fp, fp]
                f = getattr(L, "pso_crlb" + sfx)
                f.argtypes = [ct.POINTER(PsoModel), ct.c_int, fp, fp, fp, fp, fp, dp]
            L.pso_spline_compute.argtypes = [ip, fp, fp, ct.c_int]
            L.pso_glrt_f32.argtypes = [ct.POINTER(PsoModel), ct.c_int, fp, fp, fp, fp, fp]
            L.pso_detect_spots.argtypes = [fp, fp, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int,
                                           ct.c_float, ct.c_float, ct.c_int, ip, fp]
            L.pso_detect_spots.restype = ct.c_int
            L.pso_cut_rois.argtypes = [fp, ct.c_int, ct.c_int, ip, ct.c_int, ct.c_int, ip, fp]
            L.pso_sizeof_model.restype = ct.c_int
            assert L.pso_sizeof_model() == ct.sizeof(PsoModel), "oracle struct layout mismatch"
            _lib = L
    return _lib


def _fptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(ct.POINTER(ct.c_float))


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


class Model:
    """Description of one PSF model instance, mirroring the reference's creation calls."""

    def __init__(self, model: int, roisize: int, sigma=(1.0, 1.0), astig_x=None, astig_y=None, zrange=(0, 0),
                 coefs=None, spline_zrange=(0, 0), spline_xy_step=1.0):
        self.model = model
        self.roisize = int(roisize)
        self.K = NUM_PARAMS[model]
        self.numconst = 2 if model in (XYIBG_CONSTSIGMA, XYITILTEDBG) else (3 if model == INTENSITYBG else 0)
        if model == CSPLINE_BGIMAGE:
            self.numconst = self.roisize * self.roisize
        s = PsoModel()
        s.model = model
        s.roisize = self.roisize
        s.sigma[0], s.sigma[1] = (sigma, sigma) if np.isscalar(sigma) else tuple(sigma)
        ax = list(astig_x) if astig_x is not None else [1, 0, 1, 0, 0]
        ay = list(astig_y) if astig_y is not None else [1, 0, 1, 0, 0]
        ax += [0.0] * (5 - len(ax))
        ay += [0.0] * (5 - len(ay))
        for i in range(5):
            s.astig_x[i] = ax[i]
            s.astig_y[i] = ay[i]
        s.minz, s.maxz = zrange
        self._coefs = None
        if coefs is not None:
            self._coefs = np.ascontiguousarray(coefs, dtype=np.float32)
            nz, ny, nx = self._coefs.shape[:3]
            s.spline_shape[0], s.spline_shape[1], s.spline_shape[2] = nz, ny, nx
            s.spline_zmin, s.spline_zmax = spline_zrange
            s.coefs = self._coefs.ctypes.data
        s.spline_q = 1.0 / float(spline_xy_step)
        self.s = s

    # -- oracle entry points -------------------------------------------------------------
    def fit(self, samples, constants=None, initial=None, iterations=50, lambda_=1e-18, fp64=False,
            trace_len=0, nthreads=None):
        samples = _f32(samples)
        n = samples.shape[0]
        constants = _f32(constants)
        initial = _f32(initial)
        params = np.zeros((n, self.K), np.float32)
        its = np.zeros(n, np.int32)
        trace = np.zeros((n, trace_len, self.K), np.float32) if trace_len > 0 else None
        f = lib().pso_fit_f64 if fp64 else lib().pso_fit_f32
        f(ct.byref(self.s), n, _fptr(samples), _fptr(constants), _fptr(initial), int(iterations),
          float(lambda_), _fptr(params), its.ctypes.data_as(ct.POINTER(ct.c_int32)), _fptr(trace),
          int(trace_len), int(nthreads or os.cpu_count() or 1))
        if trace_len > 0:
            return params, its, trace
        return params, its

    def derivatives(self, params, constants=None, fp64=False):
        params = _f32(params)
        n = params.shape[0]
        npix = self.roisize * self.roisize
        ev = np.zeros((n, self.roisize, self.roisize), np.float32)
        deriv = np.zeros((n, self.K, self.roisize, self.roisize), np.float32)
        f = lib().pso_derivatives_f64 if fp64 else lib().pso_derivatives_f32
        f(ct.byref(self.s), n, _fptr(params), _fptr(_f32(constants)), _fptr(deriv), _fptr(ev))
        del npix
        return deriv, ev

    def expected_value(self, params, constants=None, fp64=False):
        return self.derivatives(params, constants, fp64)[1]

    def crlb(self, params, samples=None, constants=None, fp64=False, return_fisher=False):
        params = _f32(params)
        n = params.shape[0]
        crlb = np.zeros((n, self.K), np.float32)
        chisq = np.zeros(n, np.float32)
        fisher = np.zeros((n, self.K, self.K), np.float64) if return_fisher else None
        f = lib().pso_crlb_f64 if fp64 else lib().pso_crlb_f32
        f(ct.byref(self.s), n, _fptr(params), _fptr(_f32(samples)), _fptr(_f32(constants)), _fptr(crlb),
          _fptr(chisq), None if fisher is None else fisher.ctypes.data_as(ct.POINTER(ct.c_double)))
        if return_fisher:
            return crlb, chisq, fisher
        return crlb, chisq


    def glrt(self, params, samples, constants=None, mean_roi=None):
        """GLRT diagnostics {ll_on, ll_off, mean} per spot at `params` (GLRT_PSF.cu:96-131);
        mean_roi (npix samples) replaces each spot's own mean source, as the reference's loop does."""
        params = _f32(params)
        samples = _f32(samples)
        n = params.shape[0]
        out = np.zeros((n, 3), np.float32)
        lib().pso_glrt_f32(ct.byref(self.s), n, _fptr(params), _fptr(samples), _fptr(_f32(constants)),
                           _fptr(_f32(mean_roi)), _fptr(out))
        return out


def spline_compute(data, border=0):
    """CSpline_Compute restated (double LUP solve per voxel)."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    shape = np.ascontiguousarray(data.shape, dtype=np.int32)
    out = np.zeros((*(np.array(data.shape) - 3 + 2 * border), 64), np.float32)
    rc = lib().pso_spline_compute(shape.ctypes.data_as(ct.POINTER(ct.c_int32)), _fptr(data), _fptr(out),
                                  int(border))
    if rc != 0:
        raise RuntimeError("spline basis matrix is singular")
    return out


def detect_spots(frame, u1, u2, maxfilter, roisize, min_intensity, max_intensity=np.inf, background=None,
                 max_spots=100000):
    """SpotDetector::Detect + SpotDetector_ProcessFrame restated: returns (number found,
    indices y*w+x [<= max_spots], scores, corner positions [n, 2] (y, x), rois [n, roisize, roisize])."""
    frame = np.ascontiguousarray(frame, dtype=np.float32)
    h, w = frame.shape
    bg = None if background is None else np.ascontiguousarray(background, dtype=np.float32)
    idx = np.zeros(max_spots, np.int32)
    score = np.zeros(max_spots, np.float32)
    found = lib().pso_detect_spots(_fptr(frame), _fptr(bg), w, h, int(u1), int(u2), int(maxfilter), int(roisize),
                                   float(min_intensity), float(max_intensity), int(max_spots),
                                   idx.ctypes.data_as(ct.POINTER(ct.c_int32)), _fptr(score))
    n = min(found, max_spots)
    corner = np.zeros((n, 2), np.int32)
    rois = np.zeros((n, roisize, roisize), np.float32)
    lib().pso_cut_rois(_fptr(frame), w, h, idx.ctypes.data_as(ct.POINTER(ct.c_int32)), n, int(roisize),
                       corner.ctypes.data_as(ct.POINTER(ct.c_int32)), _fptr(rois))
    return found, idx[:n], score[:n], corner, rois


def camera_calibrate(frames, kind=None, gain=1.0, offset=0.0):
    """CameraCalibration.cu:19-57 restated in float32 numpy (subtract, then multiply, each
    rounded). kind: None, "gain_offset" (scalars; negatives to 0), "image" (per-pixel arrays;
    negatives to 0), "scmos" (per-pixel, no clamp; the intended transform, see the note on
    photonpy's sCMOS transform in the integration notes)."""
    x = np.asarray(frames).astype(np.float32)
    if kind is None:
        return x
    g = np.asarray(gain, dtype=np.float32)
    o = np.asarray(offset, dtype=np.float32)
    v = (x - o).astype(np.float32) * g
    v = v.astype(np.float32)
    if kind in ("gain_offset", "image"):
        v = np.where(v < 0, np.float32(0), v).astype(np.float32)
    return v


def spot_extraction_queue(frames_u16, u1, u2, maxfilter, det_roisize, min_intensity, max_intensity=np.inf,
                          background=None, sumframes=1, roi_shape=None, calib=None):
    """The spot-extraction queue restated (ImgFilterQueue.cu:117-260): 16-bit frames ->
    calibration -> sums of sumframes frames (left to right) -> spot detection on each sum ->
    ROI stacks [sumframes][rh][rw] of the calibrated frames (corner = centre - size/2, pixels
    clamped). Incomplete trailing groups are not processed. Returns (info records as an array of
    (id, score, x, y, z), rois [n, sumframes, rh, rw]) in frame order, row-major within a frame.
    calib: None or (kind, gain, offset) for camera_calibrate."""
    frames = np.asarray(frames_u16)
    n, h, w = frames.shape
    rh, rw = roi_shape if roi_shape is not None else (det_roisize, det_roisize)
    cal = camera_calibrate(frames, *calib) if calib is not None else frames.astype(np.float32)
    infos, stacks = [], []
    for g in range(n // sumframes):
        grp = cal[g * sumframes:(g + 1) * sumframes]
        s = grp[0].copy()
        for z in range(1, sumframes):
            s = (s + grp[z]).astype(np.float32)
        found, idx, score, _, _ = detect_spots(s, u1, u2, maxfilter, det_roisize, min_intensity, max_intensity,
                                               background, max_spots=h * w)
        for i, p in enumerate(idx):
            cy, cx = int(p) // w - rh // 2, int(p) % w - rw // 2
            ys = np.clip(np.arange(cy, cy + rh), 0, h - 1)
            xs = np.clip(np.arange(cx, cx + rw), 0, w - 1)
            stacks.append(grp[:, ys][:, :, xs])
            infos.append((g, score[i], cx, cy, 0))
    info = np.array(infos, dtype=[("id", "<i4"), ("score", "<f4"), ("x", "<i4"), ("y", "<i4"), ("z", "<i4")])
    rois = np.array(stacks, dtype=np.float32).reshape(len(stacks), sumframes, rh, rw)
    return info, rois


ROI_TYPE = np.dtype([("cornerpos", "<i4", 2), ("startframe", "<i4"), ("numframes", "<i4")])


def extract_rois(frames_u16, rois, roiframes, roisize, calib=None):
    """The ROI extractor restated (ImageProcessor.cpp:61-233): ROI i collects the roisize x
    roisize box at (x, y) = cornerpos of frames startframe .. startframe + numframes - 1 of the
    calibrated movie; records complete at their last frame (the start frame when numframes <= 0)
    and come out by last frame, then start frame, then request order. Boxes are clamped to the
    frame (the reference reads outside it). Returns (records, boxes [n, roiframes, roisize,
    roisize]) for the records complete within the movie; unwritten boxes are zero."""
    frames = np.asarray(frames_u16)
    n, h, w = frames.shape
    cal = camera_calibrate(frames, *calib) if calib is not None else frames.astype(np.float32)
    rois = np.asarray(rois, dtype=ROI_TYPE)
    last = rois["startframe"] + np.maximum(rois["numframes"], 1) - 1
    order = sorted(range(len(rois)), key=lambda i: (last[i], rois["startframe"][i], i))
    out_r, out_b = [], []
    for i in order:
        if last[i] >= n:
            continue
        r = rois[i]
        b = np.zeros((roiframes, roisize, roisize), np.float32)
        x0, y0 = int(r["cornerpos"][0]), int(r["cornerpos"][1])
        ys = np.clip(np.arange(y0, y0 + roisize), 0, h - 1)
        xs = np.clip(np.arange(x0, x0 + roisize), 0, w - 1)
        for f in range(min(max(int(r["numframes"]), 0), roiframes)):
            b[f] = cal[int(r["startframe"]) + f][ys][:, xs]
        out_r.append(r)
        out_b.append(b)
    return np.array(out_r, dtype=ROI_TYPE), np.array(out_b, np.float32).reshape(len(out_b), roiframes, roisize,
                                                                                roisize)
