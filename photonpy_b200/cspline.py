"""Cubic-spline PSF estimator — counterpart of photonpy/cpp/cspline.py (lines 16-213)."""
from __future__ import annotations

import ctypes

import numpy as np
import numpy.ctypeslib as ctl

from . import estimator
from .context import Context
from .lib import NullableFloatArrayType


class CSplineCalibration(ctypes.Structure):
    """(n_voxels_z, n_voxels_y, n_voxels_x, z_min, z_max, coefs) — cspline.py:16-38,
    CubicSplinePSF.h:12-23. coefs has shape [nz, ny, nx, 64]."""
    _fields_ = [
        ("n_voxels_z", ctypes.c_int32),
        ("n_voxels_y", ctypes.c_int32),
        ("n_voxels_x", ctypes.c_int32),
        ("z_min", ctypes.c_float),
        ("z_max", ctypes.c_float),
        ("coefs", ctl.ndpointer(np.float32, flags="aligned, c_contiguous")),
    ]

    def __init__(self, z_min, z_max, coefs):
        coefs = np.ascontiguousarray(coefs, dtype=np.float32)
        self.coefsx = coefs  # keep the array alive while the struct points at it
        self.n_voxels_x = coefs.shape[2]
        self.n_voxels_y = coefs.shape[1]
        self.n_voxels_z = coefs.shape[0]
        self.coefs = coefs.ctypes.data
        self.z_min = z_min
        self.z_max = z_max
        self.zrange = [z_min, z_max]

    @classmethod
    def from_file(cls, filename):
        """.npz/.npy dict with zmin/zmax in nm (stored in um, cspline.py:45-53) and 'coeff'."""
        calibration = np.load(filename, allow_pickle=True)
        z_min = calibration["zmin"] * 1e-3
        z_max = calibration["zmax"] * 1e-3
        return cls(z_min, z_max, calibration["coeff"])


class CSplinePSF(estimator.Estimator):
    def __init__(self, ctx: Context, inst, calib):
        super().__init__(ctx, inst, calib)


class CSplineMethods:
    FlatBg = 0
    TiltedBg = 1
    BgImage = 2

    def __init__(self, ctx: Context):
        smlmlib = ctx.smlm.lib
        self.ctx = ctx
        self._CSpline_CreatePSF = smlmlib.CSpline_CreatePSF
        self._CSpline_CreatePSF.argtypes = [ctypes.c_int32, ctypes.POINTER(CSplineCalibration), NullableFloatArrayType,
                                            ctypes.c_int32, ctypes.c_bool, ctypes.c_void_p]
        self._CSpline_CreatePSF.restype = ctypes.c_void_p
        self._CSpline_CreatePSF_FromFile = smlmlib.CSpline_CreatePSF_FromFile
        self._CSpline_CreatePSF_FromFile.argtypes = [ctypes.c_int32, ctypes.c_char_p, ctypes.c_int32, ctypes.c_bool,
                                                     ctypes.c_void_p]
        self._CSpline_CreatePSF_FromFile.restype = ctypes.c_void_p
        self._CSpline_CreatePSF_Oversampled = smlmlib.CSpline_CreatePSF_Oversampled
        self._CSpline_CreatePSF_Oversampled.argtypes = [ctypes.c_int32, ctypes.POINTER(CSplineCalibration),
                                                        NullableFloatArrayType, ctypes.c_int32, ctypes.c_float,
                                                        ctypes.c_bool, ctypes.c_void_p]
        self._CSpline_CreatePSF_Oversampled.restype = ctypes.c_void_p
        self._CSpline_Compute = smlmlib.CSpline_Compute
        self._CSpline_Compute.argtypes = [ctl.ndpointer(np.int32, flags="aligned, c_contiguous"),
                                          ctl.ndpointer(np.float32, flags="aligned, c_contiguous"),
                                          ctl.ndpointer(np.float32, flags="aligned, c_contiguous"), ctypes.c_int32]
        self._CSpline_Evaluate = smlmlib.CSpline_Evaluate
        self._CSpline_Evaluate.argtypes = [ctl.ndpointer(np.int32, flags="aligned, c_contiguous"),
                                           ctl.ndpointer(np.float32, flags="aligned, c_contiguous"),
                                           ctl.ndpointer(np.float32, flags="aligned, c_contiguous"), ctypes.c_int32,
                                           ctl.ndpointer(np.float32, flags="aligned, c_contiguous")]

    def CreatePSF_XYZIBg(self, roisize, calib: CSplineCalibration, fitMode=FlatBg, cuda=True,
                         xyStep=1.0) -> CSplinePSF:
        """Spline PSF estimator (x, y, z, I, bg[, bgx, bgy]). Extension: xyStep < 1 for a calibration
        sampled every xyStep ROI pixels in x and y (e.g. 0.5 for a 2x oversampled z-stack)."""
        if xyStep == 1.0:
            inst = self._CSpline_CreatePSF(roisize, calib, None, fitMode, cuda, self.ctx.inst)
        else:
            inst = self._CSpline_CreatePSF_Oversampled(roisize, calib, None, fitMode, float(xyStep), cuda,
                                                       self.ctx.inst)
        return CSplinePSF(self.ctx, inst, calib)

    def ComputeSplineCoeff(self, data, border=0):
        """Spline coefficients [*(shape-3+2*border), 64] of a 3D array (z, y, x)."""
        data = np.ascontiguousarray(data, dtype=np.float32)
        outshape = np.array(data.shape) - 3 + border * 2
        spline = np.zeros((*outshape, 64), dtype=np.float32)
        shape = np.ascontiguousarray(data.shape, dtype=np.int32)
        self._CSpline_Compute(shape, data, spline, border)
        return spline

    def Evaluate(self, splineCoefs, shift, border=0):
        """Matrix whose last dimension is (value, dv/dx, dv/dy, dv/dz)."""
        assert len(splineCoefs.shape) == 4 and splineCoefs.shape[-1] == 64
        splineCoefs = np.ascontiguousarray(splineCoefs, dtype=np.float32)
        shift = np.ascontiguousarray(shift, dtype=np.float32)
        outshape = np.array(splineCoefs.shape[:3]) - border * 2
        values = np.zeros((*outshape, 4), dtype=np.float32)
        self._CSpline_Evaluate(np.array(splineCoefs.shape, dtype=np.int32), splineCoefs, shift, border, values)
        return values

    def CreatePSFFromFile(self, roisize, filename, fitMode=FlatBg, cuda=True) -> CSplinePSF:
        if filename.endswith(".zstack"):
            zstack, zrange = load_zstack(filename)
            return self.CreatePSFFromZStack(roisize, zstack, zrange, fitMode, cuda)
        if filename.endswith(".pickle"):
            import pickle
            with open(filename, "rb") as f:
                d = pickle.load(f)
            return self.CreatePSFFromZStack(roisize, d["zstack"], d["zrange"], fitMode, cuda)
        raise RuntimeError(f"Unknown psf extension: {filename}")

    def CreatePSFFromZStack(self, roisize, zstack, zrange, fitMode=FlatBg, cuda=True, border=0) -> CSplinePSF:
        spline_coeff = self.ComputeSplineCoeff(zstack, border)
        calib = CSplineCalibration(zrange[0], zrange[-1], spline_coeff)
        calib.zstack = zstack
        return self.CreatePSF_XYZIBg(roisize, calib, fitMode, cuda)


_zstack_header = [("version", "<i4"), ("dims", "<i4", 3), ("zrange", "<f4", 2)]


def load_zstack(fn):
    """Z-stack file: header (version 1, int32[3] shape, float32[2] zrange) then float32 data
    (format of photonpy/smlm/psf.py:257-276 and CubicSplinePSF.cu:109-133)."""
    with open(fn, "rb") as f:
        d = np.fromfile(f, dtype=_zstack_header, count=1, sep="")
        version, shape, zrange = d[0]
        if version != 1:
            raise ValueError("Wrong ZStack file version (should be 1)")
        zstack = np.fromfile(f, dtype="<f4", sep="").reshape(shape)
    return zstack, zrange


def save_zstack(zstack, zrange, fn):
    with open(fn, "wb") as f:
        np.array([(1, zstack.shape, (zrange[0], zrange[-1]))], dtype=_zstack_header).tofile(f, "")
        np.ascontiguousarray(zstack, dtype=np.float32).tofile(f, "")
