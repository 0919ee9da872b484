"""Gaussian PSF estimators — counterpart of photonpy/cpp/gaussian.py (lines 15-237)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .context import Context
from .estimator import Estimator
from .lib import check_error

_F32 = np.ctypeslib.ndpointer(np.float32, flags="aligned, c_contiguous")
_I32 = np.ctypeslib.ndpointer(np.int32, flags="aligned, c_contiguous")


class Gauss3D_Calibration(ctypes.Structure):
    """Astigmatic calibration, sigma(z) = s0*sqrt(1 + tz^2/d^2 + A tz^3/d^2), tz = z - gamma,
    x/y = [s0, gamma, d, A] (gaussian.py:15-51, GaussianPSF.h:27-33)."""
    _fields_ = [("x", ctypes.c_float * 4), ("y", ctypes.c_float * 4), ("zrange", ctypes.c_float * 2)]

    def __init__(self, x=[1.3, 2, 3, 0], y=[1.3, -2, 3, 0], zrange=[-3, 3]):
        self.x = (ctypes.c_float * 4)(*x)
        self.y = (ctypes.c_float * 4)(*y)
        self.zrange = (ctypes.c_float * 2)(*zrange)

    def sigma(self):
        return self.x[0], self.y[0]

    @classmethod
    def from_file(cls, filename):
        ext = os.path.splitext(filename)[1]
        if ext == ".npy":
            calibration = np.load(filename, allow_pickle=True).item()
        else:
            import yaml
            with open(filename, "r") as f:
                calibration = yaml.safe_load(f)
        return cls(calibration.get("x"), calibration.get("y"))

    def save(self, filename):
        ext = os.path.splitext(filename)[1]
        if ext == ".npy":
            np.save(filename, self.__dict__())
        elif ext == ".yaml":
            import yaml
            with open(filename, "w") as f:
                yaml.dump(self.__dict__(), f)

    def __dict__(self):
        return {"x": np.array(self.x, dtype=float).tolist(), "y": np.array(self.y, dtype=float).tolist(),
                "range": np.array(self.zrange, dtype=float).tolist()}


class Gauss3D_CalibrationB(ctypes.Structure):
    """Extension: astigmatic calibration with a quartic term, x/y = [s0, gamma, d, A, B],
    sigma(z) = s0*sqrt(1 + tz^2/d^2 + A tz^3/d^2 + B tz^4/d^4)."""
    _fields_ = [("x", ctypes.c_float * 5), ("y", ctypes.c_float * 5), ("zrange", ctypes.c_float * 2)]

    def __init__(self, x, y, zrange):
        x = list(x) + [0.0] * (5 - len(x))
        y = list(y) + [0.0] * (5 - len(y))
        self.x = (ctypes.c_float * 5)(*x)
        self.y = (ctypes.c_float * 5)(*y)
        self.zrange = (ctypes.c_float * 2)(*zrange)


class GaussianPSFMethods:
    def __init__(self, ctx: Context):
        smlmlib = ctx.smlm.lib
        self.ctx = ctx
        self.lib = ctx.smlm
        vp = ctypes.c_void_p
        self._Gauss2D_CreatePSF_XYIBg = smlmlib.Gauss2D_CreatePSF_XYIBg
        self._Gauss2D_CreatePSF_XYIBg.argtypes = [ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_int32, vp]
        self._Gauss2D_CreatePSF_XYIBg.restype = vp
        self._Gauss2D_CreatePSF_XYIBgConstSigma = smlmlib.Gauss2D_CreatePSF_XYIBgConstSigma
        self._Gauss2D_CreatePSF_XYIBgConstSigma.argtypes = [ctypes.c_int32, ctypes.c_int32, vp]
        self._Gauss2D_CreatePSF_XYIBgConstSigma.restype = vp
        self._Gauss2D_CreatePSF_XYIBgSigma = smlmlib.Gauss2D_CreatePSF_XYIBgSigma
        self._Gauss2D_CreatePSF_XYIBgSigma.argtypes = [ctypes.c_int32, ctypes.c_float, ctypes.c_int32, vp]
        self._Gauss2D_CreatePSF_XYIBgSigma.restype = vp
        self._Gauss2D_CreatePSF_XYIBgSigmaXY = smlmlib.Gauss2D_CreatePSF_XYIBgSigmaXY
        self._Gauss2D_CreatePSF_XYIBgSigmaXY.argtypes = [ctypes.c_int32, ctypes.c_float, ctypes.c_float,
                                                         ctypes.c_int32, vp]
        self._Gauss2D_CreatePSF_XYIBgSigmaXY.restype = vp
        self._Gauss2D_CreatePSF_XYZIBg = smlmlib.Gauss2D_CreatePSF_XYZIBg
        self._Gauss2D_CreatePSF_XYZIBg.argtypes = [ctypes.c_int32, ctypes.POINTER(Gauss3D_Calibration),
                                                   ctypes.c_int32, vp]
        self._Gauss2D_CreatePSF_XYZIBg.restype = vp
        self._Gauss2D_CreatePSF_XYZIBgB = smlmlib.Gauss2D_CreatePSF_XYZIBgB
        self._Gauss2D_CreatePSF_XYZIBgB.argtypes = [ctypes.c_int32, ctypes.POINTER(Gauss3D_CalibrationB),
                                                    ctypes.c_int32, vp]
        self._Gauss2D_CreatePSF_XYZIBgB.restype = vp
        self._EstimateIBg = smlmlib.Gauss2D_EstimateIntensityBg
        self._EstimateIBg.argtypes = [_F32, _F32, _F32, ctypes.c_int32, _F32, _I32, _F32, ctypes.c_int32,
                                      ctypes.c_int32, ctypes.c_int32]
        self._EstimateIBg.restype = None
        self._Gauss2D_CreatePSF_XYITiltedBg = smlmlib.Gauss2D_CreatePSF_XYITiltedBg
        self._Gauss2D_CreatePSF_XYITiltedBg.argtypes = [ctypes.c_int32, ctypes.c_int32, vp]
        self._Gauss2D_CreatePSF_XYITiltedBg.restype = vp
        self._Gauss2D_CreatePSF_XYITiltedBgSigmaXY = smlmlib.Gauss2D_CreatePSF_XYITiltedBgSigmaXY
        self._Gauss2D_CreatePSF_XYITiltedBgSigmaXY.argtypes = [ctypes.c_int32, ctypes.c_float, ctypes.c_float,
                                                               ctypes.c_int32, vp]
        self._Gauss2D_CreatePSF_XYITiltedBgSigmaXY.restype = vp

    def CreatePSF_XYIBg(self, roisize, sigma, cuda=True) -> Estimator:
        """[x,y,I,bg] (px, px, photons, photons/px). sigma: scalar or (sx, sy); None passes
        sigma per spot as 2 constants (XYIBgConstSigma)."""
        if sigma is not None:
            if np.isscalar(sigma):
                sigma_x, sigma_y = sigma, sigma
            else:
                sigma_x, sigma_y = sigma
            inst = self._Gauss2D_CreatePSF_XYIBg(roisize, sigma_x, sigma_y, cuda, self.ctx.inst)
        else:
            inst = self._Gauss2D_CreatePSF_XYIBgConstSigma(roisize, cuda, self.ctx.inst)
        return Estimator(self.ctx, inst, sigma)

    def CreatePSF_XYIBgSigma(self, roisize, initialSigma, cuda=True) -> Estimator:
        """[x,y,I,bg,sigma]; sigma clamped to [1, roisize/2] during the fit."""
        inst = self._Gauss2D_CreatePSF_XYIBgSigma(roisize, initialSigma, cuda, self.ctx.inst)
        return Estimator(self.ctx, inst, initialSigma)

    def CreatePSF_XYIBgSigmaXY(self, roisize, initialSigma, cuda=True) -> Estimator:
        """[x,y,I,bg,sigmaX,sigmaY]; sigmas clamped to [1, roisize/2] during the fit."""
        if np.isscalar(initialSigma):
            initialSigma = [initialSigma, initialSigma]
        inst = self._Gauss2D_CreatePSF_XYIBgSigmaXY(roisize, initialSigma[0], initialSigma[1], cuda, self.ctx.inst)
        return Estimator(self.ctx, inst, initialSigma)

    def EstimateIBg(self, images, sigma, xy, roipos=None, useCuda=False):
        """Intensity and background of each ROI with the spot at a known position xy [n, 2] and
        width sigma (photonpy/cpp/gaussian.py:153-172): returns (IBg [n, 2], crlb [n, 2]).
        100 LM iterations from (I, bg) = (1, 0). Runs on the GPU whatever useCuda says."""
        images = np.ascontiguousarray(images, dtype=np.float32)
        xy = np.ascontiguousarray(xy, dtype=np.float32)
        assert len(images.shape) == 3
        numspots = len(images)
        assert np.array_equal(xy.shape, (numspots, 2))
        imgw = images.shape[1]
        result = np.zeros((numspots, 2), dtype=np.float32)
        crlb = np.zeros((numspots, 2), dtype=np.float32)
        sigma_ = np.zeros((numspots, 2), dtype=np.float32)
        sigma_[:] = sigma
        if roipos is None:
            roipos = np.zeros((numspots, 2))
        assert np.array_equal(roipos.shape, (numspots, 2))
        roipos = np.ascontiguousarray(roipos, dtype=np.int32)
        if numspots > 0:
            self._EstimateIBg(images, result, crlb, numspots, xy, roipos, sigma_, imgw, 100, useCuda)
            check_error("EstimateIBg")
        return result, crlb

    def CreatePSF_XYITiltedBg(self, roisize, cuda=True) -> Estimator:
        """[x,y,I,bg,bgx,bgy] (photonpy/cpp/gaussian.py:193-200): mu = bg + bgx (x - R/2) +
        bgy (y - R/2) + I Gaussian(x, y); sigma_x/sigma_y per spot as 2 constants."""
        inst = self._Gauss2D_CreatePSF_XYITiltedBg(roisize, cuda, self.ctx.inst)
        return Estimator(self.ctx, inst)

    def CreatePSF_XYITiltedBgSigmaXY(self, roisize, initialSigma, cuda=True) -> Estimator:
        """[x,y,I,bg,bgx,bgy,sigmaX,sigmaY] (photonpy/cpp/gaussian.py:223-232). As in photonpy,
        the tilt enters the Jacobian but not the expected value."""
        if np.isscalar(initialSigma):
            initialSigma = [initialSigma, initialSigma]
        inst = self._Gauss2D_CreatePSF_XYITiltedBgSigmaXY(roisize, initialSigma[0], initialSigma[1], cuda,
                                                          self.ctx.inst)
        return Estimator(self.ctx, inst, initialSigma)

    def CreatePSF_XYZIBg(self, roisize, calib, cuda=True) -> Estimator:
        """[x,y,z,I,bg] astigmatic 3D Gaussian. calib: Gauss3D_Calibration, or
        Gauss3D_CalibrationB for the extension with a quartic term."""
        if isinstance(calib, Gauss3D_CalibrationB):
            inst = self._Gauss2D_CreatePSF_XYZIBgB(roisize, calib, cuda, self.ctx.inst)
        else:
            inst = self._Gauss2D_CreatePSF_XYZIBg(roisize, calib, cuda, self.ctx.inst)
        return Estimator(self.ctx, inst, calib)


Gaussian = GaussianPSFMethods
