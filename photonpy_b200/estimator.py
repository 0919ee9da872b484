"""Estimator — the drop-in Python surface of photonpy/cpp/estimator.py (lines 27-397).

Same constructor, method names, argument order, shapes, defaults (LM lambda 1e-18,
50 iterations) and error behaviour (the native side reports through the debug-print
callback and leaves outputs zero). Everything computes on the GPU through
libphotonpy_b200.so. Extensions: ``Estimate(..., return_iterations=True)``,
``EstimateWithCRLB`` (fused fit + CRLB + chi-square), ``EstimateDevice`` /
``ExpectedValueDevice`` (torch CUDA tensors, no host round trip) and ``SetKernelConfig``.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import numpy.ctypeslib as ctl

from .context import Context
from .lib import NullableFloatArrayType, NullableIntArrayType, check_error


class EstimatorProperties(ct.Structure):
    _fields_ = [
        ("numParams", ct.c_int),
        ("sampleCount", ct.c_int),
        ("numDiag", ct.c_int),
        ("numConst", ct.c_int),
        ("sampleIndexDims", ct.c_int),
    ]


class LevMarParams(ct.Structure):
    _fields_ = [("iterations", ct.c_int32), ("lambda_", ct.c_float), ("factor", ct.c_float)]


_F32 = ctl.ndpointer(np.float32, flags="aligned, c_contiguous")
_I32 = ctl.ndpointer(np.int32, flags="aligned, c_contiguous")


def _ptr(t):
    """Device pointer of a torch tensor (or None)."""
    return None if t is None else ct.c_void_p(t.data_ptr())


class Estimator:
    def __init__(self, ctx: Context, psfInst, calib=None):
        if not psfInst:
            raise RuntimeError("native estimator creation failed: " + _last_error(ctx))
        self.inst = psfInst
        self.ctx = ctx
        self.calib = calib
        lib = ctx.smlm.lib
        self._lib = lib
        Inst = ct.c_void_p
        self._Estimator_Delete = lib.Estimator_Delete
        self._Estimator_Delete.argtypes = [Inst]
        self._Estimator_ParamFormat = lib.Estimator_ParamFormat
        self._Estimator_ParamFormat.restype = ct.c_char_p
        self._Estimator_ParamFormat.argtypes = [Inst]
        self._Estimator_GetProperties = lib.Estimator_GetProperties
        self._Estimator_GetProperties.argtypes = [Inst, ct.POINTER(EstimatorProperties)]
        self._Estimator_SampleDims = lib.Estimator_SampleDims
        self._Estimator_SampleDims.argtypes = [Inst, _I32]
        self._Estimator_GetParamLimits = lib.Estimator_GetParamLimits
        self._Estimator_GetParamLimits.argtypes = [Inst, _F32]
        self._Estimator_ChiSquareAndCRLB = lib.Estimator_ChiSquareAndCRLB
        self._Estimator_ChiSquareAndCRLB.argtypes = [Inst, _F32, NullableFloatArrayType, _F32, _I32, ct.c_int32, _F32,
                                                     _F32]
        self._Estimator_ComputeExpectedValue = lib.Estimator_ComputeExpectedValue
        self._Estimator_ComputeExpectedValue.argtypes = [Inst, ct.c_int32, _F32, _F32, _I32, _F32]
        self._Estimator_ComputeDerivatives = lib.Estimator_ComputeDerivatives
        self._Estimator_ComputeDerivatives.argtypes = [Inst, ct.c_int32, _F32, _F32, _I32, _F32, _F32]
        self._Estimator_Estimate = lib.Estimator_Estimate
        self._Estimator_Estimate.argtypes = [Inst, ct.c_int32, _F32, _F32, _I32, NullableFloatArrayType, _F32, _F32,
                                             NullableIntArrayType, NullableFloatArrayType, ct.c_int32]
        self._Estimator_SetLMParams = lib.Estimator_SetLMParams
        self._Estimator_SetLMParams.argtypes = [Inst, ct.POINTER(LevMarParams)]
        self._Estimator_GetLMParams = lib.Estimator_GetLMParams
        self._Estimator_GetLMParams.argtypes = [Inst, ct.POINTER(LevMarParams)]
        lib.PB200_FisherMatrix.argtypes = [Inst, ct.c_int32, _F32, _F32, _F32]
        lib.PB200_FisherMatrix.restype = None
        self._EstimateCRLB = lib.PB200_EstimateCRLB
        self._EstimateCRLB.argtypes = [Inst, ct.c_int32, _F32, NullableFloatArrayType, NullableFloatArrayType, _F32,
                                       NullableIntArrayType, NullableFloatArrayType, NullableFloatArrayType]

        props = EstimatorProperties()
        self._Estimator_GetProperties(self.inst, props)
        self.numparams = props.numParams
        self.numconst = props.numConst
        self.samplecount = props.sampleCount
        self.indexdims = props.sampleIndexDims
        self.sampleshape = np.zeros(self.indexdims, dtype=np.int32)
        self._Estimator_SampleDims(self.inst, self.sampleshape)
        self.numdiag = props.numDiag
        self.fmt = self.ParamFormat()
        self.param_names = [s.strip() for s in self.fmt.split(",")]
        self.limits = np.zeros((self.numparams, 2), dtype=np.float32)
        self._Estimator_GetParamLimits(self.inst, self.limits)
        self.SetLevMarParams(1e-18, 50)

    # ------------------------------------------------------------------ helpers
    def _checkparams(self, params, constants, roipos):
        """Normalise the per-spot arguments of one call (the contract of photonpy's Estimator,
        photonpy/cpp/estimator.py:155-186): params as float32 [n, K] (one parameter vector is one
        spot), constants as float32 [n, numconst] (required when the model has constants; any
        array with n*numconst values, or one that broadcasts to [n, numconst]), ROI positions as
        int32 [n, indexdims] (zeros when omitted). Raises ValueError when a shape does not fit."""
        p = np.asarray(params, dtype=np.float32)
        if p.ndim == 1:
            p = p.reshape(1, -1)
        p = np.ascontiguousarray(p)
        n = p.shape[0]
        nc = self.numconst
        if constants is None:
            if nc:
                raise ValueError(f"the estimator needs {nc} constants per spot: pass an array of shape {(n, nc)}")
            c = np.zeros((n, 0), dtype=np.float32)
        else:
            c = np.asarray(constants, dtype=np.float32)
            if c.size == n * nc:
                c = np.ascontiguousarray(c.reshape(n, nc))
            else:
                try:
                    c = np.ascontiguousarray(np.broadcast_to(c, (n, nc)))
                except ValueError:
                    raise ValueError(f"constants of shape {c.shape} do not fit {(n, nc)}") from None
        if roipos is None:
            rp = np.zeros((n, self.indexdims), dtype=np.int32)
        else:
            rp = np.ascontiguousarray(roipos, dtype=np.int32)
            if rp.shape != (n, self.indexdims):
                raise ValueError(f"ROI positions of shape {rp.shape}, expected {(n, self.indexdims)}")
        if p.ndim != 2 or p.shape[1] != self.numparams:
            raise ValueError(f"expected {self.numparams} parameters per spot ({self.fmt}), got shape {p.shape}")
        return p, c, rp

    # ------------------------------------------------------------------ reference API
    def ExpectedValue(self, params, roipos=None, constants=None):
        """Expected value of each pixel of the ROIs, shape [len(params), *sampleshape]."""
        params, constants, roipos = self._checkparams(params, constants, roipos)
        ev = np.zeros((len(params), *self.sampleshape), dtype=np.float32)
        if len(params) > 0:
            self._Estimator_ComputeExpectedValue(self.inst, len(params), params, constants, roipos, ev)
        return ev

    def GenerateSample(self, params, roipos=None, constants=None):
        ev = self.ExpectedValue(params, roipos, constants)
        return np.random.poisson(ev)

    def FisherMatrix(self, params, roipos=None, constants=None):
        """Fisher information of the Poisson likelihood at each spot's parameters, float32
        [n, K, K]: FI_ij = sum over pixels of dmu/dtheta_i dmu/dtheta_j / mu, computed on the GPU by
        the fit kernels' Fisher pass (FP32 sums, mu clamped at 1e-8 as the C++ CRLB path does;
        photonpy's numpy version clamps at 1e-9, photonpy/cpp/estimator.py:205-220)."""
        params, constants, roipos = self._checkparams(params, constants, roipos)
        fi = np.zeros((len(params), self.numparams, self.numparams), dtype=np.float32)
        if len(params) > 0:
            self._lib.PB200_FisherMatrix(self.inst, len(params), params, constants, fi)
            check_error("FisherMatrix")
        return fi

    def CRLBAndChiSquare(self, params, samples=None, roipos=None, constants=None):
        """(crlb, chisq) if samples are given, otherwise crlb."""
        params, constants, roipos = self._checkparams(params, constants, roipos)
        crlb = np.zeros((len(params), self.numparams), dtype=np.float32)
        chisq = np.zeros(len(params), dtype=np.float32)
        if samples is not None:
            samples = np.ascontiguousarray(samples, dtype=np.float32)
            if not np.array_equal(samples.shape, [len(params), *self.sampleshape]):
                raise ValueError(f"Sample data was expected to have shape {[len(params), *self.sampleshape]}. "
                                 f"Given: {samples.shape}")
        if len(params) > 0:
            self._Estimator_ChiSquareAndCRLB(self.inst, params, samples, constants, roipos, len(params), crlb, chisq)
        if samples is not None:
            return crlb, chisq
        return crlb

    def ChiSquare(self, params, samples, roipos=None, constants=None):
        return self.CRLBAndChiSquare(params, samples, roipos, constants)[1]

    def CRLB(self, params, roipos=None, constants=None):
        """Cramer-Rao lower bound sqrt(diag(FI^-1)) at each spot's parameters, float32 [n, K]: the
        Fisher matrix from the GPU's Fisher pass, inverted in FP64 on the GPU (LUP with partial
        pivoting; +Inf where it is singular, where photonpy's numpy version takes a
        pseudo-inverse, photonpy/cpp/estimator.py:249-253)."""
        return self.CRLBAndChiSquare(params, None, roipos, constants)

    def Derivatives(self, params, roipos=None, constants=None):
        """(deriv, ev) with deriv shaped [numspots, numparams, *roishape]."""
        params, constants, roipos = self._checkparams(params, constants, roipos)
        deriv = np.zeros((len(params), self.numparams, *self.sampleshape), dtype=np.float32)
        ev = np.zeros((len(params), *self.sampleshape), dtype=np.float32)
        if len(params) > 0:
            self._Estimator_ComputeDerivatives(self.inst, len(params), params, constants, roipos, deriv, ev)
        return deriv, ev

    def NumDeriv(self, params, roipos=None, constants=None, eps=1e-6):
        """Central differences of ExpectedValue: deriv[:, k] = (mu(theta + eps e_k) -
        mu(theta - eps e_k)) / (2 eps) in float32, with the 2K shifted parameter sets of all spots
        evaluated in one GPU call. Returns (deriv [n, K, *sampleshape], mu(theta))."""
        params, constants, roipos = self._checkparams(params, constants, roipos)
        n, K = params.shape
        ev = self.ExpectedValue(params, roipos, constants)
        shifted = np.empty((n, 2 * K, K), dtype=np.float32)
        shifted[...] = params[:, None, :]
        for k in range(K):  # theta_k +- eps rounded to float32, as a float32 parameter array holds it
            shifted[:, k, k] = params[:, k] + np.float32(eps)
            shifted[:, K + k, k] = params[:, k] - np.float32(eps)
        ev_s = self.ExpectedValue(shifted.reshape(n * 2 * K, K), np.repeat(roipos, 2 * K, axis=0),
                                  np.repeat(constants, 2 * K, axis=0))
        ev_s = ev_s.reshape(n, 2 * K, *self.sampleshape)
        deriv = ((ev_s[:, :K] - ev_s[:, K:]) / np.float32(2 * eps)).astype(np.float32)
        return deriv, ev

    def NumCRLB(self, params, roipos=None, constants=None, eps=1e-4, useNumDeriv=True):
        """CRLB from the definition, in float64 on the host: FI = J diag(1/mu) J^T over the
        pixels, with J the numerical (NumDeriv, step eps) or analytic (Derivatives) Jacobian and
        mu clamped at 1e-9; CRLB = sqrt(|diag(FI^-1)|)."""
        deriv, ev = (self.NumDeriv(params, roipos, constants, eps) if useNumDeriv
                     else self.Derivatives(params, roipos, constants))
        n, K = deriv.shape[:2]
        J = deriv.reshape(n, K, -1).astype(np.float64)
        w = 1.0 / np.maximum(ev.reshape(n, -1).astype(np.float64), 1e-9)
        fi = np.einsum("nkp,np,nlp->nkl", J, w, J)
        var = np.linalg.inv(fi)
        return np.sqrt(np.abs(np.diagonal(var, axis1=1, axis2=2)))

    def GetLevMarParams(self):
        lmp = LevMarParams()
        self._Estimator_GetLMParams(self.inst, lmp)
        self.lmparams = lmp
        return lmp

    def SetLevMarParams(self, lambda_=1e-15, iterations=50, lmFactor=0.0):
        self.lmparams = LevMarParams()
        self.lmparams.lambda_ = lambda_
        self.lmparams.iterations = iterations
        self.lmparams.factor = lmFactor
        self._Estimator_SetLMParams(self.inst, self.lmparams)

    def Estimate(self, imgs, roipos=None, constants=None, initial=None, return_iterations=False):
        """Fit every ROI. Returns (params, diag, traces) like the reference; with
        return_iterations=True also the per-spot iteration counts (i+1 at the stop,
        maxIterations+1 when capped)."""
        numspots = len(imgs)
        traceBufLen = self.lmparams.iterations
        imgs = np.ascontiguousarray(imgs, dtype=np.float32)
        if not np.array_equal(imgs.shape[1:], self.sampleshape):
            raise ValueError(f"Sample images are expected to have shape {self.sampleshape}. Given: {imgs.shape[1:]}")
        iterations = np.zeros(numspots, np.int32)
        params = np.zeros((numspots, self.numparams), dtype=np.float32)
        trace = np.zeros((numspots, traceBufLen, self.numparams), dtype=np.float32)
        diag = np.zeros((numspots, self.numdiag), dtype=np.float32)
        params, constants, roipos = self._checkparams(params, constants, roipos)
        if initial is not None:
            initial = np.ascontiguousarray(initial, dtype=np.float32)
            if not np.array_equal(initial.shape, [numspots, self.numparams]):
                raise ValueError(f"Initial value array is expected to have shape {[numspots, self.numparams]}. "
                                 f"Given: {initial.shape}")
        if numspots > 0:
            self._Estimator_Estimate(self.inst, numspots, imgs, constants, roipos, initial, params,
                                     diag if diag.size else np.zeros(1, np.float32), iterations, trace, traceBufLen)
        traces = [trace[k, 0:iterations[k], :] for k in range(numspots)]
        if return_iterations:
            return params, diag, traces, iterations
        return params, diag, traces

    # ------------------------------------------------------------------ extensions
    def EstimateWithCRLB(self, imgs, constants=None, initial=None):
        """Fused fit + Fisher/CRLB + chi-square (one kernel). Returns (params, iterations, crlb, chisq)."""
        imgs = np.ascontiguousarray(imgs, dtype=np.float32)
        n = len(imgs)
        if not np.array_equal(imgs.shape[1:], self.sampleshape):
            raise ValueError(f"Sample images are expected to have shape {self.sampleshape}. Given: {imgs.shape[1:]}")
        params = np.zeros((n, self.numparams), np.float32)
        its = np.zeros(n, np.int32)
        crlb = np.zeros((n, self.numparams), np.float32)
        chisq = np.zeros(n, np.float32)
        _, constants, _ = self._checkparams(params, constants, None)
        if initial is not None:
            initial = np.ascontiguousarray(initial, dtype=np.float32)
        if n > 0:
            self._EstimateCRLB(self.inst, n, imgs, constants if self.numconst else None, initial, params, its, crlb,
                               chisq)
            check_error("EstimateWithCRLB")
        return params, its, crlb, chisq

    def EstimateDevice(self, imgs, constants=None, initial=None, with_crlb=True, trace_len=0, stream=None,
                       out=None):
        """Fit torch CUDA tensors on the device (no host copies, no synchronisation).
        Returns dict(params, iterations, crlb, chisq[, trace]) of torch tensors; `out` may
        supply preallocated tensors for any of them."""
        import torch
        n = imgs.shape[0]
        dev = imgs.device
        assert imgs.is_cuda and imgs.dtype == torch.float32 and imgs.is_contiguous()
        out = dict(out or {})
        out.setdefault("params", torch.empty((n, self.numparams), device=dev, dtype=torch.float32))
        out.setdefault("iterations", torch.empty(n, device=dev, dtype=torch.int32))
        if with_crlb:
            out.setdefault("crlb", torch.empty((n, self.numparams), device=dev, dtype=torch.float32))
            out.setdefault("chisq", torch.empty(n, device=dev, dtype=torch.float32))
        if trace_len > 0:
            out.setdefault("trace", torch.zeros((n, trace_len, self.numparams), device=dev, dtype=torch.float32))
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        self._lib.PB200_EstimateDevice(self.inst, n, _ptr(imgs), _ptr(constants), _ptr(initial), _ptr(out["params"]),
                                       _ptr(out["iterations"]), _ptr(out.get("trace")), int(trace_len),
                                       _ptr(out.get("crlb")), _ptr(out.get("chisq")), ct.c_void_p(s.cuda_stream))
        check_error("EstimateDevice")
        return out

    def ExpectedValueDevice(self, params, constants=None, derivatives=False, stream=None):
        """ExpectedValue (and Derivatives) of torch CUDA tensors on the device."""
        import torch
        n = params.shape[0]
        R = int(self.sampleshape[0])
        ev = torch.empty((n, R, R), device=params.device, dtype=torch.float32)
        deriv = torch.empty((n, self.numparams, R, R), device=params.device, dtype=torch.float32) if derivatives \
            else None
        s = stream if stream is not None else torch.cuda.current_stream(params.device)
        self._lib.PB200_ExpectedValueDevice(self.inst, n, _ptr(params), _ptr(constants), _ptr(ev), _ptr(deriv),
                                            ct.c_void_p(s.cuda_stream))
        check_error("ExpectedValueDevice")
        return (deriv, ev) if derivatives else ev

    def SetKernelConfig(self, lanes_per_roi=0, threads_per_block=0, variant=None):
        """Lanes per ROI (2, 4, 8, 16, 32; 0 = automatic), threads per block (64..256; 0 =
        automatic) and, for the Gaussian models, the kernel family (0 = column-blocked, 1 =
        generic per-pixel table)."""
        rc = self._lib.PB200_SetKernelConfig(self.inst, int(lanes_per_roi), int(threads_per_block))
        if rc == 0 and variant is not None:
            rc = self._lib.PB200_SetKernelVariant(self.inst, int(variant))
        if rc != 0:
            raise ValueError("invalid kernel configuration")
        prev = self.kernel_config_setting()
        self._kernel_setting = (int(lanes_per_roi), int(threads_per_block), prev[2] if variant is None else int(variant))

    def kernel_config_setting(self):
        """(lanes_per_roi, threads_per_block, variant) as last given to SetKernelConfig (0 =
        automatic), for restoring a configuration; GetKernelConfig gives the values in use."""
        return getattr(self, "_kernel_setting", (0, 0, 0))

    def SetHostPipeline(self, rois_per_chunk=0, slots=4):
        """Chunking of the host-array calls (Estimate, EstimateWithCRLB, ...): ROIs per chunk
        (0 = automatic: up to 64 MB of samples, ramped up over the first three chunks, and the
        streamed path where it is faster; an explicit size always takes the chunked path) and the
        number of chunks in flight (2..8), whose copies overlap the fits of the others."""
        if self._lib.PB200_SetHostPipeline(self.inst, int(rois_per_chunk), int(slots)) != 0:
            raise ValueError("invalid host pipeline configuration")

    def GetKernelConfig(self):
        g, t = ct.c_int(), ct.c_int()
        self._lib.PB200_GetKernelConfig(self.inst, ct.byref(g), ct.byref(t))
        return g.value, t.value

    # ------------------------------------------------------------------ misc
    def Destroy(self):
        if self.inst is not None:
            self._Estimator_Delete(self.inst)
            self.inst = None

    def NumConstants(self):
        return self.numconst

    def ParamFormat(self):
        return self._Estimator_ParamFormat(self.inst).decode("utf-8")

    def ParamIndex(self, paramName):
        if type(paramName) == list:
            return [self.param_names.index(n) for n in paramName]
        return self.param_names.index(paramName)

    def NumParams(self):
        return self.numparams

    def SampleCount(self):
        return self.samplecount

    def NumDiag(self):
        return self.numdiag

    def ParamLimits(self):
        """(min[NumParams], max[NumParams])"""
        return self.limits[:, 0], self.limits[:, 1]

    def __enter__(self):
        return self

    def __exit__(self, *args):
        self.Destroy()


def _last_error(ctx) -> str:
    try:
        ctx.smlm.lib.PB200_GetLastError.restype = ct.c_char_p
        return (ctx.smlm.lib.PB200_GetLastError() or b"").decode()
    except Exception:
        return "unknown error"
