"""Loader of libphotonpy_b200.so — Linux counterpart of photonpy/cpp/lib.py.

The library is the CUDA product; there is no CPU fallback. If the shared library is
missing it is built in-tree with nvcc (photonpy_b200/csrc/build.py); if that fails the
import error propagates.
"""
from __future__ import annotations

import ctypes
import os
import sys
import threading

import numpy as np
import numpy.ctypeslib as ctl

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libphotonpy_b200.so")

# Nullable ndpointer types (photonpy/cpp/lib.py:21-38): None passes a NULL pointer.
FloatArrayTypeBase = ctl.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def _from_param_F32(cls, obj):
    if obj is None:
        return obj
    return FloatArrayTypeBase.from_param(obj)


NullableFloatArrayType = type("FloatArrayType", (FloatArrayTypeBase,), {"from_param": classmethod(_from_param_F32)})

IntArrayTypeBase = ctl.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def _from_param_I32(cls, obj):
    if obj is None:
        return obj
    return IntArrayTypeBase.from_param(obj)


NullableIntArrayType = type("IntArrayType", (IntArrayTypeBase,), {"from_param": classmethod(_from_param_I32)})

_load_lock = threading.Lock()
_cdll = None
# Every ctypes callback handed to the library stays referenced for the life of the process: the
# library keeps the last pointer it was given, and an SMLM object that installed it may be
# garbage-collected while another SMLM object is still in use.
_callbacks = []


def library_path() -> str:
    """The library the package loads: PHOTONPY_B200_LIBRARY when set (another build of the same
    sources, e.g. with different compile-time switches), else the in-tree build."""
    return os.environ.get("PHOTONPY_B200_LIBRARY") or LIB_PATH


def load_library() -> ctypes.CDLL:
    """Load (building first if needed) the CUDA shared library."""
    global _cdll
    with _load_lock:
        if _cdll is None:
            path = library_path()
            if path == LIB_PATH:
                from .csrc import build as _build
                if not _build.up_to_date():
                    _build.build()
            _cdll = ctypes.CDLL(path)
            _bind_common(_cdll)
    return _cdll


def _bind_common(L):
    L.PB200_GetLastError.restype = ctypes.c_char_p
    L.PB200_ClearError.restype = None
    L.PB200_LaunchCount.restype = ctypes.c_uint64
    L.CudaGetNumDevices.restype = ctypes.c_int32
    L.CudaSetDevice.argtypes = [ctypes.c_int32]
    L.CudaSetDevice.restype = ctypes.c_bool
    vp = ctypes.c_void_p
    L.PB200_SetKernelConfig.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.PB200_SetKernelConfig.restype = ctypes.c_int
    L.PB200_SetKernelVariant.argtypes = [vp, ctypes.c_int]
    L.PB200_SetKernelVariant.restype = ctypes.c_int
    L.PB200_SetHostPipeline.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.PB200_SetHostPipeline.restype = ctypes.c_int
    L.PB200_GetKernelConfig.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    L.PB200_ModelInfo.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.PB200_ModelInfo.restype = ctypes.c_int
    L.PB200_Fp32ProbeLaunch.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp]
    L.PB200_Fp32ProbeLaunch.restype = ctypes.c_double
    L.PB200_EstimateDevice.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp]
    L.PB200_ExpectedValueDevice.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp]
    L.PB200_ChiSquareAndCRLBDevice.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp, vp]


def last_error() -> str:
    return (load_library().PB200_GetLastError() or b"").decode("utf-8", "replace")


def clear_error() -> None:
    load_library().PB200_ClearError()


def launch_count() -> int:
    return int(load_library().PB200_LaunchCount())


class NativeError(RuntimeError):
    pass


def check_error(what: str) -> None:
    """Raise if the last C-ABI call on this thread reported an error."""
    msg = last_error()
    if msg:
        clear_error()
        raise NativeError(f"{what}: {msg}")


def debugPrint(msg):
    sys.stdout.write(msg.decode("utf-8"))
    return 1


class SMLM:
    """Handle to the native library (photonpy/cpp/lib.py:41-280, Linux loading)."""

    def __init__(self, debugMode=False):
        if ctypes.sizeof(ctypes.c_voidp) == 4:
            raise RuntimeError("The SMLM library can only be used with 64-bit python.")
        self.debugMode = debugMode
        self.lib = load_library()
        self.lib_path = library_path()
        smlmlib = self.lib
        self.numDevices = smlmlib.CudaGetNumDevices()
        self._CudaSetDevice = smlmlib.CudaSetDevice
        self._CudaGetDeviceInfo = smlmlib.CudaGetDeviceInfo
        self._CudaGetDeviceInfo.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.c_char_p,
                                            ctypes.c_int32]
        self._CudaGetDeviceInfo.restype = ctypes.c_bool
        self._CudaGetMemoryUse = smlmlib.CudaGetMemoryUse
        self._CudaGetMemoryUse.argtypes = [ctypes.POINTER(ctypes.c_uint64)] * 4
        self.DebugPrintCallback = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_char_p)
        self._SetDebugPrintCallback = smlmlib.SetDebugPrintCallback
        self._SetDebugPrintCallback.argtypes = [self.DebugPrintCallback]
        self.DebugImageCallbackType = ctypes.CFUNCTYPE(None, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                       ctypes.POINTER(ctypes.c_float), ctypes.c_char_p)
        self._SetDebugImageCallback = smlmlib.SetDebugImageCallback
        self._SetDebugImageCallback.argtypes = [self.DebugImageCallbackType]
        self._ShowDebugImage = smlmlib.ShowDebugImage
        self._ShowDebugImage.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                         ctl.ndpointer(np.float32, flags="aligned, c_contiguous"), ctypes.c_char_p]
        self.SetDebugPrintCallback(debugPrint)

        def imgcb(w, h, n, data, label):
            images = np.ctypeslib.as_array(data, shape=(n, h, w)) * 1
            if self.debugImageCallback is not None:
                self.debugImageCallback(images, label.decode("utf-8"))

        self.debugImageCallback = None
        self.debugImageCFunction = self.DebugImageCallbackType(imgcb)
        _callbacks.append(self.debugImageCFunction)
        self._SetDebugImageCallback(self.debugImageCFunction)

    def GetCudaMemUse(self):
        vals = [ctypes.c_uint64() for _ in range(4)]
        self._CudaGetMemoryUse(*vals)
        return tuple(v.value for v in vals)

    def GetCudaDevices(self):
        names = []
        for d in range(self.numDevices):
            mpu = ctypes.c_int32()
            namebuf = ctypes.create_string_buffer(100)
            self._CudaGetDeviceInfo(d, ctypes.byref(mpu), namebuf, 100)
            names.append(namebuf.value.decode("utf-8"))
        return names

    def SetCudaDevice(self, idx):
        return self._CudaSetDevice(idx)

    def SetDebugPrintCallback(self, fn):
        self.dbgPrintCallback = self.DebugPrintCallback(fn)
        _callbacks.append(self.dbgPrintCallback)
        self._SetDebugPrintCallback(self.dbgPrintCallback)

    def SetDebugImageCallback(self, fn):
        self.debugImageCallback = fn

    def ShowDebugImage(self, img, label):
        if len(img.shape) == 2:
            img = np.array([img])
        img = np.ascontiguousarray(img, dtype=np.float32)
        self._ShowDebugImage(img.shape[2], img.shape[1], img.shape[0], img, label.encode("utf-8"))

    def Close(self):
        # The library stays loaded for the life of the process (dlclose of a CUDA library
        # with live device state is unsafe); nothing to release here.
        self.lib = None

    def __enter__(self):
        return self

    def __exit__(self, *args):
        self.Close()
