"""photonpy_b200 — B200-native (sm_100a) batched Poisson-MLE PSF estimator.

Drop-in for photonpy's estimator path (photonpy/cpp/{context,estimator,gaussian,cspline,estim_queue}.py
over the Estimator_* C ABI): same classes, methods, argument order, limits and iteration
semantics, computed by hand-written CUDA kernels in libphotonpy_b200.so.
"""
from .context import Context
from .cspline import CSplineCalibration, CSplineMethods, CSplinePSF
from .estim_queue import EstimQueue, EstimQueue_Results, EstimResultDType
from .estimator import Estimator, EstimatorProperties, LevMarParams
from .gaussian import Gauss3D_Calibration, Gauss3D_CalibrationB, Gaussian, GaussianPSFMethods
from .lib import SMLM, last_error, launch_count, library_path, load_library

__all__ = [
    "Context", "Estimator", "EstimQueue", "EstimQueue_Results", "EstimResultDType", "EstimatorProperties", "LevMarParams", "GaussianPSFMethods", "Gaussian",
    "Gauss3D_Calibration", "Gauss3D_CalibrationB", "CSplineMethods", "CSplineCalibration", "CSplinePSF", "SMLM",
    "load_library", "library_path", "last_error", "launch_count",
]
