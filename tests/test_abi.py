"""C-ABI library: builds for sm_100a, loads, and exports every function include/photonpy_b200.h
declares. No compute call is made (runs without a GPU)."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "photonpy_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = []
    for m in re.finditer(r"^\s*(?!typedef|struct|#)[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", txt, flags=re.M):
        names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_reference_abi():
    names = declared_functions()
    for must in ["Estimator_Estimate", "Estimator_ChiSquareAndCRLB", "Estimator_ComputeDerivatives",
                 "Estimator_ComputeExpectedValue", "Gauss2D_CreatePSF_XYIBg", "Gauss2D_CreatePSF_XYIBgSigmaXY",
                 "Gauss2D_CreatePSF_XYZIBg", "CSpline_CreatePSF", "CSpline_Compute", "Context_Create",
                 "Context_Destroy", "Estimator_GetParamLimits", "Estimator_SetLMParams", "EstimQueue_Create",
                 "EstimQueue_Delete", "EstimQueue_Schedule", "EstimQueue_Flush", "EstimQueue_IsIdle",
                 "EstimQueue_GetResultCount", "EstimQueue_GetQueueLength", "EstimQueue_GetResults",
                 "GLRT_CreatePSF", "Gauss2D_CreatePSF_XYITiltedBg", "Gauss2D_CreatePSF_XYITiltedBgSigmaXY",
                 "Gauss2D_EstimateIntensityBg", "SpotDetector_Configure", "SpotDetector_ProcessFrame",
                 "SpotDetector_DestroyFactory", "ExtractROIs", "PSFCorrelationSpotDetector_Configure",
                 "SpotExtractionQueue_Create"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from photonpy_b200 import lib
    L = lib.load_library()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_library_is_sm100a():
    """The shared library carries sm_100a device code (cuobjdump --list-elf lists the cubins)."""
    import shutil
    import subprocess
    from photonpy_b200 import lib
    lib.load_library()
    tool = shutil.which("cuobjdump") or "/usr/local/cuda/bin/cuobjdump"
    if not os.path.exists(tool):
        return
    out = subprocess.run([tool, "--list-elf", lib.LIB_PATH], capture_output=True, text=True).stdout
    assert "sm_100a" in out


def test_struct_layouts_match_reference_ctypes():
    """ctypes layouts used by photonpy's Python bindings match the C header."""
    import photonpy_b200 as pb
    assert ctypes.sizeof(pb.Gauss3D_Calibration) == 40
    assert ctypes.sizeof(pb.CSplineCalibration) == 32
    assert pb.CSplineCalibration.coefs.offset == 24
    assert ctypes.sizeof(pb.LevMarParams) == 12
    assert ctypes.sizeof(pb.EstimatorProperties) == 20
    from photonpy_b200 import spotdetect
    assert ctypes.sizeof(spotdetect.SpotDetector) == 32
    assert spotdetect.SpotDetector.backgroundImagePtr.offset == 24


def test_mixed_standalone_threshold_setting():
    """The mixed plans' standalone threshold is host state: set, read back, restored by a
    negative value (no GPU call)."""
    from photonpy_b200 import mixed
    assert mixed.standalone_min() == 0
    try:
        mixed.set_standalone_min(1 << 30)
        assert mixed.standalone_min() == 1 << 30
        mixed.set_standalone_min(256)
        assert mixed.standalone_min() == 256
    finally:
        mixed.set_standalone_min(None)
    assert mixed.standalone_min() == 0
