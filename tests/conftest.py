import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


GOLDEN_SETS = ["xyibg_r10", "constsigma_r9", "sigma_r11", "sigmaxy_r16", "astig_r12", "spline_r13", "tiltedbg_r11",
               "tiltedsxy_r11", "spline_tilted_r13", "spline_bgimage_r13"]


@pytest.fixture(scope="session")
def ctx():
    import photonpy_b200 as pb
    c = pb.Context()
    yield c
    c.Destroy()


@pytest.fixture(autouse=True)
def no_native_error(request):
    """GPU tests fail if any C-ABI call reported an error (the reference-compatible API only
    prints errors and leaves outputs zero)."""
    if request.node.get_closest_marker("gpu") is None:
        yield
        return
    import photonpy_b200 as pb
    from photonpy_b200 import lib
    lib.clear_error()
    yield
    msg = pb.last_error()
    assert msg == "", f"native error: {msg}"
