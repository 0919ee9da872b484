"""Host-side library plumbing that needs no GPU: the debug-print callback stays valid after the
Context (and SMLM object) that installed it is destroyed and collected."""
import gc


def test_debug_callback_survives_context_destroy(capsys):
    import photonpy_b200 as pb
    from photonpy_b200 import lib
    keep = pb.Context()
    tmp = pb.Context()  # installs its own callback, replacing keep's
    tmp.Destroy()
    del tmp
    gc.collect()
    L = lib.load_library()
    # an argument error is reported through the debug-print callback without touching the GPU
    L.CSpline_Compute(None, None, None, 0)
    assert "CSpline_Compute" in lib.last_error()
    lib.clear_error()
    keep.Destroy()
