"""PB200_EstimateCRLBNoAlloc: the fused fit + CRLB for callers that cannot allocate device
memory while fitting (real-time acquisition loops with all device memory reserved up front,
hosts whose memory must come from their own pools).

Called through the C ABI with device buffers owned by the test, it must give exactly what the
allocating entry point (PB200_EstimateDevice with a CRLB request) gives, on two calls in a row
(the second sees the scratch rows the first one left behind), and it must refuse batches above
its fixed capacity with an error instead of touching memory. This file runs last so that a
failure here does not hide the results of the other tests; it also passes on its own.
"""
import ctypes as ct

import numpy as np
import pytest

from conftest import load_golden
from helpers import cuda_estimator

pytestmark = pytest.mark.gpu

MAX_SPOTS = 32768


def _bind(L):
    vp = ct.c_void_p
    L.PB200_EstimateCRLBNoAlloc.argtypes = [vp, ct.c_int, vp, vp, vp, vp, vp, vp, vp, vp]
    L.PB200_EstimateCRLBNoAlloc.restype = ct.c_int
    L.PB200_EstimateDevice.argtypes = [vp, ct.c_int, vp, vp, vp, vp, vp, vp, ct.c_int, vp, vp, vp]
    return L


def _run(L, est, x, consts, noalloc, torch):
    n = x.shape[0]
    K = est.numparams
    dev = x.device
    params = torch.full((n, K), -1.0, device=dev)
    its = torch.full((n,), -1, dtype=torch.int32, device=dev)
    crlb = torch.full((n, K), -1.0, device=dev)
    chisq = torch.full((n,), -1.0, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    cp = None if consts is None else consts.data_ptr()
    if noalloc:
        rc = L.PB200_EstimateCRLBNoAlloc(est.inst, n, x.data_ptr(), cp, None, params.data_ptr(), its.data_ptr(),
                                         crlb.data_ptr(), chisq.data_ptr(), s)
        assert rc == 0
    else:
        L.PB200_EstimateDevice(est.inst, n, x.data_ptr(), cp, None, params.data_ptr(), its.data_ptr(), None, 0,
                               crlb.data_ptr(), chisq.data_ptr(), s)
    torch.cuda.synchronize()
    return params.cpu().numpy(), its.cpu().numpy(), crlb.cpu().numpy(), chisq.cpu().numpy()


@pytest.mark.parametrize("name", ["sigmaxy_r16", "constsigma_r9"])
def test_no_alloc_matches_allocating_entry_point_twice(name, ctx):
    import torch
    import photonpy_b200 as pb
    L = _bind(pb.load_library())
    g = load_golden(name)
    est = cuda_estimator(name, g, ctx)
    consts = g.get("constants")
    # two calls in a row with different batches: all rows of the second call are rewritten
    for sl in (slice(0, None), slice(37, 181)):
        x = torch.from_numpy(np.ascontiguousarray(g["samples"][sl])).cuda()
        c = None if consts is None else torch.from_numpy(np.ascontiguousarray(consts[sl])).cuda()
        want = _run(L, est, x, c, False, torch)
        got = _run(L, est, x, c, True, torch)
        for w, h in zip(want, got):
            assert np.array_equal(w, h)
        assert np.all(got[1] >= 1)
        assert np.all(np.isfinite(got[2]))
    assert pb.last_error() == ""
    est.Destroy()


def test_no_alloc_rejects_batches_above_capacity(ctx):
    import torch
    import photonpy_b200 as pb
    from photonpy_b200 import lib as pblib
    L = _bind(pb.load_library())
    g = load_golden("xyibg_r10")
    est = cuda_estimator("xyibg_r10", g, ctx)
    n = MAX_SPOTS + 1
    # buffers sized for the rejected batch, so nothing could be read out of bounds either way
    x = torch.zeros((n, 10, 10), device="cuda")
    params = torch.zeros((n, 4), device="cuda")
    crlb = torch.zeros((n, 4), device="cuda")
    rc = L.PB200_EstimateCRLBNoAlloc(est.inst, n, x.data_ptr(), None, None, params.data_ptr(), None,
                                     crlb.data_ptr(), None, torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    msg = pb.last_error()
    assert "32768" in msg
    pblib.clear_error()
    est.Destroy()


def test_no_alloc_full_capacity_and_no_device_allocation(ctx):
    """A batch of exactly 32768 spots uses the last row of the fixed array and still equals the
    allocating entry point; warmed-up calls leave the device's free memory unchanged."""
    import torch
    import photonpy_b200 as pb
    L = _bind(pb.load_library())
    g = load_golden("xyibg_r10")
    est = cuda_estimator("xyibg_r10", g, ctx)
    reps = -(-MAX_SPOTS // len(g["samples"]))
    smp = np.ascontiguousarray(np.tile(g["samples"], (reps, 1, 1))[:MAX_SPOTS])
    x = torch.from_numpy(smp).cuda()
    want = _run(L, est, x, None, False, torch)
    got = _run(L, est, x, None, True, torch)
    for w, h in zip(want, got):
        assert np.array_equal(w, h)
    # the last spot is a copy of a golden spot fitted in the first rows
    j = (MAX_SPOTS - 1) % len(g["samples"])
    assert np.array_equal(got[0][-1], got[0][j]) and np.array_equal(got[2][-1], got[2][j])
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        _run(L, est, x, None, True, torch)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    est.Destroy()


def test_no_alloc_rejects_more_than_six_parameters(ctx):
    """The tilted-background SigmaXY Gaussian has 8 parameters; its Fisher rows do not fit the
    fixed array's rows, so the call fails before launching anything."""
    import torch
    import photonpy_b200 as pb
    from photonpy_b200 import lib as pblib
    L = _bind(pb.load_library())
    g = load_golden("tiltedsxy_r11")
    est = cuda_estimator("tiltedsxy_r11", g, ctx)
    assert est.numparams == 8
    x = torch.from_numpy(np.ascontiguousarray(g["samples"][:64])).cuda()
    params = torch.full((64, 8), -1.0, device="cuda")
    crlb = torch.full((64, 8), -1.0, device="cuda")
    n0 = pb.launch_count()
    rc = L.PB200_EstimateCRLBNoAlloc(est.inst, 64, x.data_ptr(), None, None, params.data_ptr(), None,
                                     crlb.data_ptr(), None, torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    assert "parameters" in pb.last_error()
    assert pb.launch_count() == n0
    torch.cuda.synchronize()
    assert torch.all(params == -1.0) and torch.all(crlb == -1.0)
    pblib.clear_error()
    est.Destroy()
