"""The streamed LM launch's waits for arriving ROIs: with every ROI block marked as arrived its
results equal the device-pointer fit; with none marked, every wait runs out (bounded, 1-2 s),
the launch ends with its error flag set, and the context keeps working. No GPU fault is made:
the failure is a flag that nothing sets."""
import ctypes as ct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _probe(L):
    fn = L.PB200_StreamedFitProbe
    fn.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int]
    fn.restype = ct.c_int
    return fn


def test_streamed_launch_waits_and_times_out(ctx):
    import torch
    import photonpy_b200 as pb
    from photonpy_b200 import synth
    synth.use_torch(None, 0)
    d = synth.sigmaxy(5000, seed=53)
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBgSigmaXY(d["R"], d["sigma"], True)
    x = torch.from_numpy(d["samples"]).cuda()
    ref = est.EstimateDevice(x, with_crlb=False)
    n, K = x.shape[0], est.numparams
    p = torch.zeros((n, K), device="cuda")
    its = torch.zeros(n, dtype=torch.int32, device="cuda")
    fn = _probe(pb.load_library())
    assert fn(est.inst, n, x.data_ptr(), p.data_ptr(), its.data_ptr(), 1) == 0
    assert torch.equal(p, ref["params"]) and torch.equal(its, ref["iterations"])
    assert fn(est.inst, n, x.data_ptr(), p.data_ptr(), its.data_ptr(), 0) == 1
    # the context keeps working after the waits ran out
    again = est.EstimateDevice(x, with_crlb=False)
    torch.cuda.synchronize()
    assert torch.equal(again["params"], ref["params"])
    est.Destroy()
