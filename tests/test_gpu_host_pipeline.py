"""Host-array calls at sizes that take the streamed path (one LM launch that fits the ROIs while
a copy stream brings them in, ready flags per 1024-ROI block) give exactly the results of the
device-pointer call on the same ROIs, as does the slot pipeline (chunked launches) that an
explicit chunk size selects; inputs from pageable numpy memory and from pinned torch memory."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device(est, samples, initial=None):
    import torch
    x = torch.from_numpy(samples).cuda()
    init = torch.from_numpy(initial).cuda() if initial is not None else None
    out = est.EstimateDevice(x, initial=init, with_crlb=True)
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("chunk", [0, 8192])
def test_host_calls_equal_device_call(ctx, chunk):
    import photonpy_b200 as pb
    from photonpy_b200 import synth
    synth.use_torch(None, 0)
    d = synth.sigmaxy(40_000, seed=51)
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBgSigmaXY(d["R"], d["sigma"], True)
    est.SetHostPipeline(chunk, 4)
    ref = _device(est, d["samples"])
    p, its, crlb, chisq = est.EstimateWithCRLB(d["samples"])
    assert np.array_equal(p, ref["params"]) and np.array_equal(its, ref["iterations"])
    assert np.array_equal(crlb, ref["crlb"], equal_nan=True) and np.array_equal(chisq, ref["chisq"])
    p2, _, _, its2 = est.Estimate(d["samples"], return_iterations=True)
    assert np.array_equal(p2, ref["params"]) and np.array_equal(its2, ref["iterations"])
    est.Destroy()


def test_streamed_call_with_start_values_and_pinned_input(ctx):
    import ctypes as ct
    import torch
    import photonpy_b200 as pb
    from photonpy_b200 import synth
    synth.use_torch(None, 0)
    d = synth.astig(30_000, seed=52)
    cx, cy = d["astig"]
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYZIBg(d["R"], pb.Gauss3D_Calibration(cx[:4], cy[:4], d["zrange"]), True)
    init = (d["truth"] + np.float32(0.3)).astype(np.float32)
    ref = _device(est, d["samples"], init)
    n, K = d["samples"].shape[0], est.numparams
    h = torch.from_numpy(d["samples"]).pin_memory()
    hi = torch.from_numpy(init).pin_memory()
    out = {k: torch.empty(s, dtype=t).pin_memory() for k, s, t in
           (("params", (n, K), torch.float32), ("iterations", (n,), torch.int32), ("crlb", (n, K), torch.float32),
            ("chisq", (n,), torch.float32))}
    L = pb.load_library()
    fn = L.PB200_EstimateCRLB
    fn.argtypes = [ct.c_void_p, ct.c_int] + [ct.c_void_p] * 7
    fn.restype = None
    fn(est.inst, n, h.data_ptr(), None, hi.data_ptr(), out["params"].data_ptr(), out["iterations"].data_ptr(),
       out["crlb"].data_ptr(), out["chisq"].data_ptr())
    from photonpy_b200.lib import check_error
    check_error("PB200_EstimateCRLB")
    for k in out:
        assert np.array_equal(out[k].numpy(), ref[k], equal_nan=True), k
    est.Destroy()
