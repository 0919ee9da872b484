"""ROI sizes at the ends of the supported range (5 to 64 px) for the column-blocked and the
generic kernel: fits against the oracle (the reference's arithmetic in C), and the block size the
library reports for large ROIs, whose groups need more shared memory than 256 threads allow."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("R", [5, 32, 64])
@pytest.mark.parametrize("variant", [0, 1])
def test_roi_size_extremes(ctx, R, variant):
    import photonpy_b200 as pb
    from oracle import oracle as O
    from photonpy_b200 import synth
    synth.use_torch(None, 0)
    c = (R - 1) / 2
    d = synth.xyibg(300, seed=60 + R, R=R, xy=(c - 0.5, c + 0.5))
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(R, d["sigma"], True)
    est.SetKernelConfig(16 if R > 16 else 0, 256, variant=variant)
    lanes, threads = est.GetKernelConfig()
    assert threads in (32, 64, 128, 256)
    if R == 64:
        # 16 groups of 64x64 pixels would need more than 200 KB: the block that runs is smaller
        assert threads < 256
    params, _, _, its = est.Estimate(d["samples"], return_iterations=True)
    p_ref, it_ref = O.Model(O.XYIBG, R, sigma=d["sigma"]).fit(d["samples"])
    conv = (its <= 50) & (it_ref <= 50)
    assert conv.mean() > 0.9
    dpos = np.abs(params[conv, :2] - p_ref[conv, :2]).max(axis=1)
    assert np.mean(dpos <= 1e-3) >= 0.99, np.quantile(dpos, [0.5, 0.99, 1])
    crlb, _ = est.CRLBAndChiSquare(params, d["samples"])
    crlb_ref, _ = O.Model(O.XYIBG, R, sigma=d["sigma"]).crlb(params, d["samples"])
    assert np.quantile(np.abs(crlb - crlb_ref) / crlb_ref, 0.99) < 1e-4
    est.Destroy()
