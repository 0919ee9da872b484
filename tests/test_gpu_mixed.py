"""A mixed batch over several PSF models and ROI sizes gives exactly the results of one launch
per (model, ROI size) with the lanes per ROI the plan chose, whether its buckets run in the
persistent mixed kernel (4 lanes, or 2 for large 7..10 px buckets), as launches of their own on
forked streams (each estimator's default lanes), or split between the two; a captured CUDA graph
replays the same results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NEVER = 1 << 30


@pytest.fixture
def persistent_kernel():
    """Every bucket of the MixedBatch objects created in the test runs in the persistent kernel."""
    from photonpy_b200.mixed import set_standalone_min
    set_standalone_min(NEVER)
    yield
    set_standalone_min(None)


def _buckets(ctx, n=3000, seed=5):
    import torch
    import photonpy_b200 as pb
    from photonpy_b200 import synth
    G = pb.GaussianPSFMethods(ctx)
    buckets = []
    for g in synth.mixed(n, seed=seed):
        if g["kind"] == "XYIBg":
            est = G.CreatePSF_XYIBg(g["R"], g["sigma"], True)
        elif g["kind"] == "XYIBgSigmaXY":
            est = G.CreatePSF_XYIBgSigmaXY(g["R"], g["sigma"], True)
        else:
            cx, cy = g["astig"]
            est = G.CreatePSF_XYZIBg(g["R"], pb.Gauss3D_Calibration(cx[:4], cy[:4], g["zrange"]), True)
        buckets.append((est, torch.from_numpy(g["samples"]).cuda()))
    return buckets


@pytest.mark.parametrize("tile", [1, 8, 97])
def test_mixed_launch_equals_plain_launches(ctx, tile, persistent_kernel):
    import torch
    from photonpy_b200.mixed import MixedBatch
    buckets = _buckets(ctx)
    assert len(buckets) == 12
    mb = MixedBatch(buckets, tile_rois=tile).run()
    torch.cuda.synchronize()
    fused = [{k: v.clone() for k, v in r.items()} for r in mb.results()]
    assert mb.lanes() == [4] * len(buckets)  # 3000 ROIs: no bucket is large enough for 2 lanes
    mb.run_plain()
    torch.cuda.synchronize()
    for f, p in zip(fused, mb.results()):
        for k in f:
            assert torch.equal(f[k], p[k]), k
    mb.close()


def test_large_small_roi_buckets_run_two_lanes(ctx, persistent_kernel):
    """A 9 px bucket of 200k ROIs runs 2 lanes per ROI (two groups per 4-lane slot) beside a
    4-lane 16 px bucket: its results equal the per-bucket launch at the estimator's default
    configuration (2 lanes per ROI) bit for bit."""
    import torch
    import photonpy_b200 as pb
    from photonpy_b200 import synth
    from photonpy_b200.mixed import MixedBatch
    synth.use_torch("cuda", 41)
    small = synth.xyibg(200_000, seed=41, R=9, xy=(3.0, 5.0))
    big = synth.sigmaxy(3000, seed=42)
    synth.use_torch(None, 0)
    G = pb.GaussianPSFMethods(ctx)
    e1 = G.CreatePSF_XYIBg(9, small["sigma"], True)
    e2 = G.CreatePSF_XYIBgSigmaXY(16, big["sigma"], True)
    buckets = [(e1, torch.from_numpy(small["samples"]).cuda()), (e2, torch.from_numpy(big["samples"]).cuda())]
    mb = MixedBatch(buckets, tile_rois=1).run()
    torch.cuda.synchronize()
    assert mb.lanes() == [2, 4]
    assert e1.GetKernelConfig()[0] == 2
    fused = [{k: v.clone() for k, v in r.items()} for r in mb.results()]
    for lanes in ("plan", None):
        mb.run_plain(lanes=lanes)
        torch.cuda.synchronize()
        for f, p in zip(fused, mb.results()):
            for k in f:
                assert torch.equal(f[k], p[k]), (lanes, k)
    mb.close()


def test_mixed_launch_close_to_default_config_launches(ctx, persistent_kernel):
    """With each estimator's own configuration (2 lanes per ROI for the 7 and 9 px buckets) the
    per-bucket launches sum those buckets' pixels in another order than the plan's 4 lanes: the
    fits agree to within float rounding on the ROIs both sides converge on, and the estimators'
    settings are restored."""
    import torch
    from photonpy_b200.mixed import MixedBatch
    buckets = _buckets(ctx, n=3000, seed=7)
    before = [b[0].GetKernelConfig() for b in buckets]
    assert any(c[0] == 2 for c in before)
    mb = MixedBatch(buckets, tile_rois=1).run()
    torch.cuda.synchronize()
    fused = [{k: v.clone() for k, v in r.items()} for r in mb.results()]
    mb.run_plain(lanes=4)
    torch.cuda.synchronize()
    assert [b[0].GetKernelConfig() for b in buckets] == before
    mb.run_plain()
    assert [b[0].GetKernelConfig() for b in buckets] == before
    mb.run_plain(lanes=None)
    torch.cuda.synchronize()
    for f, p in zip(fused, mb.results()):
        conv = ((f["iterations"] < 50) & (p["iterations"] < 50)).cpu().numpy()
        dp = (f["params"] - p["params"]).abs().cpu().numpy()[:, :2]
        assert np.mean(np.all(dp[conv] < 1e-3, axis=1)) > 0.97
    mb.close()


@pytest.mark.parametrize("standalone_min", [NEVER, 0, 2])
def test_mixed_graph_replay(ctx, standalone_min):
    """Graph replay of the persistent kernel, of forked per-bucket launches (threshold 0) and of a
    plan split between the two (threshold 2 ROIs per SM: the larger buckets alone)."""
    import torch
    from photonpy_b200.mixed import MixedBatch, set_standalone_min
    buckets = _buckets(ctx, n=2000, seed=6)
    set_standalone_min(standalone_min)
    try:
        mb = MixedBatch(buckets, tile_rois=32).run()
    finally:
        set_standalone_min(None)
    alone = mb.standalone()
    if standalone_min == NEVER:
        assert not any(alone)
    elif standalone_min == 0:
        assert all(alone)
    else:
        assert any(alone) and not all(alone)
    torch.cuda.synchronize()
    ref = [{k: v.clone() for k, v in r.items()} for r in mb.results()]
    for r in mb.results():
        for v in r.values():
            v.zero_()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        mb.capture(s)
        mb.run(s)
        mb.run(s)
    s.synchronize()
    for f, p in zip(ref, mb.results()):
        for k in f:
            assert torch.equal(f[k], p[k]), k
    mb.close()


@pytest.mark.parametrize("standalone_min", [0, 2])
def test_standalone_buckets_equal_plain_launches(ctx, standalone_min):
    """Buckets run as launches of their own on forked streams (all of them, or the larger ones
    beside the persistent kernel for the others) give the per-bucket launches' results bit for
    bit, at each estimator's default lanes per ROI (2 for the 7 and 9 px buckets)."""
    import torch
    from photonpy_b200.mixed import MixedBatch, set_standalone_min
    buckets = _buckets(ctx, n=3000, seed=8)
    set_standalone_min(standalone_min)
    try:
        mb = MixedBatch(buckets, tile_rois=1).run()
    finally:
        set_standalone_min(None)
    torch.cuda.synchronize()
    alone = mb.standalone()
    assert any(alone)
    defaults = [b[0].GetKernelConfig()[0] for b in buckets]
    lanes = mb.lanes()
    for a, l, dflt in zip(alone, lanes, defaults):
        assert l == (dflt if a else 4)
    fused = [{k: v.clone() for k, v in r.items()} for r in mb.results()]
    for r in mb.results():
        for v in r.values():
            v.zero_()
    mb.run_plain()
    torch.cuda.synchronize()
    for f, p in zip(fused, mb.results()):
        for k in f:
            assert torch.equal(f[k], p[k]), k
    mb.close()


def test_autotuner_picks_a_configuration_with_identical_results(ctx, tmp_path):
    import torch
    import photonpy_b200 as pb
    from photonpy_b200 import autotune, synth
    d = synth.sigmaxy(4000, seed=31)
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBgSigmaXY(d["R"], d["sigma"], True)
    x = torch.from_numpy(d["samples"]).cuda()
    ref = est.EstimateDevice(x)
    r = autotune.tune_estimator(est, samples=x, reps=1, cache_file=str(tmp_path / "t.json"))
    assert not r["cached"] and r["ms"] > 0
    r2 = autotune.tune_estimator(est, cache_file=str(tmp_path / "t.json"))
    assert r2["cached"] and tuple(r2["config"]) == tuple(r["config"])
    out = est.EstimateDevice(x)
    # other kernel configurations sum pixels in another order: same fits to the parity tolerance
    conv = (ref["iterations"] <= 50) & (out["iterations"] <= 50)
    dxy = (out["params"][:, :2] - ref["params"][:, :2]).abs().max(dim=1).values[conv]
    assert (dxy <= 1e-3).float().mean().item() > 0.97
    est.Destroy()
