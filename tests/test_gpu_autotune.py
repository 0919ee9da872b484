"""The autotuner on the GPU: it times every candidate configuration, applies the fastest, and
the tuned estimator / mixed batch still gives the untuned results (the configurations change
only how work is laid out, not the arithmetic of a ROI, except the lanes per ROI, which change
the order of the pixel sums)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_tune_estimator_applies_a_candidate(ctx, tmp_path):
    import torch
    import photonpy_b200 as pb
    from photonpy_b200 import autotune, synth
    from photonpy_b200.autograd import model_id
    d = synth.xyibg(4096, seed=3)
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(10, 1.5, True)
    x = torch.from_numpy(d["samples"]).cuda()
    r = autotune.tune_estimator(est, samples=x, reps=1, use_cache=False, write_cache=False)
    cands = [tuple(c) for c in autotune.candidates(model_id(est), 10)]
    assert tuple(r["config"]) in cands
    assert all(v is None or v > 0 for v in r["timings"].values())
    v, g, t = r["config"]
    assert est.GetKernelConfig() == (g, t)
    out = est.EstimateDevice(x, with_crlb=True)
    ref = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(10, 1.5, True).Estimate(d["samples"])[0]
    assert np.mean(np.all(np.abs(out["params"].cpu().numpy()[:, :2] - ref[:, :2]) < 1e-3, axis=1)) > 0.99
    cache = tmp_path / "c.json"
    autotune.tune_estimator(est, samples=x, reps=1, use_cache=True, write_cache=True, cache_file=str(cache))
    r2 = autotune.tune_estimator(est, samples=x, reps=1, use_cache=True, cache_file=str(cache))
    assert r2["cached"]


def test_default_kernel_config(ctx):
    """Automatic lanes and threads: 2 lanes x 128 threads for flat-background Gaussians up to
    10 px wide, 4 x 256 up to 16 px; an explicit setting replaces them and 0 restores them."""
    import photonpy_b200 as pb
    gm = pb.GaussianPSFMethods(ctx)
    small = gm.CreatePSF_XYIBg(10, 1.5, True)
    assert small.GetKernelConfig() == (2, 128)
    small.SetKernelConfig(8, 192)
    assert small.GetKernelConfig() == (8, 192)
    small.SetKernelConfig(0, 0)
    assert small.GetKernelConfig() == (2, 128)
    small.SetKernelConfig(0, 0, variant=1)  # generic table kernel: 2 lanes run as 4
    assert small.GetKernelConfig() == (4, 256)
    small.SetKernelConfig(2, 0, variant=0)
    assert small.GetKernelConfig() == (2, 128)
    assert gm.CreatePSF_XYIBgSigmaXY(16, [1.5, 1.5], True).GetKernelConfig() == (4, 256)
    with pytest.raises(ValueError):
        small.SetKernelConfig(3, 0)


def test_tune_mixed_picks_a_candidate(ctx):
    import torch
    from photonpy_b200.autotune import tune_mixed
    from photonpy_b200.mixed import MixedBatch
    from test_gpu_mixed import _buckets
    buckets = _buckets(ctx, n=3000, seed=9)
    from photonpy_b200.mixed import set_standalone_min, standalone_min
    r = tune_mixed(buckets, tiles=(1, 4), budgets=(256, 128), reps=1)
    assert r["tile"] in (1, 4) and r["threads"] in (256, 128) and r["ms"] > 0
    assert r["standalone_min"] in (0, 1 << 30)
    assert standalone_min() == 0  # restored
    # every threshold timed; the all-alone plan once, the persistent kernel at each tile and budget
    assert len(r["timings"]) == 1 + 4
    set_standalone_min(r["standalone_min"])
    try:
        mb = MixedBatch(buckets, tile_rois=r["tile"], threads=r["threads"]).run()
    finally:
        set_standalone_min(None)
    torch.cuda.synchronize()
    fused = [{k: v.clone() for k, v in x.items()} for x in mb.results()]
    mb.run_plain()
    torch.cuda.synchronize()
    for f, p in zip(fused, mb.results()):
        for k in f:
            assert torch.equal(f[k], p[k]), k
    mb.close()
