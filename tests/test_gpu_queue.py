"""Estimation queue (EstimQueue_* C ABI, photonpy_b200.EstimQueue).

The queue must return, for every scheduled spot, exactly what the direct fused call
(PB200_EstimateCRLB: same kernels, results independent of batch composition) returns, whatever
the batch size, stream count, launch grouping or scheduling pattern; ids, roipos and samples
travel with their spot. Modelled on photonpy/tests/psf_queue.py:test_queue_output (5 spots,
batchSize 4, 3 streams, results sorted by id equal Estimate's).
"""
import numpy as np
import pytest

from conftest import load_golden
from photonpy_b200 import synth

pytestmark = pytest.mark.gpu


def _run_queue(est, smp, batchSize, numStreams=3, chunks=1, ids=None, initial=None, constants=None, roipos=None,
               keepSamples=False, maxQueueLenInBatches=5):
    import photonpy_b200 as pb
    n = len(smp)
    ids = np.arange(n, dtype=np.int32) if ids is None else ids
    out = []
    with pb.EstimQueue(est, batchSize=batchSize, numStreams=numStreams, keepSamples=keepSamples,
                       maxQueueLenInBatches=maxQueueLenInBatches) as q:
        bounds = np.linspace(0, n, chunks + 1).astype(int)
        for a, b in zip(bounds[:-1], bounds[1:]):
            q.Schedule(smp[a:b], ids=ids[a:b], initial=None if initial is None else initial[a:b],
                       constants=None if constants is None else constants[a:b],
                       roipos=None if roipos is None else roipos[a:b])
            if q.GetResultCount() > 0:
                out.append(q.GetResults(getSampleData=keepSamples))
        q.WaitUntilDone()
        assert q.GetQueueLength() == 0
        out.append(q.GetResults(getSampleData=keepSamples))
        assert q.GetResultCount() == 0
    return out


def _merge(parts):
    r = parts[0]
    for p in parts[1:]:
        r.estim = np.concatenate([r.estim, p.estim])
        r.crlb = np.concatenate([r.crlb, p.crlb])
        r.chisq = np.concatenate([r.chisq, p.chisq])
        r.iterations = np.concatenate([r.iterations, p.iterations])
        r.ids = np.concatenate([r.ids, p.ids])
        r.roipos = np.concatenate([r.roipos, p.roipos])
        r.diagnostics = np.concatenate([r.diagnostics, p.diagnostics])
        if r.samples is not None:
            r.samples = np.concatenate([r.samples, p.samples])
    return r


def test_queue_output_matches_estimate(ctx):
    """photonpy/tests/psf_queue.py:test_queue_output with its sizes."""
    import photonpy_b200 as pb
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(11, 1.5, True)
    rng = np.random.default_rng(5)
    theta = np.repeat([[5.0, 5.0, 1000.0, 5.0]], 5, axis=0)
    smp = rng.poisson(est.ExpectedValue(theta)).astype(np.float32)
    estim1 = est.Estimate(smp)[0]
    r = _merge(_run_queue(est, smp, batchSize=4, numStreams=3))
    r.SortByID()
    assert np.array_equal(r.ids, np.arange(5))
    assert np.sum(np.abs(r.estim - estim1)) < 0.01
    est.Destroy()


@pytest.mark.parametrize("batchSize,numStreams,chunks", [(256, 3, 1), (1000, 2, 7), (37, 4, 13), (4096, 1, 3)])
def test_queue_equals_fused_call_bitwise(ctx, batchSize, numStreams, chunks):
    import photonpy_b200 as pb
    d = synth.sigmaxy(20000, seed=31)
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBgSigmaXY(d["R"], 1.7, True)
    p, it, crlb, chisq = est.EstimateWithCRLB(d["samples"])
    r = _merge(_run_queue(est, d["samples"], batchSize, numStreams, chunks))
    r.SortByID(isUnique=True)
    assert np.array_equal(r.ids, np.arange(len(p)))
    assert np.array_equal(r.estim, p)
    assert np.array_equal(r.iterations, it)
    assert np.array_equal(r.crlb, crlb, equal_nan=True)
    assert np.array_equal(r.chisq, chisq)
    est.Destroy()


def test_queue_constants_initial_roipos_and_samples(ctx):
    """Per-spot constants (ConstSigma model), initial values, roipos and kept samples travel
    with their spot; spots scheduled with and without initial values can alternate."""
    import photonpy_b200 as pb
    d = synth.constsigma(3000, seed=32)
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(d["R"], None, True)
    smp, consts = d["samples"], d["constants"].astype(np.float32)
    n = len(smp)
    init = d["truth"].astype(np.float32) * np.float32(1.05)
    rng = np.random.default_rng(3)
    ids = rng.permutation(n).astype(np.int32) + 1000
    roipos = rng.integers(0, 500, size=(n, 2)).astype(np.int32)
    p_init = est.EstimateWithCRLB(smp, constants=consts, initial=init)
    p_com = est.EstimateWithCRLB(smp, constants=consts)
    parts = []
    with pb.EstimQueue(est, batchSize=128, numStreams=2, keepSamples=True) as q:
        half = n // 2
        # first half with initial values in 4 calls, second half without, alternating modes
        for a, b in [(0, 500), (500, 1100), (1100, half)]:
            q.Schedule(smp[a:b], ids=ids[a:b], initial=init[a:b], constants=consts[a:b], roipos=roipos[a:b])
        q.Schedule(smp[half:], ids=ids[half:], constants=consts[half:], roipos=roipos[half:])
        q.WaitUntilDone()
        parts.append(q.GetResults(getSampleData=True))
    r = parts[0]
    order = np.argsort(r.ids)
    r.Filter(order)
    inv = np.argsort(ids)
    assert np.array_equal(r.ids, ids[inv])
    assert np.array_equal(r.roipos, roipos[inv])
    assert np.array_equal(r.samples, smp[inv])
    first = inv < half
    assert np.array_equal(r.estim[first], p_init[0][inv][first])
    assert np.array_equal(r.estim[~first], p_com[0][inv][~first])
    assert np.array_equal(r.crlb[~first], p_com[2][inv][~first], equal_nan=True)
    assert r.diagnostics.shape == (n, 0)
    est.Destroy()


def test_queue_partial_results_are_whole_batches(ctx):
    import photonpy_b200 as pb
    d = synth.xyibg(1000, seed=33)
    est = pb.GaussianPSFMethods(ctx).CreatePSF_XYIBg(d["R"], 1.5, True)
    with pb.EstimQueue(est, batchSize=100, numStreams=2) as q:
        q.Schedule(d["samples"], ids=np.arange(1000, dtype=np.int32))
        q.WaitUntilDone()
        assert q.IsIdle()
        assert q.GetResultCount() == 1000
        r = q.GetResults(maxResults=250)
        assert len(r.ids) == 200  # two whole batches of 100
        assert q.GetResultCount() == 800
        r2 = q.GetResults()
        assert len(r2.ids) == 800
        all_ids = np.sort(np.concatenate([r.ids, r2.ids]))
        assert np.array_equal(all_ids, np.arange(1000))
    est.Destroy()


def test_queue_golden_vectors(ctx):
    """Queue results on the reference's golden ROIs equal the direct fused call."""
    from helpers import cuda_estimator
    for name in ["xyibg_r10", "astig_r12", "spline_r13"]:
        g = load_golden(name)
        est = cuda_estimator(name, g, ctx)
        smp = g["samples"]
        p, it, crlb, chisq = est.EstimateWithCRLB(smp)
        r = _merge(_run_queue(est, smp, batchSize=64, numStreams=3, chunks=3))
        r.SortByID(isUnique=True)
        assert np.array_equal(r.estim, p), name
        assert np.array_equal(r.iterations, it), name
        est.Destroy()


def test_context_destroy_deletes_queue():
    """A queue created on a context is deleted by Context_Destroy (before its estimators)."""
    import photonpy_b200 as pb
    c = pb.Context()
    d = synth.xyibg(300, seed=34)
    est = pb.GaussianPSFMethods(c).CreatePSF_XYIBg(d["R"], 1.5, True)
    q = pb.EstimQueue(est, batchSize=64)
    q.Schedule(d["samples"])
    q.Flush()
    c.Destroy()  # queue with work possibly in flight, then the estimator
