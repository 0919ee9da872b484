"""EstimQueue_Results selections on the host (no GPU): every per-spot array follows a sort or
filter, as photonpy's users rely on (photonpy/smlm/process_movie.py:190 sorts by id)."""
import numpy as np

from photonpy_b200.estim_queue import EstimQueue_Results


def _results(n=50, K=5, keep_samples=True, seed=3):
    rng = np.random.default_rng(seed)
    ids = rng.permutation(n).astype(np.int32)
    estim = rng.uniform(0, 10, size=(n, K)).astype(np.float32)
    return EstimQueue_Results(["x", "y", "z", "I", "bg"][:K], (7, 7), estim, rng.normal(size=(n, 0)).astype(np.float32),
                              rng.uniform(size=(n, K)).astype(np.float32), rng.integers(1, 51, n).astype(np.int32),
                              rng.uniform(size=n).astype(np.float32), rng.integers(0, 100, (n, 3)).astype(np.int32),
                              rng.uniform(size=(n, 7, 7)).astype(np.float32) if keep_samples else None, ids)


def _rows(r):
    return {int(i): (tuple(r.estim[k]), tuple(r.crlb[k]), int(r.iterations[k]), float(r.chisq[k]), tuple(r.roipos[k]),
                     None if r.samples is None else float(r.samples[k].sum())) for k, i in enumerate(r.ids)}


def test_sort_by_unique_id_keeps_rows_together():
    r = _results()
    before = _rows(r)
    perm = r.SortByID(isUnique=True)
    assert np.array_equal(r.ids, np.arange(len(r.ids)))
    assert _rows(r) == before
    assert len(perm) == len(r.ids)


def test_sort_by_repeated_ids_is_stable():
    r = _results()
    r.ids = (r.ids % 7).astype(np.int32)
    order_before = [(int(i), k) for k, i in enumerate(r.ids)]
    estim_before = r.estim.copy()
    perm = r.SortByID()
    assert np.all(np.diff(r.ids) >= 0)
    assert np.array_equal(perm, [k for _, k in sorted(order_before)])
    assert np.array_equal(r.estim, estim_before[perm])


def test_filter_mask_and_box():
    r = _results(keep_samples=False)
    before = _rows(r)
    inside = (r.estim[:, 0] > 2) & (r.estim[:, 0] < 8) & (r.estim[:, 1] > 3) & (r.estim[:, 1] < 9)
    idx = r.FilterXY(2, 3, 8, 9)
    assert len(r.ids) == inside.sum() == len(idx)
    assert all(before[int(i)] == row for i, row in _rows(r).items())
    r2 = _results()
    mask = np.zeros(len(r2.ids), bool)
    mask[::3] = True
    r2.Filter(mask)
    assert len(r2.estim) == len(r2.samples) == len(r2.diagnostics) == mask.sum()


def test_col_idx_and_clone():
    r = _results()
    assert r.ColIdx("z") == 2
    assert list(r.ColIdx("I", "x")) == [3, 0]
    c = r.Clone()
    c.FilterXY(100, 100, 200, 200)
    assert len(c.ids) == 0 and len(r.ids) == 50
    assert r.CRLB() is r.crlb
