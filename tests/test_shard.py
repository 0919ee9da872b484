"""Multi-rank host path on CPU: world size 2 over gloo. Each rank fits its contiguous shard of
a batch (the oracle stands in for the GPU fit here) and rank 0 gathers; the result must equal
the single-process fit, and the step time is reduced with MAX."""
import os
import socket

import numpy as np
import pytest

from photonpy_b200.shard import shard_range


def test_shard_range_covers_batch():
    for n in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist
    from oracle import oracle as O
    from photonpy_b200 import synth
    from photonpy_b200.shard import gather_to_rank0, max_over_ranks, shard_range
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    d = synth.xyibg(101, seed=9)
    a, b = shard_range(len(d["samples"]), rank, world)
    m = O.Model(O.XYIBG, d["R"], sigma=d["sigma"])
    p, it = m.fit(d["samples"][a:b], nthreads=1)
    t = max_over_ranks(float(rank + 1))
    allp = gather_to_rank0(p)
    allit = gather_to_rank0(it)
    if rank == 0:
        np.savez(out_path, p=allp, it=allit, t=t)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_matches_single_process(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "gathered.npz")
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    r = np.load(out)
    from oracle import oracle as O
    from photonpy_b200 import synth
    d = synth.xyibg(101, seed=9)
    p, it = O.Model(O.XYIBG, d["R"], sigma=d["sigma"]).fit(d["samples"], nthreads=1)
    assert np.array_equal(r["p"], p)
    assert np.array_equal(r["it"], it)
    assert float(r["t"]) == 2.0
