"""
The multi-GPU path of bench.py on CPU: two ranks over gloo (127.0.0.1).
Directions are independent, so each rank takes a contiguous shard of the
batch and no collective touches the data; the ranks only agree on the timing
(max over ranks) and the totals (sums).  Checks that the shards partition the
batch exactly (disjoint, covering, in order, per-rank layouts consistent) and
that the reductions give the max / sum.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist          # noqa: E402
import torch.multiprocessing as mp        # noqa: E402

from conftest import ROOT                 # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, n_total, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    w, pg = None, None
    try:
        wsize, r, local, pg = bench.dist_init()
        assert (wsize, r, local) == (world, rank, rank)
        w, idx = bench.workload_slice("mixed", n_total, r, wsize)
        geoms, ps, pgeo = bench.layout(w, idx)
        # the layout keeps every direction of the shard exactly once
        got = sorted(tuple(p.tolist()) for p in ps)
        want = sorted(tuple(np.asarray(w.ps[i]).tolist()) for i in idx)
        assert got == want
        t = bench.allmax(pg, float(rank + 1) * 1.5)
        s = bench.allsum(pg, float(len(idx)))
        bench.barrier(pg)
        q.put((rank, idx[0], idx[-1], len(idx), t, s))
    finally:
        if pg is not None:
            pg.destroy_process_group()


def test_two_ranks_shard_the_batch_and_reduce_timing():
    world, n_total = 2, 1000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n_total, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=10) for _ in range(world))
    # contiguous shards [0, 500) and [500, 1000)
    assert [(r[1], r[2], r[3]) for r in res] == [(0, 499, 500), (500, 999, 500)]
    for r in res:
        assert r[4] == 3.0                   # max over ranks of (rank + 1) * 1.5
        assert r[5] == float(n_total)        # sum of the shard sizes
