"""
The multi-GPU path on CPU: two ranks over gloo (127.0.0.1).  Directions are
independent, so the ranks pull contiguous chunks of the batch from one shared
queue (the process group's store, pfvs_b200.multi.StoreQueue) and no
collective touches the data; the host gathers the chunks in chunk order.
Checks that every chunk is run by exactly one rank, that the gathered points
equal the one-rank result element for element in p order (the chunks'
compute here is the reference's CPU kernel, standing in for the device
call, which is the same function of a chunk), and that the timing and total
reductions give the max / sum.
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist          # noqa: E402
import torch.multiprocessing as mp        # noqa: E402

from conftest import ROOT                 # noqa: E402

N_TOTAL, CHUNK = 1000, 96


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _chunk_points(geoms, ps, pgeo, lo, hi):
    from parity import expected
    M, Kn, q, pidx, st = expected(geoms, ps[lo:hi], pgeo[lo:hi], "ref")
    return M, Kn, q, pidx, st.astype(np.int8)


def _rank_main(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    from pfvs_b200 import multi
    pg = None
    try:
        wsize, r, local, pg = bench.dist_init()
        assert (wsize, r, local) == (world, rank, rank)
        w = bench.workload_for("mixed", N_TOTAL // world, wsize)
        geoms, ps, pgeo = bench.layout(w, list(range(len(w))))
        assert len(ps) == N_TOTAL
        bounds = multi.chunk_bounds(len(ps), CHUNK)
        store = pg.distributed_c10d._get_default_store()
        mine = multi.run_chunks(multi.StoreQueue(store, "test/points"), len(bounds),
                                lambda k: _chunk_points(geoms, ps, pgeo, *bounds[k]))
        parts = [None] * world
        dist.all_gather_object(parts, mine)
        t = bench.allmax(pg, float(rank + 1) * 1.5)
        s = bench.allsum(pg, float(len(mine)))
        bench.barrier(pg)
        if rank == 0:
            claimed = [sorted(p) for p in parts]
            merged = {}
            for p in parts:
                merged.update(p)
            got = multi.gather_points(merged, bounds)
            from parity import expected
            one = expected(geoms, ps, pgeo, "ref")
            for a, b in zip(got, one):
                np.testing.assert_array_equal(a, b)
            q.put((claimed, len(bounds), len(one[2]), t, s))
        else:
            q.put(None)
    finally:
        if pg is not None:
            pg.destroy_process_group()


def test_two_ranks_pull_chunks_and_gather_in_p_order():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = [x for x in (q.get(timeout=10) for _ in range(world)) if x is not None]
    claimed, n_chunks, n_points, t, s = res[0]
    # every chunk run by exactly one rank, both ranks took part
    flat = sorted(k for c in claimed for k in c)
    assert flat == list(range(n_chunks))
    assert all(len(c) > 0 for c in claimed)
    assert n_points > 1000
    assert t == 3.0                          # max over ranks of (rank + 1) * 1.5
    assert s == float(n_chunks)              # chunks summed over the ranks


def test_local_queue_hands_each_chunk_out_once():
    import threading
    import sys
    sys.path.insert(0, ROOT)
    from pfvs_b200 import multi
    q = multi.LocalQueue()
    seen, mu = [], threading.Lock()

    def worker():
        got = multi.run_chunks(q, 500, lambda k: k)
        with mu:
            seen.extend(got)
    ths = [threading.Thread(target=worker) for _ in range(8)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    assert sorted(seen) == list(range(500))
    bounds = multi.chunk_bounds(1001, 100)
    assert bounds[0] == (0, 100) and bounds[-1] == (1000, 1001) and len(bounds) == 11
