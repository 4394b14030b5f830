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


def test_nonconi_devices_gather_equals_one_call(monkeypatch):
    """zpm_batch_devices over three (host-thread) devices, each chunk's points
    from the reference's non-coni C setup and kernel standing in for the
    device call: the gathered points equal one call's, in p order."""
    from oracle import nonconi, ref
    from pfvs_b200 import gpu, multi
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    G = np.load(os.path.join(ROOT, "tests", "golden", "nonconi.npz"))
    kappa, Mb, ps = G["c4_kappa"], G["c4_Mbasis"], G["c4_ps"]
    Qmax = int(G["c4_scal"][1])
    geoms = [dict(kappa=kappa, Mbasis=Mb, Q=Qmax, dilation=1.0)]
    qmax = nonconi.qmax_of(Qmax, 1.0)

    def fake(geoms_, sub_ps, sub_pgeo, device=0, **kw):
        Ms, Ks, qs, pid = [], [], [], []
        for i, p in enumerate(sub_ps):
            st, C, M, Kn, q = nonconi.ref_points(kappa, Mb, p, Qmax, qmax)
            Ms.append(M); Ks.append(Kn); qs.append(q); pid.append(np.full(len(q), i))
        M, Kn, q, pidx = np.vstack(Ms), np.vstack(Ks), np.concatenate(qs), np.concatenate(pid).astype(np.int64)
        o = np.lexsort(tuple(Kn[:, j] for j in range(Kn.shape[1] - 1, -1, -1)) +
                       tuple(M[:, j] for j in range(M.shape[1] - 1, -1, -1)) + (pidx,))
        return M[o], Kn[o], q[o], pidx[o], np.zeros(len(sub_ps), np.int8), 0.01 * (device + 1), {}
    monkeypatch.setattr(gpu, "zpm_batch_multi_ex", fake)
    got = multi.zpm_batch_devices(geoms, ps, np.zeros(len(ps), np.int32), devices=[0, 1, 2], chunk=16)
    one = fake(geoms, ps, np.zeros(len(ps), np.int32))
    for a, b in zip(got[:5], one[:5]):
        np.testing.assert_array_equal(a, b)
    assert len(got[2]) > 100 and got[5] > 0
