"""Helpers shared by the parity tests: lay a workload out as one
multi-geometry call (one geometry entry per (CY, dilation), as the
reference's mixed-dilation caller does, pfvs/coni.py:701-738) and compute the
oracle's answer for it in the ABI's canonical order."""
import numpy as np

from oracle import pfo, ref


def layout(w):
    """(geoms, ps, pgeo, hs): the workload as coni_batch_multi arguments."""
    geoms, ps, pgeo, hs = [], [], [], []
    for k, ((gi, dil), idx) in enumerate(sorted(w.groups().items())):
        g = w.geoms[gi]
        geoms.append(dict(kappa=g.kappa, Mbasis=g.Mbasis, Q=g.Q, dilation=dil, M0min=13))
        hs.append(g.h11)
        for i in idx:
            ps.append(np.asarray(w.ps[i], dtype=np.int64))
            pgeo.append(k)
    return geoms, ps, np.array(pgeo, dtype=np.int32), hs


def _pad(a, MH=64):
    out = np.zeros((a.shape[0], MH), dtype=np.int64)
    out[:, :a.shape[1]] = a
    return out


def expected(geoms, ps, pgeo, which="oracle"):
    """The oracle's (or the reference build's) points for the layout, as
    (M, Kn, q, pidx, status) with MH-wide rows in canonical order."""
    Ms, Ks, qs, pids, status = [], [], [], [], np.zeros(len(ps), dtype=np.int32)
    for k, g in enumerate(geoms):
        idx = np.flatnonzero(pgeo == k)
        if not len(idx):
            continue
        P = np.array([ps[i] for i in idx])
        if which == "oracle":
            M, Kn, q, pl, st, _ = pfo.coni_batch(g["kappa"], g["Mbasis"], P, g["Q"], g["dilation"],
                                                 g["M0min"])
        else:
            M, Kn, q, pl, st, _ = ref.coni_batch(g["kappa"], g["Mbasis"], P, g["Q"], g["dilation"],
                                                 g["M0min"])
        status[idx] = st
        Ms.append(_pad(M)); Ks.append(_pad(Kn)); qs.append(q); pids.append(idx[pl])
    if Ms:
        M, Kn, q, pidx = np.vstack(Ms), np.vstack(Ks), np.concatenate(qs), np.concatenate(pids)
    else:
        M = Kn = np.zeros((0, 64), np.int64)
        q = pidx = np.zeros(0, np.int64)
    o = pfo.canonical_order(M, Kn, pidx)
    return M[o], Kn[o], q[o], pidx[o], status


def _ref_chunk(args):
    g, P, idx = args
    M, Kn, q, pl, st, nodes = ref.coni_batch(g["kappa"], g["Mbasis"], P, g["Q"], g["dilation"],
                                             g["M0min"])
    return idx, M, Kn, q, pl, st, nodes


def _oracle_one(args):
    g, p = args
    from oracle.ref import linmin_of, qmax_of
    M, Kn, q, st, nodes = pfo.direction(g["kappa"], g["Mbasis"], np.asarray(p, np.int64), g["Q"],
                                        qmax_of(g["Q"], g["dilation"]), linmin_of(g["M0min"]))
    return M, Kn, q, st


def expected_full(geoms, ps, pgeo, threads=None, chunk=32, oracle_procs=None, oracle_fallback=True):
    """
    The expected points of a whole workload at sizes the oracle alone cannot
    follow: the reference build (oracle/_ref) over every direction, on
    `threads` host threads (its ctypes calls release the GIL), and the oracle
    restatement for the directions the reference's C batch leaves at status 1
    (an exact setup value beyond its int64 path; the reference hands those to
    flint/GMP code that is not built here), in a spawn process pool.  With
    oracle_fallback False those directions stay unfinished (source -1): the
    oracle prunes only with the GCD rows that fit int64, which at h11 = 60
    and deep dilations makes its trees too large to follow.

    Returns (M, Kn, q, pidx, status, source) in the canonical order: status
    per direction as the finishing implementation reports it, source 0 for
    the reference build, 1 for the oracle, -1 where neither finished.
    """
    import concurrent.futures as cf
    import multiprocessing as mp
    import os
    threads = threads or os.cpu_count() or 1
    jobs = []
    for k, g in enumerate(geoms):
        idx = np.flatnonzero(pgeo == k)
        for c in range(0, len(idx), chunk):
            ii = idx[c:c + chunk]
            jobs.append((g, np.array([ps[i] for i in ii]), ii))
    n = len(ps)
    status = np.zeros(n, dtype=np.int32)
    source = np.zeros(n, dtype=np.int8)
    Ms, Ks, qs, pids = [], [], [], []
    with cf.ThreadPoolExecutor(threads) as ex:
        for idx, M, Kn, q, pl, st, _ in ex.map(_ref_chunk, jobs):
            status[idx] = st
            ok = st[pl] == 0 if len(pl) else np.zeros(0, bool)
            Ms.append(_pad(M[ok])); Ks.append(_pad(Kn[ok])); qs.append(q[ok]); pids.append(idx[pl[ok]])
    redo = np.flatnonzero(status == 1)
    if len(redo) and oracle_fallback:
        procs = min(len(redo), oracle_procs or os.cpu_count() or 1)
        with cf.ProcessPoolExecutor(procs, mp_context=mp.get_context("spawn")) as ex:
            res = ex.map(_oracle_one, [(geoms[pgeo[i]], ps[i]) for i in redo], chunksize=1)
            for i, (M, Kn, q, st) in zip(redo, res):
                status[i] = st
                source[i] = 1 if st == 0 else -1
                if st == 0 and len(q):
                    Ms.append(_pad(M)); Ks.append(_pad(Kn)); qs.append(q)
                    pids.append(np.full(len(q), i, np.int64))
    source[(status != 0) & (source == 0)] = -1
    M, Kn = np.vstack(Ms) if Ms else np.zeros((0, 64), np.int64), np.vstack(Ks) if Ks else np.zeros((0, 64), np.int64)
    q = np.concatenate(qs) if qs else np.zeros(0, np.int64)
    pidx = np.concatenate(pids).astype(np.int64) if pids else np.zeros(0, np.int64)
    o = pfo.canonical_order(M, Kn, pidx)
    return M[o], Kn[o], q[o], pidx[o], status, source


def assert_same(got, exp, ok_mask=None):
    """GPU (M, Kn, q, pidx) equal to the expected arrays, element for
    element; ok_mask restricts to directions the reference finished."""
    gM, gK, gq, gp = got[:4]
    eM, eK, eq, ep = exp[:4]
    if ok_mask is not None:
        sel_g = ok_mask[gp] if len(gp) else np.zeros(0, bool)
        sel_e = ok_mask[ep] if len(ep) else np.zeros(0, bool)
        gM, gK, gq, gp = gM[sel_g], gK[sel_g], gq[sel_g], gp[sel_g]
        eM, eK, eq, ep = eM[sel_e], eK[sel_e], eq[sel_e], ep[sel_e]
    np.testing.assert_array_equal(gp, ep)
    np.testing.assert_array_equal(gq, eq)
    np.testing.assert_array_equal(gM, eM)
    np.testing.assert_array_equal(gK, eK)
