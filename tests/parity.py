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
