"""
coniZpK on the device: the coni PFVs of each p-vector's direction with
dilation above D0 -- the reference's coniZpK (pfvs/coni.py:554-637).  With
coniZpM at ellipsoid dilation D0 it gives every coni PFV of the direction
(the reference's tests/test_coni_zpk.py:172-205).

Stages, as the reference's:
  1. the short-vector enumeration and its lattice points (k_zpk,
     pfg_coni_zpk_pfvs; the reference's C kernel coni_zpk.h:714) followed by
     coniZpM's post-processing on the device (the reference's
     _pfvs_from_points on the host, coni.py:613);
  2. a direction the kernel does not decide (status != 0) is searched by
     coniZpM up to max(its dilation bound, D0) instead (coni.py:614-625), on
     the device too; without a bound that is an IncompleteSearchError, as in
     the reference (where the device does not decide the bound itself -- an
     exact value beyond 128 bits, which the reference decides with
     python-flint -- the error says so);
  3. the PFVs with dilation delta = gcd((Z M)_r) / gcd(K_r) > D0, once each,
     sorted by p-vector then (M, K) (coni.py:627-631, 505-524).
"""
import math

import numpy as np

from . import coni, dilation, gpu
from .nonconi import IncompleteSearchError


def dilations(kappa, ps_full, Ks, Ms, keys):
    """The dilation of each PFV (K, M) of the p-vector ps_full[key] as exact
    (numerator, denominator) object arrays: delta = gcd((Z M)_r) / gcd(K_r),
    Z = kappa . p, since (Z M)_r = delta K_r (pfvs/coni.py:505-524)."""
    kappa = np.asarray(kappa).astype(object)
    keys = np.asarray(keys, dtype=np.int64)
    n = len(keys)
    num, den = np.zeros(n, dtype=object), np.zeros(n, dtype=object)
    for k in np.unique(keys):
        sel = np.flatnonzero(keys == k)
        Z = np.tensordot(kappa, np.asarray(ps_full[k]).astype(object), axes=([2], [0]))
        ZM = np.asarray(Ms[sel]).astype(object) @ Z.T
        num[sel] = [math.gcd(*[int(x) for x in r[1:]]) for r in ZM]
    den[:] = [math.gcd(*[int(x) for x in r[1:]]) for r in np.asarray(Ks).astype(object)] if n else []
    return num, den


def coni_zpk(kappa, Mbasis, ps, Q, D0, M0min=13, device=0, max_N_pfvs=1_000_000_000, return_info=False):
    """
    The coni PFVs of each p-vector's direction with dilation > D0.

    - kappa: (h11, h11, h11) triple intersection numbers in the coni basis;
      Mbasis: (h11, h11) the M-lattice basis; Q the tadpole; D0 a positive
      integer.
    - ps: (n, h11-1) p-vectors without their (zero) coni entry.

    Returns (Ks, Ms, keys): the PFVs (N, h11), sorted by p-vector (keys, the
    row of ps), then (M, K), each once.  With return_info, also a dict:
    status (the kernel's per p-vector), fallback (the rows searched by ZpM
    to their bound instead), n_points, seconds_gpu.
    """
    item = dict(kappa=kappa, Mbasis=Mbasis, ps=ps, Q=Q, M0min=M0min)
    return coni_zpk_multi([item], D0, device=device, max_N_pfvs=max_N_pfvs, return_info=return_info)[0]


def coni_zpk_multi(items, D0, device=0, max_N_pfvs=1_000_000_000, return_info=False):
    """
    coni_zpk over several geometries (one device call per geometry, as the
    reference's coniZpK is per geometry): items is a list of dicts with
    kappa, Mbasis, ps, Q and optionally M0min (13).  Returns, per item, what
    coni_zpk returns for it.
    """
    if int(D0) != D0 or D0 < 1:
        raise ValueError(f"D0 must be a positive integer, got {D0}")
    D0 = int(D0)
    out = []
    for it in items:
        kappa = np.asarray(it["kappa"], dtype=np.int64)
        h = kappa.shape[0]
        ps = np.atleast_2d(np.asarray(it["ps"], dtype=np.int64))
        if len(ps) == 0:
            raise ValueError("ps must be non-empty.")
        if ps.shape[1] != h - 1:
            raise ValueError(f"ps must have h11 - 1 = {h - 1} columns (no coni entry), got {ps.shape[1]}")
        p_full = np.hstack([np.zeros((len(ps), 1), dtype=np.int64), ps])
        g = dict(kappa=kappa, Mbasis=np.asarray(it["Mbasis"], dtype=np.int64), h=h, ps=ps, p_full=p_full,
                 Q=int(it["Q"]), M0min=it.get("M0min", 13))
        K, M, pidx, st, n_points, secs = gpu.coni_zpk_pfvs(kappa, g["Mbasis"], p_full, g["Q"], g["M0min"], D0,
                                                           max_out=max_N_pfvs, device=device)
        pieces = [(K, M, np.asarray(pidx, dtype=np.int64))]
        bad = np.flatnonzero(st != 0)
        if len(bad):
            pieces.append(_fallback(g, bad, D0, device))
        Ks = np.vstack([pc[0] for pc in pieces]).astype(np.int64)
        Ms = np.vstack([pc[1] for pc in pieces]).astype(np.int64)
        keys = np.concatenate([np.asarray(pc[2], dtype=np.int64) for pc in pieces])
        num, den = dilations(kappa, p_full, Ks, Ms, keys)
        above = np.array([int(a) > D0 * int(b) for a, b in zip(num, den)], dtype=bool)
        Ks, Ms, keys = coni._canonical(Ks[above], Ms[above], keys[above])
        if return_info:
            out.append((Ks, Ms, keys, dict(status=st, fallback=bad, n_points=n_points, seconds_gpu=secs)))
        else:
            out.append((Ks, Ms, keys))
    return out


def _fallback(g, bad, D0, device):
    """coniZpM up to max(the dilation bound, D0) on the device for the rows
    `bad` of one geometry (pfvs/coni.py:614-625): (Ks, Ms, keys)."""
    kappa, h = g["kappa"], g["h"]
    bceil, bst = dilation.coni_dilation_bound_ceils(g["ps"][bad], kappa, g["Q"], device=device, return_status=True)
    for i, b, s in zip(bad, bceil, bst):
        if b <= 0:
            why = ("s >= 0, or S not positive definite on the lattice orthogonal to p" if s == 1 else
                   f"its dilation bound is not decided on the device (status {int(s)})")
            raise IncompleteSearchError(f"p={g['ps'][i].tolist()}: its PFVs above D0 cannot be enumerated ({why})")
    Ds = np.maximum(bceil, D0)
    dil = sorted(set(int(D) for D in Ds))
    gid = {D: j for j, D in enumerate(dil)}
    geoms = [dict(kappa=kappa, Mbasis=g["Mbasis"], Q=g["Q"], dilation=float(D), M0min=g["M0min"]) for D in dil]
    K1, M1, pidx1, pst, _, _ = gpu.coni_pfvs_multi(geoms, g["p_full"][bad],
                                                   np.array([gid[int(D)] for D in Ds], dtype=np.int32),
                                                   device=device)
    if np.any(pst != 0):
        j = int(np.flatnonzero(pst != 0)[0])
        raise IncompleteSearchError(f"p={g['ps'][bad[j]].tolist()}: coniZpM up to its dilation bound did not "
                                    f"finish on the device (status {int(pst[j])})")
    return np.asarray(K1)[:, :h], np.asarray(M1)[:, :h], bad[np.asarray(pidx1, dtype=np.int64)]


def coniZpK(data, ps, D0, Q=None, M0min=13, n_jobs=-1, max_N_pfvs=1_000_000_000, return_formal_pfvs=False,
            verbosity=0):
    """
    The reference's coniZpK signature (pfvs/coni.py:554) over a geometry
    object with the reference's CYData attributes (coni, h11, h21,
    kappa_cob, M_lattice()): (Ks, Ms) grouped by p-vector (in the order of
    ps) and sorted by (M, K) within one.  n_jobs is accepted and unused (the
    device runs every stage); return_formal_pfvs is not supported (no PFV
    class here).
    """
    del n_jobs
    if return_formal_pfvs:
        raise NotImplementedError("return_formal_pfvs needs the reference's PFV class")
    if not getattr(data, "coni", True):
        raise ValueError("coniZp/coniZpM/coniZpK only apply to coni contexts. Use ZpM for non-coni PFVs.")
    if Q is None:
        Q = data.h11 + data.h21 + 4
    Ks, Ms, keys, info = coni_zpk(data.kappa_cob, data.M_lattice(), ps, Q, D0, M0min=M0min,
                                  max_N_pfvs=max_N_pfvs, return_info=True)
    if verbosity >= 1:
        print(f"ZpK: {info['n_points']} lattice points for {len(np.atleast_2d(ps))} p-vectors "
              f"({len(info['fallback'])} searched by coniZpM to their bound instead)")
    return Ks, Ms
