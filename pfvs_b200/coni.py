"""
coniZp on the device: every coni PFV of each p-vector's direction, at any
dilation -- the reference's coniZp (pfvs/coni.py:1171-1223) and its
exhaustive driver _coni_exhaustive (pfvs/coni.py:784-857).

Both device stages are this library's kernels:
  1. the dilation bound of every direction (k_mu0 through
     pfvs_b200.dilation): b = ceil(Q / mu0), every PFV of the direction
     having dilation below Q / mu0;
  2. the batched coniZpM search with the post-processing on the device
     (pfg_coni_pfvs) at each direction's dilation, all the distinct
     dilations in one multi-geometry call, as the reference's _zpm
     (pfvs/coni.py:701-738) makes each distinct dilation its own geometry
     entry.

Routing (pfvs/coni.py:809-813).  A direction with a bound is searched to
grid_up(b) (the bound rounded up onto the grid of ratio 2^(1/16), so nearby
bounds share one search); a direction without one at fallback_dilation, and
reported incomplete.  The reference may instead split a direction at a
dilation D0 (ZpM up to D0 plus coniZpK above it on the CPU) where its cost
model favours that; every plan gives the same PFVs (its
tests/test_coni_zpk.py:172-205), and searching every bounded direction to its
bound on the device is the reference's own plan when ZpM is the cheaper
side at every split.

Differences from the reference, both reported rather than hidden:
  - a direction whose bound the device does not decide (pfvs_b200.dilation:
    an exact value beyond 128 bits; the reference decides these with
    python-flint on the host) is treated as one without a bound: searched at
    fallback_dilation, complete False;
  - a direction the device search reports with a negative status (or more
    than max_N_pfvs PFVs) contributes no PFVs and is marked incomplete,
    where the reference re-runs it on the CPU.
"""
import numpy as np

from . import dilation, gpu


def _canonical(Ks, Ms, keys):
    """Deduplicate PFVs and sort them by key (p-vector), then (M, K)
    (pfvs/coni.py:516-531)."""
    h = Ms.shape[1]
    if len(keys) == 0:
        return Ks, Ms, np.asarray(keys, dtype=np.int64)
    A = np.unique(np.hstack([np.asarray(keys, dtype=np.int64)[:, None], Ms, Ks]), axis=0)
    return A[:, 1 + h:], A[:, 1:1 + h], A[:, 0]


def route(bceil, fallback_dilation):
    """The dilation each direction is searched at: grid_up(b) where b > 0,
    else fallback_dilation (pfvs/coni.py:809-813 with every bounded
    direction routed to its bound)."""
    bceil = np.asarray(bceil, dtype=np.int64)
    return np.where(bceil > 0, dilation.grid_up(bceil).astype(np.float64), float(fallback_dilation))


def coni_zp(kappa, Mbasis, ps, Q, M0min=13, fallback_dilation=1, device=0, max_N_pfvs=1_000_000_000,
            chunk=1 << 18, return_info=False):
    """
    Every coni PFV of each p-vector's direction, at any dilation.

    - kappa: (h11, h11, h11) triple intersection numbers in the coni basis;
      Mbasis: (h11, h11) the M-lattice basis (rows); Q the tadpole.
    - ps: (n, h11-1) p-vectors without their (zero) coni entry, in the
      Kahler cone (not checked here).

    Returns (Ks, Ms, complete): the PFVs (N, h11) sorted by p-vector, then
    (M, K), each once, and per p-vector whether its search is complete (it
    has a bound and the device search finished it).  With return_info, also
    a dict: keys (the p-vector of each PFV), status (the bound's), bceil,
    dilation (the searched one), pstat (the search's), seconds of each stage.
    """
    import time
    if fallback_dilation <= 0:
        raise ValueError(f"fallback_dilation must be > 0, got {fallback_dilation}.")
    kappa = np.asarray(kappa, dtype=np.int64)
    h = kappa.shape[0]
    ps = np.atleast_2d(np.asarray(ps, dtype=np.int64))
    if len(ps) == 0:
        raise ValueError("ps must be non-empty.")
    if ps.shape[1] != h - 1:
        raise ValueError(f"ps must have h11 - 1 = {h - 1} columns (no coni entry), got {ps.shape[1]}")
    n = len(ps)
    p_full = np.hstack([np.zeros((n, 1), dtype=np.int64), ps])
    t0 = time.perf_counter()
    bceil, bst = dilation.coni_dilation_bound_ceils(ps, kappa, Q, device=device, return_status=True)
    t1 = time.perf_counter()
    dil = route(bceil, fallback_dilation)
    pieces_K, pieces_M, pieces_k = [], [], []
    pstat = np.zeros(n, dtype=np.int8)
    for lo in range(0, n, chunk):
        idx = np.arange(lo, min(n, lo + chunk))
        Ds, gi = np.unique(dil[idx], return_inverse=True)
        geoms = [dict(kappa=kappa, Mbasis=Mbasis, Q=int(Q), dilation=float(D), M0min=M0min) for D in Ds]
        K, M, pidx, pst, _, _ = gpu.coni_pfvs_multi(geoms, p_full[idx], gi.astype(np.int32), device=device)
        counts = np.bincount(pidx, minlength=len(idx)) if len(pidx) else np.zeros(len(idx), dtype=np.int64)
        pst = pst.copy()
        pst[(pst == 0) & (counts > max_N_pfvs)] = 1
        pstat[idx] = pst
        keep = pst[pidx] == 0 if len(pidx) else np.zeros(0, dtype=bool)
        pieces_K.append(np.asarray(K[keep][:, :h]))
        pieces_M.append(np.asarray(M[keep][:, :h]))
        pieces_k.append(idx[pidx[keep]])
    t2 = time.perf_counter()
    Ks, Ms, keys = _canonical(np.vstack(pieces_K), np.vstack(pieces_M), np.concatenate(pieces_k))
    complete = (bceil > 0) & (pstat == 0)
    if not return_info:
        return Ks, Ms, complete
    info = dict(keys=keys, status=bst, bceil=bceil, dilation=dil, pstat=pstat,
                seconds_bound=t1 - t0, seconds_search=t2 - t1, seconds_total=time.perf_counter() - t0)
    return Ks, Ms, complete, info


def coniZp(data, ps, Q=None, M0min=13, fallback_dilation=1, n_jobs=-1, device="auto", cost_model=None,
           max_N_pfvs=1_000_000_000, return_formal_pfvs=False, verbosity=0):
    """
    The reference's coniZp signature (pfvs/coni.py:1171) over a geometry
    object with the reference's CYData attributes (coni, h11, h21,
    kappa_cob, M_lattice()): (Ks, Ms, complete).  n_jobs and cost_model are
    accepted and unused (the device runs every stage; see the module's
    routing note); device "auto" or "gpu" (there is no CPU path);
    return_formal_pfvs is not supported (no PFV class here).
    """
    del n_jobs, cost_model
    if device not in ("auto", "gpu"):
        raise ValueError(f"device must be 'auto' or 'gpu' (this library has no CPU path), got {device!r}")
    if return_formal_pfvs:
        raise NotImplementedError("return_formal_pfvs needs the reference's PFV class")
    if not getattr(data, "coni", True):
        raise ValueError("coniZp only applies to coni contexts.")
    if Q is None:
        Q = data.h11 + data.h21 + 4
    Ks, Ms, complete, info = coni_zp(data.kappa_cob, data.M_lattice(), ps, Q, M0min=M0min,
                                     fallback_dilation=fallback_dilation, max_N_pfvs=max_N_pfvs,
                                     return_info=True)
    if verbosity >= 1:
        has = info["bceil"] > 0
        print(f"exhaustive: {len(complete)} p-vectors, {int(np.sum(~has))} without a bound (searched at "
              f"dilation {fallback_dilation}), {int(np.sum(has))} by ZpM to their bound; bounds "
              f"{info['seconds_bound']:.3f} s, search {info['seconds_search']:.3f} s")
    return Ks, Ms, complete
