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
    item = dict(kappa=kappa, Mbasis=Mbasis, ps=ps, Q=Q, M0min=M0min)
    return coni_zp_multi([item], fallback_dilation, device, max_N_pfvs, chunk, return_info)[0]


def coni_zp_multi(items, fallback_dilation=1, device=0, max_N_pfvs=1_000_000_000, chunk=1 << 18,
                  return_info=False):
    """
    coni_zp over several geometries at once: items is a list of dicts with
    kappa, Mbasis, ps, Q and optionally M0min (13).  The bounds are computed
    per geometry (one k_mu0 launch each); the searches of every geometry,
    each distinct (geometry, dilation) pair a geometry entry, go to the
    device together (one pipeline call per `chunk` p-vectors of the whole
    list).  Returns, per item, what coni_zp returns for it.
    """
    import time
    if fallback_dilation <= 0:
        raise ValueError(f"fallback_dilation must be > 0, got {fallback_dilation}.")
    t0 = time.perf_counter()
    per, P_all, key_all = [], [], []
    for it in items:
        kappa = np.asarray(it["kappa"], dtype=np.int64)
        h = kappa.shape[0]
        ps = np.atleast_2d(np.asarray(it["ps"], dtype=np.int64))
        if len(ps) == 0:
            raise ValueError("ps must be non-empty.")
        if ps.shape[1] != h - 1:
            raise ValueError(f"ps must have h11 - 1 = {h - 1} columns (no coni entry), got {ps.shape[1]}")
        Q = int(it["Q"])
        bceil, bst = dilation.coni_dilation_bound_ceils(ps, kappa, Q, device=device, return_status=True)
        dil = route(bceil, fallback_dilation)
        per.append(dict(kappa=kappa, h=h, Q=Q, M0min=it.get("M0min", 13), Mbasis=it["Mbasis"], n=len(ps),
                        bceil=bceil, bst=bst, dil=dil, base=len(P_all)))
        P_all.extend(np.hstack([np.zeros((len(ps), 1), dtype=np.int64), ps]))
        key_all.extend((len(per) - 1, float(D)) for D in dil)
    t1 = time.perf_counter()
    pairs = sorted(set(key_all))
    gid = {pk: g for g, pk in enumerate(pairs)}
    geoms = [dict(kappa=per[k]["kappa"], Mbasis=per[k]["Mbasis"], Q=per[k]["Q"], dilation=D, M0min=per[k]["M0min"])
             for k, D in pairs]
    pgeo_all = np.array([gid[pk] for pk in key_all], dtype=np.int32)
    N = len(P_all)
    pstat = np.zeros(N, dtype=np.int8)
    pieces = [([], [], []) for _ in per]
    item_of = np.repeat(np.arange(len(per)), [it["n"] for it in per])
    for lo in range(0, N, chunk):
        hi = min(N, lo + chunk)
        K, M, pidx, pst, _, _ = gpu.coni_pfvs_multi(geoms, P_all[lo:hi], pgeo_all[lo:hi], device=device)
        counts = np.bincount(pidx, minlength=hi - lo) if len(pidx) else np.zeros(hi - lo, dtype=np.int64)
        pst = pst.copy()
        pst[(pst == 0) & (counts > max_N_pfvs)] = 1
        pstat[lo:hi] = pst
        keep = pst[pidx] == 0 if len(pidx) else np.zeros(0, dtype=bool)
        gidx = lo + np.asarray(pidx)[keep]
        Kk, Mk = np.asarray(K)[keep], np.asarray(M)[keep]
        which = item_of[gidx] if len(gidx) else np.zeros(0, dtype=np.int64)
        for k in np.unique(which):
            sel = which == k
            h = per[k]["h"]
            pieces[k][0].append(Kk[sel][:, :h])
            pieces[k][1].append(Mk[sel][:, :h])
            pieces[k][2].append(gidx[sel] - per[k]["base"])
    t2 = time.perf_counter()
    out = []
    for k, it in enumerate(per):
        h, n, base = it["h"], it["n"], it["base"]
        Kp, Mp, kp = pieces[k]
        Ks, Ms, keys = _canonical(np.vstack(Kp) if Kp else np.zeros((0, h), np.int64),
                                  np.vstack(Mp) if Mp else np.zeros((0, h), np.int64),
                                  np.concatenate(kp) if kp else np.zeros(0, np.int64))
        ps_stat = pstat[base:base + n]
        complete = (it["bceil"] > 0) & (ps_stat == 0)
        if return_info:
            info = dict(keys=keys, status=it["bst"], bceil=it["bceil"], dilation=it["dil"], pstat=ps_stat,
                        seconds_bound=t1 - t0, seconds_search=t2 - t1, seconds_total=time.perf_counter() - t0)
            out.append((Ks, Ms, complete, info))
        else:
            out.append((Ks, Ms, complete))
    return out


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
