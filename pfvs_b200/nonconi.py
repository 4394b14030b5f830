"""
Non-coni ZpM on the device: the reference's ZpM (pfvs/nonconi.py:262-514),
whose lattice setup and Fincke-Pohst search run here in the library's
kernels (pfg_zpm_batch: the coni pipeline with coni = 0 -- no M0 cut, the
whole basis LLL-reduced w.r.t. mat, the non-strict GCD cut on all of K),
for every p-vector of a batch at once; the reference runs them on the CPU,
one p-vector at a time.

The post-processing is the reference's per-p host step (nonconi.py:437-495),
in exact integer numpy: primitive lattice points only (gcd(c) = 1, read off
M in the M-lattice basis: c and M's coordinates there have the same gcd,
since Binter spans a saturated sublattice), det(kappa . M) != 0 decided
exactly (determinants modulo primes, then exact Bareiss for the matrices
that vanish modulo all of them), K = Z M / gcd, Qmin <= -K.M <= Qmax; then
_allow_gcds (nonconi.py:50-84): every (a K, b M) with -a b K.M <= Qmax.

    Ks, Ms = ZpM(data, ps, Qmax=..., ellipsoid_dilation=...)   # data: CYData-like
    Ks, Ms = zpm(kappa, Mbasis, ps, Qmin, Qmax, dilation)      # arrays

The PFVs come back deduplicated in the canonical order (sorted by (K, M));
the reference returns the same set in the iteration order of a Python set.
"""
import math
from fractions import Fraction

import numpy as np

from . import gpu, intlat

PRIMES = (2147483647, 2147483629, 2147483587, 2147483579, 2147483563, 2147483549, 2147483543, 2147483497)
STATUS_TEXT = {
    -2: "more than max_N_pfvs outputs; increase max_N_pfvs",
    -8: "lattice-point coordinates exceed int32",
    -9: "the ellipsoid matrix is not positive definite, so its lattice points cannot be enumerated",
    -20: "an exact setup value exceeds the device's fixed-width integers",
    -21: "the FP64 factor of the ellipsoid could not be certified",
    -22: "the search ran past its deadline",
}


class IncompleteSearchError(RuntimeError):
    """A p-vector's search could not be completed exactly (the reference's
    pfvs.util.IncompleteSearchError)."""


def _pow_mod(x, e, p):
    """x^e mod p elementwise (int64, p < 2^31: every product below 2^62)."""
    r = np.ones_like(x)
    b = x % p
    while e:
        if e & 1:
            r = (r * b) % p
        b = (b * b) % p
        e >>= 1
    return r


def _det_mod(Ns, p):
    """det(N) mod p for a stack of integer matrices (n, m, m), entries < 2^62."""
    A = np.mod(np.asarray(Ns, dtype=np.int64), p)
    n, m, _ = A.shape
    det = np.ones(n, dtype=np.int64)
    alive = np.ones(n, dtype=bool)
    for k in range(m):
        col = A[:, k:, k]
        nz = col != 0
        has = nz.any(axis=1)
        alive &= has
        piv = k + np.argmax(nz, axis=1)
        swap = piv != k
        idx = np.arange(n)
        rk, rp = A[idx, k].copy(), A[idx, piv].copy()
        A[idx, k], A[idx, piv] = rp, rk
        det = np.where(swap, (p - det) % p, det)
        pv = A[:, k, k]
        det = (det * pv) % p
        inv = _pow_mod(pv, p - 2, p)                 # (Fermat; 0 stays 0)
        for i in range(k + 1, m):
            f = (A[:, i, k] * inv) % p
            # row_i -= f row_k (mod p), products below 2^62
            A[:, i, k:] = (A[:, i, k:] - (f[:, None] * A[:, k, k:]) % p) % p
    return np.where(alive, det, 0)


def _det_exact(N):
    """det of an integer matrix (Python ints), fraction-free (Bareiss)."""
    M = [[int(x) for x in r] for r in N]
    m, sign, prev = len(M), 1, 1
    for k in range(m):
        piv = next((i for i in range(k, m) if M[i][k] != 0), None)
        if piv is None:
            return 0
        if piv != k:
            M[k], M[piv] = M[piv], M[k]
            sign = -sign
        for i in range(k + 1, m):
            for j in range(k + 1, m):
                M[i][j] = (M[i][j] * M[k][k] - M[i][k] * M[k][j]) // prev
        prev = M[k][k]
    return sign * M[m - 1][m - 1]


def singular_mask(Ns):
    """Exactly which integer matrices of the stack Ns (n, m, m) are singular."""
    Ns = np.asarray(Ns)
    if Ns.shape[0] == 0:
        return np.zeros(0, dtype=bool)
    if Ns.dtype == object or np.max(np.abs(Ns)) >= 2 ** 62:
        return np.array([_det_exact(N) == 0 for N in Ns], dtype=bool)
    nonzero = np.zeros(Ns.shape[0], dtype=bool)
    for p in PRIMES:
        todo = np.flatnonzero(~nonzero)
        if not len(todo):
            break
        nonzero[todo] = _det_mod(Ns[todo], p) != 0
    sing = ~nonzero
    # det = 0 modulo every prime: det is a multiple of their product P, so it is 0
    # when |det| < P, i.e. when Hadamard's bound (the product of the rows' lengths)
    # is below P (log2 taken with a margin of two bits); otherwise exactly
    rows = np.sum(np.asarray(Ns, dtype=np.float64) ** 2, axis=2)
    with np.errstate(divide="ignore"):
        log_hb = 0.5 * np.sum(np.log2(rows), axis=1)
    log_p = sum(np.log2(float(p)) for p in PRIMES)
    for i in np.flatnonzero(sing & ~(log_hb + 2.0 < log_p)):
        sing[i] = _det_exact(Ns[i]) == 0
    return sing


def _adjugate(Mb):
    """(adj(Mb), det(Mb)) exactly, as Python ints (Mb^-1 = adj / det)."""
    h = len(Mb)
    inv = [[Fraction(int(Mb[i][j])) for j in range(h)] + [Fraction(int(i == j)) for j in range(h)] for i in range(h)]
    for k in range(h):
        piv = next(i for i in range(k, h) if inv[i][k] != 0)
        inv[k], inv[piv] = inv[piv], inv[k]
        f = inv[k][k]
        inv[k] = [x / f for x in inv[k]]
        for i in range(h):
            if i != k and inv[i][k] != 0:
                g = inv[i][k]
                inv[i] = [a - g * b for a, b in zip(inv[i], inv[k])]
    det = _det_exact(Mb)
    return [[int(inv[i][h + j] * det) for j in range(h)] for i in range(h)], det


def _primitive(M, Mbasis):
    """gcd(c) == 1 for each row M = Mbasis x (x = the coordinates in the
    M-lattice basis, with gcd(x) = gcd(c)): gcd(adj(Mbasis) M) == |det|."""
    adj, det = _adjugate(np.asarray(Mbasis))
    h = len(adj)
    amax = max(abs(v) for r in adj for v in r)
    if len(M) and amax * int(np.max(np.abs(M))) * h < 2 ** 62:
        X = np.asarray(M, dtype=np.int64) @ np.array(adj, dtype=np.int64).T      # det x, exact in int64
        return np.gcd.reduce(np.abs(X), axis=1) == abs(det)
    X = (np.array(adj, dtype=object) @ np.asarray(M).astype(object).T).T
    g = np.array([math.gcd(*[int(v) for v in row]) for row in X], dtype=object)
    return np.array([int(x) == abs(det) for x in g], dtype=bool)


def pfvs_from_points(M, Kn, kappa, Mbasis, Qmin, Qmax):
    """(Ks, Ms) of lattice points (M, Kn = Z M rows), as nonconi.py:437-495,
    of any number of p-vectors at once (each point's test is its own)."""
    h = np.asarray(kappa).shape[0]
    M, Kn = np.asarray(M)[:, :h], np.asarray(Kn)[:, :h]
    empty = (np.zeros((0, h), np.int64), np.zeros((0, h), np.int64))
    if not len(M):
        return empty
    keep = _primitive(M, Mbasis)
    M, Kn = M[keep], Kn[keep]
    if not len(M):
        return empty
    kap = np.asarray(kappa, dtype=np.int64)
    if np.max(np.abs(kap)) * np.max(np.abs(M)) * h < 2 ** 62:
        Ns = np.einsum("abc,nc->nab", kap, M)
    else:
        Ns = np.einsum("abc,nc->nab", kap.astype(object), M.astype(object))
    sing = singular_mask(Ns)
    M, Kn = M[~sing], Kn[~sing]
    if not len(M):
        return empty
    g = np.gcd.reduce(np.abs(Kn), axis=1)
    K = Kn // g[:, None]
    if np.max(np.abs(K)) * np.max(np.abs(M)) * h < 2 ** 62:
        Q = -np.einsum("ij,ij->i", K, M)
    else:
        Q = -np.sum(K.astype(object) * M.astype(object), axis=1)
    inq = np.array([Qmin <= int(q) <= Qmax for q in Q], dtype=bool) if Q.dtype == object else \
        (Q >= Qmin) & (Q <= Qmax)
    return K[inq].astype(np.int64), M[inq].astype(np.int64)


def allow_gcds(Ks, Ms, Qmax, h11):
    """Every (a K, b M), a, b >= 1, with -a b K.M <= Qmax (nonconi.py:50-84),
    each once, sorted by (K, M).  A pair with -K.M <= 0 has no multiples (the
    reference's numpy Qmax // 0 is 0)."""
    Ks, Ms = np.asarray(Ks, dtype=np.int64).reshape(-1, h11), np.asarray(Ms, dtype=np.int64).reshape(-1, h11)
    q = -np.einsum("ij,ij->i", Ks.astype(object), Ms.astype(object)) if len(Ks) else np.zeros(0, object)
    ok = np.array([int(x) > 0 for x in q], dtype=bool)
    Ks, Ms = Ks[ok], Ms[ok]
    q = np.array([int(x) for x in q[ok]], dtype=np.int64)
    parts = []
    for a in range(1, int(Qmax) + 1):
        sel = a * q <= Qmax
        if not sel.any():
            break
        Ka, Ma, qa = Ks[sel] * a, Ms[sel], q[sel] * a
        for b in range(1, int(Qmax) // a + 1):
            sb = b * qa <= Qmax
            if not sb.any():
                break
            parts.append(np.hstack([Ka[sb], Ma[sb] * b]))
    if not parts:
        z = np.zeros((0, h11), dtype=np.int64)
        return z, z.copy()
    A = np.unique(np.vstack(parts), axis=0)
    return A[:, :h11], A[:, h11:]


def zpm(kappa, Mbasis, ps, Qmin, Qmax, dilation, device=0, max_N_pfvs=1_000_000_000, return_info=False):
    """
    Non-coni PFVs of the p-vectors ps ((n, h11), in the Kahler cone): the
    device's lattice points (gpu.zpm_batch_multi_ex) through the reference's
    post-processing.  Raises IncompleteSearchError, as the reference, for a
    p-vector whose search the device could not finish exactly (or with more
    than max_N_pfvs points).  Returns (Ks, Ms) (and a dict of statistics).
    """
    kappa = np.asarray(kappa, dtype=np.int64)
    h = kappa.shape[0]
    ps = np.atleast_2d(np.asarray(ps, dtype=np.int64))
    geoms = [dict(kappa=kappa, Mbasis=np.asarray(Mbasis, dtype=np.int64), Q=int(Qmax), dilation=float(dilation))]
    M, Kn, q, pidx, pstat, secs, stats = gpu.zpm_batch_multi_ex(geoms, ps, np.zeros(len(ps), np.int32),
                                                                device=device)
    counts = np.bincount(pidx, minlength=len(ps)) if len(pidx) else np.zeros(len(ps), np.int64)
    for i in np.flatnonzero((pstat != 0) | (counts > max_N_pfvs)):
        st = int(pstat[i]) if pstat[i] else -2
        raise IncompleteSearchError(f"p={ps[i].tolist()}: the device search returned status {st} "
                                    f"({STATUS_TEXT.get(st, 'not finished')})")
    K, Mm = pfvs_from_points(M, Kn, kappa, Mbasis, Qmin, Qmax)     # (every point's test is its own)
    Ks, Ms = allow_gcds(K, Mm, int(Qmax), h)
    if return_info:
        return Ks, Ms, dict(stats, points=int(len(q)), seconds_gpu=secs)
    return Ks, Ms


def ZpM(data, ps, Qmax=None, Qmin=0, ellipsoid_dilation=1, use_c_kernel=True, use_c_lattice=True, n_jobs=-1,
        extra_checks=False, extra_lll_reduction=True, max_N_pfvs=1_000_000_000, return_formal_pfvs=False,
        verbosity=0, device=0):
    """
    The reference's ZpM signature (pfvs/nonconi.py:262) over a geometry
    object with the reference's CYData attributes (coni, kappa, h11, h21, H,
    c2 or M_lattice()): the same checks and errors, the search on the
    device.  use_c_kernel, use_c_lattice, n_jobs, extra_checks and
    extra_lll_reduction select among the reference's CPU routes, which all
    give the same PFVs, and are accepted and unused here; return_formal_pfvs
    needs the reference's PFV class and is not supported.
    """
    del use_c_kernel, use_c_lattice, n_jobs, extra_checks, extra_lll_reduction, verbosity
    if getattr(data, "coni", False):
        raise ValueError("ZpM and ZpK only apply to non-coni contexts. Use coniZpM for coni PFVs.")
    if return_formal_pfvs:
        raise NotImplementedError("return_formal_pfvs needs the reference's PFV class")
    if len(ps) == 0:
        raise ValueError("ps must be non-empty.")
    ps = np.array(ps)
    if not np.all(np.asarray(data.H) @ ps.T >= 1):
        raise ValueError("some p-vectors are not in the kahler cone (H@ps.T >= 1 failed)")
    kappa = np.asarray(data.kappa, dtype=np.int64)
    h11, h21 = int(data.h11), int(data.h21)
    if Qmax is None:
        Qmax = h11 + h21 + 2
    if Qmax < Qmin:
        raise ValueError(f"Qmax ({Qmax}) must be >= Qmin ({Qmin}).")
    if ellipsoid_dilation <= 0:
        raise ValueError(f"ellipsoid_dilation must be > 0, got {ellipsoid_dilation}.")
    Mbasis = data.M_lattice() if hasattr(data, "M_lattice") else intlat.m_lattice(kappa, data.c2, coni=False)
    return zpm(kappa, Mbasis, ps, Qmin, Qmax, ellipsoid_dilation, device=device, max_N_pfvs=max_N_pfvs)
