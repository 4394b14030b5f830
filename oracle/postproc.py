"""
ORACLE / TEST INFRASTRUCTURE -- never part of the product path.

Restatement of coniZpM's post-processing `_pfvs_from_points`
(pfvs/coni.py:275-412): lattice points (M = Binter c, Kn = ZB c, q) of any
number of p-vectors -> coni PFVs (K, M), in exact integer arithmetic
(Python ints), with the exact singularity test of `util.singular_mask`
(pfvs/util.py:224-243) done by modular determinants plus an exact
fraction-free fallback.
"""
import numpy as np

PRIMES = (2147483629, 2147483587, 2147483579)     # < 2^31: products fit int64


def _gcd(a, b):
    a, b = abs(a), abs(b)
    while b:
        a, b = b, a % b
    return a


def det_mod_p(A, p):
    """det of each matrix in the stack A (n, m, m) int64 modulo prime p
    (Gaussian elimination, vectorized over the stack)."""
    A = np.mod(np.array(A, dtype=np.int64), p)
    n, m, _ = A.shape
    det = np.ones(n, dtype=np.int64)
    alive = np.ones(n, dtype=bool)
    ar = np.arange(n)
    for k in range(m):
        sub = A[:, k:, k]
        nz = sub != 0
        has = nz.any(axis=1)
        alive &= has
        piv = k + np.argmax(nz, axis=1)
        # swap row k and row piv
        rk = A[ar, k].copy()
        A[ar, k] = A[ar, piv]
        A[ar, piv] = rk
        det = np.where(piv != k, (p - det) % p, det)
        pk = A[:, k, k]
        det = (det * pk) % p
        inv = np.array([pow(int(x), p - 2, p) if x else 0 for x in pk], dtype=np.int64)
        f = (A[:, k + 1:, k] * inv[:, None]) % p                    # (n, m-k-1)
        A[:, k + 1:, k:] = (A[:, k + 1:, k:] - (f[:, :, None] * A[:, None, k, k:]) % p) % p
    return np.where(alive, det, 0)


def det_exact(A):
    """Exact determinant of an integer matrix (fraction-free Bareiss)."""
    M = [[int(x) for x in r] for r in A]
    m = len(M)
    sign, prev = 1, 1
    for k in range(m - 1):
        if M[k][k] == 0:
            sw = next((i for i in range(k + 1, m) if M[i][k] != 0), None)
            if sw is None:
                return 0
            M[k], M[sw] = M[sw], M[k]
            sign = -sign
        for i in range(k + 1, m):
            for j in range(k + 1, m):
                M[i][j] = (M[i][j] * M[k][k] - M[i][k] * M[k][j]) // prev
        prev = M[k][k]
    return sign * M[m - 1][m - 1] if m else 1


def singular_mask(Ns):
    """Exactly which integer matrices in the stack Ns (n, m, m) are singular."""
    Ns = np.asarray(Ns)
    n = Ns.shape[0]
    if n == 0:
        return np.zeros(0, dtype=bool)
    if Ns.dtype == object or np.max(np.abs(Ns)) >= 2**62:
        return np.array([det_exact(N) == 0 for N in Ns], dtype=bool)
    nonzero = np.zeros(n, dtype=bool)
    for p in PRIMES:
        nonzero |= det_mod_p(Ns, p) != 0
    sing = ~nonzero
    for i in np.flatnonzero(sing):          # zero mod every prime: decide exactly
        sing[i] = det_exact(Ns[i]) == 0
    return sing


def pfvs_from_points(Ms, Kns, Qs, key, kappa, h11, Q, M0min):
    """
    Lattice points -> coni PFVs, as pfvs/coni.py:275-412.  Ms, Kns: (N, h11)
    rows (one per point); Qs, key: (N,).  Returns (Ks, Ms, keys): (n, h11),
    (n, h11) as int64 (object if any entry exceeds int64), (n,), grouped by
    key (stable) in the reference's canonical order.
    """
    empty = (np.zeros((0, h11), dtype=np.int64), np.zeros((0, h11), dtype=np.int64),
             np.zeros(0, dtype=np.int64))
    Ms = [[int(x) for x in r] for r in np.asarray(Ms)]
    Kns = [[int(x) for x in r] for r in np.asarray(Kns)]
    Qs = [int(x) for x in np.asarray(Qs)]
    key = [int(x) for x in np.asarray(key)]
    if not Qs:
        return empty
    if M0min <= 0:
        raise ValueError("coniZpM requires M0min > 0")
    # strict cut: q < Q * gcd(Kn[1:]) (coni.py:314-318), gcd < 1 -> 1
    pts = []
    for M, K, q, k in zip(Ms, Kns, Qs, key):
        g = 0
        for x in K[1:]:
            g = _gcd(g, x)
        g = max(g, 1)
        if q < Q * g:
            pts.append((k, M, K, q, g))
    if not pts:
        return empty
    # canonical order (key, M, Kn) (coni.py:322-324)
    pts.sort(key=lambda t: (t[0], t[1], t[2]))
    # expand by admissible gcds g = 1..(Q*Kg - 1)//q, in (key, g, point) order
    exp = []
    for ip, (k, M, K, q, Kg) in enumerate(pts):
        gcap = (Q * Kg - 1) // max(q, 1)
        for g in range(1, gcap + 1):
            exp.append((k, g, ip))
    exp.sort()
    Ks_out, Ms_out, key_out = [], [], []
    for k, g, ip in exp:
        _, M, K, q, Kg = pts[ip]
        nat_K0 = K[0]
        Kperp = [x // Kg for x in K[1:]]
        M0 = M[0]
        rawQperp = (q + M0 * nat_K0) // Kg
        Qperp = g * rawQperp
        lo = -((Q - Qperp) // M0)
        up = (Qperp - Q) // M0
        up = min(up, -((-nat_K0 * g) // Kg) - 1)
        for K0 in range(lo, up + 1):
            Kv = [K0] + [g * x for x in Kperp]
            tad = -sum(a * b for a, b in zip(Kv, M))
            if tad > Q:
                raise RuntimeError(f"Tadpole violation: -dot(K,M)={tad} > Q={Q}")
            Ks_out.append(Kv)
            Ms_out.append(M)
            key_out.append(k)
    if not Ks_out:
        return empty
    # det((kappa . M)[1:, 1:]) != 0 (coni.py:388-404)
    kap = np.asarray(kappa).astype(object)
    Mo = np.array(Ms_out, dtype=object)
    Ns = np.einsum("ijk,nk->nij", kap, Mo)[:, 1:, 1:]
    big = any(abs(int(x)) >= 2**62 for x in Ns.ravel()) if Ns.size else False
    sing = singular_mask(Ns if big else Ns.astype(np.int64))
    keep = ~sing
    Ks = np.array(Ks_out, dtype=object)[keep]
    Msel = Mo[keep]
    keys = np.array(key_out, dtype=np.int64)[keep]
    order = np.argsort(keys, kind="stable")
    Ks, Msel, keys = Ks[order], Msel[order], keys[order]

    def tight(a):
        a = np.asarray(a, dtype=object).reshape(-1, h11)
        if a.size and max(abs(int(x)) for x in a.ravel()) >= 2**63:
            return a
        return a.astype(np.int64)
    return tight(Ks), tight(Msel), keys
