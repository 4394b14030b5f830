"""
Exact integer-lattice helpers for per-geometry input preparation on the
host (Python ints; no floating point in any result, floats only choose
unimodular LLL steps).

The reference computes the M-lattice basis with python-flint
(pfvs/cydata.py:307-356, `CYData.M_lattice`: LLL of the primal
[b/24; a/2; I], dual lattice, LLL).  Any basis of the same lattice gives the
same coniZpM output (the output is put in canonical order,
pfvs/coni.py:322-324), so this module computes the lattice directly from the
congruences and LLL-reduces it.
"""
import numpy as np


def _xgcd(a, b):
    """(g, s, t) with s a + t b = g = gcd(a, b) >= 0."""
    s0, s1, t0, t1 = 1, 0, 0, 1
    while b:
        q, r = divmod(a, b)
        a, b = b, r
        s0, s1 = s1, s0 - q * s1
        t0, t1 = t1, t0 - q * t1
    if a < 0:
        a, s0, t0 = -a, -s0, -t0
    return a, s0, t0


def refine_congruence(B, c, m):
    """
    Given a basis B (list of h column vectors, Python ints) of a lattice L,
    return a basis of {M in L : c . M = 0 (mod m)}.  The residues
    v_j = c . b_j mod m are brought to (g, 0, ..., 0) by unimodular 2x2
    Bezout steps on the columns (small numbers: residues are < m); then
    the first column is scaled by m / gcd(g, m).
    """
    B = [list(b) for b in B]
    h = len(B)
    v = [sum(int(x) * int(y) for x, y in zip(c, b)) % m for b in B]
    # move a nonzero residue to position 0
    for j in range(h):
        if v[j]:
            B[0], B[j] = B[j], B[0]
            v[0], v[j] = v[j], v[0]
            break
    else:
        return B                              # every column already satisfies it
    for j in range(1, h):
        if v[j] == 0:
            continue
        g, s, t = _xgcd(v[0], v[j])
        a0, aj = v[0] // g, v[j] // g
        b0, bj = B[0], B[j]
        B[0] = [s * x + t * y for x, y in zip(b0, bj)]
        B[j] = [-aj * x + a0 * y for x, y in zip(b0, bj)]
        v[0], v[j] = g % m, 0
    f = m // _xgcd(v[0], m)[0]
    B[0] = [f * x for x in B[0]]
    return B


def lll_rows_fast(B, delta=0.99, max_swaps=10**6):
    """
    LLL-reduce the rows of an integer matrix (Lenstra-Lenstra-Lovasz 1982,
    textbook form): exact integer row operations and an exact integer Gram
    matrix; floating-point Gram-Schmidt coefficients, recomputed from the
    exact Gram row after each size reduction, only choose the steps.  The
    result always spans the same lattice.
    """
    B = [[int(x) for x in row] for row in B]
    m = len(B)
    if m < 2:
        return B
    G = [[sum(x * y for x, y in zip(B[i], B[j])) for j in range(m)] for i in range(m)]
    mu = [[0.0] * m for _ in range(m)]
    bb = [0.0] * m

    def gso_row(k):
        for j in range(k):
            t = float(G[k][j])
            for l in range(j):
                t -= mu[j][l] * mu[k][l] * bb[l]
            mu[k][j] = t / bb[j]
        t = float(G[k][k])
        for l in range(k):
            t -= mu[k][l] * mu[k][l] * bb[l]
        bb[k] = t

    def sub(k, j, q):                   # b_k -= q b_j, exactly (vectors and Gram)
        B[k] = [x - q * y for x, y in zip(B[k], B[j])]
        gkk = G[k][k] - 2 * q * G[k][j] + q * q * G[j][j]
        for l in range(m):
            if l != k:
                G[k][l] -= q * G[j][l]
                G[l][k] = G[k][l]
        G[k][k] = gkk

    gso_row(0)
    gso_row(1)
    k, swaps = 1, 0
    while k < m:
        for _ in range(8):
            changed = False
            for j in range(k - 1, -1, -1):
                q = round(mu[k][j])
                if q:
                    sub(k, j, q)
                    for l in range(j):
                        mu[k][l] -= q * mu[j][l]
                    mu[k][j] -= q
                    changed = True
            if not changed:
                break
            gso_row(k)
        if bb[k] < (delta - mu[k][k - 1] ** 2) * bb[k - 1]:
            swaps += 1
            if swaps > max_swaps:
                raise RuntimeError("LLL did not converge")
            B[k], B[k - 1] = B[k - 1], B[k]
            G[k], G[k - 1] = G[k - 1], G[k]
            for row in G:
                row[k], row[k - 1] = row[k - 1], row[k]
            k = max(k - 1, 1)
            if k == 1:
                gso_row(0)
            gso_row(k - 1)
            gso_row(k)
        else:
            k += 1
            if k < m:
                gso_row(k)
    return B


def a_matrix(kappa, coni=True):
    """The a-matrix (pfvs/cydata.py:252-283): a_ij = kappa_iij (i >= j),
    kappa_ijj (i < j); in the coni basis with the coni row dropped (coni), or
    whole (a non-coni geometry)."""
    h = kappa.shape[0]
    a = np.zeros((h, h), dtype=np.int64)
    for x in range(h):
        for y in range(h):
            a[x, y] = kappa[x, x, y] if x >= y else kappa[x, y, y]
    return a[1:] if coni else a


def b_vector(c2, coni=True):
    """b = c2 + 2 e0 in the coni basis (coni), or c2 (non-coni)
    (pfvs/cydata.py:285-303)."""
    b = np.array(c2, dtype=np.int64).copy()
    if coni:
        b[0] += 2
    return b


def m_lattice(kappa, c2, coni=True):
    """
    Basis (columns, h x h int64) of {M in Z^h : (a/2) M integral and
    (b/24) . M integral}: the lattice of `CYData.M_lattice`
    (pfvs/cydata.py:307-356), computed by refining Z^h one congruence at
    a time (`refine_congruence`: b . M = 0 mod 24, then each row of a mod 2),
    LLL-reducing after each step to keep the entries small.  a and b as
    a_matrix / b_vector for a coni geometry (kappa, c2 in the coni basis) or
    a non-coni one.
    """
    kappa = np.asarray(kappa, dtype=np.int64)
    h = kappa.shape[0]
    a = a_matrix(kappa, coni)
    b = b_vector(c2, coni)
    B = [[int(i == j) for i in range(h)] for j in range(h)]   # columns of I
    B = refine_congruence(B, [int(x) for x in b], 24)
    for row in a:
        B = refine_congruence(B, [int(x) for x in row], 2)
        B = lll_rows_fast(B)
    basis = lll_rows_fast(B)
    Mb = np.array(basis, dtype=np.int64).T      # columns
    # verify (pfvs/cydata.py:349-353)
    if not np.all((a @ Mb) % 2 == 0) or not np.all((b @ Mb) % 24 == 0):
        raise RuntimeError("M-lattice verification failed")
    det = abs(round(np.linalg.det(Mb.astype(float))))
    if det == 0:
        raise RuntimeError("M-lattice basis is singular")
    return Mb
