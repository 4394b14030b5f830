"""
ORACLE / TEST INFRASTRUCTURE -- never part of the product path.

CPU restatement, in exact Python integers, of the reference's per-direction
lattice setup and exact factorization for the coni pipeline:

- `build`   restates pfl_build (pfvs/fp_kernel/pfv_lattice.h:604-680):
            Z = kappa.p, T = Z p, v = T Mbasis; the lattice orthogonal to v
            (pfl_unimodular, :162-188) LLL-reduced (pfl_lll, :508-521);
            Binter^T = O Mbasis^T; coni column order (:643-653);
            ZB = Z Binter, mat = -Binter^T ZB (:655-666); the cut-aware basis
            change (pfl_m0_basis, :554-602).  Python ints never overflow, so
            the reference's overflow statuses do not arise here.
- `hnf`     the canonical row-HNF (flint's, pfl_hnf :205-313 / GMP :320-368).
- `factor`  the exact LDL^T / Cholesky data of fpk_factor_fast /
            fpk_factor_exact (pfvs/fpk_common.h:259-309, fp_kernel.h:193-306):
            U (upper, U^T U = mat), and the M0 bound data N, V, |V|-sums,
            computed exactly (fraction-free Bareiss, exact rationals) and
            rounded once to double.

Any basis of the same lattice gives the same output set, so this module need
not reproduce the reference's basis bit for bit; it follows its steps.
"""
from fractions import Fraction
import math

import numpy as np


def xgcd_floor(a, b):
    """(g, s, t): s a + t b = g, Euclid with floor division
    (pfv_lattice.h:116-130, util.extended_euclidean)."""
    r0, r1, s0, s1, t0, t1 = a, b, 1, 0, 0, 1
    while r1 != 0:
        q = r0 // r1
        r0, r1 = r1, r0 - q * r1
        s0, s1 = s1, s0 - q * s1
        t0, t1 = t1, t0 - q * t1
    return r0, s0, t0


def unimodular(v):
    """U (list of rows) with U v = (gcd, 0, ..., 0) by sequential Bezout
    steps on (w0, wk) (pfv_lattice.h:162-188)."""
    n = len(v)
    w = [int(x) for x in v]
    U = [[int(i == j) for j in range(n)] for i in range(n)]
    for k in range(1, n):
        if w[k] == 0:
            continue
        g, s, t = xgcd_floor(w[0], w[k])
        if g == 0:
            raise ValueError("degenerate vector")
        m10, m11 = -(w[k] // g), w[0] // g
        w[0], w[k] = g, 0
        r0, rk = U[0], U[k]
        U[0] = [s * x + t * y for x, y in zip(r0, rk)]
        U[k] = [m10 * x + m11 * y for x, y in zip(r0, rk)]
    return U


def lll(B, gram, last=None, delta=0.99):
    """
    LLL (delta 0.99) of the rows of B w.r.t. the exact Gram matrix `gram`
    ((m + [last]) x (m + [last]) Python ints), then size-reduce `last`
    against the reduced rows (pfv_lattice.h:389-505).  Floating-point
    Gram-Schmidt from the exact Gram only chooses the unimodular steps.
    Returns (B, last).
    """
    B = [list(r) for r in B]
    m = len(B)
    rows = B + ([list(last)] if last is not None else [])
    M = len(rows)
    G = [list(r) for r in gram]
    mu = [[0.0] * M for _ in range(M)]
    bb = [0.0] * M

    def gs(k):
        for j in range(k):
            t = float(G[k][j])
            for l in range(j):
                t -= mu[j][l] * mu[k][l] * bb[l]
            mu[k][j] = t / bb[j]
        t = float(G[k][k])
        for l in range(k):
            t -= mu[k][l] * mu[k][l] * bb[l]
        bb[k] = t

    def sub(k, j, q):
        rows[k] = [x - q * y for x, y in zip(rows[k], rows[j])]
        gkk = G[k][k] - 2 * q * G[k][j] + q * q * G[j][j]
        for l in range(M):
            if l != k:
                G[k][l] -= q * G[j][l]
                G[l][k] = G[k][l]
        G[k][k] = gkk

    if m >= 1:
        gs(0)
        if not bb[0] > 0:
            raise ValueError("rank loss in LLL")
    if m >= 2:
        gs(1)
    k = 1
    while k < m:
        for _ in range(4):
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
            gs(k)
        if not bb[k] > 0:
            raise ValueError("rank loss in LLL")
        if bb[k] < (delta - mu[k][k - 1] ** 2) * bb[k - 1]:
            rows[k], rows[k - 1] = rows[k - 1], rows[k]
            G[k], G[k - 1] = G[k - 1], G[k]
            for r in G:
                r[k], r[k - 1] = r[k - 1], r[k]
            k = max(k - 1, 1)
            if k == 1:
                gs(0)
            gs(k - 1)
            gs(k)
        else:
            k += 1
            if k < m:
                gs(k)
    if last is not None and m > 0:
        for _ in range(4):
            mw = [0.0] * m
            for j in range(m):
                t = float(G[m][j])
                for l in range(j):
                    t -= mu[j][l] * mw[l] * bb[l]
                mw[j] = t / bb[j]
            changed = False
            for j in range(m - 1, -1, -1):
                q = round(mw[j])
                if q:
                    sub(m, j, q)
                    for l in range(j):
                        mw[l] -= q * mu[j][l]
                    mw[j] -= q
                    changed = True
            if not changed:
                break
    return rows[:m], (rows[m] if last is not None else None)


def _gram(rows, form=None):
    if form is None:
        return [[sum(a * b for a, b in zip(x, y)) for y in rows] for x in rows]
    Fy = [[sum(form[i][c] * y[c] for c in range(len(y))) for i in range(len(y))] for y in rows]
    return [[sum(a * b for a, b in zip(x, fy)) for fy in Fy] for x in rows]


def matmul(A, B):
    return [[sum(a * b for a, b in zip(row, col)) for col in zip(*B)] for row in A]


class NotPositiveDefinite(ValueError):
    """The ellipsoid matrix is not positive definite: the reference's kernel
    status -9 (fpk_common.h:259-309), which coniZpM raises as
    IncompleteSearchError (coni.py:446-453)."""


def is_positive_definite(mat):
    """Sylvester's criterion, exactly: every leading principal minor of the
    symmetric integer matrix is > 0 (fraction-free Bareiss elimination; the
    pivots are the leading minors)."""
    A = [[int(x) for x in r] for r in mat]
    d = len(A)
    prev = 1
    for k in range(d):
        pk = A[k][k]
        if pk <= 0:
            return False
        for i in range(k + 1, d):
            for j in range(k + 1, d):
                A[i][j] = (pk * A[i][j] - A[i][k] * A[k][j]) // prev
        prev = pk
    return True


def build(kappa, Mbasis, p):
    """
    Per-direction lattice data (pfl_build, coni, extra_lll, m0_basis).
    kappa (h,h,h), Mbasis (h,h) columns, p (h,) with p[0] = 0.  Returns a dict
    of Python-int matrices: Z (h,h), Binter (h,d), ZB (h,d), mat (d,d).
    """
    kappa = np.asarray(kappa).astype(object)
    Mb = [[int(x) for x in r] for r in np.asarray(Mbasis)]
    p = [int(x) for x in p]
    h = len(p)
    d = h - 1
    Z = [[sum(int(kappa[i, j, k]) * p[k] for k in range(h)) for j in range(h)] for i in range(h)]
    T = [sum(Z[i][k] * p[k] for k in range(h)) for i in range(h)]
    v = [sum(T[i] * Mb[i][j] for i in range(h)) for j in range(h)]
    if all(x == 0 for x in v):
        raise ValueError("p.Z.Mbasis == 0")
    O = unimodular(v)[1:]                                     # (d, h) rows
    O, _ = lll(O, _gram(O))
    BT = [[sum(Mb[i][l] * O[a][l] for l in range(h)) for i in range(h)] for a in range(d)]
    order = [a for a in range(d) if BT[a][0] == 0] + [a for a in range(d) if BT[a][0] != 0]
    Binter = [[BT[order[a]][i] for a in range(d)] for i in range(h)]
    ZB = matmul(Z, Binter)
    mat = [[-sum(Binter[i][a] * ZB[i][b] for i in range(h)) for b in range(d)] for a in range(d)]
    # A direction whose kappa.p lacks the signature (1, h11-1) gives an
    # indefinite mat.  The reference's C setup fails on it (the LLL w.r.t.
    # mat below meets a non-positive norm), its Python path rebuilds mat with
    # the Euclidean reduction only, and the exact factorization then reports
    # -9 (coni.py:1025-1046, fpk_common.h:259-309): decide that here.
    if not is_positive_definite(mat):
        raise NotPositiveDefinite("the ellipsoid matrix is not positive definite")
    # cut-aware basis change (pfv_lattice.h:554-602)
    l = Binter[0]
    if any(x != 0 for x in l):
        V = unimodular(l)
        K, w = V[1:], V[0]
        K, w = lll(K, _gram(K + [w], mat), last=w)
        Tm = [[K[a][i] for a in range(d - 1)] + [w[i]] for i in range(d)]   # columns
        Binter = matmul(Binter, Tm)
        ZB = matmul(ZB, Tm)
        TT = [list(r) for r in zip(*Tm)]
        mat = matmul(TT, matmul(mat, Tm))
    return dict(h=h, d=d, Z=Z, Binter=Binter, ZB=ZB, mat=mat)


def hnf(A):
    """Canonical row-HNF (upper echelon, positive pivots, entries above a
    pivot in [0, pivot), zero rows last) of an integer matrix."""
    A = [[int(x) for x in r] for r in A]
    r = len(A)
    n = len(A[0]) if r else 0
    row = 0
    for col in range(n):
        if row >= r:
            break
        while True:
            nz = [i for i in range(row, r) if A[i][col] != 0]
            if not nz:
                break
            piv = min(nz, key=lambda i: abs(A[i][col]))
            A[row], A[piv] = A[piv], A[row]
            clean = True
            for i in range(row + 1, r):
                if A[i][col]:
                    q = A[i][col] // A[row][col]
                    A[i] = [x - q * y for x, y in zip(A[i], A[row])]
                    if A[i][col]:
                        clean = False
            if clean:
                break
        if A[row][col] == 0:
            continue
        if A[row][col] < 0:
            A[row] = [-x for x in A[row]]
        for i in range(row):
            q = A[i][col] // A[row][col]
            if q:
                A[i] = [x - q * y for x, y in zip(A[i], A[row])]
        row += 1
    return A


def _fdiv(a, b):
    """a / b correctly rounded to double (Python int true division)."""
    return a / b


def factor(mat, linvec=None):
    """
    Exact LDL^T of a symmetric integer matrix, rounded once: returns
    (status, U, N, V, Va) with U upper triangular (U^T U = mat),
    N[i] = sum_{k<=i} z_k^2 / d_k, V[i][j] = sum_{k<=i} R_kj z_k (j > i),
    Va[i][j] = |V[i][j]| (exact V, so |V| bounds its rounding), z = R^-T linvec
    (fp_kernel.h:193-306).  status -9 if mat is not positive definite.
    """
    d = len(mat)
    A = [[int(x) for x in r] for r in mat]
    piv = []
    prev = 1
    rowsk = []                      # A^(k)[k][j], j >= k, after step k
    for k in range(d):
        pk = A[k][k]
        if pk <= 0:
            return -9, None, None, None, None
        rowsk.append(list(A[k]))
        for i in range(k + 1, d):
            for j in range(i, d):
                x = (pk * A[i][j] - A[i][k] * A[k][j])
                q, rem = divmod(x, prev)
                assert rem == 0
                A[i][j] = q
                if j != i:
                    A[j][i] = q
        piv.append(pk)
        prev = pk
    U = np.zeros((d, d))
    pprev = 1
    for k in range(d):
        pk = piv[k]
        ukk = math.sqrt(_fdiv(pk, pprev))
        U[k, k] = ukk
        for j in range(k + 1, d):
            U[k, j] = ukk * _fdiv(rowsk[k][j], pk)
        pprev = pk
    N = V = Va = None
    if linvec is not None:
        lv = [int(x) for x in linvec]
        R = [[Fraction(rowsk[k][j], piv[k]) if j >= k else Fraction(0) for j in range(d)]
             for k in range(d)]
        z = []
        for k in range(d):
            zk = Fraction(lv[k]) - sum((R[m][k] * z[m] for m in range(k)), Fraction(0))
            z.append(zk)
        N = np.zeros(d)
        V = np.zeros((d, d))
        Vx = [Fraction(0)] * d
        acc = Fraction(0)
        pprev = 1
        for i in range(d):
            acc += z[i] * z[i] * Fraction(pprev, piv[i])
            N[i] = float(acc)
            for j in range(i + 1, d):
                Vx[j] += R[i][j] * z[i]
                V[i, j] = float(Vx[j])
            pprev = piv[i]
        Va = np.abs(V)
    return 0, U, N, V, Va
