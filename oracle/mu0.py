"""
ORACLE / TEST INFRASTRUCTURE -- never part of the product path.

The coni dilation bound of the reference (pfvs/dilation.py:47-200, C path
pfvs/fp_kernel/coni_bound.h:255), restated in exact Python integers and
fractions (no flint):

    A      = kappa . p_hat              p_hat = (0, p_r)
    s      = a00 - a_r0^T A_rr^-1 a_r0,  S = -A_rr^-1
    Lambda = {K in Z^(h11-1) : p_r . K = 0}
    mu0    = min over nonzero K in Lambda of K^T S K

Every coni PFV with direction p_hat has dilation delta < Q / mu0 when s <= 0
and S is positive definite on Lambda; otherwise there is no bound.

  coni_mu0(kappa, p_r) -> (status, mu0 Fraction or None, K list or None)
      status 0: decided; 1: no bound (A_rr singular, s > 0, or S not
      positive definite on Lambda)
  dilation_bound(kappa, p_r, Q) -> Fraction Q / mu0, or None
  grid_up(D) -> D rounded up onto the grid of ratio 2^(1/16)
      (pfvs/coni.py:647-653, the reference's _grid_up)
"""
import math
from fractions import Fraction

import numpy as np

from . import lattice


def _solve_exact(A, rhs_cols):
    """A^-1 applied to the columns in rhs_cols (lists), Gauss-Jordan over the
    rationals; None if A is singular."""
    m = len(A)
    M = [[Fraction(int(x)) for x in A[i]] + [Fraction(int(c[i])) for c in rhs_cols] for i in range(m)]
    w = len(M[0])
    for k in range(m):
        piv = next((i for i in range(k, m) if M[i][k] != 0), None)
        if piv is None:
            return None
        M[k], M[piv] = M[piv], M[k]
        inv = 1 / M[k][k]
        M[k] = [x * inv for x in M[k]]
        for i in range(m):
            if i != k and M[i][k] != 0:
                f = M[i][k]
                M[i] = [a - f * b for a, b in zip(M[i], M[k])]
    return [[M[i][m + c] for i in range(m)] for c in range(w - m)]


def _shortest(G):
    """Exact min of y^T G y over nonzero integer y and a minimizer, for a
    positive definite integer Gram matrix G (n x n lists), by Fincke-Pohst
    over its exact LDL^T (rational pivots d_i, multipliers m[j][i])."""
    n = len(G)
    d = [Fraction(0)] * n
    m = [[Fraction(0)] * n for _ in range(n)]
    for i in range(n):
        d[i] = Fraction(G[i][i]) - sum(m[i][k] ** 2 * d[k] for k in range(i))
        for j in range(i + 1, n):
            m[j][i] = (Fraction(G[j][i]) - sum(m[j][k] * m[i][k] * d[k] for k in range(i))) / d[i]
    k0 = min(range(n), key=lambda k: G[k][k])
    best = [Fraction(G[k0][k0]), [int(i == k0) for i in range(n)]]
    y = [0] * n

    def level(i, partial):
        if i < 0:
            if any(y) and partial < best[0]:
                best[0], best[1] = partial, list(y)
            return
        c = -sum((m[j][i] * y[j] for j in range(i + 1, n)), Fraction(0))
        room = best[0] - partial
        r = math.sqrt(float(room / d[i])) if room > 0 else 0.0
        for v in range(math.floor(float(c) - r) - 1, math.ceil(float(c) + r) + 2):
            t = d[i] * (v - c) ** 2
            if partial + t <= best[0]:
                y[i] = v
                level(i - 1, partial + t)
        y[i] = 0

    level(n - 1, Fraction(0))
    return best[0], best[1]


def coni_mu0(kappa, p_r):
    kappa = np.asarray(kappa)
    h = kappa.shape[0]
    p_r = [int(x) for x in np.asarray(p_r).ravel()]
    p_hat = [0] + p_r
    A = [[sum(int(kappa[a, b, c]) * p_hat[c] for c in range(h)) for b in range(h)] for a in range(h)]
    Arr = [row[1:] for row in A[1:]]
    a_r0 = [A[i][0] for i in range(1, h)]
    O = [list(r) for r in lattice.unimodular(p_r)[1:]]          # rows span Lambda
    sol = _solve_exact(Arr, [a_r0] + O)                         # A_rr^-1 a_r0, A_rr^-1 O_k
    if sol is None:
        return 1, None, None
    x = sol[0]
    s = Fraction(A[0][0]) - sum(Fraction(a) * b for a, b in zip(a_r0, x))
    if s > 0:
        return 1, None, None
    n = len(O)
    # the form S = -A_rr^-1 on Lambda's basis, made integral
    Gq = [[-sum(Fraction(O[a][i]) * sol[1 + b][i] for i in range(h - 1)) for b in range(n)] for a in range(n)]
    L = 1
    for row in Gq:
        for v in row:
            L = L * v.denominator // math.gcd(L, v.denominator)
    G = [[int(v * L) for v in row] for row in Gq]
    if not lattice.is_positive_definite(G):
        return 1, None, None
    T, _ = lattice.lll([[int(i == j) for j in range(n)] for i in range(n)], G)
    Gr = [[sum(T[a][i] * G[i][j] * T[b][j] for i in range(n) for j in range(n)) for b in range(n)]
          for a in range(n)]
    val, y = _shortest(Gr)
    coef = [sum(y[a] * T[a][j] for a in range(n)) for j in range(n)]       # in O's basis
    K = [sum(coef[a] * O[a][i] for a in range(n)) for i in range(h - 1)]
    return 0, Fraction(val) / L, K


def dilation_bound(kappa, p_r, Q):
    st, mu0, _ = coni_mu0(kappa, p_r)
    return None if st else Fraction(int(Q)) / mu0


def grid_up(D):
    """D (integer >= 1) rounded up onto the grid ceil(2^(k/16)), nearby bounds
    sharing one search; D itself where the grid point is below it."""
    D = np.maximum(np.asarray(D, dtype=np.int64), 1)
    k = np.ceil(16 * np.log2(D)).astype(np.int64)
    g = np.ceil(2.0 ** (k / 16)).astype(np.int64)
    return np.where(g >= D, g, D)
