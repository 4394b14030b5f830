"""
ORACLE / TEST INFRASTRUCTURE -- never part of the product path.

Non-coni ZpM (pfvs/nonconi.py:262-514, its C route: use_c_lattice and
use_c_kernel), restated:

  build(kappa, Mbasis, p)      the setup of pfl_build with coni = 0
                               (pfv_lattice.h:604-680): Z = kappa.p, T = Z p,
                               v = T Mbasis, O the lattice orthogonal to v (LLL),
                               Binter = Mbasis O^T, ZB = Z Binter,
                               mat = -Binter^T ZB; then, with no M0 cut, the whole
                               basis LLL-reduced w.r.t. mat (pfv_lattice.h:560-566)
  points(kappa, Mbasis, p, Qmax, qmax)
                               the lattice points c with c^T mat c <= qmax and
                               the non-strict GCD cut g == 0 or Qmax g >= q,
                               g = gcd(ZB c) (pfv_kernel, fp_kernel.pyx:321-352):
                               (c, M = Binter c, Kn = ZB c, q)
  pfvs_from_points(C, M, Kn, kappa, Qmin, Qmax)
                               the reference's per-p post-processing
                               (nonconi.py:437-495): primitive c only,
                               det(kappa.M) != 0, K = Z M / gcd, Qmin <= -K.M <= Qmax
  allow_gcds(Ks, Ms, Qmax, h11) nonconi.py:50-84
  zpm(kappa, Mbasis, ps, Qmin, Qmax, dilation) -> set of (K, M) tuples

and the same data from the reference's own C code (oracle/_ref), composed as
nonconi.ZpM composes it: ref_points() = _lattice_build(coni = 0), the HNF of
ZB when the C setup leaves it to the caller (status -15), pfv_kernel.
"""
import math

import numpy as np

from . import lattice, pfo
from .postproc import singular_mask


def qmax_of(Q, dilation):
    """floor(dilation * Q) as the reference's _qmax (fp_kernel.pyx:146-148)."""
    return int(math.floor(dilation * Q + 1e-7))


def build(kappa, Mbasis, p):
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
    O = lattice.unimodular(v)[1:]
    O, _ = lattice.lll(O, lattice._gram(O))
    BT = [[sum(Mb[i][l] * O[a][l] for l in range(h)) for i in range(h)] for a in range(d)]
    Binter = [[BT[a][i] for a in range(d)] for i in range(h)]
    ZB = lattice.matmul(Z, Binter)
    mat = [[-sum(Binter[i][a] * ZB[i][b] for i in range(h)) for b in range(d)] for a in range(d)]
    if not lattice.is_positive_definite(mat):
        raise lattice.NotPositiveDefinite("the ellipsoid matrix is not positive definite")
    V, _ = lattice.lll([[int(i == j) for j in range(d)] for i in range(d)], mat)
    Tm = [[V[a][i] for a in range(d)] for i in range(d)]          # columns: the reduced basis
    Binter = lattice.matmul(Binter, Tm)
    ZB = lattice.matmul(ZB, Tm)
    mat = lattice.matmul([list(r) for r in zip(*Tm)], lattice.matmul(mat, Tm))
    return dict(h=h, d=d, Z=Z, Binter=Binter, ZB=ZB, mat=mat)


def _emit(Binter, ZB, pts, h):
    Bn, Zn = np.array(Binter, dtype=object), np.array(ZB, dtype=object)
    C = pts.astype(object).T
    if not pts.shape[0]:
        z = np.zeros((0, h), np.int64)
        return z, z.copy()
    M, Kn = (Bn @ C).T, (Zn @ C).T
    if np.max(np.abs(M)) >= 2 ** 63 or np.max(np.abs(Kn)) >= 2 ** 63:
        raise OverflowError("M or Kn beyond int64")
    return np.array(M, dtype=np.int64), np.array(Kn, dtype=np.int64)


def points(kappa, Mbasis, p, Qmax, qmax, eps=1e-4, max_out=10 ** 9):
    """(status, C (n, d) int32, M (n, h), Kn (n, h), q (n,)): status 0, or -9
    (mat not positive definite), or the kernel's status."""
    h = np.asarray(Mbasis).shape[0]
    empty = (np.zeros((0, h - 1), np.int32), np.zeros((0, h), np.int64), np.zeros((0, h), np.int64),
             np.zeros(0, np.int64))
    try:
        L = build(kappa, Mbasis, p)
    except lattice.NotPositiveDefinite:
        return (-9,) + empty
    st, U, _, _, _ = lattice.factor(L["mat"])
    if st:
        return (st,) + empty
    H = lattice.hnf(L["ZB"])
    pts, qs, st, _ = pfo.search(L["mat"], U, Qmax, qmax, 0, None, None, prune_rows=H, leaf_rows=L["ZB"],
                                strict=False, eps=eps, max_out=max_out)
    if st:
        return (st,) + empty
    M, Kn = _emit(L["Binter"], L["ZB"], pts, h)
    return 0, pts, M, Kn, qs.astype(np.int64)


def ref_points(kappa, Mbasis, p, Qmax, qmax, eps=1e-4, max_out=10 ** 9, return_nodes=False):
    """The same from the reference's own C setup and kernel (oracle/_ref):
    status 1 where its C setup fails (the reference then builds the lattice
    in python-flint code that is not built here); with return_nodes, also the
    kernel's tree nodes."""
    from . import ref
    h = np.asarray(Mbasis).shape[0]
    empty = (np.zeros((0, h - 1), np.int32), np.zeros((0, h), np.int64), np.zeros((0, h), np.int64),
             np.zeros(0, np.int64))
    st, Z, B, ZB, mat, H = ref.lattice_build(kappa, Mbasis, p, coni=False)
    nodes = 0
    if st not in (0, -15):
        res = (1,) + empty
    else:
        if H is None:
            H = lattice.hnf(ZB.tolist())
        pts, qs, st, nodes = ref.kernel(mat, Qmax, qmax, H, strict=False, max_N_out=max_out, eps=eps)
        if st:
            res = (st,) + empty
        else:
            M, Kn = _emit(B.tolist(), ZB.tolist(), pts, h)
            res = (0, pts, M, Kn, qs.astype(np.int64))
    return res + (nodes,) if return_nodes else res


def pfvs_from_points(C, M, Kn, kappa, Qmin, Qmax):
    """(Ks, Ms) of one p-vector's points, as nonconi.py:437-495 (rows)."""
    h = np.asarray(kappa).shape[0]
    if not len(C):
        return np.zeros((0, h), np.int64), np.zeros((0, h), np.int64)
    prim = np.gcd.reduce(np.abs(C.astype(np.int64)), axis=1) == 1
    M, Kn = M[prim], Kn[prim]
    if not len(M):
        return np.zeros((0, h), np.int64), np.zeros((0, h), np.int64)
    kap = np.asarray(kappa, dtype=object)
    Ns = np.array([np.tensordot(kap, m.astype(object), axes=([2], [0])) for m in M], dtype=object)
    sing = singular_mask(Ns)
    M, Kn = M[~sing], Kn[~sing]
    g = np.gcd.reduce(np.abs(Kn), axis=1)
    K = Kn // g[:, None]
    Q = -np.sum(K.astype(object) * M.astype(object), axis=1)
    keep = np.array([Qmin <= int(q) <= Qmax for q in Q], dtype=bool)
    return K[keep].astype(np.int64), M[keep].astype(np.int64)


def allow_gcds(Ks, Ms, Qmax, h11):
    """Every (a K, b M), a, b >= 1, with -a b K.M <= Qmax (nonconi.py:50-84),
    as a set of (K tuple, M tuple)."""
    out = set()
    for K, M in zip(Ks, Ms):
        q = -int(np.dot(np.asarray(K, dtype=object), np.asarray(M, dtype=object)))
        if q <= 0:                      # (numpy's Qmax // 0 is 0: no multiples, as the reference)
            continue
        for a in range(1, Qmax // q + 1):
            for b in range(1, Qmax // (a * q) + 1):
                out.add((tuple(int(a * x) for x in K), tuple(int(b * x) for x in M)))
    return out


def zpm(kappa, Mbasis, ps, Qmin, Qmax, dilation, source="oracle"):
    """Non-coni ZpM over the p-vectors ps: (set of (K, M), statuses)."""
    fn = points if source == "oracle" else ref_points
    qmax = qmax_of(Qmax, dilation)
    h = np.asarray(kappa).shape[0]
    allK, allM, sts = [], [], []
    for p in np.atleast_2d(ps):
        st, C, M, Kn, q = fn(kappa, Mbasis, p, Qmax, qmax)
        sts.append(st)
        if st == 0:
            K, Mm = pfvs_from_points(C, M, Kn, kappa, Qmin, Qmax)
            allK.append(K)
            allM.append(Mm)
    Ks = np.vstack(allK) if allK else np.zeros((0, h), np.int64)
    Ms = np.vstack(allM) if allM else np.zeros((0, h), np.int64)
    return allow_gcds(Ks, Ms, Qmax, h), np.array(sts, dtype=np.int32)
