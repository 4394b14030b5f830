"""
ORACLE / TEST INFRASTRUCTURE -- never part of the product path.

The oracle for the batched coniZpM path: this repository's CPU restatement of
the reference algorithm (setup in exact Python ints, oracle/lattice.py;
search in C, oracle/pfo.c), with the reference batch driver's semantics
(pfvs/fp_kernel/fp_kernel.pyx:480-622):

  coni_batch(...) -> (M, Kn, q, pidx, status, nodes)

for every lattice point c of every direction: M = Binter c, Kn = ZB c,
q = c^T mat c, pidx; then put in the canonical order the GPU ABI promises
(grouped by p ascending, sorted by (M, Kn) within a p; pfvs/gpu.py:155-159).

The GCD cut's leaf test uses the exact gcd of Kn[1:] = (ZB c)[1:] (the
kernel's g = gcd(H c) for H the row-HNF of ZB[1:], a unimodular image of
ZB[1:]); HNF rows that fit int64 prune.
"""
import ctypes
import os
import subprocess

import numpy as np

from . import lattice

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libpfvs_oracle.so")

_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


class _Problem(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("Q", ctypes.c_int64), ("qmax", ctypes.c_int64),
                ("linmin", ctypes.c_int64), ("strict", ctypes.c_int), ("eps", ctypes.c_double),
                ("U", _f64p), ("mat", _i64p), ("linvec", _i64p),
                ("m0N", _f64p), ("m0V", _f64p), ("m0Va", _f64p),
                ("nprune", ctypes.c_int), ("Hp", _i64p), ("nleaf", ctypes.c_int), ("Hl", _i64p),
                ("leaf_gcd", ctypes.c_int), ("max_out", ctypes.c_long)]


_lib = None


def build_lib():
    """Compile oracle/pfo.c (make -C oracle oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_lib()
        lib = ctypes.CDLL(LIB_PATH)
        lib.pfo_search.restype = ctypes.c_int
        lib.pfo_search.argtypes = [ctypes.POINTER(_Problem), ctypes.POINTER(_i32p),
                                   ctypes.POINTER(_i64p), ctypes.POINTER(ctypes.c_long),
                                   ctypes.POINTER(ctypes.c_long)]
        lib.pfo_free.argtypes = [ctypes.c_void_p]
        _lib = lib
    return _lib


def _i64(a):
    return np.ascontiguousarray(np.array(a, dtype=np.int64))


def search(mat, U, Q, qmax, linmin, linvec=None, m0=None, prune_rows=(), leaf_rows=None,
           strict=True, eps=1e-4, max_out=10**9):
    """One run of the restated kernel.  leaf_rows None: the exact GCD test is
    left to the caller.  Returns (pts (n, d) int32, qs (n,) int64, status, nodes)."""
    lib = _load()
    mat = _i64(mat)
    d = mat.shape[0]
    U = np.ascontiguousarray(U, dtype=np.float64)
    keep = [mat, U]
    P = _Problem()
    P.dim, P.Q, P.qmax, P.linmin, P.strict, P.eps = d, int(Q), int(qmax), int(linmin), int(strict), eps
    P.U = U.ctypes.data_as(_f64p)
    P.mat = mat.ctypes.data_as(_i64p)
    if linvec is not None:
        lv = _i64(linvec)
        N, V, Va = (np.ascontiguousarray(x, dtype=np.float64) for x in m0)
        keep += [lv, N, V, Va]
        P.linvec = lv.ctypes.data_as(_i64p)
        P.m0N, P.m0V, P.m0Va = (x.ctypes.data_as(_f64p) for x in (N, V, Va))
    rows = [r for r in prune_rows if all(abs(int(x)) < 2**63 for x in r)]
    Hp = _i64(rows).reshape(-1, d) if rows else np.zeros((1, d), dtype=np.int64)
    keep.append(Hp)
    P.nprune = len(rows)
    P.Hp = Hp.ctypes.data_as(_i64p)
    if leaf_rows is not None:
        Hl = _i64(leaf_rows).reshape(-1, d)
        keep.append(Hl)
        P.nleaf, P.Hl, P.leaf_gcd = Hl.shape[0], Hl.ctypes.data_as(_i64p), 1
    else:
        P.nleaf, P.leaf_gcd = 0, 0
    P.max_out = int(max_out)
    pts_p, qs_p = _i32p(), _i64p()
    n, nn = ctypes.c_long(0), ctypes.c_long(0)
    st = lib.pfo_search(ctypes.byref(P), ctypes.byref(pts_p), ctypes.byref(qs_p),
                        ctypes.byref(n), ctypes.byref(nn))
    try:
        m = n.value
        pts = np.ctypeslib.as_array(pts_p, shape=(m, d)).copy() if m else np.zeros((0, d), np.int32)
        qs = np.ctypeslib.as_array(qs_p, shape=(m,)).copy() if m else np.zeros(0, np.int64)
    finally:
        lib.pfo_free(ctypes.cast(pts_p, ctypes.c_void_p))
        lib.pfo_free(ctypes.cast(qs_p, ctypes.c_void_p))
    return pts, qs, st, nn.value


def kernel(mat, Q, qmax, H, linvec=None, linmin=0, strict=True, eps=1e-12, max_out=10**9):
    """
    The kernel boundary (conipfv_kernel / pfv_kernel semantics): exact output
    for an integral ellipsoid mat, GCD rows H (Python ints, any size; rows
    beyond int64 only lose pruning), optional M0 cut.  The exact GCD test on
    all of H is done here in Python ints.  Returns (pts, qs, status, nodes).
    """
    st, U, N, V, Va = lattice.factor(mat, linvec)
    if st:
        return np.zeros((0, len(mat)), np.int32), np.zeros(0, np.int64), st, 0
    m0 = (N, V, Va) if linvec is not None else None
    pts, qs, st, nodes = search(mat, U, Q, qmax, linmin, linvec, m0, prune_rows=H,
                                leaf_rows=None, strict=strict, eps=eps, max_out=max_out)
    Hl = [[int(x) for x in r] for r in H]
    keep = []
    for c, q in zip(pts.tolist(), qs.tolist()):
        g = 0
        for r in Hl:
            g = _gcd(g, sum(a * b for a, b in zip(r, c)))
        keep.append(g == 0 or (Q * g > q if strict else Q * g >= q))
    keep = np.array(keep, dtype=bool) if len(keep) else np.zeros(0, bool)
    return pts[keep], qs[keep], st, nodes


def _gcd(a, b):
    a, b = abs(a), abs(b)
    while b:
        a, b = b, a % b
    return a


def direction(kappa, Mbasis, p, Q, qmax, linmin, eps=1e-4, max_out=10**9, prune=True):
    """Setup + search + emission for one direction.  Returns
    (M (n,h), Kn (n,h), q (n,), status, nodes)."""
    try:
        L = lattice.build(kappa, Mbasis, p)
    except lattice.NotPositiveDefinite:
        h = np.asarray(Mbasis).shape[0]
        return (np.zeros((0, h), np.int64), np.zeros((0, h), np.int64), np.zeros(0, np.int64), -9, 0)
    h, d = L["h"], L["d"]
    B, ZB, mat = L["Binter"], L["ZB"], L["mat"]
    st, U, N, V, Va = lattice.factor(mat, B[0])
    empty = (np.zeros((0, h), np.int64), np.zeros((0, h), np.int64), np.zeros(0, np.int64))
    if st:
        return empty + (st, 0)
    H = lattice.hnf([r for r in ZB[1:]]) if prune else []
    for r in ZB + mat:
        if any(abs(x) >= 2**63 for x in r):
            raise OverflowError("lattice data beyond int64")
    pts, qs, st, nodes = search(mat, U, Q, qmax, linmin, B[0], (N, V, Va), prune_rows=H,
                                leaf_rows=ZB[1:], eps=eps, max_out=max_out)
    if st:
        return empty + (st, nodes)
    Bn = np.array(B, dtype=object)
    Zn = np.array(ZB, dtype=object)
    C = pts.astype(object).T
    M = (Bn @ C).T if len(qs) else np.zeros((0, h), dtype=object)
    Kn = (Zn @ C).T if len(qs) else np.zeros((0, h), dtype=object)
    if len(qs) and (np.max(np.abs(M)) >= 2**63 or np.max(np.abs(Kn)) >= 2**63):
        raise OverflowError("M or Kn beyond int64")
    return (np.array(M, dtype=np.int64).reshape(-1, h), np.array(Kn, dtype=np.int64).reshape(-1, h),
            qs.astype(np.int64), 0, nodes)


def canonical_order(M, Kn, pidx):
    """Indices sorting points by (pidx, M, Kn) lexicographically
    (pfvs/gpu.py:155-159; pfvs/coni.py:322-324)."""
    keys = tuple(Kn[:, j] for j in range(Kn.shape[1] - 1, -1, -1)) + \
        tuple(M[:, j] for j in range(M.shape[1] - 1, -1, -1)) + (pidx,)
    return np.lexsort(keys) if len(pidx) else np.zeros(0, dtype=np.int64)


def coni_batch(kappa, Mbasis, ps, Q, dilation, M0min, eps=1e-4, max_out=10**9, prune=True):
    """
    The oracle for one geometry: (M, Kn, q, pidx, status, nodes), points in
    the canonical order.  status per direction: 0 done, < 0 the kernel status.
    """
    from .ref import qmax_of, linmin_of
    ps = np.asarray(ps, dtype=np.int64)
    h = np.asarray(Mbasis).shape[0]
    qmax, linmin = qmax_of(Q, dilation), linmin_of(M0min)
    Ms, Ks, qs, pid, status, nodes = [], [], [], [], [], []
    for ip, p in enumerate(ps.reshape(-1, h)):
        M, Kn, q, st, nn = direction(kappa, Mbasis, p, Q, qmax, linmin, eps, max_out, prune)
        status.append(st)
        nodes.append(nn)
        if st == 0:
            Ms.append(M); Ks.append(Kn); qs.append(q); pid.append(np.full(len(q), ip, np.int64))
    if Ms:
        M, Kn, q, pidx = np.vstack(Ms), np.vstack(Ks), np.concatenate(qs), np.concatenate(pid)
    else:
        M = Kn = np.zeros((0, h), np.int64)
        q = pidx = np.zeros(0, np.int64)
    o = canonical_order(M, Kn, pidx)
    return M[o], Kn[o], q[o], pidx[o], np.array(status, np.int32), np.array(nodes, np.int64)
