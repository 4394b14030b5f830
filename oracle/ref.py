"""
ORACLE / TEST INFRASTRUCTURE -- never part of the product path.

ctypes wrapper around oracle/_ref/libpfvs_ref.so: the reference's own CPU
kernel (pfvs/fp_kernel/pfv_lattice.h + fp_kernel.h, compiled in place by
oracle/Makefile) behind the driver oracle/ref_harness.c.

- `coni_batch`   -- the reference batch loop `_coni_batch`
                    (pfvs/fp_kernel/fp_kernel.pyx:480-622): per p-vector
                    lattice setup + Fincke-Pohst search -> (M, Kn, q, pidx,
                    status), plus per-p search-tree node counts.
- `kernel`       -- the kernel boundary `conipfv_kernel` / `pfv_kernel`
                    (fp_kernel.pyx:258-350), H with arbitrary-precision rows.
- `lattice_build`-- `_lattice_build` (fp_kernel.pyx:355-401).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use it.
"""
import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libpfvs_ref.so")

_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)


class _Points(ctypes.Structure):
    _fields_ = [("M", _i64p), ("Kn", _i64p), ("q", _i64p), ("pidx", _i64p),
                ("n", ctypes.c_long), ("cap", ctypes.c_long)]


_lib = None


def available():
    return os.path.exists(LIB_PATH)


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built (make -C oracle ref)")
        lib = ctypes.CDLL(LIB_PATH)
        lib.ref_coni_batch.restype = ctypes.c_int
        lib.ref_coni_batch.argtypes = [
            ctypes.c_int, _i64p, _i64p, _i64p, ctypes.c_long, ctypes.c_int64,
            ctypes.c_int64, ctypes.c_int64, ctypes.c_long, ctypes.c_double,
            ctypes.c_long, ctypes.c_int, ctypes.POINTER(_Points), _i32p, _i64p]
        lib.ref_points_free.argtypes = [ctypes.POINTER(_Points)]
        lib.ref_kernel.restype = ctypes.c_int
        lib.ref_kernel.argtypes = [
            ctypes.c_int, _i64p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
            ctypes.POINTER(ctypes.c_int8), ctypes.POINTER(ctypes.c_uint64), ctypes.c_int,
            ctypes.c_int, _i64p, ctypes.c_int64, ctypes.c_long, ctypes.c_double,
            ctypes.POINTER(_i32p), ctypes.POINTER(_i64p), ctypes.POINTER(ctypes.c_long),
            ctypes.POINTER(ctypes.c_long)]
        lib.ref_free.argtypes = [ctypes.c_void_p]
        lib.ref_coni_mu0.restype = ctypes.c_int
        lib.ref_coni_mu0.argtypes = [ctypes.c_int, _i64p, _i64p, _i64p, _i64p, _i64p]
        lib.ref_coni_mu0_batch.restype = None
        lib.ref_coni_mu0_batch.argtypes = [ctypes.c_int, _i64p, ctypes.c_int64, _i64p,
                                           ctypes.POINTER(ctypes.c_int32), _i64p, _i64p, _i64p]
        lib.ref_coni_zpk_batch.restype = ctypes.c_long
        lib.ref_coni_zpk_batch.argtypes = [
            ctypes.c_int, _i64p, _i64p, _i64p, ctypes.c_long, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
            ctypes.c_long, ctypes.POINTER(_i64p), ctypes.POINTER(_i64p), ctypes.POINTER(_i64p),
            ctypes.POINTER(_i64p), _i32p]
        lib.ref_lattice_build.restype = ctypes.c_int
        lib.ref_lattice_build.argtypes = [
            ctypes.c_int, _i64p, _i64p, _i64p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            _i64p, _i64p, _i64p, _i64p, _i64p, ctypes.POINTER(ctypes.c_int)]
        _lib = lib
    return _lib


def qmax_of(Q, dilation):
    """floor(dilation * Q), tolerant of float noise (fp_kernel.pyx:145-147)."""
    return int(math.floor(dilation * Q + 1e-7))


def linmin_of(M0min):
    """ceil(M0min - 1e-9) (fp_kernel.pyx:524)."""
    return int(math.ceil(M0min - 1e-9))


def _p(a):
    return a.ctypes.data_as(_i64p)


def coni_batch(kappa, Mbasis, ps, Q, dilation, M0min, max_N_out=10**9, eps=1e-4,
               pidx_base=0, per_p=True):
    """
    The reference CPU batch (fp_kernel.pyx:_coni_batch) for one geometry.
    ps: (n, h) int64 p-vectors *with* the leading 0.  Returns
    (M, Kn, q, pidx, status, nodes): points in per-p DFS order, status per p
    (0 done, 1 exact per-p path needed, <0 kernel status) and the kernel's
    search-tree node count per p.  With per_p (default), directions the
    batch loop hands on because H does not fit int64 are finished as the
    reference's per-p path does (H rows in GMP); only a setup overflow then
    leaves status 1.
    """
    lib = _load()
    kappa = np.ascontiguousarray(kappa, dtype=np.int64)
    Mbasis = np.ascontiguousarray(Mbasis, dtype=np.int64)
    h = Mbasis.shape[0]
    ps = np.ascontiguousarray(ps, dtype=np.int64).reshape(-1, h)
    n = ps.shape[0]
    status = np.zeros(max(n, 1), dtype=np.int32)
    nodes = np.zeros(max(n, 1), dtype=np.int64)
    out = _Points()
    rc = lib.ref_coni_batch(h, _p(kappa), _p(Mbasis), _p(ps), n, int(Q),
                            qmax_of(Q, dilation), linmin_of(M0min), int(max_N_out),
                            float(eps), int(pidx_base), int(bool(per_p)), ctypes.byref(out),
                            status.ctypes.data_as(_i32p), _p(nodes))
    try:
        if rc != 0:
            raise MemoryError("reference batch ran out of memory")
        m = out.n

        def arr(ptr, shape):
            if m == 0:
                return np.zeros(shape, dtype=np.int64)
            return np.ctypeslib.as_array(ptr, shape=shape).copy()
        M, Kn = arr(out.M, (m, h)), arr(out.Kn, (m, h))
        q, pidx = arr(out.q, (m,)), arr(out.pidx, (m,))
    finally:
        lib.ref_points_free(ctypes.byref(out))
    return M, Kn, q, pidx, status[:n], nodes[:n]


def kernel(mat, Q, qmax, H, linvec=None, linmin=0, strict=True, max_N_out=10**9,
           eps=1e-12):
    """
    The reference kernel boundary (fpk_enumerate via conipfv_kernel /
    pfv_kernel).  H: rows of Python ints (any size).  Returns
    (pts (n, dim) int32, qs (n,) int64, status, n_nodes).
    """
    lib = _load()
    mat = np.ascontiguousarray(np.array([[int(x) for x in r] for r in mat], dtype=np.int64))
    dim = mat.shape[0]
    Hl = [[int(x) for x in r] for r in H]
    nrows = len(Hl)
    bits = max([abs(x).bit_length() for r in Hl for x in r] + [1])
    nl = max(1, (bits + 63) // 64)
    sign = np.ones(max(nrows * dim, 1), dtype=np.int8)
    limbs = np.zeros(max(nrows * dim, 1) * nl, dtype=np.uint64)
    for r in range(nrows):
        for j in range(dim):
            e = r * dim + j
            x = Hl[r][j]
            if x < 0:
                sign[e] = -1
                x = -x
            for k in range(nl):
                limbs[e * nl + k] = (x >> (64 * k)) & 0xFFFFFFFFFFFFFFFF
    lv = None
    if linvec is not None:
        lv = np.ascontiguousarray(np.array([int(x) for x in linvec], dtype=np.int64))
    pts_p = _i32p()
    qs_p = _i64p()
    n = ctypes.c_long(0)
    nn = ctypes.c_long(0)
    st = lib.ref_kernel(dim, _p(mat), int(qmax), int(Q), nrows,
                        sign.ctypes.data_as(ctypes.POINTER(ctypes.c_int8)),
                        limbs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), nl,
                        int(bool(strict)), _p(lv) if lv is not None else None, int(linmin),
                        int(max_N_out), float(eps), ctypes.byref(pts_p), ctypes.byref(qs_p),
                        ctypes.byref(n), ctypes.byref(nn))
    try:
        m = n.value
        pts = np.ctypeslib.as_array(pts_p, shape=(m, dim)).copy() if m else \
            np.zeros((0, dim), dtype=np.int32)
        qs = np.ctypeslib.as_array(qs_p, shape=(m,)).copy() if m else np.zeros(0, dtype=np.int64)
    finally:
        lib.ref_free(ctypes.cast(pts_p, ctypes.c_void_p))
        lib.ref_free(ctypes.cast(qs_p, ctypes.c_void_p))
    return pts, qs, st, nn.value


def lattice_build(kappa, Mbasis, p, coni=True, extra_lll=True, m0_basis=True):
    """The reference per-p setup (pfl_build).  Returns (status, Z, Binter,
    ZB, mat, H) with H as Python-int rows (None unless status 0)."""
    lib = _load()
    kappa = np.ascontiguousarray(kappa, dtype=np.int64)
    Mbasis = np.ascontiguousarray(Mbasis, dtype=np.int64)
    h = Mbasis.shape[0]
    d = h - 1
    p = np.ascontiguousarray(p, dtype=np.int64)
    Z = np.zeros(h * h, dtype=np.int64)
    B = np.zeros(h * d, dtype=np.int64)
    ZB = np.zeros(h * d, dtype=np.int64)
    mat = np.zeros(d * d, dtype=np.int64)
    Hw = np.zeros(2 * h * d, dtype=np.int64)
    nr = ctypes.c_int(0)
    st = lib.ref_lattice_build(h, _p(kappa), _p(Mbasis), _p(p), int(coni), int(extra_lll),
                               int(m0_basis), _p(Z), _p(B), _p(ZB), _p(mat), _p(Hw),
                               ctypes.byref(nr))
    if st not in (0, -15):
        return st, None, None, None, None, None
    H = None
    if st == 0:
        H = []
        for r in range(nr.value):
            row = []
            for j in range(d):
                k = r * d + j
                lo = int(Hw[2 * k]) & 0xFFFFFFFFFFFFFFFF
                hi = int(Hw[2 * k + 1])
                row.append((hi << 64) + lo)
            H.append(row)
    return (st, Z.reshape(h, h), B.reshape(h, d), ZB.reshape(h, d), mat.reshape(d, d), H)


def coni_mu0(kappa, p_r):
    """The reference's C dilation bound (coni_bound.h:255): (status, mu0 as a
    Fraction or None, K) with status 0 decided, 1 no bound, < 0 undecided in C."""
    from fractions import Fraction
    lib = _load()
    kappa = np.ascontiguousarray(kappa, dtype=np.int64)
    h = kappa.shape[0]
    p_r = np.ascontiguousarray(p_r, dtype=np.int64).reshape(h - 1)
    num, den = np.zeros(1, np.int64), np.zeros(1, np.int64)
    K = np.zeros(h - 1, np.int64)
    st = lib.ref_coni_mu0(h, _p(kappa), _p(p_r), _p(num), _p(den), _p(K))
    return st, (Fraction(int(num[0]), int(den[0])) if st == 0 else None), K


def coni_mu0_batch(kappa, P):
    """The reference's C dilation bound over the rows of P ((n, h-1)), in one
    C loop: (status int32, mu_num, mu_den, K) arrays."""
    lib = _load()
    kappa = np.ascontiguousarray(kappa, dtype=np.int64)
    h = kappa.shape[0]
    P = np.ascontiguousarray(np.atleast_2d(P), dtype=np.int64).reshape(-1, h - 1)
    n = len(P)
    st = np.zeros(max(n, 1), np.int32)
    num, den = np.zeros(max(n, 1), np.int64), np.zeros(max(n, 1), np.int64)
    K = np.zeros((max(n, 1), h - 1), np.int64)
    lib.ref_coni_mu0_batch(h, _p(kappa), n, _p(P), st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _p(num),
                           _p(den), _p(K))
    return st[:n], num[:n], den[:n], K[:n]


def coni_zpk_batch(kappa, Mbasis, ps, Q, M0min, D0, max_out=10**9):
    """The reference's C coniZpK above D0 (coni_zpk.h:714) over the rows of ps
    ((n, h), p[0] = 0): (M (N, h), Kn (N, h), q (N,), pidx (N,), status (n,)
    int32), the points of the rows with status 0, in the reference's order."""
    lib = _load()
    kappa = np.ascontiguousarray(kappa, dtype=np.int64)
    Mbasis = np.ascontiguousarray(Mbasis, dtype=np.int64)
    h = Mbasis.shape[0]
    ps = np.ascontiguousarray(np.atleast_2d(ps), dtype=np.int64).reshape(-1, h)
    n = len(ps)
    st = np.zeros(max(n, 1), np.int32)
    Mp, Kp, qp, pp = _i64p(), _i64p(), _i64p(), _i64p()
    N = lib.ref_coni_zpk_batch(h, _p(kappa), _p(Mbasis), _p(ps), n, int(Q), int(M0min), int(D0), int(max_out),
                               ctypes.byref(Mp), ctypes.byref(Kp), ctypes.byref(qp), ctypes.byref(pp),
                               st.ctypes.data_as(_i32p))
    try:
        M = np.ctypeslib.as_array(Mp, shape=(N, h)).copy() if N else np.zeros((0, h), np.int64)
        Kn = np.ctypeslib.as_array(Kp, shape=(N, h)).copy() if N else np.zeros((0, h), np.int64)
        q = np.ctypeslib.as_array(qp, shape=(N,)).copy() if N else np.zeros(0, np.int64)
        pidx = np.ctypeslib.as_array(pp, shape=(N,)).copy() if N else np.zeros(0, np.int64)
    finally:
        for a in (Mp, Kp, qp, pp):
            if a:
                lib.ref_free(ctypes.cast(a, ctypes.c_void_p))
    return M, Kn, q, pidx, st[:n]
