"""TEST INFRASTRUCTURE: ctypes wrapper for tests/emu/_build/libpfvs_emu.so
(the library's device kernels run on CPU threads under warp_emu.h)."""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libpfvs_emu.so")
SRCS = [os.path.join(HERE, f) for f in ("emu_driver.cpp", "warp_emu.h")] + [
    os.path.join(HERE, "..", "..", "pfvs_b200", "csrc", f) for f in
    ("pfg_int.cuh", "pfg_types.cuh", "pfg_setup.cuh", "pfg_search.cuh", "pfg_out.cuh", "pfg_mu0.cuh", "pfg_zpk.cuh")] + [
    os.path.join(HERE, "..", "..", "include", "pfvs_gpu.h")]
_lib = None


def build():
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if os.path.exists(LIB) and all(os.path.getmtime(s) <= os.path.getmtime(LIB) for s in SRCS):
        return
    # -DPFG_SORT_CAP=1: the output sort starts from runs of one point here, so that
    # every direction with 2 or more points goes through the run-merge passes
    subprocess.run(["g++", "-std=c++20", "-O1", "-g", "-pthread", "-shared", "-fPIC", "-w",
                    "-DPFG_SORT_CAP=1", os.path.join(HERE, "emu_driver.cpp"), "-o", LIB], check=True)


def _load():
    global _lib
    if _lib is None:
        build()
        from pfvs_b200 import gpu
        lib = ctypes.CDLL(LIB)
        lib.emu_coni_batch.argtypes = [ctypes.POINTER(gpu._Input), ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(gpu._Output), ctypes.POINTER(ctypes.c_int64),
                                       ctypes.POINTER(ctypes.c_int32)]
        lib.emu_coni_batch.restype = ctypes.c_int
        lib.emu_output_free.argtypes = [ctypes.POINTER(gpu._Output)]
        lib.emu_witness_not_pd.argtypes = [ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
        lib.emu_witness_not_pd.restype = ctypes.c_int
        lib.emu_last_fp32_check.argtypes = [ctypes.POINTER(ctypes.c_double)]
        lib.emu_set_gcd_min_tree.argtypes = [ctypes.c_double]
        lib.emu_set_coni.argtypes = [ctypes.c_int]
        _lib = lib
    return _lib


def coni_batch_multi(geoms, ps, pgeo, precision=2, n_warps=2, coni=True):
    """As pfvs_b200.gpu.coni_batch_multi, on the emulated warps (default: FP32
    pruning with the FP64 retry, so that both search instantiations run); with
    coni False the non-coni ZpM of pfg_zpm_batch (geometry Q = Qmax).  Returns
    (M, Kn, q, pidx, pstat, dir_nodes, setup_failure_stage)."""
    from pfvs_b200 import gpu
    lib = _load()
    MH = 64
    h, Q, qmax, linmin, kap, Mb, P, pgeo, n_p = gpu._pack(geoms, ps, pgeo, MH)
    i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
    inp = gpu._Input(len(geoms), h.ctypes.data_as(i32p), Q.ctypes.data_as(i64p),
                     qmax.ctypes.data_as(i64p), linmin.ctypes.data_as(i64p),
                     kap.ctypes.data_as(i64p), Mb.ctypes.data_as(i64p), n_p,
                     P.ctypes.data_as(i64p), pgeo.ctypes.data_as(i32p), 0, 0, 0)
    out = gpu._Output()
    dn = np.zeros(max(n_p, 1), np.int64)
    dbg = np.zeros(max(n_p, 1), np.int32)
    lib.emu_set_coni(int(bool(coni)))
    try:
        rc = lib.emu_coni_batch(ctypes.byref(inp), int(precision), int(n_warps), ctypes.byref(out),
                                dn.ctypes.data_as(i64p), dbg.ctypes.data_as(i32p))
    finally:
        lib.emu_set_coni(1)
    if rc:
        raise RuntimeError(out.err.decode())
    try:
        n = out.n
        arr = (lambda p, s: np.ctypeslib.as_array(p, shape=s).copy() if n else np.zeros(s, np.int64))
        M, Kn = arr(out.M, (n, MH)), arr(out.Kn, (n, MH))
        q, pidx = arr(out.q, (n,)), arr(out.pidx, (n,))
        pstat = np.ctypeslib.as_array(out.pstat, shape=(n_p,)).copy()
    finally:
        lib.emu_output_free(ctypes.byref(out))
    return M, Kn, q, pidx, pstat, dn[:n_p], dbg[:n_p]


def witness_not_pd(A):
    """The setup's exact witness that the symmetric integer matrix A is not
    positive definite (True: proved indefinite; False: no witness found)."""
    lib = _load()
    A = np.ascontiguousarray(A, dtype=np.int64)
    return bool(lib.emu_witness_not_pd(A.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), A.shape[0]))


def last_fp32_check():
    """After coni_batch_multi(..., precision=3) (FP32 pruning in the bound-check
    form): dict of the FP32-versus-FP64 bound errors of that run."""
    lib = _load()
    b = (ctypes.c_double * 4)()
    lib.emu_last_fp32_check(b)
    return dict(rem_err=b[0], margin_frac=b[1], end_err=b[2], narrower=int(b[3]))


def set_gcd_min_tree(v):
    """GCD-row policy of the emulated setup, as pfg_options.gcd_min_tree
    (0: the library default; < 0: rows for every direction)."""
    _load().emu_set_gcd_min_tree(float(v))


def coni_mu0_batch(kappa, p_r):
    """The device's coni dilation bound on the emulated warp: (status, mu_num,
    mu_den, K) for the rows of p_r ((n, h-1))."""
    lib = _load()
    i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
    lib.emu_coni_mu0_batch.argtypes = [ctypes.c_int, i64p, ctypes.c_int64, i64p, i32p, i64p, i64p, i64p]
    kappa = np.ascontiguousarray(kappa, dtype=np.int64)
    h = kappa.shape[0]
    p_r = np.ascontiguousarray(p_r, dtype=np.int64).reshape(-1, h - 1)
    n = len(p_r)
    st = np.zeros(max(n, 1), np.int32)
    num, den = np.zeros(max(n, 1), np.int64), np.zeros(max(n, 1), np.int64)
    K = np.zeros((max(n, 1), h - 1), np.int64)
    lib.emu_coni_mu0_batch(h, kappa.ctypes.data_as(i64p), n, p_r.ctypes.data_as(i64p), st.ctypes.data_as(i32p),
                           num.ctypes.data_as(i64p), den.ctypes.data_as(i64p), K.ctypes.data_as(i64p))
    return st[:n], num[:n], den[:n], K[:n]


def coni_zpk_batch(kappa, Mbasis, ps, Q, M0min, D0, max_out=10**9, budget=10**9):
    """The device's coniZpK above D0 on the emulated warp: (M (N, h), Kn, q,
    pidx, status) for the rows of ps ((n, h), p[0] = 0); points of every row
    (the caller keeps those whose row has status 0)."""
    lib = _load()
    i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
    lib.emu_coni_zpk_batch.restype = ctypes.c_longlong
    lib.emu_coni_zpk_batch.argtypes = [ctypes.c_int, i64p, i64p, i64p, ctypes.c_int64, ctypes.c_int64,
                                       ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_longlong,
                                       ctypes.c_ulonglong, i64p, i64p, i64p, i64p, i32p]
    kappa = np.ascontiguousarray(kappa, dtype=np.int64)
    Mbasis = np.ascontiguousarray(Mbasis, dtype=np.int64)
    h = Mbasis.shape[0]
    ps = np.ascontiguousarray(np.atleast_2d(ps), dtype=np.int64).reshape(-1, h)
    n = len(ps)
    st = np.zeros(max(n, 1), np.int32)
    cap = 1024
    while True:
        M, Kn = np.zeros((cap, 64), np.int64), np.zeros((cap, 64), np.int64)
        q, pidx = np.zeros(cap, np.int64), np.zeros(cap, np.int64)
        N = lib.emu_coni_zpk_batch(h, kappa.ctypes.data_as(i64p), Mbasis.ctypes.data_as(i64p),
                                   ps.ctypes.data_as(i64p), n, int(Q), int(M0min), int(D0), int(max_out),
                                   int(budget), cap, M.ctypes.data_as(i64p), Kn.ctypes.data_as(i64p),
                                   q.ctypes.data_as(i64p), pidx.ctypes.data_as(i64p), st.ctypes.data_as(i32p))
        if N <= cap:
            return M[:N, :h], Kn[:N, :h], q[:N], pidx[:N], st[:n]
        cap = N
