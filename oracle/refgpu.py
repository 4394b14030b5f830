"""
ORACLE / TEST INFRASTRUCTURE -- never part of the product path.

The reference's own CUDA backend (pfvs/fp_kernel/cuda/pfvs_gpu.cu, built
unmodified for sm_100a by `make -C oracle refgpu` into
oracle/_refgpu/libpfvs_refgpu{12,24}.so, PFL_MAX_H11 = 12 and 24) as a
comparator: the same C ABI as libpfvs_gpu.so (pfg_input / pfg_output,
pfvs_gpu.cu:66-88).  Each call runs in a subprocess of its own, so that this
library and the reference's never share a process (each links its own CUDA
runtime).

  coni_batch_multi(geoms, ps, pgeo, max_h11=24) ->
      (M, Kn, q, pidx, pstat, seconds_gpu, wall_seconds)

pstat 1 marks directions that build hands to the reference's CPU path
(none of their points are returned).
"""
import ctypes
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


def lib_path(max_h11):
    return os.path.join(_HERE, "_refgpu", f"libpfvs_refgpu{int(max_h11)}.so")


def available(max_h11=24):
    return os.path.exists(lib_path(max_h11))


_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)


class _In(ctypes.Structure):
    _fields_ = [("n_geo", ctypes.c_int), ("h", _i32p), ("Q", _i64p), ("qmax", _i64p),
                ("linmin", _i64p), ("kappa", _i64p), ("Mbasis", _i64p), ("n_p", ctypes.c_int64),
                ("ps", _i64p), ("pgeo", _i32p), ("device", ctypes.c_int), ("batch", ctypes.c_int64),
                ("verbose", ctypes.c_int)]


class _Out(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("M", _i64p), ("Kn", _i64p), ("q", _i64p), ("pidx", _i64p),
                ("pstat", ctypes.POINTER(ctypes.c_int8)), ("seconds_gpu", ctypes.c_double),
                ("err", ctypes.c_char * 256)]


def _child(path_in, path_out, so, reps):
    """Subprocess body: load the reference backend, run the saved call `reps`
    times (the first untimed), save the last result."""
    z = np.load(path_in)
    lib = ctypes.CDLL(so)
    lib.pfg_max_h11.restype = ctypes.c_int
    lib.pfg_coni_batch.argtypes = [ctypes.POINTER(_In), ctypes.POINTER(_Out)]
    lib.pfg_coni_batch.restype = ctypes.c_int
    lib.pfg_output_free.argtypes = [ctypes.POINTER(_Out)]
    MH = lib.pfg_max_h11()
    h, Q, qmax, linmin = (np.ascontiguousarray(z[k]) for k in ("h", "Q", "qmax", "linmin"))
    kap, Mb, pgeo = (np.ascontiguousarray(z[k]) for k in ("kappa", "Mbasis", "pgeo"))
    ps = np.ascontiguousarray(z["ps"][:, :MH]) if z["ps"].shape[1] >= MH else None
    if ps is None:
        ps = np.zeros((z["ps"].shape[0], MH), np.int64)
        ps[:, :z["ps"].shape[1]] = z["ps"]
    n_p = len(pgeo)
    inp = _In(len(h), h.ctypes.data_as(_i32p), Q.ctypes.data_as(_i64p), qmax.ctypes.data_as(_i64p),
              linmin.ctypes.data_as(_i64p), kap.ctypes.data_as(_i64p), Mb.ctypes.data_as(_i64p), n_p,
              ps.ctypes.data_as(_i64p), pgeo.ctypes.data_as(_i32p), 0, 0, 0)
    secs, walls, res = [], [], None
    for r in range(reps):
        out = _Out()
        t0 = time.perf_counter()
        rc = lib.pfg_coni_batch(ctypes.byref(inp), ctypes.byref(out))
        wall = time.perf_counter() - t0
        if rc != 0:
            raise SystemExit("reference GPU backend failed: " + out.err.decode(errors="replace"))
        n = out.n
        arr = (lambda p, s: np.ctypeslib.as_array(p, shape=s).copy() if n else np.zeros(s, np.int64))
        res = (arr(out.M, (n, MH)), arr(out.Kn, (n, MH)), arr(out.q, (n,)), arr(out.pidx, (n,)),
               np.ctypeslib.as_array(out.pstat, shape=(n_p,)).copy())
        lib.pfg_output_free(ctypes.byref(out))
        if r > 0 or reps == 1:
            secs.append(out.seconds_gpu)
            walls.append(wall)
    np.savez(path_out, M=res[0], Kn=res[1], q=res[2], pidx=res[3], pstat=res[4],
             seconds_gpu=np.array(secs), wall=np.array(walls))


def coni_batch_multi(geoms, ps, pgeo, max_h11=24, reps=1, timeout=1800):
    """The reference backend's pfg_coni_batch on the layout (a subprocess).
    With reps > 1 the first call is a warm-up and the times are those of the
    other calls.  Rows are 64 wide (zero-padded from the build's MH)."""
    so = lib_path(max_h11)
    if not os.path.exists(so):
        raise RuntimeError(f"{so} is not built (make -C oracle refgpu)")
    h = np.array([np.asarray(g["kappa"]).shape[0] for g in geoms], dtype=np.int32)
    if h.max() > max_h11:
        raise ValueError(f"the reference GPU build supports h11 <= {max_h11}")
    Q = np.array([int(g["Q"]) for g in geoms], dtype=np.int64)
    qmax = np.array([int(math.floor(g["dilation"] * int(g["Q"]) + 1e-7)) for g in geoms], dtype=np.int64)
    linmin = np.array([math.ceil(g["M0min"] - 1e-9) for g in geoms], dtype=np.int64)
    kap = np.concatenate([np.asarray(g["kappa"], np.int64).ravel() for g in geoms])
    Mb = np.concatenate([np.asarray(g["Mbasis"], np.int64).ravel() for g in geoms])
    P = np.zeros((len(ps), 64), dtype=np.int64)
    for i, p in enumerate(ps):
        P[i, :len(p)] = p
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.npz"), os.path.join(td, "out.npz")
        np.savez(fin, h=h, Q=Q, qmax=qmax, linmin=linmin, kappa=kap, Mbasis=Mb, ps=P,
                 pgeo=np.asarray(pgeo, dtype=np.int32))
        root = os.path.dirname(_HERE)
        subprocess.run([sys.executable, "-c",
                        "import sys; sys.path.insert(0, %r); from oracle import refgpu; "
                        "refgpu._child(%r, %r, %r, %d)" % (root, fin, fout, so, int(reps))],
                       check=True, timeout=timeout)
        z = np.load(fout)
        MH = z["M"].shape[1]
        pad = (lambda a: np.concatenate([a, np.zeros((a.shape[0], 64 - MH), np.int64)], axis=1))
        return (pad(z["M"]), pad(z["Kn"]), z["q"], z["pidx"], z["pstat"],
                float(np.mean(z["seconds_gpu"])), float(np.mean(z["wall"])))
