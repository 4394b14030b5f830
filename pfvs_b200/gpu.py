"""
The B200 backend of the batched coni pipeline, loaded with ctypes -- the
same module interface as the reference's `pfvs.gpu` (pfvs/gpu.py:26-232):
`available`, `unavailable_reason`, `backend`, `release`, `max_h11`,
`coni_batch_multi`, `coni_batch`.  The library is libpfvs_gpu.so next to
this module (pfvs_b200/fp_kernel/) or the file named by PFVS_GPU_LIB, as
the reference looks it up (pfvs/gpu.py:57-82).

Differences from the reference backend (all within its contract): every
direction is finished on the device -- `pstat` is 0, or a negative kernel
status (-8 coordinates beyond int32, -9 not positive definite, -20 exact
values beyond the device's integers, -21 FP64 factor not certified) that
`coniZpM` turns into IncompleteSearchError; never 1 ("redo on the CPU").
`coni_batch_multi_ex` adds the search form, the pruning precision and
statistics.
"""
import ctypes
import glob
import math
import os

import numpy as np

_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)

FORM_BATCHED, FORM_PLAIN = 0, 1
PREC_AUTO, PREC_FP64, PREC_FP32 = 0, 1, 2


class _Input(ctypes.Structure):
    _fields_ = [("n_geo", ctypes.c_int), ("h", _i32p),
                ("Q", _i64p), ("qmax", _i64p), ("linmin", _i64p),
                ("kappa", _i64p), ("Mbasis", _i64p),
                ("n_p", ctypes.c_int64), ("ps", _i64p), ("pgeo", _i32p),
                ("device", ctypes.c_int), ("batch", ctypes.c_int64),
                ("verbose", ctypes.c_int)]


class _Output(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("M", _i64p), ("Kn", _i64p),
                ("q", _i64p), ("pidx", _i64p),
                ("pstat", ctypes.POINTER(ctypes.c_int8)),
                ("seconds_gpu", ctypes.c_double), ("err", ctypes.c_char * 256)]


class _Options(ctypes.Structure):
    _fields_ = [("form", ctypes.c_int), ("precision", ctypes.c_int),
                ("blocks_per_sm", ctypes.c_int), ("warps_per_block", ctypes.c_int),
                ("gcd_min_tree", ctypes.c_double), ("wait_s", ctypes.c_double),
                ("deadline_s", ctypes.c_double), ("check_fp32", ctypes.c_int),
                ("compact_rows", ctypes.c_int)]


class _PfvOutput(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("K", _i64p), ("M", _i64p), ("pidx", _i64p),
                ("n_points", ctypes.c_int64), ("pstat", ctypes.POINTER(ctypes.c_int8)),
                ("seconds_gpu", ctypes.c_double), ("err", ctypes.c_char * 256)]


class _Stats(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_int64), ("candidates", ctypes.c_int64),
                ("leaves", ctypes.c_int64), ("points", ctypes.c_int64),
                ("donated", ctypes.c_int64), ("fp64_retries", ctypes.c_int64),
                ("ms_setup", ctypes.c_double), ("ms_search", ctypes.c_double),
                ("ms_output", ctypes.c_double), ("launches", ctypes.c_int64),
                ("batch_retries", ctypes.c_int64), ("fp32_rem_err", ctypes.c_double),
                ("fp32_margin_frac", ctypes.c_double), ("fp32_end_err", ctypes.c_double),
                ("fp32_narrower", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_lib_error = None
LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fp_kernel")


def library_path():
    """The shared library this module loads (PFVS_GPU_LIB, else the in-tree build)."""
    path = os.environ.get("PFVS_GPU_LIB")
    if path:
        return path
    found = sorted(glob.glob(os.path.join(LIB_DIR, "libpfvs_gpu*.so")))
    return found[0] if found else None


def _load():
    global _lib, _lib_error
    if _lib is not None or _lib_error is not None:
        return _lib
    path = library_path()
    if not path:
        _lib_error = ("the B200 backend was not built (python -c 'import pfvs_b200.build as b; "
                      "b.build()', or __graft_entry__.build())")
        return None
    try:
        lib = ctypes.CDLL(path)
    except OSError as e:
        _lib_error = f"could not load {path}: {e}"
        return None
    lib.pfg_max_h11.restype = ctypes.c_int
    lib.pfg_backend.restype = ctypes.c_char_p
    lib.pfg_device_count.restype = ctypes.c_int
    lib.pfg_coni_batch.argtypes = [ctypes.POINTER(_Input), ctypes.POINTER(_Output)]
    lib.pfg_coni_batch.restype = ctypes.c_int
    lib.pfg_coni_batch_ex.argtypes = [ctypes.POINTER(_Input), ctypes.POINTER(_Options),
                                      ctypes.POINTER(_Output), ctypes.POINTER(_Stats), _i64p]
    lib.pfg_coni_batch_ex.restype = ctypes.c_int
    lib.pfg_zpm_batch.argtypes = lib.pfg_coni_batch_ex.argtypes
    lib.pfg_zpm_batch.restype = ctypes.c_int
    lib.pfg_output_free.argtypes = [ctypes.POINTER(_Output)]
    lib.pfg_coni_pfvs.argtypes = [ctypes.POINTER(_Input), ctypes.POINTER(_Options),
                                  ctypes.POINTER(_PfvOutput), ctypes.POINTER(_Stats)]
    lib.pfg_coni_pfvs.restype = ctypes.c_int
    lib.pfg_pfv_output_free.argtypes = [ctypes.POINTER(_PfvOutput)]
    lib.pfg_release.argtypes = [ctypes.c_int]
    lib.pfg_debug_fail_alloc.argtypes = [ctypes.c_int]
    lib.pfg_coni_mu0_batch.argtypes = [ctypes.c_int, _i64p, ctypes.c_int64, _i64p, ctypes.c_int, _i32p,
                                       _i64p, _i64p, _i64p, ctypes.c_char_p]
    lib.pfg_coni_mu0_batch.restype = ctypes.c_int
    zpk_args = [ctypes.c_int, _i64p, _i64p, ctypes.c_int64, _i64p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                ctypes.c_int64, ctypes.c_int]
    lib.pfg_coni_zpk_batch.argtypes = zpk_args + [ctypes.POINTER(_Output), _i32p]
    lib.pfg_coni_zpk_batch.restype = ctypes.c_int
    lib.pfg_coni_zpk_pfvs.argtypes = zpk_args + [ctypes.POINTER(_PfvOutput), _i32p]
    lib.pfg_coni_zpk_pfvs.restype = ctypes.c_int
    _lib = lib
    return lib


def _require():
    lib = _load()
    if lib is None:
        raise RuntimeError(_lib_error)
    return lib


def available() -> bool:
    """Whether the backend is built and a CUDA device is present
    (pfvs/gpu.py:85-95)."""
    lib = _load()
    return lib is not None and lib.pfg_device_count() > 0


def unavailable_reason() -> str:
    """Why `available()` is False ('' if it is True)."""
    lib = _load()
    if lib is None:
        return _lib_error
    if lib.pfg_device_count() == 0:
        return "no CUDA device found"
    return ""


def backend() -> str:
    """'cuda'."""
    return _require().pfg_backend().decode()


def release(device: int = 0) -> None:
    """Free the device buffers kept between calls on `device`."""
    lib = _load()
    if lib is not None:
        lib.pfg_release(int(device))


def debug_fail_alloc(k: int) -> None:
    """Test hook: the k-th device allocation of the library from now on fails
    once (out of memory), without allocating; k <= 0 cancels."""
    _require().pfg_debug_fail_alloc(int(k))


def max_h11() -> int:
    """The largest h11 the build supports (64)."""
    return _require().pfg_max_h11()


def _qmax(Q, dilation):
    return int(math.floor(dilation * Q + 1e-7))


def _geometry_arrays(geoms, MH):
    """pfg_input's per-geometry arrays: h11, Q, qmax = floor(dilation Q),
    linmin = ceil(M0min), and the kappa and Mbasis blocks end to end."""
    n_geo = len(geoms)
    h = np.zeros(n_geo, dtype=np.int32)
    Q, qmax, linmin = (np.zeros(n_geo, dtype=np.int64) for _ in range(3))
    blocks_k, blocks_m = [], []
    for k, g in enumerate(geoms):
        kap_k = np.ascontiguousarray(g["kappa"], dtype=np.int64)
        h[k] = kap_k.shape[0]
        if not 3 <= h[k] <= MH:
            raise ValueError(f"the GPU build supports 3 <= h11 <= {MH}")
        Q[k] = int(g["Q"])
        qmax[k] = _qmax(int(Q[k]), g["dilation"])
        linmin[k] = math.ceil(g.get("M0min", 0) - 1e-9)
        blocks_k.append(kap_k.reshape(-1))
        blocks_m.append(np.ascontiguousarray(g["Mbasis"], dtype=np.int64).reshape(-1))
    kap = np.concatenate(blocks_k) if blocks_k else np.zeros(1, dtype=np.int64)
    Mb = np.concatenate(blocks_m) if blocks_m else np.zeros(1, dtype=np.int64)
    return h, Q, qmax, linmin, kap, Mb


def _pack(geoms, ps, pgeo, MH):
    n_geo = len(geoms)
    h, Q, qmax, linmin, kap, Mb = _geometry_arrays(geoms, MH)
    pgeo = np.ascontiguousarray(pgeo, dtype=np.int32)
    n_p = len(pgeo)
    if n_p and (np.any(pgeo < 0) or np.any(pgeo >= n_geo)):
        raise ValueError("pgeo: geometry index out of range")
    if isinstance(ps, np.ndarray) and ps.ndim == 2:
        W = ps.shape[1]
        if W > MH:
            raise ValueError("a p-vector is longer than its geometry's h11")
        if ps.shape[0] != n_p:
            raise ValueError("ps and pgeo differ in length")
        if n_p:
            hp = h[pgeo]
            if W > hp.min():                                  # entries beyond h11 must be 0
                if np.any((ps != 0) & (np.arange(W)[None, :] >= hp[:, None])):
                    raise ValueError("a p-vector is longer than its geometry's h11")
        if n_p and W == MH and ps.dtype == np.int64 and ps.flags.c_contiguous:
            P = ps                                            # already the library's layout
        else:
            P = np.zeros((max(n_p, 1), MH), dtype=np.int64)
            P[:n_p, :W] = ps
    else:
        P = np.zeros((max(n_p, 1), MH), dtype=np.int64)
        if n_p:
            # one flat copy and one scatter (a list of 1-d arrays)
            lens = np.fromiter((len(p) for p in ps), dtype=np.int64, count=n_p)
            if lens.max() > MH:
                raise ValueError("a p-vector is longer than its geometry's h11")
            flat = np.concatenate([np.asarray(p, dtype=np.int64).ravel() for p in ps])
            rows = np.repeat(np.arange(n_p), lens)
            cols = np.arange(len(flat)) - np.repeat(np.cumsum(lens) - lens, lens)
            P[rows, cols] = flat
            long_rows = np.flatnonzero(lens > h[pgeo])
            if len(long_rows):
                hh = h[pgeo[long_rows]]
                if np.any(P[long_rows][np.arange(MH)[None, :] >= hh[:, None]] != 0):
                    raise ValueError("a p-vector is longer than its geometry's h11")
    return h, Q, qmax, linmin, kap, Mb, P, pgeo, n_p


class _OutputOwner:
    """Owns one pfg_output; frees it (pfg_output_free) when collected."""

    def __init__(self, lib, out):
        self.lib, self.out = lib, out

    def __del__(self):
        try:
            self.lib.pfg_output_free(ctypes.byref(self.out))
        except Exception:
            pass


def _view(owner, ptr, shape):
    """int64 array of `shape` over the library buffer at `ptr`, keeping `owner` alive."""
    n = int(np.prod(shape))
    if n == 0:
        return np.zeros(shape, dtype=np.int64)
    buf = (ctypes.c_int64 * n).from_address(ctypes.cast(ptr, ctypes.c_void_p).value)
    buf._owner = owner
    return np.ctypeslib.as_array(buf).reshape(shape)


def coni_batch_multi_ex(geoms, ps, pgeo, device=0, batch=0, verbose=False,
                        form=FORM_BATCHED, precision=PREC_AUTO, blocks_per_sm=0,
                        warps_per_block=0, want_dir_nodes=False, gcd_min_tree=0.0,
                        wait_s=0.0, deadline_s=0.0, check_fp32=False, compact_rows=False):
    """
    `coni_batch_multi` with the search form (FORM_BATCHED: one persistent
    work-stealing launch; FORM_PLAIN: one warp per direction in one launch, FP64 pruning, no work sharing), the pruning
    precision (PREC_AUTO: the library's choice, FP64 on B200; PREC_FP64;
    PREC_FP32: FP32 where qmax < 2^22 with an FP64 retry on -11), the
    bounds on the search's waits (wait_s: a warp's wait for work, counted
    from the launch, past which the call fails; deadline_s: one subtree's
    search, past which its direction gets status -22; 0: 30 s and 120 s),
    check_fp32 (with PREC_FP32: the FP32 pass with an FP64 shadow of its
    pruning bounds; their errors in stats["fp32_*"]), compact_rows (M and
    Kn rows as wide as the largest h11 of `geoms` instead of max_h11(): fewer
    bytes copied back) and the call's statistics.  Returns
    (M, Kn, q, pidx, pstat, seconds_gpu, stats dict[, dir_nodes]).
    """
    return _batch_ex("pfg_coni_batch_ex", geoms, ps, pgeo, device, batch, verbose, form, precision,
                     blocks_per_sm, warps_per_block, want_dir_nodes, gcd_min_tree, wait_s, deadline_s,
                     check_fp32, compact_rows)


def zpm_batch_multi_ex(geoms, ps, pgeo, device=0, batch=0, verbose=False,
                       form=FORM_BATCHED, precision=PREC_AUTO, blocks_per_sm=0,
                       warps_per_block=0, want_dir_nodes=False, gcd_min_tree=0.0,
                       wait_s=0.0, deadline_s=0.0, check_fp32=False, compact_rows=False):
    """
    Non-coni ZpM's lattice points on the device (pfg_zpm_batch): as
    `coni_batch_multi_ex`, with each geometry's `Q` the search's Qmax
    (qmax = floor(dilation Qmax); `M0min` is ignored: no M0 cut) and the
    p-vectors with all h11 entries (any p in the Kahler cone).  The points c
    satisfy c^T mat c <= qmax and the non-strict GCD cut (g == 0 or
    Qmax g >= q, g = gcd(K)), as the reference's pfv_kernel
    (pfvs/fp_kernel/fp_kernel.pyx:321-352) returns them for nonconi.ZpM.
    """
    return _batch_ex("pfg_zpm_batch", geoms, ps, pgeo, device, batch, verbose, form, precision,
                     blocks_per_sm, warps_per_block, want_dir_nodes, gcd_min_tree, wait_s, deadline_s,
                     check_fp32, compact_rows)


def _batch_ex(entry, geoms, ps, pgeo, device, batch, verbose, form, precision, blocks_per_sm,
              warps_per_block, want_dir_nodes, gcd_min_tree, wait_s, deadline_s, check_fp32, compact_rows):
    lib = _require()
    MH = lib.pfg_max_h11()
    h, Q, qmax, linmin, kap, Mb, P, pgeo, n_p = _pack(geoms, ps, pgeo, MH)
    inp = _Input(len(geoms), h.ctypes.data_as(_i32p), Q.ctypes.data_as(_i64p),
                 qmax.ctypes.data_as(_i64p), linmin.ctypes.data_as(_i64p),
                 kap.ctypes.data_as(_i64p), Mb.ctypes.data_as(_i64p),
                 n_p, P.ctypes.data_as(_i64p), pgeo.ctypes.data_as(_i32p),
                 int(device), int(batch), int(bool(verbose)))
    opt = _Options(int(form), int(precision), int(blocks_per_sm), int(warps_per_block), float(gcd_min_tree),
                   float(wait_s), float(deadline_s), int(bool(check_fp32)), int(bool(compact_rows)))
    st = _Stats()
    dn = np.zeros(max(n_p, 1), dtype=np.int64)
    out = _Output()
    rc = getattr(lib, entry)(ctypes.byref(inp), ctypes.byref(opt), ctypes.byref(out),
                             ctypes.byref(st), dn.ctypes.data_as(_i64p))
    if rc != 0:
        raise RuntimeError(f"GPU pipeline failed: {out.err.decode(errors='replace')}")
    width = max(3, int(h.max())) if (compact_rows and len(h)) else MH
    res = _points(lib, out, n_p, width) + (st.as_dict(),)
    return res + (dn[:n_p],) if want_dir_nodes else res


def _points(lib, out, n_p, width):
    """(M, Kn, q, pidx, pstat, seconds_gpu) of a filled pfg_output (rows of
    `width` entries).  The row arrays view the library's (pinned) output
    blocks without a copy; the blocks go back to the library when the last
    view is collected."""
    owner = _OutputOwner(lib, out)
    n = out.n
    M, Kn = _view(owner, out.M, (n, width)), _view(owner, out.Kn, (n, width))
    q, pidx = _view(owner, out.q, (n,)), _view(owner, out.pidx, (n,))
    pstat = np.ctypeslib.as_array(out.pstat, shape=(n_p,)).astype(np.int8) if n_p \
        else np.zeros(0, dtype=np.int8)
    return M, Kn, q, pidx, pstat, out.seconds_gpu


class _PfvOwner:
    """Owns one pfg_pfv_output; frees it (pfg_pfv_output_free) when collected."""

    def __init__(self, lib, out):
        self.lib, self.out = lib, out

    def __del__(self):
        try:
            self.lib.pfg_pfv_output_free(ctypes.byref(self.out))
        except Exception:
            pass


def coni_pfvs_multi(geoms, ps, pgeo, device=0, batch=0, verbose=False, form=FORM_BATCHED,
                    precision=PREC_AUTO, gcd_min_tree=0.0):
    """
    The batched pipeline and coniZpM's post-processing (pfvs/coni.py:275-412,
    `_pfvs_from_points`), both on the device: the coni PFVs of every
    p-vector.  Arguments as `coni_batch_multi` (M0min > 0).  Returns
    (Ks, Ms, pidx, pstat, seconds_gpu, stats dict): Ks, Ms of shape
    (n, max_h11()) (first h11 entries valid), grouped by p-vector (ascending)
    in the reference's order within one.
    """
    lib = _require()
    MH = lib.pfg_max_h11()
    h, Q, qmax, linmin, kap, Mb, P, pgeo, n_p = _pack(geoms, ps, pgeo, MH)
    inp = _Input(len(geoms), h.ctypes.data_as(_i32p), Q.ctypes.data_as(_i64p),
                 qmax.ctypes.data_as(_i64p), linmin.ctypes.data_as(_i64p),
                 kap.ctypes.data_as(_i64p), Mb.ctypes.data_as(_i64p),
                 n_p, P.ctypes.data_as(_i64p), pgeo.ctypes.data_as(_i32p),
                 int(device), int(batch), int(bool(verbose)))
    opt = _Options(int(form), int(precision), 0, 0, float(gcd_min_tree), 0.0, 0.0, 0, 0)
    st = _Stats()
    out = _PfvOutput()
    rc = lib.pfg_coni_pfvs(ctypes.byref(inp), ctypes.byref(opt), ctypes.byref(out), ctypes.byref(st))
    if rc != 0:
        raise RuntimeError(f"GPU pipeline failed: {out.err.decode(errors='replace')}")
    owner = _PfvOwner(lib, out)
    n = out.n
    K, M = _view(owner, out.K, (n, MH)), _view(owner, out.M, (n, MH))
    pidx = _view(owner, out.pidx, (n,))
    pstat = np.ctypeslib.as_array(out.pstat, shape=(n_p,)).copy() if n_p \
        else np.zeros(0, dtype=np.int8)
    stats = st.as_dict()
    stats["points"] = out.n_points
    secs = out.seconds_gpu
    del owner
    return K, M, pidx, pstat.astype(np.int8), secs, stats


def coni_batch_multi(geoms, ps, pgeo, device=0, batch=0, verbose=False):
    """
    The batched coni pipeline on the GPU for p-vectors of several geometries
    at once (pfvs/gpu.py:136-211), through the exported pfg_coni_batch (the
    entry point the reference's loader binds).

    - `geoms`: per geometry a dict with `kappa` (h, h, h), `Mbasis` (h, h),
      `Q`, `dilation`, `M0min`.
    - `ps`: the p-vectors, each of length h of its geometry, *with* the
      leading 0.
    - `pgeo`: the geometry index of each p-vector.

    Returns (M, Kn, q, pidx, pstat, seconds_gpu): for every lattice point
    M = Binter c and Kn = Z Binter c (rows of width max_h11(), first h
    entries valid), q = c^T mat c, its p-vector index; points grouped by
    p-vector (ascending), sorted by (M, Kn) within one.
    """
    lib = _require()
    MH = lib.pfg_max_h11()
    h, Q, qmax, linmin, kap, Mb, P, pgeo, n_p = _pack(geoms, ps, pgeo, MH)
    inp = _Input(len(geoms), h.ctypes.data_as(_i32p), Q.ctypes.data_as(_i64p),
                 qmax.ctypes.data_as(_i64p), linmin.ctypes.data_as(_i64p),
                 kap.ctypes.data_as(_i64p), Mb.ctypes.data_as(_i64p),
                 n_p, P.ctypes.data_as(_i64p), pgeo.ctypes.data_as(_i32p),
                 int(device), int(batch), int(bool(verbose)))
    out = _Output()
    if lib.pfg_coni_batch(ctypes.byref(inp), ctypes.byref(out)) != 0:
        raise RuntimeError(f"GPU pipeline failed: {out.err.decode(errors='replace')}")
    return _points(lib, out, n_p, MH)


def coni_batch(kappa, Mbasis, ps, Q, dilation, M0min, max_N_out, device=0):
    """
    One geometry (pfvs/gpu.py:214-232): (M, Kn, q, pidx, pstat), rows cut to
    h columns.  A p-vector with more than max_N_out points gets pstat -2
    ("more than max_N_pfvs outputs", as the reference kernel's status) and
    none of its points are returned.
    """
    ps = np.asarray(ps, dtype=np.int64)
    n_p = len(ps)
    geom = {"kappa": kappa, "Mbasis": Mbasis, "Q": Q, "dilation": dilation, "M0min": M0min}
    M, Kn, q, pidx, pstat, _ = coni_batch_multi([geom], ps, np.zeros(n_p, dtype=np.int32), device=device)
    hh = np.asarray(kappa).shape[0]
    rows_of = np.zeros(n_p, dtype=np.int64)
    np.add.at(rows_of, pidx, 1)
    too_many = np.flatnonzero(rows_of > max_N_out)
    if too_many.size:
        pstat[too_many] = -2
        kept = ~np.isin(pidx, too_many)
        M, Kn, q, pidx = M[kept], Kn[kept], q[kept], pidx[kept]
    return M[:, :hh], Kn[:, :hh], q, pidx, pstat


def _zpk_arrays(kappa, Mbasis, ps):
    kappa = np.ascontiguousarray(kappa, dtype=np.int64)
    Mbasis = np.ascontiguousarray(Mbasis, dtype=np.int64)
    h = Mbasis.shape[0]
    if kappa.shape != (h, h, h):
        raise ValueError(f"kappa must be ({h}, {h}, {h}), got {kappa.shape}")
    ps = np.ascontiguousarray(np.atleast_2d(ps), dtype=np.int64)
    if ps.shape[1] != h:
        raise ValueError(f"ps must have h11 = {h} columns (p[0] = 0), got {ps.shape[1]}")
    return kappa, Mbasis, ps, h


def coni_zpk_points(kappa, Mbasis, ps, Q, M0min, D0, max_out=10**9, device=0):
    """
    coniZpK above D0 on the device (pfg_coni_zpk_batch; the reference's
    _coni_zpk_batch, pfvs/fp_kernel/fp_kernel.pyx:434): for each row p of ps
    ((n, h11), p[0] = 0) the lattice points of its coni PFVs with dilation
    > D0.  Returns (M (N, h11), Kn (N, h11), q (N,), pidx (N,), status (n,)
    int32, seconds_gpu); points only of the rows with status 0.
    """
    lib = _require()
    MH = lib.pfg_max_h11()
    kappa, Mbasis, ps, h = _zpk_arrays(kappa, Mbasis, ps)
    n = len(ps)
    st = np.zeros(max(n, 1), np.int32)
    out = _Output()
    rc = lib.pfg_coni_zpk_batch(h, kappa.ctypes.data_as(_i64p), Mbasis.ctypes.data_as(_i64p), n,
                                ps.ctypes.data_as(_i64p), int(Q), int(M0min), int(D0), int(max_out), int(device),
                                ctypes.byref(out), st.ctypes.data_as(_i32p))
    if rc != 0:
        raise RuntimeError(f"coniZpK failed: {out.err.decode(errors='replace')}")
    M, Kn, q, pidx, _, secs = _points(lib, out, 0, MH)
    return M[:, :h].copy(), Kn[:, :h].copy(), q.copy(), pidx.copy(), st[:n], secs


def coni_zpk_pfvs(kappa, Mbasis, ps, Q, M0min, D0, max_out=10**9, device=0):
    """
    coniZpK above D0 and coniZpM's post-processing, both on the device
    (pfg_coni_zpk_pfvs): (Ks (N, h11), Ms, pidx, status (n,) int32,
    n_points, seconds_gpu) -- the PFVs of the points, not yet filtered by
    dilation > D0.
    """
    lib = _require()
    MH = lib.pfg_max_h11()
    kappa, Mbasis, ps, h = _zpk_arrays(kappa, Mbasis, ps)
    n = len(ps)
    st = np.zeros(max(n, 1), np.int32)
    out = _PfvOutput()
    rc = lib.pfg_coni_zpk_pfvs(h, kappa.ctypes.data_as(_i64p), Mbasis.ctypes.data_as(_i64p), n,
                               ps.ctypes.data_as(_i64p), int(Q), int(M0min), int(D0), int(max_out), int(device),
                               ctypes.byref(out), st.ctypes.data_as(_i32p))
    if rc != 0:
        raise RuntimeError(f"coniZpK failed: {out.err.decode(errors='replace')}")
    owner = _PfvOwner(lib, out)
    N = out.n
    K, M = _view(owner, out.K, (N, MH)), _view(owner, out.M, (N, MH))
    pidx = _view(owner, out.pidx, (N,))
    res = (K[:, :h].copy(), M[:, :h].copy(), pidx.copy(), st[:n], int(out.n_points), out.seconds_gpu)
    del owner
    return res

