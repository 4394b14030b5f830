"""
The coni dilation bound on the device: the reference's pfvs/dilation.py
(coni_mu0 :145, coni_dilation_bound :187, coni_dilation_bound_ceils :214,
coni_dilation_bounds :243), computed by the library's k_mu0 kernel (one warp
per direction, exact integers; pfvs_b200/csrc/pfg_mu0.cuh) through the C
entry point pfg_coni_mu0_batch.

For a direction p_hat = (0, p_r) of a geometry with triple intersection
numbers kappa (coni basis) and tadpole Q,

    A = kappa . p_hat,   S = -A_rr^-1,   Lambda = {K in Z^(h11-1) : p_r . K = 0}
    mu0 = min over nonzero K in Lambda of K^T S K

and every coni PFV of the direction has dilation delta < Q / mu0 when the
hypotheses hold (s = a00 - a_r0^T A_rr^-1 a_r0 <= 0, S positive definite on
Lambda); otherwise the direction has no bound.

Statuses per direction, as the reference's C path reports them
(_coni_mu0_batch, pfvs/fp_kernel/coni_bound.h:255): 0 decided, 1 no bound,
< 0 not decided on the device (an exact value beyond the device's 128-bit
range, an ill-conditioned form, the enumeration's node budget).  The
reference decides those with python-flint on the host; this library does not
fall back to the host: `coni_mu0` and `coni_dilation_bound` raise
UndecidedBound, and the batch functions report the direction as undecided
(no bound value, status < 0), so that coni_zp searches it at the fallback
dilation and marks it incomplete.
"""
import ctypes
from fractions import Fraction

import numpy as np

from . import gpu

MAX_H11 = 32                  # the device bound's largest h11


class UndecidedBound(RuntimeError):
    """The device could not decide mu0 for a direction (status < 0)."""

    def __init__(self, status):
        super().__init__(f"the coni dilation bound is not decided on the device (status {status}: "
                         f"an exact value beyond 128 bits, an ill-conditioned form, or the node budget)")
        self.status = int(status)


def coni_mu0_batch(ps, kappa, device=0):
    """
    mu0 for each row of ps ((n, h11-1), the directions without their coni
    entry) on the device: (status int32 (n,), mu_num int64 (n,), mu_den int64
    (n,), K int64 (n, h11-1)); for status 0, mu0 = mu_num / mu_den in lowest
    terms and K a nonzero minimizer in Lambda.  The reference's
    _coni_mu0_batch(kappa, ps) (pfvs/dilation.py:134-142).
    """
    lib = gpu._require()
    kappa = np.ascontiguousarray(kappa, dtype=np.int64)
    h = kappa.shape[0]
    if kappa.shape != (h, h, h) or not 3 <= h <= MAX_H11:
        raise ValueError(f"kappa must be (h11, h11, h11) with 3 <= h11 <= {MAX_H11}, got {kappa.shape}")
    ps = np.ascontiguousarray(np.atleast_2d(np.asarray(ps, dtype=np.int64)))
    if ps.shape[1] != h - 1:
        raise ValueError(f"ps must have h11 - 1 = {h - 1} columns, got {ps.shape[1]}")
    n = len(ps)
    st = np.zeros(max(n, 1), dtype=np.int32)
    num, den = np.zeros(max(n, 1), dtype=np.int64), np.zeros(max(n, 1), dtype=np.int64)
    K = np.zeros((max(n, 1), h - 1), dtype=np.int64)
    buf = ctypes.create_string_buffer(256)
    rc = lib.pfg_coni_mu0_batch(h, kappa.ctypes.data_as(gpu._i64p), n, ps.ctypes.data_as(gpu._i64p), int(device),
                                st.ctypes.data_as(gpu._i32p), num.ctypes.data_as(gpu._i64p),
                                den.ctypes.data_as(gpu._i64p), K.ctypes.data_as(gpu._i64p), buf)
    if rc != 0:
        raise RuntimeError(f"GPU dilation bound failed: {buf.value.decode(errors='replace')}")
    return st[:n], num[:n], den[:n], K[:n]


def coni_mu0(p, kappa, device=0):
    """(mu0 as a Fraction, K as a list) for one direction p ((h11-1,)), or
    None when the direction has no bound (pfvs/dilation.py:145); raises
    UndecidedBound where the device cannot decide it."""
    st, num, den, K = coni_mu0_batch(np.asarray(p)[None], kappa, device)
    if st[0] == 1:
        return None
    if st[0] != 0:
        raise UndecidedBound(st[0])
    return Fraction(int(num[0]), int(den[0])), [int(x) for x in K[0]]


def coni_dilation_bound(p, kappa, Q, device=0):
    """Q / mu0 (exact; the bound is strict), or None without a bound
    (pfvs/dilation.py:187)."""
    r = coni_mu0(p, kappa, device)
    return None if r is None else Fraction(int(Q)) / r[0]


BOUND_RANGE = -36            # status: the bound's ceiling exceeds int64 (no searchable bound)


def _ceil_q_over(Q, num, den):
    """(ceil(Q den / num) per entry (num > 0), whether it fits int64): in
    int64 where Q den fits, else exactly; 0 where the ceiling does not fit."""
    out = np.zeros(len(num), dtype=np.int64)
    fits = np.ones(len(num), dtype=bool)
    small = den < 2 ** 62 // max(int(Q), 1)
    out[small] = -((-int(Q) * den[small]) // num[small])
    for i in np.flatnonzero(~small):
        c = -((-int(Q) * int(den[i])) // int(num[i]))
        if c < 2 ** 63:
            out[i] = c
        else:
            fits[i] = False
    return out, fits


def coni_dilation_bound_ceils(ps, kappa, Q, n_jobs=1, device=0, return_status=False):
    """
    ceil(coni_dilation_bound) for each row of ps as int64, 0 where there is
    no bound or the device did not decide it (pfvs/dilation.py:214); with
    return_status, also the per-direction status (0, 1, < 0; BOUND_RANGE
    where the ceiling exceeds int64).  n_jobs is
    accepted for the reference's signature (the device takes every row at
    once).
    """
    del n_jobs
    st, num, den, _ = coni_mu0_batch(ps, kappa, device)
    out = np.zeros(len(st), dtype=np.int64)
    ok = np.flatnonzero(st == 0)
    out[ok], fits = _ceil_q_over(Q, num[ok], den[ok])
    st = st.copy()
    st[ok[~fits]] = BOUND_RANGE
    return (out, st) if return_status else out


def coni_dilation_bounds(ps, kappa, Q, n_jobs=1, device=0):
    """coni_dilation_bound for each row of ps (pfvs/dilation.py:243): a
    Fraction, None without a bound; raises UndecidedBound for a direction
    the device did not decide."""
    del n_jobs
    st, num, den, _ = coni_mu0_batch(ps, kappa, device)
    out = []
    for s, a, b in zip(st, num, den):
        if s == 1:
            out.append(None)
        elif s == 0:
            out.append(Fraction(int(Q)) / Fraction(int(a), int(b)))
        else:
            raise UndecidedBound(s)
    return out


def grid_up(D):
    """
    D rounded up onto the grid ceil(2^(k/16)), k integer, so that nearby
    bounds share one search; D itself where the grid point falls below it
    (the reference's _grid_up, pfvs/coni.py:647-653: the same formula, so
    that a routed direction is searched at the same dilation).
    """
    D = np.maximum(np.asarray(D, dtype=np.int64), 1)
    k = np.ceil(16 * np.log2(D)).astype(np.int64)
    g = np.ceil(2.0 ** (k / 16)).astype(np.int64)
    return np.where(g >= D, g, D)
