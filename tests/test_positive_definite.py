"""
The positive-definiteness decision (the reference's status -9).

A direction whose kappa.p lacks the signature (1, h11-1) has an indefinite
ellipsoid matrix.  The reference decides that exactly (the Bareiss pivots of
fpk_common.h:259-309 are the leading minors; a non-positive one is -9, which
coniZpM raises as IncompleteSearchError, coni.py:446-453) after its C setup
hands such a direction to its Python path (status 1 from the C batch).  The
oracle decides it by Sylvester's criterion in Python integers; the device
by an integer witness x with x^T mat x <= 0 evaluated exactly
(pfg_setup.cuh, witness_not_pd).  These tests run the device code on the
CPU warp emulator (tests/emu), so they need no GPU.
"""
import math

import numpy as np
import pytest

from oracle import lattice, pfo, ref
from pfvs_b200 import workloads
from parity import layout


def _non_lorentzian(g, n, emax, seed):
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        p = np.concatenate([[0], rng.integers(1, emax + 1, g.h11 - 1)]).astype(np.int64)
        if math.gcd(*[int(x) for x in p]) == 1 and not workloads.lorentzian_ok(g.kappa, p):
            out.append(p)
    return out


@pytest.mark.parametrize("name", ["small", "plain", "mixed"])
def test_indefinite_directions_give_status_minus_9(name):
    from emu import emu
    w = workloads.build(name, n_p=8)
    g = w.geoms[0]
    bad = _non_lorentzian(g, 4, 6, seed=5)
    good = [np.asarray(p) for p, k in zip(w.ps, w.pgeo) if k == 0][:2]
    ps = bad + good
    geoms = [dict(kappa=g.kappa, Mbasis=g.Mbasis, Q=g.Q, dilation=1.0, M0min=13)]
    pgeo = np.zeros(len(ps), dtype=np.int32)
    # the oracle: -9 exactly for the indefinite ones, 0 for the others
    for p, want in zip(ps, [-9] * len(bad) + [0] * len(good)):
        assert pfo.direction(g.kappa, g.Mbasis, p, g.Q, g.Q, 13)[3] == want
    # the reference's C batch hands the indefinite ones to its exact Python path
    if ref.available():
        st = ref.coni_batch(g.kappa, g.Mbasis, np.array(bad), g.Q, 1.0, 13)[4]
        assert np.all(st == 1)
    # the device code: -9 for those, and the good directions unaffected
    M, Kn, q, pidx, pstat, nodes, stage = emu.coni_batch_multi(geoms, ps, pgeo, precision=1)
    np.testing.assert_array_equal(pstat, [-9] * len(bad) + [0] * len(good))
    assert np.all(pidx >= len(bad))


def _rand_sym(rng, d, lo=-9, hi=10):
    A = rng.integers(lo, hi, (d, d))
    return A + A.T


@pytest.mark.parametrize("d", [2, 5, 12, 31, 47, 63])
def test_witness_on_crafted_matrices(d):
    from emu import emu
    rng = np.random.default_rng(d)
    B = rng.integers(-20, 21, (d, d))
    pd = B.T @ B + d * np.eye(d, dtype=np.int64)             # positive definite
    assert lattice.is_positive_definite(pd)
    assert not emu.witness_not_pd(pd)                          # (never a false proof)
    # indefinite: one direction of negative curvature added
    v = rng.integers(-3, 4, d)
    v[0] = 1
    ind = pd - (int(v @ pd @ v) + 5) * np.outer(pd @ v, pd @ v) // max(1, int(v @ pd @ pd @ v))
    ind = (ind + ind.T) // 2
    if not lattice.is_positive_definite(ind):
        assert emu.witness_not_pd(ind)
    # random symmetric matrices are indefinite for d >= 2 almost surely
    A = _rand_sym(rng, d)
    assert lattice.is_positive_definite(A) == (not emu.witness_not_pd(A))
    # a negative diagonal entry deep inside
    N = pd.copy()
    N[d // 2, d // 2] = -1
    assert emu.witness_not_pd(N)


def test_witness_finds_a_negative_pivot_lost_among_large_entries():
    """Indefinite only in the last leading minor, with entries near 2^40
    (the witness's scale adapts to the entries' size)."""
    from emu import emu
    rng = np.random.default_rng(3)
    d = 20
    B = rng.integers(-2**18, 2**18, (d, d))
    A = B.T @ B
    # make the trailing Schur complement -1 exactly: A' = A with A_dd lowered
    Ainv_col = np.linalg.solve(A[:-1, :-1].astype(float), A[:-1, -1].astype(float))
    schur = A[-1, -1] - A[:-1, -1].astype(float) @ Ainv_col
    A[-1, -1] -= int(round(schur)) + 1
    if lattice.is_positive_definite(A):
        pytest.skip("rounding left it positive definite")
    assert emu.witness_not_pd(A)


def test_ill_conditioned_positive_definite_is_not_called_indefinite():
    """A positive definite matrix whose FP64 factor cannot be certified is
    never called indefinite (the device reports -21, 'not certified', for it:
    no witness exists)."""
    from emu import emu
    d = 12
    A = np.zeros((d, d), dtype=np.int64)
    for i in range(d):                      # a path of nearly dependent rows
        A[i, i] = 2 * 10**6 + (1 if i == 0 else 0)
        if i:
            A[i, i - 1] = A[i - 1, i] = -10**6
    assert lattice.is_positive_definite(A)
    assert not emu.witness_not_pd(A)


def test_is_positive_definite_matches_eigenvalues():
    rng = np.random.default_rng(11)
    for _ in range(200):
        d = int(rng.integers(1, 7))
        A = _rand_sym(rng, d, -4, 5) + int(rng.integers(0, 12)) * np.eye(d, dtype=np.int64)
        ev = np.linalg.eigvalsh(A.astype(float))
        if np.min(np.abs(ev)) < 1e-9:
            continue
        assert lattice.is_positive_definite(A) == bool(np.all(ev > 0))
