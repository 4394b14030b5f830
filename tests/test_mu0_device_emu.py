"""
The device's coni dilation bound (pfvs_b200/csrc/pfg_mu0.cuh, k_mu0) run on
the CPU warp emulator (tests/emu), against the reference:

- every PFV direction of the reference's fixtures (tests/golden/mu0.npz):
  status 0, mu0 equal to the reference's C code's (coni_bound.h:255), the
  PFV's dilation below Q / mu0 (tests/test_dilation_bound.py:110-117 of the
  reference), the minimizer K in Lambda and attaining mu0;
- the fixtures' seeded non-PFV directions: the C code's status and value
  wherever it decides (0 or 1), and the exact oracle's where it does not;
- mu0 invariant under signed permutations of the non-coni directions
  (tests/test_dilation_bound.py:164-181 of the reference);
- the hypothesis failures (a singular A_rr, a negative definite form) are
  "no bound" (tests/test_dilation_bound.py:184-197 of the reference);
- beyond the C code: at h11 = 16 the 256-bit elimination decides directions
  whose Bareiss products overflow int128, equal to the exact oracle.
The host logic of pfvs_b200.coni (routing, ceilings, canonical order) is
checked with the oracle standing in for the device.
"""
import os
from fractions import Fraction

import numpy as np
import pytest

from conftest import ROOT
from emu import emu
from oracle import mu0 as omu0
from pfvs_b200 import coni, dilation, workloads

G = np.load(os.path.join(ROOT, "tests", "golden", "mu0.npz"))


def _frac(num, den):
    return Fraction(int(num), int(den))


def _form_value(kappa, p_r, K):
    h = kappa.shape[0]
    p_hat = [0] + [int(x) for x in p_r]
    A = [[sum(int(kappa[a, b, c]) * p_hat[c] for c in range(h)) for b in range(h)] for a in range(h)]
    x = omu0._solve_exact([row[1:] for row in A[1:]], [[int(k) for k in K]])[0]
    return -sum(Fraction(int(k)) * v for k, v in zip(K, x))


def test_device_mu0_on_every_fixture_pfv():
    n = len(G["status"])
    assert n > 300
    by_geo = {}
    for i in range(n):
        by_geo.setdefault(int(G["gidx"][i]), []).append(i)
    for k, rows in by_geo.items():
        kappa = G[f"kappa{k}"]
        h = kappa.shape[0]
        p_r = np.array([G["p"][i][1:h] for i in rows])
        st, num, den, K = emu.coni_mu0_batch(kappa, p_r)
        for j, i in enumerate(rows):
            assert st[j] == 0 == int(G["status"][i]), (k, i)
            m = _frac(num[j], den[j])
            assert m == _frac(*G["mu0"][i])
            assert _frac(*G["delta"][i]) < Fraction(int(G["Q"][i])) / m
            assert K[j].any() and int(np.dot(K[j], p_r[j])) == 0
            if j % 5 == 0:
                assert _form_value(kappa, p_r[j], K[j]) == m


def test_device_mu0_on_other_directions():
    n = len(G["r_status"])
    seen = {0: 0, 1: 0, "oracle": 0}
    for i in range(n):
        kappa = G[f"kappa{int(G['r_gidx'][i])}"]
        h = kappa.shape[0]
        p_r = G["r_p"][i][:h - 1]
        st, num, den, K = emu.coni_mu0_batch(kappa, p_r[None])
        rs = int(G["r_status"][i])
        if rs >= 0:
            assert st[0] == rs, i
            if rs == 0:
                assert _frac(num[0], den[0]) == _frac(*G["r_mu0"][i])
            seen[rs] += 1
        else:                                                   # the C code did not decide: the oracle
            so, mo, _ = omu0.coni_mu0(kappa, p_r)
            assert st[0] == so and (so == 1 or _frac(num[0], den[0]) == mo), i
            seen["oracle"] += 1
    assert seen[0] > 50 and seen[1] > 100 and seen["oracle"] > 20


def test_device_mu0_unimodular_invariance():
    rng = np.random.default_rng(0)
    for i in range(0, len(G["status"]), 25):
        kappa = G[f"kappa{int(G['gidx'][i])}"]
        h = kappa.shape[0]
        p_hat = G["p"][i][:h]
        perm = rng.permutation(h - 1)
        signs = rng.choice([-1, 1], size=h - 1)
        U = np.eye(h, dtype=np.int64)
        U[1:, 1:] = 0
        U[1 + np.arange(h - 1), 1 + perm] = signs
        Uinv = np.round(np.linalg.inv(U)).astype(np.int64)
        kappa2 = np.einsum("ia,jb,kc,ijk->abc", Uinv, Uinv, Uinv, kappa)
        p2 = U @ p_hat
        a = emu.coni_mu0_batch(kappa, p_hat[1:][None])
        b = emu.coni_mu0_batch(kappa2, p2[1:][None])
        assert a[0][0] == b[0][0] == 0
        assert _frac(a[1][0], a[2][0]) == _frac(b[1][0], b[2][0])


def test_device_mu0_hypothesis_failures():
    h = 4
    st, *_ = emu.coni_mu0_batch(np.zeros((h, h, h), dtype=np.int64), np.array([[1, 2, 3]]))
    assert st[0] == 1                                           # A_rr singular
    kappa = np.zeros((h, h, h), dtype=np.int64)
    for i in (1, 2, 3):
        for a, b, c in {(i, i, 1), (i, 1, i), (1, i, i)}:
            kappa[a, b, c] = 1
    st, *_ = emu.coni_mu0_batch(kappa, np.array([[1, 0, 0]]))
    assert st[0] == 1                                           # S = -I: negative definite


def test_device_mu0_beyond_int128_products():
    """mixed's h11 = 16 geometries: the reference's C code stops on int128
    overflow (status -3); the device's 256-bit elimination decides them, equal
    to the exact oracle.  At h11 = 24 the determinant itself passes 2^127 and
    the device reports the direction undecided (< 0)."""
    w = workloads.build("mixed", n_p=8)
    decided = {16: 0, 24: 0}
    for p, k in zip(w.ps, w.pgeo):
        g = w.geoms[int(k)]
        if g.h11 not in decided:
            continue
        st, num, den, K = emu.coni_mu0_batch(g.kappa, np.asarray(p[1:])[None])
        if g.h11 == 24:
            assert st[0] < 0
            continue
        so, mo, _ = omu0.coni_mu0(g.kappa, p[1:])
        assert st[0] == so == 0 and _frac(num[0], den[0]) == mo
        decided[16] += 1
    assert decided[16] >= 2


def test_grid_up_is_the_reference_grid():
    D = np.concatenate([np.arange(1, 20000), [10 ** 6, 12345678, 2 ** 40 + 1]])
    np.testing.assert_array_equal(dilation.grid_up(D), omu0.grid_up(D))
    g = dilation.grid_up(np.array([1, 2, 3, 100, 799, 800, 801, 12345, 10 ** 6]))
    D = np.array([1, 2, 3, 100, 799, 800, 801, 12345, 10 ** 6])
    assert np.all(g >= D) and np.all(g <= np.ceil(D * 2 ** (1 / 16)) + 1)


def test_ceilings_exact_beyond_int64():
    num = np.array([3, 7, 1, 5, 2 ** 60], dtype=np.int64)
    den = np.array([10, 2 ** 61, 1, 2 ** 62 + 1, 2 ** 62 + 3], dtype=np.int64)
    Q = 118
    got, fits = dilation._ceil_q_over(Q, num, den)
    want = [-((-Q * int(d)) // int(a)) for a, d in zip(num, den)]
    assert [int(x) for x, f in zip(got, fits) if f] == [w for w in want if w < 2 ** 63]
    assert list(fits) == [w < 2 ** 63 for w in want] == [True, False, True, False, True]


def _fake_device(monkeypatch, zpm_points):
    """coni_zp's device calls replaced by the oracle: mu0 per direction, and
    the PFVs of each (direction, dilation) from zpm_points."""
    def mu0_batch(ps, kappa, device=0):
        ps = np.atleast_2d(ps)
        st = np.zeros(len(ps), np.int32)
        num, den = np.zeros(len(ps), np.int64), np.zeros(len(ps), np.int64)
        K = np.zeros_like(ps)
        for i, p in enumerate(ps):
            s, m, k = omu0.coni_mu0(kappa, p)
            st[i] = s
            if s == 0:
                num[i], den[i], K[i] = m.numerator, m.denominator, k
        return st, num, den, K

    def pfvs_multi(geoms, ps, pgeo, device=0):
        Ks, Ms, pidx = [], [], []
        for i, (p, k) in enumerate(zip(ps, pgeo)):
            for K, M in zpm_points(tuple(int(x) for x in p), geoms[int(k)]["dilation"]):
                Ks.append(K)
                Ms.append(M)
                pidx.append(i)
        h = len(ps[0])
        Ks = np.array(Ks, dtype=np.int64).reshape(-1, h)
        Ms = np.array(Ms, dtype=np.int64).reshape(-1, h)
        return Ks, Ms, np.array(pidx, dtype=np.int64), np.zeros(len(ps), np.int8), 0.0, {}
    monkeypatch.setattr(dilation, "coni_mu0_batch", mu0_batch)
    monkeypatch.setattr(coni.gpu, "coni_pfvs_multi", pfvs_multi)


def test_coni_zp_routing_and_canonical_order(monkeypatch):
    """Each direction is searched at grid_up(ceil(Q / mu0)), one without a
    bound at fallback_dilation and marked incomplete; the PFVs come back once
    each, sorted by p-vector then (M, K)."""
    k = int(G["gidx"][0])
    kappa = G[f"kappa{k}"]
    h = kappa.shape[0]
    Q = int(G["Q"][0])
    rows = [i for i in range(len(G["status"])) if int(G["gidx"][i]) == k][:3]
    ps = [G["p"][i][1:h] for i in rows]
    nb = [G["r_p"][i][:h - 1] for i in range(len(G["r_status"]))
          if int(G["r_gidx"][i]) == k and int(G["r_status"][i]) == 1][:1]
    assert nb
    ps = np.array(ps + nb + ps[:1])                            # (a repeated p-vector too)
    searched = {}

    def zpm_points(p, D):
        searched.setdefault(p, []).append(D)
        v = int(sum(p))                                        # two synthetic PFVs per direction, one repeated
        return [([0] + [v] * (h - 1), [1] + [2] * (h - 1)), ([0] + [v] * (h - 1), [1] + [2] * (h - 1)),
                ([0] * h, [int(D)] + [0] * (h - 1))]
    _fake_device(monkeypatch, zpm_points)
    Ks, Ms, complete, info = coni.coni_zp(kappa, np.eye(h, dtype=np.int64), ps, Q, fallback_dilation=30,
                                          return_info=True)
    for i, p in enumerate(ps):
        st, m, _ = omu0.coni_mu0(kappa, p)
        D = searched[tuple([0] + [int(x) for x in p])][0]
        if st == 0:
            b = -((-Q * m.denominator) // m.numerator)
            assert D == omu0.grid_up([b])[0] and complete[i]
            assert info["bceil"][i] == b
        else:
            assert D == 30 and not complete[i]
    keys = info["keys"]
    assert np.all(np.diff(keys) >= 0)
    assert len(keys) == 2 * len(ps)                            # the repeated PFV once per p-vector
    rows_ = np.hstack([keys[:, None], Ms, Ks])
    assert len(np.unique(rows_, axis=0)) == len(rows_)
    np.testing.assert_array_equal(np.unique(rows_, axis=0), rows_)


def test_coni_zp_multi_equals_one_geometry_at_a_time(monkeypatch):
    """coni_zp_multi (every geometry's searches in one device call) returns,
    per geometry, what coni_zp returns for it alone."""
    hs = {int(k): G[f"kappa{k}"].shape[0] for k in np.unique(G["gidx"])}
    h = next(v for v in sorted(set(hs.values())) if sum(1 for x in hs.values() if x == v) >= 2)
    ks = [k for k, v in hs.items() if v == h][:2]
    items = []
    for k in ks:
        rows = [i for i in range(len(G["status"])) if int(G["gidx"][i]) == k][:3]
        items.append(dict(kappa=G[f"kappa{k}"], Mbasis=np.eye(h, dtype=np.int64) * (k + 1),
                          ps=np.array([G["p"][i][1:h] for i in rows]), Q=int(G["Q"][rows[0]]), M0min=13))

    def zpm_points(p, D):
        v = int(sum(p)) + int(D)
        return [([0] + [v] * (h - 1), [1] + [2] * (h - 1)), ([0] * h, [int(D) % 7] + [1] * (h - 1))]
    _fake_device(monkeypatch, zpm_points)
    multi = coni.coni_zp_multi(items, return_info=True)
    for it, (Ks, Ms, complete, info) in zip(items, multi):
        one = coni.coni_zp(it["kappa"], it["Mbasis"], it["ps"], it["Q"], return_info=True)
        np.testing.assert_array_equal(Ks, one[0])
        np.testing.assert_array_equal(Ms, one[1])
        np.testing.assert_array_equal(complete, one[2])
        np.testing.assert_array_equal(info["keys"], one[3]["keys"])
        np.testing.assert_array_equal(info["dilation"], one[3]["dilation"])
        assert len(Ks) > 0
