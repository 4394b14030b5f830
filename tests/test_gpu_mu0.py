"""
GPU: the coni dilation bound on the device (k_mu0 through
pfvs_b200.dilation) and the exhaustive coniZp driver (pfvs_b200.coni) on the
reference's coni dataset geometries (tests/golden/dataset_pfvs.npz: 30
geometries, h11 3..9, 10,399 p-vectors of the coni cones' boxes) and the
fixtures' PFV directions (tests/golden/mu0.npz):

- mu0 equals the reference's C code's (coni_bound.h:255, oracle/_ref) on
  every direction it decides, and the exact oracle's elsewhere; every
  fixture PFV's dilation is below Q / mu0;
- coniZp equals coniZpM run at each direction's ceil(Q / mu0), each PFV
  once, every direction complete (the check of the reference's
  tests/test_coni_zpk.py:172-188), with the searches at ceil(b) computed by
  the reference build plus the oracle's post-processing on a sample of the
  directions and by the device on all of them;
- it contains every published PFV of the p-vectors (found at dilation 150);
- searching past the bound finds nothing more
  (tests/test_dilation_bound.py:216-238 of the reference).
"""
import os
from fractions import Fraction

import numpy as np
import pytest

from conftest import ROOT
from oracle import mu0 as omu0
from oracle import postproc, ref
from pfvs_b200 import coni, dilation, gpu, workloads

pytestmark = pytest.mark.gpu

G = np.load(os.path.join(ROOT, "tests", "golden", "mu0.npz"))


def _need_gpu():
    if not gpu.available():
        pytest.fail("no CUDA device: " + gpu.unavailable_reason())


def _dataset():
    D = np.load(os.path.join(ROOT, "tests", "golden", "dataset_pfvs.npz"))
    out = []
    for k in range(int(D["n_geometries"][0])):
        h, Q, m0 = (int(x) for x in D[f"g{k}_scal"])
        pub = {(tuple(a), tuple(b)) for a, b in zip(D[f"g{k}_K"].tolist(), D[f"g{k}_M"].tolist())}
        out.append(dict(kappa=D[f"g{k}_kappa"], Mbasis=D[f"g{k}_Mbasis"], Q=Q, M0min=m0,
                        ps=D[f"g{k}_ps"][:, 1:], pub=pub))
    return out


def _as_set(Ks, Ms, keys=None):
    if keys is None:
        return {(tuple(int(x) for x in k), tuple(int(x) for x in m)) for k, m in zip(Ks, Ms)}
    return {(int(i), tuple(int(x) for x in k), tuple(int(x) for x in m)) for i, k, m in zip(keys, Ks, Ms)}


def test_device_mu0_on_fixture_pfvs_and_other_directions():
    _need_gpu()
    for k in np.unique(G["gidx"]):
        kappa = G[f"kappa{k}"]
        h = kappa.shape[0]
        rows = np.flatnonzero(G["gidx"] == k)
        st, num, den, K = dilation.coni_mu0_batch(G["p"][rows][:, 1:h], kappa)
        for j, i in enumerate(rows):
            assert st[j] == 0
            m = Fraction(int(num[j]), int(den[j]))
            assert m == Fraction(*(int(x) for x in G["mu0"][i]))
            assert Fraction(*(int(x) for x in G["delta"][i])) < Fraction(int(G["Q"][i])) / m
            assert int(np.dot(K[j], G["p"][i][1:h])) == 0 and K[j].any()
        rr = np.flatnonzero(G["r_gidx"] == k)
        st, num, den, _ = dilation.coni_mu0_batch(G["r_p"][rr][:, :h - 1], kappa)
        for j, i in enumerate(rr):
            rs = int(G["r_status"][i])
            if rs >= 0:
                assert st[j] == rs
                if rs == 0:
                    assert Fraction(int(num[j]), int(den[j])) == Fraction(*(int(x) for x in G["r_mu0"][i]))
            else:
                so, mo, _ = omu0.coni_mu0(kappa, G["r_p"][i][:h - 1])
                assert st[j] == so and (so == 1 or Fraction(int(num[j]), int(den[j])) == mo)


def test_device_mu0_on_dataset_directions_equals_reference_c():
    _need_gpu()
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    n = 0
    for g in _dataset():
        st, num, den, _ = dilation.coni_mu0_batch(g["ps"], g["kappa"])
        for j, p in enumerate(g["ps"]):
            sr, mr, _ = ref.coni_mu0(g["kappa"], p)
            if sr >= 0:
                assert st[j] == sr and (sr == 1 or Fraction(int(num[j]), int(den[j])) == mr)
            else:
                so, mo, _ = omu0.coni_mu0(g["kappa"], p)
                assert st[j] == so and (so == 1 or Fraction(int(num[j]), int(den[j])) == mo)
            n += 1
    assert n > 10000


def test_device_mu0_beyond_the_reference_c_range():
    """h11 = 16 (int128 products: the C code stops, the device's 256-bit
    elimination decides) equals the exact oracle; at h11 = 24 and 32 the
    device reports the directions undecided."""
    _need_gpu()
    w = workloads.build("mixed", n_p=64)
    seen = 0
    for k, g in enumerate(w.geoms):
        sel = np.flatnonzero(np.asarray(w.pgeo) == k)[:4]
        if not len(sel):
            continue
        P = np.array([w.ps[i][1:] for i in sel])
        st, num, den, _ = dilation.coni_mu0_batch(P, g.kappa)
        if g.h11 > 16:
            assert np.all(st < 0)
            continue
        for j, p in enumerate(P):
            so, mo, _ = omu0.coni_mu0(g.kappa, p)
            assert st[j] == so and (so == 1 or Fraction(int(num[j]), int(den[j])) == mo)
            seen += g.h11 == 16
    assert seen >= 4


def _zpm_at(g, ps, dil):
    """Device coniZpM PFVs of each p-vector at its own dilation: (Ks, Ms, keys)."""
    h = g["kappa"].shape[0]
    Ds, gi = np.unique(dil, return_inverse=True)
    geoms = [dict(kappa=g["kappa"], Mbasis=g["Mbasis"], Q=g["Q"], dilation=float(D), M0min=g["M0min"]) for D in Ds]
    P = np.hstack([np.zeros((len(ps), 1), np.int64), ps])
    K, M, pidx, pstat, _, _ = gpu.coni_pfvs_multi(geoms, P, gi.astype(np.int32))
    assert np.all(pstat == 0)
    return K[:, :h], M[:, :h], pidx


def test_coni_zp_exhaustive_on_dataset():
    _need_gpu()
    n_pfvs = 0
    for g in _dataset():
        Ks, Ms, complete, info = coni.coni_zp(g["kappa"], g["Mbasis"], g["ps"], g["Q"], M0min=g["M0min"],
                                              return_info=True)
        assert complete.all()
        b = info["bceil"]
        np.testing.assert_array_equal(info["dilation"], dilation.grid_up(b))
        want = _as_set(*_zpm_at(g, g["ps"], b.astype(np.float64)))
        got = _as_set(Ks, Ms, info["keys"])
        assert got == want and len(got) == len(Ks)
        assert g["pub"] <= _as_set(Ks, Ms)
        n_pfvs += len(Ks)
    assert n_pfvs > 400                          # (431: the 367 published ones and the rest at dilations above 150)


def test_coni_zp_matches_reference_build_on_a_sample():
    """coniZp's PFVs of a sample of directions equal the reference build's
    points (oracle/_ref) at ceil(Q / mu0) run through the oracle's
    post-processing."""
    _need_gpu()
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(0)
    checked = 0
    for g in _dataset():
        h = g["kappa"].shape[0]
        sel = np.sort(rng.choice(len(g["ps"]), min(len(g["ps"]), 24), replace=False))
        ps = g["ps"][sel]
        Ks, Ms, complete, info = coni.coni_zp(g["kappa"], g["Mbasis"], ps, g["Q"], M0min=g["M0min"],
                                              return_info=True)
        want = set()
        for i, p in enumerate(ps):
            P = np.concatenate([[0], p])[None]
            M, Kn, q, pl, st, _ = ref.coni_batch(g["kappa"], g["Mbasis"], P, g["Q"], float(info["bceil"][i]),
                                                 g["M0min"])
            assert st[0] == 0
            eK, eM, _ = postproc.pfvs_from_points(M[:, :h], Kn[:, :h], q, np.full(len(q), i), g["kappa"], h,
                                                  g["Q"], g["M0min"])
            want |= {(i, tuple(int(x) for x in k), tuple(int(x) for x in m)) for k, m in zip(eK, eM)}
        assert _as_set(Ks, Ms, info["keys"]) == want
        checked += len(ps)
    assert checked > 500


def test_search_past_the_bound_finds_nothing_more():
    _need_gpu()
    for g in _dataset()[:12]:
        ps = g["ps"][:4]
        b = dilation.coni_dilation_bound_ceils(ps, g["kappa"], g["Q"])
        assert np.all(b > 0)
        at = _as_set(*_zpm_at(g, ps, b.astype(np.float64)))
        big = _as_set(*_zpm_at(g, ps, 2.0 * b + 20))
        assert at == big


def test_coni_zp_multi_equals_per_geometry():
    """All dataset geometries through coni_zp_multi (their searches in one
    device call) give each geometry's coni_zp result."""
    _need_gpu()
    data = _dataset()
    items = [dict(kappa=g["kappa"], Mbasis=g["Mbasis"], ps=g["ps"], Q=g["Q"], M0min=g["M0min"]) for g in data]
    multi = coni.coni_zp_multi(items)
    for g, (Ks, Ms, complete) in zip(data, multi):
        one = coni.coni_zp(g["kappa"], g["Mbasis"], g["ps"], g["Q"], M0min=g["M0min"])
        np.testing.assert_array_equal(Ks, one[0])
        np.testing.assert_array_equal(Ms, one[1])
        np.testing.assert_array_equal(complete, one[2])
