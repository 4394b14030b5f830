"""
The coni dilation bound mu0 (pfvs/dilation.py:145, C path
pfvs/fp_kernel/coni_bound.h:255) in the oracle (oracle/mu0.py), pinned to the
reference:

- on every PFV of the reference's fixtures (tests/golden/mu0.npz, made by
  tests/golden/make_mu0_golden.py from its fixtures and its own C code), the
  oracle's mu0 equals the reference's, and the PFV's dilation is below the
  bound Q / mu0 (the property the reference's tests/test_dilation_bound.py:110-117
  checks);
- the minimizer K lies in Lambda (p_r . K = 0) and attains mu0;
- on synthetic directions the oracle equals the reference's C code wherever
  that code decides (it stops at h11 = 20 and on int128 overflow).
"""
import os
from fractions import Fraction

import numpy as np
import pytest

from conftest import ROOT
from oracle import mu0, ref
from pfvs_b200 import workloads

G = np.load(os.path.join(ROOT, "tests", "golden", "mu0.npz"))


def test_oracle_matches_reference_on_every_fixture_pfv():
    n = len(G["status"])
    assert n > 300
    for i in range(n):
        h, Q = int(G["h"][i]), int(G["Q"][i])
        kappa = G[f"kappa{int(G['gidx'][i])}"]
        p_r = G["p"][i][1:h]
        st, m, K = mu0.coni_mu0(kappa, p_r)
        assert st == 0 == int(G["status"][i])
        assert m == Fraction(int(G["mu0"][i][0]), int(G["mu0"][i][1]))
        delta = Fraction(int(G["delta"][i][0]), int(G["delta"][i][1]))
        assert delta < Fraction(Q) / m
        assert sum(int(a) * int(b) for a, b in zip(K, p_r)) == 0 and any(K)


def test_minimizer_attains_mu0():
    for i in range(0, len(G["status"]), 11):
        h = int(G["h"][i])
        kappa = G[f"kappa{int(G['gidx'][i])}"]
        p_r = [int(x) for x in G["p"][i][1:h]]
        st, m, K = mu0.coni_mu0(kappa, p_r)
        p_hat = [0] + p_r
        A = [[sum(int(kappa[a, b, c]) * p_hat[c] for c in range(h)) for b in range(h)] for a in range(h)]
        x = mu0._solve_exact([row[1:] for row in A[1:]], [K])[0]       # A_rr^-1 K
        assert -sum(Fraction(k) * v for k, v in zip(K, x)) == m


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name,n", [("small", 32), ("plain", 16), ("mixed", 8)])
def test_oracle_matches_reference_c_on_synthetic_directions(name, n):
    w = workloads.build(name, n_p=n)
    decided = 0
    for p, k in zip(w.ps, w.pgeo):
        g = w.geoms[int(k)]
        sr, mr, _ = ref.coni_mu0(g.kappa, p[1:])
        so, mo, _ = mu0.coni_mu0(g.kappa, p[1:])
        if sr >= 0:
            assert so == sr and mo == mr
            decided += 1
    assert decided >= 2


def test_grid_up():
    D = np.arange(1, 5000)
    g = mu0.grid_up(D)
    assert np.all(g >= D)
    assert np.all(g <= np.maximum(D + 1, np.ceil(D * 2 ** (1 / 16)) + 1))
    assert len(np.unique(g)) < len(D) / 5                     # nearby bounds share a grid point
    assert np.all(np.diff(g) >= 0)                            # monotone
