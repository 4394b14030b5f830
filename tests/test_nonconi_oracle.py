"""
Non-coni ZpM (pfvs/nonconi.py:262) in the oracle (oracle/nonconi.py),
pinned to the reference (tests/golden/nonconi.npz, made by
tests/golden/make_nonconi_golden.py from its paper examples, its Manwe test
geometry and its own C setup and kernel):

- the oracle's lattice points of every p-vector equal the reference's;
- its PFV set equals the reference route's, and contains each paper vacuum
  (the check of the reference's tests/test_paper_examples.py:93-101);
- the non-coni M-lattice (b = c2, the whole a-matrix) holds every paper M.
"""
import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import nonconi
from pfvs_b200 import intlat

G = np.load(os.path.join(ROOT, "tests", "golden", "nonconi.npz"))
CASES = range(int(G["n_cases"][0]))


def _rows(M, Kn, q, pidx):
    return {(int(i), tuple(int(x) for x in m), tuple(int(x) for x in k), int(v))
            for i, m, k, v in zip(pidx, M, Kn, q)}


@pytest.mark.parametrize("k", CASES)
def test_oracle_points_equal_reference(k):
    kappa, Mb, ps = G[f"c{k}_kappa"], G[f"c{k}_Mbasis"], G[f"c{k}_ps"]
    Qmin, Qmax = (int(x) for x in G[f"c{k}_scal"])
    D = float(G[f"c{k}_D"][0])
    np.testing.assert_array_equal(intlat.m_lattice(kappa, G[f"c{k}_c2"], coni=False), Mb)
    qmax = nonconi.qmax_of(Qmax, D)
    got = set()
    sel = range(len(ps)) if len(ps) < 50 else range(0, len(ps), 3)
    for i in sel:
        st, C, M, Kn, q = nonconi.points(kappa, Mb, ps[i], Qmax, qmax)
        assert st == 0
        got |= _rows(M, Kn, q, np.full(len(q), i))
    ref = _rows(G[f"c{k}_M"], G[f"c{k}_Kn"], G[f"c{k}_q"], G[f"c{k}_pidx"])
    ref = {r for r in ref if r[0] in set(sel)}
    assert got == ref and len(ref) > 0


@pytest.mark.parametrize("k", CASES)
def test_oracle_pfvs_equal_reference(k):
    kappa, Mb, ps = G[f"c{k}_kappa"], G[f"c{k}_Mbasis"], G[f"c{k}_ps"]
    Qmin, Qmax = (int(x) for x in G[f"c{k}_scal"])
    D = float(G[f"c{k}_D"][0])
    if len(ps) > 50 and D > 1:
        pytest.skip("(the dilation-3 Manwe case is covered point for point above)")
    pf, sts = nonconi.zpm(kappa, Mb, ps, Qmin, Qmax, D)
    assert np.all(sts == 0)
    want = {(tuple(int(x) for x in a), tuple(int(x) for x in b)) for a, b in zip(G[f"c{k}_pfvK"], G[f"c{k}_pfvM"])}
    assert pf == want and len(want) > 0
    if f"c{k}_knownK" in G:
        assert (tuple(int(x) for x in G[f"c{k}_knownK"]), tuple(int(x) for x in G[f"c{k}_knownM"])) in pf
