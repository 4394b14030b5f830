"""
Non-coni ZpM on the device code (pfg_zpm_batch's setup and search:
pfvs_b200/csrc/pfg_setup.cuh with coni = 0 -- no coni column order, the whole
basis LLL-reduced w.r.t. mat, GCD rows of all of ZB -- and pfg_search.cuh's
non-strict cut on all of K) run on the CPU warp emulator (tests/emu), against
the reference's own C setup and kernel (tests/golden/nonconi.npz, made by
tests/golden/make_nonconi_golden.py): the same lattice points (M, Kn, q) of
every p-vector, with FP64 and with FP32 pruning.  The paper's vacuum 6.4
(p = (293, 163, 163, 65)) has a mat entry of 2.6e10, beyond the search's
int32 staging: its direction is searched with mat read from the slab
(Dir.wide), its sums bounded through the ellipsoid's coordinate ranges.
"""
import os

import numpy as np
import pytest

from conftest import ROOT
from emu import emu

G = np.load(os.path.join(ROOT, "tests", "golden", "nonconi.npz"))
CASES = range(int(G["n_cases"][0]))


@pytest.mark.parametrize("k", CASES)
def test_device_nonconi_points_equal_reference(k):
    kappa, Mb, ps = G[f"c{k}_kappa"], G[f"c{k}_Mbasis"], G[f"c{k}_ps"]
    Qmin, Qmax = (int(x) for x in G[f"c{k}_scal"])
    D = float(G[f"c{k}_D"][0])
    h = kappa.shape[0]
    geoms = [dict(kappa=kappa, Mbasis=Mb, Q=Qmax, dilation=D, M0min=0)]
    sel = np.arange(len(ps)) if len(ps) < 50 else np.arange(0, len(ps), 4)
    for prec in ((2, 1) if len(sel) < 50 and D == 1 else (2,)):
        M, Kn, q, pidx, pstat, _, _ = emu.coni_batch_multi(geoms, ps[sel], np.zeros(len(sel), np.int32),
                                                           precision=prec, coni=False)
        assert np.all(pstat == 0)
        got = [(int(sel[i]), tuple(m[:h]), tuple(x[:h]), int(v)) for i, m, x, v in
               zip(pidx, M.tolist(), Kn.tolist(), q)]
        ref = [(int(i), tuple(m), tuple(x), int(v)) for i, m, x, v in
               zip(G[f"c{k}_pidx"], G[f"c{k}_M"].tolist(), G[f"c{k}_Kn"].tolist(), G[f"c{k}_q"])
               if int(i) in set(sel.tolist())]
        assert got == ref and len(ref) > 0           # (both in the canonical order)


@pytest.mark.parametrize("k", CASES)
def test_host_postprocessing_gives_the_reference_pfvs(k):
    """The product's post-processing (pfvs_b200.nonconi: primitive points,
    exact singularity, K, tadpole window, the GCD multiples) on the
    reference's points gives the reference route's PFV set; on the emulated
    device's points (the small cases) the same."""
    from pfvs_b200 import nonconi
    kappa, Mb, ps = G[f"c{k}_kappa"], G[f"c{k}_Mbasis"], G[f"c{k}_ps"]
    Qmin, Qmax = (int(x) for x in G[f"c{k}_scal"])
    h = kappa.shape[0]
    want = {(tuple(int(x) for x in a), tuple(int(x) for x in b)) for a, b in zip(G[f"c{k}_pfvK"], G[f"c{k}_pfvM"])}
    pidx, M, Kn = G[f"c{k}_pidx"], G[f"c{k}_M"], G[f"c{k}_Kn"]
    Ks, Ms = [], []
    for i in range(len(ps)):
        sel = pidx == i
        K, Mm = nonconi.pfvs_from_points(M[sel], Kn[sel], kappa, Mb, Qmin, Qmax)
        Ks.append(K)
        Ms.append(Mm)
    Ks, Ms = nonconi.allow_gcds(np.vstack(Ks), np.vstack(Ms), Qmax, h)
    got = {(tuple(int(x) for x in a), tuple(int(x) for x in b)) for a, b in zip(Ks, Ms)}
    assert got == want and len(got) == len(Ks) > 0
    rows = np.hstack([Ks, Ms])
    np.testing.assert_array_equal(np.unique(rows, axis=0), rows)       # sorted by (K, M), each once
    if f"c{k}_knownK" in G:
        assert (tuple(int(x) for x in G[f"c{k}_knownK"]), tuple(int(x) for x in G[f"c{k}_knownM"])) in got


def test_singular_mask_exact():
    from pfvs_b200 import nonconi
    rng = np.random.default_rng(3)
    Ns = rng.integers(-5, 6, size=(200, 5, 5))
    Ns[::7, 2] = Ns[::7, 0] * 2 - Ns[::7, 1]                    # singular by construction
    Ns[1] = 0
    big = Ns[:20].astype(object) * (2 ** 40)
    want = np.array([round(np.linalg.det(N.astype(float))) == 0 for N in Ns])
    np.testing.assert_array_equal(nonconi.singular_mask(Ns), want)
    np.testing.assert_array_equal(nonconi.singular_mask(big), want[:20])
    assert want[::7].all() and not want.all()
