"""
CPU tests (no GPU): the oracle pinned to the reference, the committed golden
vectors, the device sources under the CPU warp emulator, and the workload
generator's properties.

- the restated kernel vs the reference's 219 kernel fixtures (812 cases;
  tests/test_kernels.py:64-77 of the reference) -- needs the reference tree;
- the restated pipeline vs the published PFV sets of the reference's dataset
  geometries under the rule of tests/test_dataset.py:59-86 (h11 <= 5 here,
  so that the CPU suite stays within minutes);
- the restated pipeline vs the reference build (oracle/_ref) and vs the
  golden vectors generated from it (tests/golden/make_golden.py).
"""
import gzip
import json
import os

import numpy as np
import pytest

from conftest import REFERENCE, ROOT
from oracle import pfo, postproc, pvecs, ref
from parity import assert_same, expected, layout
from pfvs_b200 import intlat, workloads

FIXTURES = os.path.join(REFERENCE, "tests", "data", "fixtures.json.gz")
needs_reference = pytest.mark.skipif(not os.path.exists(FIXTURES), reason="reference tree not present")
needs_ref_build = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")


def _fixtures():
    with gzip.open(FIXTURES) as f:
        return json.load(f)


@needs_reference
def test_oracle_kernel_matches_reference_fixtures():
    F = _fixtures()
    n = 0
    for k in F["kernel"]:
        for dil, exp in k["expected"].items():
            qmax = ref.qmax_of(k["Q"], float(dil))
            pts, qs, st, _ = pfo.kernel(k["mat"], k["Q"], qmax, k["H"], k["linvec"],
                                        ref.linmin_of(k["M0min"]), strict=True)
            assert st == 0
            assert [tuple(map(int, r)) for r in pts] == [tuple(c) for c in exp["pts"]]
            assert [int(x) for x in qs] == exp["qs"]
            n += 1
    assert n == 812


@needs_reference
def test_reference_build_matches_reference_fixtures(ref_available):
    if not ref_available:
        pytest.skip("oracle/_ref not built")
    F = _fixtures()
    for k in F["kernel"][::7]:
        for dil, exp in k["expected"].items():
            pts, qs, st, _ = ref.kernel(k["mat"], k["Q"], ref.qmax_of(k["Q"], float(dil)), k["H"],
                                        k["linvec"], ref.linmin_of(k["M0min"]), strict=True)
            assert st == 0 and [tuple(map(int, r)) for r in pts] == [tuple(c) for c in exp["pts"]]


def _cydata(g):
    h = g["h11"]
    kappa = np.zeros((h,) * 3, dtype=np.int64)
    for i, j, k, v in g["kappa_coo"]:
        for a, b, c in {(i, j, k), (i, k, j), (j, i, k), (j, k, i), (k, i, j), (k, j, i)}:
            kappa[a, b, c] = v
    Hc = np.array(g["H"], dtype=np.int64)
    return kappa, Hc[np.any(Hc != 0, axis=1)]


@needs_reference
def test_oracle_pipeline_reproduces_dataset_pfvs():
    F = _fixtures()
    done = 0
    for g in F["geometries"]:
        h = g["h11"]
        if h > 5:
            continue
        kappa, Hc = _cydata(g)
        Mb = intlat.m_lattice(kappa, np.array(g["c2"]))
        ps = pvecs.box_enum(g["B"], Hc)
        Q = h + g["h21"] + 4
        exp = {(tuple(K), tuple(M)) for K, M in zip(g["K"], g["M"])}
        if len(ps) == 0:
            assert exp == set()
            continue
        pfull = np.hstack([np.zeros((len(ps), 1), np.int64), ps])
        M, Kn, q, pidx, st, _ = pfo.coni_batch(kappa, Mb, pfull, Q, g["D"], 13)
        assert np.all(st == 0)
        Ks, Ms, _ = postproc.pfvs_from_points(M, Kn, q, pidx, kappa, h, Q, 13)
        got = {(tuple(int(x) for x in K), tuple(int(x) for x in m)) for K, m in zip(Ks, Ms)}
        primitive = {KM for KM in got if np.gcd.reduce(np.array(KM[0][1:])) == 1}
        assert exp <= got and primitive == exp
        for K, m in got - exp:
            assert np.gcd.reduce(np.array(K[1:])) >= 2
            assert -int(np.dot(K, m)) == Q and m[0] >= 13
        done += 1
    assert done >= 10


@needs_ref_build
@pytest.mark.parametrize("name,n,dils", [("plain", 64, (150.0,)), ("mixed", 48, None),
                                         ("precision", 4, None)])
def test_oracle_matches_reference_build(name, n, dils):
    w = workloads.build(name, n_p=n, dilations=dils)
    geoms, ps, pgeo, _ = layout(w)
    a = expected(geoms, ps, pgeo, "oracle")
    b = expected(geoms, ps, pgeo, "ref")
    assert_same(a, b, ok_mask=b[4] == 0)


GOLDEN = sorted(f[:-4] for f in os.listdir(os.path.join(ROOT, "tests", "golden"))
                if f.endswith(".npz") and f not in ("dataset_pfvs.npz", "mu0.npz", "nonconi.npz", "zpk.npz"))


@pytest.mark.parametrize("key", GOLDEN)
def test_oracle_matches_golden(key):
    """The oracle against the reference build's committed answers."""
    G = np.load(os.path.join(ROOT, "tests", "golden", key + ".npz"))
    dils = tuple(G["dilations"].tolist()) or None
    w = workloads.build(str(G["workload"]), n_p=int(G["n"]), dilations=dils)
    geoms, ps, pgeo, _ = layout(w)
    M, Kn, q, pidx, st = expected(geoms, ps, pgeo, "oracle")
    ok = G["status"] == 0
    h = G["M"].shape[1]
    sel = ok[pidx] if len(pidx) else np.zeros(0, bool)
    np.testing.assert_array_equal(pidx[sel], G["pidx"])
    np.testing.assert_array_equal(q[sel], G["q"])
    np.testing.assert_array_equal(M[sel][:, :h], G["M"])
    np.testing.assert_array_equal(Kn[sel][:, :h], G["Kn"])


def test_postproc_singular_mask():
    A = np.array([[[1, 2], [2, 4]], [[1, 0], [0, 1]], [[3, 5], [6, 10]]], dtype=np.int64)
    np.testing.assert_array_equal(postproc.singular_mask(A), [True, False, True])


def test_m_lattice_properties():
    for h, rows, ones, sw in [(5, 8, (1, 3), (1, 3)), (11, 8, (1, 4), (1, 3))]:
        g = workloads.make_geometry(h, 2 * h + 40, rows, ones, sw, seed=3)
        a, b = intlat.a_matrix(g.kappa), intlat.b_vector(g.c2)
        Mb = g.Mbasis
        assert np.all((a @ Mb) % 2 == 0) and np.all((b @ Mb) % 24 == 0)
        # index of the lattice = number of residue classes of Z^h it keeps, by counting mod 24
        det = abs(round(np.linalg.det(Mb.astype(float))))
        rng = np.random.default_rng(0)
        # every integer vector satisfying the congruences is in the lattice
        for _ in range(50):
            x = rng.integers(-5, 6, h)
            M = 24 * x
            coeff = np.linalg.solve(Mb.astype(float), M.astype(float))
            assert np.allclose(coeff, np.round(coeff))
        assert det > 0


def test_workload_prefix_property():
    a = workloads.build("mixed", n_p=64)
    b = workloads.build("mixed", n_p=16)
    for i in range(16):
        assert np.array_equal(a.ps[i], b.ps[i]) and a.pgeo[i] == b.pgeo[i] and a.dil[i] == b.dil[i]
    assert all(workloads.lorentzian_ok(a.geoms[a.pgeo[i]].kappa, a.ps[i]) for i in range(64))


def test_device_code_under_warp_emulator():
    """The library's device sources, run on CPU threads (tests/emu), equal the
    oracle on a small case; divergent warp collectives abort the run."""
    from emu import emu
    # plain h11 = 11 at dilation 150: three directions with points (one with two)
    w = workloads.build("plain", n_p=96, dilations=(150.0,))
    geoms, ps, pgeo, _ = layout(w)
    sel = [3, 25, 65, 86]
    ps, pgeo = [ps[i] for i in sel], pgeo[sel]
    M, Kn, q, pidx, pstat, nodes, stage = emu.coni_batch_multi(geoms, ps, pgeo)
    assert np.all(pstat == 0) and nodes.sum() > 0 and len(q) == 4
    assert_same((M, Kn, q, pidx), expected(geoms, ps, pgeo, "oracle"))
    # mixed h11 = 8 .. 32: directions of the h11 = 32 geometry with 3 and 47 points
    # (the emulator build sorts from runs of one point, so these go through the merges)
    w = workloads.build("mixed", n_p=96)
    geoms, ps, pgeo, _ = layout(w)
    sel = [3, 83, 85, 87]
    ps, pgeo = [ps[i] for i in sel], pgeo[sel]
    got = emu.coni_batch_multi(geoms, ps, pgeo)
    assert np.all(got[4] == 0) and len(got[2]) == 51
    assert_same(got[:4], expected(geoms, ps, pgeo, "oracle"))


def test_device_code_under_warp_emulator_on_dataset_geometries():
    """The device sources (CPU warp emulator) on the reference's own coni
    dataset geometries (tests/golden/dataset_pfvs.npz, h11 3..9): the first
    4 p-vectors of each of the 30 geometries, points equal to the oracle's."""
    from emu import emu
    G = np.load(os.path.join(ROOT, "tests", "golden", "dataset_pfvs.npz"))
    geoms, ps, pgeo = [], [], []
    for k in range(int(G["n_geometries"][0])):
        h, Q, m0 = (int(x) for x in G[f"g{k}_scal"])
        geoms.append(dict(kappa=G[f"g{k}_kappa"], Mbasis=G[f"g{k}_Mbasis"], Q=Q,
                          dilation=float(G[f"g{k}_D"][0]), M0min=m0))
        for p in G[f"g{k}_ps"][:4]:
            ps.append(np.asarray(p, dtype=np.int64))
            pgeo.append(k)
    pgeo = np.array(pgeo, dtype=np.int32)
    got = emu.coni_batch_multi(geoms, ps, pgeo)
    assert np.all(got[4] == 0) and len(got[2]) > 20
    assert_same(got[:4], expected(geoms, ps, pgeo, "oracle"))



def test_device_code_under_warp_emulator_with_gcd_rows_everywhere():
    """The device search with GCD-cut rows built for every direction (the
    reference's pruning): points equal the oracle's, and the rows prune
    (fewer nodes than without them)."""
    from emu import emu
    w = workloads.build("mixed", n_p=96)
    geoms, ps, pgeo, _ = layout(w)
    sel = [3, 83, 85, 87]
    ps, pgeo = [ps[i] for i in sel], pgeo[sel]
    try:
        emu.set_gcd_min_tree(-1.0)
        rows = emu.coni_batch_multi(geoms, ps, pgeo, precision=1)
        emu.set_gcd_min_tree(1e30)
        none = emu.coni_batch_multi(geoms, ps, pgeo, precision=1)
    finally:
        emu.set_gcd_min_tree(0.0)
    assert np.all(rows[4] == 0)
    exp = expected(geoms, ps, pgeo, "oracle")
    assert_same(rows[:4], exp)
    assert_same(none[:4], exp)
    assert rows[5].sum() < none[5].sum()


def test_fp32_bound_check_under_warp_emulator():
    """The FP32 search's bound-check form (an FP64 shadow of its pruning
    quantities, pfg_options.check_fp32) on the emulated device: the FP32
    remaining-norm error is a small part of the FP32 safety margin, no level's
    FP32 range misses part of the FP64 one, and the points equal the FP64
    form's."""
    from emu import emu
    for name, n, dils in (("mixed", 24, None),):
        w = workloads.build(name, n_p=n, dilations=dils)
        geoms, ps, pgeo, _ = layout(w)
        a = emu.coni_batch_multi(geoms, ps, pgeo, precision=3)
        chk = emu.last_fp32_check()
        b = emu.coni_batch_multi(geoms, ps, pgeo, precision=1)
        assert_same(a[:4], b[:4])
        assert chk["narrower"] == 0
        assert 0 < chk["margin_frac"] < 0.5
        assert chk["rem_err"] > 0
