"""
The device's coniZpK above D0 (pfvs_b200/csrc/pfg_zpk.cuh, k_zpk) run on the
CPU warp emulator (tests/emu), against the reference's own C kernel
(czk_batch, pfvs/fp_kernel/coni_zpk.h:714) through the committed golden
vectors (tests/golden/zpk.npz, made by tests/golden/make_zpk_golden.py):

- on the 30 dataset geometries (h11 3..9), 8 directions each, D0 in
  (20, 150): the same statuses and the same multiset of lattice points
  (pidx, M, Kn, q), although the device's bases of the M-lattice and of
  Lambda are its own (the points do not depend on them);
- the argument and hypothesis failures: D0 < 1 or M0min < 1 (-100, as the
  reference), h11 beyond the kernel (-20), and directions without a bound
  (s > 0 or S not positive definite) status 1, as the reference's C code;
- max_out: a direction with more points than max_out ends with -80 and
  keeps none (the reference's rule);
- D0 = 1, 2, 5 (the most points per direction) on the h11 3..5 geometries
  against the reference's czk_batch run here (where oracle/_ref is built);
- the driver's host logic (pfvs_b200.zpk) with the emulated kernel and the
  oracle's post-processing standing in for the device.
"""
import os

import numpy as np
import pytest

from conftest import ROOT
from emu import emu

Z = np.load(os.path.join(ROOT, "tests", "golden", "zpk.npz"))
D = np.load(os.path.join(ROOT, "tests", "golden", "dataset_pfvs.npz"))
N_GEO = len([k for k in D.files if k.endswith("_kappa")])


def _rows(M, Kn, q, pidx, st):
    ok = st[pidx] == 0 if len(pidx) else np.zeros(0, dtype=bool)
    A = np.hstack([pidx[ok, None], M[ok], Kn[ok], q[ok, None]]).astype(np.int64)
    return A[np.lexsort(A.T[::-1])] if len(A) else A.reshape(0, A.shape[1] if A.ndim == 2 else 0)


def _geo(g):
    h, Q, M0min = (int(x) for x in D[f"g{g}_scal"])
    return D[f"g{g}_kappa"], D[f"g{g}_Mbasis"], Z[f"g{g}_ps"], h, Q, M0min


@pytest.mark.parametrize("D0", [20, 150])
def test_device_zpk_points_equal_the_reference(D0):
    total = 0
    for g in range(N_GEO):
        kappa, Mb, ps, h, Q, M0min = _geo(g)
        M, Kn, q, pidx, st = emu.coni_zpk_batch(kappa, Mb, ps, Q, M0min, D0)
        np.testing.assert_array_equal(st, Z[f"g{g}_d{D0}_status"], err_msg=f"geometry {g}")
        want = Z[f"g{g}_d{D0}_points"]
        got = _rows(M, Kn, q, pidx, st)
        assert got.shape[0] == want.shape[0], (g, D0)
        if len(want):
            np.testing.assert_array_equal(got, want, err_msg=f"geometry {g}")
        total += len(want)
    assert total > (1500 if D0 == 20 else 500)


def test_device_zpk_argument_failures():
    kappa, Mb, ps, h, Q, M0min = _geo(5)
    for D0, m0 in ((0, M0min), (20, 0)):
        M, Kn, q, pidx, st = emu.coni_zpk_batch(kappa, Mb, ps[:2], Q, m0, D0)
        assert list(st) == [-100, -100]
    M, Kn, q, pidx, st = emu.coni_zpk_batch(np.zeros((2, 2, 2), np.int64), np.eye(2, dtype=np.int64),
                                            np.array([[0, 1]]), Q, M0min, 20)
    assert list(st) == [-20]


def test_device_zpk_max_out_drops_the_direction():
    kappa, Mb, ps, h, Q, M0min = _geo(13)
    pts = Z["g13_d20_points"]
    per = np.bincount(pts[:, 0], minlength=len(ps))
    assert per.max() > 3
    M, Kn, q, pidx, st = emu.coni_zpk_batch(kappa, Mb, ps, Q, M0min, 20, max_out=3)
    np.testing.assert_array_equal(st == -80, per > 3)
    kept = _rows(M, Kn, q, pidx, st)
    want = pts[np.isin(pts[:, 0], np.flatnonzero(per <= 3))]
    np.testing.assert_array_equal(kept, want)


def test_device_zpk_no_bound_directions_match_the_reference():
    """Directions whose dilation bound has no value (mu0 status 1: s > 0 or
    S not positive definite on Lambda) have no ZpK either: status 1, as the
    reference's C code says for the same inputs."""
    from oracle import ref
    if not ref.available():
        pytest.skip("the reference's C build (oracle/_ref) is not present")
    G = np.load(os.path.join(ROOT, "tests", "golden", "mu0.npz"))
    done = 0
    for i in range(len(G["r_status"])):
        if int(G["r_status"][i]) != 1 or done >= 6:
            continue
        k = int(G["r_gidx"][i])
        kappa = G[f"kappa{k}"]
        h = kappa.shape[0]
        if h > 20:
            continue
        p = np.concatenate([[0], G["r_p"][i][:h - 1]]).astype(np.int64)[None]
        Mb = np.eye(h, dtype=np.int64)
        _, _, _, _, st_ref = ref.coni_zpk_batch(kappa, Mb, p, 100, 13, 20)
        _, _, _, _, st = emu.coni_zpk_batch(kappa, Mb, p, 100, 13, 20)
        if st_ref[0] in (0, 1):
            assert st[0] == st_ref[0], i
            done += 1
    assert done >= 3


def test_zpk_driver_host_logic(monkeypatch):
    """pfvs_b200.zpk.coni_zpk_multi with the emulated kernel and the oracle's
    post-processing standing in for the device: each geometry's PFVs are the
    reference's coniZpK PFVs (tests/golden/zpk.npz: dilation > D0, once each,
    sorted by p-vector then (M, K)), and a direction the kernel drops (more
    points than max_N_pfvs) goes to coniZpM up to max(its bound, D0)."""
    from oracle import postproc
    from pfvs_b200 import dilation, gpu, zpk
    D0 = 20
    gs = [5, 13, 15, 17]

    def fake_pfvs(kappa, Mbasis, ps, Q, M0min, D0_, max_out=10**9, device=0):
        h = ps.shape[1]
        M, Kn, q, pidx, st = emu.coni_zpk_batch(kappa, Mbasis, ps, Q, M0min, D0_, max_out=max_out)
        ok = st[pidx] == 0
        K1, M1, k1 = postproc.pfvs_from_points(M[ok], Kn[ok], q[ok], pidx[ok], kappa, h, Q, M0min)
        return (np.asarray(K1, np.int64).reshape(-1, h), np.asarray(M1, np.int64).reshape(-1, h),
                np.asarray(k1, np.int64), st, int(ok.sum()), 0.0)

    searched = []

    def fake_bounds(ps, kappa, Q, device=0, return_status=False):
        return np.full(len(ps), 400, np.int64), np.zeros(len(ps), np.int32)

    def fake_zpm(geoms, ps, pgeo, device=0):
        searched.append([g["dilation"] for g in geoms])
        z = np.zeros((0, 64), np.int64)
        return z, z, np.zeros(0, np.int64), np.zeros(len(ps), np.int8), 0.0, {}

    monkeypatch.setattr(gpu, "coni_zpk_pfvs", fake_pfvs)
    monkeypatch.setattr(dilation, "coni_dilation_bound_ceils", fake_bounds)
    monkeypatch.setattr(gpu, "coni_pfvs_multi", fake_zpm)
    items = []
    for g in gs:
        kappa, Mb, ps, h, Q, M0min = _geo(g)
        items.append(dict(kappa=kappa, Mbasis=Mb, ps=ps[:, 1:], Q=Q, M0min=M0min))
    for g, (Ks, Ms, keys) in zip(gs, zpk.coni_zpk_multi(items, D0)):
        h = Ks.shape[1]
        got = np.hstack([keys[:, None], Ms, Ks]) if len(keys) else np.zeros((0, 1 + 2 * h), np.int64)
        np.testing.assert_array_equal(got, Z[f"g{g}_d{D0}_pfvs"], err_msg=f"geometry {g}")
    assert not searched
    # max_N_pfvs = 3: geometry 13's directions with more points go to ZpM at max(bound, D0) = 400
    Ks, Ms, keys, info = zpk.coni_zpk(items[1]["kappa"], items[1]["Mbasis"], items[1]["ps"], items[1]["Q"], D0,
                                      M0min=items[1]["M0min"], max_N_pfvs=3, return_info=True)
    per = np.bincount(Z["g13_d20_points"][:, 0], minlength=len(items[1]["ps"]))
    np.testing.assert_array_equal(info["fallback"], np.flatnonzero(per > 3))
    assert searched == [[400.0]]
    with pytest.raises(ValueError):
        zpk.coni_zpk(items[1]["kappa"], items[1]["Mbasis"], items[1]["ps"], items[1]["Q"], 0)


@pytest.mark.parametrize("D0", [1, 2, 5])
def test_device_zpk_small_D0_against_the_reference_build(D0):
    """Small D0 (the most points per direction) on the h11 3..5 dataset
    geometries, 6 directions each: the emulated kernel against the
    reference's own czk_batch (oracle/_ref) run here."""
    from oracle import ref
    if not ref.available():
        pytest.skip("the reference's C build (oracle/_ref) is not present")
    total = 0
    for g in range(16):
        kappa, Mb, ps, h, Q, M0min = _geo(g)
        ps = ps[:6]
        want = _rows(*ref.coni_zpk_batch(kappa, Mb, ps, Q, M0min, D0))
        st_ref = ref.coni_zpk_batch(kappa, Mb, ps, Q, M0min, D0)[4]
        M, Kn, q, pidx, st = emu.coni_zpk_batch(kappa, Mb, ps, Q, M0min, D0)
        np.testing.assert_array_equal(st, st_ref, err_msg=f"geometry {g}")
        got = _rows(M, Kn, q, pidx, st)
        assert got.shape == want.shape, (g, D0)
        np.testing.assert_array_equal(got, want, err_msg=f"geometry {g}")
        total += len(want)
    assert total > 500
