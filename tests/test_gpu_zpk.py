"""
GPU: coniZpK above D0 on the device (k_zpk through pfg_coni_zpk_batch /
pfg_coni_zpk_pfvs and pfvs_b200.zpk), on the reference's coni dataset
geometries (tests/golden/dataset_pfvs.npz: 30 geometries, h11 3..9) and the
golden vectors of the reference's own C kernel (tests/golden/zpk.npz):

- the lattice points and statuses equal the reference's (czk_batch,
  pfvs/fp_kernel/coni_zpk.h:714) for every geometry, 8 directions each, at
  D0 = 20 and 150;
- the PFVs equal the reference's coniZpK (pfvs/coni.py:554-637: its points,
  the post-processing, dilation > D0);
- ZpK above D0 is exactly the part above D0 of the exhaustive coniZp (the
  reference's tests/test_coni_zpk.py:172-205: every split gives the same
  PFVs), with both on the device;
- a direction the kernel drops (more than max_N_pfvs points) is searched by
  coniZpM to its dilation bound instead, with the same PFVs.
"""
import os

import numpy as np
import pytest

from conftest import ROOT
from pfvs_b200 import coni, gpu, zpk

pytestmark = pytest.mark.gpu

Z = np.load(os.path.join(ROOT, "tests", "golden", "zpk.npz"))
D = np.load(os.path.join(ROOT, "tests", "golden", "dataset_pfvs.npz"))
N_GEO = len([k for k in D.files if k.endswith("_kappa")])


def _need_gpu():
    if not gpu.available():
        pytest.fail("no CUDA device: " + gpu.unavailable_reason())


def _geo(g):
    h, Q, M0min = (int(x) for x in D[f"g{g}_scal"])
    return D[f"g{g}_kappa"], D[f"g{g}_Mbasis"], Z[f"g{g}_ps"], h, Q, M0min


def _sorted(A):
    A = np.asarray(A, dtype=np.int64)
    return A[np.lexsort(A.T[::-1])] if len(A) else A


@pytest.mark.parametrize("D0", [20, 150])
def test_gpu_zpk_points_equal_the_reference(D0):
    _need_gpu()
    total = 0
    for g in range(N_GEO):
        kappa, Mb, ps, h, Q, M0min = _geo(g)
        M, Kn, q, pidx, st, _ = gpu.coni_zpk_points(kappa, Mb, ps, Q, M0min, D0)
        np.testing.assert_array_equal(st, Z[f"g{g}_d{D0}_status"], err_msg=f"geometry {g}")
        want = Z[f"g{g}_d{D0}_points"]
        got = _sorted(np.hstack([pidx[:, None], M, Kn, q[:, None]])) if len(q) else np.zeros((0, want.shape[1]))
        assert got.shape == want.shape, (g, D0)
        np.testing.assert_array_equal(got, want, err_msg=f"geometry {g}")
        total += len(want)
    assert total > (1500 if D0 == 20 else 500)


@pytest.mark.parametrize("D0", [20, 150])
def test_gpu_zpk_pfvs_equal_the_reference(D0):
    _need_gpu()
    total = 0
    for g in range(N_GEO):
        kappa, Mb, ps, h, Q, M0min = _geo(g)
        Ks, Ms, keys, info = zpk.coni_zpk(kappa, Mb, ps[:, 1:], Q, D0, M0min=M0min, return_info=True)
        assert np.all(info["status"] == 0) and len(info["fallback"]) == 0, g
        got = np.hstack([keys[:, None], Ms, Ks]) if len(keys) else np.zeros((0, 1 + 2 * h), np.int64)
        want = Z[f"g{g}_d{D0}_pfvs"]
        np.testing.assert_array_equal(got, want, err_msg=f"geometry {g}")
        total += len(want)
    assert total >= (20 if D0 == 20 else 5)


def test_gpu_zpk_is_the_part_of_conizp_above_D0():
    _need_gpu()
    D0, checked = 20, 0
    for g in range(N_GEO):
        kappa, Mb, ps, h, Q, M0min = _geo(g)
        Ks, Ms, complete, info = coni.coni_zp(kappa, Mb, ps[:, 1:], Q, M0min=M0min, return_info=True)
        assert complete.all(), g
        keys = info["keys"]
        num, den = zpk.dilations(kappa, ps, Ks, Ms, keys)
        above = np.array([int(a) > D0 * int(b) for a, b in zip(num, den)], dtype=bool)
        want = np.hstack([keys[above, None], Ms[above], Ks[above]]) if above.any() else np.zeros((0, 1 + 2 * h))
        K2, M2, k2 = zpk.coni_zpk(kappa, Mb, ps[:, 1:], Q, D0, M0min=M0min)
        got = np.hstack([k2[:, None], M2, K2]) if len(k2) else np.zeros((0, 1 + 2 * h))
        np.testing.assert_array_equal(got, want, err_msg=f"geometry {g}")
        checked += len(want)
    assert checked >= 20


def test_gpu_zpk_fallback_to_zpm_at_the_bound():
    _need_gpu()
    kappa, Mb, ps, h, Q, M0min = _geo(13)
    D0 = 20
    Ks, Ms, keys, info = zpk.coni_zpk(kappa, Mb, ps[:, 1:], Q, D0, M0min=M0min, max_N_pfvs=3, return_info=True)
    per = np.bincount(Z["g13_d20_points"][:, 0], minlength=len(ps))
    np.testing.assert_array_equal(info["status"] == -80, per > 3)
    assert len(info["fallback"]) == int(np.sum(per > 3)) > 0
    got = np.hstack([keys[:, None], Ms, Ks])
    np.testing.assert_array_equal(got, Z["g13_d20_pfvs"])


def test_gpu_zpk_multi_equals_the_reference():
    """coni_zpk_multi over the 30 geometries returns, per geometry, the
    reference's coniZpK PFVs, and every direction is decided by the kernel."""
    _need_gpu()
    D0 = 20
    items, hs = [], []
    for g in range(N_GEO):
        kappa, Mb, ps, h, Q, M0min = _geo(g)
        items.append(dict(kappa=kappa, Mbasis=Mb, ps=ps[:, 1:], Q=Q, M0min=M0min))
        hs.append(h)
    res = zpk.coni_zpk_multi(items, D0, return_info=True)
    for g, (Ks, Ms, keys, info) in enumerate(res):
        assert np.all(info["status"] == 0), g
        got = np.hstack([keys[:, None], Ms, Ks]) if len(keys) else np.zeros((0, 1 + 2 * hs[g]), np.int64)
        np.testing.assert_array_equal(got, Z[f"g{g}_d{D0}_pfvs"], err_msg=f"geometry {g}")
