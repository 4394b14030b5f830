"""
GPU: lattice points -> coni PFVs on the device (pfg_coni_pfvs), on the
reference's own coni dataset geometries (tests/golden/dataset_pfvs.npz, made
by tests/golden/make_dataset_golden.py from the reference's fixtures): 30
geometries with h11 3..9 and their p-vectors in one multi-geometry call.

- The PFVs equal, row for row and in order, the oracle's restatement of
  coniZpM's post-processing (pfvs/coni.py:275-412) applied to the same
  points (pfg_coni_batch's);
- the primitive ones (gcd(K[1:]) = 1) are exactly the published PFV set of
  each geometry (the rule of the reference's tests/test_dataset.py:59-86).
"""
import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import postproc
from pfvs_b200 import gpu

pytestmark = pytest.mark.gpu


def _dataset():
    G = np.load(os.path.join(ROOT, "tests", "golden", "dataset_pfvs.npz"))
    geoms, ps, pgeo, pub = [], [], [], []
    for k in range(int(G["n_geometries"][0])):
        h, Q, m0 = (int(x) for x in G[f"g{k}_scal"])
        geoms.append(dict(kappa=G[f"g{k}_kappa"], Mbasis=G[f"g{k}_Mbasis"], Q=Q,
                          dilation=float(G[f"g{k}_D"][0]), M0min=m0))
        for p in G[f"g{k}_ps"]:
            ps.append(np.asarray(p, dtype=np.int64))
            pgeo.append(k)
        pub.append({(tuple(a), tuple(b)) for a, b in zip(G[f"g{k}_K"].tolist(), G[f"g{k}_M"].tolist())})
    return geoms, ps, np.array(pgeo, dtype=np.int32), pub


def test_device_pfvs_match_reference_postprocessing_and_dataset():
    if not gpu.available():
        pytest.fail("no CUDA device: " + gpu.unavailable_reason())
    geoms, ps, pgeo, pub = _dataset()
    K, M, pidx, pstat, secs, stats = gpu.coni_pfvs_multi(geoms, ps, pgeo)
    assert np.all(pstat == 0)
    Mp, Kp, qp, pp, pst, _ = gpu.coni_batch_multi(geoms, ps, pgeo)
    assert stats["points"] == len(qp)
    total = 0
    for k, g in enumerate(geoms):
        h = np.asarray(g["kappa"]).shape[0]
        selp = pgeo[pp] == k if len(pp) else np.zeros(0, bool)
        eK, eM, ek = postproc.pfvs_from_points(Mp[selp][:, :h], Kp[selp][:, :h], qp[selp], pp[selp],
                                               g["kappa"], h, g["Q"], g["M0min"])
        sel = pgeo[pidx] == k if len(pidx) else np.zeros(0, bool)
        np.testing.assert_array_equal(pidx[sel], ek)
        np.testing.assert_array_equal(K[sel][:, :h], np.asarray(eK, dtype=np.int64).reshape(-1, h))
        np.testing.assert_array_equal(M[sel][:, :h], np.asarray(eM, dtype=np.int64).reshape(-1, h))
        assert not K[sel][:, h:].any() and not M[sel][:, h:].any()
        got = {(tuple(int(x) for x in a[:h]), tuple(int(x) for x in b[:h])) for a, b in zip(K[sel], M[sel])}
        prim = {km for km in got if np.gcd.reduce(np.abs(np.array(km[0][1:]))) == 1}
        assert prim == pub[k], k
        total += int(sel.sum())
    assert total >= sum(len(s) for s in pub) > 300
