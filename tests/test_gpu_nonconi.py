"""
GPU: non-coni ZpM on the device (pfg_zpm_batch through
pfvs_b200.gpu.zpm_batch_multi_ex and pfvs_b200.nonconi.zpm), against the
reference (tests/golden/nonconi.npz: its four non-coni paper vacua and its
non-coni Manwe test geometry, points from its own C setup and kernel):

- the device's lattice points of every p-vector equal the reference's, in
  the canonical order, with FP64 and with FP32 pruning, all cases in one
  multi-geometry call;
- the PFVs through the product's post-processing equal the reference
  route's set, and contain each paper vacuum (6.4's mat, beyond the
  search's int32 staging, is read from the slab);
- a larger batch (the Manwe geometry's 11,386 primitive p-vectors of the
  box |p| <= 6, at dilation 3) equals the reference's C code on a sample
  and its points are independent of the search form.
"""
import os

import numpy as np
import pytest

from conftest import ROOT
from oracle import nonconi as onc
from oracle import pvecs, ref
from pfvs_b200 import gpu, nonconi

pytestmark = pytest.mark.gpu

G = np.load(os.path.join(ROOT, "tests", "golden", "nonconi.npz"))
CASES = list(range(int(G["n_cases"][0])))


def _need_gpu():
    if not gpu.available():
        pytest.fail("no CUDA device: " + gpu.unavailable_reason())


def _case(k):
    kappa, Mb, ps = G[f"c{k}_kappa"], G[f"c{k}_Mbasis"], G[f"c{k}_ps"]
    Qmin, Qmax = (int(x) for x in G[f"c{k}_scal"])
    return kappa, Mb, ps, Qmin, Qmax, float(G[f"c{k}_D"][0])


def _rows(M, Kn, q, pidx, h):
    return [(int(i), tuple(int(x) for x in m[:h]), tuple(int(x) for x in y[:h]), int(v))
            for i, m, y, v in zip(pidx, M, Kn, q)]


@pytest.mark.parametrize("precision", [gpu.PREC_FP64, gpu.PREC_FP32])
def test_device_points_equal_reference_all_cases_in_one_call(precision):
    _need_gpu()
    geoms, ps, pgeo, base = [], [], [], []
    for k in CASES:
        kappa, Mb, P, Qmin, Qmax, D = _case(k)
        geoms.append(dict(kappa=kappa, Mbasis=Mb, Q=Qmax, dilation=D))
        base.append(len(ps))
        ps += [p for p in P]
        pgeo += [k] * len(P)
    M, Kn, q, pidx, pstat, _, _ = gpu.zpm_batch_multi_ex(geoms, ps, np.array(pgeo, np.int32), precision=precision)
    for k in CASES:
        kappa = G[f"c{k}_kappa"]
        h = kappa.shape[0]
        n = len(G[f"c{k}_ps"])
        mine = (pidx >= base[k]) & (pidx < base[k] + n)
        assert np.all(pstat[base[k]:base[k] + n] == 0)
        got = _rows(M[mine], Kn[mine], q[mine], pidx[mine] - base[k], h)
        want = _rows(G[f"c{k}_M"], G[f"c{k}_Kn"], G[f"c{k}_q"], G[f"c{k}_pidx"], h)
        assert got == want and len(want) > 0, k


@pytest.mark.parametrize("k", CASES)
def test_device_pfvs_equal_reference(k):
    _need_gpu()
    kappa, Mb, ps, Qmin, Qmax, D = _case(k)
    Ks, Ms = nonconi.zpm(kappa, Mb, ps, Qmin, Qmax, D)
    got = {(tuple(int(x) for x in a), tuple(int(x) for x in b)) for a, b in zip(Ks, Ms)}
    want = {(tuple(int(x) for x in a), tuple(int(x) for x in b)) for a, b in zip(G[f"c{k}_pfvK"], G[f"c{k}_pfvM"])}
    assert got == want and len(got) == len(Ks) > 0
    if f"c{k}_knownK" in G:
        assert (tuple(int(x) for x in G[f"c{k}_knownK"]), tuple(int(x) for x in G[f"c{k}_knownM"])) in got


def test_larger_batch_equals_reference_sample_and_forms_agree():
    _need_gpu()
    kappa, Mb, _, Qmin, Qmax, _ = _case(4)
    ps = np.array(pvecs.box_enum(6, G["c4_H"]), dtype=np.int64)
    assert len(ps) > 10000
    geoms = [dict(kappa=kappa, Mbasis=Mb, Q=Qmax, dilation=3.0)]
    pg = np.zeros(len(ps), np.int32)
    a = gpu.zpm_batch_multi_ex(geoms, ps, pg)
    b = gpu.zpm_batch_multi_ex(geoms, ps, pg, form=gpu.FORM_PLAIN)
    assert np.all(a[4] == 0) and np.all(b[4] == 0)
    for x, y in zip(a[:4], b[:4]):
        np.testing.assert_array_equal(x, y)
    h = kappa.shape[0]
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(0)
    qmax = onc.qmax_of(Qmax, 3.0)
    for i in np.sort(rng.choice(len(ps), 200, replace=False)):
        st, C, M, Kn, q = onc.ref_points(kappa, Mb, ps[i], Qmax, qmax)
        assert st == 0
        sel = a[3] == i
        got = sorted(_rows(a[0][sel], a[1][sel], a[2][sel], a[3][sel], h))
        want = sorted(_rows(M, Kn, q, np.full(len(q), i), h))
        assert got == want
