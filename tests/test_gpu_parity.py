"""
GPU parity of the batched coniZpM pipeline: the B200 library's points
(M, Kn, q, pidx, in the canonical order) equal the oracle's -- this
repository's CPU restatement -- and the reference's own CPU kernel
(oracle/_ref) element for element, on seeded synthetic workloads, in both
search forms and both pruning precisions (as the reference's
tests/test_gpu.py:51-81 compares its GPU and CPU arrays).
"""
import numpy as np
import pytest

from pfvs_b200 import gpu, workloads
from parity import assert_same, expected, layout

pytestmark = pytest.mark.gpu

CASES = [
    ("small", 256, None),
    ("small", 128, (150.0,)),
    ("small", 64, (800.0,)),
    ("plain", 256, None),
    ("plain", 96, (150.0,)),
    ("mixed", 256, None),
    ("precision", 24, None),
    ("large", 6, None),
]


@pytest.fixture(scope="module", autouse=True)
def _built(lib):
    if not gpu.available():
        pytest.fail("no CUDA device: " + gpu.unavailable_reason())


def _ids(c):
    return f"{c[0]}-{c[1]}-dil{'x'.join(str(int(d)) for d in c[2]) if c[2] else 'cfg'}"


@pytest.mark.parametrize("case", CASES, ids=[_ids(c) for c in CASES])
def test_batched_matches_oracle(case):
    name, n, dils = case
    w = workloads.build(name, n_p=n, dilations=dils)
    geoms, ps, pgeo, hs = layout(w)
    got = gpu.coni_batch_multi(geoms, ps, pgeo)
    M, Kn, q, pidx, pstat, _ = got
    assert np.all(pstat == 0), np.unique(pstat)
    exp = expected(geoms, ps, pgeo, "oracle")
    assert_same(got, exp)


@pytest.mark.parametrize("case", CASES, ids=[_ids(c) for c in CASES])
def test_batched_matches_reference_build(case, ref_available, record_property):
    if not ref_available:
        pytest.skip("oracle/_ref not built")
    name, n, dils = case
    w = workloads.build(name, n_p=n, dilations=dils)
    geoms, ps, pgeo, hs = layout(w)
    got = gpu.coni_batch_multi(geoms, ps, pgeo)
    exp = expected(geoms, ps, pgeo, "ref")
    ok = exp[4] == 0            # (directions the reference's C path finished)
    record_property("finished_by_reference_build", float(ok.mean()))
    print(f"{_ids(case)}: reference build finished {ok.mean():.4f} of {len(ok)} directions")
    assert ok.mean() >= 0.9
    assert_same(got, exp, ok_mask=ok)


@pytest.mark.parametrize("case", [CASES[2], CASES[4], CASES[5]], ids=_ids)
def test_forms_and_precisions_agree(case):
    name, n, dils = case
    w = workloads.build(name, n_p=n, dilations=dils)
    geoms, ps, pgeo, hs = layout(w)
    a = gpu.coni_batch_multi_ex(geoms, ps, pgeo, precision=gpu.PREC_FP32)
    b = gpu.coni_batch_multi_ex(geoms, ps, pgeo, precision=gpu.PREC_FP64)
    c = gpu.coni_batch_multi_ex(geoms, ps, pgeo, form=gpu.FORM_PLAIN, precision=gpu.PREC_FP64)
    for x in (b, c):
        assert_same(x, a)
        np.testing.assert_array_equal(x[4], a[4])
    assert a[6]["nodes"] > 0


def test_repeat_calls_identical():
    w = workloads.build("mixed", n_p=128)
    geoms, ps, pgeo, _ = layout(w)
    a = gpu.coni_batch_multi(geoms, ps, pgeo)
    b = gpu.coni_batch_multi(geoms, ps, pgeo)
    assert_same(b, a)


def test_gcd_row_policy_keeps_points():
    """GCD-cut rows only prune: building them for every direction (the
    reference's pruning), for the large trees only (the default), or for none
    gives the same points; only the node counts differ."""
    w = workloads.build("mixed", n_p=4096)
    geoms, ps, pgeo, _ = layout(w)
    always = gpu.coni_batch_multi_ex(geoms, ps, pgeo, gcd_min_tree=-1.0)
    default = gpu.coni_batch_multi_ex(geoms, ps, pgeo)
    never = gpu.coni_batch_multi_ex(geoms, ps, pgeo, gcd_min_tree=1e30)
    for x in (default, never):
        assert_same(x, always)
        np.testing.assert_array_equal(x[4], always[4])
    assert always[6]["nodes"] <= default[6]["nodes"] <= never[6]["nodes"]
    assert always[6]["nodes"] < never[6]["nodes"]


def _is_canonical(M, Kn, pidx):
    """rows strictly increasing in (pidx, M, Kn) lexicographic order"""
    keys = np.concatenate([pidx[:, None], M, Kn], axis=1)
    a, b = keys[:-1], keys[1:]
    diff = a != b
    first = np.argmax(diff, axis=1)
    rows = np.arange(len(a))
    return bool(np.all(diff.any(axis=1)) and np.all(a[rows, first] < b[rows, first]))


def test_output_canonical_on_a_large_batch():
    """Size-independent check at a size the oracle cannot follow: 16,384
    directions of the mixed batch, including directions with more points
    than the shared-memory sort holds (the global-memory sort path); the
    rows come out in the canonical order and equal the plain form's."""
    w = workloads.build("mixed", n_p=16384)
    geoms, ps, pgeo, _ = layout(w)
    a = gpu.coni_batch_multi_ex(geoms, ps, pgeo)
    M, Kn, q, pidx = a[:4]
    counts = np.bincount(pidx, minlength=len(ps))
    assert counts.max() > 2048
    assert _is_canonical(M, Kn, pidx)
    b = gpu.coni_batch_multi_ex(geoms, ps, pgeo, precision=gpu.PREC_FP64)
    assert_same(b, a)


def test_batch_splits_give_identical_rows():
    """The rows do not depend on how the directions are split into batches:
    one batch (explicit and default) and six batches (both device output
    slots reused, each batch's rows copied out while the next computes)."""
    w = workloads.build("mixed", n_p=16384)
    geoms, ps, pgeo, _ = layout(w)
    one = gpu.coni_batch_multi_ex(geoms, ps, pgeo, batch=len(ps))
    for b in (0, 3000):
        x = gpu.coni_batch_multi_ex(geoms, ps, pgeo, batch=b)
        assert_same(x, one)
        np.testing.assert_array_equal(x[4], one[4])
        assert x[6]["nodes"] == one[6]["nodes"]


@pytest.mark.parametrize("name,n", [("mixed", 4096), ("precision", 64)])
def test_compact_rows_equal_the_padded_rows(name, n):
    """compact_rows: M and Kn rows as wide as the call's largest h11; the
    entries equal the leading columns of the reference-layout rows (whose
    other columns are zero)."""
    w = workloads.build(name, n_p=n)
    geoms, ps, pgeo, hs = layout(w)
    full = gpu.coni_batch_multi_ex(geoms, ps, pgeo)
    comp = gpu.coni_batch_multi_ex(geoms, ps, pgeo, compact_rows=True)
    width = max(hs)
    assert comp[0].shape[1] == width and comp[1].shape[1] == width
    np.testing.assert_array_equal(comp[0], full[0][:, :width])
    np.testing.assert_array_equal(comp[1], full[1][:, :width])
    assert not full[0][:, width:].any() and not full[1][:, width:].any()
    for a, b in zip(comp[2:5], full[2:5]):
        np.testing.assert_array_equal(a, b)
