"""
GPU failure paths, driven from the host without faulting the device:

- a search deadline that runs out marks the directions it cut short with
  status -22 and the call returns; every other direction keeps its points;
- a bound on a warp's wait for work that runs out fails the call with the
  library's error (rc 1, a RuntimeError here) and leaves the context usable;
- a device allocation made to fail (pfg_debug_fail_alloc, the host-side
  hook) inside the batch loop halves the batch and carries on, with the same
  points, as the reference's backend does on cudaErrorMemoryAllocation
  (pfvs/fp_kernel/cuda/pfvs_gpu.cu:729-747); one made to fail before the
  loop (the geometries' buffers) fails the call cleanly.

After each, an ordinary call returns the ordinary result.
"""
import numpy as np
import pytest

from pfvs_b200 import gpu, workloads
from parity import assert_same, layout

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch():
    if not gpu.available():
        pytest.fail("no CUDA device: " + gpu.unavailable_reason())
    w = workloads.build("mixed", n_p=4096)
    geoms, ps, pgeo, _ = layout(w)
    base = gpu.coni_batch_multi_ex(geoms, ps, pgeo)
    assert np.all(base[4] == 0)
    return geoms, ps, pgeo, base


@pytest.fixture(scope="module")
def mixed_depths(batch):
    """The mixed batch (small trees) with 32 directions of plain at dilation
    3200 (trees of about a million nodes) appended, so that a short deadline
    always cuts some directions and spares others."""
    geoms, ps, pgeo, _ = batch
    g2, p2, q2, _ = layout(workloads.build("plain", n_p=32, dilations=(3200.0,)))
    geoms = list(geoms) + list(g2)
    ps = list(ps) + list(p2)
    pgeo = np.concatenate([pgeo, np.asarray(q2) + len(batch[0])]).astype(np.int32)
    base = gpu.coni_batch_multi_ex(geoms, ps, pgeo)
    assert np.all(base[4] == 0)
    return geoms, ps, pgeo, base


def _same_as_base(res, base):
    assert_same(res, base)
    np.testing.assert_array_equal(res[4], base[4])


def test_deadline_marks_cut_directions_and_keeps_the_rest(mixed_depths):
    geoms, ps, pgeo, base = mixed_depths
    r = gpu.coni_batch_multi_ex(geoms, ps, pgeo, deadline_s=1e-6)
    cut = r[4] == -22
    assert cut.any() and not cut.all()
    assert set(np.unique(r[4]).tolist()) <= {0, -22}
    assert_same(r, base, ok_mask=~cut)
    assert not np.isin(r[3], np.flatnonzero(cut)).any()        # no rows of a cut direction
    _same_as_base(gpu.coni_batch_multi_ex(geoms, ps, pgeo), base)


def test_wait_bound_fails_the_call_cleanly(batch):
    geoms, ps, pgeo, base = batch
    try:
        r = gpu.coni_batch_multi_ex(geoms, ps, pgeo, wait_s=1e-6)
    except RuntimeError as e:
        assert "bounded device wait ran out" in str(e)
    else:                           # (no warp had to wait: the ordinary result)
        _same_as_base(r, base)
    _same_as_base(gpu.coni_batch_multi_ex(geoms, ps, pgeo), base)


@pytest.mark.parametrize("k", [4, 9, 16, 25])
def test_out_of_memory_in_the_batch_loop_halves_the_batch(batch, k):
    geoms, ps, pgeo, base = batch
    gpu.release(0)                  # (so that the call allocates again)
    gpu.debug_fail_alloc(k)
    try:
        r = gpu.coni_batch_multi_ex(geoms, ps, pgeo)
    finally:
        gpu.debug_fail_alloc(0)
    assert r[6]["batch_retries"] >= 1
    _same_as_base(r, base)


def test_out_of_memory_before_the_batch_loop_fails_cleanly(batch):
    geoms, ps, pgeo, base = batch
    gpu.release(0)
    gpu.debug_fail_alloc(1)         # the geometries' buffer
    try:
        with pytest.raises(RuntimeError, match="out of memory"):
            gpu.coni_batch_multi_ex(geoms, ps, pgeo)
    finally:
        gpu.debug_fail_alloc(0)
    _same_as_base(gpu.coni_batch_multi_ex(geoms, ps, pgeo), base)
