"""
GPU: the autotuner on a sample of the mixed batch picks valid options, stores
them, and a call with the tuned options returns the default call's arrays
(the knobs change time only).
"""
import numpy as np
import pytest

from pfvs_b200 import gpu, tune, workloads
from parity import assert_same, layout

pytestmark = pytest.mark.gpu


def test_autotune_keeps_the_points(tmp_path):
    if not gpu.available():
        pytest.fail("no CUDA device: " + gpu.unavailable_reason())
    w = workloads.build("mixed", n_p=4096)
    geoms, ps, pgeo, _ = layout(w)
    path = str(tmp_path / "tune.json")
    opts = tune.autotune(geoms, ps, pgeo, n_sample=2048, reps=1, path=path)
    assert set(opts) == set(tune.KNOBS)
    assert tune.load(path)
    a = gpu.coni_batch_multi_ex(geoms, ps, pgeo, **opts)
    b = gpu.coni_batch_multi_ex(geoms, ps, pgeo)
    assert_same(a, b)
    np.testing.assert_array_equal(a[4], b[4])
