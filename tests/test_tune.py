"""
The autotuner's host logic (pfvs_b200/tune.py) with a fake timing function:
coordinate descent picks the fastest setting along each knob, the result is
stored per (device, batch class) as JSON and reused without timing again,
and the tuning sample keeps every geometry entry of the batch.
"""
import json

import numpy as np

from pfvs_b200 import tune, workloads
from parity import layout


def _fake(best):
    """ms of a setting: smallest at `best`, a penalty per knob away from it."""
    calls = []

    def run(opts):
        calls.append(dict(opts))
        ms = 100.0
        for k, v in best.items():
            ms += 0 if opts[k] == v else 7.0 + abs(float(opts[k]) - float(v)) * 1e-3
        return ms
    return run, calls


def test_search_finds_the_fastest_setting():
    best = {"gcd_min_tree": 3000.0, "warps_per_block": 3, "blocks_per_sm": 2}
    run, calls = _fake(best)
    got, ms, trials = tune.search(run)
    assert got == best and ms == 100.0
    assert len(calls) == len(trials) <= 1 + sum(len(v) for v in (tune.GCD_MIN_TREE, tune.WARPS, tune.BLOCKS))


def test_results_are_stored_and_reused(tmp_path):
    w = workloads.build("mixed", n_p=64)
    geoms, ps, pgeo, _ = layout(w)
    path = str(tmp_path / "tune.json")
    best = {"gcd_min_tree": 300.0, "warps_per_block": 4, "blocks_per_sm": 3}
    run, calls = _fake(best)
    assert tune.autotune(geoms, ps, pgeo, path=path, run=run) == best
    n = len(calls)
    table = json.load(open(path))
    (key,) = table
    assert key.endswith(tune.batch_class(geoms)) and table[key]["options"] == best
    assert table[key]["ms"] < table[key]["default_ms"]
    assert tune.autotune(geoms, ps, pgeo, path=path, run=run) == best      # stored: no timing
    assert len(calls) == n
    tune.autotune(geoms, ps, pgeo, path=path, run=run, retune=True)         # retune: timed again
    assert len(calls) > n


def test_sample_is_stratified_and_batch_class():
    pgeo = np.repeat(np.arange(5), [1000, 10, 3000, 1, 500])
    idx = tune.sample(pgeo, 400)
    assert set(np.unique(pgeo[idx]).tolist()) == {0, 1, 2, 3, 4}
    assert 350 <= len(idx) <= 450 and np.all(np.diff(idx) > 0)
    assert np.array_equal(tune.sample(pgeo[:20], 400), np.arange(20))
    w = workloads.build("mixed", n_p=8)
    geoms, ps, pg, _ = layout(w)
    assert tune.batch_class(geoms) == "h32-d4"
