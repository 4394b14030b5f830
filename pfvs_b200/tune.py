"""
Autotuner for the batched search's runtime knobs, persisted as JSON.

The knobs (pfg_options): the persistent search grid -- blocks per SM and
warps per block -- and `gcd_min_tree`, the estimated tree size from which a
direction gets GCD-cut rows (they cost setup time and save search time).
These stand in for the reference's fixed compile-time choices of subtree
split depth, block size and warp cooperation (PFG_SD, PFG_EXP_BLOCK,
PFG_COOP, pfvs/fp_kernel/cuda/pfvs_gpu.cu:323-331,494-497): here subtrees
are split dynamically by donation, so the grid and the row policy are what
is left to choose.  None of them changes the points (only time and node
counts), so a tuned call returns the same arrays as an untuned one.

The tuner times candidate settings on the batch itself, or on a stratified
sample of it (the library's own device time of setup + search, best of
`reps`); a sample much smaller than the batch can mislead it (on 8,192 of the
mixed batch's 65,536 directions it preferred a smaller grid that ran the full
batch's search 38 % slower), so the default is the whole batch, by
coordinate descent: the row policy first, then the block shape, then the
grid.  Results are kept per (device name, batch class) in a JSON file
(default ~/.cache/pfvs_b200/tune.json, or PFVS_B200_TUNE), where the batch
class is the largest h11 (which selects the kernel instantiation and the
staging size) and the largest dilation (which sets the tree sizes).

    opts = tune.autotune(geoms, ps, pgeo)        # tunes, or reuses a stored result
    gpu.coni_batch_multi_ex(geoms, ps, pgeo, **opts)
"""
import json
import math
import os

import numpy as np

GCD_MIN_TREE = (300.0, 1000.0, 3000.0, 10000.0)   # 1000: the library default
WARPS = (2, 3, 4)                                   # at most 4 (the search kernels' launch bounds)
BLOCKS = (0, 1, 2, 3, 4)                            # 0: as many as fit (the occupancy API)
KNOBS = ("gcd_min_tree", "warps_per_block", "blocks_per_sm")
DEFAULTS = {"gcd_min_tree": 0.0, "warps_per_block": 0, "blocks_per_sm": 0}


def store_path():
    return os.environ.get("PFVS_B200_TUNE") or os.path.join(
        os.path.expanduser("~"), ".cache", "pfvs_b200", "tune.json")


def batch_class(geoms):
    """The key of a batch: largest h11 and largest dilation (rounded up to a power of 2)."""
    hmax = max(int(np.asarray(g["kappa"]).shape[0]) for g in geoms)
    dmax = max(float(g["dilation"]) for g in geoms)
    return f"h{hmax}-d{2 ** math.ceil(math.log2(max(dmax, 1.0))):g}"


def load(path=None):
    try:
        with open(path or store_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save(table, path=None):
    path = path or store_path()
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def sample(pgeo, n, seed=0):
    """Up to n direction indices, stratified over the geometry entries."""
    pgeo = np.asarray(pgeo)
    if len(pgeo) <= n:
        return np.arange(len(pgeo))
    rng = np.random.default_rng(seed)
    out = []
    for k in np.unique(pgeo):
        idx = np.flatnonzero(pgeo == k)
        take = max(1, int(round(n * len(idx) / len(pgeo))))
        out.append(np.sort(rng.choice(idx, size=min(take, len(idx)), replace=False)))
    return np.sort(np.concatenate(out))


def _device_time(geoms, ps, pgeo, device, reps):
    """The library's device time (setup + search) of one setting, best of reps."""
    from . import gpu

    def run(opts):
        best = math.inf
        for _ in range(reps):
            st = gpu.coni_batch_multi_ex(geoms, ps, pgeo, device=device, **opts)[6]
            best = min(best, st["ms_setup"] + st["ms_search"])
        return best
    return run


def search(run, candidates=None):
    """Coordinate descent over the knobs with `run(opts) -> ms` (lower is
    better).  Returns (best options, best ms, {setting: ms} of every trial)."""
    cand = candidates or {"gcd_min_tree": GCD_MIN_TREE, "warps_per_block": WARPS, "blocks_per_sm": BLOCKS}
    best = dict(DEFAULTS)
    trials = {}

    def timed(opts):
        key = json.dumps(opts, sort_keys=True)
        if key not in trials:
            trials[key] = float(run(dict(opts)))
        return trials[key]
    best_ms = timed(best)
    for knob in KNOBS:
        for v in cand[knob]:
            trial = dict(best, **{knob: v})
            ms = timed(trial)
            if ms < best_ms:
                best, best_ms = trial, ms
    return best, best_ms, trials


def autotune(geoms, ps, pgeo, device=0, n_sample=None, reps=2, path=None, retune=False, run=None):
    """
    Options for coni_batch_multi_ex tuned for this batch's class on this
    device: a stored result when there is one (unless retune), else a
    coordinate-descent search on the batch (or a stratified sample of
    n_sample directions), stored.
    `run` (opts -> ms) replaces the device timing (tests).
    """
    key_dev = "cpu"
    if run is None:
        try:
            import torch
            key_dev = torch.cuda.get_device_name(device).replace(" ", "_")
        except Exception:
            key_dev = f"device{device}"
    key = f"{key_dev}|{batch_class(geoms)}"
    table = load(path)
    if key in table and not retune:
        return dict(table[key]["options"])
    if run is None:
        from . import gpu
        idx = sample(pgeo, n_sample or len(pgeo))
        sps = ps[idx] if isinstance(ps, np.ndarray) else [ps[i] for i in idx]
        spgeo = np.asarray(pgeo)[idx]
        gpu.coni_batch_multi_ex(geoms, sps, spgeo, device=device)      # (warm: buffers, module)
        run = _device_time(geoms, sps, spgeo, device, reps)
    best, best_ms, trials = search(run)
    table[key] = {"options": best, "ms": best_ms, "default_ms": trials[json.dumps(DEFAULTS, sort_keys=True)],
                  "trials": len(trials)}
    save(table, path)
    return dict(best)
