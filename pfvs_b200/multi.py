"""
Several GPUs on one batch: the directions are independent, so a batch is cut
into contiguous chunks of directions that the devices pull from one shared
queue (dynamic balancing: the tree sizes differ by more than 1000x, so a
static split by count leaves devices idle); each chunk's points come back in
the canonical order of the chunk, and concatenating the chunks in chunk order
is the canonical order of the batch (grouped by p-vector ascending, (M, Kn)
within one).  No data crosses between devices; only the host gathers.

This is the single-node counterpart of the reference's distributed GPU
workers, which pull work units from a coordinator (pfvs/distributed.py:710-850,
one worker per GPU, :887).

- `LocalQueue`: an in-process chunk counter (threads).
- `StoreQueue`: the same over a torch.distributed key-value store (one
  process per GPU, e.g. under torchrun).
- `run_chunks(queue, n_chunks, fn)`: pull chunks until none is left;
  returns {chunk: fn(chunk)} for the chunks this worker ran.
- `gather_points(parts, offsets)`: the per-chunk (M, Kn, q, pidx, pstat)
  results in batch order, with pidx and pstat in batch indexing.
- `coni_batch_devices(geoms, ps, pgeo, devices, chunk)`: the batched pipeline
  over several devices of this process, one host thread per device (the
  ctypes call releases the GIL).
"""
import threading

import numpy as np


def chunk_bounds(n, chunk):
    """[(lo, hi)] contiguous chunks of n directions, each of at most `chunk`."""
    chunk = max(1, int(chunk))
    return [(lo, min(n, lo + chunk)) for lo in range(0, n, chunk)]


class LocalQueue:
    """Chunk indices 0, 1, 2, ... handed out once each to the threads of this process."""

    def __init__(self):
        self._next = 0
        self._mu = threading.Lock()

    def take(self):
        with self._mu:
            k = self._next
            self._next += 1
            return k


class StoreQueue:
    """Chunk indices handed out once each across processes, through the
    atomic add of a torch.distributed store (every rank uses the same key
    for the same batch; a fresh key per batch)."""

    def __init__(self, store, key):
        self.store, self.key = store, key

    def take(self):
        return int(self.store.add(self.key, 1)) - 1


def run_chunks(queue, n_chunks, fn):
    """Pull chunk indices from `queue` until they run out; {k: fn(k)}."""
    done = {}
    while True:
        k = queue.take()
        if k >= n_chunks:
            return done
        done[k] = fn(k)


def gather_points(parts, bounds):
    """parts: {chunk k: (M, Kn, q, pidx, pstat)} with pidx local to chunk k,
    bounds: chunk_bounds(...).  Returns the batch's (M, Kn, q, pidx, pstat) in
    batch order (every chunk must be present)."""
    ks = sorted(parts)
    if ks != list(range(len(bounds))):
        raise ValueError(f"chunks missing from the gather: have {len(ks)} of {len(bounds)}")
    n = bounds[-1][1] if bounds else 0
    pstat = np.zeros(n, dtype=np.int8)
    Ms, Ks, qs, ps_ = [], [], [], []
    for k in ks:
        M, Kn, q, pidx, st = parts[k][:5]
        lo, hi = bounds[k]
        pstat[lo:hi] = st
        Ms.append(M); Ks.append(Kn); qs.append(q); ps_.append(np.asarray(pidx, dtype=np.int64) + lo)
    MH = Ms[0].shape[1] if Ms else 64
    cat = (lambda xs, shape: np.concatenate(xs) if xs else np.zeros(shape, np.int64))
    return cat(Ms, (0, MH)), cat(Ks, (0, MH)), cat(qs, (0,)), cat(ps_, (0,)), pstat


def _subset(ps, pgeo, lo, hi):
    if isinstance(ps, np.ndarray):
        return ps[lo:hi], pgeo[lo:hi]
    return list(ps[lo:hi]), pgeo[lo:hi]


def coni_batch_devices(geoms, ps, pgeo, devices, chunk=8192):
    """
    `coni_batch_multi` over several GPUs of this process: the directions in
    contiguous chunks of `chunk`, pulled by one host thread per device.
    Returns (M, Kn, q, pidx, pstat, seconds_gpu) as coni_batch_multi, in the
    same order; seconds_gpu is the largest per-device total.
    """
    from . import gpu
    return _batch_devices(lambda g, p, pg, dev: gpu.coni_batch_multi(g, p, pg, device=dev),
                          geoms, ps, pgeo, devices, chunk)


def zpm_batch_devices(geoms, ps, pgeo, devices, chunk=8192, **opts):
    """
    Non-coni ZpM's points (`gpu.zpm_batch_multi_ex`) over several GPUs of
    this process, as `coni_batch_devices`: (M, Kn, q, pidx, pstat,
    seconds_gpu) in the one-call order.
    """
    from . import gpu
    return _batch_devices(lambda g, p, pg, dev: gpu.zpm_batch_multi_ex(g, p, pg, device=dev, **opts)[:6],
                          geoms, ps, pgeo, devices, chunk)


def _batch_devices(call, geoms, ps, pgeo, devices, chunk):
    pgeo = np.ascontiguousarray(pgeo, dtype=np.int32)
    bounds = chunk_bounds(len(pgeo), chunk)
    queue = LocalQueue()
    parts, secs, errors = {}, {}, []
    mu = threading.Lock()

    def worker(dev):
        def one(k):
            lo, hi = bounds[k]
            sub_ps, sub_pgeo = _subset(ps, pgeo, lo, hi)
            M, Kn, q, pidx, pstat, s = call(geoms, sub_ps, sub_pgeo, dev)
            return (M, Kn, q, pidx, pstat), s
        try:
            got = run_chunks(queue, len(bounds), one)
        except Exception as e:          # re-raised in the caller's thread
            with mu:
                errors.append(e)
            return
        with mu:
            for k, (res, s) in got.items():
                parts[k] = res
                secs[dev] = secs.get(dev, 0.0) + s

    threads = [threading.Thread(target=worker, args=(int(d),)) for d in devices]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    if not bounds:
        return call(geoms, ps, pgeo, int(devices[0]))
    return gather_points(parts, bounds) + (max(secs.values()) if secs else 0.0,)
