"""
Benchmark of the batched coniZpM search on B200 (one JSON line on rank 0).

Workload: the "mixed" synthetic batch -- 4 Calabi-Yau geometries with
h11 in {8, 16, 24, 32} (h21 = 2 h11 + 40), 65,536 p-hat directions with
entries in [1, 10], dilation per direction from {1, 2, 3, 4}
(pfvs_b200/workloads.py).  A step is one pass of the pipeline over the whole
batch: per-direction lattice setup, FP32-pruned search (FP64 retry on -11)
and the canonical output, in one multi-geometry call.

Metric: lattice nodes/s.  A node is one search-tree node entered; the work
unit of the batch is the node count of its FP64-pruned tree (counted once,
untimed), so FP32's extra nodes are not counted.  PFVs/s is reported beside
it (points -> (K, M) PFVs by the exact post-processing).

- value: device time of the K timed steps (CUDA events on the launching
  stream inside the library, inputs resident), nodes / time.
- e2e:  the same metric through the public C-ABI entry point pfg_coni_batch
  with host buffers (inputs copied in, points copied out every step),
  wall clock around the K calls.
- cpu_baseline: the reference's own CPU kernel (oracle/_ref, compiled from
  its sources) on a bounded sample of the batch, all host cores.
- --impl reference: that CPU kernel as the timed arm.

Multi-GPU: directions are independent, so each rank takes a contiguous
1/N of the batch (weak scaling: the batch grows with N), no collective on
the data path; timing is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Roofline of the dominant kernel, k_search<double, 1> (the persistent
# FP64-pruned search, about 33 % of the launch list): scalar integer / FP64
# warp code, neither HBM- nor tensor-bound, so its ceiling is the
# warp-instruction issue rate, 148 SMs x 4 schedulers x SM clock.  Per-unit
# figures from one ncu --set full capture of the timed form's search on the
# first 16,384 directions of this batch (20,582,107 nodes): executed warp
# instructions and DRAM bytes per search node.
SEARCH_INST_PER_NODE = 14_977_918_824 / 20_582_107
SEARCH_DRAM_PER_NODE = (248_137_216 + 110_171_648) / 20_582_107
# The setup's three phase kernels (k_setup<32, 0..2>) together, from the
# same kind of capture on the same 16,384 directions: per direction.
SETUP_INST_PER_DIR = (3_785_943_035 + 6_529_456_061 + 1_841_800_499) / 16384
SETUP_DRAM_PER_DIR = (10_734_080 + 253_480_192 + 191_088_384 + 196_837_376 + 215_589_376 + 138_622_720) / 16384
N_SM, SCHEDULERS = 148, 4


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed")
    ap.add_argument("--n", type=int, default=0, help="directions per GPU (0: the workload's size)")
    ap.add_argument("--form", default="batched", choices=["batched", "plain"])
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "fp32"])
    ap.add_argument("--cpu-sample", type=int, default=0, help="directions in the CPU sample (0: auto)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def allmax(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def allsum(pg, x):
    if pg is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


class Clocks:
    """nvidia-smi clock / throttle samples during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.samples, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if len(s) > 3 + k and s[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def workload_slice(name, n_total, rank, world):
    from pfvs_b200 import workloads
    w = workloads.build(name, n_p=n_total)
    per = (len(w) + world - 1) // world
    lo, hi = rank * per, min(len(w), (rank + 1) * per)
    return w, list(range(lo, hi))


def layout(w, idx):
    geoms, ps, pgeo = [], [], []
    groups = {}
    for i in idx:
        groups.setdefault((int(w.pgeo[i]), float(w.dil[i])), []).append(i)
    for k, ((gi, dil), ii) in enumerate(sorted(groups.items())):
        g = w.geoms[gi]
        geoms.append(dict(kappa=g.kappa, Mbasis=g.Mbasis, Q=g.Q, dilation=dil, M0min=13))
        for i in ii:
            ps.append(np.asarray(w.ps[i], dtype=np.int64))
            pgeo.append(k)
    return geoms, ps, np.array(pgeo, dtype=np.int32)


def cpu_reference_run(geoms, ps, pgeo, threads, deadline_s=None):
    """The reference CPU kernel (oracle/_ref) over the given directions, split
    over `threads` host threads (ctypes releases the GIL).  Returns
    (seconds, reference nodes, points, directions done)."""
    from oracle import ref
    jobs = []
    for k, g in enumerate(geoms):
        idx = np.flatnonzero(pgeo == k)
        for c in range(0, len(idx), 16):
            jobs.append((g, [ps[i] for i in idx[c:c + 16]]))
    res = []
    lock = threading.Lock()
    it = iter(jobs)
    t0 = time.perf_counter()

    def worker():
        while True:
            with lock:
                job = next(it, None)
            if job is None or (deadline_s and time.perf_counter() - t0 > deadline_s):
                return
            g, P = job
            M, Kn, q, pidx, st, nodes = ref.coni_batch(g["kappa"], g["Mbasis"], np.array(P), g["Q"],
                                                       g["dilation"], g["M0min"])
            with lock:
                res.append((int(nodes.sum()), len(q), len(P)))
    ths = [threading.Thread(target=worker) for _ in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    dt = time.perf_counter() - t0
    return dt, sum(r[0] for r in res), sum(r[1] for r in res), sum(r[2] for r in res)


def workload_desc(args, w):
    """The config's workload string (the same for both arms)."""
    return (f"{args.workload}: {len(w)} p-hat directions over {len(w.geoms)} geometries "
            f"h11={[g.h11 for g in w.geoms]}, dilations {list(w.info.get('dilations', []))}")


def run_reference(args, world, rank, pg):
    if rank != 0:
        return
    from oracle import ref
    metric = "lattice nodes/s"
    if not ref.available():
        print(json.dumps({"impl": "reference", "metric": metric,
                          "unavailable": "oracle/_ref (the reference CPU kernel) is not built"}))
        return
    w, idx = workload_slice(args.workload, args.n or None, 0, 1)
    threads = os.cpu_count() or 1
    sample = args.cpu_sample or 2048
    rng = np.random.default_rng(1)
    pick = sorted(rng.choice(len(idx), size=min(sample, len(idx)), replace=False).tolist())
    geoms, ps, pgeo = layout(w, [idx[i] for i in pick])
    for _ in range(args.warmup):
        cpu_reference_run(geoms, ps[:64], pgeo[:64], threads)
    times, nodes, pts, dirs = [], 0, 0, 0
    for _ in range(args.steps):
        dt, nn, npt, nd = cpu_reference_run(geoms, ps, pgeo, threads)
        times.append(dt)
        nodes, pts, dirs = nn, npt, nd
    t = float(np.mean(times))
    v = nodes / t
    line = {"impl": "reference", "metric": metric, "value": v, "unit": "nodes/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded)",
            "config": {"workload": workload_desc(args, w),
                       "sample": f"{len(pick)} random directions (seed 1) of the batch per step",
                       "threads": threads},
            "directions_per_s": dirs / t, "points_per_s": pts / t,
            "cpu_baseline": {"value": v, "unit": "nodes/s", "cores": threads, "kind": "reference",
                             "sample": f"{len(pick)} directions of the {args.workload} batch; "
                                       f"the reference's own tree nodes"},
            "e2e": {"value": v, "unit": "nodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    world, rank, local, pg = dist_init()
    if args.impl == "reference":
        run_reference(args, world, rank, pg)
        return
    from pfvs_b200 import build, gpu
    build.build()
    if not gpu.available():
        raise SystemExit("bench: " + gpu.unavailable_reason())
    device = local
    n_total = (args.n * world) if args.n else None
    w, idx = workload_slice(args.workload, n_total, rank, world)
    geoms, ps_list, pgeo = layout(w, idx)
    # the p-vectors as one zero-padded 2-D array, the form the reference's coniZpM passes
    ps = np.zeros((len(ps_list), max((len(p) for p in ps_list), default=1)), dtype=np.int64)
    for i, p in enumerate(ps_list):
        ps[i, :len(p)] = p
    form = gpu.FORM_PLAIN if args.form == "plain" else gpu.FORM_BATCHED
    prec = {"auto": gpu.PREC_AUTO, "fp64": gpu.PREC_FP64, "fp32": gpu.PREC_FP32}[args.precision]

    # work unit: nodes of the FP64-pruned tree with every GCD-cut row built (the
    # reference's pruning), counted once, untimed; the timed steps build the
    # rows only where they pay off, which changes time but not the points
    r64 = gpu.coni_batch_multi_ex(geoms, ps, pgeo, device=device, precision=gpu.PREC_FP64,
                                  gcd_min_tree=-1.0)
    nodes_fp64 = r64[6]["nodes"]
    n_points = len(r64[2])
    for _ in range(args.warmup):
        r = gpu.coni_batch_multi_ex(geoms, ps, pgeo, device=device, form=form, precision=prec)
    # parity guard: the timed form returns the FP64 form's arrays
    for a, b in zip(r[:5], r64[:5]):
        if not np.array_equal(a, b):
            raise SystemExit("bench: timed form differs from the FP64 form")
    # timed steps: device time (CUDA events inside the library)
    barrier(pg)
    with Clocks(device) as clk:
        dev_s, stats = 0.0, None
        t0 = time.perf_counter()
        for _ in range(args.steps):
            r = gpu.coni_batch_multi_ex(geoms, ps, pgeo, device=device, form=form, precision=prec)
            dev_s += r[5]
            stats = r[6]
        wall_s = time.perf_counter() - t0
    barrier(pg)
    dev_s = allmax(pg, dev_s)
    tot_nodes = allsum(pg, nodes_fp64)
    value = tot_nodes * args.steps / dev_s
    # e2e: the public C ABI (pfg_coni_batch) with host buffers, wall clock
    e2e = None
    if not args.no_e2e:
        del r
        out = gpu.coni_batch_multi(geoms, ps, pgeo, device=device)    # (warm-up: pinned output blocks)
        del out
        barrier(pg)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            out = gpu.coni_batch_multi(geoms, ps, pgeo, device=device)
        e2e_s = allmax(pg, time.perf_counter() - t0)
        MH = 64
        h2d = len(ps) * MH * 8 + len(ps) * 4 + sum(np.asarray(g["kappa"]).size * 8 + np.asarray(g["Mbasis"]).size * 8
                                                  for g in geoms) + len(geoms) * 32
        d2h = len(out[2]) * (2 * MH * 8 + 16) + len(ps)
        e2e = {"value": tot_nodes * args.steps / e2e_s, "unit": "nodes/s",
               "h2d_bytes_per_step": int(allsum(pg, h2d)), "d2h_bytes_per_step": int(allsum(pg, d2h)),
               "ms_per_step": e2e_s / args.steps * 1e3}
    # CPU baseline: the reference kernel on a bounded sample (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import ref
        if ref.available():
            threads = os.cpu_count() or 1
            sample = args.cpu_sample or 2048
            rng = np.random.default_rng(1)
            pick = sorted(rng.choice(len(idx), size=min(sample, len(idx)), replace=False).tolist())
            g2, p2, pg2 = layout(w, [idx[i] for i in pick])
            dt, rn, rp, rd = cpu_reference_run(g2, p2, pg2, threads)
            cpu = {"value": rn / dt, "unit": "nodes/s", "cores": threads, "kind": "reference",
                   "sample": f"{len(pick)} random directions (seed 1) of the batch, "
                             f"{dt:.1f} s on {threads} threads; the reference's own tree nodes",
                   "directions_per_s": rd / dt}
    # PFVs: the same batch through the device post-processing (pfg_coni_pfvs), once, untimed
    pfv = None
    if not args.no_e2e:
        Kp, Mp, pp, sp, secs_p, st_p = gpu.coni_pfvs_multi(geoms, ps, pgeo, device=device)
        pfv = {"pfvs_per_step": int(allsum(pg, len(pp))), "points_in": int(allsum(pg, st_p["points"])),
               "device_ms": allmax(pg, secs_p) * 1e3,
               "pfvs_per_s": allsum(pg, len(pp)) / max(allmax(pg, secs_p), 1e-12)}
        del Kp, Mp, pp
    # roofline of the search kernel: executed warp instructions per launch (ncu
    # per-node figure x the launch's nodes) over its CUDA-event time (the
    # search stage: k_flip, a few microseconds, then k_search<double, 1>); the
    # setup's three phase kernels beside it, per direction
    peaks, peaks_kind = measured_peaks()
    clk_sum = clk.summary()
    mhz = clk_sum.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    peak = N_SM * SCHEDULERS * mhz * 1e6
    search_s = stats["ms_search"] / 1e3
    achieved = SEARCH_INST_PER_NODE * stats["nodes"] / search_s
    roofline = {"kernel": "k_search<double, 1>", "bound": "issue", "achieved": achieved, "peak": peak,
                "unit": "warp-inst/s", "frac": achieved / peak,
                "traffic": SEARCH_DRAM_PER_NODE * stats["nodes"],
                "basis": f"ncu: {SEARCH_INST_PER_NODE:.0f} warp-inst and {SEARCH_DRAM_PER_NODE:.1f} DRAM bytes per "
                         f"search node x {stats['nodes']} nodes per launch; peak = {N_SM} SMs x {SCHEDULERS} x "
                         f"{mhz:.0f} MHz (sampled SM clock); HBM for context: {peaks.get('hbm_gbs')} GB/s {peaks_kind}"}
    setup_s = stats["ms_setup"] / 1e3
    setup_ach = SETUP_INST_PER_DIR * len(idx) / setup_s
    roofline_setup = {"kernel": "k_setup<32, 0..2>", "bound": "issue", "achieved": setup_ach, "peak": peak,
                      "unit": "warp-inst/s", "frac": setup_ach / peak,
                      "traffic": SETUP_DRAM_PER_DIR * len(idx),
                      "basis": f"ncu: {SETUP_INST_PER_DIR:.0f} warp-inst and {SETUP_DRAM_PER_DIR:.0f} DRAM bytes "
                               f"per direction over the three phases x {len(idx)} directions"}
    if rank == 0:
        line = {"metric": "lattice nodes/s", "value": value, "unit": "nodes/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": dev_s / args.steps * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "int64+fp32" if args.precision == "fp32" else "int64+fp64",
                "data": "synthetic (seeded CY instances, pfvs_b200/workloads.py)",
                "config": {"workload": workload_desc(args, w),
                           "form": args.form, "precision": args.precision,
                           "directions_per_gpu": len(idx),
                           "l2": "working set per step > 126 MB (slabs + points); no flush needed",
                           "parallelism": f"directions sharded over {world} GPU(s)"},
                "nodes_fp64_per_step": int(tot_nodes), "points_per_step": int(allsum(pg, n_points)),
                "directions_per_s": allsum(pg, len(idx)) * args.steps / dev_s,
                "stage_ms": {"setup": stats["ms_setup"], "search": stats["ms_search"],
                             "output": stats["ms_output"]},
                "timed_form_nodes_per_step": stats["nodes"], "wall_ms_per_step": wall_s / args.steps * 1e3,
                "clocks": clk_sum, "e2e": e2e, "cpu_baseline": cpu, "roofline": roofline, "roofline_setup": roofline_setup, "pfvs": pfv,
                "gpu_launches": int(stats.get("launches", 0)) * args.steps}
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
