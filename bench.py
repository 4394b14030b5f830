"""
Benchmark of the batched coniZpM search on B200 (one JSON line on rank 0).

Workload: the "mixed" synthetic batch -- 4 Calabi-Yau geometries with
h11 in {8, 16, 24, 32} (h21 = 2 h11 + 40), 65,536 p-hat directions with
entries in [1, 10], dilation per direction from {1, 2, 3, 4}
(pfvs_b200/workloads.py).  A step is one pass of the pipeline over the whole
batch: per-direction lattice setup, the persistent search with the library's
default pruning (FP64 on B200; --precision fp32 gives the FP32-pruned form
with its FP64 retry on -11) and the canonical output, in one
multi-geometry call.

Metric: lattice nodes/s.  A node is one search-tree node entered; the work
unit of the batch is the node count of its FP64-pruned tree (counted once,
untimed), so FP32's extra nodes are not counted.  Directions/s and points/s
are printed beside it in both arms (units the reference counts the same way).

- value: device time of the K timed steps (CUDA events on the launching
  stream inside the library, inputs resident), nodes / time.
- e2e:  the same metric through the library's public entry point
  (pfvs_b200.gpu.coni_batch_multi -> the C ABI) with host buffers (inputs
  copied in, points copied out every step), wall clock around the K calls.
- failed_directions: directions the device did not finish, by status
  (none on the benchmark's workloads).
- cpu_baseline: the reference's own CPU kernel (oracle/_ref, compiled from
  its sources) over the whole batch once, on all host threads.
- --impl reference: that CPU kernel as the timed arm: the K steps cover the
  batch exactly once (step k takes the k-th of K disjoint slices), so the
  arm times the same directions as this one.
- plain / fp32 forms and PFVs/s: see `extras` below.

Multi-GPU: directions are independent.  The batch has N x 65,536
directions (weak scaling), cut into contiguous chunks that the ranks pull
from one shared queue (the process group's store: dynamic balancing, as the
tree sizes differ by more than 1000x); no collective on the data path, the
chunks' points concatenate in p order; timing is the max over ranks.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Roofline of the dominant kernel, k_search<double, 1> (the persistent
# FP64-pruned search, about 40 % of a timed call in the launch list): scalar integer / FP64
# warp code, neither HBM- nor tensor-bound, so its ceiling is the
# warp-instruction issue rate, 148 SMs x 4 schedulers x SM clock.  Per-unit
# figures from one ncu --set full capture of the timed form's search on the
# first 16,384 directions of this batch (20,582,108 nodes): executed warp
# instructions and DRAM bytes per search node.
SEARCH_INST_PER_NODE = 14_639_379_767 / 20_582_108
SEARCH_DRAM_PER_NODE = (246_358_784 + 109_123_072) / 20_582_108
# The setup's four phase kernels (k_setup<32, 0..3>) together, from the
# same capture on the same 16,384 directions: per direction.
SETUP_INST_PER_DIR = (3_554_488_661 + 5_946_675_448 + 255_177_793 + 1_180_743_953) / 16384
SETUP_DRAM_PER_DIR = (111_877_632 + 256_222_208 + 224_210_176 + 14_457_088
                      + 390_921_472 + 315_255_040 + 139_578_880 + 386_816) / 16384
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
    ap.add_argument("--cpu-sample", type=int, default=0, help="directions in the CPU baseline (0: the whole batch)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the forms and PFV figures")
    ap.add_argument("--no-tune", action="store_true", help="the library's default grid and row policy")
    ap.add_argument("--chunk", type=int, default=8192, help="directions per queue chunk (N > 1)")
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


def workload_for(name, n_per_gpu, world):
    """The benchmark batch: n_per_gpu directions (0: the workload's own size)
    for each of the `world` GPUs (weak scaling), the same on every rank."""
    from pfvs_b200 import workloads
    n = (n_per_gpu or workloads.SPECS[name][1]) * world
    return workloads.build(name, n_p=n)


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


def failed_by_status(pstat):
    """{status: directions} of the directions the device did not finish."""
    st, n = np.unique(np.asarray(pstat)[np.asarray(pstat) != 0], return_counts=True)
    return {int(a): int(b) for a, b in zip(st, n)}


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
    w = workload_for(args.workload, args.n, world)
    idx = list(range(len(w)))
    threads = os.cpu_count() or 1
    # the K steps cover the batch once: step k takes every K-th direction from k
    # (each slice has the batch's mix of geometries and dilations)
    K = max(1, args.steps)
    slices = [idx[k::K] for k in range(K)]
    wg, wp, wpg = layout(w, idx[:64])
    for _ in range(args.warmup):
        cpu_reference_run(wg, wp, wpg, threads)
    t_tot, nodes, pts, dirs = 0.0, 0, 0, 0
    for sl in slices:
        geoms, ps, pgeo = layout(w, sl)
        dt, nn, npt, nd = cpu_reference_run(geoms, ps, pgeo, threads)
        t_tot += dt
        nodes += nn
        pts += npt
        dirs += nd
    t = t_tot / K
    v = nodes / t_tot
    line = {"impl": "reference", "metric": metric, "value": v, "unit": "nodes/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64+fp32",
            "data": "synthetic (seeded CY instances, pfvs_b200/workloads.py)",
            "config": {"workload": workload_desc(args, w),
                       "steps_cover": f"the whole batch once: step k of {K} takes directions k, k+{K}, ...",
                       "threads": threads},
            "directions_per_s": dirs / t_tot, "points_per_s": pts / t_tot,
            "reference_nodes": int(nodes), "directions_done": int(dirs), "points": int(pts),
            "cpu_baseline": {"value": v, "unit": "nodes/s", "cores": threads, "kind": "reference",
                             "sample": f"all {len(idx)} directions of the {args.workload} batch once over the "
                                       f"{K} steps; the reference kernel's own tree nodes (its float-pruned "
                                       f"tree on its HNF basis)"},
            "e2e": {"value": v, "unit": "nodes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def padded(ps_list):
    """The p-vectors as one zero-padded 2-D array, the form the reference's coniZpM passes."""
    ps = np.zeros((len(ps_list), max((len(p) for p in ps_list), default=1)), dtype=np.int64)
    for i, p in enumerate(ps_list):
        ps[i, :len(p)] = p
    return ps


def dataset_layout():
    """The reference's own coni dataset geometries (tests/golden/dataset_pfvs.npz:
    30 geometries, h11 3..9, 12,000 p-vectors), the workload on which the
    post-processing produces PFVs."""
    G = np.load(os.path.join(ROOT, "tests", "golden", "dataset_pfvs.npz"))
    geoms, ps, pgeo = [], [], []
    for k in range(int(G["n_geometries"][0])):
        h, Q, m0 = (int(x) for x in G[f"g{k}_scal"])
        geoms.append(dict(kappa=G[f"g{k}_kappa"], Mbasis=G[f"g{k}_Mbasis"], Q=Q,
                          dilation=float(G[f"g{k}_D"][0]), M0min=m0))
        for p in G[f"g{k}_ps"]:
            ps.append(np.asarray(p, dtype=np.int64))
            pgeo.append(k)
    return geoms, ps, np.array(pgeo, dtype=np.int32)


def pfv_rates(gpu, device, threads):
    """PFVs/s on the dataset geometries: the device pipeline with its
    post-processing (pfg_coni_pfvs) against the reference CPU kernel plus the
    oracle's restatement of coniZpM's post-processing (pfvs/coni.py:275-412)."""
    from oracle import postproc, ref
    geoms, ps, pgeo = dataset_layout()
    P = padded(ps)
    gpu.coni_pfvs_multi(geoms, P, pgeo, device=device)                # warm
    reps, dev_s, n_pfv = 5, 0.0, 0
    for _ in range(reps):
        K, M, pidx, pstat, secs, st = gpu.coni_pfvs_multi(geoms, P, pgeo, device=device)
        dev_s += secs
        n_pfv = len(pidx)
    out = {"workload": f"{len(geoms)} reference dataset geometries (h11 3..9), {len(ps)} p-vectors",
           "pfvs": int(n_pfv), "points": int(st["points"]), "device_ms": dev_s / reps * 1e3,
           "pfvs_per_s": n_pfv * reps / dev_s if dev_s > 0 else None}
    if ref.available():
        t0 = time.perf_counter()
        n_cpu = 0
        lock = threading.Lock()

        def one(k):
            nonlocal n_cpu
            g = geoms[k]
            idx = np.flatnonzero(pgeo == k)
            h = np.asarray(g["kappa"]).shape[0]
            M_, Kn_, q_, pl, stt, _ = ref.coni_batch(g["kappa"], g["Mbasis"], np.array([ps[i] for i in idx]),
                                                     g["Q"], g["dilation"], g["M0min"])
            eK, eM, ek = postproc.pfvs_from_points(M_, Kn_, q_, pl, g["kappa"], h, g["Q"], g["M0min"])
            with lock:
                n_cpu += len(ek)
        import concurrent.futures as cf
        with cf.ThreadPoolExecutor(threads) as ex:
            list(ex.map(one, range(len(geoms))))
        dt = time.perf_counter() - t0
        out["cpu_reference"] = {"pfvs": int(n_cpu), "seconds": dt, "pfvs_per_s": n_cpu / dt, "threads": threads,
                                "what": "oracle/_ref kernel + the oracle's restated post-processing"}
    return out


def coni_zp_rates(device, threads):
    """The exhaustive coniZp driver (pfvs_b200.coni.coni_zp_multi: the dilation
    bound of every direction on the device, then coniZpM at each direction's
    grid_up bound with the device post-processing, all geometries' searches in
    one call) on the dataset geometries, against
    the same plan on the host: the reference's C bound (coni_bound.h:255),
    the reference kernel at the same dilations and the oracle's restated
    post-processing, on `threads` threads.  And the bound alone at volume:
    directions/s of k_mu0 against the reference's C bound on a batch of
    the mixed workload's h11 = 8 and 16 directions."""
    import concurrent.futures as cf
    from oracle import postproc, ref
    from pfvs_b200 import coni, dilation, workloads
    G = np.load(os.path.join(ROOT, "tests", "golden", "dataset_pfvs.npz"))
    data = []
    for k in range(int(G["n_geometries"][0])):
        h, Q, m0 = (int(x) for x in G[f"g{k}_scal"])
        data.append(dict(kappa=G[f"g{k}_kappa"], Mbasis=G[f"g{k}_Mbasis"], Q=Q, M0min=m0, ps=G[f"g{k}_ps"][:, 1:]))
    n_dirs = sum(len(g["ps"]) for g in data)

    def device_run():
        # every geometry's bounds, then all their searches in one device call (coni_zp_multi)
        t0 = time.perf_counter()
        res = coni.coni_zp_multi([dict(kappa=g["kappa"], Mbasis=g["Mbasis"], ps=g["ps"], Q=g["Q"], M0min=g["M0min"])
                                  for g in data], device=device, return_info=True)
        n_pfv = sum(len(r[0]) for r in res)
        t_b = res[0][3]["seconds_bound"]
        dil_max = max(int(r[3]["dilation"].max()) for r in res)
        return time.perf_counter() - t0, t_b, n_pfv, dil_max
    device_run()                                                    # (warm)
    runs = [device_run() for _ in range(3)]
    best = min(runs)
    out = {"workload": f"{len(data)} reference dataset geometries (h11 3..9), {n_dirs} p-vectors, every PFV of "
                       f"each direction at any dilation (searched to grid_up(ceil(Q / mu0)), up to {best[3]})",
           "pfvs": int(best[2]), "wall_s": best[0], "bound_wall_s": best[1], "pfvs_per_s": best[2] / best[0],
           "directions_per_s": n_dirs / best[0]}
    if ref.available():
        def host_one(g):
            st, num, den, _ = ref.coni_mu0_batch(g["kappa"], g["ps"])
            bc, fits = dilation._ceil_q_over(g["Q"], num[st == 0], den[st == 0])
            b = np.zeros(len(st), np.int64)
            b[st == 0] = bc
            dil = coni.route(b, 1)
            h = g["kappa"].shape[0]
            P = np.hstack([np.zeros((len(g["ps"]), 1), np.int64), g["ps"]])
            n = 0
            for D in np.unique(dil):
                sel = np.flatnonzero(dil == D)
                M_, Kn_, q_, pl, stt, _ = ref.coni_batch(g["kappa"], g["Mbasis"], P[sel], g["Q"], float(D), g["M0min"])
                eK, eM, ek = postproc.pfvs_from_points(M_, Kn_, q_, pl, g["kappa"], h, g["Q"], g["M0min"])
                n += len(ek)
            return n
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(threads) as ex:
            n_host = sum(ex.map(host_one, sorted(data, key=lambda g: -len(g["ps"]) * g["kappa"].shape[0] ** 3)))
        dt = time.perf_counter() - t0
        out["cpu_reference"] = {"pfvs": int(n_host), "wall_s": dt, "pfvs_per_s": n_host / dt, "threads": threads,
                                "what": "oracle/_ref: the reference's C bound + its kernel at the same dilations "
                                        "+ the oracle's restated post-processing"}
        out["device_vs_cpu_reference"] = dt / best[0]
    # the bound at volume
    w = workloads.build("mixed")
    vol = {}
    for k, g in enumerate(w.geoms):
        if g.h11 not in (8, 16) or f"h11={g.h11}" in vol:
            continue
        P = np.array([w.ps[i][1:] for i in np.flatnonzero(np.asarray(w.pgeo) == k)])
        dilation.coni_mu0_batch(P, g.kappa, device=device)          # (warm: buffers sized for P)
        dt = math.inf
        for _ in range(3):
            t0 = time.perf_counter()
            st, *_ = dilation.coni_mu0_batch(P, g.kappa, device=device)
            dt = min(dt, time.perf_counter() - t0)
        ent = {"directions": int(len(P)), "device_directions_per_s": len(P) / dt,
               "device_decided": float(np.mean(st >= 0))}
        if ref.available():
            t1 = time.perf_counter()
            with cf.ThreadPoolExecutor(threads) as ex:
                parts = list(ex.map(lambda c: ref.coni_mu0_batch(g.kappa, c), np.array_split(P, 4 * threads)))
            dr = time.perf_counter() - t1
            sr = np.concatenate([x[0] for x in parts])
            ent.update({"cpu_reference_directions_per_s": len(P) / dr, "cpu_reference_decided": float(np.mean(sr >= 0)),
                        "threads": threads})
        vol[f"h11={g.h11}"] = ent
    out["bound_at_volume"] = vol
    return out


def zpk_rates(device, threads):
    """coniZpK above D0 (pfg_coni_zpk_batch; the reference runs it on the CPU
    only: coni_zpk.h:714 behind coniZpK) on the dataset geometries' 10,399
    directions at D0 = 20 and 150: the kernel's device time and the whole
    call, points/s and directions/s, and the PFVs through pfvs_b200.zpk; against
    the reference's own C kernel (oracle/_ref) over the same directions on
    `threads` threads."""
    import concurrent.futures as cf
    from oracle import ref
    from pfvs_b200 import gpu, zpk
    G = np.load(os.path.join(ROOT, "tests", "golden", "dataset_pfvs.npz"))
    data = []
    for k in range(int(G["n_geometries"][0])):
        h, Q, m0 = (int(x) for x in G[f"g{k}_scal"])
        data.append((G[f"g{k}_kappa"], G[f"g{k}_Mbasis"], G[f"g{k}_ps"], Q, m0))
    n_dirs = sum(len(g[2]) for g in data)
    out = {"workload": f"{len(data)} reference dataset geometries (h11 3..9), {n_dirs} p-vectors, the points and "
                       f"PFVs of dilation above D0"}
    items = [dict(kappa=g[0], Mbasis=g[1], ps=g[2][:, 1:], Q=g[3], M0min=g[4]) for g in data]
    for D0 in (20, 150):
        for g in data[:2]:
            gpu.coni_zpk_points(g[0], g[1], g[2], g[3], g[4], D0, device=device)     # (warm)
        best = None
        for _ in range(2):
            t0 = time.perf_counter()
            dev = pts = bad = 0
            for g in data:                      # (one device call per geometry, as the reference's czk_batch)
                M, Kn, q, pidx, st, secs = gpu.coni_zpk_points(g[0], g[1], g[2], g[3], g[4], D0, device=device)
                dev += secs
                pts += len(q)
                bad += int(np.sum(st != 0))
            wall = time.perf_counter() - t0
            if best is None or wall < best[0]:
                best = (wall, dev, pts, bad)
        t0 = time.perf_counter()
        n_pfv = sum(len(r[2]) for r in zpk.coni_zpk_multi(items, D0, device=device))
        pfv_wall = time.perf_counter() - t0
        ent = {"points": int(best[2]), "not_decided": int(best[3]), "device_kernel_s": best[1], "wall_s": best[0],
               "directions_per_s": n_dirs / best[0], "pfvs": int(n_pfv), "pfvs_wall_s": pfv_wall,
               "what": "one device call per geometry (pfg_coni_zpk_batch); pfvs through "
                       "pfvs_b200.zpk.coni_zpk_multi (the kernel, the device post-processing, the dilation filter)"}
        if ref.available():
            jobs = [(g, c) for g in data for c in np.array_split(g[2], max(1, min(4 * threads, len(g[2]) // 8)))]
            t1 = time.perf_counter()
            with cf.ThreadPoolExecutor(threads) as ex:
                parts = list(ex.map(lambda j: ref.coni_zpk_batch(j[0][0], j[0][1], j[1], j[0][3], j[0][4], D0),
                                    sorted(jobs, key=lambda j: -len(j[1]) * j[0][0].shape[0] ** 3)))
            dt = time.perf_counter() - t1
            ent["cpu_reference"] = {"points": int(sum(len(x[2]) for x in parts)), "wall_s": dt,
                                    "directions_per_s": n_dirs / dt, "threads": threads,
                                    "what": "oracle/_ref: the reference's czk_batch (ctypes, the GIL released)"}
            ent["device_vs_cpu_reference"] = dt / best[0]
        out[f"D0={D0}"] = ent
    return out


def nonconi_rates(device, threads):
    """Non-coni ZpM (pfg_zpm_batch; the reference runs it on the CPU only) on
    the reference's non-coni Manwe test geometry (tests/golden/nonconi.npz):
    the 11,386 primitive p-vectors of the box |p| <= 6 in its Kahler cone at
    dilation 3, Qmax = h11 + h21 + 2.  Device: setup + search time, nodes/s,
    and PFVs/s through the product's host post-processing; against the
    reference's C setup and kernel (oracle/_ref, composed as nonconi.ZpM
    composes them) on `threads` threads."""
    import concurrent.futures as cf
    from oracle import nonconi as onc
    from oracle import pvecs, ref
    from pfvs_b200 import gpu, nonconi
    G = np.load(os.path.join(ROOT, "tests", "golden", "nonconi.npz"))
    kappa, Mb, H = G["c4_kappa"], G["c4_Mbasis"], G["c4_H"]
    Qmin, Qmax = (int(x) for x in G["c4_scal"])
    ps = np.array(pvecs.box_enum(6, H), dtype=np.int64)
    geoms = [dict(kappa=kappa, Mbasis=Mb, Q=Qmax, dilation=3.0)]
    pg = np.zeros(len(ps), np.int32)
    gpu.zpm_batch_multi_ex(geoms, ps, pg, device=device)            # (warm)
    runs = [gpu.zpm_batch_multi_ex(geoms, ps, pg, device=device) for _ in range(3)]
    r = min(runs, key=lambda x: x[5])
    st = r[6]
    dev_s = (st["ms_setup"] + st["ms_search"] + st["ms_output"]) / 1e3
    t0 = time.perf_counter()
    Ks, Ms = nonconi.zpm(kappa, Mb, ps, Qmin, Qmax, 3.0, device=device)
    wall = time.perf_counter() - t0
    out = {"workload": f"non-coni Manwe geometry (h11 = 8), {len(ps)} p-vectors (box |p| <= 6), dilation 3, "
                       f"Qmax {Qmax}",
           "points": int(len(r[2])), "nodes": int(st["nodes"]), "device_ms": dev_s * 1e3,
           "stage_ms": {"setup": st["ms_setup"], "search": st["ms_search"], "output": st["ms_output"]},
           "nodes_per_s": st["nodes"] / dev_s, "directions_per_s": len(ps) / dev_s,
           "pfvs": int(len(Ks)), "zpm_wall_s": wall, "pfvs_per_s": len(Ks) / wall,
           "failed": int(np.sum(r[4] != 0))}
    if ref.available():
        qmax = onc.qmax_of(Qmax, 3.0)

        def chunk(c):
            n_pts = n_nodes = 0
            for p in c:
                res = onc.ref_points(kappa, Mb, p, Qmax, qmax, return_nodes=True)
                n_pts += len(res[4])
                n_nodes += res[5]
            return n_pts, n_nodes
        t1 = time.perf_counter()
        with cf.ThreadPoolExecutor(threads) as ex:
            parts = list(ex.map(chunk, np.array_split(ps, 8 * threads)))
        dt = time.perf_counter() - t1
        out["cpu_reference"] = {"points": int(sum(x[0] for x in parts)), "nodes": int(sum(x[1] for x in parts)),
                                "seconds": dt, "nodes_per_s": sum(x[1] for x in parts) / dt,
                                "directions_per_s": len(ps) / dt, "threads": threads,
                                "what": "oracle/_ref: the reference's pfl_build (coni = 0) + its kernel per "
                                        "p-vector (ctypes calls, the GIL released)"}
        out["device_vs_cpu_reference_directions"] = out["directions_per_s"] / out["cpu_reference"]["directions_per_s"]
    return out


def main():
    args = parse()
    world, rank, local, pg = dist_init()
    if args.impl == "reference":
        run_reference(args, world, rank, pg)
        return
    from pfvs_b200 import build, gpu, multi
    build.build()
    if not gpu.available():
        raise SystemExit("bench: " + gpu.unavailable_reason())
    device = local
    w = workload_for(args.workload, args.n, world)
    idx = list(range(len(w)))
    geoms, ps_list, pgeo = layout(w, idx)
    ps = padded(ps_list)
    form = gpu.FORM_PLAIN if args.form == "plain" else gpu.FORM_BATCHED
    prec = {"auto": gpu.PREC_AUTO, "fp64": gpu.PREC_FP64, "fp32": gpu.PREC_FP32}[args.precision]
    # one GPU: one call over the whole batch; several: contiguous chunks pulled
    # by the ranks from a shared queue (the process group's store)
    bounds = multi.chunk_bounds(len(ps), len(ps) if world == 1 else args.chunk)
    store = pg.distributed_c10d._get_default_store() if pg is not None else None

    def queue(key):
        return multi.StoreQueue(store, "bench/" + key) if store is not None else multi.LocalQueue()

    def call(k, **kw):
        lo, hi = bounds[k]
        return gpu.coni_batch_multi_ex(geoms, ps[lo:hi], pgeo[lo:hi], device=device, **kw)

    # the search grid and GCD-row policy from the autotuner (tuned on the batch, or
    # read from its JSON store), untimed; they change time only
    tuned = {}
    if not args.no_tune and args.form == "batched":
        from pfvs_b200 import tune
        tuned = tune.autotune(geoms, ps, pgeo, device=device)

    # work unit: nodes of the FP64-pruned tree with every GCD-cut row built (the
    # reference's pruning), counted once, untimed; the timed steps build the
    # rows only where they pay off, which changes time but not the points.
    # Parity guard: the timed form returns the FP64 form's arrays.
    def unit(k):
        r64 = call(k, precision=gpu.PREC_FP64, gcd_min_tree=-1.0)
        r = call(k, form=form, precision=prec, **tuned)
        for a, b in zip(r[:5], r64[:5]):
            if not np.array_equal(a, b):
                raise SystemExit("bench: timed form differs from the FP64 form")
        return r64[6]["nodes"], len(r64[2]), failed_by_status(r64[4]), len(r64[4])
    got = multi.run_chunks(queue("unit"), len(bounds), unit)
    nodes_fp64 = sum(g[0] for g in got.values())
    n_points = sum(g[1] for g in got.values())
    failed = {}
    for g in got.values():
        for k, v in g[2].items():
            failed[k] = failed.get(k, 0) + v
    for s_ in range(args.warmup):
        multi.run_chunks(queue(f"warm{s_}"), len(bounds), lambda k: call(k, form=form, precision=prec, **tuned)[5])
    # timed steps: device time (CUDA events inside the library)
    tot = dict(ms_setup=0.0, ms_search=0.0, ms_output=0.0, nodes=0, launches=0)
    failed_timed = {}
    barrier(pg)
    with Clocks(device) as clk:
        dev_s = 0.0
        t0 = time.perf_counter()
        for s_ in range(args.steps):
            def timed(k):
                r = call(k, form=form, precision=prec, **tuned)
                for key in tot:
                    tot[key] += r[6][key]
                for st_, v in failed_by_status(r[4]).items():
                    failed_timed[st_] = failed_timed.get(st_, 0) + v
                return r[5]
            dev_s += sum(multi.run_chunks(queue(f"step{s_}"), len(bounds), timed).values())
        wall_s = time.perf_counter() - t0
    barrier(pg)
    dev_s = allmax(pg, dev_s)
    tot_nodes = allsum(pg, nodes_fp64)
    value = tot_nodes * args.steps / dev_s
    per_step = {k: v / args.steps for k, v in tot.items()}
    # e2e: the public entry point (coni_batch_multi -> pfg_coni_batch) with host
    # buffers (inputs copied in, rows copied out, every step), wall clock
    e2e = None
    if not args.no_e2e:
        def e2e_call(k):
            lo, hi = bounds[k]
            out = gpu.coni_batch_multi(geoms, ps[lo:hi], pgeo[lo:hi], device=device)
            return len(out[2]), hi - lo
        multi.run_chunks(queue("e2e_warm"), len(bounds), e2e_call)   # (pinned output blocks)
        barrier(pg)
        t0 = time.perf_counter()
        rows = dirs = 0
        for s_ in range(args.steps):
            for nr, nd in multi.run_chunks(queue(f"e2e{s_}"), len(bounds), e2e_call).values():
                rows += nr
                dirs += nd
        e2e_s = allmax(pg, time.perf_counter() - t0)
        MH = 64
        geo_bytes = sum(np.asarray(g["kappa"]).size * 8 + np.asarray(g["Mbasis"]).size * 8 for g in geoms) \
            + len(geoms) * 32
        h2d = dirs * (MH * 8 + 4) / args.steps + geo_bytes
        d2h = rows * (2 * MH * 8 + 16) / args.steps + dirs / args.steps
        e2e = {"value": tot_nodes * args.steps / e2e_s, "unit": "nodes/s",
               "h2d_bytes_per_step": int(allsum(pg, h2d)), "d2h_bytes_per_step": int(allsum(pg, d2h)),
               "ms_per_step": e2e_s / args.steps * 1e3,
               "path": "pfvs_b200.gpu.coni_batch_multi -> pfg_coni_batch (the reference's ABI: 64-wide rows)"}
        # the same through the extension entry point with compact rows (as wide as the
        # call's largest h11): the user-side option for fewer bytes copied back
        wmax = max(int(np.asarray(g["kappa"]).shape[0]) for g in geoms)

        def e2e_compact(k):
            lo, hi = bounds[k]
            out = gpu.coni_batch_multi_ex(geoms, ps[lo:hi], pgeo[lo:hi], device=device, compact_rows=True)
            return len(out[2])
        multi.run_chunks(queue("e2ec_warm"), len(bounds), e2e_compact)
        barrier(pg)
        t0 = time.perf_counter()
        rows_c = 0
        for s_ in range(args.steps):
            rows_c += sum(multi.run_chunks(queue(f"e2ec{s_}"), len(bounds), e2e_compact).values())
        e2ec_s = allmax(pg, time.perf_counter() - t0)
        e2e["compact_rows"] = {"value": tot_nodes * args.steps / e2ec_s, "unit": "nodes/s",
                               "ms_per_step": e2ec_s / args.steps * 1e3, "row_width": wmax,
                               "d2h_bytes_per_step": int(allsum(pg, rows_c * (2 * wmax * 8 + 16) / args.steps
                                                                + dirs / args.steps)),
                               "path": "pfvs_b200.gpu.coni_batch_multi_ex(compact_rows=True) -> pfg_coni_batch_ex"}
    threads = os.cpu_count() or 1
    # CPU baseline: the reference kernel over the whole batch once (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import ref
        if ref.available():
            sel = idx if not args.cpu_sample else idx[::max(1, len(idx) // args.cpu_sample)]
            g2, p2, pg2 = layout(w, sel)
            dt, rn, rp, rd = cpu_reference_run(g2, p2, pg2, threads)
            cpu = {"value": rn / dt, "unit": "nodes/s", "cores": threads, "kind": "reference",
                   "sample": f"{len(sel)} of the batch's {len(idx)} directions, {dt:.1f} s on {threads} "
                             f"threads; the reference kernel's own tree nodes ({rn})",
                   "directions_per_s": rd / dt, "points_per_s": rp / dt}
    # forms (N = 1): the plain form and the FP32-pruned form on the same work unit
    forms = None
    if rank == 0 and world == 1 and not args.no_extras:
        forms = {}
        for name, kw in (("plain", dict(form=gpu.FORM_PLAIN, precision=gpu.PREC_FP64)),
                         ("fp32", dict(precision=gpu.PREC_FP32))):
            call(0, **kw)
            r = call(0, **kw)
            if any(not np.array_equal(a, b) for a, b in zip(r[:4], call(0)[:4])):
                raise SystemExit(f"bench: the {name} form's points differ")
            forms[name] = {"ms_per_step": r[5] * 1e3, "search_ms": r[6]["ms_search"],
                           "nodes_per_s": tot_nodes / r[5], "nodes_entered": r[6]["nodes"],
                           "fp64_retries": r[6]["fp64_retries"]}
        forms["batched_vs_plain"] = {"step": forms["plain"]["ms_per_step"] / (dev_s / args.steps * 1e3),
                                     "search": forms["plain"]["search_ms"] / per_step["ms_search"]}
        forms["batched_fp32_vs_plain"] = {"step": forms["plain"]["ms_per_step"] / forms["fp32"]["ms_per_step"],
                                          "search": forms["plain"]["search_ms"] / forms["fp32"]["search_ms"]}
        # the FP32 pruning bounds against FP64 on this batch (the bound-check form, untimed)
        rc_ = call(0, precision=gpu.PREC_FP32, check_fp32=True)
        forms["fp32_bound_error"] = {k: rc_[6][k] for k in ("fp32_rem_err", "fp32_margin_frac", "fp32_end_err",
                                                            "fp32_narrower")}
        forms["fp32_bound_error"]["what"] = ("max over the FP32 pass of |FP32 - FP64| remaining norm (q units), its "
                                             "fraction of the FP32 test's safety margin, interval endpoints "
                                             "(coordinate units, including the FP32 margin's widening), and levels "
                                             "whose FP32 range misses part of the FP64 one")
    # the reference's own CUDA backend (oracle/_refgpu, its PFL_MAX_H11 = 24 build, in a process
    # of its own) on the batch's h11 <= 24 directions, beside this library on the same directions
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_extras:
        from oracle import refgpu
        keep_g = [k for k, g in enumerate(geoms) if np.asarray(g["kappa"]).shape[0] <= 24]
        if refgpu.available(24) and keep_g:
            remap = {k: i for i, k in enumerate(keep_g)}
            sel = np.flatnonzero(np.isin(pgeo, keep_g))
            g24 = [geoms[k] for k in keep_g]
            p24 = ps[sel]
            pg24 = np.array([remap[int(x)] for x in pgeo[sel]], dtype=np.int32)
            rr = refgpu.coni_batch_multi(g24, list(p24), pg24, max_h11=24, reps=3)
            ours = [gpu.coni_batch_multi_ex(g24, p24, pg24, device=device, **tuned) for _ in range(3)][1:]
            ref_gpu = {"directions": int(len(sel)), "reference_finished": float(np.mean(rr[4] == 0)),
                       "reference_device_ms": rr[5] * 1e3, "reference_wall_ms": rr[6] * 1e3,
                       "ours_device_ms": float(np.mean([o[5] for o in ours])) * 1e3,
                       "what": "pfvs/fp_kernel/cuda/pfvs_gpu.cu built for sm_100a (PFL_MAX_H11 = 24), the same "
                               "directions; it hands the directions it does not finish (pstat 1) to the CPU, "
                               "whose time is not in its figure"}
            ref_gpu["ours_vs_reference_device"] = ref_gpu["reference_device_ms"] / ref_gpu["ours_device_ms"]
    # PFVs: the batch through the device post-processing (pfg_coni_pfvs), once,
    # untimed, and PFVs/s on the reference's dataset geometries (which have PFVs)
    pfv = None
    if not args.no_extras:
        def pfv_chunk(k):
            lo, hi = bounds[k]
            Kp, Mp, pp, sp, secs_p, st_p = gpu.coni_pfvs_multi(geoms, ps[lo:hi], pgeo[lo:hi], device=device)
            return len(pp), st_p["points"], secs_p
        pr = multi.run_chunks(queue("pfv"), len(bounds), pfv_chunk).values()
        pfv = {"pfvs_per_step": int(allsum(pg, sum(x[0] for x in pr))),
               "points_in": int(allsum(pg, sum(x[1] for x in pr))),
               "device_ms": allmax(pg, sum(x[2] for x in pr)) * 1e3}
        if rank == 0 and world == 1:
            pfv["dataset"] = pfv_rates(gpu, device, threads)
            pfv["coni_zp"] = coni_zp_rates(device, threads)
            pfv["nonconi_zpm"] = nonconi_rates(device, threads)
            pfv["coni_zpk"] = zpk_rates(device, threads)
    # roofline of the search kernel: executed warp instructions per launch (ncu
    # per-node figure x the launch's nodes) over its CUDA-event time (the
    # search stage: k_flip, a few microseconds, then k_search<double, 1>); the
    # setup's three phase kernels beside it, per direction
    peaks, peaks_kind = measured_peaks()
    clk_sum = clk.summary()
    mhz = clk_sum.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    peak = N_SM * SCHEDULERS * mhz * 1e6
    search_s = per_step["ms_search"] / 1e3
    achieved = SEARCH_INST_PER_NODE * per_step["nodes"] / search_s
    roofline = {"kernel": "k_search<double, 1>", "bound": "issue", "achieved": achieved, "peak": peak,
                "unit": "warp-inst/s", "frac": achieved / peak,
                "traffic": SEARCH_DRAM_PER_NODE * per_step["nodes"],
                "basis": f"ncu: {SEARCH_INST_PER_NODE:.0f} warp-inst and {SEARCH_DRAM_PER_NODE:.1f} DRAM bytes per "
                         f"search node x {per_step['nodes']:.0f} nodes per step; peak = {N_SM} SMs x {SCHEDULERS} x "
                         f"{mhz:.0f} MHz (sampled SM clock); HBM for context: {peaks.get('hbm_gbs')} GB/s {peaks_kind}"}
    setup_s = per_step["ms_setup"] / 1e3
    n_here = len(idx) / world
    setup_ach = SETUP_INST_PER_DIR * n_here / setup_s
    roofline_setup = {"kernel": "k_setup<32, 0..3>", "bound": "issue", "achieved": setup_ach, "peak": peak,
                      "unit": "warp-inst/s", "frac": setup_ach / peak,
                      "traffic": SETUP_DRAM_PER_DIR * n_here,
                      "basis": f"ncu: {SETUP_INST_PER_DIR:.0f} warp-inst and {SETUP_DRAM_PER_DIR:.0f} DRAM bytes "
                               f"per direction over the four phases x {n_here:.0f} directions"}
    failed_all = {str(k): int(allsum(pg, v)) for k, v in sorted(failed.items())}
    failed_step = {str(k): allsum(pg, v) / args.steps for k, v in sorted(failed_timed.items())}
    if rank == 0:
        line = {"metric": "lattice nodes/s", "value": value, "unit": "nodes/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": dev_s / args.steps * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "int64+fp32" if args.precision == "fp32" else "int64+fp64",
                "data": "synthetic (seeded CY instances, pfvs_b200/workloads.py)",
                "config": {"workload": workload_desc(args, w),
                           "form": args.form, "precision": args.precision,
                           "tuned_options": tuned or "library defaults",
                           "directions_per_gpu": len(idx) // world,
                           "l2": "working set per step > 126 MB (slabs + points); no flush needed",
                           "parallelism": (f"directions in chunks of {bounds[0][1]} pulled by {world} GPUs "
                                           f"from a shared queue" if world > 1 else "one GPU, one call")},
                "nodes_fp64_per_step": int(tot_nodes), "points_per_step": int(allsum(pg, n_points)),
                "directions_per_s": len(idx) * args.steps / dev_s,
                "points_per_s": allsum(pg, n_points) * args.steps / dev_s,
                "failed_directions": failed_all, "failed_directions_timed_per_step": failed_step,
                "stage_ms": {"setup": per_step["ms_setup"], "search": per_step["ms_search"],
                             "output": per_step["ms_output"]},
                "timed_form_nodes_per_step": int(per_step["nodes"]), "wall_ms_per_step": wall_s / args.steps * 1e3,
                "clocks": clk_sum, "e2e": e2e, "cpu_baseline": cpu, "roofline": roofline,
                "roofline_setup": roofline_setup, "forms": forms, "pfvs": pfv, "ref_gpu": ref_gpu,
                "gpu_launches": int(tot["launches"])}
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
