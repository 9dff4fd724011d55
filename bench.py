"""Benchmark driver: one JSON line per run (rank 0).

Default workload (config 2 of the reference's benchmark set): plain EDR top-k similarity over
100,000 synthetic random-walk trajectories (lengths lognormal(ln 200, 0.6) clipped to 32..1024),
256 query trajectories drawn from the set, k = 32, eps = 5e-4 deg, frequency vectors on the
256 x 256 virtual grid (cell 0.0025 deg, virtual-cell shift 2), one query per launch sequence.
A step is one pass over the 256 queries. Other workloads: --workload c1 (plain GT-quadtree range
queries), c3 (batched range queries over the three indexes), c4 (batched EDR pairs).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c2]

Multi-GPU runs are replicas (one process per GPU, each with its own copy of the set and its own
queries); value is the work of all ranks over the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

OPS_PER_CELL = 12  # int32 / fp32 instructions per DP cell of the EDR recurrence


def log(*a):
    print("[bench]", *a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------- distributed plumbing
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init_dist(world, backend="nccl"):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as td

    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    td.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return td


def max_over_ranks(td, value: float, device) -> float:
    if td is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def barrier(td, device=None):
    if td is not None:
        if device is not None:
            td.barrier(device_ids=[device.index])
        else:
            td.barrier()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = os.path.join("/tmp", f"gat_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax.append(float(f[2]))
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- peaks
def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


# ---------------------------------------------------------------- workload: config 2
C2 = dict(n=100_000, nq=256, k=32, eps=5e-4, cell=0.0025, vparam=2, leaf_cap=512)


def c2_workload(seed: int):
    from gat_b200 import data as D

    t, qids = D.config2(seed=seed, n=C2["n"], nq=C2["nq"])
    return t, qids


def run_c2(args, world, rank, local, td):
    import torch

    import gat_b200 as G
    from gat_b200 import _lib as L

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t, qids = c2_workload(seed=0)
    log("workload generated", t.n, len(t.lon))
    # replicas: each rank queries its own sample of the same set
    if rank > 0:
        from gat_b200 import data as D

        qids = D.sample_ids(C2["nq"], C2["n"], 1000 + rank)
    ctx = G.Context(local)
    db = G.TrajectorySet(ctx, t)
    g = G.Grid(ctx, db, G.BOX, C2["cell"], C2["vparam"], C2["leaf_cap"])
    log("index built", g.info())
    q = t.subset(qids)
    nq, k = q.n, C2["k"]
    qoff = np.zeros(nq + 1, np.int64)
    qoff[1:] = np.cumsum(q.lengths)
    xy = np.stack([q.lon, q.lat], 1).astype(np.float32)
    d_len = torch.from_numpy(q.lengths.astype(np.int32)).to(dev)
    d_off = torch.from_numpy(qoff).to(dev)
    d_xy = torch.from_numpy(xy).to(dev)
    d_ids = torch.empty(nq * k, dtype=torch.int32, device=dev)
    d_dist = torch.empty(nq * k, dtype=torch.int32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    lib = L.lib
    stream = torch.cuda.ExternalStream(ctx.stream)
    maxlen = int(q.lengths.max())
    stats = np.zeros(4, np.int64)
    acc = np.zeros(4, np.int64)

    def step(execution: int) -> float:
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = lib.gat_topk_dev(ctx.h, g.h, nq, d_len.data_ptr(), d_off.data_ptr(), d_xy.data_ptr(), maxlen, k, C2["eps"], execution,
                              d_ids.data_ptr(), d_dist.data_ptr(), stats.ctypes.data_as(L.P_i64))
        ctx.check(rc, "gat_topk_dev")
        e1.record(stream)
        e1.synchronize()
        acc[:] += stats
        return e0.elapsed_time(e1)

    # pinned host buffers for the end-to-end leg
    h_len = torch.from_numpy(q.lengths.astype(np.int32)).pin_memory()
    h_lon = torch.from_numpy(q.lon.astype(np.float32)).pin_memory()
    h_lat = torch.from_numpy(q.lat.astype(np.float32)).pin_memory()
    h_ids = torch.empty(nq * k, dtype=torch.int32).pin_memory()
    h_dist = torch.empty(nq * k, dtype=torch.int32).pin_memory()

    def step_e2e(execution: int) -> float:
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = lib.gat_topk(ctx.h, g.h, nq, h_len.numpy().ctypes.data_as(L.P_i32), h_lon.numpy().ctypes.data_as(L.P_f32),
                          h_lat.numpy().ctypes.data_as(L.P_f32), k, C2["eps"], execution, h_ids.numpy().ctypes.data_as(L.P_i32),
                          h_dist.numpy().ctypes.data_as(L.P_i32), None)
        ctx.check(rc, "gat_topk")
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    plain, batched = L.GAT_EXEC_PLAIN, L.GAT_EXEC_BATCHED
    log("warmup")
    for _ in range(args.warmup):
        log("step", step(plain))
    # ---- timed: plain (the workload as specified), with per-kernel timing
    ctx.set_timing(True)
    l0 = ctx.launches
    clocks = ClockSampler(local)
    barrier(td, dev)
    torch.cuda.synchronize()
    clocks.start()
    ms = []
    acc[:] = 0
    for _ in range(args.steps):
        ms.append(step(plain))
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = ctx.launches - l0
    timed_ms_for_gcups = None
    pairs, cells = int(acc[0]), int(acc[1])
    kstats = {c: ctx.kernel_stats(c) for c in (L.GAT_KERNEL_EDR, L.GAT_KERNEL_BOUNDS)}
    ctx.set_timing(False)
    total_ms = sum(ms)
    total_ms_max = max_over_ranks(td, total_ms, dev)
    barrier(td, dev)
    log("timed plain", ms)
    # ---- batched form of the same queries
    for _ in range(max(1, args.warmup)):
        step(batched)
    bms = [step(batched) for _ in range(args.steps)]
    bms_max = max_over_ranks(td, sum(bms), dev)
    # ---- end to end through the host-buffer C ABI call (plain), H2D + D2H inside
    for _ in range(max(1, args.warmup)):
        step_e2e(plain)
    ems = [step_e2e(plain) for _ in range(args.steps)]
    log("batched", bms, "e2e", ems)
    ems_max = max_over_ranks(td, sum(ems), dev)
    # results agree across forms
    ids_plain = d_ids.cpu().numpy().copy()
    ok_same = np.array_equal(ids_plain, h_ids.numpy())
    if rank != 0:
        ctx.close()
        return None
    nqs = nq * world * args.steps
    value = nqs / (total_ms_max / 1e3)
    # roofline: dominant timed kernel
    edr, bnd = kstats[L.GAT_KERNEL_EDR], kstats[L.GAT_KERNEL_BOUNDS]
    peaks = measured_peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    roof = roofline_c2(edr, bnd, hbm, clk)
    line = {
        "metric": "EDR top-k similarity queries/s (plain: one query per launch sequence)",
        "value": round(value, 2),
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_ms_max / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic (seeded random walks; no dataset)",
        "config": {"workload": "C2 plain EDR top-k: 100k trajectories, lognormal(ln200,0.6) lengths 32..1024, 256 queries "
                               "from the set, k=32, eps=5e-4 deg, FV grid 256x256 (cell 0.0025, shift 2), one query per launch",
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}"},
        "e2e": {"value": round(nqs / (ems_max / 1e3), 2), "unit": "queries/s",
                "h2d_bytes_per_step": int(q.lengths.nbytes + q.lon.nbytes + q.lat.nbytes),
                "d2h_bytes_per_step": int(2 * 4 * nq * k)},
        "gpu_launches": int(launches),
        "batched": {"value": round(nq * world * args.steps / (bms_max / 1e3), 2), "unit": "queries/s",
                    "speedup_vs_plain": round(total_ms_max / bms_max, 2)},
        "gcups_evaluated": round(cells / (total_ms / 1e3) / 1e9, 3),
        "edr_pairs_per_query": round(pairs / (nq * args.steps), 1),
        "kernels": {"edr": edr, "bounds": bnd},
        "roofline": roof,
        "clocks": clk,
        "results_identical_across_forms": bool(ok_same),
    }
    if world == 1 and not args.no_cpu_baseline:
        log("cpu baseline")
        line["cpu_baseline"] = cpu_baseline_c2(t, qids, sample=args.cpu_sample)
    ctx.close()
    return line


def roofline_c2(edr, bnd, hbm_gbs, clk):
    """Roofline of the kernel with the most device time in the timed region."""
    if bnd["ms"] >= edr["ms"]:
        per_launch_bytes = bnd["work"] / max(1, bnd["launches"])
        per_launch_s = bnd["ms"] / max(1, bnd["launches"]) / 1e3
        achieved = per_launch_bytes / per_launch_s / 1e9
        return {"kernel": "k_lower_bounds", "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_gbs,
                "unit": "GB/s", "frac": round(achieved / hbm_gbs, 4), "traffic": None,
                "work_per_launch": per_launch_bytes, "note": "algorithmic bytes: FV entries (8 B) + offsets and bound (12 B) per (query, trajectory); of measured"}
    per_launch_cells = edr["work"] / max(1, edr["launches"])
    per_launch_s = edr["ms"] / max(1, edr["launches"]) / 1e3
    achieved = per_launch_cells / per_launch_s / 1e9
    mhz = clk.get("sm_mhz") or 1965.0
    peak = 148 * 128 * mhz * 1e6 / OPS_PER_CELL / 1e9
    return {"kernel": "k_edr", "bound": "alu", "achieved": round(achieved, 2), "peak": round(peak, 1), "unit": "Gcell/s",
            "frac": round(achieved / peak, 4), "traffic": None,
            "note": f"peak = 148 SM x 128 int32 lanes x measured SM clock / {OPS_PER_CELL} ops per cell"}


def cpu_baseline_c2(t, qids, sample=32, reps=1):
    """The reference's own CPU top-k (Grid::SimilarityQueryBatchCPUParallel) on a sample of the
    queries, compiled from its sources (oracle/_ref/gatref); the oracle port otherwise."""
    from oracle import pyoracle as po

    qs = np.asarray(qids[:sample], np.int32)
    if po.ref_available():
        r = po.RefRunner().topk(t, qs, (121.0, 30.7, 122.0, 31.7), C2["cell"], C2["k"], C2["eps"], reps=reps)
        sec = float(np.sum(r["t_reps"]))
        return {"value": round(len(qs) * reps / sec, 3), "unit": "queries/s", "cores": min(os.cpu_count() or 1, len(qs)),
                "kind": "reference", "sample": f"{len(qs)} of the 256 queries x {reps}, Grid::SimilarityQueryBatchCPUParallel "
                                                f"(one thread per query for the bounds, 20 for EDR)"}
    o = po.OracleGrid(t, (121.0, 30.7, 122.0, 31.7), C2["cell"], C2["vparam"], C2["leaf_cap"])
    t0 = time.time()
    for qid in qs:
        o.topk(*t.points(int(qid)), C2["k"], C2["eps"], pruned=True, threads=1)
    sec = time.time() - t0
    return {"value": round(len(qs) / sec, 3), "unit": "queries/s", "cores": 1, "kind": "port",
            "sample": f"{len(qs)} of the 256 queries, oracle restatement, 1 thread"}


def run_reference_c2(args, world, rank):
    if rank != 0:
        return None
    from oracle import pyoracle as po

    t, qids = c2_workload(seed=0)
    sample = args.cpu_sample
    qs = np.asarray(qids[:sample], np.int32)
    if po.ref_available():
        r = po.RefRunner().topk(t, qs, (121.0, 30.7, 122.0, 31.7), C2["cell"], C2["k"], C2["eps"], reps=args.warmup + args.steps)
        times = list(r["t_reps"])[args.warmup:]
        kind = "reference"
        cores = min(os.cpu_count() or 1, len(qs))
        desc = f"{len(qs)} of the 256 queries per step, Grid::SimilarityQueryBatchCPUParallel compiled from the reference"
    else:
        o = __import__("oracle.pyoracle", fromlist=["OracleGrid"]).OracleGrid(t, (121.0, 30.7, 122.0, 31.7), C2["cell"], 2, 512)
        times = []
        for s in range(args.warmup + args.steps):
            t0 = time.time()
            for qid in qs:
                o.topk(*t.points(int(qid)), C2["k"], C2["eps"], pruned=True, threads=os.cpu_count() or 1)
            if s >= args.warmup:
                times.append(time.time() - t0)
        kind, cores, desc = "port", os.cpu_count() or 1, f"{len(qs)} queries per step, oracle restatement"
    sec = float(sum(times))
    value = len(qs) * args.steps / sec
    return {
        "impl": "reference",
        "metric": "EDR top-k similarity queries/s (plain: one query per launch sequence)",
        "value": round(value, 3),
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(sec / args.steps * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic (seeded random walks; no dataset)",
        "config": {"workload": "C2 plain EDR top-k: 100k trajectories, 256 queries from the set (bounded sample per step), k=32, eps=5e-4"},
        "cpu_baseline": {"value": round(value, 3), "unit": "queries/s", "cores": cores, "kind": kind, "sample": desc},
        "e2e": {"value": round(value, 3), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c2"])
    ap.add_argument("--cpu-sample", type=int, default=32)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_env()
    if args.impl == "reference":
        line = run_reference_c2(args, world, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    td = init_dist(world)
    try:
        line = run_c2(args, world, rank, local, td)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if td is not None:
            td.destroy_process_group()


if __name__ == "__main__":
    main()
