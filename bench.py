"""Benchmark driver: one JSON line per run (rank 0).

Default workload (config 2 of the reference's benchmark set): plain EDR top-k similarity over
100,000 synthetic random-walk trajectories (lengths lognormal(ln 200, 0.6) clipped to 32..1024),
256 query trajectories drawn from the set, k = 32, eps = 5e-4 deg, frequency vectors on the
256 x 256 virtual grid (cell 0.0025 deg, virtual-cell shift 2), one query per launch sequence.
A step is one pass over the 256 queries. Other workloads: --workload c1 (plain GT-quadtree range
queries), c3 (batched range queries over the three indexes), c4 (batched EDR pairs), c5 (served
mix of range and top-k requests through the serving loop at three offered loads), c4k (batched
top-k of 1024 long queries against the 1M-trajectory set), build (Grid and FSG index builds over
the 1M-trajectory set).

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

OPS_PER_CELL = 12  # int32 / fp32 instructions per DP cell of the EDR recurrence (match test, three-way min, carries)
# ALU-pipe instructions per DP cell of k_edr_tiles (8 rows per lane, row tiles) from an ncu capture of the
# C4 launch: ALU pipe 76.7% busy over the active cycles at 64 lanes per clock per SM, 2.257 G cells
ALU_PER_CELL = 10.2


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


def c2_workload(seed: int, lib: bool = True):
    """The config 2 set and query ids, from the library's generator (lib) or the oracle's copy of
    it (the reference arm loads no part of the library); both give the same arrays."""
    if lib:
        from gat_b200 import data as D

        return D.config2(seed=seed, n=C2["n"], nq=C2["nq"])
    from oracle import pyoracle as po

    return po.config2(seed=seed, n=C2["n"], nq=C2["nq"])


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
    if args.queries:
        # a prefix of the query sample, for launch-list captures under a profiler
        qids = qids[:args.queries]
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
    # ---- timed: plain (the workload as specified): one launch of the query graph per query
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
    pairs, cells = int(acc[0]), int(acc[1])
    total_ms = sum(ms)
    total_ms_max = max_over_ranks(td, total_ms, dev)
    ids_graph = d_ids.cpu().numpy().copy()
    barrier(td, dev)
    log("timed plain", ms)
    # ---- per-kernel device time: the same plain steps with CUDA events around every timed
    # kernel (events cannot sit inside the graph, so these kernels are launched one by one)
    ctx.set_timing(True)
    kms = [step(plain) for _ in range(args.steps)]
    kstats = {c: ctx.kernel_stats(c) for c in (L.GAT_KERNEL_EDR, L.GAT_KERNEL_BOUNDS)}
    ctx.set_timing(False)
    ids_stream = d_ids.cpu().numpy().copy()
    log("kernel-timing pass", kms)
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
    ok_same = np.array_equal(ids_graph, h_ids.numpy()) and np.array_equal(ids_graph, ids_stream)
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
        "config": {"workload": f"C2 plain EDR top-k: 100k trajectories, lognormal(ln200,0.6) lengths 32..1024, {nq} queries "
                               "from the set, k=32, eps=5e-4 deg, FV grid 256x256 (cell 0.0025, shift 2), one query per "
                               "launch (one CUDA-graph launch per query)",
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}",
                   "kernel_timing": "per-kernel device time from a second pass of the same steps with CUDA events "
                                    "around each timed kernel, launched one by one"},
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

    qs = np.asarray(qids[::max(1, len(qids) // sample)][:sample], np.int32)
    if po.ref_available():
        r = po.RefRunner().topk(t, qs, (121.0, 30.7, 122.0, 31.7), C2["cell"], C2["k"], C2["eps"], reps=reps)
        sec = float(np.sum(r["t_reps"]))
        return {"value": round(len(qs) * reps / sec, 3), "unit": "queries/s", "cores": min(os.cpu_count() or 1, len(qs)),
                "kind": "reference", "sample": f"{len(qs)} of the 256 queries (evenly spaced) x {reps}, Grid::SimilarityQueryBatchCPUParallel "
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

    t, qids = c2_workload(seed=0, lib=False)
    sample = args.cpu_sample
    # evenly spaced over the query sample, so light and heavy queries are both represented
    qs = np.asarray(qids[::max(1, len(qids) // sample)][:sample], np.int32)
    if po.ref_available():
        r = po.RefRunner().topk(t, qs, (121.0, 30.7, 122.0, 31.7), C2["cell"], C2["k"], C2["eps"], reps=args.warmup + args.steps)
        times = list(r["t_reps"])[args.warmup:]
        kind = "reference"
        cores = min(os.cpu_count() or 1, len(qs))
        desc = (f"{len(qs)} of the 256 queries (every {max(1, len(qids) // sample)}th) per step, "
                "Grid::SimilarityQueryBatchCPUParallel compiled from the reference")
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


# ---------------------------------------------------------------- shared GPU harness
class Harness:
    """CUDA-event timing on the library's stream, L2 flush between timed steps, clocks."""

    def __init__(self, ctx, dev):
        import torch

        self.torch = torch
        self.ctx = ctx
        self.dev = dev
        self.stream = torch.cuda.ExternalStream(ctx.stream)
        self.flush_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def time(self, fn) -> float:
        torch = self.torch
        self.flush_buf.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        fn()
        e1.record(self.stream)
        e1.synchronize()
        return e0.elapsed_time(e1)


def hbm_peak():
    p = measured_peaks()
    return float(p.get("hbm_gbs", 6650.0)), ("measured" if "hbm_gbs" in p else "fallback")


# DRAM read + write / algorithmic bytes of k_range_hash, from one-pass ncu captures (dram__bytes_read.sum,
# dram__bytes_write.sum) of the C3 batch on the 1M-walk set in the tuned shape (small queries one per warp):
# Grid (4.319 + 0.088) GB / 20.79 GB; FSG (block mode) (5.333 + 0.088) GB / 41.29 GB. The locality order serves
# neighbouring queries' points from L2.
RANGE_TRAFFIC_RATIO = {"grid": 0.212, "fsg": 0.131}


def range_roofline(st, name, index="grid"):
    gbs, src = hbm_peak()
    if st["launches"] == 0 or st["ms"] <= 0:
        return None
    per_bytes = st["work"] / st["launches"]
    per_s = st["ms"] / st["launches"] / 1e3
    ach = per_bytes / per_s / 1e9
    ratio = RANGE_TRAFFIC_RATIO.get(index)
    return {"kernel": name, "bound": "hbm", "achieved": round(ach, 1), "peak": gbs, "unit": "GB/s",
            "frac": round(ach / gbs, 4), "traffic": round(ratio * per_bytes) if ratio else None,
            "work_per_launch": per_bytes,
            "note": f"algorithmic bytes: 8 B (x, y) per tested point + 4 B per hit + 4 B per point of an all-hit item; "
                    f"peak of {src}; traffic = "
                    + (f"{ratio} x algorithmic, the dram read+write / algorithmic ratio of a one-pass ncu capture of "
                       f"this index's k_range_hash on the 1M-walk C3 batch" if ratio else "not captured for this index")
                    + "; DRAM traffic well below the algorithmic bytes means L2 serves most of them (locality order), "
                      "so the kernel is issue-bound, not HBM-bound"}


def edr_roofline(st, clk):
    if st["launches"] == 0 or st["ms"] <= 0:
        return None
    per_cells = st["work"] / st["launches"]
    per_s = st["ms"] / st["launches"] / 1e3
    ach = per_cells / per_s / 1e9
    mhz = clk.get("sm_mhz") or 1965.0
    peak = 148 * 128 * mhz * 1e6 / OPS_PER_CELL / 1e9
    alu = 148 * 64 * mhz * 1e6 / ALU_PER_CELL / 1e9
    return {"kernel": "k_edr", "bound": "alu", "achieved": round(ach, 2), "peak": round(peak, 1), "unit": "Gcell/s",
            "frac": round(ach / peak, 4), "traffic": None, "work_per_launch": per_cells,
            "note": f"peak = 148 SM x 128 int32 lanes x sampled SM clock / {OPS_PER_CELL} ops per cell (nominal issue rate)",
            "alu_pipe": {"peak": round(alu, 1), "frac": round(ach / alu, 4), "alu_instructions_per_cell": ALU_PER_CELL,
                         "note": "148 SM x 64 ALU-pipe lanes per clock x sampled SM clock / the kernel's measured ALU "
                                 "instructions per cell (ncu, C4 launch, 8 rows per lane)"}}


def base_line(args, world, metric, unit, value, ms_total, config, dtype="fp32-compare/int32"):
    return {"metric": metric, "value": round(value, 3), "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_total / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded random walks; no dataset)",
            "config": config}


# ---------------------------------------------------------------- workload: config 1
C1 = dict(n=10_000, nq=1_000, cell=0.01, leaf_cap=512)


def run_c1(args, world, rank, local, td):
    """Plain GT-quadtree range queries: 10k walks, 1k squares of 0.01 deg, leaf cap 512; id sets."""
    import torch

    import gat_b200 as G
    from gat_b200 import _lib as L
    from gat_b200 import data as D

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t, q = D.config1(seed=0, n=C1["n"], nq=C1["nq"])
    if rank > 0:
        q = D.boxes(C1["nq"], L.GAT_SIDE_FIXED, 0.01, 0.01, 1000 + rank)
    ctx = G.Context(local)
    db = G.TrajectorySet(ctx, t)
    g = G.Grid(ctx, db, G.BOX, C1["cell"], 2, C1["leaf_cap"])
    H = Harness(ctx, dev)
    nq = q.shape[0]
    cap = nq * 512
    d_q = torch.from_numpy(q).to(dev)
    d_off = torch.empty(nq + 1, dtype=torch.int64, device=dev)
    d_tid = torch.empty(cap, dtype=torch.int32, device=dev)
    import ctypes as C

    need = C.c_int64(0)

    def call(execution):
        ctx.check(L.lib.gat_range_query_dev(ctx.h, g.h, d_q.data_ptr(), nq, L.GAT_RESULT_IDS, execution, d_off.data_ptr(),
                                            d_tid.data_ptr(), None, cap, C.byref(need)), "gat_range_query_dev")

    h_q = torch.from_numpy(q).pin_memory()
    h_off = torch.empty(nq + 1, dtype=torch.int64).pin_memory()
    h_tid = torch.empty(cap, dtype=torch.int32).pin_memory()

    def call_e2e(execution):
        ctx.check(L.lib.gat_range_query(ctx.h, g.h, h_q.data_ptr(), nq, L.GAT_RESULT_IDS, execution,
                                        h_off.numpy().ctypes.data_as(L.P_i64), h_tid.numpy().ctypes.data_as(L.P_i32), None,
                                        cap, C.byref(need)), "gat_range_query")

    plain, batched = L.GAT_EXEC_PLAIN, L.GAT_EXEC_BATCHED
    for _ in range(args.warmup):
        H.time(lambda: call(plain))
    ctx.set_timing(True)
    l0 = ctx.launches
    clocks = ClockSampler(local)
    barrier(td, dev)
    clocks.start()
    ms = [H.time(lambda: call(plain)) for _ in range(args.steps)]
    clk = clocks.stop()
    launches = ctx.launches - l0
    scan = ctx.kernel_stats(L.GAT_KERNEL_RANGE_SCAN)
    ctx.set_timing(False)
    tot = max_over_ranks(td, sum(ms), dev)
    for _ in range(args.warmup):
        H.time(lambda: call(batched))
    ctx.set_timing(True)
    bms = [H.time(lambda: call(batched)) for _ in range(args.steps)]
    bscan = ctx.kernel_stats(L.GAT_KERNEL_RANGE_SCAN)
    ctx.set_timing(False)
    btot = max_over_ranks(td, sum(bms), dev)
    for _ in range(args.warmup):
        H.time(lambda: call_e2e(plain))
    ems = [H.time(lambda: call_e2e(plain)) for _ in range(args.steps)]
    etot = max_over_ranks(td, sum(ems), dev)
    total_ids = int(need.value)
    if rank != 0:
        ctx.close()
        return None
    line = base_line(args, world, "range queries/s (plain: one query per launch sequence)", "queries/s",
                     nq * world * args.steps / (tot / 1e3), tot,
                     {"workload": "C1 plain GT-quadtree range: 10k walks U[20,200], 1k squares 0.01 deg, leaf cap 512, "
                                  "cell 0.01 deg, trajectory-id sets", "l2": "flushed between steps (256 MiB write)",
                      "parallelism": f"replicas x{world}"})
    line.update({
        "e2e": {"value": round(nq * world * args.steps / (etot / 1e3), 3), "unit": "queries/s",
                "h2d_bytes_per_step": int(q.nbytes), "d2h_bytes_per_step": int((nq + 1) * 8 + total_ids * 4)},
        "gpu_launches": int(launches),
        "batched": {"value": round(nq * world * args.steps / (btot / 1e3), 3), "unit": "queries/s",
                    "speedup_vs_plain": round(tot / btot, 2), "roofline": range_roofline(bscan, "k_range_hash", None)},
        "roofline": range_roofline(scan, "k_plain_scan", None),
        "clocks": clk,
        "result_ids": total_ids,
    })
    if world == 1 and not args.no_cpu_baseline:
        from oracle import pyoracle as po

        if po.ref_available():
            r = po.RefRunner().gtq(t, q, (121.0, 30.7, 122.0, 31.7), C1["cell"], C1["leaf_cap"], layout=False, threads=0)
            line["cpu_baseline"] = {"value": round(nq / float(r["t_query"][0]), 1), "unit": "queries/s", "cores": 1,
                                    "kind": "reference", "sample": "all 1k queries, Grid::rangeQueryBatch on one core"}
    ctx.close()
    return line


def run_reference_c1(args, world, rank):
    if rank != 0:
        return None
    from oracle import pyoracle as po

    t, q = po.config1(seed=0, n=C1["n"], nq=C1["nq"])
    threads = os.cpu_count() or 1
    times = []
    R = po.RefRunner()
    for s in range(args.warmup + args.steps):
        r = R.gtq(t, q, (121.0, 30.7, 122.0, 31.7), C1["cell"], C1["leaf_cap"], layout=False, threads=threads)
        if s >= args.warmup:
            times.append(float(r["t_query"][0]))
    sec = sum(times)
    v = len(q) * args.steps / sec
    line = base_line(args, world, "range queries/s (plain: one query per launch sequence)", "queries/s", v, sec * 1e3,
                     {"workload": "C1 plain GT-quadtree range: 10k walks U[20,200], 1k squares 0.01 deg, leaf cap 512"})
    line.update({"impl": "reference",
                 "cpu_baseline": {"value": round(v, 3), "unit": "queries/s", "cores": threads, "kind": "reference",
                                  "sample": f"all 1k queries per step, Grid::rangeQueryBatch on {threads} threads (query slices)"},
                 "e2e": {"value": round(v, 3), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    return line


# ---------------------------------------------------------------- workload: config 3
C3 = dict(n=1_000_000, nq=100_000, cell=0.001, leaf_cap=512, stig_block=10240)


def run_c3(args, world, rank, local, td):
    """Batched range queries over the three indexes: 1M walks U[50,350], 100k rectangles with
    log-uniform sides in [0.001, 0.05] deg; trajectory-id sets."""
    import ctypes as C

    import torch

    import gat_b200 as G
    from gat_b200 import _lib as L
    from gat_b200 import data as D

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t0 = time.time()
    t, q = D.config3(seed=0, n=args.c3_n, nq=C3["nq"])
    log("c3 data", t.n, len(t.lon), round(time.time() - t0, 1))
    ctx = G.Context(local)
    if args.range_shape:
        ctx.set_tuning(L.GAT_TUNE_RANGE_SHAPE, args.range_shape)
    db = G.TrajectorySet(ctx, t)
    idx = {}
    t0 = time.time()
    idx["grid"] = G.Grid(ctx, db, G.BOX, C3["cell"], 2, C3["leaf_cap"])
    log("grid built", round(time.time() - t0, 1), idx["grid"].info())
    t0 = time.time()
    idx["fsg"] = G.FSG(ctx, db, G.BOX, C3["cell"])
    log("fsg built", round(time.time() - t0, 1))
    if "stig" in args.c3_indexes:
        t0 = time.time()
        idx["stig"] = G.STIG(ctx, db, C3["stig_block"])
        log("stig built", round(time.time() - t0, 1))
    H = Harness(ctx, dev)
    nq = q.shape[0]
    cap = 64 * 1024 * 1024
    d_q = torch.from_numpy(q).to(dev)
    d_off = torch.empty(nq + 1, dtype=torch.int64, device=dev)
    d_tid = torch.empty(cap, dtype=torch.int32, device=dev)
    need = C.c_int64(0)

    def call(ix, n=nq, execution=L.GAT_EXEC_BATCHED):
        ctx.check(L.lib.gat_range_query_dev(ctx.h, ix.h, d_q.data_ptr(), n, L.GAT_RESULT_IDS, execution, d_off.data_ptr(),
                                            d_tid.data_ptr(), None, cap, C.byref(need)), "gat_range_query_dev")

    res = {}
    for name, ix in idx.items():
        for _ in range(args.warmup):
            H.time(lambda: call(ix))
        l0 = ctx.launches
        clocks = ClockSampler(local)
        clocks.start()
        ms = [H.time(lambda: call(ix)) for _ in range(args.steps)]
        clk = clocks.stop()
        launches = ctx.launches - l0
        # kernel time and algorithmic bytes: two more steps with the library's per-kernel timing on
        ctx.set_timing(True)
        for _ in range(2):
            H.time(lambda: call(ix))
        st = ctx.kernel_stats(L.GAT_KERNEL_RANGE_SCAN)
        ctx.set_timing(False)
        res[name] = dict(ms=max_over_ranks(td, sum(ms), dev), launches=launches, ids=int(need.value), scan=st, clk=clk)
        log(name, ms, res[name]["ids"])
    # plain form on a sample of queries, for the batched-vs-plain ratio
    ns = min(nq, args.c3_plain_sample)
    pms = [H.time(lambda: call(idx["grid"], ns, L.GAT_EXEC_PLAIN)) for _ in range(max(1, args.steps // 2))]
    plain_qps = ns * len(pms) / (sum(pms) / 1e3)
    # end to end (host buffers) on the Grid
    h_q = torch.from_numpy(q).pin_memory()
    h_off = torch.empty(nq + 1, dtype=torch.int64).pin_memory()
    h_tid = torch.empty(cap, dtype=torch.int32).pin_memory()

    def call_e2e():
        ctx.check(L.lib.gat_range_query(ctx.h, idx["grid"].h, h_q.data_ptr(), nq, L.GAT_RESULT_IDS, L.GAT_EXEC_BATCHED,
                                        h_off.numpy().ctypes.data_as(L.P_i64), h_tid.numpy().ctypes.data_as(L.P_i32), None,
                                        cap, C.byref(need)), "gat_range_query")

    H.time(call_e2e)
    ems = [H.time(call_e2e) for _ in range(args.steps)]
    etot = max_over_ranks(td, sum(ems), dev)
    if rank != 0:
        ctx.close()
        return None
    g = res["grid"]
    line = base_line(args, world, "range queries/s (batched, GT-quadtree, trajectory-id sets)", "queries/s",
                     nq * world * args.steps / (g["ms"] / 1e3), g["ms"],
                     {"workload": f"C3 batched range: {t.n} walks U[50,350] ({len(t.lon)} points), 100k rectangles "
                                  "log-U[0.001,0.05] deg, cell 0.001 deg, leaf cap 512, STIG block 10240",
                      "l2": "flushed between steps (256 MiB write); point arrays 3.2 GB per index",
                      "parallelism": f"replicas x{world}"})
    line.update({
        "e2e": {"value": round(nq * world * args.steps / (etot / 1e3), 3), "unit": "queries/s",
                "h2d_bytes_per_step": int(q.nbytes), "d2h_bytes_per_step": int((nq + 1) * 8 + g["ids"] * 4)},
        "gpu_launches": int(g["launches"]),
        "indexes": {k: {"queries_per_s": round(nq * world * args.steps / (v["ms"] / 1e3), 1), "result_ids": v["ids"],
                        "roofline": range_roofline(v["scan"], "k_range_hash", k)} for k, v in res.items()},
        "plain_sample": {"queries": ns, "queries_per_s": round(plain_qps, 1),
                         "batched_speedup": round(nq * world * args.steps / (g["ms"] / 1e3) / plain_qps, 1)},
        "roofline": range_roofline(g["scan"], "k_range_hash"),
        "clocks": g["clk"],
    })
    ctx.close()
    return line


# ---------------------------------------------------------------- workload: config 4
def run_c4(args, world, rank, local, td):
    """Batched EDR: 4096 pairs, both lengths log-uniform in [16, 4096], eps 5e-4."""
    import torch

    import gat_b200 as G
    from gat_b200 import _lib as L
    from gat_b200 import data as D

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    la, a, lb, b = D.config4_pairs(seed=rank, npairs=args.pairs)
    n = len(la)
    cells = float(np.sum(la.astype(np.float64) * lb.astype(np.float64)))
    ctx = G.Context(local)
    H = Harness(ctx, dev)
    oa = np.zeros(n, np.int64)
    ob = np.zeros(n, np.int64)
    oa[1:] = np.cumsum(la)[:-1]
    ob[1:] = np.cumsum(lb)[:-1]
    T = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    d_la, d_oa, d_a, d_lb, d_ob, d_b = T(la.astype(np.int32)), T(oa), T(a), T(lb.astype(np.int32)), T(ob), T(b)
    d_out = torch.empty(n, dtype=torch.int32, device=dev)

    def call(lo=0, hi=n):
        ctx.check(L.lib.gat_edr_pairs_dev(ctx.h, hi - lo, d_la.data_ptr() + 4 * lo, d_oa.data_ptr() + 8 * lo, d_a.data_ptr(),
                                          d_lb.data_ptr() + 4 * lo, d_ob.data_ptr() + 8 * lo, d_b.data_ptr(), 5e-4,
                                          d_out.data_ptr() + 4 * lo), "gat_edr_pairs_dev")

    for _ in range(args.warmup):
        H.time(call)
    ctx.set_timing(True)
    l0 = ctx.launches
    clocks = ClockSampler(local)
    barrier(td, dev)
    clocks.start()
    ms = [H.time(call) for _ in range(args.steps)]
    clk = clocks.stop()
    st = ctx.kernel_stats(L.GAT_KERNEL_EDR)
    st["work"] = cells * args.steps
    ctx.set_timing(False)
    launches = ctx.launches - l0
    tot = max_over_ranks(td, sum(ms), dev)
    # plain: one pair per launch
    def plain():
        for i in range(n):
            call(i, i + 1)

    pms = [H.time(plain) for _ in range(1)]
    ptot = max_over_ranks(td, sum(pms), dev)
    # end to end through the host-buffer call
    import gat_b200.api as A

    ems = []
    for _ in range(args.steps):
        t0 = time.time()
        A.edr_pairs(ctx, la, a, lb, b, 5e-4)
        ems.append((time.time() - t0) * 1e3)
    etot = max_over_ranks(td, sum(ems), dev)
    if rank != 0:
        ctx.close()
        return None
    g = cells * world * args.steps / (tot / 1e3) / 1e9
    line = base_line(args, world, "EDR GCUPS (batched pairs)", "GCUPS", g, tot,
                     {"workload": f"C4 batched EDR: {n} pairs, lengths log-U[16,4096] both sides, eps 5e-4 deg, "
                                  f"{cells:.3g} DP cells per step", "l2": "flushed between steps (256 MiB write)",
                      "parallelism": f"replicas x{world}"}, dtype="int32")
    line.update({
        "e2e": {"value": round(cells * world * args.steps / (etot / 1e3) / 1e9, 3), "unit": "GCUPS",
                "h2d_bytes_per_step": int(a.nbytes + b.nbytes + 24 * n), "d2h_bytes_per_step": int(4 * n),
                "timer": "host wall clock around gat_edr_pairs (synchronous call)"},
        "gpu_launches": int(launches),
        "plain": {"value": round(cells * world / (ptot / 1e3) / 1e9, 3), "unit": "GCUPS", "note": "one pair per launch",
                  "batched_speedup": round(ptot / (tot / args.steps), 2)},
        "roofline": edr_roofline(st, clk),
        "clocks": clk,
    })
    if world == 1 and not args.no_cpu_baseline:
        from oracle import pyoracle as po

        idx = np.arange(0, n, 64)
        sa = np.concatenate([a[oa[i]:oa[i] + la[i]] for i in idx])
        sb = np.concatenate([b[ob[i]:ob[i] + lb[i]] for i in idx])
        sc = float(np.sum(la[idx].astype(np.float64) * lb[idx]))
        thr = os.cpu_count() or 1
        if po.ref_available():
            r = po.RefRunner().edr(la[idx], sa, lb[idx], sb, 5e-4, threads=thr)
            line["cpu_baseline"] = {"value": round(sc / float(r["t_query"][0]) / 1e9, 4), "unit": "GCUPS", "cores": thr,
                                    "kind": "reference", "sample": f"{len(idx)} of the {n} pairs, Grid::SimilarityExecuter"}
    ctx.close()
    return line


def run_reference_c4(args, world, rank):
    if rank != 0:
        return None
    from oracle import pyoracle as po

    la, a, lb, b = po.config4_pairs(seed=0, npairs=4096)
    n = len(la)
    oa = np.zeros(n, np.int64)
    ob = np.zeros(n, np.int64)
    oa[1:] = np.cumsum(la)[:-1]
    ob[1:] = np.cumsum(lb)[:-1]
    idx = np.arange(0, n, 32)
    sa = np.concatenate([a[oa[i]:oa[i] + la[i]] for i in idx])
    sb = np.concatenate([b[ob[i]:ob[i] + lb[i]] for i in idx])
    sc = float(np.sum(la[idx].astype(np.float64) * lb[idx]))
    thr = os.cpu_count() or 1
    R = po.RefRunner()
    times = []
    for s in range(args.warmup + args.steps):
        r = R.edr(la[idx], sa, lb[idx], sb, 5e-4, threads=thr)
        if s >= args.warmup:
            times.append(float(r["t_query"][0]))
    sec = sum(times)
    v = sc * args.steps / sec / 1e9
    line = base_line(args, world, "EDR GCUPS (batched pairs)", "GCUPS", v, sec * 1e3,
                     {"workload": "C4 batched EDR: 4096 pairs log-U[16,4096] (every 32nd pair per step)"}, dtype="int32")
    line.update({"impl": "reference",
                 "cpu_baseline": {"value": round(v, 4), "unit": "GCUPS", "cores": thr, "kind": "reference",
                                  "sample": f"{len(idx)} of 4096 pairs per step, Grid::SimilarityExecuter on {thr} threads"},
                 "e2e": {"value": round(v, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    return line


# ---------------------------------------------------------------- workload: config 4, top-k part
C4K = dict(nq=1024, k=64, eps=5e-4, cell=0.0025, vparam=2, leaf_cap=512, check=8)


def run_c4k(args, world, rank, local, td):
    """Batched top-k: 1024 query walks with lengths log-U[16, 4096] (the pair length
    distribution of config 4), k = 64, eps 5e-4, against the 1M-trajectory set of config 3 with
    frequency-vector pruning (FV on 256 x 256 virtual cells: cell 0.0025, shift 2). A sample of
    queries is checked against exhaustive EDR over the whole set (every pair on the GPU)."""
    import torch

    import gat_b200 as G
    from gat_b200 import _lib as L
    from gat_b200 import data as D

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t0 = time.time()
    t, _ = D.config3(seed=0, n=args.c3_n, nq=1)
    ctx = G.Context(local)
    db = G.TrajectorySet(ctx, t)
    grid = G.Grid(ctx, db, G.BOX, C4K["cell"], C4K["vparam"], C4K["leaf_cap"])
    log("c4k set and grid", t.n, round(time.time() - t0, 1))
    nq, k = args.c4k_queries, C4K["k"]
    qlen = D.lengths(nq, L.GAT_LEN_LOGUNIFORM, 0, 0, 16, 4096, 41 + rank)
    qs = D.walks(qlen, 42 + rank)
    qoff = np.zeros(nq + 1, np.int64)
    qoff[1:] = np.cumsum(qlen)
    T = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    d_len, d_off, d_xy = T(qlen.astype(np.int32)), T(qoff), T(np.stack([qs.lon, qs.lat], 1).astype(np.float32))
    d_ids = torch.empty(nq * k, dtype=torch.int32, device=dev)
    d_dist = torch.empty(nq * k, dtype=torch.int32, device=dev)
    stats = np.zeros(4, np.int64)
    H = Harness(ctx, dev)

    def call():
        stats[:] = 0
        ctx.check(L.lib.gat_topk_dev(ctx.h, grid.h, nq, d_len.data_ptr(), d_off.data_ptr(), d_xy.data_ptr(), int(qlen.max()), k,
                                     C4K["eps"], L.GAT_EXEC_BATCHED, d_ids.data_ptr(), d_dist.data_ptr(),
                                     stats.ctypes.data_as(L.P_i64)), "gat_topk_dev")

    for _ in range(args.warmup):
        log("warmup", H.time(call))
    ctx.set_timing(True)
    l0 = ctx.launches
    clocks = ClockSampler(local)
    clocks.start()
    ms = []
    for _ in range(args.steps):
        ms.append(H.time(call))
        log("step", ms[-1], stats.tolist())
    clk = clocks.stop()
    edr = ctx.kernel_stats(L.GAT_KERNEL_EDR)
    bnd = ctx.kernel_stats(L.GAT_KERNEL_BOUNDS)
    ctx.set_timing(False)
    launches = ctx.launches - l0
    tot = max_over_ranks(td, sum(ms), dev)
    ids = d_ids.cpu().numpy().reshape(nq, k)
    dist = d_dist.cpu().numpy().reshape(nq, k)
    # exhaustive check of a sample: EDR of the query against every trajectory of the set
    d_B = T(np.stack([t.lon, t.lat], 1).astype(np.float32))
    d_blen = T(t.lengths.astype(np.int32))
    d_boff = T(t.offsets[:-1].astype(np.int64))
    out = torch.empty(t.n, dtype=torch.int32, device=dev)
    chk = np.random.default_rng(43).choice(nq, size=min(nq, args.c4k_check), replace=False)
    ok = True
    for i in chk:
        a_len = torch.full((t.n,), int(qlen[i]), dtype=torch.int32, device=dev)
        a_off = torch.full((t.n,), int(qoff[i]), dtype=torch.int64, device=dev)
        ctx.check(L.lib.gat_edr_pairs_dev(ctx.h, t.n, a_len.data_ptr(), a_off.data_ptr(), d_xy.data_ptr(), d_blen.data_ptr(),
                                          d_boff.data_ptr(), d_B.data_ptr(), C4K["eps"], out.data_ptr()), "gat_edr_pairs_dev")
        ctx.sync()
        d_all = out.cpu().numpy()
        order = np.lexsort((np.arange(1, t.n + 1), d_all))[:k]
        ok &= bool(np.array_equal(ids[i], order + 1) and np.array_equal(dist[i], d_all[order]))
    log("exhaustive check", ok)
    if rank != 0:
        ctx.close()
        return None
    cells = edr["work"]
    line = base_line(args, world, "top-k queries/s (batched, 1M-trajectory set)", "queries/s",
                     nq * world * args.steps / (tot / 1e3), tot,
                     {"workload": f"C4 top-k: {nq} query walks log-U[16,4096], k=64, eps 5e-4, against {t.n} walks "
                                  "U[50,350]; FV 256x256 virtual cells (cell 0.0025, shift 2)",
                      "l2": "flushed between steps (256 MiB write); set 3.2 GB", "parallelism": f"replicas x{world}"},
                     dtype="int32")
    line.update({
        "gpu_launches": int(launches),
        "pairs_evaluated_per_query": round(float(stats[0]) / nq, 1),
        "pruned_fraction": round(1.0 - float(stats[0]) / (nq * t.n), 6),
        "gcups_evaluated": round(cells / (edr["ms"] / 1e3) / 1e9, 2) if edr["ms"] else None,
        "kernels": {"edr": edr, "bounds": bnd},
        "roofline": edr_roofline(edr, clk),
        "exhaustive_check": {"queries": int(len(chk)), "identical": ok},
        "clocks": clk,
    })
    ctx.close()
    return line


# ---------------------------------------------------------------- workload: config 5
C5 = dict(requests=4000, range_frac=0.7, loads=(0.25, 0.5, 0.8), lanes=4, budget=40 << 30, eps=5e-4)


def run_c5(args, world, rank, local, td):
    """Served mix over the C3 set and its three indexes, resident on the device: open-loop
    Poisson arrivals of 70% range requests (rectangles log-U[0.001, 0.05] deg, spread over the
    GT-quadtree, STIG and FSG; trajectory-id sets) and 30% top-k requests (query walks with
    lengths log-U[16, 2048], k uniform in [8, 64], eps 5e-4) through the serving loop
    (continuous batching, 4 lanes, 40 GiB budget). First a burst of all requests gives the
    saturation throughput; then three offered loads (fractions of it) give the achieved
    throughput and p50/p99 latency (arrival to completion, host clock)."""
    import torch

    import gat_b200 as G
    from gat_b200 import data as D

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t0 = time.time()
    t, _ = D.config3(seed=0, n=args.c3_n, nq=1)
    ctx = G.Context(local)
    db = G.TrajectorySet(ctx, t)
    grid = G.Grid(ctx, db, G.BOX, C3["cell"], 2, C3["leaf_cap"])
    stig = G.STIG(ctx, db, C3["stig_block"])
    fsg = G.FSG(ctx, db, G.BOX, C3["cell"])
    log("c5 set and indexes", t.n, round(time.time() - t0, 1))
    clocks = ClockSampler(local)
    r = served_mix(ctx, grid, stig, fsg, args.c5_requests, args.warmup, rank, clocks)
    if rank != 0:
        ctx.close()
        return None
    top = r["loads"][-1]
    n = args.c5_requests
    line = base_line(args, world, "served mixed requests/s (continuous batching; 70% range / 30% top-k)", "requests/s",
                     top["achieved_per_s"] * world, 1e3 * n / max(top["achieved_per_s"], 1e-9) * args.steps,
                     {"workload": f"C5 served mix: {t.n} walks U[50,350] resident with GT-quadtree (cell 0.001, leaf 512), "
                                  f"STIG (block 10240) and FSG (cell 0.001); {n} requests per load: 70% range "
                                  "(log-U[0.001,0.05] deg rectangles over the three indexes, id sets), 30% top-k "
                                  "(query lengths log-U[16,2048], k U[8,64], eps 5e-4); open-loop Poisson arrivals",
                      "server": r["server"], "l2": "inputs (3.2 GB per index) larger than L2",
                      "parallelism": f"replicas x{world}"})
    line.update({
        "e2e": {"value": round(top["achieved_per_s"] * world, 1), "unit": "requests/s", "h2d_bytes_per_step": r["h2d"],
                "d2h_bytes_per_step": int(top["result_entries"] * 4 * 2),
                "timer": "host clock from each request's submission to its completion (the serving path is end to end)"},
        "saturation": r["saturation"],
        "loads": r["loads"],
        "server_stats": r["server_stats"],
        "results_equal_direct_calls": r["results_equal_direct_calls"],
        "clocks": r["clocks"],
    })
    ctx.close()
    return line


def served_mix(ctx, grid, stig, fsg, n, warmup, rank, clocks):
    """The C5 measurement on indexes already resident: n requests (70% range over the three
    indexes, 30% top-k) through a G.Server; a burst for the saturation rate, then the offered
    loads of C5['loads'] (fractions of it), then a sample of requests against the direct calls."""
    import threading

    import gat_b200 as G
    from gat_b200 import _lib as L
    from gat_b200 import data as D

    rng = np.random.default_rng(500 + rank)
    is_range = rng.random(n) < C5["range_frac"]
    ikind = rng.integers(0, 3, n)
    boxes = D.boxes(n, L.GAT_SIDE_LOGUNIFORM, 0.001, 0.05, 501 + rank)
    qlen = D.lengths(n, L.GAT_LEN_LOGUNIFORM, 0, 0, 16, 2048, 502 + rank)
    qs = D.walks(qlen, 503 + rank)
    ks = rng.integers(8, 65, n)
    qoff = np.zeros(n + 1, np.int64)
    qoff[1:] = np.cumsum(qlen)
    srv = G.Server(ctx, grid, stig, fsg, lanes=C5["lanes"], budget_bytes=C5["budget"])

    def submit(i):
        if is_range[i]:
            return srv.submit_range(boxes[i], int(ikind[i]), "ids")
        a, b = qoff[i], qoff[i + 1]
        return srv.submit_topk(qs.lon[a:b], qs.lat[a:b], int(ks[i]), C5["eps"])

    def run(idx, rate=None):
        """Submits requests idx (open loop at `rate` per second, or all at once), waits for all;
        returns per-request (arrival, completion) ns and the result entries returned."""
        ids = [None] * len(idx)
        gaps = rng.exponential(1.0 / rate, len(idx)) if rate else np.zeros(len(idx))
        due = np.cumsum(gaps)

        def producer():
            start = time.perf_counter()
            for j, i in enumerate(idx):
                while True:
                    wait = start + due[j] - time.perf_counter()
                    if wait <= 0:
                        break
                    time.sleep(min(wait, 0.0005) if wait > 0.0002 else 0)
                ids[j] = submit(i)

        th = threading.Thread(target=producer)
        th.start()
        th.join()
        times = np.zeros((len(idx), 3), np.int64)
        entries = 0
        for j, r in enumerate(ids):
            st = srv.wait(r)
            if st != L.GAT_OK:
                raise RuntimeError(f"request {idx[j]} failed with status {st}")
            times[j] = srv.times(r)
            if is_range[idx[j]]:
                entries += len(srv.range_result(r))
            else:
                entries += int(ks[idx[j]])
            srv.release(r)
        return times, entries

    def summary(idx, times, entries):
        lat = (times[:, 2] - times[:, 0]) / 1e6
        span = (times[:, 2].max() - times[:, 0].min()) / 1e9
        rg = np.array([is_range[i] for i in idx])
        pct = lambda a, p: round(float(np.percentile(a, p)), 3) if len(a) else None
        return {"requests": len(idx), "achieved_per_s": round(len(idx) / span, 1), "p50_ms": pct(lat, 50),
                "p99_ms": pct(lat, 99), "range_p50_ms": pct(lat[rg], 50), "range_p99_ms": pct(lat[rg], 99),
                "topk_p50_ms": pct(lat[~rg], 50), "topk_p99_ms": pct(lat[~rg], 99), "result_entries": entries}

    # warm-up: every lane sees both request kinds (first launches tune the EDR tiles)
    for _ in range(warmup):
        run(np.arange(0, min(n, 400)))
    clocks.start()
    allidx = np.arange(n)
    times, entries = run(allidx)
    sat = summary(allidx, times, entries)
    loads = []
    for f in C5["loads"]:
        rate = f * sat["achieved_per_s"]
        times, entries = run(allidx, rate)
        s = summary(allidx, times, entries)
        s["offered_per_s"] = round(rate, 1)
        loads.append(s)
        log("load", f, s)
    clk = clocks.stop()
    st = srv.stats()
    # a sample of requests against the direct calls (each result must equal the request alone)
    ok = True
    chk = rng.choice(n, size=min(n, 24), replace=False)
    for i in chk:
        r = submit(i)
        srv.wait(r)
        if is_range[i]:
            got = srv.range_result(r)
            want = {0: grid, 1: stig, 2: fsg}[int(ikind[i])].range_query(boxes[i:i + 1]).tids
            ok &= bool(np.array_equal(got, want))
        else:
            got = srv.topk_result(r, int(ks[i]))
            a, b = qoff[i], qoff[i + 1]
            wi, wd, _ = grid.topk(D.Trajectories(np.array([b - a], np.int32), qs.lon[a:b], qs.lat[a:b]), int(ks[i]), C5["eps"])
            ok &= bool(np.array_equal(got[0], wi[0]) and np.array_equal(got[1], wd[0]))
        srv.release(r)
    srv.close()
    return {"saturation": sat, "loads": loads, "server_stats": st, "results_equal_direct_calls": ok, "clocks": clk,
            "checked_requests": int(len(chk)),
            "h2d": int(sum(32 if is_range[i] else 8 * qlen[i] + 16 for i in range(n))),
            "server": {"lanes": C5["lanes"], "budget_bytes": C5["budget"], "max_range_batch": 4096, "max_topk_batch": 32}}


# ---------------------------------------------------------------- workload: index builds
BUILD = dict(cell=0.001, vparam=2, leaf_cap=512, ref_n=40_000)


# dram read+write / algorithmic bytes of k_point_cells + k_expand_runs: (228.1 + 501.3) MB / 804.0 MB in an
# ncu capture of one Grid build over 100k walks (20M points, every array above L2)
BUILD_TRAFFIC_RATIO = 0.907


def build_roofline(st):
    gbs, src = hbm_peak()
    if st["launches"] == 0 or st["ms"] <= 0:
        return None
    ach = st["work"] / (st["ms"] / 1e3) / 1e9
    per = st["work"] / st["launches"]
    return {"kernel": "k_point_cells + k_expand_runs", "bound": "hbm", "achieved": round(ach, 1), "peak": gbs,
            "unit": "GB/s", "frac": round(ach / gbs, 4),
            "traffic": round(BUILD_TRAFFIC_RATIO * per) if BUILD_TRAFFIC_RATIO else None, "work_per_launch": per,
            "note": "achieved = algorithmic bytes of both placement kernels / their summed event time; k_point_cells "
                    "13 B per point (x, y read; cell and run flag written), k_expand_runs 24 B per point (x, y read; "
                    f"x, y, trajectory, key written) + 20 B per run (packed run, destination); peak of {src}; "
                    f"traffic = {BUILD_TRAFFIC_RATIO} x algorithmic, the dram read+write / algorithmic ratio of an ncu "
                    "capture of both kernels on a 100k-walk set (20M points)"}


def build_reference_sample():
    """The reference's own Grid::addDatasetToGrid and FSG::addDatasetToGrid over the first
    BUILD['ref_n'] trajectories of the set: (points placed per second over both builds, seconds)."""
    from oracle import pyoracle as po

    t, _ = po.config3(seed=0, n=BUILD["ref_n"], nq=1)
    R = po.RefRunner()
    r = R.gtq(t, np.zeros((0, 4), np.float32), po.BOX, BUILD["cell"], BUILD["leaf_cap"])
    f = R.fsg(t, po.BOX, BUILD["cell"])
    sec = float(r["t_build"][0]) + float(f["t_build"][0])
    return 2 * len(t.lon) / sec, sec, len(t.lon)


def run_build(args, world, rank, local, td):
    """Index builds over the C3 set (1M walks U[50,350], 200M points): a GT-quadtree Grid with its
    FVTable (cell 0.001 deg, virtual cells of 4x4 cells, leaf cap 512) and an FSG (cell 0.001 deg),
    both built in HBM from a resident trajectory set."""
    import torch

    import gat_b200 as G
    from gat_b200 import _lib as L
    from gat_b200 import data as D

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t, _ = D.config3(seed=0, n=args.c3_n, nq=1)
    P = len(t.lon)
    ctx = G.Context(local)
    ctx.set_tuning(L.GAT_TUNE_INDEX_BUILD, 2)
    db = G.TrajectorySet(ctx, t)
    H = Harness(ctx, dev)

    def build(dbh):
        return [G.Grid(ctx, dbh, G.BOX, BUILD["cell"], BUILD["vparam"], BUILD["leaf_cap"]),
                G.FSG(ctx, dbh, G.BOX, BUILD["cell"])]

    def step():
        out = []
        ms = H.time(lambda: out.extend(build(db)))
        info = [ix.info() for ix in out]
        for ix in out:
            ix.close()
        return ms, info

    for _ in range(args.warmup):
        step()
    ctx.set_timing(True)
    l0 = ctx.launches
    clocks = ClockSampler(local)
    barrier(td, dev)
    clocks.start()
    ms, info = [], None
    for _ in range(args.steps):
        m, info = step()
        ms.append(m)
    clk = clocks.stop()
    st = ctx.kernel_stats(L.GAT_KERNEL_INDEX_BUILD)
    ctx.set_timing(False)
    launches = ctx.launches - l0
    tot = max_over_ranks(td, sum(ms), dev)
    # end to end through the public API: the trajectory set uploaded from host arrays, both
    # builds, and each index's counts read back
    ems = []
    for _ in range(args.steps):
        keep = []

        def e2e():
            dbh = G.TrajectorySet(ctx, t)
            keep.append(dbh)
            keep.extend(build(dbh))
            for ix in keep[1:]:
                ix.info()

        ems.append(H.time(e2e))
        for ix in keep[1:]:
            ix.close()
        keep[0].close()
    etot = max_over_ranks(td, sum(ems), dev)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        v, sec, ps = build_reference_sample()
        cpu = {"value": round(v, 1), "unit": "points/s", "cores": 1, "kind": "reference",
               "sample": f"first {BUILD['ref_n']} trajectories ({ps} points): Grid::addDatasetToGrid + "
                         f"FSG::addDatasetToGrid, {sec:.2f} s on one core"}
    if rank != 0:
        ctx.close()
        return None
    line = base_line(args, world, "index build points/s (GT-quadtree Grid + FVTable, and FSG)", "points/s",
                     2 * P * world * args.steps / (tot / 1e3), tot,
                     {"workload": f"index builds over the C3 set: {t.n} walks U[50,350] ({P} points), Grid cell 0.001 "
                                  "deg (2048 x 2048 Morton cells), virtual cells 4x4, leaf cap 512; FSG cell 0.001 deg",
                      "l2": "flushed between steps (256 MiB write); point arrays 1.6 GB in, 3.2 GB out per index",
                      "parallelism": f"replicas x{world}"}, dtype="fp32-cell/int32")
    line.update({
        "e2e": {"value": round(2 * P * world * args.steps / (etot / 1e3), 1), "unit": "points/s",
                "h2d_bytes_per_step": int(t.lon.nbytes + t.lat.nbytes + t.lengths.nbytes),
                "d2h_bytes_per_step": 2 * 8 * 8},
        "gpu_launches": int(launches),
        "launches_note": "counts this library's kernels and the CUB radix-sort / scan passes it issues",
        "indexes": {"grid": info[0], "fsg": info[1]},
        "roofline": build_roofline(st),
        "cpu_baseline": cpu,
        "clocks": clk,
    })
    ctx.close()
    return line


def run_reference_build(args, world, rank):
    if rank != 0:
        return None
    times, v, ps = [], 0.0, 0
    for s in range(args.warmup + args.steps):
        v, sec, ps = build_reference_sample()
        if s >= args.warmup:
            times.append(sec)
    sec = sum(times)
    v = 2 * ps * args.steps / sec
    line = base_line(args, world, "index build points/s (GT-quadtree Grid + FVTable, and FSG)", "points/s", v, sec * 1e3,
                     {"workload": f"index builds: first {BUILD['ref_n']} trajectories of the C3 set ({ps} points), "
                                  "Grid cell 0.001 deg, leaf cap 512; FSG cell 0.001 deg"}, dtype="fp32-cell/int32")
    line.update({"impl": "reference",
                 "cpu_baseline": {"value": round(v, 1), "unit": "points/s", "cores": 1, "kind": "reference",
                                  "sample": f"first {BUILD['ref_n']} of the 1M trajectories per step (the reference's "
                                            "Grid build allocates and clears a cell-sized array per trajectory, "
                                            "Grid.cpp:268-269, so the full set takes about 3 minutes per build)"},
                 "e2e": {"value": round(v, 1), "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    return line


# ---------------------------------------------------------------- workload: the range and EDR suite (default)
SUITE = dict(n=1_000_000, nq=100_000, cell=0.001, vparam=2, leaf_cap=512, stig_block=10240, plain_queries=2000,
             parity_queries=1000, pairs=4096, eps=5e-4, c5_requests=2000, ref_per_step=2000, ref_pair_every=32)
SUITE_METRIC = "range queries/s & EDR GCUPS, batched vs plain, 1 B200, bit-exact; p50/p99 ms"


def host_cpu() -> tuple[int, str]:
    """(host cores this process may run on, CPU model name)."""
    try:
        cores = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        cores = os.cpu_count() or 1
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return cores, model


def suite_config(world: int, n: int) -> dict:
    """The configuration both arms print (the reference arm times the same workload on the host)."""
    return {"workload": f"C3 batched range queries over the GT-quadtree, STIG, FSG and MortonGrid: {n} random walks U[50,350] "
                        "points, 100k rectangles with log-U[0.001,0.05] deg sides, cell 0.001 deg, leaf cap 512, STIG "
                        "block 10240, trajectory-id sets; value = GT-quadtree batched queries/s. Beside it: the plain "
                        "form (one query per launch sequence), C4 batched EDR (4096 pairs, both sides log-U[16,4096], "
                        "eps 5e-4 deg) and its plain form (one pair per launch), and the C5 served mix (p50/p99)",
            "l2": "flushed between steps (256 MiB write); point arrays 3.2 GB per index",
            "parallelism": f"replicas x{world}"}


def sample_rows(off: np.ndarray, vals: np.ndarray, rows: np.ndarray):
    """CSR rows `rows` of (off, vals) as a new CSR."""
    counts = off[rows + 1] - off[rows]
    o = np.zeros(len(rows) + 1, np.int64)
    np.cumsum(counts, out=o[1:])
    v = np.concatenate([vals[off[r]:off[r + 1]] for r in rows]) if len(rows) else np.zeros(0, vals.dtype)
    return o, v


def oracle_range_parallel(o, q, threads: int):
    """The oracle's id sets for q on `threads` host threads (query slices); (off, ids, seconds)."""
    from concurrent.futures import ThreadPoolExecutor

    nq = len(q)
    per = max(1, (nq + threads - 1) // threads)
    slices = [(s, min(nq, s + per)) for s in range(0, nq, per)]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        parts = list(ex.map(lambda se: o.range(q[se[0]:se[1]]), slices))
    sec = time.perf_counter() - t0
    counts = np.concatenate([np.diff(p[0]) for p in parts])
    off = np.zeros(nq + 1, np.int64)
    np.cumsum(counts, out=off[1:])
    return off, np.concatenate([p[1] for p in parts]), sec


def run_suite(args, world, rank, local, td):
    """Config 3 batched range queries (the line's value) with their plain form, config 4 batched and
    plain EDR, and the config 5 served mix, on one resident 1M-walk set and its three indexes."""
    import ctypes as C

    import torch

    import gat_b200 as G
    from gat_b200 import _lib as L
    from gat_b200 import data as D

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t0 = time.time()
    n, nq = args.c3_n, SUITE["nq"]
    t, q = D.config3(seed=0, n=n, nq=nq)
    if rank > 0:  # replicas: each rank its own rectangles over the same set
        q = D.boxes(nq, L.GAT_SIDE_LOGUNIFORM, 0.001, 0.05, 1000 + rank)
    log("suite data", t.n, len(t.lon), round(time.time() - t0, 1))
    ctx = G.Context(local)
    db = G.TrajectorySet(ctx, t)
    t0 = time.time()
    idx = {"grid": G.Grid(ctx, db, G.BOX, SUITE["cell"], SUITE["vparam"], SUITE["leaf_cap"]),
           "fsg": G.FSG(ctx, db, G.BOX, SUITE["cell"])}
    idx["morton"] = G.MortonGrid(idx["grid"])
    log("grid + fsg + morton built", round(time.time() - t0, 1))
    t0 = time.time()
    idx["stig"] = G.STIG(ctx, db, SUITE["stig_block"])
    log("stig built", round(time.time() - t0, 1))
    H = Harness(ctx, dev)
    cap = 64 * 1024 * 1024
    d_q = torch.from_numpy(q).to(dev)
    d_off = torch.empty(nq + 1, dtype=torch.int64, device=dev)
    d_tid = torch.empty(cap, dtype=torch.int32, device=dev)
    need = C.c_int64(0)

    def call(ix, dq=d_q, m=nq, execution=L.GAT_EXEC_BATCHED):
        ctx.check(L.lib.gat_range_query_dev(ctx.h, ix.h, dq.data_ptr(), m, L.GAT_RESULT_IDS, execution, d_off.data_ptr(),
                                            d_tid.data_ptr(), None, cap, C.byref(need)), "gat_range_query_dev")

    # ---- timed: batched range steps on each index (the GT-quadtree's are the line's value)
    res = {}
    clk = None
    for name in ("grid", "fsg", "stig", "morton"):
        ix = idx[name]
        for _ in range(args.warmup):
            H.time(lambda: call(ix))
        l0 = ctx.launches
        clocks = ClockSampler(local)
        barrier(td, dev)
        clocks.start()
        ms = [H.time(lambda: call(ix)) for _ in range(args.steps)]
        c = clocks.stop()
        launches = ctx.launches - l0
        # kernel device time and algorithmic bytes for the roofline: two more steps with the library's
        # per-kernel timing on (it also counts the bytes, which the timed steps skip)
        ctx.set_timing(True)
        for _ in range(2):
            H.time(lambda: call(ix))
        st = ctx.kernel_stats(L.GAT_KERNEL_RANGE_SCAN)
        ctx.set_timing(False)
        res[name] = dict(ms=max_over_ranks(td, sum(ms), dev), launches=launches, ids=int(need.value), scan=st)
        if name == "grid":
            clk = c
        log(name, [round(x, 3) for x in ms], res[name]["ids"])
    # ---- plain form: one query per launch sequence, on an evenly spaced sample of the rectangles
    ps = min(nq, SUITE["plain_queries"])
    sel = np.arange(0, nq, nq // ps)[:ps]
    d_qs = d_q[torch.from_numpy(sel).to(dev)].contiguous()
    H.time(lambda: call(idx["grid"], d_qs, ps, L.GAT_EXEC_PLAIN))
    pms = [H.time(lambda: call(idx["grid"], d_qs, ps, L.GAT_EXEC_PLAIN)) for _ in range(max(1, min(args.steps, 5)))]
    plain_off = d_off[:ps + 1].cpu().numpy()
    plain_ids = d_tid[:int(plain_off[-1])].cpu().numpy()
    ptot = max_over_ranks(td, sum(pms), dev)
    plain_qps = ps * world * len(pms) / (ptot / 1e3)
    # ---- config 1 in both forms (10k walks, 1k squares of 0.01 deg): the plain form's own workload
    t1, q1 = D.config1(seed=0, n=C1["n"], nq=C1["nq"])
    db1 = G.TrajectorySet(ctx, t1)
    g1 = G.Grid(ctx, db1, G.BOX, C1["cell"], 2, C1["leaf_cap"])
    d_q1 = torch.from_numpy(q1).to(dev)
    H.time(lambda: call(g1, d_q1, len(q1), L.GAT_EXEC_PLAIN))
    c1_pms = [H.time(lambda: call(g1, d_q1, len(q1), L.GAT_EXEC_PLAIN)) for _ in range(max(1, min(args.steps, 5)))]
    c1_off = d_off[:len(q1) + 1].cpu().numpy()
    c1_ids = d_tid[:int(c1_off[-1])].cpu().numpy()
    H.time(lambda: call(g1, d_q1, len(q1)))
    c1_bms = [H.time(lambda: call(g1, d_q1, len(q1))) for _ in range(max(1, min(args.steps, 5)))]
    c1_plain = len(q1) * world * len(c1_pms) / (max_over_ranks(td, sum(c1_pms), dev) / 1e3)
    c1_batched = len(q1) * world * len(c1_bms) / (max_over_ranks(td, sum(c1_bms), dev) / 1e3)
    # ---- end to end through the host-buffer call (pinned host rectangles in, id sets out)
    h_q = torch.from_numpy(q).pin_memory()
    h_off = torch.empty(nq + 1, dtype=torch.int64).pin_memory()
    h_tid = torch.empty(cap, dtype=torch.int32).pin_memory()

    def call_e2e():
        ctx.check(L.lib.gat_range_query(ctx.h, idx["grid"].h, h_q.data_ptr(), nq, L.GAT_RESULT_IDS, L.GAT_EXEC_BATCHED,
                                        h_off.numpy().ctypes.data_as(L.P_i64), h_tid.numpy().ctypes.data_as(L.P_i32), None,
                                        cap, C.byref(need)), "gat_range_query")

    H.time(call_e2e)
    ems = [H.time(call_e2e) for _ in range(args.steps)]
    etot = max_over_ranks(td, sum(ems), dev)
    grid_off = h_off.numpy().copy()
    grid_ids = h_tid.numpy()[:int(grid_off[-1])].copy()
    # FSG id sets of the parity sample
    pq = min(nq, SUITE["parity_queries"])
    psel = np.arange(0, nq, nq // pq)[:pq]
    fsg_r = idx["fsg"].range_query(q[psel])
    morton_r = idx["morton"].range_query(q[psel])
    # ---- config 4: batched EDR pairs and their plain form
    edr = measure_edr_pairs(ctx, H, args, td, rank, local, dev)
    # ---- config 5: served mix on the same resident set
    c5 = served_mix(ctx, idx["grid"], idx["stig"], idx["fsg"], args.c5_requests, min(args.warmup, 3), rank,
                    ClockSampler(local))
    if rank != 0:
        ctx.close()
        return None
    g = res["grid"]
    value = nq * world * args.steps / (g["ms"] / 1e3)
    line = base_line(args, world, SUITE_METRIC, "queries/s", value, g["ms"], suite_config(world, t.n))
    line.update({
        "e2e": {"value": round(nq * world * args.steps / (etot / 1e3), 3), "unit": "queries/s",
                "h2d_bytes_per_step": int(q.nbytes), "d2h_bytes_per_step": int((nq + 1) * 8 + len(grid_ids) * 4),
                "call": "gat_range_query (pinned host rectangles in, CSR id sets out), GT-quadtree, batched"},
        "gpu_launches": int(g["launches"]),
        "roofline": range_roofline(g["scan"], "k_range_hash"),
        "clocks": clk,
        "range": {
            "indexes": {k: {"queries_per_s": round(nq * world * args.steps / (v["ms"] / 1e3), 1), "result_ids": v["ids"],
                            "ms_per_step": round(v["ms"] / args.steps, 4),
                            "roofline": range_roofline(v["scan"], "k_range_hash", k)} for k, v in res.items()},
            "plain": {"queries": ps, "steps": len(pms), "queries_per_s": round(plain_qps, 1),
                      "form": "gat_range_query_dev with GAT_EXEC_PLAIN: one query per launch sequence",
                      "sample": f"every {nq // ps}th of the 100k rectangles"},
            "batched_over_plain": round(value / plain_qps, 1),
            "c1": {"workload": "10k walks U[20,200], 1k squares of 0.01 deg, cell 0.01, leaf cap 512, GT-quadtree",
                   "plain_queries_per_s": round(c1_plain, 1), "batched_queries_per_s": round(c1_batched, 1),
                   "batched_over_plain": round(c1_batched / c1_plain, 1)},
        },
        "edr": edr,
        "served": {"requests_per_load": args.c5_requests, "saturation": c5["saturation"], "loads": c5["loads"],
                   "server": c5["server"], "server_stats": c5["server_stats"],
                   "results_equal_direct_calls": c5["results_equal_direct_calls"], "clocks": c5["clocks"]},
    })
    # ---- parity against the oracle and the CPU baseline (rank 0, one GPU)
    if world == 1 and not args.no_cpu_baseline:
        from oracle import pyoracle as po

        cores, model = host_cpu()
        t0 = time.time()
        og = po.OracleGrid(t, G.BOX, SUITE["cell"], SUITE["vparam"], SUITE["leaf_cap"])
        of = po.OracleFSG(t, G.BOX, SUITE["cell"])
        log("oracle grid + fsg built", round(time.time() - t0, 1))
        o_off, o_ids, sec = oracle_range_parallel(og, q[psel], cores)
        g_off, g_ids = sample_rows(grid_off, grid_ids, psel)
        f_off, f_ids = of.range(q[psel])
        p_off, p_ids = sample_rows(plain_off, plain_ids, np.arange(0, ps, max(1, ps // pq))[:pq])
        po_off, po_ids = og.range(q[sel][np.arange(0, ps, max(1, ps // pq))[:pq]])
        c1o_off, c1o_ids = po.OracleGrid(t1, G.BOX, C1["cell"], 2, C1["leaf_cap"]).range(q1)
        checks = {"grid_batched": bool(np.array_equal(g_off, o_off) and np.array_equal(g_ids, o_ids)),
                  "c1_plain": bool(np.array_equal(c1_off, c1o_off) and np.array_equal(c1_ids, c1o_ids)),
                  "fsg_batched": bool(np.array_equal(fsg_r.offsets, f_off) and np.array_equal(fsg_r.tids, f_ids)),
                  "morton_batched": bool(np.array_equal(morton_r.offsets, o_off) and np.array_equal(morton_r.tids, o_ids)),
                  "grid_plain": bool(np.array_equal(p_off, po_off) and np.array_equal(p_ids, po_ids)),
                  "edr_batched": edr.pop("_parity_ok")}
        line["parity"] = {"checked": {"range_queries": int(pq), "c1_plain_queries": int(len(q1)), "edr_pairs": int(edr["pairs"])},
                          "against": "oracle restatement (pinned to the reference's compiled CPU code by the CPU tests)",
                          "stig": "checked against the oracle by tests/test_gpu_configs.py (its oracle build takes minutes)",
                          "cases": checks, "equal": all(checks.values())}
        line["cpu_baseline"] = {"value": round(pq / sec, 1), "unit": "queries/s", "cores": cores, "cpu": model,
                                "kind": "port",
                                "sample": f"{pq} of the 100k rectangles (every {nq // pq}th), the oracle's GT-quadtree "
                                          f"range query on {cores} threads (query slices)"}
        line["edr"]["cpu_baseline"]["cpu"] = model
    else:
        edr.pop("_parity_ok", None)
    ctx.close()
    return line


def measure_edr_pairs(ctx, H, args, td, rank, local, dev):
    """Config 4: 4096 pairs, both lengths log-U[16, 4096], eps 5e-4. Batched (one launch for all
    pairs) timed steps with the tile kernel's own event time; plain (one pair per launch); the
    oracle's distances on every pair as the parity check and the CPU baseline (rank 0)."""
    import torch

    import gat_b200.api as A
    from gat_b200 import _lib as L
    from gat_b200 import data as D

    la, a, lb, b = D.config4_pairs(seed=rank, npairs=SUITE["pairs"])
    n = len(la)
    cells = float(np.sum(la.astype(np.float64) * lb.astype(np.float64)))
    oa = np.zeros(n, np.int64)
    ob = np.zeros(n, np.int64)
    oa[1:] = np.cumsum(la)[:-1]
    ob[1:] = np.cumsum(lb)[:-1]
    T = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    d_la, d_oa, d_a, d_lb, d_ob, d_b = T(la.astype(np.int32)), T(oa), T(a), T(lb.astype(np.int32)), T(ob), T(b)
    d_out = torch.empty(n, dtype=torch.int32, device=dev)
    eps = SUITE["eps"]

    def call(lo=0, hi=n):
        ctx.check(L.lib.gat_edr_pairs_dev(ctx.h, hi - lo, d_la.data_ptr() + 4 * lo, d_oa.data_ptr() + 8 * lo, d_a.data_ptr(),
                                          d_lb.data_ptr() + 4 * lo, d_ob.data_ptr() + 8 * lo, d_b.data_ptr(), eps,
                                          d_out.data_ptr() + 4 * lo), "gat_edr_pairs_dev")

    for _ in range(args.warmup):
        H.time(call)
    ctx.set_timing(True)
    l0 = ctx.launches
    clocks = ClockSampler(local)
    barrier(td, dev)
    clocks.start()
    ms = [H.time(call) for _ in range(args.steps)]
    clk = clocks.stop()
    st = ctx.kernel_stats(L.GAT_KERNEL_EDR)
    st["work"] = cells * args.steps
    ctx.set_timing(False)
    launches = ctx.launches - l0
    tot = max_over_ranks(td, sum(ms), dev)
    got = d_out.cpu().numpy().copy()

    def plain():
        for i in range(n):
            call(i, i + 1)

    H.time(lambda: [call(i, i + 1) for i in range(0, n, 64)])  # warm the one-pair shape class
    pms = [H.time(plain)]
    ptot = max_over_ranks(td, sum(pms), dev)
    plain_ok = bool(np.array_equal(d_out.cpu().numpy(), got))
    ems = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_out = A.edr_pairs(ctx, la, a, lb, b, eps)
        ems.append((time.perf_counter() - t0) * 1e3)
    etot = max_over_ranks(td, sum(ems), dev)
    gcups = cells * args.steps / (tot / 1e3) / 1e9
    pg = cells / (ptot / 1e3) / 1e9
    out = {"workload": f"{n} pairs, both lengths log-U[16,4096], eps 5e-4 deg, {cells:.4g} DP cells per step",
           "batched": {"gcups": round(gcups, 3), "ms_per_step": round(tot / args.steps, 4), "gpu_launches": int(launches)},
           "plain": {"gcups": round(pg, 3), "ms_per_step": round(ptot, 3), "form": "one pair per gat_edr_pairs_dev call",
                     "results_equal_batched": plain_ok},
           "batched_over_plain": round(gcups / pg, 1),
           "e2e": {"gcups": round(cells * args.steps / (etot / 1e3) / 1e9, 3), "timer": "host clock around gat_edr_pairs "
                   "(synchronous; host arrays in, distances out)", "h2d_bytes_per_step": int(a.nbytes + b.nbytes + 24 * n),
                   "d2h_bytes_per_step": int(4 * n), "results_equal_batched": bool(np.array_equal(e2e_out, got))},
           "roofline": edr_roofline(st, clk),
           "clocks": clk, "pairs": n, "_parity_ok": True}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import pyoracle as po

        cores, _ = host_cpu()
        t0 = time.perf_counter()
        want = po.edr_batch(la, a, lb, b, eps, threads=cores)
        sec = time.perf_counter() - t0
        out["_parity_ok"] = bool(np.array_equal(want, got))
        out["cpu_baseline"] = {"value": round(cells / sec / 1e9, 4), "unit": "GCUPS", "cores": cores, "kind": "port",
                               "sample": f"all {n} pairs, the oracle's EDR on {cores} threads"}
    return out


def run_reference_suite(args, world, rank):
    """The reference's own CPU code on the suite's workload (rank 0): gatref rangebench builds the
    reference's Grid over the same generated set and times Grid::rangeQueryBatch on strided samples
    of the same rectangles on every host core; gatref edr times Grid::SimilarityExecuter on a
    sample of the config 4 pairs. No part of this library is loaded."""
    if rank != 0:
        return None
    from oracle import pyoracle as po

    cores, model = host_cpu()
    n, nq = args.c3_n, SUITE["nq"]
    cfg = suite_config(world, n)
    if not po.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/gatref (the reference's CPU code compiled from its "
                "sources) was not built in this tree", "config": cfg}
    steps = args.warmup + args.steps
    per_step = min(SUITE["ref_per_step"], nq // steps)
    R = po.RefRunner()
    t0 = time.time()
    r = R.rangebench(n, 50, 350, 0, nq, 0.001, 0.05, SUITE["cell"], SUITE["leaf_cap"], po.BOX, per_step, steps, cores)
    log("reference rangebench", round(time.time() - t0, 1), "build", float(r["t_build"][0]))
    ts = [float(x) for x in r["t_step"][args.warmup:]]
    sec = sum(ts)
    value = per_step * args.steps / sec
    la, a, lb, b = po.config4_pairs(seed=0, npairs=SUITE["pairs"])
    sel = np.arange(0, len(la), SUITE["ref_pair_every"])
    oa = np.concatenate([[0], np.cumsum(la)]).astype(np.int64)
    ob = np.concatenate([[0], np.cumsum(lb)]).astype(np.int64)
    sa = np.concatenate([a[oa[i]:oa[i + 1]] for i in sel])
    sb = np.concatenate([b[ob[i]:ob[i + 1]] for i in sel])
    sc = float(np.sum(la[sel].astype(np.float64) * lb[sel]))
    e = R.edr(la[sel], sa, lb[sel], sb, SUITE["eps"], threads=cores)
    edr_gcups = sc / float(e["t_query"][0]) / 1e9
    line = base_line(args, world, SUITE_METRIC, "queries/s", value, sec * 1e3, cfg)
    line.update({
        "impl": "reference",
        "cpu_baseline": {"value": round(value, 3), "unit": "queries/s", "cores": cores, "cpu": model, "kind": "reference",
                         "sample": f"per step {per_step} of the 100k rectangles (every {nq // per_step}th, a different "
                                   f"offset each step), Grid::rangeQueryBatch on {cores} threads (query slices), over "
                                   f"the reference's Grid of the same {n} walks (built in {float(r['t_build'][0]):.1f} s)"},
        "e2e": {"value": round(value, 3), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "result_ids_per_step": int(np.mean(r["ids_step"][args.warmup:])),
        "edr": {"gcups": round(edr_gcups, 4), "unit": "GCUPS", "cores": cores,
                "sample": f"{len(sel)} of the {len(la)} config 4 pairs (every {SUITE['ref_pair_every']}th), "
                          f"Grid::SimilarityExecuter on {cores} threads"},
        "served": {"unavailable": "the reference has no serving loop"},
    })
    return line


WORKLOADS = {"suite": run_suite, "c1": run_c1, "c2": run_c2, "c3": run_c3, "c4": run_c4, "c4k": run_c4k, "c5": run_c5,
             "build": run_build}
REFERENCE = {"suite": run_reference_suite, "c1": run_reference_c1, "c2": run_reference_c2, "c4": run_reference_c4,
             "build": run_reference_build}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="suite", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-sample", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--queries", type=int, default=0, help="C2: use only the first N of the 256 queries")
    ap.add_argument("--pairs", type=int, default=4096, help="C4: pairs per launch")
    ap.add_argument("--c3-indexes", default="grid,fsg,stig")
    ap.add_argument("--c3-n", type=int, default=C3["n"])
    ap.add_argument("--c3-plain-sample", type=int, default=2000)
    ap.add_argument("--range-shape", type=int, default=0,
                    help="c3: block shape of the batched range scan (0 = autotuned, 1 = 256 threads, 2 = 128 threads, "
                         "3 = split by query size)")
    ap.add_argument("--c5-requests", type=int, default=0, help="C5 requests per load (default 4000; 2000 in the suite)")
    ap.add_argument("--c4k-queries", type=int, default=C4K["nq"])
    ap.add_argument("--c4k-check", type=int, default=C4K["check"])
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if not args.c5_requests:
        args.c5_requests = SUITE["c5_requests"] if args.workload == "suite" else C5["requests"]
    world, rank, local = dist_env()
    if args.impl == "reference":
        fn = REFERENCE.get(args.workload)
        if args.workload == "c3":
            line = {"impl": "reference", "unavailable": "the reference's Grid build clears a cell-sized array per "
                    "trajectory (Grid.cpp:268-269): about 3 minutes on one core for the 1M-trajectory set before any "
                    "query, and its 100k queries then scan on one core; a bench step cannot hold that"}
        elif args.workload == "c4k":
            line = {"impl": "reference", "unavailable": "the reference's Grid build over the 1M-trajectory set takes about "
                    "3 minutes on one core (Grid.cpp:268-269), and its GPU EDR kernel stops at 1024 points per side "
                    "(kernel.cu:249-501) while these queries reach 4096"}
        elif args.workload == "c5":
            line = {"impl": "reference", "unavailable": "the reference has no serving loop, and its Grid build over the "
                    "1M-trajectory set takes about 3 minutes on one core (Grid.cpp:268-269)"}
        else:
            line = fn(args, world, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    td = init_dist(world)
    try:
        fn = WORKLOADS[args.workload]
        line = fn(args, world, rank, local, td)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if td is not None:
            td.destroy_process_group()


if __name__ == "__main__":
    main()
