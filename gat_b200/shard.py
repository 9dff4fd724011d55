"""A trajectory set split across the ranks of a torch.distributed process group.

Rank r of W keeps the contiguous id range `shard_bounds(n, W)[r]` of the set and builds its own
GT-quadtree over it. A top-k query runs on every shard, one all-gather exchanges each shard's k
(distance, id) pairs per query, and `gat_topk_merge_dev` (NCCL, device buffers) or
`gat_topk_merge` (other backends, host buffers) keeps the k smallest: the unsharded result,
since every shard's list holds its own k best in the canonical (distance, id) order. Range
queries gather each shard's id sets, which are disjoint and increase with the rank, and
concatenate them per query.

The reference's two-GPU mode (Grid.cpp:1758-2332) splits the queries, not the set; a split by
queries needs no exchange and is what `bench.py --gpus N` runs (replicas).
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .api import Context, Grid, RangeResult, TrajectorySet, _p
from .data import Trajectories

lib = L.lib


def shard_bounds(n: int, world: int) -> list[tuple[int, int]]:
    """Contiguous 1-based id ranges [lo, hi) of n trajectories over `world` shards."""
    per, extra = divmod(n, world)
    out, lo = [], 1
    for r in range(world):
        hi = lo + per + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def merge_topk_host(ids: np.ndarray, dist: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """[nparts, nq, k] per-shard lists (global ids) -> the merged [nq, k] lists (gat_topk_merge)."""
    ids = np.ascontiguousarray(ids, np.int32)
    dist = np.ascontiguousarray(dist, np.int32)
    nparts, nq, k = ids.shape
    oi, od = np.zeros((nq, k), np.int32), np.zeros((nq, k), np.int32)
    rc = lib.gat_topk_merge(nq, k, nparts, _p(ids, L.P_i32), _p(dist, L.P_i32), _p(oi, L.P_i32), _p(od, L.P_i32))
    if rc != L.GAT_OK:
        raise RuntimeError(f"gat_topk_merge failed with status {rc}")
    return oi, od


def merge_topk_device(ctx: Context, ids, dist):
    """Device form: torch int32 CUDA tensors [nparts, nq, k] -> merged [nq, k] (gat_topk_merge_dev)."""
    import torch

    nparts, nq, k = ids.shape
    ids, dist = ids.contiguous(), dist.contiguous()
    oi = torch.empty((nq, k), dtype=torch.int32, device=ids.device)
    od = torch.empty((nq, k), dtype=torch.int32, device=ids.device)
    stream = torch.cuda.current_stream(ids.device)
    stream.synchronize()  # the gathered lists were written on torch's stream
    ctx.check(lib.gat_topk_merge_dev(ctx.h, nq, k, nparts, ids.data_ptr(), dist.data_ptr(), oi.data_ptr(), od.data_ptr()),
              "gat_topk_merge_dev")
    ctx.check(lib.gat_ctx_sync(ctx.h), "gat_ctx_sync")
    return oi, od


def gather_topk(ids: np.ndarray, dist: np.ndarray, group=None, ctx: Context | None = None):
    """This rank's [nq, k] top-k (global ids) -> the merged [nq, k] over all ranks. With an NCCL
    group (and ctx) the exchange and the merge run on the device; otherwise on the host."""
    import torch
    import torch.distributed as td

    world = td.get_world_size(group)
    ids = np.ascontiguousarray(ids, np.int32)
    dist = np.ascontiguousarray(dist, np.int32)
    nq, k = ids.shape
    if td.get_backend(group) == "nccl":
        if ctx is None:
            raise ValueError("an NCCL group needs the context whose device holds the shard")
        dev = torch.device("cuda", ctx.device)
        mine = torch.from_numpy(np.stack([ids, dist])).to(dev)
        allv = torch.empty((world, 2, nq, k), dtype=torch.int32, device=dev)
        td.all_gather_into_tensor(allv, mine, group=group)
        oi, od = merge_topk_device(ctx, allv[:, 0], allv[:, 1])
        return oi.cpu().numpy(), od.cpu().numpy()
    mine = torch.from_numpy(np.stack([ids, dist]))
    parts = [torch.empty_like(mine) for _ in range(world)]
    td.all_gather(parts, mine, group=group)
    allv = torch.stack(parts).numpy()
    return merge_topk_host(allv[:, 0], allv[:, 1])


def gather_ranges(offsets: np.ndarray, tids: np.ndarray, group=None, device=None) -> RangeResult:
    """This rank's range result (CSR over queries, global ids) -> the union over all ranks: per
    query the ranks' ids concatenated in rank order, which keeps them sorted."""
    import torch
    import torch.distributed as td

    world = td.get_world_size(group)
    offsets = np.asarray(offsets, np.int64)
    tids = np.asarray(tids, np.int32)
    nq = len(offsets) - 1
    dev = device if device is not None else torch.device("cpu")
    counts = torch.from_numpy(np.diff(offsets)).to(dev)
    all_counts = [torch.empty_like(counts) for _ in range(world)]
    td.all_gather(all_counts, counts, group=group)
    totals = [int(c.sum()) for c in all_counts]
    width = max(1, max(totals))
    mine = torch.full((width,), -1, dtype=torch.int32, device=dev)
    if len(tids):
        mine[: len(tids)] = torch.from_numpy(tids).to(dev)
    all_ids = [torch.empty_like(mine) for _ in range(world)]
    td.all_gather(all_ids, mine, group=group)
    cnt = np.stack([c.cpu().numpy() for c in all_counts])  # [world, nq]
    ids = np.concatenate([all_ids[r].cpu().numpy()[: totals[r]] for r in range(world)])
    query = np.concatenate([np.repeat(np.arange(nq), cnt[r]) for r in range(world)])
    # a stable sort by query keeps the ranks in order within each query
    out = ids[np.argsort(query, kind="stable")].astype(np.int32)
    out_off = np.zeros(nq + 1, np.int64)
    out_off[1:] = np.cumsum(cnt.sum(axis=0))
    return RangeResult(out_off, out, None)


class ShardedGrid:
    """The GT-quadtree over this rank's contiguous share of a trajectory set; queries answer over
    the whole set. Every rank must make the same calls in the same order (they exchange data)."""

    def __init__(self, ctx: Context, traj: Trajectories, box, cell_size: float, virtual_cell_param: int = 2,
                 leaf_cap: int = 512, group=None):
        import torch.distributed as td

        self.ctx, self.group = ctx, group
        world, rank = td.get_world_size(group), td.get_rank(group)
        self.n = traj.n
        self.lo, self.hi = shard_bounds(traj.n, world)[rank]
        self.offset = self.lo - 1  # local id + offset = global id
        self.shard = traj.subset(np.arange(self.lo, self.hi))
        self.db = TrajectorySet(ctx, self.shard)
        self.grid = Grid(ctx, self.db, box, cell_size, virtual_cell_param, leaf_cap)

    def topk(self, queries: Trajectories, k: int, eps: float, execution: str = "batched"):
        """(ids, dist): the k nearest trajectories of the whole set per query, sorted by
        (distance, id), equal to gat_topk over the unsharded set."""
        ids, dist, _ = self.grid.topk(queries, k, eps, execution)
        ids = np.where(ids > 0, ids + self.offset, -1).astype(np.int32)
        return gather_topk(ids, dist, self.group, self.ctx)

    def range_query(self, queries) -> RangeResult:
        """Trajectory-id sets over the whole set (sorted per query)."""
        import torch
        import torch.distributed as td

        r = self.grid.range_query(queries)
        dev = torch.device("cuda", self.ctx.device) if td.get_backend(self.group) == "nccl" else None
        return gather_ranges(r.offsets, r.tids + self.offset, self.group, dev)

    def close(self):
        self.grid.close()
        self.db.close()
