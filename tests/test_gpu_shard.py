"""Sharded sets on the GPU: per-shard gat_topk lists (ids made global) merged on the device
(gat_topk_merge_dev) equal the unsharded gat_topk and the host merge; a ShardedGrid in an NCCL
group of one rank answers top-k and range queries like the unsharded Grid. Two or more GPUs are
not available to these tests; the exchange between ranks is covered on CPU (test_shard.py)."""
import datetime
import socket

import numpy as np
import pytest

import gat_b200 as G
from gat_b200 import data as D
from gat_b200 import shard as S

pytestmark = pytest.mark.gpu


def test_device_merge_equals_unsharded(gpu_ctx):
    import torch

    t = D.walks(D.lengths(6000, 0, 0, 0, 20, 300, 83), 83)
    q = t.subset([5, 1000, 4321, 5999])
    full = G.Grid(gpu_ctx, G.TrajectorySet(gpu_ctx, t), D.BOX, 0.0025, 2, 512)
    for k in (1, 8, 64):
        want_i, want_d, _ = full.topk(q, k, 5e-4)
        ids, dist = [], []
        for lo, hi in S.shard_bounds(t.n, 3):
            db = G.TrajectorySet(gpu_ctx, t.subset(np.arange(lo, hi)))
            g = G.Grid(gpu_ctx, db, D.BOX, 0.0025, 2, 512)
            i, d, _ = g.topk(q, k, 5e-4)
            ids.append(np.where(i > 0, i + lo - 1, -1))
            dist.append(d)
            g.close()
            db.close()
        ids, dist = np.stack(ids).astype(np.int32), np.stack(dist).astype(np.int32)
        di, dd = S.merge_topk_device(gpu_ctx, torch.from_numpy(ids).cuda(), torch.from_numpy(dist).cuda())
        assert np.array_equal(di.cpu().numpy(), want_i) and np.array_equal(dd.cpu().numpy(), want_d)
        hi_, hd = S.merge_topk_host(ids, dist)
        assert np.array_equal(hi_, want_i) and np.array_equal(hd, want_d)


def test_sharded_grid_in_nccl_group_of_one(gpu_ctx):
    import torch.distributed as td

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    td.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                          timeout=datetime.timedelta(seconds=60))
    try:
        t = D.walks(D.lengths(3000, 0, 0, 0, 20, 300, 84), 84)
        sg = S.ShardedGrid(gpu_ctx, t, D.BOX, 0.0025, 2, 512)
        full = G.Grid(gpu_ctx, G.TrajectorySet(gpu_ctx, t), D.BOX, 0.0025, 2, 512)
        q = t.subset([1, 2999, 1500])
        i1, d1 = sg.topk(q, 16, 5e-4)
        i2, d2, _ = full.topk(q, 16, 5e-4)
        assert np.array_equal(i1, i2) and np.array_equal(d1, d2)
        boxes = D.boxes(50, 1, 0.002, 0.05, 85)
        a, b = sg.range_query(boxes), full.range_query(boxes)
        assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.tids, b.tids)
        sg.close()
    finally:
        td.destroy_process_group()
