"""A trajectory set split across ranks by contiguous id ranges (gat_b200.shard): the host merge of
per-shard top-k lists (gat_topk_merge) equals the unsharded top-k of the oracle, shards with
fewer than k trajectories included; two gloo ranks on CPU exchange their shards' top-k lists
and range id sets and both obtain the unsharded results."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gat_b200 import _lib as L
from gat_b200 import data as D
from gat_b200 import shard as S
from oracle import pyoracle as po

CELL, EPS, K = 0.01, 5e-4, 6


def _set():
    return D.walks(D.lengths(240, 0, 0, 0, 5, 60, 81), 81)


def _queries(t):
    return [t.points(i) for i in (3, 77, 200)]


def shard_topk(t, lo, hi, q, k=K):
    """oracle top-k of each query over trajectories lo..hi-1, with global ids"""
    sub = t.subset(np.arange(lo, hi))
    o = po.OracleGrid(sub, D.BOX, CELL, 2, 512)
    ids, dist = [], []
    for lon, lat in q:
        i, d, _ = o.topk(lon, lat, k, EPS, pruned=False)
        ids.append(np.where(i > 0, i + lo - 1, -1))
        dist.append(d)
    return np.array(ids, np.int32), np.array(dist, np.int32)


def test_shard_bounds():
    for n, w in ((10, 3), (7, 7), (5, 8), (240, 2)):
        b = S.shard_bounds(n, w)
        assert len(b) == w and b[0][0] == 1 and b[-1][1] == n + 1
        assert all(b[i][1] == b[i + 1][0] for i in range(w - 1))
        assert max(h - l for l, h in b) - min(h - l for l, h in b) <= 1


def test_host_merge_equals_unsharded():
    t = _set()
    q = _queries(t)
    want = shard_topk(t, 1, t.n + 1, q)
    for bounds in (S.shard_bounds(t.n, 3), [(1, 4), (4, 200), (200, 241)]):  # (1, 4): fewer than k
        parts = [shard_topk(t, lo, hi, q) for lo, hi in bounds]
        ids, dist = S.merge_topk_host(np.stack([p[0] for p in parts]), np.stack([p[1] for p in parts]))
        assert np.array_equal(ids, want[0]) and np.array_equal(dist, want[1])
    # a set smaller than k pads with (-1, -1), as gat_topk does
    small = shard_topk(t, 1, 3, q, k=4)
    ids, dist = S.merge_topk_host(small[0][None], small[1][None])
    assert (ids[:, 2:] == -1).all() and (dist[:, 2:] == -1).all()
    assert L.lib.gat_topk_merge(1, 4, 3000, None, None, None, None) == L.GAT_ERR_ARG  # nparts x k > 8192


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as td

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t = _set()
    q = _queries(t)
    lo, hi = S.shard_bounds(t.n, world)[rank]
    ids, dist = S.gather_topk(*shard_topk(t, lo, hi, q))
    boxes = D.boxes(20, 1, 0.002, 0.05, 82)
    sub = t.subset(np.arange(lo, hi))
    off, rids = po.OracleGrid(sub, D.BOX, CELL, 2, 512).range(boxes, 0)
    rr = S.gather_ranges(off, np.asarray(rids) + lo - 1)
    out.put((rank, ids.tolist(), dist.tolist(), rr.offsets.tolist(), rr.tids.tolist()))
    td.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    t = _set()
    want = shard_topk(t, 1, t.n + 1, _queries(t))
    woff, wids = po.OracleGrid(t, D.BOX, CELL, 2, 512).range(D.boxes(20, 1, 0.002, 0.05, 82), 0)
    for rank, ids, dist, roff, rids in got:
        assert np.array_equal(ids, want[0]) and np.array_equal(dist, want[1])
        assert np.array_equal(roff, woff) and np.array_equal(rids, wids)
