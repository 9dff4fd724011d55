"""Multi-GPU runs are replicas (the hot paths shard by query with no exchange step). The host
logic bench.py uses for N > 1 (rank discovery, per-rank query samples, barrier and max-over-
ranks device time) is exercised here with two gloo ranks on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as td

    import bench
    from gat_b200 import data as D

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    td.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    w, r, loc = bench.dist_env()
    qids = D.sample_ids(16, 1000, 1000 + r)
    mine = float(10.0 + r)
    worst = bench.max_over_ranks(td, mine, torch.device("cpu"))
    bench.barrier(td)
    q.put((r, w, worst, sorted(qids.tolist())))
    td.destroy_process_group()


def test_two_rank_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [2, 2]
    assert out[0][2] == out[1][2] == 11.0  # max over ranks
    assert out[0][3] != out[1][3]  # each replica has its own queries
