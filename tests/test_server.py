"""Serving loop host logic on a host-only context: request lifecycle, admission by the memory
budget, errors. (Execution needs a GPU; on a host-only context every admitted batch reports
GAT_ERR_STATE, which exercises the same scheduling and completion paths.)"""
import threading

import numpy as np
import pytest

import gat_b200 as G
from gat_b200 import _lib as L
from gat_b200 import data as D


@pytest.fixture(scope="module")
def host_indexes(host_ctx):
    t = D.walks(D.lengths(500, 0, 0, 0, 10, 60, 81), 81)
    db = G.TrajectorySet(host_ctx, t)
    return t, G.Grid(host_ctx, db, D.BOX, 0.01), G.STIG(host_ctx, db, 64), G.FSG(host_ctx, db, D.BOX, 0.01)


def test_lifecycle_host_only(host_ctx, host_indexes):
    t, g, s, f = host_indexes
    srv = G.Server(host_ctx, g, s, f, lanes=3, budget_bytes=1 << 30, max_range_batch=8, max_topk_batch=2)
    boxes = D.boxes(40, 1, 0.002, 0.05, 82)
    ids = []

    def submit(lo, hi):
        for i in range(lo, hi):
            ids.append(srv.submit_range(boxes[i], index_kind=i % 3, result="ids" if i % 2 else "points"))

    th = [threading.Thread(target=submit, args=(a, a + 20)) for a in (0, 20)]
    [x.start() for x in th]
    [x.join() for x in th]
    lon, lat = t.points(3)
    tk = [srv.submit_topk(lon, lat, 5, 5e-4) for _ in range(3)]
    for r in ids + tk:
        assert srv.wait(r, 10000) == L.GAT_ERR_STATE  # host-only: no device
        a, b, c = srv.times(r)
        assert 0 <= a <= b <= c
    st = srv.stats()
    assert st["submitted"] == st["completed"] == 43 and st["failed"] == 43
    assert 1 <= st["batches"] <= 43 and st["largest_batch"] <= 8
    for r in ids:
        srv.release(r)
    with pytest.raises(G.GatError):
        srv.release(ids[0])  # already released
    with pytest.raises(G.GatError):
        srv.wait(10 ** 9, 10)  # unknown id
    srv.close()


def test_budget_rejects_oversize(host_ctx, host_indexes):
    t, g, s, f = host_indexes
    # a top-k request reserves 32 bytes per trajectory + 64 KB: more than this budget
    srv = G.Server(host_ctx, g, None, None, lanes=1, budget_bytes=32 << 10)
    lon, lat = t.points(7)
    r = srv.submit_topk(lon, lat, 3, 5e-4)
    assert srv.wait(r, 10000) == L.GAT_ERR_OOM
    with pytest.raises(G.GatError):
        srv.topk_result(r, 3)
    with pytest.raises(G.GatError) as e:
        srv.submit_range((121, 31, 121.1, 31.1), index_kind=L.GAT_INDEX_STIG)  # no STIG given
    assert e.value.status == L.GAT_ERR_ARG
    with pytest.raises(G.GatError):
        srv.submit_topk(lon, lat, 0, 5e-4)
    srv.close()


def test_config_errors(host_ctx, host_indexes):
    t, g, s, f = host_indexes
    for kw in (dict(lanes=0), dict(budget_bytes=0), dict(max_range_batch=0), dict(max_topk_batch=0)):
        with pytest.raises(G.GatError):
            G.Server(host_ctx, g, s, f, **kw)
    with pytest.raises(G.GatError):
        G.Server(host_ctx, s, None, None)  # a STIG where the grid belongs
