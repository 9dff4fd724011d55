"""Serving loop on the GPU: a mix of range requests (three indexes, both result kinds) and
top-k requests of different lengths and k, submitted from two threads and run with continuous
batching on three lanes, gives for every request exactly the result of the same request run
alone; a sample is checked against the oracle; a tight budget still completes everything
without admitting more than it allows."""
import threading

import numpy as np
import pytest

import gat_b200 as G
from gat_b200 import _lib as L
from gat_b200 import data as D
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(gpu_ctx):
    t = D.walks(D.lengths(20000, 0, 0, 0, 20, 200, 91), 91)
    db = G.TrajectorySet(gpu_ctx, t)
    g = G.Grid(gpu_ctx, db, D.BOX, 0.0025, 2, 512)
    s = G.STIG(gpu_ctx, db, 256)
    f = G.FSG(gpu_ctx, db, D.BOX, 0.01)
    rng = np.random.default_rng(92)
    boxes = D.boxes(300, 1, 0.001, 0.05, 93)
    ql = D.lengths(24, 2, 0, 0, 16, 512, 94)
    qs = D.walks(ql, 95)
    ks = rng.integers(4, 33, size=24)
    kinds = rng.integers(0, 3, size=300)
    res = rng.integers(0, 2, size=300)
    return t, g, s, f, boxes, qs, ks, kinds, res


def _submit_all(srv, boxes, qs, ks, kinds, res):
    """300 range and 24 top-k requests, interleaved, submitted from two threads."""
    plan = []
    for i in range(300):
        plan.append(("r", i))
        if i % 12 == 5 and i // 12 < 24:
            plan.append(("t", i // 12))
    out = {}
    lock = threading.Lock()

    def worker(part):
        for key in plan[part::2]:
            if key[0] == "r":
                i = key[1]
                r = srv.submit_range(boxes[i], int(kinds[i]), "points" if res[i] else "ids")
            else:
                lon, lat = qs.points(key[1] + 1)
                r = srv.submit_topk(lon, lat, int(ks[key[1]]), 5e-4)
            with lock:
                out[key] = r

    th = [threading.Thread(target=worker, args=(p,)) for p in (0, 1)]
    [x.start() for x in th]
    [x.join() for x in th]
    assert len(out) == len(plan) == 324
    return out


def _collect(srv, ids, ks, res):
    got = {}
    for key, r in ids.items():
        assert srv.wait(r, 600000) == L.GAT_OK
        if key[0] == "r":
            got[key] = srv.range_result(r, points=bool(res[key[1]]))
        else:
            got[key] = srv.topk_result(r, int(ks[key[1]]))
    return got


def test_mix_equals_alone(gpu_ctx, setup):
    t, g, s, f, boxes, qs, ks, kinds, res = setup
    idx = {0: g, 1: s, 2: f}
    srv = G.Server(gpu_ctx, g, s, f, lanes=3, budget_bytes=4 << 30, max_range_batch=64, max_topk_batch=4)
    ids = _submit_all(srv, boxes, qs, ks, kinds, res)
    got = _collect(srv, ids, ks, res)
    st = srv.stats()
    assert st["completed"] == st["submitted"] == len(ids) and st["failed"] == 0
    assert st["batches"] < len(ids) and st["peak_admitted_bytes"] <= 4 << 30
    # alone, through the server (one request in flight) and through the direct call
    for key in list(got)[::7]:
        if key[0] == "r":
            i = key[1]
            r = srv.submit_range(boxes[i], int(kinds[i]), "points" if res[i] else "ids")
            assert srv.wait(r) == L.GAT_OK
            alone = srv.range_result(r, points=bool(res[i]))
            direct = idx[int(kinds[i])].range_query(boxes[i:i + 1], result="points" if res[i] else "ids")
            if res[i]:
                assert np.array_equal(got[key][0], alone[0]) and np.array_equal(got[key][1], alone[1])
                assert np.array_equal(got[key][0], direct.tids) and np.array_equal(got[key][1], direct.pidx)
            else:
                assert np.array_equal(got[key], alone) and np.array_equal(got[key], direct.tids)
        else:
            j = key[1]
            lon, lat = qs.points(j + 1)
            r = srv.submit_topk(lon, lat, int(ks[j]), 5e-4)
            assert srv.wait(r) == L.GAT_OK
            a_ids, a_d = srv.topk_result(r, int(ks[j]))
            d_ids, d_d, _ = g.topk(qs.subset([j + 1]), int(ks[j]), 5e-4)
            assert np.array_equal(got[key][0], a_ids) and np.array_equal(got[key][1], a_d)
            assert np.array_equal(a_ids, d_ids[0]) and np.array_equal(a_d, d_d[0])
    srv.close()
    # a sample against the oracle
    og = po.OracleGrid(t, D.BOX, 0.0025, 2, 512)
    for i in range(0, 300, 37):
        if kinds[i] == 0:
            off, want = og.range(boxes[i:i + 1], 1 if res[i] else 0)[:2]
            have = got[("r", i)][0] if res[i] else got[("r", i)]
            assert np.array_equal(have, want)
    for j in (0, 5):
        wi, wd, _ = og.topk(*qs.points(j + 1), int(ks[j]), 5e-4)
        assert np.array_equal(got[("t", j)][0], wi) and np.array_equal(got[("t", j)][1], wd)


def test_tight_budget_serialises(gpu_ctx, setup):
    t, g, s, f, boxes, qs, ks, kinds, res = setup
    one = 20000 * 32 + (64 << 10)  # one top-k request's reservation
    srv = G.Server(gpu_ctx, g, None, None, lanes=4, budget_bytes=int(one * 1.5), max_topk_batch=8)
    rs = []
    for j in range(6):
        lon, lat = qs.points(j + 1)
        rs.append(srv.submit_topk(lon, lat, int(ks[j]), 5e-4))
    for j, r in enumerate(rs):
        assert srv.wait(r) == L.GAT_OK
        ids, d = srv.topk_result(r, int(ks[j]))
        d_ids, d_d, _ = g.topk(qs.subset([j + 1]), int(ks[j]), 5e-4)
        assert np.array_equal(ids, d_ids[0]) and np.array_equal(d, d_d[0])
    st = srv.stats()
    assert st["peak_admitted_bytes"] <= int(one * 1.5) and st["largest_batch"] == 1
    srv.close()
