"""FV lower bounds and top-k on the GPU against the oracle (FVTable.cpp:77-207 and an
exhaustive (distance, id) ranking over Grid::SimilarityExecuter)."""
import numpy as np
import pytest

import gat_b200 as G
from gat_b200 import data as D
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(gpu_ctx):
    t = D.walks(D.lengths(6000, 1, float(np.log(200.0)), 0.6, 32, 1024, 3), 3)
    db = G.TrajectorySet(gpu_ctx, t)
    g = G.Grid(gpu_ctx, db, D.BOX, 0.0025, 2, 512)
    o = po.OracleGrid(t, D.BOX, 0.0025, 2, 512)
    qids = D.sample_ids(12, t.n, 4)
    return t, g, o, qids


def test_lower_bounds(small):
    t, g, o, qids = small
    q = t.subset(qids)
    lb = g.fv_lower_bounds(q)
    for j, qid in enumerate(qids):
        lon, lat = t.points(int(qid))
        want = o.fv_lb(lon, lat)
        assert np.array_equal(lb[j, 1:], want[1:])


@pytest.mark.parametrize("execution", ["batched", "plain"])
@pytest.mark.parametrize("k", [1, 5, 32])
def test_topk_matches_exhaustive(small, execution, k):
    t, g, o, qids = small
    q = t.subset(qids)
    ids, dist, stats = g.topk(q, k, 5e-4, execution)
    for j, qid in enumerate(qids):
        lon, lat = t.points(int(qid))
        wi, wd, _ = o.topk(lon, lat, k, 5e-4, pruned=False)
        assert np.array_equal(dist[j], wd), (j, dist[j], wd)
        assert np.array_equal(ids[j], wi), (j, ids[j], wi)
    assert stats["pairs"] > 0 and stats["cells"] > 0


def test_topk_external_queries_and_big_eps(small):
    """queries that are not in the set (lengths 16..900) and a coarse eps = 0.005"""
    t, g, o, _ = small
    q = D.walks(D.lengths(6, 2, 0, 0, 16, 900, 9), 9)
    ids, dist, _ = g.topk(q, 8, 0.005)
    for j in range(q.n):
        lon, lat = q.points(j + 1)
        wi, wd, _ = o.topk(lon, lat, 8, 0.005, pruned=False)
        assert np.array_equal(dist[j], wd) and np.array_equal(ids[j], wi)


def test_k_larger_than_set(gpu_ctx):
    t = D.walks(D.lengths(20, 0, 0, 0, 5, 30, 12), 12)
    db = G.TrajectorySet(gpu_ctx, t)
    g = G.Grid(gpu_ctx, db, D.BOX, 0.0025, 2, 512)
    o = po.OracleGrid(t, D.BOX, 0.0025, 2, 512)
    q = t.subset([3])
    ids, dist, _ = g.topk(q, 25, 5e-4)
    wi, wd, _ = o.topk(*t.points(3), 25, 5e-4, pruned=False)
    assert np.array_equal(ids[0], wi) and np.array_equal(dist[0], wd)
    assert np.all(ids[0, 20:] == -1)


def test_long_queries_against_short_set(gpu_ctx):
    """Query walks up to 4096 points (the pair lengths of the batched-EDR configuration) against
    a set of shorter walks (U[50, 350], the batched-range configuration's set): the walk's
    bound order and stop rule with k = 64, batched and plain, against the oracle."""
    t = D.walks(D.lengths(20000, 0, 0, 0, 50, 350, 44), 44)
    db = G.TrajectorySet(gpu_ctx, t)
    g = G.Grid(gpu_ctx, db, D.BOX, 0.0025, 2, 512)
    o = po.OracleGrid(t, D.BOX, 0.0025, 2, 512)
    ql = np.concatenate([[4096, 16], D.lengths(4, 2, 0, 0, 16, 4096, 45)]).astype(np.int32)
    qs = D.walks(ql, 46)
    for execution in ("batched", "plain"):
        ids, dist, _ = g.topk(qs, 64, 5e-4, execution=execution)
        for j in range(qs.n):
            wi, wd, _ = o.topk(*qs.points(j + 1), 64, 5e-4)
            assert np.array_equal(ids[j], wi) and np.array_equal(dist[j], wd), (execution, j, int(ql[j]))


def test_plain_graph_matches_stream_path(gpu_ctx, small):
    """The plain form runs each query as one launch of a CUDA graph (rounds in a device-side
    loop); with per-kernel timing on, the same kernels are launched one by one. Both, over
    repeated calls (graph reuse), several k (several cached graphs, one evicted) and a single
    query (the uncaptured sizing run only), equal the batched form."""
    t, g, o, qids = small
    q = t.subset(qids)
    for k in (4, 16, 8, 16):
        b_ids, b_d, _ = g.topk(q, k, 5e-4, execution="batched")
        p_ids, p_d, st = g.topk(q, k, 5e-4, execution="plain")
        assert np.array_equal(p_ids, b_ids) and np.array_equal(p_d, b_d), k
        assert st["launches"] > 0 and st["pairs"] > 0
    gpu_ctx.set_timing(True)
    try:
        s_ids, s_d, _ = g.topk(q, 16, 5e-4, execution="plain")
    finally:
        gpu_ctx.set_timing(False)
    b_ids, b_d, _ = g.topk(q, 16, 5e-4, execution="batched")
    assert np.array_equal(s_ids, b_ids) and np.array_equal(s_d, b_d)
    one = t.subset(qids[:1])
    i1, d1, _ = g.topk(one, 5, 5e-4, execution="plain")
    assert np.array_equal(i1[0], b_ids[0, :5]) and np.array_equal(d1[0], b_d[0, :5])


def test_dependent_launch_does_not_change_results(gpu_ctx, small):
    """GAT_TUNE_DEP_LAUNCH 0 (plain launches) and 1 (programmatic dependent launches) give the
    same top-k lists in the plain graph and batched forms, and the same EDR of pairs."""
    from gat_b200 import _lib as L

    t, g, o, qids = small
    q = t.subset(qids)
    res = {}
    try:
        for dep in (0, 1):
            gpu_ctx.set_tuning(L.GAT_TUNE_DEP_LAUNCH, dep)
            assert gpu_ctx.tuning(L.GAT_TUNE_DEP_LAUNCH) == dep
            res[dep] = [g.topk(q, 16, 5e-4, execution=e)[:2] for e in ("plain", "batched", "plain")]
            la, a, lb, b = D.config4_pairs(seed=3, npairs=64, lo=16, hi=600)
            res[dep].append((G.api.edr_pairs(gpu_ctx, la, a, lb, b, 5e-4),))
    finally:
        gpu_ctx.set_tuning(L.GAT_TUNE_DEP_LAUNCH, 1)
    for x, y in zip(res[0], res[1]):
        for u, v in zip(x, y):
            assert np.array_equal(u, v)

