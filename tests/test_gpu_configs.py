"""GPU results at the full sizes the benchmark times, against the oracle (and the reference's own
compiled CPU code where it is built):

* config 2: the 100k-walk set (lognormal lengths 32..1024), 8 of its 256 query trajectories,
  k = 32, eps 5e-4, frequency vectors on 256 x 256 virtual cells; ids and distances equal the
  oracle's exhaustive ranking in both execution forms, and the distance multisets equal the
  reference's Grid::SimilarityQueryBatchCPUParallel (Grid.cpp:1133);
* config 3: the 1M-walk set (200M points) and 250 of its 100k rectangles, trajectory-id sets of
  the GT-quadtree, FSG and STIG equal the oracle's (Grid.cpp:341-405, FSG.cpp:145-393,
  STIG.cpp:179-338), batched and plain.

Both build large host-side oracles (about a minute each)."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import gat_b200 as G
from gat_b200 import data as D
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

EPS = 5e-4


def _cores():
    import os

    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def test_topk_on_the_100k_set(gpu_ctx):
    t, qids = D.config2(seed=0, n=100_000, nq=256)
    sel = qids[::32]
    k = 32
    db = G.TrajectorySet(gpu_ctx, t)
    g = G.Grid(gpu_ctx, db, G.BOX, 0.0025, 2, 512)
    q = t.subset(sel)
    got = {ex: g.topk(q, k, EPS, execution=ex)[:2] for ex in ("plain", "batched")}
    o = po.OracleGrid(t, G.BOX, 0.0025, 2, 512)
    for j, qid in enumerate(sel):
        wi, wd, _ = o.topk(*t.points(int(qid)), k, EPS, pruned=False, threads=_cores())
        for ex, (ids, dist) in got.items():
            assert np.array_equal(ids[j], wi), f"{ex}: ids of query {qid}"
            assert np.array_equal(dist[j], wd), f"{ex}: distances of query {qid}"
    if po.ref_available():
        r = po.RefRunner().topk(t, sel, G.BOX, 0.0025, k, EPS)
        for j in range(len(sel)):
            assert np.array_equal(np.sort(r["dist"][j]), got["plain"][1][j])
    g.close()
    db.close()


def test_ranges_on_the_1m_set(gpu_ctx):
    t, q = D.config3(seed=0, n=1_000_000, nq=100_000)
    sel = np.arange(0, 100_000, 400)
    qs = q[sel]
    with ThreadPoolExecutor(max_workers=3) as ex:
        fut = {"grid": ex.submit(po.OracleGrid, t, G.BOX, 0.001, 2, 512),
               "fsg": ex.submit(po.OracleFSG, t, G.BOX, 0.001),
               "stig": ex.submit(po.OracleSTIG, t, 10240)}
        db = G.TrajectorySet(gpu_ctx, t)
        ix = {"grid": G.Grid(gpu_ctx, db, G.BOX, 0.001, 2, 512), "fsg": G.FSG(gpu_ctx, db, G.BOX, 0.001),
              "stig": G.STIG(gpu_ctx, db, 10240)}
        oracle = {k: f.result() for k, f in fut.items()}
    for name in ("grid", "fsg", "stig"):
        off, ids = oracle[name].range(qs)
        r = ix[name].range_query(qs)
        assert np.array_equal(r.offsets, off) and np.array_equal(r.tids, ids), f"{name} batched"
        r = ix[name].range_query(qs[:40], execution="plain")
        n40 = int(off[40])
        assert np.array_equal(r.offsets, off[:41]) and np.array_equal(r.tids, ids[:n40]), f"{name} plain"
    for v in ix.values():
        v.close()
    db.close()
