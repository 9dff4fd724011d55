"""Range queries on the GPU against the oracle (Grid.cpp:341-405 restated), all three indexes,
plain and batched execution, id sets and point lists. Bit-exact: integer results."""
import numpy as np
import pytest

import gat_b200 as G
from gat_b200 import data as D
from oracle import pyoracle as po
from tests.conftest import csr_equal

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1(gpu_ctx):
    """config-1 shaped: 10k walks U[20,200], leaf cap 512, CELL_LEN 0.01; mixed query sizes."""
    t, q = D.config1(seed=0)
    q2 = D.boxes(500, 1, 0.001, 0.05, 11)  # uneven selectivity, some boxes cross the grid edge
    edge = np.array([[121.0, 30.7, 121.01, 30.71], [121.995, 31.69, 122.05, 31.8], [120.9, 30.6, 121.2, 30.75],
                     [121.5, 31.2, 121.5, 31.2], [121.3, 31.0, 121.3000001, 31.4], [122.5, 32.0, 122.6, 32.1]],
                    np.float32)
    qs = np.concatenate([q, q2, edge])
    db = G.TrajectorySet(gpu_ctx, t)
    return t, qs, db


@pytest.mark.parametrize("execution", ["batched", "plain"])
def test_grid_ids(gpu_ctx, c1, execution):
    t, q, db = c1
    g = G.Grid(gpu_ctx, db, D.BOX, 0.01, 2, 512)
    o = po.OracleGrid(t, D.BOX, 0.01, 2, 512)
    qq = q if execution == "batched" else q[::7]
    r = g.range_query(qq, "ids", execution)
    off, ids = o.range(qq, 0)
    assert csr_equal(r.offsets, r.tids, off, ids)
    assert gpu_ctx.launches > 0


@pytest.mark.parametrize("execution", ["batched", "plain"])
def test_grid_points(gpu_ctx, c1, execution):
    t, q, db = c1
    g = G.Grid(gpu_ctx, db, D.BOX, 0.01, 2, 512)
    o = po.OracleGrid(t, D.BOX, 0.01, 2, 512)
    qq = q if execution == "batched" else q[::9]
    r = g.range_query(qq, "points", execution)
    off, tid, pidx = o.range(qq, 1)
    assert csr_equal(r.offsets, r.tids, off, tid)
    assert np.array_equal(r.pidx, pidx)


@pytest.mark.parametrize("result", ["ids", "points"])
def test_stig(gpu_ctx, c1, result):
    t, q, db = c1
    s = G.STIG(gpu_ctx, db, 512)
    o = po.OracleSTIG(t, 512)
    r = s.range_query(q, result)
    ref = o.range(q, 0 if result == "ids" else 1)
    assert csr_equal(r.offsets, r.tids, ref[0], ref[1])
    if result == "points":
        assert np.array_equal(r.pidx, ref[2])


@pytest.mark.parametrize("result", ["ids", "points"])
def test_fsg(gpu_ctx, c1, result):
    t, q, db = c1
    f = G.FSG(gpu_ctx, db, D.BOX, 0.01)
    o = po.OracleFSG(t, D.BOX, 0.01)
    r = f.range_query(q, result)
    ref = o.range(q, 0 if result == "ids" else 1)
    assert csr_equal(r.offsets, r.tids, ref[0], ref[1])
    if result == "points":
        assert np.array_equal(r.pidx, ref[2])


def test_empty_and_single(gpu_ctx, c1):
    t, q, db = c1
    g = G.Grid(gpu_ctx, db, D.BOX, 0.01, 2, 512)
    r = g.range_query(np.zeros((0, 4), np.float32))
    assert r.offsets.tolist() == [0] and len(r.tids) == 0
    far = np.array([[10.0, 10.0, 11.0, 11.0]], np.float32)
    r = g.range_query(far)
    assert r.offsets.tolist() == [0, 0]


def test_truncation_reports_needed(gpu_ctx, c1):
    t, q, db = c1
    g = G.Grid(gpu_ctx, db, D.BOX, 0.01, 2, 512)
    full = g.range_query(q[:50])
    with pytest.raises(G.GatError) as e:
        g.range_query(q[:50], capacity=max(0, len(full.tids) - 1))
    assert e.value.status == 4


def test_tiny_leaf_cap_and_single_leaf(gpu_ctx):
    """leaf cap 1 drives every node to the maximum level; a huge cap keeps the root a leaf."""
    t = D.walks(D.lengths(300, 0, 0, 0, 1, 40, 5), 5)
    q = D.boxes(100, 1, 0.001, 0.2, 6)
    db = G.TrajectorySet(gpu_ctx, t)
    for cap in (1, 10_000_000):
        g = G.Grid(gpu_ctx, db, D.BOX, 0.02, 2, cap)
        o = po.OracleGrid(t, D.BOX, 0.02, 2, cap)
        r = g.range_query(q)
        off, ids = o.range(q, 0)
        assert csr_equal(r.offsets, r.tids, off, ids)


@pytest.mark.parametrize("kind", ["grid", "stig", "fsg"])
def test_id_sets_beyond_shared_memory_set(gpu_ctx, c1, kind):
    """Queries whose result holds more distinct trajectories than the kernel's shared-memory
    set (4096) go to the bitmap form; mixed with small queries in one batch, every result must
    still equal the oracle's, in any mix and order."""
    t, q, db = c1
    ix = {"grid": lambda: G.Grid(gpu_ctx, db, D.BOX, 0.01, 2, 512), "stig": lambda: G.STIG(gpu_ctx, db, 512),
          "fsg": lambda: G.FSG(gpu_ctx, db, D.BOX, 0.01)}[kind]()
    o = {"grid": lambda: po.OracleGrid(t, D.BOX, 0.01, 2, 512), "stig": lambda: po.OracleSTIG(t, 512),
         "fsg": lambda: po.OracleFSG(t, D.BOX, 0.01)}[kind]()
    big = np.array([[121.0, 30.7, 122.0, 31.7], [121.0, 30.7, 121.7, 31.5], [121.2, 30.9, 122.0, 31.7]], np.float32)
    qq = np.concatenate([q[:40], big[:1], q[40:80], big[1:], q[80:100]])
    r = ix.range_query(qq)
    off, ids = o.range(qq, 0)
    assert np.array_equal(r.offsets, off) and np.array_equal(r.tids, ids)
    assert off[41] - off[40] > 4096  # the whole-box query really overflows the set


@pytest.mark.parametrize("kind", ["grid", "stig", "fsg"])
def test_plain_and_ordered_batches_with_overflow(gpu_ctx, c1, kind):
    """Plain execution (one launch sequence per query, no host wait in between) and batches of
    at least 256 queries (scanned in the locality order of their first candidate) on every
    index, with whole-box queries that overflow the shared-memory set in both forms."""
    t, q, db = c1
    ix = {"grid": lambda: G.Grid(gpu_ctx, db, D.BOX, 0.01, 2, 512), "stig": lambda: G.STIG(gpu_ctx, db, 512),
          "fsg": lambda: G.FSG(gpu_ctx, db, D.BOX, 0.01)}[kind]()
    o = {"grid": lambda: po.OracleGrid(t, D.BOX, 0.01, 2, 512), "stig": lambda: po.OracleSTIG(t, 512),
         "fsg": lambda: po.OracleFSG(t, D.BOX, 0.01)}[kind]()
    big = np.array([[121.0, 30.7, 122.0, 31.7], [121.2, 30.9, 122.0, 31.7]], np.float32)
    batch = np.concatenate([q[:700], big[:1], q[700:], big[1:]])
    r = ix.range_query(batch)
    off, ids = o.range(batch, 0)
    assert np.array_equal(r.offsets, off) and np.array_equal(r.tids, ids)
    plain = np.concatenate([q[::23], big[:1], q[5:40]])
    r = ix.range_query(plain, execution="plain")
    off, ids = o.range(plain, 0)
    assert np.array_equal(r.offsets, off) and np.array_equal(r.tids, ids)


def test_plain_truncation_reports_needed(gpu_ctx, c1):
    t, q, db = c1
    g = G.Grid(gpu_ctx, db, D.BOX, 0.01, 2, 512)
    full = g.range_query(q[:60], execution="plain")
    with pytest.raises(G.GatError) as e:
        g.range_query(q[:60], execution="plain", capacity=max(0, len(full.tids) - 1))
    assert e.value.status == 4
    again = g.range_query(q[:60], execution="plain")
    assert np.array_equal(again.offsets, full.offsets) and np.array_equal(again.tids, full.tids)


@pytest.mark.parametrize("cell,cap", [(0.01, 512), (0.02, 1), (0.02, 10_000_000), (0.005, 64)])
def test_morton_grid_leaves_and_results(gpu_ctx, c1, cell, cap):
    """MortonGrid (MortonGrid.cpp:238-393): its leaf bitmap holds exactly the Grid's leaves as
    (level, id) (the oracle's quadtree, Grid.cpp:58-94), and its implicit-tree walk with computed
    node boxes returns the oracle's id sets and point lists, batched and plain."""
    t, q, db = c1
    g = G.Grid(gpu_ctx, db, D.BOX, cell, 2, cap)
    m = G.MortonGrid(g)
    o = po.OracleGrid(t, D.BOX, cell, 2, cap)
    nd = o.nodes()
    want = sorted(zip(nd["level"][nd["leaf"] == 1].tolist(), nd["id"][nd["leaf"] == 1].tolist()))
    lv, ids = m.leaves()
    assert sorted(zip(lv.tolist(), ids.tolist())) == want
    assert m.info()["kind"] == 3 and m.info()["points"] == g.info()["points"]
    off, tids = o.range(q, 0)
    r = m.range_query(q)
    assert np.array_equal(r.offsets, off) and np.array_equal(r.tids, tids)
    qq = q[::11]
    off, tids = o.range(qq, 0)
    r = m.range_query(qq, execution="plain")
    assert np.array_equal(r.offsets, off) and np.array_equal(r.tids, tids)
    off, tid, pidx = o.range(qq, 1)
    r = m.range_query(qq, "points")
    assert csr_equal(r.offsets, r.tids, off, tid) and np.array_equal(r.pidx, pidx)
    m.close()
    g.close()


def test_morton_grid_rejects_other_kinds(gpu_ctx, c1):
    t, q, db = c1
    f = G.FSG(gpu_ctx, db, D.BOX, 0.01)
    with pytest.raises(G.GatError) as e:
        G.MortonGrid(f)
    assert e.value.status == 1
    g = G.Grid(gpu_ctx, db, D.BOX, 0.01, 2, 512)
    m = G.MortonGrid(g)
    with pytest.raises(G.GatError):
        m.save("/tmp/gat_morton_snapshot.bin")


@pytest.mark.parametrize("shape", [1, 2, 3])
def test_hash_shapes(gpu_ctx, c1, shape):
    """Every block shape of the batched id-set scan (256 threads, 128 threads, small queries one
    per warp after the others in block mode) returns the oracle's sets, on the Grid and on STIG."""
    from gat_b200 import _lib as L
    t, q, db = c1
    qq = np.concatenate([q] * 3)  # enough queries for the locality order
    gpu_ctx.set_tuning(L.GAT_TUNE_RANGE_SHAPE, shape)
    try:
        g = G.Grid(gpu_ctx, db, D.BOX, 0.01, 2, 512)
        off, ids = po.OracleGrid(t, D.BOX, 0.01, 2, 512).range(qq, 0)
        r = g.range_query(qq, "ids")
        assert csr_equal(r.offsets, r.tids, off, ids)
        s = G.STIG(gpu_ctx, db, 512)
        ref = po.OracleSTIG(t, 512).range(qq, 0)
        r = s.range_query(qq, "ids")
        assert csr_equal(r.offsets, r.tids, ref[0], ref[1])
    finally:
        gpu_ctx.set_tuning(L.GAT_TUNE_RANGE_SHAPE, 0)
