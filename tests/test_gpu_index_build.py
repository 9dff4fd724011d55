"""Grid and FSG indexes placed on the device (GAT_TUNE_INDEX_BUILD = 2) against the host
placement (= 1) of the same set: every device array of the index byte for byte (read back through
an index snapshot), the host copies (gat_index_points), the counts, range results and FV lower
bounds; and the device layout against the oracle's (Grid.cpp:210-316, FSG.cpp:95-143). Edge
sets: points on the grid's borders and cell boundaries, a coordinate just outside xmin (which
truncates into column 0 in the reference), empty and one-point trajectories, revisited cells,
a set with no points; a point outside the grid and a NaN coordinate fail alike on both paths."""
import struct

import numpy as np
import pytest

import gat_b200 as G
from gat_b200 import _lib as L
from gat_b200 import data as D
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

HOST, DEVICE = 1, 2


def build(ctx, db, kind, mode, **kw):
    ctx.set_tuning(L.GAT_TUNE_INDEX_BUILD, mode)
    try:
        if kind == "grid":
            return G.Grid(ctx, db, kw.get("box", D.BOX), kw["cell"], kw.get("vparam", 2), kw.get("leaf", 512))
        return G.FSG(ctx, db, kw.get("box", D.BOX), kw["cell"])
    finally:
        ctx.set_tuning(L.GAT_TUNE_INDEX_BUILD, 0)


def snapshot_arrays(ix, path):
    """The index's device arrays as saved by gat_index_save: (count, [bytes...])."""
    ix.save(path)
    raw = open(path, "rb").read()
    npts = ix.info()["points"]
    # the array list starts with its count (u32) and the x array's size ((points + 1) * 4)
    narr = 11 if ix.kind == L.GAT_INDEX_GRID else 6
    at = raw.find(struct.pack("<IQ", narr, (npts + 1) * 4))
    assert at > 0
    p, out = at + 4, []
    for _ in range(narr):
        (size,) = struct.unpack_from("<Q", raw, p)
        out.append(raw[p + 8:p + 8 + size])
        p += 8 + size
    return out


def assert_same_index(ctx, db, kind, tmp_path, queries=None, fv_queries=None, **kw):
    h = build(ctx, db, kind, HOST, **kw)
    d = build(ctx, db, kind, DEVICE, **kw)
    assert h.info() == d.info()
    for a, b in zip(h.points(), d.points()):
        assert np.array_equal(a, b)
    ah, ad = snapshot_arrays(h, str(tmp_path / "h.idx")), snapshot_arrays(d, str(tmp_path / "d.idx"))
    for i, (a, b) in enumerate(zip(ah, ad)):
        assert a == b, f"device array {i} differs"
    if queries is not None:
        for res in ("ids", "points"):
            x, y = h.range_query(queries, result=res), d.range_query(queries, result=res)
            assert np.array_equal(x.offsets, y.offsets) and np.array_equal(x.tids, y.tids)
    if fv_queries is not None and kind == "grid":
        assert np.array_equal(h.fv_lower_bounds(fv_queries), d.fv_lower_bounds(fv_queries))
    return h, d


@pytest.mark.parametrize("cell,vparam,leaf", [(0.0025, 2, 512), (0.01, 0, 7), (0.005, 8, 64), (0.5, 2, 1)])
def test_grid_device_matches_host_and_oracle(gpu_ctx, tmp_path, cell, vparam, leaf):
    t = D.walks(D.lengths(4000, 0, 0, 0, 1, 300, 61), 61)
    db = G.TrajectorySet(gpu_ctx, t)
    q = D.boxes(300, 1, 0.001, 0.05, 62)
    _, d = assert_same_index(gpu_ctx, db, "grid", tmp_path, q, t.subset([1, 500, 3999]), cell=cell, vparam=vparam,
                             leaf=leaf)
    o = po.OracleGrid(t, D.BOX, cell, vparam, leaf)
    for a, b in zip(d.points(), o.points()):
        assert np.array_equal(a, b)
    info, meta = d.info(), o.meta()
    assert info["leaves"] == meta["leaves"] and info["nodes"] == meta["nodes"]


@pytest.mark.parametrize("cell", [0.01, 0.0031, 0.3])
def test_fsg_device_matches_host_and_oracle(gpu_ctx, tmp_path, cell):
    t = D.walks(D.lengths(3000, 0, 0, 0, 1, 250, 63), 63)
    db = G.TrajectorySet(gpu_ctx, t)
    _, d = assert_same_index(gpu_ctx, db, "fsg", tmp_path, D.boxes(300, 1, 0.001, 0.05, 64), cell=cell)
    for a, b in zip(d.points(), po.OracleFSG(t, D.BOX, cell).points()):
        assert np.array_equal(a, b)


def edge_set():
    """Border and cell-boundary points, revisits, empty and one-point trajectories."""
    x0, y0, x1, y1 = (np.float32(v) for v in D.BOX)
    c = np.float32(0.01)
    bx = [x0 + c * np.float32(k) for k in (0, 1, 7, 50, 99)]
    by = [y1 - c * np.float32(k) for k in (0, 1, 3, 64, 99)]
    below = np.nextafter(x0, np.float32(0))  # just left of xmin: (lon - xmin) / cell truncates to 0
    trajs = [
        [(x0, y1), (x1, y0), (x0, y0), (x1, y1)],                  # the four corners
        [],
        [(bx[i], by[j]) for i in range(5) for j in range(5)],       # on cell boundaries
        [(below, y1), (below, by[2])],
        [(bx[1], by[1])],
        [],
        [(bx[2], by[2]), (bx[3], by[3]), (bx[2], by[2]), (bx[3], by[3]), (bx[2], by[2])],  # revisits
        [(bx[0], by[0])] * 6,                                       # duplicates
        [],
    ]
    lens = np.array([len(p) for p in trajs], np.int32)
    pts = [p for tr in trajs for p in tr]
    lon = np.array([p[0] for p in pts], np.float32)
    lat = np.array([p[1] for p in pts], np.float32)
    return D.Trajectories(lens, lon, lat)


def test_edge_sets(gpu_ctx, tmp_path):
    t = edge_set()
    db = G.TrajectorySet(gpu_ctx, t)
    q = np.array([[121.0, 30.7, 122.0, 31.7], [121.0, 31.69, 121.011, 31.7], [121.5, 31.1, 121.51, 31.11]], np.float32)
    for vparam in (0, 1, 2):
        assert_same_index(gpu_ctx, db, "grid", tmp_path, q, t.subset([1, 3, 7]), cell=0.01, vparam=vparam, leaf=2)
    assert_same_index(gpu_ctx, db, "fsg", tmp_path, q, cell=0.01)
    for a, b in zip(build(gpu_ctx, db, "grid", DEVICE, cell=0.01, leaf=2).points(),
                    po.OracleGrid(t, D.BOX, 0.01, 2, 2).points()):
        assert np.array_equal(a, b)
    empty = D.Trajectories(np.zeros(3, np.int32), np.zeros(0, np.float32), np.zeros(0, np.float32))
    edb = G.TrajectorySet(gpu_ctx, empty)
    assert_same_index(gpu_ctx, edb, "grid", tmp_path, cell=0.01)
    assert_same_index(gpu_ctx, edb, "fsg", tmp_path, cell=0.01)


@pytest.mark.parametrize("bad", [(121.5, 31.2, 122.5, 31.2), (121.5, 31.2, float("nan"), 31.2),
                                 (121.5, 31.2, 121.6, float("nan")), (121.5, 31.2, 121.6, 40.0)])
def test_out_of_grid_fails_on_both_paths(gpu_ctx, bad):
    t = D.Trajectories(np.array([2, 2], np.int32), np.array([bad[0], bad[0], bad[2], bad[0]], np.float32),
                       np.array([bad[1], bad[1], bad[3], bad[1]], np.float32))
    db = G.TrajectorySet(gpu_ctx, t)
    for kind in ("grid", "fsg"):
        for mode in (HOST, DEVICE):
            with pytest.raises(G.GatError) as e:
                build(gpu_ctx, db, kind, mode, cell=0.01)
            assert e.value.status == L.GAT_ERR_ARG


def test_point_index_beyond_the_key(gpu_ctx, tmp_path):
    """2^17 trajectories and one of 40000 points: trajectory and point index need 18 + 16 bits,
    more than the 32-bit key holds, so the device keeps the point index apart; the host copies
    read back later must still match the host build's."""
    lens = np.full(1 << 17, 2, np.int32)
    lens[1000] = 40000
    t = D.walks(lens, 65)
    db = G.TrajectorySet(gpu_ctx, t)
    assert_same_index(gpu_ctx, db, "grid", tmp_path, cell=0.01)
    assert_same_index(gpu_ctx, db, "fsg", tmp_path, cell=0.02)


def test_long_trajectories_and_deep_trees(gpu_ctx, tmp_path):
    """Trajectories of 1 to 2049 points (many runs of virtual cells per trajectory), and a leaf
    cap of 1 over a fine grid, whose quadtree outgrows the builder's first node buffer."""
    q = D.boxes(200, 1, 0.001, 0.05, 67)
    for top in (2048, 2049):
        lens = D.lengths(400, 0, 0, 0, 1, 300, 68).astype(np.int32)
        lens[[5, 100, 399]] = [top, 2047, 1]
        t = D.walks(lens, 69)
        db = G.TrajectorySet(gpu_ctx, t)
        assert_same_index(gpu_ctx, db, "grid", tmp_path, q, t.subset([6, 101, 400]), cell=0.0025, vparam=2, leaf=64)
    rng = np.random.default_rng(70)
    x0, y0, x1, y1 = D.BOX
    t = D.Trajectories(np.ones(60000, np.int32), rng.uniform(x0, x1, 60000).astype(np.float32),
                       rng.uniform(y0, y1, 60000).astype(np.float32))
    db = G.TrajectorySet(gpu_ctx, t)
    h, d = assert_same_index(gpu_ctx, db, "grid", tmp_path, q, cell=0.001, vparam=3, leaf=1)
    assert d.info()["nodes"] > 1 << 16


def test_build_temporaries_kept_until_trim(gpu_ctx):
    """A device build leaves its temporaries in the context's pool for the next build (counted by
    scratch_bytes); trim returns them, and a build after the trim still gives the same index."""
    t = D.walks(D.lengths(3000, 0, 0, 0, 1, 250, 71), 71)
    db = G.TrajectorySet(gpu_ctx, t)
    a = build(gpu_ctx, db, "grid", DEVICE, cell=0.005)
    assert gpu_ctx.scratch_bytes > 0
    gpu_ctx.trim()
    assert gpu_ctx.scratch_bytes == 0
    b = build(gpu_ctx, db, "grid", DEVICE, cell=0.005)
    for x, y in zip(a.points(), b.points()):
        assert np.array_equal(x, y)
