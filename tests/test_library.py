"""CPU checks of the product library: every symbol include/gat_b200.h declares is exported,
host index builders reproduce the reference layouts (host-only context, no GPU), the
generator is deterministic, arguments are validated with status codes."""
import os
import re
import subprocess

import numpy as np
import pytest

import gat_b200 as G
from gat_b200 import _lib as L
from gat_b200 import data as D
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "gat_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gat_[a-z0-9_]+)\s*\(", src)))


def test_all_declared_symbols_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (gat_[a-z0-9_]+)", out))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    assert set(L.EXPORTED) == set(declared_functions())


def test_generator_deterministic_and_shaped():
    a = D.lengths(1000, L.GAT_LEN_LOGNORMAL, float(np.log(200.0)), 0.6, 32, 1024, 1)
    b = D.lengths(1000, L.GAT_LEN_LOGNORMAL, float(np.log(200.0)), 0.6, 32, 1024, 1)
    assert np.array_equal(a, b) and a.min() >= 32 and a.max() <= 1024
    assert 150 < np.median(a) < 260
    t = D.walks(a, 2)
    assert np.all(t.lon >= 121.0) and np.all(t.lon <= 122.0) and np.all(t.lat >= 30.7) and np.all(t.lat <= 31.7)
    steps = np.diff(t.lon[:a[0]].astype(np.float64))
    assert np.std(steps) < 3e-4
    q = D.boxes(1000, L.GAT_SIDE_LOGUNIFORM, 0.001, 0.05, 3)
    w = q[:, 2] - q[:, 0]
    assert w.min() > 0.0009 and w.max() < 0.0501
    ids = D.sample_ids(256, 1000, 4)
    assert len(set(ids.tolist())) == 256 and ids.min() >= 1 and ids.max() <= 1000


@pytest.mark.parametrize("cell,leaf", [(0.01, 512), (0.0025, 512), (0.005, 7)])
def test_host_grid_layout_matches_oracle(host_ctx, cell, leaf):
    t = D.walks(D.lengths(2500, 0, 0, 0, 1, 200, 20), 20)
    db = G.TrajectorySet(host_ctx, t)
    g = G.Grid(host_ctx, db, D.BOX, cell, 2, leaf)
    o = po.OracleGrid(t, D.BOX, cell, 2, leaf)
    for a, b in zip(g.points(), o.points()):
        assert np.array_equal(a, b)
    info, meta = g.info(), o.meta()
    assert info["leaves"] == meta["leaves"] and info["nodes"] == meta["nodes"] and info["nx"] == meta["axis"]


@pytest.mark.parametrize("block", [2, 3, 50, 777, 100000])
def test_host_stig_layout_matches_oracle(host_ctx, block):
    t = D.walks(D.lengths(1500, 0, 0, 0, 1, 120, 21), 21)
    db = G.TrajectorySet(host_ctx, t)
    s = G.STIG(host_ctx, db, block)
    for a, b in zip(s.points(), po.OracleSTIG(t, block).points()):
        assert np.array_equal(a, b)


def test_host_fsg_layout_matches_oracle(host_ctx):
    t = D.walks(D.lengths(2000, 0, 0, 0, 1, 200, 22), 22)
    db = G.TrajectorySet(host_ctx, t)
    f = G.FSG(host_ctx, db, D.BOX, 0.01)
    for a, b in zip(f.points(), po.OracleFSG(t, D.BOX, 0.01).points()):
        assert np.array_equal(a, b)


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref/gatref not built")
def test_host_layouts_match_reference(host_ctx):
    t = D.walks(D.lengths(2000, 0, 0, 0, 5, 150, 23), 23)
    db = G.TrajectorySet(host_ctx, t)
    R = po.RefRunner()
    r = R.gtq(t, np.zeros((1, 4), np.float32), D.BOX, 0.01, 512, layout=True)
    x, y, tid, _ = G.Grid(host_ctx, db, D.BOX, 0.01, 2, 512).points()
    assert np.array_equal(x, r["px"]) and np.array_equal(y, r["py"]) and np.array_equal(tid, r["ptid"])
    r = R.stig(t, np.zeros((1, 4), np.float32), 300, layout=True)
    x, y, tid, _ = G.STIG(host_ctx, db, 300).points()
    assert np.array_equal(x, r["px"]) and np.array_equal(y, r["py"]) and np.array_equal(tid, r["ptid"])
    r = R.fsg(t, D.BOX, 0.01)
    x, y, tid, _ = G.FSG(host_ctx, db, D.BOX, 0.01).points()
    assert np.array_equal(tid, r["ptid"]) and np.array_equal(x, r["px"])


def test_argument_errors(host_ctx):
    t = D.walks(D.lengths(10, 0, 0, 0, 1, 10, 24), 24)
    db = G.TrajectorySet(host_ctx, t)
    with pytest.raises(G.GatError) as e:
        G.Grid(host_ctx, db, D.BOX, -1.0)
    assert e.value.status == L.GAT_ERR_ARG
    with pytest.raises(G.GatError) as e:
        G.Grid(host_ctx, db, (121.5, 30.7, 122.0, 31.7), 0.01)  # points left of the grid
    assert e.value.status == L.GAT_ERR_ARG
    with pytest.raises(G.GatError) as e:
        G.STIG(host_ctx, db, 1)  # the reference recurses without end below 2
    assert e.value.status == L.GAT_ERR_ARG
    g = G.Grid(host_ctx, db, D.BOX, 0.01)
    with pytest.raises(G.GatError) as e:
        g.range_query(np.zeros((1, 4), np.float32))
    assert e.value.status == L.GAT_ERR_STATE  # host-only context has no device


def test_tuning_knob(host_ctx):
    """GAT_TUNE_EDR_ROWS accepts 0 (autotune), 2, 4 and 8 and nothing else."""
    for v in (2, 4, 8, 0):
        host_ctx.set_edr_rows(v)
        assert host_ctx.tuning(L.GAT_TUNE_EDR_ROWS) == v
    assert host_ctx.tuning(L.GAT_TUNE_EDR_TUNED) == 0
    for bad in (1, 3, 16, -1):
        with pytest.raises(G.GatError) as e:
            host_ctx.set_edr_rows(bad)
        assert e.value.status == L.GAT_ERR_ARG
    with pytest.raises(G.GatError):
        host_ctx.tuning(99)


def test_topk_walk_knobs(host_ctx):
    """GAT_TUNE_TOPK_CHUNK (0..2^24), GAT_TUNE_TOPK_GROWTH (0 or 2..64), the test knob
    GAT_TUNE_TEST_STALL_CARRY (>= 0), GAT_TUNE_SERVE_RESERVE (0..90), GAT_TUNE_RANGE_SHAPE (0..3)
    and GAT_TUNE_EDR_RESERVE (0..90) round-trip; other values are refused."""
    for knob, good, bad in ((L.GAT_TUNE_TOPK_CHUNK, (512, 0), (-1, 1 << 25)),
                            (L.GAT_TUNE_TOPK_GROWTH, (2, 8, 0), (1, 65, -2)),
                            (L.GAT_TUNE_TEST_STALL_CARRY, (3, 0), (-1,)),
                            (L.GAT_TUNE_SERVE_RESERVE, (25, 90, 0), (-1, 91)),
                            (L.GAT_TUNE_RANGE_SHAPE, (1, 2, 3, 0), (-1, 4)),
                            (L.GAT_TUNE_EDR_RESERVE, (50, 0), (-1, 91))):
        for v in good:
            host_ctx.set_tuning(knob, v)
            assert host_ctx.tuning(knob) == v
        for v in bad:
            with pytest.raises(G.GatError):
                host_ctx.set_tuning(knob, v)


def test_index_build_knob(host_ctx):
    """GAT_TUNE_INDEX_BUILD takes 0, 1 and 2; a device build on a host-only context is refused
    and the host build (0 or 1) still works there."""
    t = D.walks(D.lengths(50, 0, 0, 0, 1, 20, 26), 26)
    db = G.TrajectorySet(host_ctx, t)
    try:
        for v in (1, 2, 0):
            host_ctx.set_tuning(L.GAT_TUNE_INDEX_BUILD, v)
            assert host_ctx.tuning(L.GAT_TUNE_INDEX_BUILD) == v
        for v in (-1, 3):
            with pytest.raises(G.GatError) as e:
                host_ctx.set_tuning(L.GAT_TUNE_INDEX_BUILD, v)
            assert e.value.status == L.GAT_ERR_ARG
        host_ctx.set_tuning(L.GAT_TUNE_INDEX_BUILD, 2)
        for build in (lambda: G.Grid(host_ctx, db, D.BOX, 0.01), lambda: G.FSG(host_ctx, db, D.BOX, 0.01)):
            with pytest.raises(G.GatError) as e:
                build()
            assert e.value.status == L.GAT_ERR_STATE
        host_ctx.set_tuning(L.GAT_TUNE_INDEX_BUILD, 1)
        a = G.Grid(host_ctx, db, D.BOX, 0.01).points()
        host_ctx.set_tuning(L.GAT_TUNE_INDEX_BUILD, 0)
        b = G.Grid(host_ctx, db, D.BOX, 0.01).points()
        assert all(np.array_equal(x, y) for x, y in zip(a, b))
    finally:
        host_ctx.set_tuning(L.GAT_TUNE_INDEX_BUILD, 0)


def test_dependent_launch_knob(host_ctx):
    """GAT_TUNE_DEP_LAUNCH takes 0 or 1 (default 1)."""
    assert host_ctx.tuning(L.GAT_TUNE_DEP_LAUNCH) == 1
    try:
        host_ctx.set_tuning(L.GAT_TUNE_DEP_LAUNCH, 0)
        assert host_ctx.tuning(L.GAT_TUNE_DEP_LAUNCH) == 0
        for v in (-1, 2):
            with pytest.raises(G.GatError):
                host_ctx.set_tuning(L.GAT_TUNE_DEP_LAUNCH, v)
    finally:
        host_ctx.set_tuning(L.GAT_TUNE_DEP_LAUNCH, 1)


def test_topk_merge_arguments(host_ctx):
    """gat_topk_merge validates its sizes; the device form needs a device context."""
    ids = np.array([[[3, 7]], [[1, -1]]], np.int32)
    dist = np.array([[[2, 5]], [[2, -1]]], np.int32)
    oi, od = np.zeros((1, 2), np.int32), np.zeros((1, 2), np.int32)
    P = lambda a: a.ctypes.data_as(L.P_i32)
    assert L.lib.gat_topk_merge(1, 2, 2, P(ids), P(dist), P(oi), P(od)) == L.GAT_OK
    assert oi.tolist() == [[1, 3]] and od.tolist() == [[2, 2]]  # (distance, id) order
    for nq, k, parts in ((-1, 2, 2), (1, 0, 2), (1, 2, 0), (1, 1025, 1), (1, 1024, 9)):
        assert L.lib.gat_topk_merge(nq, k, parts, P(ids), P(dist), P(oi), P(od)) == L.GAT_ERR_ARG
    assert L.lib.gat_topk_merge_dev(host_ctx.h, 1, 2, 2, None, None, None, None) == L.GAT_ERR_ARG
    assert L.lib.gat_topk_merge_dev(host_ctx.h, 1, 2, 2, ids.ctypes.data, dist.ctypes.data, oi.ctypes.data,
                                    od.ctypes.data) == L.GAT_ERR_STATE


def test_snapshot_errors(host_ctx, tmp_path):
    """Saving needs a device context; loading refuses missing and foreign files."""
    t = D.walks(D.lengths(50, 0, 0, 0, 1, 20, 25), 25)
    db = G.TrajectorySet(host_ctx, t)
    g = G.Grid(host_ctx, db, D.BOX, 0.01)
    with pytest.raises(G.GatError) as e:
        g.save(str(tmp_path / "g.idx"))
    assert e.value.status == L.GAT_ERR_STATE
    with pytest.raises(G.GatError) as e:
        G.api.Index.load(host_ctx, db, str(tmp_path / "missing.idx"))
    assert e.value.status == L.GAT_ERR_ARG
    (tmp_path / "junk.idx").write_bytes(b"GATIDX01" + bytes(64))
    with pytest.raises(G.GatError) as e:
        G.api.Index.load(host_ctx, db, str(tmp_path / "junk.idx"))
    assert e.value.status == L.GAT_ERR_ARG
