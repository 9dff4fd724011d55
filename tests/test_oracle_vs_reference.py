"""The oracle restatement against the reference's own CPU code run live (oracle/_ref/gatref),
on seeded inputs larger than the committed fixtures. Runs on CPU; skipped without gatref."""
import numpy as np
import pytest

from gat_b200 import data as D
from oracle import pyoracle as po

pytestmark = pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref/gatref not built")
BOX = D.BOX


@pytest.fixture(scope="module")
def ref():
    return po.RefRunner()


@pytest.mark.parametrize("cell,leaf", [(0.01, 512), (0.005, 100), (0.02, 20000)])
def test_grid(ref, cell, leaf):
    t, _ = D.config1(seed=3, n=3000, nq=1)
    q = D.boxes(200, 1, 0.001, 0.1, 4)
    r = ref.gtq(t, q, BOX, cell, leaf, layout=True)
    o = po.OracleGrid(t, BOX, cell, 2, leaf)
    x, y, tid, _ = o.points()
    assert np.array_equal(x, r["px"]) and np.array_equal(y, r["py"]) and np.array_equal(tid, r["ptid"])
    nd = o.nodes()
    assert np.array_equal(nd["id"], r["node_id"]) and np.array_equal(nd["leaf"], r["node_leaf"])
    assert np.array_equal(nd["mbb"].ravel(), r["node_mbb"])
    off, ids = o.range(q, 0)
    assert np.array_equal(off, r["id_off"]) and np.array_equal(ids, r["ids"])
    fo, fc, fn = o.fv()
    assert np.array_equal(fo, r["fv_off"]) and np.array_equal(fc, r["fv_cell"]) and np.array_equal(fn, r["fv_count"])


def test_stig_and_fsg(ref):
    t, _ = D.config1(seed=5, n=3000, nq=1)
    q = D.boxes(200, 1, 0.001, 0.1, 6)
    for block in (64, 1000):
        r = ref.stig(t, q, block, layout=True)
        o = po.OracleSTIG(t, block)
        x, y, tid, _ = o.points()
        assert np.array_equal(x, r["px"]) and np.array_equal(y, r["py"]) and np.array_equal(tid, r["ptid"])
        off, ids = o.range(q, 0)
        assert np.array_equal(off, r["id_off"]) and np.array_equal(ids, r["ids"])
    r = ref.fsg(t, BOX, 0.01)
    o = po.OracleFSG(t, BOX, 0.01)
    x, y, tid, _ = o.points()
    s, e = o.cells()
    assert np.array_equal(tid, r["ptid"]) and np.array_equal(s, r["cell_start"]) and np.array_equal(e, r["cell_end"])


@pytest.mark.parametrize("eps", [5e-4, 5e-3, 1e-3])
def test_edr(ref, eps):
    la = D.lengths(800, 2, 0, 0, 1, 500, 14)
    lb = D.lengths(800, 2, 0, 0, 1, 500, 15)
    a, b = D.pairs(la, lb, 16)
    assert np.array_equal(po.edr_batch(la, a, lb, b, eps), ref.edr(la, a, lb, b, eps)["dist"])


def test_bounds_topk_neighbours(ref):
    t = D.walks(D.lengths(8000, 1, float(np.log(200.0)), 0.6, 32, 1024, 17), 17)
    qids = D.sample_ids(10, t.n, 18)
    lbr = ref.fvlb(t, qids, BOX, 0.0025)
    o = po.OracleGrid(t, BOX, 0.0025, 2, 512)
    for j, qid in enumerate(qids):
        assert np.array_equal(o.fv_lb(*t.points(int(qid)))[1:], lbr[j, 1:])
    rt = ref.topk(t, qids, BOX, 0.0025, 24, 5e-4)
    for j, qid in enumerate(qids):
        ids, dist, _ = o.topk(*t.points(int(qid)), 24, 5e-4, pruned=True)
        assert np.array_equal(np.sort(rt["dist"][j]), dist)
        # the reference's ids carry exactly the distances it reports
        for tid, d in zip(rt["ids"][j], rt["dist"][j]):
            assert po.edr(np.stack(t.points(int(qid)), 1), np.stack(t.points(int(tid)), 1), 5e-4) == d
    vc = (512 * 512) >> 2
    cells = np.arange(0, vc, 97, dtype=np.int32)
    nb, grid = ref.nbr(cells, vc)
    assert np.array_equal(nb, np.array([po.fv_neighbors(vc, int(c)) for c in cells]))
