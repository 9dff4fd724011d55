"""The oracle restatement against fixtures written by the reference's own CPU code
(tests/golden/make_golden.py; oracle/_ref/gatref). Runs on CPU."""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from tests.golden.make_golden import BOX, digest, inputs

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))


@pytest.fixture(scope="module")
def ins():
    return inputs()


def test_generator_unchanged(ins):
    t, q, la, a, lb, b, tk, qids = ins
    assert digest(t.lengths, t.lon, t.lat, q, la, a, lb, b, tk.lengths, tk.lon, tk.lat, qids) == str(G["input_digest"])


def test_grid_layout_ids_candidates(ins):
    t, q = ins[0], ins[1]
    o = po.OracleGrid(t, BOX, 0.01, 2, 64)
    m = o.meta()
    assert [m["axis"], m["cellnum"], m["points"]] == list(G["gtq_meta"][:3])
    x, y, tid, _ = o.points()
    s, e, _ = o.cells()
    assert digest(x, y, tid, s, e) == str(G["gtq_layout"])
    assert digest(*o.fv()) == str(G["gtq_fv"])
    off, ids = o.range(q, 0)
    assert np.array_equal(off, G["gtq_id_off"]) and np.array_equal(ids, G["gtq_ids"])
    co = G["gtq_cand_off"]
    for i in range(len(q)):
        nid, lv = o.candidates(q[i])
        assert np.array_equal(nid, G["gtq_cand_node"][co[i]:co[i + 1]])
        assert np.array_equal(lv, G["gtq_cand_level"][co[i]:co[i + 1]])


def test_stig(ins):
    t, q = ins[0], ins[1]
    o = po.OracleSTIG(t, 256)
    x, y, tid, _ = o.points()
    assert digest(x, y, tid) == str(G["stig_layout"])
    off, ids = o.range(q, 0)
    assert np.array_equal(off, G["stig_id_off"]) and np.array_equal(ids, G["stig_ids"])
    bo = G["stig_blk_off"]
    for i in range(len(q)):
        assert np.array_equal(o.candidates(q[i]).ravel(), G["stig_blk"][2 * bo[i]:2 * bo[i + 1]])


def test_fsg_layout(ins):
    o = po.OracleFSG(ins[0], BOX, 0.01)
    m = o.meta()
    assert [m["nx"], m["ny"], m["cellnum"], m["points"]] == list(G["fsg_meta"])
    x, y, tid, _ = o.points()
    s, e = o.cells()
    assert digest(x, y, tid, s, e) == str(G["fsg_layout"])


@pytest.mark.parametrize("eps,key", [(5e-4, "edr_5e-4"), (5e-3, "edr_5e-3")])
def test_edr(ins, eps, key):
    la, a, lb, b = ins[2], ins[3], ins[4], ins[5]
    assert np.array_equal(po.edr_batch(la, a, lb, b, eps), G[key])


def test_fv_lower_bounds_and_topk(ins):
    tk, qids = ins[6], ins[7]
    o = po.OracleGrid(tk, BOX, 0.0025, 2, 512)
    for j, qid in enumerate(qids):
        lb = o.fv_lb(*tk.points(int(qid)))
        assert np.array_equal(lb[1:], G["fvlb"][j, 1:])
        _, dist, _ = o.topk(*tk.points(int(qid)), 16, 5e-4, pruned=True)
        assert np.array_equal(dist, G["topk_dist_sorted"][j])


def test_neighbour_keys():
    vc = (512 * 512) >> 2
    for c, want in zip(G["nbr_cells"], G["nbr"]):
        assert np.array_equal(po.fv_neighbors(vc, int(c)), want)
