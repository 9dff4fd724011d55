"""The oracle's workload generator (oracle/datagen.cpp) against the library's (csrc/gen.cpp): the
CPU baseline of the reference builds its inputs with the former, the GPU runs with the latter,
so both must produce the same arrays bit for bit. Also the reference's timed range leg
(gatref rangebench) against the oracle on a small set. Runs on CPU."""
import numpy as np
import pytest

from gat_b200 import _lib as L
from gat_b200 import data as D
from oracle import pyoracle as po


@pytest.mark.parametrize("kind,p0,p1,lo,hi", [(L.GAT_LEN_UNIFORM, 0, 0, 20, 200),
                                              (L.GAT_LEN_LOGNORMAL, float(np.log(200.0)), 0.6, 32, 1024),
                                              (L.GAT_LEN_LOGUNIFORM, 0, 0, 16, 4096)])
def test_lengths_and_walks(kind, p0, p1, lo, hi):
    for seed in (0, 7):
        a = D.lengths(9000, kind, p0, p1, lo, hi, seed)
        b = po.gen_lengths(9000, kind, p0, p1, lo, hi, seed)
        assert np.array_equal(a, b)
        wa, wb = D.walks(a, seed), po.gen_walks(b, seed)
        assert np.array_equal(wa.lon, wb.lon) and np.array_equal(wa.lat, wb.lat)


def test_boxes_samples_pairs():
    for kind, s0, s1 in ((L.GAT_SIDE_FIXED, 0.01, 0.01), (L.GAT_SIDE_LOGUNIFORM, 0.001, 0.05)):
        assert np.array_equal(D.boxes(5000, kind, s0, s1, 3), po.gen_boxes(5000, kind, s0, s1, 3))
    assert np.array_equal(D.sample_ids(256, 100_000, 0), po.gen_sample_ids(256, 100_000, 0))
    la, a, lb, b = D.config4_pairs(seed=2, npairs=300)
    la2, a2, lb2, b2 = po.config4_pairs(seed=2, npairs=300)
    assert np.array_equal(la, la2) and np.array_equal(lb, lb2) and np.array_equal(a, a2) and np.array_equal(b, b2)


def test_configs():
    t, q = D.config3(seed=0, n=5000, nq=1000)
    t2, q2 = po.config3(seed=0, n=5000, nq=1000)
    assert np.array_equal(t.lengths, t2.lengths) and np.array_equal(t.lon, t2.lon) and np.array_equal(q, q2)
    t, qi = D.config2(seed=0, n=3000, nq=16)
    t2, qi2 = po.config2(seed=0, n=3000, nq=16)
    assert np.array_equal(t.lat, t2.lat) and np.array_equal(qi, qi2)


@pytest.mark.skipif(not po.ref_available(), reason="oracle/_ref/gatref not built")
def test_reference_rangebench_equals_oracle():
    """gatref rangebench generates its set and rectangles itself; its step-0 id sets (the
    reference's Grid::rangeQueryBatch on 3 threads) equal the oracle's on the same inputs."""
    n, nq, per_step = 4000, 3000, 150
    r = po.RefRunner().rangebench(n, 50, 350, 0, nq, 0.001, 0.05, 0.001, 512, po.BOX, per_step, 4, 3)
    t, q = po.config3(seed=0, n=n, nq=nq)
    assert list(r["q_index"]) == list(range(0, nq, nq // per_step))
    off, ids = po.OracleGrid(t, po.BOX, 0.001, 2, 512).range(q[r["q_index"]])
    assert np.array_equal(off, r["id_off"]) and np.array_equal(ids, r["ids"])
    assert len(r["t_step"]) == 4 and r["ids_step"][0] == len(ids)
