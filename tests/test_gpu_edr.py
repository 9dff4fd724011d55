"""EDR pairs on the GPU against the oracle restatement of Grid::SimilarityExecuter
(Grid.cpp:1222-1318). Bit-exact integer distances."""
import numpy as np
import pytest

import gat_b200 as G
from gat_b200 import data as D
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("eps", [5e-4, 0.005])
def test_random_lengths(gpu_ctx, eps):
    la = D.lengths(1500, 2, 0, 0, 1, 700, 21)
    lb = D.lengths(1500, 2, 0, 0, 1, 700, 22)
    a, b = D.pairs(la, lb, 23)
    got = G.edr_pairs(gpu_ctx, la, a, lb, b, eps)
    want = po.edr_batch(la, a, lb, b, eps)
    assert np.array_equal(got, want)


def test_edge_lengths(gpu_ctx):
    """lengths 1 and 2, equal lengths (query is the rows), tile boundaries 128/256/257."""
    ls = [1, 2, 3, 31, 32, 33, 127, 128, 129, 255, 256, 257, 300]
    la, lb = [], []
    for x in ls:
        for y in ls:
            la.append(x)
            lb.append(y)
    la, lb = np.array(la, np.int32), np.array(lb, np.int32)
    a, b = D.pairs(la, lb, 31, jitter=1e-4)
    for eps in (5e-4, 0.005):
        assert np.array_equal(G.edr_pairs(gpu_ctx, la, a, lb, b, eps), po.edr_batch(la, a, lb, b, eps))


def test_identical_and_disjoint(gpu_ctx):
    la = D.lengths(64, 0, 0, 0, 16, 400, 41)
    t = D.walks(la, 42)
    xy = np.stack([t.lon, t.lat], 1)
    got = G.edr_pairs(gpu_ctx, la, xy, la, xy, 5e-4)
    assert np.array_equal(got, po.edr_batch(la, xy, la, xy, 5e-4))
    assert np.all(got == 0)
    far = xy + np.float32(5.0)
    got = G.edr_pairs(gpu_ctx, la, xy, la, far, 5e-4)
    assert np.array_equal(got, po.edr_batch(la, xy, la, far, 5e-4))


def test_long_pairs_sampled(gpu_ctx):
    """config-4 lengths (log-uniform 16..4096), a sample the oracle finishes quickly."""
    la, a, lb, b = D.config4_pairs(seed=0, npairs=4096)
    idx = np.arange(0, 4096, 64)
    oa = np.zeros(len(la) + 1, np.int64); oa[1:] = np.cumsum(la)
    ob = np.zeros(len(lb) + 1, np.int64); ob[1:] = np.cumsum(lb)
    sa = np.concatenate([a[oa[i]:oa[i + 1]] for i in idx])
    sb = np.concatenate([b[ob[i]:ob[i + 1]] for i in idx])
    got = G.edr_pairs(gpu_ctx, la[idx], sa, lb[idx], sb, 5e-4)
    assert np.array_equal(got, po.edr_batch(la[idx], sa, lb[idx], sb, 5e-4))


def test_full_config4_properties(gpu_ctx):
    """All 4096 config-4 pairs: distance bounds that hold for the recurrence
    (0 <= D <= len1 + len2 and D >= |len1 - len2|), and symmetry of the orientation rule."""
    la, a, lb, b = D.config4_pairs(seed=0, npairs=4096)
    d = G.edr_pairs(gpu_ctx, la, a, lb, b, 5e-4)
    assert np.all(d >= np.abs(la - lb)) and np.all(d <= la + lb)
    d2 = G.edr_pairs(gpu_ctx, lb, b, la, a, 5e-4)
    eq = la == lb
    # with unequal lengths the shorter side is always the row side, so swapping is invariant
    assert np.array_equal(d[~eq], d2[~eq])
