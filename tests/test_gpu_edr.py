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


def _mixed_pairs():
    la = np.concatenate([D.lengths(600, 2, 0, 0, 1, 900, 51), [1, 64, 65, 128, 129, 256, 257, 512, 513]]).astype(np.int32)
    lb = np.concatenate([D.lengths(600, 2, 0, 0, 1, 900, 52), [700, 64, 66, 900, 129, 257, 256, 1024, 2000]]).astype(np.int32)
    a, b = D.pairs(la, lb, 53)
    return la, a, lb, b


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("rows", [2, 4, 8])
def test_tile_shapes(gpu_ctx, rows, form):
    """Every tile shape (64, 128 or 256 points per tile; row tiles or column tiles) gives the
    oracle's distances, across single-tile pairs, pipelined multi-tile pairs and the tile
    boundaries."""
    from gat_b200 import _lib as L

    la, a, lb, b = _mixed_pairs()
    want = po.edr_batch(la, a, lb, b, 5e-4)
    gpu_ctx.set_edr_rows(rows)
    gpu_ctx.set_tuning(L.GAT_TUNE_EDR_FORM, form)
    try:
        got = G.edr_pairs(gpu_ctx, la, a, lb, b, 5e-4)
        got2 = G.edr_pairs(gpu_ctx, la, a, lb, b, 5e-3)
    finally:
        gpu_ctx.set_edr_rows(0)
        gpu_ctx.set_tuning(L.GAT_TUNE_EDR_FORM, 0)
    assert np.array_equal(got, want)
    assert np.array_equal(got2, po.edr_batch(la, a, lb, b, 5e-3))


def test_autotune_classes(gpu_ctx):
    """Autotune (the default) records the shape class on first use; both the tuning launch
    and the tuned launch give the oracle's distances."""
    from gat_b200 import _lib as L

    gpu_ctx.set_edr_rows(0)  # clears the table
    assert gpu_ctx.tuning(L.GAT_TUNE_EDR_TUNED) == 0
    la, a, lb, b = _mixed_pairs()
    want = po.edr_batch(la, a, lb, b, 5e-4)
    assert np.array_equal(G.edr_pairs(gpu_ctx, la, a, lb, b, 5e-4), want)
    assert gpu_ctx.tuning(L.GAT_TUNE_EDR_TUNED) >= 1
    assert np.array_equal(G.edr_pairs(gpu_ctx, la, a, lb, b, 5e-4), want)
    with pytest.raises(G.GatError):
        gpu_ctx.set_edr_rows(3)


def test_device_api_beyond_cooperative_pool(gpu_ctx):
    """gat_edr_pairs_dev sizes carry rows for the longest allowed side, which caps the
    cooperative pool at a few thousand pairs; more multi-tile pairs than that run tile by
    tile on one warp each. Both kinds must agree with the oracle."""
    import torch

    from gat_b200 import _lib as L

    la = D.lengths(5000, 0, 0, 0, 65, 300, 61)
    lb = D.lengths(5000, 0, 0, 0, 65, 300, 62)
    a, b = D.pairs(la, lb, 63)
    oa = np.zeros(len(la), np.int64); oa[1:] = np.cumsum(la)[:-1]
    ob = np.zeros(len(lb), np.int64); ob[1:] = np.cumsum(lb)[:-1]
    dev = torch.device("cuda", 0)
    T = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    d = [T(la.astype(np.int32)), T(oa), T(a), T(lb.astype(np.int32)), T(ob), T(b)]
    want = po.edr_batch(la, a, lb, b, 5e-4)
    for form in (1, 2):
        out = torch.full((len(la),), -7, dtype=torch.int32, device=dev)
        gpu_ctx.set_edr_rows(2)
        gpu_ctx.set_tuning(L.GAT_TUNE_EDR_FORM, form)
        try:
            torch.cuda.synchronize()
            gpu_ctx.check(L.lib.gat_edr_pairs_dev(gpu_ctx.h, len(la), d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(),
                                                  d[3].data_ptr(), d[4].data_ptr(), d[5].data_ptr(), 5e-4, out.data_ptr()),
                          "gat_edr_pairs_dev")
            gpu_ctx.check(L.lib.gat_ctx_sync(gpu_ctx.h), "gat_ctx_sync")
        finally:
            gpu_ctx.set_edr_rows(0)
            gpu_ctx.set_tuning(L.GAT_TUNE_EDR_FORM, 0)
        assert np.array_equal(out.cpu().numpy(), want), form


def test_device_api_rejects_bad_lengths(gpu_ctx):
    """gat_edr_pairs_dev reads lengths on the device: a side outside 1..GAT_EDR_MAX_LEN gets
    -1 (its points are never read) and the call returns GAT_ERR_ARG; other pairs are exact."""
    import torch

    from gat_b200 import _lib as L

    la = np.array([10, 0, 40, 20000, 7], np.int32)
    lb = np.array([12, 5, 33, 9, 7], np.int32)
    ra, rb = np.maximum(la, 0), lb.copy()
    ra[3] = 0  # no points stored for the oversize side
    a, b = D.pairs(np.where(ra > 0, ra, 1), rb, 71)
    oa = np.zeros(5, np.int64); oa[1:] = np.cumsum(np.where(ra > 0, ra, 1))[:-1]
    ob = np.zeros(5, np.int64); ob[1:] = np.cumsum(rb)[:-1]
    dev = torch.device("cuda", 0)
    T = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    d = [T(la), T(oa), T(a), T(lb), T(ob), T(b)]
    out = torch.full((5,), -7, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    rc = L.lib.gat_edr_pairs_dev(gpu_ctx.h, 5, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(),
                                 d[4].data_ptr(), d[5].data_ptr(), 5e-4, out.data_ptr())
    assert rc == L.GAT_ERR_ARG
    got = out.cpu().numpy()
    assert got[1] == -1 and got[3] == -1
    ok = np.array([0, 2, 4])
    la_ok = la[ok]
    sa = np.concatenate([a[oa[i]:oa[i] + la[i]] for i in ok])
    sb = np.concatenate([b[ob[i]:ob[i] + lb[i]] for i in ok])
    assert np.array_equal(got[ok], po.edr_batch(la_ok, sa, lb[ok], sb, 5e-4))
    # the context stays usable
    assert np.array_equal(G.edr_pairs(gpu_ctx, la_ok, sa, lb[ok], sb, 5e-4), got[ok])


def test_bounded_carry_wait_gives_up(gpu_ctx):
    """The wait of a pipelined tile for its predecessor's carry words is bounded: with the test
    knob, the first tile of one pair writes no carries, the next tile gives up after ~4096
    polls, the call returns GAT_ERR_TIMEOUT and that pair -1; every other pair is exact, and the
    same context then answers exactly with the knob off. No fault, no hang: the wait ends by
    itself and the kernel returns."""
    from gat_b200 import _lib as L

    ctx = G.Context(0)
    try:
        ctx.set_tuning(L.GAT_TUNE_EDR_ROWS, 4)  # one tile shape: no autotune launches
        ctx.set_tuning(L.GAT_TUNE_EDR_FORM, 1)  # row tiles of 128 rows
        la = np.array([600, 40, 900, 300], np.int32)
        lb = np.array([700, 50, 800, 2000], np.int32)
        a, b = D.pairs(la, lb, 61)
        want = po.edr_batch(la, a, lb, b, 5e-4)
        ctx.set_tuning(L.GAT_TUNE_TEST_STALL_CARRY, 3)  # pair 2 (900 x 800: 7 pipelined tiles)
        assert ctx.tuning(L.GAT_TUNE_TEST_STALL_CARRY) == 3
        with pytest.raises(G.GatError) as e:
            G.edr_pairs(ctx, la, a, lb, b, 5e-4)
        assert e.value.status == L.GAT_ERR_TIMEOUT
        # the device arrays of the failed call: pair 2 is -1, the others exact
        import torch

        dev = torch.device("cuda", 0)
        T = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
        oa = np.concatenate([[0], np.cumsum(la)[:-1]]).astype(np.int64)
        ob = np.concatenate([[0], np.cumsum(lb)[:-1]]).astype(np.int64)
        d = [T(la), T(oa), T(a), T(lb), T(ob), T(b)]
        out = torch.full((4,), -7, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        rc = L.lib.gat_edr_pairs_dev(ctx.h, 4, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(),
                                     d[4].data_ptr(), d[5].data_ptr(), 5e-4, out.data_ptr())
        assert rc == L.GAT_ERR_TIMEOUT
        got = out.cpu().numpy()
        assert got[2] == -1
        assert np.array_equal(got[[0, 1, 3]], want[[0, 1, 3]])
        ctx.set_tuning(L.GAT_TUNE_TEST_STALL_CARRY, 0)
        assert np.array_equal(G.edr_pairs(ctx, la, a, lb, b, 5e-4), want)
    finally:
        ctx.close()
