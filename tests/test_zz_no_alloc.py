"""The allocation-free EDR entry point, gat_edr_pairs_dev_noalloc.

It serves callers that cannot call cudaMalloc (inside a capture they do not own, under a
no-allocation policy, or with a fixed device footprint): it takes only a stream and device
arrays and keeps its working memory in a fixed device array inside the library. These tests call
it through the C ABI twice in a row, with different pair sets, and check each result against the
regular entry point gat_edr_pairs_dev and against the oracle, exactly (EDR distances are
integers); pairs with a side beyond the caller's max_len must come back as -1 with the rest
exact; and a warmed-up call must leave the device's free memory unchanged. The tests allocate
their own buffers; the entry point allocates nothing. Collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev_pairs(torch, dev, la, a, lb, b):
    oa = np.zeros(len(la), np.int64)
    ob = np.zeros(len(lb), np.int64)
    oa[1:] = np.cumsum(la)[:-1]
    ob[1:] = np.cumsum(lb)[:-1]
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    return t(la.astype(np.int32)), t(oa), t(a.astype(np.float32)), t(lb.astype(np.int32)), t(ob), t(b.astype(np.float32))


def _noalloc(L, stream, n, max_len, d, out):
    ql, qo, qxy, cl, co, cxy = d
    return L.lib.gat_edr_pairs_dev_noalloc(C.c_void_p(stream.cuda_stream), n, max_len, ql.data_ptr(), qo.data_ptr(),
                                           qxy.data_ptr(), cl.data_ptr(), co.data_ptr(), cxy.data_ptr(), 5e-4,
                                           out.data_ptr())


def test_noalloc_matches_regular_entry_and_oracle_twice():
    import torch

    import gat_b200 as G
    from gat_b200 import _lib as L
    from gat_b200 import data as D
    from oracle import pyoracle as po

    dev = torch.device("cuda", 0)
    ctx = G.Context(0)
    stream = torch.cuda.Stream(dev)
    for call, (n, lo, hi, seed) in enumerate([(700, 1, 1500, 51), (300, 16, 4096, 52)]):
        la = D.lengths(n, L.GAT_LEN_LOGUNIFORM, 0, 0, lo, hi, seed)
        lb = D.lengths(n, L.GAT_LEN_LOGUNIFORM, 0, 0, lo, hi, seed + 100)
        a, b = D.pairs(la, lb, seed + 200)
        d = _dev_pairs(torch, dev, la, a, lb, b)
        want = torch.empty(n, dtype=torch.int32, device=dev)
        got = torch.full((n,), -7, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        rc = L.lib.gat_edr_pairs_dev(ctx.h, n, *[x.data_ptr() for x in d], 5e-4, want.data_ptr())
        assert rc == L.GAT_OK
        rc = _noalloc(L, stream, n, int(max(la.max(), lb.max())), d, got)
        assert rc == L.GAT_OK, f"call {call}"
        stream.synchronize()
        assert torch.equal(got, want), f"call {call}: no-alloc results differ from gat_edr_pairs_dev"
        assert np.array_equal(got.cpu().numpy(), po.edr_batch(la, a, lb, b, 5e-4)), f"call {call}: differ from the oracle"
    ctx.close()


def test_noalloc_sides_beyond_max_len_get_minus_one():
    """max_len 1000 with sides up to 1500: exactly the pairs with a longer side get -1, every
    other pair equals the regular entry point; a second call, warmed up, changes no free memory."""
    import torch

    import gat_b200 as G
    from gat_b200 import _lib as L
    from gat_b200 import data as D

    dev = torch.device("cuda", 0)
    ctx = G.Context(0)
    stream = torch.cuda.Stream(dev)
    n, max_len = 400, 1000
    la = D.lengths(n, L.GAT_LEN_LOGUNIFORM, 0, 0, 1, 1500, 71)
    lb = D.lengths(n, L.GAT_LEN_LOGUNIFORM, 0, 0, 1, 1500, 72)
    a, b = D.pairs(la, lb, 73)
    d = _dev_pairs(torch, dev, la, a, lb, b)
    want = torch.empty(n, dtype=torch.int32, device=dev)
    got = torch.full((n,), -7, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    assert L.lib.gat_edr_pairs_dev(ctx.h, n, *[x.data_ptr() for x in d], 5e-4, want.data_ptr()) == L.GAT_OK
    torch.cuda.synchronize()
    over = (la > max_len) | (lb > max_len)
    assert over.any() and (~over).any()
    for call in range(2):
        free0 = torch.cuda.mem_get_info(dev)[0]
        assert _noalloc(L, stream, n, max_len, d, got) == L.GAT_OK
        stream.synchronize()
        free1 = torch.cuda.mem_get_info(dev)[0]
        g, w = got.cpu().numpy(), want.cpu().numpy()
        assert np.all(g[over] == -1), f"call {call}"
        assert np.array_equal(g[~over], w[~over]), f"call {call}"
        if call == 1:
            assert free1 == free0, "a warmed-up call changed the device's free memory"
    ctx.close()


def test_noalloc_rejects_lengths_beyond_its_scratch():
    from gat_b200 import _lib as L

    rc = L.lib.gat_edr_pairs_dev_noalloc(None, 1, L.GAT_EDR_NOALLOC_MAX_LEN + 1, None, None, None, None, None, None,
                                         5e-4, None)
    assert rc == L.GAT_ERR_ARG
