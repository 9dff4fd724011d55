"""The allocation-free EDR entry point, gat_edr_pairs_dev_noalloc.

It serves callers that cannot call cudaMalloc (inside a capture they do not own, under a
no-allocation policy, or with a fixed device footprint): it takes only a stream and device
arrays and keeps its working memory in a fixed device array inside the library. This test
calls it through the C ABI twice in a row, with different pair sets, and checks each result
against the regular entry point gat_edr_pairs_dev, exactly (EDR distances are integers). The
test allocates its own buffers; the entry point allocates nothing. Collected last on purpose.
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


def test_noalloc_matches_regular_entry_twice():
    import torch

    import gat_b200 as G
    from gat_b200 import _lib as L
    from gat_b200 import data as D

    dev = torch.device("cuda", 0)
    ctx = G.Context(0)
    stream = torch.cuda.Stream(dev)
    for call, (n, lo, hi, seed) in enumerate([(700, 1, 1500, 51), (300, 16, 4096, 52)]):
        la = D.lengths(n, L.GAT_LEN_LOGUNIFORM, 0, 0, lo, hi, seed)
        lb = D.lengths(n, L.GAT_LEN_LOGUNIFORM, 0, 0, lo, hi, seed + 100)
        a, b = D.pairs(la, lb, seed + 200)
        ql, qo, qxy, cl, co, cxy = _dev_pairs(torch, dev, la, a, lb, b)
        want = torch.empty(n, dtype=torch.int32, device=dev)
        got = torch.full((n,), -7, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        rc = L.lib.gat_edr_pairs_dev(ctx.h, n, ql.data_ptr(), qo.data_ptr(), qxy.data_ptr(), cl.data_ptr(), co.data_ptr(),
                                     cxy.data_ptr(), 5e-4, want.data_ptr())
        assert rc == L.GAT_OK
        max_len = int(max(la.max(), lb.max()))
        rc = L.lib.gat_edr_pairs_dev_noalloc(C.c_void_p(stream.cuda_stream), n, max_len, ql.data_ptr(), qo.data_ptr(),
                                             qxy.data_ptr(), cl.data_ptr(), co.data_ptr(), cxy.data_ptr(), 5e-4,
                                             got.data_ptr())
        assert rc == L.GAT_OK, f"call {call}"
        stream.synchronize()
        assert torch.equal(got, want), f"call {call}: no-alloc results differ from gat_edr_pairs_dev"
    ctx.close()


def test_noalloc_rejects_lengths_beyond_its_scratch():
    from gat_b200 import _lib as L

    rc = L.lib.gat_edr_pairs_dev_noalloc(None, 1, L.GAT_EDR_NOALLOC_MAX_LEN + 1, None, None, None, None, None, None,
                                         5e-4, None)
    assert rc == L.GAT_ERR_ARG
