"""Index snapshots on the GPU: each index kind saved and loaded back answers range queries (id
sets and point lists) and top-k exactly as the built one; a different set, a truncated and a
corrupted file are refused."""
import numpy as np
import pytest

import gat_b200 as G
from gat_b200 import _lib as L
from gat_b200 import data as D

pytestmark = pytest.mark.gpu


def test_save_load_every_kind(gpu_ctx, tmp_path):
    t = D.walks(D.lengths(5000, 0, 0, 0, 20, 200, 33), 33)
    db = G.TrajectorySet(gpu_ctx, t)
    q = D.boxes(200, 1, 0.001, 0.05, 34)
    built = {"grid": G.Grid(gpu_ctx, db, D.BOX, 0.0025, 2, 512), "stig": G.STIG(gpu_ctx, db, 256),
             "fsg": G.FSG(gpu_ctx, db, D.BOX, 0.01)}
    for name, ix in built.items():
        p = str(tmp_path / f"{name}.idx")
        ix.save(p)
        back = G.api.Index.load(gpu_ctx, db, p)
        assert type(back) is type(ix) and back.info() == ix.info()
        for res in ("ids", "points"):
            a, b = ix.range_query(q, result=res), back.range_query(q, result=res)
            assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.tids, b.tids)
            if res == "points":
                assert np.array_equal(a.pidx, b.pidx)
        for x, y in zip(ix.points(), back.points()):
            assert np.array_equal(x, y)
        if name == "grid":
            qs = t.subset([3, 77, 4000])
            i1, d1, _ = ix.topk(qs, 8, 5e-4)
            i2, d2, _ = back.topk(qs, 8, 5e-4)
            assert np.array_equal(i1, i2) and np.array_equal(d1, d2)
    p = str(tmp_path / "grid.idx")
    other = G.TrajectorySet(gpu_ctx, D.walks(D.lengths(5000, 0, 0, 0, 20, 200, 35), 35))
    with pytest.raises(G.GatError) as e:
        G.api.Index.load(gpu_ctx, other, p)
    assert e.value.status == L.GAT_ERR_ARG
    raw = open(p, "rb").read()
    (tmp_path / "trunc.idx").write_bytes(raw[: len(raw) // 2])
    with pytest.raises(G.GatError):
        G.api.Index.load(gpu_ctx, db, str(tmp_path / "trunc.idx"))
    bad = bytearray(raw)
    bad[len(bad) // 2] ^= 0xFF
    (tmp_path / "flip.idx").write_bytes(bytes(bad))
    with pytest.raises(G.GatError):
        G.api.Index.load(gpu_ctx, db, str(tmp_path / "flip.idx"))
