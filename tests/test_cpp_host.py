"""The C++ host layer (include/gat_b200.hpp): a GAT-style program using gat::SystemTest, Grid,
STIG, FSG and MortonGrid over the C ABI, compiled with g++ and checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

from gat_b200 import _lib as L
from gat_b200 import data as D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "gat_b200")


@pytest.fixture(scope="module")
def demo(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "systemtest_demo")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "systemtest_demo.cpp"), "-L", LIBDIR, "-lgat_b200",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def run(exe, device, n=2000, path=None):
    r = subprocess.run([exe, str(device), str(n)] + ([path] if path else []), capture_output=True, text=True, timeout=600)
    out = {}
    for line in r.stdout.splitlines():
        f = line.split()
        if len(f) >= 2 and f[0] in ("build", "mortonbuild", "rangeQueryTest", "STIGrangeQueryTest", "FSGrangeQueryTest",
                                    "rangeQueryTestWithoutMorton", "MortonGridRangeQueryTest", "rangeQueryBatch",
                                    "similarityQueryTest", "file_roundtrip", "tuning"):
            out[f[0]] = int(f[1])
        elif len(f) >= 2:
            out[f[0]] = np.array([int(x) for x in f[2:]], np.int64)
            assert len(out[f[0]]) == int(f[1])
    return r.returncode, out, r.stdout + r.stderr


def test_host_only(demo, tmp_path):
    """Without a GPU the indexes build through the C++ classes and every query reports
    GAT_ERR_STATE instead of aborting; the trajectory file helpers round-trip."""
    rc, out, log = run(demo, -1, path=str(tmp_path / "tradb.txt"))
    assert rc == 0, log
    assert out["build"] == 0 and out["file_roundtrip"] == 1 and out["tuning"] == 3
    assert out["mortonbuild"] == L.GAT_ERR_STATE
    for k in ("rangeQueryTest", "STIGrangeQueryTest", "FSGrangeQueryTest", "rangeQueryTestWithoutMorton",
              "MortonGridRangeQueryTest", "rangeQueryBatch", "similarityQueryTest"):
        assert out[k] == L.GAT_ERR_STATE, (k, log)


@pytest.mark.gpu
def test_systemtest_matches_oracle(demo):
    from oracle import pyoracle as po

    rc, out, log = run(demo, 0)
    assert rc == 0, log
    assert out["mortonbuild"] == 0  # MortonGridRangeQueryTest below runs the MortonGrid
    t = D.walks(D.lengths(2000, 0, 0, 0, 20, 200, 0), 0)
    q = np.array([[121.40, 31.00, 121.45, 31.06]], np.float32)
    off, ids = po.OracleGrid(t, D.BOX, 0.01, 2, 512).range(q, 0)
    assert np.array_equal(out["grid_off"], np.arange(4) * off[1]) and np.array_equal(out["grid_ids"], np.tile(ids, 3))
    soff, sids = po.OracleSTIG(t, 256).range(q)
    assert np.array_equal(out["stig_ids"], np.tile(sids, 2)) and out["stig_off"][1] == soff[1]
    foff, fids = po.OracleFSG(t, D.BOX, 0.01).range(q)
    assert np.array_equal(out["fsg_ids"], np.tile(fids, 2)) and out["fsg_off"][1] == foff[1]
    assert np.array_equal(out["nonmorton_ids"], np.tile(ids, 2)) and np.array_equal(out["mortongrid_ids"], np.tile(ids, 2))
    qs = D.boxes(16, 1, 0.002, 0.05, 5)
    poff, ptid, ppidx = po.OracleGrid(t, D.BOX, 0.01, 2, 512).range(qs, 1)
    assert np.array_equal(out["pts_off"], poff) and np.array_equal(out["pts_tid"], ptid)
    assert np.array_equal(out["pts_pidx"], ppidx)
    wi, wd, _ = po.OracleGrid(t, D.BOX, 0.01, 2, 512).topk(*t.points(47), 8, 5e-4, pruned=False)
    assert np.array_equal(out["topk_ids"], np.tile(wi, 2)) and np.array_equal(out["topk_dist"], np.tile(wd, 2))
