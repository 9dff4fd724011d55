"""The reference's formatted trajectory file (PreProcess.cpp:203-315): the writer reproduces
the reference writer's bytes, the reader returns what was written (at the %f precision of the
format), headers and malformed files are handled."""
import os

import numpy as np
import pytest

from gat_b200 import data as D
from oracle import pyoracle as po


def _set():
    t = D.walks(D.lengths(300, 0, 0, 0, 1, 40, 17), 17)
    return t


def test_round_trip(tmp_path):
    t = _set()
    times = np.arange(len(t.lon), dtype=np.int32) * 7
    p = str(tmp_path / "t.txt")
    D.write_trajectory_file(p, t, D.BOX, times)
    r, box, rt = D.read_trajectory_file(p)
    assert np.array_equal(r.lengths, t.lengths) and np.array_equal(rt, times)
    # %f keeps 6 decimals: the read value is the float nearest to the printed decimal
    want_lon = np.array([float(f"{v:f}") for v in t.lon.astype(np.float64)], np.float32)
    want_lat = np.array([float(f"{v:f}") for v in t.lat.astype(np.float64)], np.float32)
    assert np.array_equal(r.lon, want_lon) and np.array_equal(r.lat, want_lat)
    assert np.allclose(box, D.BOX)
    # a second round trip is exact
    p2 = str(tmp_path / "t2.txt")
    D.write_trajectory_file(p2, r, box, rt)
    assert open(p, "rb").read() == open(p2, "rb").read()


@pytest.mark.skipif(not po.ref_available(), reason="the reference's own code is not built here")
def test_writer_matches_reference_bytes(tmp_path):
    t = _set()
    mine, theirs = str(tmp_path / "mine.txt"), str(tmp_path / "ref.txt")
    D.write_trajectory_file(mine, t, D.BOX)
    po.RefRunner().wfile(t, theirs, D.BOX)
    assert open(mine, "rb").read() == open(theirs, "rb").read()


def test_empty_trajectories_and_errors(tmp_path):
    t = D.Trajectories(np.array([0, 3, 0], np.int32), np.array([121.1, 121.2, 121.3], np.float32),
                       np.array([31.1, 31.2, 31.3], np.float32))
    p = str(tmp_path / "e.txt")
    D.write_trajectory_file(p, t, D.BOX)
    r, _, _ = D.read_trajectory_file(p)
    assert np.array_equal(r.lengths, [0, 3, 0]) and len(r.lon) == 3
    bad = tmp_path / "bad.txt"
    bad.write_text("2\n121,30.7,122,31.7\n1;1;\n31.0,121.0,1,0;\n")  # second trajectory missing
    with pytest.raises(RuntimeError):
        D.read_trajectory_file(str(bad))
    bad.write_text("2\n121,30.7,122\n1;1;\n")  # short box line
    with pytest.raises(RuntimeError):
        D.read_trajectory_file(str(bad))
    bad.write_text("1\n121,30.7,122,31.7\n1;\n--31.5,121.0,1,0;\n")  # two signs: strtod converts nothing
    with pytest.raises(RuntimeError):
        D.read_trajectory_file(str(bad))
    with pytest.raises(RuntimeError):
        D.read_trajectory_file(str(tmp_path / "missing.txt"))


def test_reader_accepts_what_strtod_accepts(tmp_path):
    """Fields parse as the reference's strtod / strtol parse them: leading blanks and '+', an
    exponent, hexadecimal floats, inf and nan, integers beyond the int range (saturated, then
    converted to int32 as the old reader did)."""
    p = tmp_path / "odd.txt"
    p.write_text("2\n121,30.7,122,31.7\n2;2;\n"
                 " +31.5, 121.25,1, +7;3.15e1,0x1.e4p+6,1,-8;\n"
                 "inf,-nan,2,99999999999999;1.0,2.0,2,99999999999999999999999;\n")
    r, _, times = D.read_trajectory_file(str(p))
    assert r.lengths.tolist() == [2, 2]
    assert r.lat[0] == np.float32(31.5) and r.lon[0] == np.float32(121.25)
    assert r.lat[1] == np.float32(31.5) and r.lon[1] == np.float32(float.fromhex("0x1.e4p+6"))
    assert np.isinf(r.lat[2]) and np.isnan(r.lon[2])
    assert times[0] == 7 and times[1] == -8
    assert times[2] == np.int64(99999999999999).astype(np.int32)  # a long, converted to int32
    assert times[3] == np.int64(2**63 - 1).astype(np.int32)  # beyond a long: strtol saturates
