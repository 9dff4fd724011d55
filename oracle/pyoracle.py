"""Python access to the test oracles. TEST INFRASTRUCTURE ONLY.

- `Oracle*` classes wrap oracle/liboracle.so, the CPU restatement of the reference's
  algorithms (oracle/oracle.cpp).
- `RefRunner` runs oracle/_ref/gatref, the reference's own CPU code compiled from its sources
  (oracle/Makefile + oracle/ref_driver.cpp), through the binary file format ref_driver.cpp
  documents.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
GATREF = os.path.join(HERE, "_ref", "gatref")

P_i32 = C.POINTER(C.c_int32)
P_i64 = C.POINTER(C.c_int64)
P_f32 = C.POINTER(C.c_float)
c_p = C.c_void_p

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise ImportError(f"{ORACLE_SO} missing: run `make -C oracle`")
        L = C.CDLL(ORACLE_SO)
        sig = {
            "orc_grid_build": (c_p, [C.c_int, P_i32, P_f32, P_f32, P_f32, C.c_float, C.c_int, C.c_int]),
            "orc_grid_free": (None, [c_p]),
            "orc_grid_meta": (None, [c_p, P_i32]),
            "orc_grid_points": (None, [c_p, P_f32, P_f32, P_i32, P_i32]),
            "orc_grid_cells": (None, [c_p, P_i32, P_i32, P_f32]),
            "orc_grid_nodes": (None, [c_p, P_i32, P_i32, P_i32, P_i32, P_f32]),
            "orc_grid_fv": (C.c_int64, [c_p, P_i64, P_i32, P_i32]),
            "orc_grid_range": (None, [c_p, P_f32, C.c_int, C.c_int, P_i64, P_i32, P_i32]),
            "orc_grid_candidates": (C.c_int, [c_p, P_f32, P_i32, P_i32]),
            "orc_stig_build": (c_p, [C.c_int, P_i32, P_f32, P_f32, C.c_int]),
            "orc_stig_free": (None, [c_p]),
            "orc_stig_npoints": (C.c_int64, [c_p]),
            "orc_stig_points": (None, [c_p, P_f32, P_f32, P_i32, P_i32]),
            "orc_stig_leaves": (C.c_int, [c_p, P_i32, P_f32]),
            "orc_stig_candidates": (C.c_int, [c_p, P_f32, P_i32]),
            "orc_stig_range": (None, [c_p, P_f32, C.c_int, C.c_int, P_i64, P_i32, P_i32]),
            "orc_fsg_build": (c_p, [C.c_int, P_i32, P_f32, P_f32, P_f32, C.c_float]),
            "orc_fsg_free": (None, [c_p]),
            "orc_fsg_meta": (None, [c_p, P_i32]),
            "orc_fsg_points": (None, [c_p, P_f32, P_f32, P_i32, P_i32]),
            "orc_fsg_cells": (None, [c_p, P_i32, P_i32]),
            "orc_fsg_candidates": (C.c_int, [c_p, P_f32, P_i32]),
            "orc_fsg_range": (None, [c_p, P_f32, C.c_int, C.c_int, P_i64, P_i32, P_i32]),
            "orc_edr": (C.c_int32, [P_f32, C.c_int, P_f32, C.c_int, C.c_double]),
            "orc_edr_batch": (None, [C.c_int, P_i32, P_i64, P_f32, P_i32, P_i64, P_f32, C.c_double, C.c_int, P_i32]),
            "orc_fv_neighbors": (None, [C.c_int, C.c_int, P_i32]),
            "orc_grid_query_fv": (C.c_int, [c_p, P_f32, P_f32, C.c_int, P_i32, P_i32]),
            "orc_grid_fv_lb": (None, [c_p, C.c_int, P_i32, P_i32, P_i32]),
            "orc_grid_topk": (None, [c_p, P_f32, P_f32, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, P_i32, P_i32, P_i64]),
            "orc_gen_lengths": (None, [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_uint64, P_i32]),
            "orc_gen_walks": (None, [C.c_int, P_i32, P_f32, C.c_double, C.c_uint64, P_f32, P_f32]),
            "orc_gen_boxes": (None, [C.c_int, C.c_int, C.c_double, C.c_double, P_f32, C.c_uint64, P_f32]),
            "orc_gen_sample_ids": (None, [C.c_int, C.c_int, C.c_uint64, P_i32]),
            "orc_gen_pairs": (None, [C.c_int, P_i32, P_i32, P_f32, C.c_double, C.c_double, C.c_uint64, P_f32, P_f32]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _csr_from_counts(counts):
    off = np.zeros(len(counts) + 1, dtype=np.int64)
    np.cumsum(counts, out=off[1:])
    return off


class _RangeMixin:
    _range_fn = None

    def range(self, queries, mode: int = 0):
        """mode 0: (offsets, ids); mode 1: (offsets, tids, pidx). Sorted per query."""
        q = _c(queries, np.float32).reshape(-1, 4)
        nq = q.shape[0]
        counts = np.zeros(nq, dtype=np.int64)
        fn = getattr(lib(), self._range_fn)
        fn(self.h, _p(q, P_f32), nq, mode, _p(counts, P_i64), None, None)
        off = _csr_from_counts(counts)
        a = np.zeros(int(off[-1]), dtype=np.int32)
        b = np.zeros(int(off[-1]), dtype=np.int32)
        fn(self.h, _p(q, P_f32), nq, mode, _p(counts, P_i64), _p(a, P_i32), _p(b, P_i32))
        return (off, a) if mode == 0 else (off, a, b)


class OracleGrid(_RangeMixin):
    _range_fn = "orc_grid_range"

    def __init__(self, traj, box, cell: float, vparam: int = 2, leaf_cap: int = 512):
        self.lengths = _c(traj.lengths, np.int32)
        self.lon = _c(traj.lon, np.float32)
        self.lat = _c(traj.lat, np.float32)
        self.box = np.asarray(box, dtype=np.float32)
        self.n = len(self.lengths)
        self.h = lib().orc_grid_build(self.n, _p(self.lengths, P_i32), _p(self.lon, P_f32), _p(self.lat, P_f32),
                                      _p(self.box, P_f32), cell, vparam, leaf_cap)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_grid_free(self.h)
            self.h = None

    def meta(self):
        m = np.zeros(6, dtype=np.int32)
        lib().orc_grid_meta(self.h, _p(m, P_i32))
        return dict(axis=int(m[0]), cellnum=int(m[1]), points=int(m[2]), levels=int(m[3]), leaves=int(m[4]), nodes=int(m[5]))

    def points(self):
        n = self.meta()["points"]
        x, y = np.zeros(n, np.float32), np.zeros(n, np.float32)
        t, p = np.zeros(n, np.int32), np.zeros(n, np.int32)
        lib().orc_grid_points(self.h, _p(x, P_f32), _p(y, P_f32), _p(t, P_i32), _p(p, P_i32))
        return x, y, t, p

    def cells(self):
        n = self.meta()["cellnum"]
        s, e, m = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros((n, 4), np.float32)
        lib().orc_grid_cells(self.h, _p(s, P_i32), _p(e, P_i32), _p(m, P_f32))
        return s, e, m

    def nodes(self):
        n = self.meta()["nodes"]
        a = [np.zeros(n, np.int32) for _ in range(4)]
        m = np.zeros((n, 4), np.float32)
        lib().orc_grid_nodes(self.h, *[_p(x, P_i32) for x in a], _p(m, P_f32))
        return dict(id=a[0], level=a[1], npts=a[2], leaf=a[3], mbb=m)

    def fv(self):
        k = lib().orc_grid_fv(self.h, None, None, None)
        off = np.zeros(self.n + 2, np.int64)
        cell, cnt = np.zeros(k, np.int32), np.zeros(k, np.int32)
        lib().orc_grid_fv(self.h, _p(off, P_i64), _p(cell, P_i32), _p(cnt, P_i32))
        return off, cell, cnt

    def candidates(self, q):
        q = _c(q, np.float32)
        k = lib().orc_grid_candidates(self.h, _p(q, P_f32), None, None)
        ids, lv = np.zeros(k, np.int32), np.zeros(k, np.int32)
        lib().orc_grid_candidates(self.h, _p(q, P_f32), _p(ids, P_i32), _p(lv, P_i32))
        return ids, lv

    def query_fv(self, lon, lat):
        lon, lat = _c(lon, np.float32), _c(lat, np.float32)
        k = lib().orc_grid_query_fv(self.h, _p(lon, P_f32), _p(lat, P_f32), len(lon), None, None)
        c, n = np.zeros(k, np.int32), np.zeros(k, np.int32)
        lib().orc_grid_query_fv(self.h, _p(lon, P_f32), _p(lat, P_f32), len(lon), _p(c, P_i32), _p(n, P_i32))
        return c, n

    def fv_lb(self, lon, lat):
        c, n = self.query_fv(lon, lat)
        lb = np.zeros(self.n + 1, np.int32)
        lib().orc_grid_fv_lb(self.h, len(c), _p(c, P_i32), _p(n, P_i32), _p(lb, P_i32))
        return lb

    def topk(self, lon, lat, k: int, eps: float, pruned: bool = True, threads: int = 8):
        lon, lat = _c(lon, np.float32), _c(lat, np.float32)
        ids, dist = np.zeros(k, np.int32), np.zeros(k, np.int32)
        ev = np.zeros(1, np.int64)
        lib().orc_grid_topk(self.h, _p(lon, P_f32), _p(lat, P_f32), len(lon), k, eps, int(pruned), threads,
                            _p(ids, P_i32), _p(dist, P_i32), _p(ev, P_i64))
        return ids, dist, int(ev[0])


class OracleSTIG(_RangeMixin):
    _range_fn = "orc_stig_range"

    def __init__(self, traj, block: int):
        self.lengths = _c(traj.lengths, np.int32)
        self.lon = _c(traj.lon, np.float32)
        self.lat = _c(traj.lat, np.float32)
        self.h = lib().orc_stig_build(len(self.lengths), _p(self.lengths, P_i32), _p(self.lon, P_f32), _p(self.lat, P_f32), block)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_stig_free(self.h)
            self.h = None

    def points(self):
        n = lib().orc_stig_npoints(self.h)
        x, y = np.zeros(n, np.float32), np.zeros(n, np.float32)
        t, p = np.zeros(n, np.int32), np.zeros(n, np.int32)
        lib().orc_stig_points(self.h, _p(x, P_f32), _p(y, P_f32), _p(t, P_i32), _p(p, P_i32))
        return x, y, t, p

    def leaves(self):
        k = lib().orc_stig_leaves(self.h, None, None)
        lr, m = np.zeros((k, 2), np.int32), np.zeros((k, 4), np.float32)
        lib().orc_stig_leaves(self.h, _p(lr, P_i32), _p(m, P_f32))
        return lr, m

    def candidates(self, q):
        q = _c(q, np.float32)
        k = lib().orc_stig_candidates(self.h, _p(q, P_f32), None)
        b = np.zeros((k, 2), np.int32)
        lib().orc_stig_candidates(self.h, _p(q, P_f32), _p(b, P_i32))
        return b


class OracleFSG(_RangeMixin):
    _range_fn = "orc_fsg_range"

    def __init__(self, traj, box, cell: float):
        self.lengths = _c(traj.lengths, np.int32)
        self.lon = _c(traj.lon, np.float32)
        self.lat = _c(traj.lat, np.float32)
        self.box = np.asarray(box, dtype=np.float32)
        self.h = lib().orc_fsg_build(len(self.lengths), _p(self.lengths, P_i32), _p(self.lon, P_f32), _p(self.lat, P_f32),
                                     _p(self.box, P_f32), cell)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_fsg_free(self.h)
            self.h = None

    def meta(self):
        m = np.zeros(4, np.int32)
        lib().orc_fsg_meta(self.h, _p(m, P_i32))
        return dict(nx=int(m[0]), ny=int(m[1]), cellnum=int(m[2]), points=int(m[3]))

    def points(self):
        n = self.meta()["points"]
        x, y = np.zeros(n, np.float32), np.zeros(n, np.float32)
        t, p = np.zeros(n, np.int32), np.zeros(n, np.int32)
        lib().orc_fsg_points(self.h, _p(x, P_f32), _p(y, P_f32), _p(t, P_i32), _p(p, P_i32))
        return x, y, t, p

    def cells(self):
        n = self.meta()["cellnum"]
        s, e = np.zeros(n, np.int32), np.zeros(n, np.int32)
        lib().orc_fsg_cells(self.h, _p(s, P_i32), _p(e, P_i32))
        return s, e

    def candidates(self, q):
        q = _c(q, np.float32)
        k = lib().orc_fsg_candidates(self.h, _p(q, P_f32), None)
        c = np.zeros(k, np.int32)
        lib().orc_fsg_candidates(self.h, _p(q, P_f32), _p(c, P_i32))
        return c


# ---------------------------------------------------------------- seeded workloads (oracle/datagen.cpp)
BOX = (121.0, 30.7, 122.0, 31.7)
STEP = 1e-4
LEN_UNIFORM, LEN_LOGNORMAL, LEN_LOGUNIFORM = 0, 1, 2
SIDE_FIXED, SIDE_LOGUNIFORM = 0, 1


class Walks:
    """A trajectory set (ids 1..n) with the attributes the oracle classes and RefRunner read."""

    def __init__(self, lengths, lon, lat):
        self.lengths, self.lon, self.lat = lengths, lon, lat

    @property
    def n(self) -> int:
        return int(self.lengths.shape[0])

    @property
    def offsets(self):
        off = np.zeros(self.n + 1, dtype=np.int64)
        np.cumsum(self.lengths, out=off[1:])
        return off

    def points(self, tid: int):
        off = self.offsets
        return self.lon[off[tid - 1]:off[tid]], self.lat[off[tid - 1]:off[tid]]


def gen_lengths(n, kind, p0, p1, lo, hi, seed):
    out = np.empty(n, np.int32)
    lib().orc_gen_lengths(n, kind, p0, p1, lo, hi, seed, _p(out, P_i32))
    return out


def gen_walks(lens, seed, box=BOX, step=STEP):
    lens = _c(lens, np.int32)
    total = int(lens.astype(np.int64).sum())
    lon, lat = np.empty(total, np.float32), np.empty(total, np.float32)
    b = np.asarray(box, np.float32)
    lib().orc_gen_walks(len(lens), _p(lens, P_i32), _p(b, P_f32), step, seed, _p(lon, P_f32), _p(lat, P_f32))
    return Walks(lens, lon, lat)


def gen_boxes(n, kind, s0, s1, seed, box=BOX):
    out = np.empty((n, 4), np.float32)
    b = np.asarray(box, np.float32)
    lib().orc_gen_boxes(n, kind, s0, s1, _p(b, P_f32), seed, _p(out, P_f32))
    return out


def gen_sample_ids(k, n, seed):
    out = np.empty(k, np.int32)
    lib().orc_gen_sample_ids(k, n, seed, _p(out, P_i32))
    return out


def gen_pairs(la, lb, seed, jitter=2.5e-4, box=BOX, step=STEP):
    la, lb = _c(la, np.int32), _c(lb, np.int32)
    a = np.empty((int(la.astype(np.int64).sum()), 2), np.float32)
    bb = np.empty((int(lb.astype(np.int64).sum()), 2), np.float32)
    b = np.asarray(box, np.float32)
    lib().orc_gen_pairs(len(la), _p(la, P_i32), _p(lb, P_i32), _p(b, P_f32), step, jitter, seed, _p(a, P_f32), _p(bb, P_f32))
    return a, bb


def config1(seed=0, n=10_000, nq=1_000):
    """10k walks of U[20, 200] points; nq squares of side 0.01 deg."""
    t = gen_walks(gen_lengths(n, LEN_UNIFORM, 0, 0, 20, 200, seed), seed)
    return t, gen_boxes(nq, SIDE_FIXED, 0.01, 0.01, seed)


def config2(seed=0, n=100_000, nq=256):
    """100k walks, lengths lognormal(ln 200, 0.6) clipped to [32, 1024]; nq query ids from the set."""
    t = gen_walks(gen_lengths(n, LEN_LOGNORMAL, float(np.log(200.0)), 0.6, 32, 1024, seed), seed)
    return t, gen_sample_ids(nq, n, seed)


def config3(seed=0, n=1_000_000, nq=100_000):
    """1M walks of U[50, 350] points; nq rectangles with sides log-U[0.001, 0.05] deg."""
    t = gen_walks(gen_lengths(n, LEN_UNIFORM, 0, 0, 50, 350, seed), seed)
    return t, gen_boxes(nq, SIDE_LOGUNIFORM, 0.001, 0.05, seed)


def config4_pairs(seed=0, npairs=4096, lo=16, hi=4096):
    """EDR pairs with both lengths log-uniform in [lo, hi]."""
    la = gen_lengths(npairs, LEN_LOGUNIFORM, 0, 0, lo, hi, seed)
    lb = gen_lengths(npairs, LEN_LOGUNIFORM, 0, 0, lo, hi, seed + 1)
    a, b = gen_pairs(la, lb, seed)
    return la, a, lb, b


def edr(a_xy, b_xy, eps: float) -> int:
    a, b = _c(a_xy, np.float32).reshape(-1, 2), _c(b_xy, np.float32).reshape(-1, 2)
    return int(lib().orc_edr(_p(a, P_f32), a.shape[0], _p(b, P_f32), b.shape[0], eps))


def edr_batch(la, a_xy, lb, b_xy, eps: float, threads: int = 8) -> np.ndarray:
    la, lb = _c(la, np.int32), _c(lb, np.int32)
    oa, ob = _csr_from_counts(la)[:-1].copy(), _csr_from_counts(lb)[:-1].copy()
    a, b = _c(a_xy, np.float32), _c(b_xy, np.float32)
    out = np.zeros(len(la), np.int32)
    lib().orc_edr_batch(len(la), _p(la, P_i32), _p(oa, P_i64), _p(a, P_f32), _p(lb, P_i32), _p(ob, P_i64), _p(b, P_f32),
                        eps, threads, _p(out, P_i32))
    return out


def fv_neighbors(vcells: int, cell: int) -> np.ndarray:
    out = np.zeros(8, np.int32)
    lib().orc_fv_neighbors(vcells, cell, _p(out, P_i32))
    return out


# ---------------------------------------------------------------- the reference binary
def ref_available() -> bool:
    return os.path.exists(GATREF)


def write_data(path: str, traj) -> None:
    with open(path, "wb") as f:
        f.write(b"GATD")
        f.write(struct.pack("<iq", traj.n, int(len(traj.lon))))
        f.write(_c(traj.lengths, np.int32).tobytes())
        f.write(_c(traj.lon, np.float32).tobytes())
        f.write(_c(traj.lat, np.float32).tobytes())


def write_queries(path: str, q) -> None:
    q = _c(q, np.float32).reshape(-1, 4)
    with open(path, "wb") as f:
        f.write(b"GATQ")
        f.write(struct.pack("<i", q.shape[0]))
        f.write(q.tobytes())


def write_ids(path: str, ids) -> None:
    ids = _c(ids, np.int32)
    with open(path, "wb") as f:
        f.write(b"GATI")
        f.write(struct.pack("<i", len(ids)))
        f.write(ids.tobytes())


def write_pairs(path: str, la, a_xy, lb, b_xy) -> None:
    la, lb = _c(la, np.int32), _c(lb, np.int32)
    with open(path, "wb") as f:
        f.write(b"GATP")
        f.write(struct.pack("<i", len(la)))
        f.write(la.tobytes())
        f.write(lb.tobytes())
        f.write(_c(a_xy, np.float32).tobytes())
        f.write(_c(b_xy, np.float32).tobytes())


def read_out(path: str) -> dict:
    out = {}
    dt = {b"i": np.int32, b"l": np.int64, b"f": np.float32, b"d": np.float64}
    with open(path, "rb") as f:
        buf = f.read()
    pos = 0
    while pos < len(buf):
        (nl,) = struct.unpack_from("<i", buf, pos)
        pos += 4
        name = buf[pos:pos + nl].decode()
        pos += nl
        code = buf[pos:pos + 1]
        pos += 1
        (cnt,) = struct.unpack_from("<q", buf, pos)
        pos += 8
        t = dt[code]
        nbytes = cnt * np.dtype(t).itemsize
        out[name] = np.frombuffer(buf, dtype=t, count=cnt, offset=pos).copy()
        pos += nbytes
    return out


class RefRunner:
    """Runs the compiled reference (oracle/_ref/gatref) in a scratch directory."""

    def __init__(self):
        if not ref_available():
            raise FileNotFoundError(f"{GATREF} missing (build with `make -C oracle` where the reference sources exist)")
        self.dir = tempfile.mkdtemp(prefix="gatref_")

    def _run(self, args, timeout=3600):
        r = subprocess.run([GATREF] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"gatref {args[0]} failed ({r.returncode}): {r.stderr[-2000:]}")
        return r

    def _path(self, name):
        return os.path.join(self.dir, name)

    def gtq(self, traj, queries, box, cell, leaf_cap, layout=False, threads=0):
        d, q, o = self._path("d.bin"), self._path("q.bin"), self._path("o.bin")
        write_data(d, traj)
        write_queries(q, queries)
        self._run(["gtq", d, q, o, repr(float(cell)), leaf_cap, *[repr(float(v)) for v in box], int(layout), threads])
        return read_out(o)

    def wfile(self, traj, path, box):
        """PreProcess::writeTraDataToFile of the given trajectories (point times 0) to path."""
        d = self._path("d.bin")
        write_data(d, traj)
        self._run(["wfile", d, path, *[repr(float(v)) for v in box]])

    def stig(self, traj, queries, block, layout=False):
        d, q, o = self._path("d.bin"), self._path("q.bin"), self._path("o.bin")
        write_data(d, traj)
        write_queries(q, queries)
        self._run(["stig", d, q, o, block, int(layout)])
        return read_out(o)

    def fsg(self, traj, box, cell):
        d, o = self._path("d.bin"), self._path("o.bin")
        write_data(d, traj)
        self._run(["fsg", d, o, repr(float(cell)), *[repr(float(v)) for v in box]])
        return read_out(o)

    def edr(self, la, a_xy, lb, b_xy, eps, threads=1):
        p, o = self._path("p.bin"), self._path("o.bin")
        write_pairs(p, la, a_xy, lb, b_xy)
        self._run(["edr", p, o, repr(float(eps)), threads])
        return read_out(o)

    def fvlb(self, traj, qids, box, cell):
        d, i, o = self._path("d.bin"), self._path("i.bin"), self._path("o.bin")
        write_data(d, traj)
        write_ids(i, qids)
        self._run(["fvlb", d, i, o, repr(float(cell)), *[repr(float(v)) for v in box]])
        r = read_out(o)
        return r["lb"].reshape(len(qids), traj.n + 1)

    def topk(self, traj, qids, box, cell, k, eps, reps=1, timeout=3600):
        d, i, o = self._path("d.bin"), self._path("i.bin"), self._path("o.bin")
        write_data(d, traj)
        write_ids(i, qids)
        self._run(["topk", d, i, o, repr(float(cell)), k, repr(float(eps)), *[repr(float(v)) for v in box], reps],
                  timeout=timeout)
        r = read_out(o)
        r["ids"] = r["ids"].reshape(len(qids), k)
        r["dist"] = r["dist"].reshape(len(qids), k)
        return r

    def rangebench(self, n, len_lo, len_hi, seed, nq, side_lo, side_hi, cell, leaf_cap, box, per_step, steps,
                   threads, timeout=3600):
        """The reference's Grid over n generated walks and Grid::rangeQueryBatch over `steps`
        strided samples of per_step of the nq generated rectangles, on `threads` threads
        (ref_driver.cpp cmd_rangebench)."""
        o = self._path("o.bin")
        self._run(["rangebench", o, n, len_lo, len_hi, seed, nq, repr(float(side_lo)), repr(float(side_hi)),
                   repr(float(cell)), leaf_cap, *[repr(float(v)) for v in box], per_step, steps, threads], timeout=timeout)
        return read_out(o)

    def nbr(self, cells, vcells):
        i, o = self._path("i.bin"), self._path("o.bin")
        write_ids(i, cells)
        self._run(["nbr", i, o, vcells])
        r = read_out(o)
        return r["nbr"].reshape(-1, 8), r["idx_grid"].reshape(12, 12)
