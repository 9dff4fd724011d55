"""Seeded synthetic workloads (host arrays), produced by the library's generator.

The reference measures on a taxi trajectory file that is not available; these stand in for it
with the shapes and distributions of the five workloads (random walks in the
[121, 122] x [30.7, 31.7] degree box, N(0, 1e-4 deg) steps clamped to the box).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L

BOX = (121.0, 30.7, 122.0, 31.7)  # xmin, ymin, xmax, ymax
STEP = 1e-4


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _check(rc: int, what: str) -> None:
    if rc != L.GAT_OK:
        raise RuntimeError(f"{what} failed with status {rc}")


@dataclass
class Trajectories:
    """Trajectory set: ids 1..n; lengths[i] points of trajectory i+1 at lon/lat[off[i]:off[i+1]]."""

    lengths: np.ndarray  # int32 [n]
    lon: np.ndarray  # float32 [P]
    lat: np.ndarray  # float32 [P]

    @property
    def n(self) -> int:
        return int(self.lengths.shape[0])

    @property
    def offsets(self) -> np.ndarray:
        off = np.zeros(self.n + 1, dtype=np.int64)
        np.cumsum(self.lengths, out=off[1:])
        return off

    def points(self, tid: int) -> tuple[np.ndarray, np.ndarray]:
        off = self.offsets
        s, e = off[tid - 1], off[tid]
        return self.lon[s:e], self.lat[s:e]

    def subset(self, ids) -> "Trajectories":
        """Trajectories with the given ids, concatenated in that order."""
        off = self.offsets
        ids = np.asarray(ids, dtype=np.int64)
        lens = self.lengths[ids - 1].astype(np.int32)
        idx = np.concatenate([np.arange(off[i - 1], off[i]) for i in ids]) if len(ids) else np.zeros(0, np.int64)
        return Trajectories(lens, self.lon[idx].copy(), self.lat[idx].copy())


def lengths(n: int, kind: int, p0: float, p1: float, lo: int, hi: int, seed: int) -> np.ndarray:
    out = np.empty(n, dtype=np.int32)
    _check(L.lib.gat_gen_lengths(n, kind, p0, p1, lo, hi, seed, _p(out, L.P_i32)), "gat_gen_lengths")
    return out


def walks(lens: np.ndarray, seed: int, box=BOX, step: float = STEP) -> Trajectories:
    lens = np.ascontiguousarray(lens, dtype=np.int32)
    total = int(lens.astype(np.int64).sum())
    lon = np.empty(total, dtype=np.float32)
    lat = np.empty(total, dtype=np.float32)
    b = np.asarray(box, dtype=np.float32)
    _check(L.lib.gat_gen_walks(len(lens), _p(lens, L.P_i32), _p(b, L.P_f32), step, seed, _p(lon, L.P_f32), _p(lat, L.P_f32)), "gat_gen_walks")
    return Trajectories(lens, lon, lat)


def boxes(n: int, side_kind: int, s0: float, s1: float, seed: int, box=BOX) -> np.ndarray:
    out = np.empty((n, 4), dtype=np.float32)
    b = np.asarray(box, dtype=np.float32)
    _check(L.lib.gat_gen_boxes(n, side_kind, s0, s1, _p(b, L.P_f32), seed, _p(out, L.P_f32)), "gat_gen_boxes")
    return out


def sample_ids(k: int, n: int, seed: int) -> np.ndarray:
    out = np.empty(k, dtype=np.int32)
    _check(L.lib.gat_gen_sample_ids(k, n, seed, _p(out, L.P_i32)), "gat_gen_sample_ids")
    return out


def pairs(len_a: np.ndarray, len_b: np.ndarray, seed: int, jitter: float = 2.5e-4, box=BOX, step: float = STEP):
    la = np.ascontiguousarray(len_a, dtype=np.int32)
    lb = np.ascontiguousarray(len_b, dtype=np.int32)
    a = np.empty((int(la.astype(np.int64).sum()), 2), dtype=np.float32)
    bb = np.empty((int(lb.astype(np.int64).sum()), 2), dtype=np.float32)
    b = np.asarray(box, dtype=np.float32)
    _check(L.lib.gat_gen_pairs(len(la), _p(la, L.P_i32), _p(lb, L.P_i32), _p(b, L.P_f32), step, jitter, seed, _p(a, L.P_f32), _p(bb, L.P_f32)), "gat_gen_pairs")
    return a, bb


# ---------------------------------------------------------------- the five workloads
def config1(seed: int = 0, n: int = 10_000, nq: int = 1_000):
    """Plain GT-quadtree range query: 10k walks of U[20, 200] points, 1k squares of 0.01 deg."""
    t = walks(lengths(n, L.GAT_LEN_UNIFORM, 0, 0, 20, 200, seed), seed)
    q = boxes(nq, L.GAT_SIDE_FIXED, 0.01, 0.01, seed)
    return t, q


def config2(seed: int = 0, n: int = 100_000, nq: int = 256):
    """Plain EDR top-k: 100k walks, lengths lognormal(ln 200, 0.6) clipped to [32, 1024];
    256 query trajectories sampled from the set."""
    t = walks(lengths(n, L.GAT_LEN_LOGNORMAL, float(np.log(200.0)), 0.6, 32, 1024, seed), seed)
    qids = sample_ids(nq, n, seed)
    return t, qids


def config3(seed: int = 0, n: int = 1_000_000, nq: int = 100_000):
    """Batched range: 1M walks of U[50, 350] points, 100k rectangles, sides log-U[0.001, 0.05]."""
    t = walks(lengths(n, L.GAT_LEN_UNIFORM, 0, 0, 50, 350, seed), seed)
    q = boxes(nq, L.GAT_SIDE_LOGUNIFORM, 0.001, 0.05, seed)
    return t, q


def config4_pairs(seed: int = 0, npairs: int = 4096, lo: int = 16, hi: int = 4096):
    """Batched EDR: pairs with both lengths log-uniform in [16, 4096]."""
    la = lengths(npairs, L.GAT_LEN_LOGUNIFORM, 0, 0, lo, hi, seed)
    lb = lengths(npairs, L.GAT_LEN_LOGUNIFORM, 0, 0, lo, hi, seed + 1)
    a, b = pairs(la, lb, seed)
    return la, a, lb, b


# ---------------------------------------------------------------- trajectory files
def read_trajectory_file(path: str):
    """(Trajectories, box, times) from the reference's formatted trajectory file
    (PreProcess::readTraFromFormatedFile)."""
    n, npts = C.c_int32(0), C.c_int64(0)
    box = np.zeros(4, np.float32)
    _check(L.lib.gat_traj_file_info(path.encode(), C.byref(n), C.byref(npts), _p(box, L.P_f32)), "gat_traj_file_info")
    lens = np.zeros(n.value, np.int32)
    lon, lat = np.zeros(npts.value, np.float32), np.zeros(npts.value, np.float32)
    times = np.zeros(npts.value, np.int32)
    _check(L.lib.gat_traj_file_read(path.encode(), n.value, npts.value, _p(lens, L.P_i32), _p(lon, L.P_f32),
                                    _p(lat, L.P_f32), _p(times, L.P_i32)), "gat_traj_file_read")
    return Trajectories(lens, lon, lat), tuple(float(v) for v in box), times


def write_trajectory_file(path: str, t: Trajectories, box=BOX, times=None) -> None:
    """The reference's formatted trajectory file (PreProcess::writeTraDataToFile)."""
    lens = np.ascontiguousarray(t.lengths, np.int32)
    lon, lat = np.ascontiguousarray(t.lon, np.float32), np.ascontiguousarray(t.lat, np.float32)
    b = np.asarray(box, np.float32)
    tm = None if times is None else np.ascontiguousarray(times, np.int32)
    _check(L.lib.gat_traj_file_write(path.encode(), t.n, _p(lens, L.P_i32), _p(lon, L.P_f32), _p(lat, L.P_f32),
                                     None if tm is None else _p(tm, L.P_i32), _p(b, L.P_f32)), "gat_traj_file_write")
