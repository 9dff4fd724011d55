"""Python mirror of the library's C ABI (include/gat_b200.h) with the reference's entry points.

Objects own their native handles and release them on `close()` / garbage collection. Every
call goes through libgat_b200.so; results come back as numpy arrays.

The reference's harness API (SystemTest.h:27-33) is mirrored by `SystemTest`:
`rangeQueryTest`, `STIGrangeQueryTest`, `FSGrangeQueryTest` take one MBB repeated
`rangeQueryNum` times (SystemTest.cpp:29-33) and `similarityQueryTest` takes a query trajectory
(or, as in the reference README, a trajectory number) repeated `similarityScale` times.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .data import Trajectories

lib = L.lib


class GatError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"status {status}: {message}")
        self.status = status


def _p(a, t):
    return a.ctypes.data_as(t)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class Context:
    """A CUDA device (device >= 0) with its stream, or a host-only context (device = -1) that
    only builds index layouts."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        rc = lib.gat_ctx_create(device, C.byref(h))
        if rc != L.GAT_OK:
            raise GatError(rc, f"gat_ctx_create({device}) failed")
        self.h = h
        self.device = device
        self._children = weakref.WeakSet()

    def adopt(self, obj) -> None:
        """Handles built on this context; they are released before the context is."""
        self._children.add(obj)

    def check(self, rc: int, what: str = "") -> None:
        if rc != L.GAT_OK:
            msg = lib.gat_last_error(self.h)
            raise GatError(rc, f"{what}: {msg.decode() if msg else ''}")

    @property
    def stream(self) -> int:
        return lib.gat_ctx_stream(self.h) or 0

    def sync(self) -> None:
        self.check(lib.gat_ctx_sync(self.h), "sync")

    @property
    def launches(self) -> int:
        return int(lib.gat_ctx_launches(self.h))

    def set_timing(self, on: bool) -> None:
        self.check(lib.gat_ctx_set_timing(self.h, int(on)), "gat_ctx_set_timing")

    def kernel_stats(self, cls: int) -> dict:
        ms, n, w = C.c_double(0), C.c_int64(0), C.c_double(0)
        self.check(lib.gat_ctx_kernel_stats(self.h, cls, C.byref(ms), C.byref(n), C.byref(w)), "gat_ctx_kernel_stats")
        return dict(ms=ms.value, launches=int(n.value), work=w.value)

    def set_edr_rows(self, rows: int) -> None:
        """Rows per lane of the EDR wavefront: 0 = autotune (default), 2, 4 or 8."""
        self.check(lib.gat_ctx_set_tuning(self.h, L.GAT_TUNE_EDR_ROWS, int(rows)), "gat_ctx_set_tuning")

    def set_tuning(self, knob: int, value: int) -> None:
        self.check(lib.gat_ctx_set_tuning(self.h, knob, int(value)), "gat_ctx_set_tuning")

    def tuning(self, knob: int) -> int:
        v = C.c_int32(0)
        self.check(lib.gat_ctx_get_tuning(self.h, knob, C.byref(v)), "gat_ctx_get_tuning")
        return int(v.value)

    @property
    def scratch_bytes(self) -> int:
        """Device bytes held by the scratch arena and the index-build temporaries kept for reuse."""
        return int(lib.gat_ctx_scratch_bytes(self.h))

    def trim(self) -> None:
        """Returns the scratch arena and kept index-build temporaries to the device (gat_ctx_trim)."""
        self.check(lib.gat_ctx_trim(self.h), "gat_ctx_trim")

    def close(self) -> None:
        if getattr(self, "h", None):
            # indexes first, then trajectory sets: native handles must not outlive the context
            kids = list(self._children)
            for o in kids:
                if isinstance(o, Server):
                    o.close()
            for o in kids:
                if isinstance(o, Index):
                    o.close()
            for o in kids:
                o.close()
            lib.gat_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class TrajectorySet:
    """gat_db: the trajectory set resident in device memory (ids 1..n)."""

    def __init__(self, ctx: Context, traj: Trajectories):
        self.ctx = ctx
        self.traj = traj
        self._keep = (_c(traj.lengths, np.int32), _c(traj.lon, np.float32), _c(traj.lat, np.float32))
        h = C.c_void_p()
        ctx.check(lib.gat_db_create(ctx.h, traj.n, _p(self._keep[0], L.P_i32), _p(self._keep[1], L.P_f32),
                                    _p(self._keep[2], L.P_f32), C.byref(h)), "gat_db_create")
        self.h = h
        ctx.adopt(self)

    def close(self):
        if getattr(self, "h", None) and getattr(self.ctx, "h", None):
            lib.gat_db_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()


@dataclass
class RangeResult:
    offsets: np.ndarray  # int64 [nq+1]
    tids: np.ndarray  # int32
    pidx: np.ndarray | None = None

    def query(self, i: int):
        s, e = self.offsets[i], self.offsets[i + 1]
        return self.tids[s:e] if self.pidx is None else (self.tids[s:e], self.pidx[s:e])


def _mbbs(queries) -> np.ndarray:
    q = _c(queries, np.float32).reshape(-1, 4)
    return q


class Index:
    kind = -1

    def __init__(self, ctx: Context, db: TrajectorySet):
        self.ctx, self.db = ctx, db
        self.h = None
        ctx.adopt(self)

    def close(self):
        if getattr(self, "h", None) and getattr(self.ctx, "h", None):
            lib.gat_index_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def info(self) -> dict:
        a = np.zeros(8, np.int64)
        self.ctx.check(lib.gat_index_info(self.h, _p(a, L.P_i64)), "gat_index_info")
        return dict(kind=int(a[0]), points=int(a[1]), leaves=int(a[2]), nodes=int(a[3]), nx=int(a[4]), ny=int(a[5]),
                    device_bytes=int(a[6]))

    def save(self, path: str) -> None:
        """Index snapshot (gat_index_save): reload with Index.load instead of rebuilding."""
        self.ctx.check(lib.gat_index_save(self.ctx.h, self.h, path.encode()), "gat_index_save")

    @staticmethod
    def load(ctx: "Context", db: "TrajectorySet", path: str) -> "Index":
        """The index saved at path, over the trajectory set it was built from."""
        h = C.c_void_p()
        ctx.check(lib.gat_index_load(ctx.h, db.h, path.encode(), C.byref(h)), "gat_index_load")
        a = np.zeros(8, np.int64)
        lib.gat_index_info(h, _p(a, L.P_i64))
        cls = {L.GAT_INDEX_GRID: Grid, L.GAT_INDEX_STIG: STIG, L.GAT_INDEX_FSG: FSG}[int(a[0])]
        ix = cls.__new__(cls)
        Index.__init__(ix, ctx, db)
        ix.h = h
        return ix

    def points(self):
        n = self.info()["points"]
        x, y = np.zeros(n, np.float32), np.zeros(n, np.float32)
        t, p = np.zeros(n, np.int32), np.zeros(n, np.int32)
        self.ctx.check(lib.gat_index_points(self.ctx.h, self.h, n, _p(x, L.P_f32), _p(y, L.P_f32), _p(t, L.P_i32),
                                            _p(p, L.P_i32)), "gat_index_points")
        return x, y, t, p

    def range_query(self, queries, result: str = "ids", execution: str = "batched", capacity: int | None = None) -> RangeResult:
        """Sorted per-query results: trajectory ids ('ids') or (tid, point index) ('points')."""
        q = _mbbs(queries)
        nq = q.shape[0]
        kind = L.GAT_RESULT_IDS if result == "ids" else L.GAT_RESULT_POINTS
        ex = L.GAT_EXEC_BATCHED if execution == "batched" else L.GAT_EXEC_PLAIN
        cap = capacity if capacity is not None else max(1024, nq * 64)
        while True:
            off = np.zeros(nq + 1, np.int64)
            tid = np.zeros(cap, np.int32)
            pid = np.zeros(cap if kind == L.GAT_RESULT_POINTS else 1, np.int32)
            need = C.c_int64(0)
            rc = lib.gat_range_query(self.ctx.h, self.h, q.ctypes.data_as(C.c_void_p), nq, kind, ex, _p(off, L.P_i64),
                                     _p(tid, L.P_i32), _p(pid, L.P_i32), cap, C.byref(need))
            if rc == L.GAT_ERR_TRUNCATED and capacity is None:
                cap = int(need.value)
                continue
            self.ctx.check(rc, "gat_range_query")
            n = int(need.value)
            return RangeResult(off, tid[:n].copy(), pid[:n].copy() if kind == L.GAT_RESULT_POINTS else None)


class Grid(Index):
    """GT-quadtree (Grid.h:34) with its FVTable: Grid(range, cell, vparam) + addDatasetToGrid."""

    kind = L.GAT_INDEX_GRID

    def __init__(self, ctx: Context, db: TrajectorySet, box, cell_size: float, virtual_cell_param: int = 2, leaf_cap: int = 512):
        super().__init__(ctx, db)
        m = L.MBB(*[float(v) for v in box])
        h = C.c_void_p()
        ctx.check(lib.gat_grid_build(ctx.h, db.h, m, float(cell_size), int(virtual_cell_param), int(leaf_cap), C.byref(h)),
                  "gat_grid_build")
        self.h = h
        self.box, self.cell_size, self.vparam, self.leaf_cap = box, cell_size, virtual_cell_param, leaf_cap

    def fv_lower_bounds(self, queries: Trajectories) -> np.ndarray:
        n = self.db.traj.n
        out = np.zeros((queries.n, n + 1), np.int32)
        lens = _c(queries.lengths, np.int32)
        self.ctx.check(lib.gat_fv_lower_bounds(self.ctx.h, self.h, queries.n, _p(lens, L.P_i32), _p(_c(queries.lon, np.float32), L.P_f32),
                                               _p(_c(queries.lat, np.float32), L.P_f32), _p(out, L.P_i32)), "gat_fv_lower_bounds")
        return out

    def topk(self, queries: Trajectories, k: int, eps: float, execution: str = "batched"):
        """(ids, dist, stats): k nearest trajectories per query by EDR, sorted by (dist, id)."""
        ids = np.zeros((queries.n, k), np.int32)
        dist = np.zeros((queries.n, k), np.int32)
        stats = np.zeros(4, np.int64)
        lens = _c(queries.lengths, np.int32)
        ex = L.GAT_EXEC_BATCHED if execution == "batched" else L.GAT_EXEC_PLAIN
        self.ctx.check(lib.gat_topk(self.ctx.h, self.h, queries.n, _p(lens, L.P_i32), _p(_c(queries.lon, np.float32), L.P_f32),
                                    _p(_c(queries.lat, np.float32), L.P_f32), k, eps, ex, _p(ids, L.P_i32), _p(dist, L.P_i32),
                                    _p(stats, L.P_i64)), "gat_topk")
        return ids, dist, dict(pairs=int(stats[0]), cells=int(stats[1]), launches=int(stats[2]))


class STIG(Index):
    """STIG KD-tree (STIG.h:41): STIG::initial(block_size, 2, db, n)."""

    kind = L.GAT_INDEX_STIG

    def __init__(self, ctx: Context, db: TrajectorySet, block_size: int = 10240):
        super().__init__(ctx, db)
        h = C.c_void_p()
        ctx.check(lib.gat_stig_build(ctx.h, db.h, int(block_size), C.byref(h)), "gat_stig_build")
        self.h = h


class FSG(Index):
    """Flat row-major grid (FSG.h:9): FSG(range, cell) + addDatasetToGrid."""

    kind = L.GAT_INDEX_FSG

    def __init__(self, ctx: Context, db: TrajectorySet, box, cell_size: float):
        super().__init__(ctx, db)
        m = L.MBB(*[float(v) for v in box])
        h = C.c_void_p()
        ctx.check(lib.gat_fsg_build(ctx.h, db.h, m, float(cell_size), C.byref(h)), "gat_fsg_build")
        self.h = h


class MortonGrid(Index):
    """MortonGrid (MortonGrid.h:27): the quadtree of `grid` as a leaf bitmap over implicit node ids
    with computed node boxes; the same range results as the Grid, over the Grid's points (keep the
    Grid alive while this is used)."""

    kind = L.GAT_INDEX_MORTON

    def __init__(self, grid: Grid):
        super().__init__(grid.ctx, grid.db)
        h = C.c_void_p()
        grid.ctx.check(lib.gat_morton_grid_build(grid.ctx.h, grid.h, C.byref(h)), "gat_morton_grid_build")
        self.h = h
        self.grid = grid

    def leaves(self):
        """(level, id) of every leaf, in bitmap order."""
        n = C.c_int64(0)
        lib.gat_morton_grid_leaves(self.ctx.h, self.h, None, None, 0, C.byref(n))
        lv, ids = np.zeros(n.value, np.int32), np.zeros(n.value, np.int32)
        self.ctx.check(lib.gat_morton_grid_leaves(self.ctx.h, self.h, _p(lv, L.P_i32), _p(ids, L.P_i32), n.value, C.byref(n)),
                       "gat_morton_grid_leaves")
        return lv, ids


def edr_pairs(ctx: Context, q_len, q_xy, c_len, c_xy, eps: float) -> np.ndarray:
    """EDR of pair i = (q_xy[q_off[i]:...], c_xy[c_off[i]:...]) with offsets from the lengths."""
    ql, cl = _c(q_len, np.int32), _c(c_len, np.int32)
    qo = np.zeros(len(ql), np.int64)
    co = np.zeros(len(cl), np.int64)
    if len(ql):
        qo[1:] = np.cumsum(ql)[:-1]
        co[1:] = np.cumsum(cl)[:-1]
    qa, ca = _c(q_xy, np.float32).reshape(-1, 2), _c(c_xy, np.float32).reshape(-1, 2)
    out = np.zeros(len(ql), np.int32)
    ctx.check(lib.gat_edr_pairs(ctx.h, len(ql), _p(ql, L.P_i32), _p(qo, L.P_i64), _p(qa, L.P_f32), qa.shape[0],
                                _p(cl, L.P_i32), _p(co, L.P_i64), _p(ca, L.P_f32), ca.shape[0], eps, _p(out, L.P_i32)),
              "gat_edr_pairs")
    return out


class Server:
    """The serving loop (gat_server_*): continuous batching of range and top-k requests over the
    given device-resident indexes, admitted by a device-memory budget."""

    def __init__(self, ctx: Context, grid: Index | None = None, stig: Index | None = None, fsg: Index | None = None,
                 lanes: int = 4, budget_bytes: int = 40 << 30, max_range_batch: int = 4096, max_topk_batch: int = 32):
        self.ctx = ctx
        self.h = None
        cfg = L.ServerConfig(lanes, budget_bytes, max_range_batch, max_topk_batch)
        h = C.c_void_p()
        hs = [x.h if x is not None else None for x in (grid, stig, fsg)]
        ctx.check(lib.gat_server_create(ctx.h, hs[0], hs[1], hs[2], C.byref(cfg), C.byref(h)), "gat_server_create")
        self.h = h
        self._keep = (grid, stig, fsg)
        ctx.adopt(self)

    def close(self) -> None:
        if getattr(self, "h", None):
            lib.gat_server_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def submit_range(self, box, index_kind: int = L.GAT_INDEX_GRID, result: str = "ids") -> int:
        b = np.asarray(box, np.float32).reshape(4)
        rid = C.c_int64(0)
        kind = L.GAT_RESULT_IDS if result == "ids" else L.GAT_RESULT_POINTS
        rc = lib.gat_server_submit_range(self.h, index_kind, L.MBB(*[float(v) for v in b]), kind, C.byref(rid))
        if rc != L.GAT_OK:
            raise GatError(rc, "gat_server_submit_range")
        return int(rid.value)

    def submit_topk(self, lon, lat, k: int, eps: float) -> int:
        x, y = _c(lon, np.float32), _c(lat, np.float32)
        rid = C.c_int64(0)
        rc = lib.gat_server_submit_topk(self.h, len(x), _p(x, L.P_f32), _p(y, L.P_f32), k, eps, C.byref(rid))
        if rc != L.GAT_OK:
            raise GatError(rc, "gat_server_submit_topk")
        return int(rid.value)

    def wait(self, rid: int, timeout_ms: int = -1) -> int:
        """The request's own status (GAT_OK, GAT_ERR_OOM, ...)."""
        st = C.c_int32(0)
        rc = lib.gat_server_wait(self.h, rid, timeout_ms, C.byref(st))
        if rc != L.GAT_OK:
            raise GatError(rc, "gat_server_wait")
        return int(st.value)

    def range_result(self, rid: int, points: bool = False):
        n = C.c_int64(0)
        rc = lib.gat_server_range_result(self.h, rid, None, None, 0, C.byref(n))
        if rc not in (L.GAT_OK, L.GAT_ERR_TRUNCATED):
            raise GatError(rc, "gat_server_range_result")
        t = np.zeros(max(1, n.value), np.int32)
        p = np.zeros(max(1, n.value), np.int32)
        rc = lib.gat_server_range_result(self.h, rid, _p(t, L.P_i32), _p(p, L.P_i32), n.value, C.byref(n))
        if rc != L.GAT_OK:
            raise GatError(rc, "gat_server_range_result")
        return (t[:n.value], p[:n.value]) if points else t[:n.value]

    def topk_result(self, rid: int, k: int):
        ids, dist = np.zeros(k, np.int32), np.zeros(k, np.int32)
        rc = lib.gat_server_topk_result(self.h, rid, _p(ids, L.P_i32), _p(dist, L.P_i32), k)
        if rc != L.GAT_OK:
            raise GatError(rc, "gat_server_topk_result")
        return ids, dist

    def times(self, rid: int) -> np.ndarray:
        """(arrival, admission, completion) in ns since the server started."""
        t = np.zeros(3, np.int64)
        rc = lib.gat_server_request_times(self.h, rid, _p(t, L.P_i64))
        if rc != L.GAT_OK:
            raise GatError(rc, "gat_server_request_times")
        return t

    def release(self, rid: int) -> None:
        rc = lib.gat_server_release(self.h, rid)
        if rc != L.GAT_OK:
            raise GatError(rc, "gat_server_release")

    def stats(self) -> dict:
        a = np.zeros(8, np.int64)
        lib.gat_server_stats(self.h, _p(a, L.P_i64))
        keys = ["submitted", "completed", "batches", "range_batches", "topk_batches", "peak_admitted_bytes",
                "largest_batch", "failed"]
        return dict(zip(keys, (int(v) for v in a)))


class SystemTest:
    """The reference's harness entry points (SystemTest.h:13-35) over this library."""

    def __init__(self, tradb: Trajectories, g: Grid | None, stig: STIG | None, fsg: FSG | None, eps: float = 0.005,
                 mgrid: MortonGrid | None = None):
        self.tradb, self.g, self.stig, self.fsg, self.eps, self.mgrid = tradb, g, stig, fsg, eps, mgrid

    @staticmethod
    def _repeat(mbb, n):
        return np.tile(np.asarray(mbb, np.float32).reshape(1, 4), (n, 1))

    def rangeQueryTest(self, rangeQueryMBB, rangeQueryNum: int) -> RangeResult:
        return self.g.range_query(self._repeat(rangeQueryMBB, rangeQueryNum))

    def STIGrangeQueryTest(self, rangeQueryMBB, rangeQueryNum: int) -> RangeResult:
        return self.stig.range_query(self._repeat(rangeQueryMBB, rangeQueryNum))

    def FSGrangeQueryTest(self, rangeQueryMBB, rangeQueryNum: int) -> RangeResult:
        return self.fsg.range_query(self._repeat(rangeQueryMBB, rangeQueryNum))

    def rangeQueryTestWithoutMorton(self, rangeQueryMBB, rangeQueryNum: int) -> RangeResult:
        """SystemTest.h:29. The reference's pretend-row-major walk (Grid.cpp:544-662) never
        advances its segment offsets (Grid.cpp:818-827), so its results are not the Grid's and
        there is nothing of its own to reproduce; this runs the GT-quadtree path."""
        return self.rangeQueryTest(rangeQueryMBB, rangeQueryNum)

    def MortonGridRangeQueryTest(self, rangeQueryMBB, rangeQueryNum: int) -> RangeResult:
        """SystemTest.h:33: the MortonGrid's implicit-tree walk (MortonGrid.cpp:268-393); its id
        sets are the Grid's. Without a MortonGrid the Grid answers."""
        ix = self.mgrid if self.mgrid is not None else self.g
        return ix.range_query(self._repeat(rangeQueryMBB, rangeQueryNum))

    def similarityQueryTest(self, t, similarityScale: int, similarityKValue: int):
        """t: a Trajectories holding one query, or an int trajectory number (README.md:30)."""
        if isinstance(t, (int, np.integer)):
            t = self.tradb.subset([int(t)])
        q = t.subset(np.ones(similarityScale, np.int64))
        return self.g.topk(q, similarityKValue, self.eps)
