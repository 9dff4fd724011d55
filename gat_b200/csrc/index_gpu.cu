/* Device builders of the Grid (GT-quadtree + FVTable) and FSG indexes, in the layouts of
 * Grid::addDatasetToGrid (Grid.cpp:210-316, quadtree Grid.cpp:58-94, frequency vectors
 * Grid.cpp:152-166 / FVTable.cpp:18-30) and FSG::addDatasetToGrid (FSG.cpp:95-143).
 *
 * Both indexes order points by cell, trajectories ascending within a cell and points in
 * trajectory order within a trajectory: a stable sort by cell of the set's points taken in
 * trajectory order, which is a stable sort of the maximal runs of consecutive points sharing a
 * cell (a walk stays in one cell for several points). The build runs entirely in HBM:
 *   1. cells      every point's cell from the builders' float expressions (IEEE single
 *                 subtract and divide, truncation toward zero) and a flag where a run starts;
 *   2. runs       run starts compacted; per run its cell, trajectory (from a per-256-point hint
 *                 table and a short search of the offsets) and length; runs stably radix-sorted
 *                 by cell, their lengths scanned into destinations;
 *   3. expand     each block fills 2048 consecutive index positions from the runs covering
 *                 them (staged in shared memory): x, y, trajectory, key;
 *   4. bounds     cell boundaries from the sorted runs' cells and destinations;
 *   5. quadtree   (Grid) level by level: split flags, a scan, children written in parents' order,
 *                 which is the breadth-first order of the reference's queue; node MBBs from the
 *                 same float expressions as the host builder;
 *   6. vectors    (Grid) each trajectory's (virtual cell, count) list in ascending cell order:
 *                 cell runs merged into runs of equal virtual cells, keyed (trajectory, virtual
 *                 cell), radix-sorted, counts summed per key.
 * The host copies of the points are downloaded only when asked for (gat_index_points,
 * snapshots). The radix sorts, scans, selection and reduce-by-key are CUB's (the CUDA toolkit's
 * header library); an index build runs once per trajectory set and is not on the query path. */
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "cells.cuh"
#include "internal.h"

namespace gat {
namespace {

constexpr int kHintShift = 8;   /* one trajectory hint per 256 points */
constexpr int kMaxLevels = 32;

/* the trajectory holding every 256th point: hint[b] = the trajectory of point b << kHintShift */
__global__ void k_hints(int n, const int64_t* __restrict__ off, int32_t* hint) {
    for (int t = 1 + blockIdx.x * blockDim.x + threadIdx.x; t <= n; t += gridDim.x * blockDim.x) {
        const int64_t e = off[t + 1];
        for (int64_t b = (off[t] + (1 << kHintShift) - 1) >> kHintShift; (b << kHintShift) < e; b++) hint[b] = t;
    }
}

/* the trajectory holding point s: the largest t with off[t] <= s, searched between the hints of
 * s's block and the next (an empty trajectory shares its successor's offset and so is never the
 * largest) */
__device__ __forceinline__ int holder(int64_t s, int n, const int64_t* __restrict__ off, const int32_t* __restrict__ hint,
                                      int64_t nhint) {
    const int64_t b = s >> kHintShift;
    int lo = hint[b], hi = b + 1 < nhint ? hint[b + 1] : n;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= s)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

constexpr int kPerThread = 4; /* points each lane of k_point_cells keeps in flight */

/* 1. every point's cell (trajectory order) and the run heads: 1 where a point's cell differs
 * from its predecessor's (trajectory starts are marked by k_run_starts). Each warp takes chunks
 * of 32 x kPerThread consecutive points; a point's predecessor is in the lane below, in lane 31
 * of the previous step, or (for the chunk's first point) recomputed from the point before. */
__global__ void k_point_cells(int64_t P, const float2* __restrict__ xy, CellParams p, uint32_t* cell, uint8_t* head,
                              int32_t* flag) {
    constexpr int kChunk = 32 * kPerThread;
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    bool bad = false;
    for (int64_t base = (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * kChunk; base < P; base += nw * kChunk) {
        float2 v[kPerThread];
#pragma unroll
        for (int k = 0; k < kPerThread; k++) {
            const int64_t i = base + k * 32 + lane;
            v[k] = i < P ? xy[i] : make_float2(0.f, 0.f);
        }
        const float2 before = (lane == 0 && base > 0) ? xy[base - 1] : make_float2(0.f, 0.f);
        int carry = (lane == 0 && base > 0) ? max(point_cell(p, before.x, before.y), 0) : -1;
#pragma unroll
        for (int k = 0; k < kPerThread; k++) {
            const int64_t i = base + k * 32 + lane;
            int c = i < P ? point_cell(p, v[k].x, v[k].y) : 0;
            if (c < 0) {
                bad = true;
                c = 0;
            }
            int prev = __shfl_up_sync(0xffffffffu, c, 1);
            if (lane == 0) prev = carry;
            carry = __shfl_sync(0xffffffffu, c, 31);
            if (i < P) {
                cell[i] = (uint32_t)c;
                head[i] = (i == 0 || c != prev) ? 1 : 0;
            }
        }
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicCAS(flag, 0, GAT_ERR_ARG);
}

/* a run never spans two trajectories */
__global__ void k_run_starts(int n, const int64_t* __restrict__ off, uint8_t* head) {
    for (int t = 1 + blockIdx.x * blockDim.x + threadIdx.x; t <= n; t += gridDim.x * blockDim.x)
        if (off[t + 1] > off[t]) head[off[t]] = 1;
}

/* 2. per run (trajectory order): its cell, index, trajectory and length */
__global__ void k_runs(int64_t R, int64_t P, int n, const int32_t* __restrict__ starts, const int64_t* __restrict__ off,
                       const int32_t* __restrict__ hint, int64_t nhint, const uint32_t* __restrict__ cells,
                       uint32_t* run_cell, int32_t* run_idx, int32_t* run_tid, int32_t* run_len) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < R; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = starts[r], e = r + 1 < R ? starts[r + 1] : P;
        run_cell[r] = cells[s];
        run_idx[r] = (int32_t)r;
        run_tid[r] = holder(s, n, off, hint, nhint);
        run_len[r] = (int32_t)(e - s);
    }
}

/* the runs in sorted order, packed (source start, trajectory, point index of the start, length),
 * and their lengths for the scan into destinations (len[R] = 0 closes it) */
__global__ void k_sorted_runs(int64_t R, const int32_t* __restrict__ order, const int32_t* __restrict__ starts,
                              const int32_t* __restrict__ run_tid, const int32_t* __restrict__ run_len,
                              const int64_t* __restrict__ off, int4* rec, int32_t* len) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j <= R; j += (int64_t)gridDim.x * blockDim.x) {
        if (j == R) {
            len[j] = 0;
            continue;
        }
        const int r = order[j];
        const int st = starts[r], t = run_tid[r], L = run_len[r];
        rec[j] = make_int4(st, t, (int)(st - off[t]), L);
        len[j] = L;
    }
}

constexpr int kExpandTile = 2048;  /* output positions per block of k_expand_runs */
constexpr int kExpandThreads = 256;

/* first[b] = the last sorted run whose destination is <= b * kExpandTile */
__global__ void k_tile_first(int64_t ntiles, int64_t R, const int32_t* __restrict__ dest, int32_t* first) {
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < ntiles; b += (int64_t)gridDim.x * blockDim.x) {
        const int64_t lo = b * kExpandTile;
        int64_t a = 0, e = R - 1;
        while (a < e) {
            const int64_t mid = (a + e + 1) >> 1;
            if (dest[mid] <= lo)
                a = mid;
            else
                e = mid - 1;
        }
        first[b] = (int32_t)a;
    }
}

/* 3. points to their index positions: block b fills the kExpandTile positions from b * kExpandTile.
 * It stages the sorted runs covering them in shared memory, marks each run's first position
 * with its index and fills the tile with a block-wide max-scan, so each position reads its run
 * directly; then writes x, y, trajectory and key = tid << pidx_bits | pidx (0 when the pair does
 * not fit 32 bits; pidx_bits < 0, the point index then goes to pidx). */
__global__ void __launch_bounds__(kExpandThreads) k_expand_runs(
    int64_t P, int64_t R, int64_t ntiles, const int32_t* __restrict__ first, const int4* __restrict__ rec,
    const int32_t* __restrict__ dest, const float2* __restrict__ xy, float* x, float* y, int32_t* tid, uint32_t* key,
    int32_t* pidx, int pidx_bits) {
    constexpr int kPer = kExpandTile / kExpandThreads;
    constexpr int kWarps = kExpandThreads / 32;
    __shared__ int s_dest[kExpandTile + 1], s_src[kExpandTile + 1], s_tid[kExpandTile + 1], s_k0[kExpandTile + 1];
    __shared__ int s_run[kExpandTile];
    __shared__ int s_warp[kWarps];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t b = blockIdx.x;
    const int64_t lo = b * kExpandTile;
    const int64_t hi = min(P, lo + kExpandTile);
    const int a0 = first[b];
    const int a1 = b + 1 < ntiles ? first[b + 1] : (int)(R - 1);
    /* runs a0 .. a1 cover [lo, hi); each run holds at least one point, so there are at most
     * kExpandTile + 1 of them */
    const int m = a1 - a0 + 1;
    for (int k = threadIdx.x; k < kExpandTile; k += kExpandThreads) s_run[k] = 0;
    __syncthreads();
    for (int q = threadIdx.x; q < m; q += kExpandThreads) {
        const int4 v = rec[a0 + q];
        const int d = dest[a0 + q];
        s_dest[q] = d;
        s_src[q] = v.x;
        s_tid[q] = v.y;
        s_k0[q] = v.z;
        /* run 0 starts at or before lo and covers position 0 */
        if (q > 0 && d - lo < kExpandTile) s_run[d - lo] = q;
    }
    __syncthreads();
    /* inclusive max-scan of s_run: each thread its kPer consecutive entries, then across threads */
    int loc[kPer];
    int run = 0;
#pragma unroll
    for (int k = 0; k < kPer; k++) {
        run = max(run, s_run[threadIdx.x * kPer + k]);
        loc[k] = run;
    }
    int incl = run;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl = max(incl, o);
    }
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    int carry = 0;
    for (int k = 0; k < w; k++) carry = max(carry, s_warp[k]);
    int excl = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl = 0;
    carry = max(carry, excl);
#pragma unroll
    for (int k = 0; k < kPer; k++) s_run[threadIdx.x * kPer + k] = max(loc[k], carry);
    __syncthreads();
    for (int64_t i = lo + threadIdx.x; i < hi; i += kExpandThreads) {
        const int a = s_run[i - lo];
        const int d = (int)(i - s_dest[a]);
        const float2 v = xy[s_src[a] + d];
        const int t = s_tid[a], q = s_k0[a] + d;
        x[i] = v.x;
        y[i] = v.y;
        tid[i] = t;
        key[i] = pidx_bits >= 0 ? ((uint32_t)t << pidx_bits) | (uint32_t)q : 0u;
        if (pidx) pidx[i] = q;
    }
}

/* 4. cell boundaries from the sorted runs: cb[c] = destination of the first run whose cell is >= c */
__global__ void k_cell_bounds(int64_t R, int64_t ncells, const uint32_t* __restrict__ run_cell_s,
                              const int32_t* __restrict__ dest, int64_t* cb) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c <= ncells; c += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = R;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((int64_t)run_cell_s[mid] < c)
                lo = mid + 1;
            else
                hi = mid;
        }
        cb[c] = dest[lo];
    }
}

/* 4. bound[j] = the first position p in the sorted keys with keys[p] >= j << shift, j = 0..m */
template <class K>
__global__ void k_bounds(int64_t P, int64_t m, const K* __restrict__ keys, int shift, int64_t* bound) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j <= m; j += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long want = (unsigned long long)j << shift;
        int64_t lo = 0, hi = P;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((unsigned long long)keys[mid] < want)
                lo = mid + 1;
            else
                hi = mid;
        }
        bound[j] = lo;
    }
}

/* FSG cell ranges [cbeg, cend) from the boundaries (FSG.cpp:119-140) */
__global__ void k_fsg_cells(int64_t ncells, const int64_t* __restrict__ cb, int32_t* cbeg, int32_t* cend) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells; c += (int64_t)gridDim.x * blockDim.x) {
        cbeg[c] = (int32_t)cb[c];
        cend[c] = (int32_t)cb[c + 1];
    }
}

/* ---------------------------------------------------------------- 5. quadtree */
struct TreeParams {
    float rxmin, rymax, cell;
    int total_level, leaf_cap;
};

__device__ __forceinline__ int64_t node_span(int level, int total_level) {
    return (int64_t)1 << (2 * (total_level - level));
}

/* split flag of each node of one level; flags[m] = 0 closes the scan */
__global__ void k_tree_split(int64_t m, int level, const int32_t* __restrict__ ids, const int64_t* __restrict__ cb,
                             TreeParams tp, int32_t* flags) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j <= m; j += (int64_t)gridDim.x * blockDim.x) {
        if (j == m) {
            flags[j] = 0;
            continue;
        }
        const int64_t span = node_span(level, tp.total_level);
        const int64_t first = (int64_t)ids[j] * span, last = first + span - 1;
        const int64_t pts = cb[last + 1] - cb[first];
        /* Grid::buildQuadTree (Grid.cpp:58-94): a leaf below the point cap or at the last level */
        flags[j] = (pts < tp.leaf_cap || level == tp.total_level) ? 0 : 1;
    }
}

/* children of the split nodes of one level, in their parents' order (the breadth-first queue) */
__global__ void k_tree_children(int64_t m, const int32_t* __restrict__ ids, const int32_t* __restrict__ flags,
                                const int32_t* __restrict__ spos, int64_t base_next, int32_t* next_ids, int32_t* child) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x) {
        if (!flags[j]) {
            child[j] = -1;
            continue;
        }
        const int64_t c0 = base_next + 4 * (int64_t)spos[j];
        child[j] = (int32_t)c0;
        for (int c = 0; c < 4; c++) next_ids[c0 - base_next + c] = (ids[j] << 2) + c;
    }
}

struct LevelTable {
    int64_t base[kMaxLevels + 1];
    int nlevels;
};

__device__ __forceinline__ float4 cell_box(const TreeParams& tp, int c) { return morton_cell_box(tp.rxmin, tp.rymax, tp.cell, c); }

/* node arrays in breadth-first order: MBB, first child, point range */
__global__ void k_tree_nodes(int64_t N, LevelTable lt, const int32_t* __restrict__ ids, const int32_t* __restrict__ child_in,
                             const int64_t* __restrict__ cb, TreeParams tp, float4* mbb, int32_t* child, int32_t* pbeg,
                             int32_t* pend) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < N; j += (int64_t)gridDim.x * blockDim.x) {
        int level = 0;
        while (level + 1 < lt.nlevels && lt.base[level + 1] <= j) level++;
        const int64_t span = node_span(level, tp.total_level);
        const int64_t first = (int64_t)ids[j] * span, last = first + span - 1;
        const float4 a = cell_box(tp, (int)first), b = cell_box(tp, (int)last);
        mbb[j] = make_float4(a.x, b.y, b.z, a.w);
        child[j] = child_in[j];
        pbeg[j] = (int32_t)cb[first];
        pend[j] = (int32_t)cb[last + 1];
    }
}

/* ---------------------------------------------------------------- 6. frequency vectors */
/* heads of runs of equal virtual cells: a cell run whose trajectory or virtual cell differs from
 * the previous run's */
__global__ void k_vrun_heads(int64_t R, const uint32_t* __restrict__ run_cell, const int32_t* __restrict__ run_tid,
                             int vparam, uint8_t* vhead) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < R; r += (int64_t)gridDim.x * blockDim.x)
        vhead[r] = (r == 0 || run_tid[r] != run_tid[r - 1] || (run_cell[r] >> vparam) != (run_cell[r - 1] >> vparam)) ? 1 : 0;
}

/* per virtual-cell run: key (trajectory << 32 | virtual cell) and point count */
__global__ void k_vruns(int64_t Rv, int64_t R, int64_t P, const int32_t* __restrict__ vstarts,
                        const int32_t* __restrict__ starts, const uint32_t* __restrict__ run_cell,
                        const int32_t* __restrict__ run_tid, int vparam, unsigned long long* key, int32_t* cnt) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < Rv; v += (int64_t)gridDim.x * blockDim.x) {
        const int a = vstarts[v];
        const int64_t b = v + 1 < Rv ? vstarts[v + 1] : R;
        key[v] = ((unsigned long long)(unsigned)run_tid[a] << 32) | (run_cell[a] >> vparam);
        cnt[v] = (int32_t)((b < R ? (int64_t)starts[b] : P) - starts[a]);
    }
}

struct AddInt {
    __device__ __forceinline__ int operator()(int a, int b) const { return a + b; }
};

/* frequency-vector cells: the low half of each (trajectory, virtual cell) key */
__global__ void k_fv_cells(int64_t R, const unsigned long long* __restrict__ runs, int32_t* cell) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < R; r += (int64_t)gridDim.x * blockDim.x)
        cell[r] = (int32_t)(runs[r] & 0xffffffffull);
}

/* ---------------------------------------------------------------- host side */
/* device temporaries of one build, taken from the context's pool in stream order and returned
 * to it (after the work queued on the stream) when the build ends */
struct Temps {
    gat_ctx* ctx;
    cudaMemPool_t pool;
    std::vector<void*> ptrs;
    cudaError_t err = cudaSuccess;
    explicit Temps(gat_ctx* c) : ctx(c), pool(build_pool(c)) {}
    Temps(const Temps&) = delete;
    Temps& operator=(const Temps&) = delete;
    ~Temps() {
        for (void* p : ptrs)
            if (p) drop(p);
    }
    void drop(void* p) {
        if (pool)
            cudaFreeAsync(p, ctx->stream);
        else
            cudaFree(p);
    }
    template <class T>
    T* get(size_t n) {
        if (err != cudaSuccess) return nullptr;
        void* p = nullptr;
        const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
        err = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, ctx->stream) : cudaMalloc(&p, bytes);
        if (err != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    /* returns one temporary early (stream-ordered: after the work already queued) */
    void release(void* p) {
        for (auto& q : ptrs)
            if (q && q == p) {
                drop(q);
                q = nullptr;
            }
    }
};

int bits_to_hold(int64_t v) {
    int b = 1;
    while (b < 62 && (int64_t(1) << b) <= v) b++;
    return b;
}

int grid_size(const gat_ctx* ctx, int64_t work, int per_block = 256) {
    const int64_t want = (work + per_block - 1) / per_block;
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)std::max(1, ctx->sm_count) * 8));
}

/* index array of `count` elements of T plus the host builder's one element of padding, zeroed */
template <class T>
T* alloc_padded(gat_index* ix, int64_t count, int* st) {
    T* p = (T*)index_alloc(ix, (size_t)(count + 1) * sizeof(T), st);
    if (!p) return nullptr;
    const cudaError_t e = cudaMemsetAsync(p + count, 0, sizeof(T), ix->ctx->stream);
    if (e != cudaSuccess) {
        *st = cuda_fail(ix->ctx, e, "index build");
        return nullptr;
    }
    return p;
}

/* Steps 1-4: the points in index order (x, y, tid, key allocated first, as the host builder
 * uploads them), the cell boundaries d_cb[0..ncells] and, for the Grid, the runs' vector keys. */
struct Placement {
    int64_t* d_cb = nullptr;
    int64_t R = 0;               /* runs of equal cells, in trajectory order: */
    int32_t* starts = nullptr;   /*   first point */
    uint32_t* run_cell = nullptr; /*   cell */
    int32_t* run_tid = nullptr;  /*   trajectory */
};

int place(gat_index* ix, const DevicePlaceArgs& a, Temps& tmp, Placement& out) {
    gat_ctx* ctx = ix->ctx;
    const gat_db* db = ix->db;
    cudaStream_t s = ctx->stream;
    const int64_t P = db->npoints;
    const int n = db->n;
    if (P >= ((int64_t)1 << 31) - 1) return fail(ctx, GAT_ERR_ARG, std::string(a.what) + ": more than 2^31 - 2 points");
    const int64_t nhint = (P + (1 << kHintShift) - 1) >> kHintShift; /* blocks holding points */
    uint32_t* cells = tmp.get<uint32_t>(P);
    uint8_t* head = tmp.get<uint8_t>(P);
    int32_t* starts = tmp.get<int32_t>(P);
    int32_t* nsel = tmp.get<int32_t>(1);
    int32_t* hint = tmp.get<int32_t>(nhint);
    int64_t* d_cb = tmp.get<int64_t>((size_t)a.ncells + 1);
    if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
    CellParams cp{a.rxmin, a.rymax, a.cell, a.morton ? 1 : 0, a.axis, a.nx, a.ny, a.vparam};
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_flag, 0, sizeof(int32_t), s), "index build");
    int32_t R = 0;
    if (P > 0) {
        /* 1. cells and run heads */
        k_hints<<<grid_size(ctx, n), 256, 0, s>>>(n, db->d_off, hint);
        count_launch(ctx);
        timed_begin(ctx, GAT_KERNEL_INDEX_BUILD);
        k_point_cells<<<grid_size(ctx, (P + kPerThread - 1) / kPerThread), 256, 0, s>>>(P, db->d_xy, cp, cells, head,
                                                                                   ctx->d_flag);
        timed_end(ctx, GAT_KERNEL_INDEX_BUILD, (double)P * 13);
        k_run_starts<<<grid_size(ctx, n), 256, 0, s>>>(n, db->d_off, head);
        count_launch(ctx, 2);
        GAT_CUDA_TRY(ctx, cudaGetLastError(), "index build (cells)");
        if (check_device_flag(ctx, "index build") != GAT_OK)
            return fail(ctx, GAT_ERR_ARG, std::string(a.what) + ": a point lies outside the grid range");
        /* run starts, in position order */
        size_t need = 0;
        thrust::counting_iterator<int> iota(0);
        GAT_CUDA_TRY(ctx, cub::DeviceSelect::Flagged(nullptr, need, iota, head, starts, nsel, (int)P, s), "index build runs");
        void* t0 = tmp.get<char>(need);
        if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
        GAT_CUDA_TRY(ctx, cub::DeviceSelect::Flagged(t0, need, iota, head, starts, nsel, (int)P, s), "index build runs");
        count_launch(ctx, 2);
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(&R, nsel, 4, cudaMemcpyDeviceToHost, s), "index build runs");
        GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "index build runs");
        tmp.release(t0);
        tmp.release(head);
    }
    /* 3. index-order arrays */
    const int tid_bits = bits_to_hold(n);
    int pidx_bits = bits_to_hold(std::max(1, db->maxlen - 1));
    if (tid_bits + pidx_bits > 32) pidx_bits = -1; /* point-level results unavailable for this set */
    ix->pidx_bits = pidx_bits;
    ix->npoints = P;
    int st = GAT_OK;
    float* dx = alloc_padded<float>(ix, P, &st);
    float* dy = dx ? alloc_padded<float>(ix, P, &st) : nullptr;
    int32_t* dt = dy ? alloc_padded<int32_t>(ix, P, &st) : nullptr;
    uint32_t* dk = dt ? alloc_padded<uint32_t>(ix, P, &st) : nullptr;
    if (!dk) return st;
    ix->d_x = dx;
    ix->d_y = dy;
    ix->d_tid = dt;
    ix->d_key = dk;
    if (pidx_bits < 0) GAT_CUDA_TRY(ctx, cudaMalloc(&ix->d_pidx, std::max<size_t>((size_t)P, 1) * 4), "index build");
    out.R = R;
    if (R == 0) {
        GAT_CUDA_TRY(ctx, cudaMemsetAsync(d_cb, 0, ((size_t)a.ncells + 1) * 8, s), "index build");
        out.d_cb = d_cb;
        ix->host_pending = true;
        return GAT_OK;
    }
    /* 2. the runs, stably sorted by cell */
    uint32_t* run_cell = tmp.get<uint32_t>(R);
    uint32_t* run_cell_s = tmp.get<uint32_t>(R);
    int32_t* run_idx = tmp.get<int32_t>(R);
    int32_t* order = tmp.get<int32_t>(R);
    int32_t* run_tid = tmp.get<int32_t>(R);
    int32_t* run_len = tmp.get<int32_t>(R);
    int32_t* len_s = tmp.get<int32_t>(R + 1);
    int32_t* dest = tmp.get<int32_t>(R + 1);
    int4* rec = tmp.get<int4>(R);
    const int64_t ntiles = (P + kExpandTile - 1) / kExpandTile;
    int32_t* tfirst = tmp.get<int32_t>(ntiles);
    if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
    k_runs<<<grid_size(ctx, R), 256, 0, s>>>(R, P, n, starts, db->d_off, hint, nhint, cells, run_cell, run_idx, run_tid,
                                             run_len);
    count_launch(ctx);
    const int end_bit = bits_to_hold(a.ncells);
    size_t b1 = 0, b2 = 0;
    GAT_CUDA_TRY(ctx, cub::DeviceRadixSort::SortPairs(nullptr, b1, run_cell, run_cell_s, run_idx, order, R, 0, end_bit, s),
                 "index build sort");
    GAT_CUDA_TRY(ctx, cub::DeviceScan::ExclusiveSum(nullptr, b2, len_s, dest, R + 1, s), "index build scan");
    void* t1 = tmp.get<char>(std::max(b1, b2));
    if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
    GAT_CUDA_TRY(ctx, cub::DeviceRadixSort::SortPairs(t1, b1, run_cell, run_cell_s, run_idx, order, R, 0, end_bit, s),
                 "index build sort");
    k_sorted_runs<<<grid_size(ctx, R + 1), 256, 0, s>>>(R, order, starts, run_tid, run_len, db->d_off, rec, len_s);
    GAT_CUDA_TRY(ctx, cub::DeviceScan::ExclusiveSum(t1, b2, len_s, dest, R + 1, s), "index build scan");
    count_launch(ctx, 2 * ((end_bit + 7) / 8) + 4);
    /* 3. points to their index positions */
    timed_begin(ctx, GAT_KERNEL_INDEX_BUILD);
    k_tile_first<<<grid_size(ctx, ntiles), 256, 0, s>>>(ntiles, R, dest, tfirst);
    count_launch(ctx);
    k_expand_runs<<<(unsigned)ntiles, kExpandThreads, 0, s>>>(P, R, ntiles, tfirst, rec, dest, db->d_xy, dx, dy, dt, dk,
                                                              ix->d_pidx, pidx_bits);
    timed_end(ctx, GAT_KERNEL_INDEX_BUILD, (double)P * (24 + (pidx_bits < 0 ? 4 : 0)) + (double)R * 20);
    count_launch(ctx);
    /* 4. cell boundaries */
    k_cell_bounds<<<grid_size(ctx, a.ncells + 1), 256, 0, s>>>(R, a.ncells, run_cell_s, dest, d_cb);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "index build (placement)");
    ix->host_pending = true;
    out.d_cb = d_cb;
    out.starts = starts;
    out.run_cell = run_cell;
    out.run_tid = run_tid;
    return GAT_OK;
}

/* Step 5: quadtree node arrays (node_mbb, node_child, node_pbeg, node_pend) in breadth-first
 * order. */
int build_tree(gat_index* ix, const Placement& pl, const TreeParams& tp, Temps& tmp) {
    gat_ctx* ctx = ix->ctx;
    cudaStream_t s = ctx->stream;
    /* node ids and child links in queue order; grown as levels are added */
    int64_t cap = 1 << 16;
    int32_t* ids = tmp.get<int32_t>(cap);
    int32_t* child = tmp.get<int32_t>(cap);
    int32_t* flags = tmp.get<int32_t>(cap + 1);
    int32_t* spos = tmp.get<int32_t>(cap + 1);
    if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
    size_t scan_bytes = 0;
    void* scan_tmp = nullptr;
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(ids, 0, 4, s), "index build tree");
    LevelTable lt{};
    int64_t base = 0, m = 1, splits = 0;
    for (int level = 0;; level++) {
        if (level >= kMaxLevels) return fail(ctx, GAT_ERR_ARG, "gat_grid_build: quadtree deeper than supported");
        lt.base[level] = base;
        lt.nlevels = level + 1;
        k_tree_split<<<grid_size(ctx, m + 1), 256, 0, s>>>(m, level, ids + base, pl.d_cb, tp, flags);
        count_launch(ctx);
        size_t need = 0;
        GAT_CUDA_TRY(ctx, cub::DeviceScan::ExclusiveSum(nullptr, need, flags, spos, (int)(m + 1), s), "index build tree");
        if (need > scan_bytes) {
            if (scan_tmp) tmp.release(scan_tmp);
            scan_tmp = tmp.get<char>(need);
            if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
            scan_bytes = need;
        }
        GAT_CUDA_TRY(ctx, cub::DeviceScan::ExclusiveSum(scan_tmp, need, flags, spos, (int)(m + 1), s), "index build tree");
        count_launch(ctx);
        int32_t S = 0;
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(&S, spos + m, 4, cudaMemcpyDeviceToHost, s), "index build tree");
        GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "index build tree");
        const int64_t next = base + m + 4 * (int64_t)S;
        if (next > (int64_t)INT32_MAX) return fail(ctx, GAT_ERR_ARG, "gat_grid_build: quadtree larger than 2^31 nodes");
        if (next > cap || 4 * (int64_t)S + 1 > cap) {
            /* grow: room for the next level's nodes, and flags for a level of that size */
            int64_t ncap = cap;
            while (ncap < next || ncap < 4 * (int64_t)S + 1) ncap *= 2;
            int32_t* nids = tmp.get<int32_t>(ncap);
            int32_t* nchild = tmp.get<int32_t>(ncap);
            int32_t* nflags = tmp.get<int32_t>(ncap + 1);
            int32_t* nspos = tmp.get<int32_t>(ncap + 1);
            if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
            GAT_CUDA_TRY(ctx, cudaMemcpyAsync(nids, ids, (size_t)(base + m) * 4, cudaMemcpyDeviceToDevice, s), "index build tree");
            GAT_CUDA_TRY(ctx, cudaMemcpyAsync(nchild, child, (size_t)std::max<int64_t>(base, 1) * 4, cudaMemcpyDeviceToDevice, s),
                         "index build tree");
            GAT_CUDA_TRY(ctx, cudaMemcpyAsync(nflags, flags, (size_t)(m + 1) * 4, cudaMemcpyDeviceToDevice, s), "index build tree");
            GAT_CUDA_TRY(ctx, cudaMemcpyAsync(nspos, spos, (size_t)(m + 1) * 4, cudaMemcpyDeviceToDevice, s), "index build tree");
            GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "index build tree");
            tmp.release(ids);
            tmp.release(child);
            tmp.release(flags);
            tmp.release(spos);
            ids = nids;
            child = nchild;
            flags = nflags;
            spos = nspos;
            cap = ncap;
        }
        k_tree_children<<<grid_size(ctx, m), 256, 0, s>>>(m, ids + base, flags, spos, base + m, ids + base + m, child + base);
        count_launch(ctx);
        splits += S;
        base += m;
        m = 4 * (int64_t)S;
        if (m == 0) break;
    }
    const int64_t N = base;
    GridDev& g = ix->grid;
    g.nnodes = (int)N;
    ix->nodes = N;
    ix->leaves = N - splits;
    int st = GAT_OK;
    float4* nmbb = alloc_padded<float4>(ix, N, &st);
    int32_t* nchild = nmbb ? alloc_padded<int32_t>(ix, N, &st) : nullptr;
    int32_t* npbeg = nchild ? alloc_padded<int32_t>(ix, N, &st) : nullptr;
    int32_t* npend = npbeg ? alloc_padded<int32_t>(ix, N, &st) : nullptr;
    if (!npend) return st;
    g.node_mbb = nmbb;
    g.node_child = nchild;
    g.node_pbeg = npbeg;
    g.node_pend = npend;
    k_tree_nodes<<<grid_size(ctx, N), 256, 0, s>>>(N, lt, ids, child, pl.d_cb, tp, nmbb, nchild, npbeg, npend);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "index build tree");
    return GAT_OK;
}

/* Step 6: the frequency-vector CSR (fv_off [n+2], fv_cell, fv_cnt), allocated after the nodes:
 * cell runs merged into runs of equal virtual cells, keyed (trajectory, virtual cell), sorted, and
 * their point counts summed per key. */
int build_vectors(gat_index* ix, const Placement& pl, int vparam, Temps& tmp) {
    gat_ctx* ctx = ix->ctx;
    cudaStream_t s = ctx->stream;
    const int n = ix->db->n;
    const int64_t P = ix->db->npoints;
    const int64_t R = pl.R;
    int st = GAT_OK;
    int64_t* off = alloc_padded<int64_t>(ix, n + 2, &st);
    if (!off) return st;
    ix->d_fv_off = off;
    int32_t E = 0;
    unsigned long long* uk = nullptr;
    int32_t* sums = nullptr;
    if (R > 0) {
        uint8_t* vhead = tmp.get<uint8_t>(R);
        int32_t* vstarts = tmp.get<int32_t>(R);
        int32_t* nsel = tmp.get<int32_t>(1);
        if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
        k_vrun_heads<<<grid_size(ctx, R), 256, 0, s>>>(R, pl.run_cell, pl.run_tid, vparam, vhead);
        count_launch(ctx);
        size_t need = 0;
        thrust::counting_iterator<int> iota(0);
        GAT_CUDA_TRY(ctx, cub::DeviceSelect::Flagged(nullptr, need, iota, vhead, vstarts, nsel, (int)R, s), "index build fv");
        void* t0 = tmp.get<char>(need);
        if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
        GAT_CUDA_TRY(ctx, cub::DeviceSelect::Flagged(t0, need, iota, vhead, vstarts, nsel, (int)R, s), "index build fv");
        count_launch(ctx, 2);
        int32_t Rv = 0;
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(&Rv, nsel, 4, cudaMemcpyDeviceToHost, s), "index build fv");
        GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "index build fv");
        unsigned long long* key = tmp.get<unsigned long long>(Rv);
        int32_t* cnt = tmp.get<int32_t>(Rv);
        unsigned long long* key_s = tmp.get<unsigned long long>(Rv);
        int32_t* cnt_s = tmp.get<int32_t>(Rv);
        uk = tmp.get<unsigned long long>(Rv);
        sums = tmp.get<int32_t>(Rv);
        int32_t* nuniq = tmp.get<int32_t>(1);
        if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
        k_vruns<<<grid_size(ctx, Rv), 256, 0, s>>>(Rv, R, P, vstarts, pl.starts, pl.run_cell, pl.run_tid, vparam, key, cnt);
        count_launch(ctx);
        /* keys hold the trajectory above bit 32 and the virtual cell below it */
        const int kbits = 32 + bits_to_hold(n);
        size_t b1 = 0, b2 = 0;
        GAT_CUDA_TRY(ctx, cub::DeviceRadixSort::SortPairs(nullptr, b1, key, key_s, cnt, cnt_s, Rv, 0, kbits, s),
                     "index build fv");
        GAT_CUDA_TRY(ctx, cub::DeviceReduce::ReduceByKey(nullptr, b2, key_s, uk, cnt_s, sums, nuniq, AddInt(), Rv, s),
                     "index build fv");
        void* t2 = tmp.get<char>(std::max(b1, b2));
        if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
        GAT_CUDA_TRY(ctx, cub::DeviceRadixSort::SortPairs(t2, b1, key, key_s, cnt, cnt_s, Rv, 0, kbits, s), "index build fv");
        GAT_CUDA_TRY(ctx, cub::DeviceReduce::ReduceByKey(t2, b2, key_s, uk, cnt_s, sums, nuniq, AddInt(), Rv, s),
                     "index build fv");
        count_launch(ctx, 2 * ((kbits + 7) / 8) + 3);
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(&E, nuniq, 4, cudaMemcpyDeviceToHost, s), "index build fv");
        GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "index build fv");
    }
    int32_t* cell = alloc_padded<int32_t>(ix, E, &st);
    int32_t* cnt = cell ? alloc_padded<int32_t>(ix, E, &st) : nullptr;
    if (!cnt) return st;
    ix->d_fv_cell = cell;
    ix->d_fv_cnt = cnt;
    if (E > 0) {
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(cnt, sums, (size_t)E * 4, cudaMemcpyDeviceToDevice, s), "index build fv");
        k_fv_cells<<<grid_size(ctx, E), 256, 0, s>>>(E, uk, cell);
        count_launch(ctx);
    }
    /* off[t] = entries of trajectories below t: the first entry whose key is >= t << 32 */
    k_bounds<unsigned long long><<<grid_size(ctx, n + 2), 256, 0, s>>>(E, n + 1, uk, 32, off);
    count_launch(ctx);
    std::vector<int64_t> h((size_t)n + 2);
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), off, h.size() * 8, cudaMemcpyDeviceToHost, s), "index build fv");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "index build fv");
    int hmx = 0;
    for (int t = 0; t <= n; t++) hmx = std::max<int>(hmx, (int)(h[(size_t)t + 1] - h[(size_t)t]));
    ix->fv_max_nnz = hmx;
    ix->fv_entries = E;
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "index build fv");
    return GAT_OK;
}

}  // namespace

/* The context's pool for scratch slots and index-build temporaries: stream-ordered, and it keeps freed memory
 * (release threshold unbounded), so repeated builds do not map and unmap gigabytes each time;
 * gat_ctx_trim returns it. Null when the device has no memory pools. */
cudaMemPool_t build_pool(gat_ctx* ctx) {
    if (ctx->build_pool) return ctx->build_pool;
    int ok = 0;
    if (cudaDeviceGetAttribute(&ok, cudaDevAttrMemoryPoolsSupported, ctx->device) != cudaSuccess || !ok) return nullptr;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctx->device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    ctx->build_pool = pool;
    return pool;
}


int device_build_grid(gat_index* ix, const DevicePlaceArgs& a, int total_level, int leaf_cap) {
    gat_ctx* ctx = ix->ctx;
    Temps tmp(ctx);
    Placement pl;
    if (int st = place(ix, a, tmp, pl)) return st;
    TreeParams tp{a.rxmin, a.rymax, a.cell, total_level, leaf_cap};
    if (int st = build_tree(ix, pl, tp, tmp)) return st;
    if (int st = build_vectors(ix, pl, a.vparam, tmp)) return st;
    /* the temporaries are freed on return: wait for the work that reads them */
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "gat_grid_build");
    return GAT_OK;
}

int device_build_fsg(gat_index* ix, const DevicePlaceArgs& a) {
    gat_ctx* ctx = ix->ctx;
    Temps tmp(ctx);
    Placement pl;
    if (int st = place(ix, a, tmp, pl)) return st;
    int st = GAT_OK;
    int32_t* cbeg = alloc_padded<int32_t>(ix, a.ncells, &st);
    int32_t* cend = cbeg ? alloc_padded<int32_t>(ix, a.ncells, &st) : nullptr;
    if (!cend) return st;
    ix->fsg.cbeg = cbeg;
    ix->fsg.cend = cend;
    ix->leaves = a.ncells;
    k_fsg_cells<<<grid_size(ctx, a.ncells), 256, 0, ctx->stream>>>(a.ncells, pl.d_cb, cbeg, cend);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "gat_fsg_build");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "gat_fsg_build");
    return GAT_OK;
}

namespace {
__global__ void k_interleave(int64_t P, const float* __restrict__ lon, const float* __restrict__ lat, float2* xy) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < P; i += (int64_t)gridDim.x * blockDim.x)
        xy[i] = make_float2(lon[i], lat[i]);
}
}  // namespace

int upload_set_points(gat_ctx* ctx, const float* lon, const float* lat, int64_t P, float2* d_xy) {
    if (P == 0) return GAT_OK;
    Temps tmp(ctx);
    float* d_lon = tmp.get<float>(P);
    float* d_lat = tmp.get<float>(P);
    if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "gat_db_create");
    cudaStream_t s = ctx->stream;
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(d_lon, lon, (size_t)P * 4, cudaMemcpyHostToDevice, s), "gat_db_create");
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(d_lat, lat, (size_t)P * 4, cudaMemcpyHostToDevice, s), "gat_db_create");
    k_interleave<<<grid_size(ctx, P), 256, 0, s>>>(P, d_lon, d_lat, d_xy);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "gat_db_create");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "gat_db_create");
    return GAT_OK;
}

int db_host_copies(const gat_db* cdb) {
    gat_db* db = const_cast<gat_db*>(cdb);
    std::lock_guard<std::mutex> lk(db->host_mu);
    if (!db->host_pending) return GAT_OK;
    gat_ctx* ctx = db->ctx;
    const size_t P = (size_t)db->npoints;
    std::vector<float2> xy(P);
    cudaSetDevice(ctx->device);
    if (P > 0) GAT_CUDA_TRY(ctx, cudaMemcpy(xy.data(), db->d_xy, P * 8, cudaMemcpyDeviceToHost), "trajectory set host copy");
    std::vector<float> x(P), y(P);
    for (size_t i = 0; i < P; i++) {
        x[i] = xy[i].x;
        y[i] = xy[i].y;
    }
    db->h_x.swap(x);
    db->h_y.swap(y);
    db->host_pending = false;
    return GAT_OK;
}

int index_points_device(const gat_index* ix, float* x, float* y, int32_t* tid, int32_t* pidx) {
    gat_ctx* ctx = ix->ctx;
    const int64_t P = ix->npoints;
    if (P == 0) return GAT_OK;
    cudaSetDevice(ctx->device);
    const size_t b = (size_t)P * 4;
    if (x) GAT_CUDA_TRY(ctx, cudaMemcpy(x, ix->d_x, b, cudaMemcpyDeviceToHost), "index points");
    if (y) GAT_CUDA_TRY(ctx, cudaMemcpy(y, ix->d_y, b, cudaMemcpyDeviceToHost), "index points");
    if (tid) GAT_CUDA_TRY(ctx, cudaMemcpy(tid, ix->d_tid, b, cudaMemcpyDeviceToHost), "index points");
    if (pidx && ix->pidx_bits >= 0) {
        /* the point index is the key's low pidx_bits bits */
        GAT_CUDA_TRY(ctx, cudaMemcpy(pidx, ix->d_key, b, cudaMemcpyDeviceToHost), "index points");
        const uint32_t mask = (uint32_t)((1ull << ix->pidx_bits) - 1);
        for (int64_t i = 0; i < P; i++) pidx[i] = (int32_t)((uint32_t)pidx[i] & mask);
    } else if (pidx) {
        GAT_CUDA_TRY(ctx, cudaMemcpy(pidx, ix->d_pidx, b, cudaMemcpyDeviceToHost), "index points");
    }
    return GAT_OK;
}

int index_host_copies(gat_index* ix) {
    std::lock_guard<std::mutex> lk(ix->host_mu);
    if (!ix->host_pending) return GAT_OK;
    const size_t P = (size_t)ix->npoints;
    std::vector<float> x(P), y(P);
    std::vector<int32_t> tid(P), pidx(P);
    if (int st = index_points_device(ix, x.data(), y.data(), tid.data(), pidx.data())) return st;
    ix->h_x.swap(x);
    ix->h_y.swap(y);
    ix->h_tid.swap(tid);
    ix->h_pidx.swap(pidx);
    ix->host_pending = false;
    return GAT_OK;
}

}  // namespace gat
