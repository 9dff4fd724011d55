/* Range queries over the Grid (GT-quadtree), STIG and FSG indexes.
 *
 * Pipeline for a batch of queries (all launches on the context stream):
 *   1. candidates  64 threads per query walk the index, each its own subtree (Grid: quadtree
 *                  with BoxIntersect, Grid.cpp:428-446; STIG: median slabs + leaf MBBs,
 *                  STIG.cpp:179-252; FSG: the rows of the candidate cell rectangle,
 *                  FSG.cpp:183-262) and emit point ranges, contiguous ranges joined and cut into
 *                  chunks of at most 1024 points; a count pass and a scan give each thread its
 *                  item slice.
 *   2. scan        id sets: persistent CTAs take queries from a counter; each warp scans one
 *                  chunk at a time with 128-bit loads of x / y / tid and the inclusive
 *                  MBB::pInBox (MBB.cpp:21-26), inserting the trajectory id of each run of hits
 *                  into a shared-memory hash set, which is then sorted and written (the
 *                  reference's per-query vector<bool>, Grid.cpp:384-387, as a sorted id list);
 *                  queries with more distinct ids than the set holds use a bitmap over all
 *                  trajectory ids instead. Point lists: one CTA per query compacts hit keys with
 *                  warp ballots and prefix sums, sorts them with a stable in-CTA radix sort and
 *                  de-duplicates.
 *   3. offsets     scan of per-query result counts; one CTA per query copies its segment.
 * Plain execution runs the same pipeline once per query.
 */
#include <algorithm>
#include <climits>

#include "cells.cuh"
#include "internal.h"
#include "launch.cuh"

namespace gat {
namespace {

constexpr int kThreads = 256;
constexpr int kStack = 96;
constexpr int kChunk = 1024;       /* candidate points per scan item */
constexpr int kChunkAllHit = 4096; /* points per item whose every point is a hit (ids only) */
constexpr int kAllHit = (int)0x80000000; /* item start flag: every point of the item is a hit */

struct Box {
    float xmin, ymin, xmax, ymax;
};

__device__ __forceinline__ bool in_box(const Box& q, float x, float y) {
    /* MBB::pInBox (MBB.cpp:21-26) */
    return x <= q.xmax && x >= q.xmin && y <= q.ymax && y >= q.ymin;
}

/* BoxIntersect (MBB.cpp:28-73) reduced to its zero / non-zero outcome, the only use the
 * traversals make of it. */
__device__ __forceinline__ bool box_intersect(const Box& a1, const Box& b1) {
    Box a, b;
    if (a1.xmin < b1.xmin) {
        a = a1;
        b = b1;
    } else if (a1.xmin == b1.xmin) {
        if (a1.xmax > b1.xmax) {
            a = a1;
            b = b1;
        } else {
            b = a1;
            a = b1;
        }
    } else {
        b = a1;
        a = b1;
    }
    if (b.xmin >= a.xmax) return false;
    if (b.ymax <= a.ymin) return false;
    if (b.ymin >= a.ymax) return false;
    return true;
}

__device__ __forceinline__ Box load_box(const gat_mbb* q, int i) {
    gat_mbb m = q[i];
    return Box{m.xmin, m.ymin, m.xmax, m.ymax};
}

__device__ __forceinline__ void set_flag(int32_t* flag, int code) { atomicCAS(flag, 0, code); }

/* ---------------------------------------------------------------- candidates */
/* Whole subtrees. Quadtree node boxes (the Grid's and the MortonGrid's) are made from the first
 * and last cell of the node by float expressions that are monotone in the cell's column and row
 * (Grid.cpp:121), so every descendant's box lies within its ancestor's. When a node's box lies
 * strictly inside the query, BoxIntersect is therefore non-zero for every descendant, the
 * traversal takes every leaf below it, and those leaves' point ranges tile the node's own range
 * [pbeg, pend) in visiting order (children in Morton order). The walks emit such a node as that
 * one range: the range joiner of walk_ranges turns the leaves' ranges into exactly the same
 * joined range, so the items are unchanged and the walk visits only the nodes that straddle the
 * query's border. */
__device__ __forceinline__ bool box_inside(const Box& q, const float4& m) {
    return q.xmin < m.x && m.z < q.xmax && q.ymin < m.y && m.w < q.ymax;
}

/* All points hit. A range the walk takes (a leaf, or a whole subtree as above) whose exact point
 * box (pbox.cu) lies inside the query under MBB::pInBox's inclusive comparisons has every point
 * in the query: the scan takes its ids without testing coordinates. False without point boxes. */
__device__ __forceinline__ bool points_inside(const Box& q, const float4* pbox, int nd) {
    if (!pbox) return false;
    const float4 b = pbox[nd];
    return b.x >= q.xmin && b.z <= q.xmax && b.y >= q.ymin && b.w <= q.ymax;
}

/* emit(pbeg, pend, all_hit) for each candidate leaf (or whole subtree, above); returns false on
 * stack overflow. Stack entries are node indices, complemented for a subtree inside the query. */
template <class Emit>
__device__ bool grid_walk(const GridDev& g, const Box& q, Emit emit, int start = 0) {
    int stack[kStack];
    int sp = 0;
    stack[sp++] = start;
    while (sp > 0) {
        const int e = stack[--sp];
        if (e < 0) {
            emit(g.node_pbeg[~e], g.node_pend[~e], points_inside(q, g.node_pbox, ~e));
            continue;
        }
        const int ch = g.node_child[e];
        if (ch < 0) {
            /* leaves are taken without a test (Grid.cpp:430-433) */
            emit(g.node_pbeg[e], g.node_pend[e], points_inside(q, g.node_pbox, e));
            continue;
        }
        /* push in reverse so children are visited UL, UR, DL, DR (Grid.cpp:436-443) */
        for (int c = 3; c >= 0; c--) {
            const float4 m = g.node_mbb[ch + c];
            if (box_intersect(q, Box{m.x, m.y, m.z, m.w})) {
                if (sp >= kStack) return false;
                stack[sp++] = box_inside(q, m) ? ~(ch + c) : ch + c;
            }
        }
    }
    return true;
}

template <class Emit>
__device__ bool stig_walk(const StigDev& s, const Box& q, Emit emit, int start = 0) {
    int stack[kStack];
    int sp = 0;
    stack[sp++] = start;
    while (sp > 0) {
        int nd = stack[--sp];
        if (s.kind[nd]) {
            /* STIG::searchNode(LeafNode*) (STIG.cpp:241-252): leaf MBB against the query */
            float4 m = s.mbb[nd];
            if (box_intersect(Box{m.x, m.y, m.z, m.w}, q)) emit(s.lo[nd], s.hi[nd] + 1, points_inside(q, s.pbox, nd));
            continue;
        }
        /* STIG::searchNode(InternalNode*) (STIG.cpp:201-239) with intersectBlock (:340-347) */
        float lo = s.dim[nd] == 0 ? q.xmin : q.ymin;
        float hi = s.dim[nd] == 0 ? q.xmax : q.ymax;
        float med = s.median[nd];
        bool go_left = !(hi < 0.0f) && !(lo > med);
        bool go_right = !(hi < med) && !(lo > 180.0f);
        if (sp + 2 > kStack) return false;
        if (go_right) stack[sp++] = s.right[nd];
        if (go_left) stack[sp++] = s.left[nd];
    }
    return true;
}

template <class Emit>
__device__ void fsg_walk(const FsgDev& f, const Box& q, Emit emit, int first = 0, int step = 1) {
    /* FSG::rangeQueryBatchGPU (FSG.cpp:183-262): the border ring plus the interior cover the
     * cells (row, col) for rows g3..g4 and cols g1..g2, addressed row * nx + col without
     * clamping. Row r is one contiguous run of cell ids; ids outside the grid are skipped (the
     * reference reads out of bounds there and no point lies in such a cell). */
    int g1 = (int)__fdiv_rn(__fsub_rn(q.xmin, f.rxmin), f.cell);
    int g2 = (int)__fdiv_rn(__fsub_rn(q.xmax, f.rxmin), f.cell);
    int g3 = (int)__fdiv_rn(__fsub_rn(f.rymax, q.ymax), f.cell);
    int g4 = (int)__fdiv_rn(__fsub_rn(f.rymax, q.ymin), f.cell);
    for (long long r = (long long)g3 + first; r <= g4; r += step) {
        long long lo = (long long)g1 + (long long)r * f.nx;
        long long hi = (long long)g2 + (long long)r * f.nx;
        if (lo < 0) lo = 0;
        if (hi > f.cellnum - 1) hi = f.cellnum - 1;
        if (lo > hi) continue;
        int b = f.cbeg[lo], e = f.cend[hi];
        if (b < e) emit(b, e, false);
    }
}

/* MortonGrid implicit nodes: the leaf bit of (level, id) (findIdxInBitmap, MortonGrid.cpp:8-13),
 * the node's box from its first and last Morton cells (generateMBBfromNode,
 * MortonGrid.cpp:261-265) and its point range. */
__device__ __forceinline__ bool morton_leaf(const MortonDev& m, int level, uint32_t id) {
    const uint64_t idx = (((uint64_t)1 << (2 * level)) - 1) / 3 + id;
    return (__ldg(m.leaf + (idx >> 5)) >> (idx & 31)) & 1u;
}
__device__ __forceinline__ Box morton_box(const MortonDev& m, int level, uint32_t id) {
    const uint32_t span = 1u << (2 * (m.total_level - level));
    const float4 a = morton_cell_box(m.rxmin, m.rymax, m.cell, (int)(id * span));
    const float4 b = morton_cell_box(m.rxmin, m.rymax, m.cell, (int)(id * span + span - 1));
    return Box{a.x, b.y, b.z, a.w};
}
template <class Emit>
__device__ __forceinline__ void morton_emit(const MortonDev& m, int level, uint32_t id, Emit emit) {
    const uint32_t span = 1u << (2 * (m.total_level - level));
    emit(__ldg(m.cbeg + id * span), __ldg(m.cbeg + id * span + span), false);
}

/* MortonGrid::findMatchNodeInQuadTree (MortonGrid.cpp:356-393): leaves are taken without a
 * test, children in the order UL, UR, DL, DR when BoxIntersect(query, child box) is non-zero.
 * Stack entries pack (id << 4) | level (level <= 13, id < 2^26); bit 31 marks a subtree inside
 * the query, emitted whole (box_inside). */
template <class Emit>
__device__ bool morton_walk(const MortonDev& m, const Box& q, Emit emit, int level0, uint32_t id0) {
    constexpr uint32_t kWhole = 0x80000000u;
    uint32_t stack[kStack];
    int sp = 0;
    stack[sp++] = (id0 << 4) | (uint32_t)level0;
    while (sp > 0) {
        const uint32_t e = stack[--sp];
        const int level = (int)(e & 15u);
        const uint32_t id = (e & ~kWhole) >> 4;
        if ((e & kWhole) || morton_leaf(m, level, id)) {
            morton_emit(m, level, id, emit);
            continue;
        }
        for (int c = 3; c >= 0; c--) {
            const uint32_t cid = (id << 2) + (uint32_t)c;
            const Box b = morton_box(m, level + 1, cid);
            if (box_intersect(q, b)) {
                if (sp >= kStack) return false;
                const bool whole = box_inside(q, make_float4(b.xmin, b.ymin, b.xmax, b.ymax));
                stack[sp++] = (cid << 4) | (uint32_t)(level + 1) | (whole ? kWhole : 0u);
            }
        }
    }
    return true;
}

/* kSub threads per query: thread `sub` takes the path given by its digits (base 4 over
 * kGridDepth quadtree levels, base 2 over kStigDepth STIG levels), with the traversal's own
 * intersection tests, and walks the subtree it reaches; a leaf met on the way belongs to the
 * thread whose remaining digits are all zero. FSG rows are dealt round robin. Concatenated in
 * thread order the items are the sequential traversal's, cut at subtree boundaries. */
constexpr int kGridDepth = 3, kSub = 64;
/* plain execution walks one query with 1024 threads: the split goes two levels deeper */
constexpr int kPlainDepth = 5, kPlainSub = 1024;

/* The candidate ranges of sub-thread `sub` of a query, joined and cut into items. Writes them
 * to items[0..] when items is non-NULL; returns how many there are. Sets GAT_ERR_ARG in flag when
 * a walk's stack overflows. */
template <int KIND, int GD, class Sink>
__device__ int64_t walk_ranges(const GridDev& g, const StigDev& s, const FsgDev& f, const MortonDev& m, const Box& q,
                               int sub, Sink sink, int32_t* flag) {
    constexpr int SD = 2 * GD, NSUB = 1 << (2 * GD); /* STIG levels and threads of the split */
    int64_t cnt = 0;
    /* Ranges that continue the previous one (neighbouring leaves / cells are contiguous in the
     * index's point order) are joined, and everything is cut into chunks of at most kChunk
     * points ending on multiples of 4, so the warps of the scan get balanced, 16-byte-aligned
     * pieces. Chunking only regroups the same points. */
    /* Ranges whose every point is a hit (points_inside) are joined only with each other and
     * flagged in bit 31 of the item's start (kAllHit); their chunks are longer, since the scan
     * reads only their ids. */
    int cur_b = -1, cur_e = -1;
    bool cur_all = false;
    auto flush = [&]() {
        const int chunk = cur_all ? kChunkAllHit : kChunk;
        while (cur_b < cur_e) {
            int e = cur_e;
            if (e - cur_b > chunk) e = (cur_b + chunk) & ~3;
            sink(cnt, make_int2(cur_b | (cur_all ? kAllHit : 0), e));
            cnt++;
            cur_b = e;
        }
    };
    auto emit = [&](int b, int e, bool all) {
        if (b >= e) return;
        if (b == cur_e && all == cur_all) {
            cur_e = e;
            return;
        }
        flush();
        cur_b = b;
        cur_e = e;
        cur_all = all;
    };
    bool ok = true;
    if (KIND == GAT_INDEX_GRID) {
        int nd = 0; /* the root is taken without a test (Grid.cpp:428-446) */
        bool walk = true;
        for (int lev = 0; lev < GD && walk; lev++) {
            const int ch = g.node_child[nd];
            if (ch < 0) {
                if ((sub & ((1 << (2 * (GD - lev))) - 1)) == 0)
                    emit(g.node_pbeg[nd], g.node_pend[nd], points_inside(q, g.node_pbox, nd));
                walk = false;
                break;
            }
            const int c = ch + ((sub >> (2 * (GD - 1 - lev))) & 3);
            const float4 m = g.node_mbb[c];
            if (!box_intersect(q, Box{m.x, m.y, m.z, m.w})) walk = false;
            nd = c;
        }
        if (walk) ok = grid_walk(g, q, emit, nd);
    }
    if (KIND == GAT_INDEX_STIG) {
        int nd = 0;
        bool walk = true;
        for (int lev = 0; lev < SD && walk; lev++) {
            if (s.kind[nd]) {
                if ((sub & ((1 << (SD - lev)) - 1)) == 0) {
                    const float4 m = s.mbb[nd];
                    if (box_intersect(Box{m.x, m.y, m.z, m.w}, q)) emit(s.lo[nd], s.hi[nd] + 1, points_inside(q, s.pbox, nd));
                }
                walk = false;
                break;
            }
            const float lo = s.dim[nd] == 0 ? q.xmin : q.ymin;
            const float hi = s.dim[nd] == 0 ? q.xmax : q.ymax;
            const float med = s.median[nd];
            const bool right = (sub >> (SD - 1 - lev)) & 1;
            const bool go = right ? (!(hi < med) && !(lo > 180.0f)) : (!(hi < 0.0f) && !(lo > med));
            if (!go) walk = false;
            nd = right ? s.right[nd] : s.left[nd];
        }
        if (walk) ok = stig_walk(s, q, emit, nd);
    }
    if (KIND == GAT_INDEX_FSG) fsg_walk(f, q, emit, sub, NSUB);
    if (KIND == GAT_INDEX_MORTON) {
        int level = 0; /* the Grid's digit split over the implicit nodes */
        uint32_t id = 0;
        bool walk = true;
        for (int lev = 0; lev < GD && walk; lev++) {
            if (morton_leaf(m, level, id)) {
                if ((sub & ((1 << (2 * (GD - lev))) - 1)) == 0) morton_emit(m, level, id, emit);
                walk = false;
                break;
            }
            const uint32_t cid = (id << 2) + (uint32_t)((sub >> (2 * (GD - 1 - lev))) & 3);
            if (!box_intersect(q, morton_box(m, level + 1, cid))) walk = false;
            level++;
            id = cid;
        }
        if (walk) ok = morton_walk(m, q, emit, level, id);
    }
    flush();
    if (!ok) set_flag(flag, GAT_ERR_ARG);
    return cnt;
}

/* walk_ranges writing the items to items[0..] (nothing when items is NULL) */
template <int KIND, int GD = kGridDepth>
__device__ int64_t walk_items(const GridDev& g, const StigDev& s, const FsgDev& f, const MortonDev& m, const Box& q,
                              int sub, int2* items, int32_t* flag) {
    return walk_ranges<KIND, GD>(
        g, s, f, m, q, sub,
        [items](int64_t c, int2 v) {
            if (items) items[c] = v;
        },
        flag);
}

/* items of queries 0..nq-1, or of the nq queries listed in qlist (offsets by list position) */
template <int KIND>
__global__ void k_items(GridDev g, StigDev s, FsgDev f, MortonDev m, const gat_mbb* queries, int nq, const int* qlist,
                        const int64_t* ioff, int64_t* icnt, int2* items, int32_t* flag) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (int64_t)nq * kSub) return;
    const int qi = qlist ? qlist[tid / kSub] : (int)(tid / kSub), sub = (int)(tid % kSub);
    const Box q = load_box(queries, qi);
    const int64_t cnt = walk_items<KIND>(g, s, f, m, q, sub, ioff ? items + ioff[tid] : nullptr, flag);
    if (!ioff) icnt[tid] = cnt;
}

/* ---------------------------------------------------------------- candidate items by tasks */
/* The walk of a query's 64 sub-threads is lopsided: a box meets few of the subtrees its digits
 * select, so in a warp of one query's sub-threads a handful of lanes do all the walking (2.2 of
 * 32 lanes active on average in a 300k-walk profile). The items are therefore built from a task
 * list: a first pass keeps the (query, sub-thread) pairs whose digit path reaches a subtree or
 * leaf to walk, and the walks run over the compacted list, so a warp's lanes all walk. Tasks
 * stay in (query, sub-thread) order, so every query's items stay contiguous and in the
 * traversal's order. */

/* whether the digits of `sub` reach a subtree (or a leaf this sub-thread emits) */
template <int KIND>
__device__ bool has_walk(const GridDev& g, const StigDev& s, const MortonDev& m, const Box& q, int sub) {
    constexpr int GD = kGridDepth, SD = 2 * kGridDepth;
    if (KIND == GAT_INDEX_GRID) {
        int nd = 0;
        for (int lev = 0; lev < GD; lev++) {
            const int ch = g.node_child[nd];
            if (ch < 0) return (sub & ((1 << (2 * (GD - lev))) - 1)) == 0;
            const int c = ch + ((sub >> (2 * (GD - 1 - lev))) & 3);
            const float4 b = g.node_mbb[c];
            if (!box_intersect(q, Box{b.x, b.y, b.z, b.w})) return false;
            nd = c;
        }
        return true;
    }
    if (KIND == GAT_INDEX_MORTON) {
        int level = 0;
        uint32_t id = 0;
        for (int lev = 0; lev < GD; lev++) {
            if (morton_leaf(m, level, id)) return (sub & ((1 << (2 * (GD - lev))) - 1)) == 0;
            const uint32_t cid = (id << 2) + (uint32_t)((sub >> (2 * (GD - 1 - lev))) & 3);
            if (!box_intersect(q, morton_box(m, level + 1, cid))) return false;
            level++;
            id = cid;
        }
        return true;
    }
    /* STIG */
    int nd = 0;
    for (int lev = 0; lev < SD; lev++) {
        if (s.kind[nd]) return (sub & ((1 << (SD - lev)) - 1)) == 0;
        const float lo = s.dim[nd] == 0 ? q.xmin : q.ymin;
        const float hi = s.dim[nd] == 0 ? q.xmax : q.ymax;
        const float med = s.median[nd];
        const bool right = (sub >> (SD - 1 - lev)) & 1;
        const bool go = right ? (!(hi < med) && !(lo > 180.0f)) : (!(hi < 0.0f) && !(lo > med));
        if (!go) return false;
        nd = right ? s.right[nd] : s.left[nd];
    }
    return true;
}

template <int KIND>
__global__ void k_task_flags(GridDev g, StigDev s, MortonDev m, const gat_mbb* queries, int nq, int64_t* flags) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (int64_t)nq * kSub) return;
    flags[tid] = has_walk<KIND>(g, s, m, load_box(queries, (int)(tid / kSub)), (int)(tid % kSub)) ? 1 : 0;
}

/* tasks[tpos[t]] = t for every flagged (query, sub-thread) t */
__global__ void k_task_list(int64_t nsub, const int64_t* __restrict__ flags, const int64_t* __restrict__ tpos,
                            int32_t* tasks) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nsub; t += (int64_t)gridDim.x * blockDim.x)
        if (flags[t]) tasks[tpos[t]] = (int32_t)t;
}

/* the walks of the tasks: counts (toff NULL) or items at toff[task] */
template <int KIND>
__global__ void k_task_walk(GridDev g, StigDev s, FsgDev f, MortonDev m, const gat_mbb* queries,
                            const int32_t* __restrict__ tasks, const int64_t* ntasks, const int64_t* toff,
                            int64_t* tcnt, int2* items, int32_t* flag) {
    const int64_t n = *ntasks;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int t = tasks[i];
        const Box q = load_box(queries, t / kSub);
        const int64_t c = walk_items<KIND>(g, s, f, m, q, t % kSub, toff ? items + toff[i] : nullptr, flag);
        if (!toff) tcnt[i] = c;
    }
}

/* every query's first item: ioff[qi * kSub] = toff[first task of qi] (the only entries the scan
 * kernels read) */
__global__ void k_task_qoff(int nq, const int64_t* __restrict__ tpos, const int64_t* __restrict__ toff, int64_t* ioff) {
    for (int qi = blockIdx.x * blockDim.x + threadIdx.x; qi <= nq; qi += gridDim.x * blockDim.x)
        ioff[(int64_t)qi * kSub] = toff[tpos[(int64_t)qi * kSub]];
}

/* Plain execution (one query per launch sequence of three kernels, nothing waiting on the host
 * in between), step 1: one CTA of kPlainSub threads walks query qi, each thread the subtree its
 * digits select (two levels deeper than the batched split, so every thread's walk is short),
 * counts its items, and after a block scan writes them at their offsets. ioff[0] receives the
 * query's item count. item_cap bounds the items of any single query; a query beyond it
 * (impossible with the bound the host computes) raises GAT_ERR_ARG and scans nothing. */
template <int KIND>
__global__ void __launch_bounds__(kPlainSub) k_plain_items(GridDev g, StigDev s, FsgDev f, MortonDev m,
                                                           const gat_mbb* queries, int qi, int64_t* ioff, int2* items,
                                                           int64_t item_cap, int32_t* flag) {
    dep_wait();
    __shared__ int64_t wsum[kPlainSub / 32 + 1];
    const Box q = load_box(queries, qi);
    const int sub = threadIdx.x, lane = sub & 31, warp = sub >> 5;
    const int64_t c = walk_items<KIND, kPlainDepth>(g, s, f, m, q, sub, nullptr, flag);
    int64_t x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (sub == 0) {
        int64_t run = 0;
        for (int w = 0; w < kPlainSub / 32; w++) {
            const int64_t t = wsum[w];
            wsum[w] = run;
            run += t;
        }
        wsum[kPlainSub / 32] = run;
    }
    __syncthreads();
    const int64_t total = wsum[kPlainSub / 32];
    const bool fits = total <= item_cap;
    if (sub == 0) {
        ioff[0] = fits ? total : 0;
        if (!fits) set_flag(flag, GAT_ERR_ARG);
    }
    if (fits) walk_items<KIND, kPlainDepth>(g, s, f, m, q, sub, items + wsum[warp] + x - c, flag);
}

/* Plain execution, step 2: warps of the whole grid take the query's items (ioff[0] of them) and
 * mark the trajectory id of every run of hits (MBB::pInBox, MBB.cpp:21-26) in a bitmap over the
 * set's ids, with 128-bit loads of x / y / tid. work (optional) accumulates algorithmic bytes. */
__global__ void __launch_bounds__(kThreads) k_plain_scan(const gat_mbb* queries, int qi, const int64_t* __restrict__ ioff,
                                                         const int2* __restrict__ items, const float* __restrict__ X,
                                                         const float* __restrict__ Y, const int32_t* __restrict__ tid,
                                                         uint32_t* bitmap, unsigned long long* work) {
    dep_wait();
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t nitems = ioff[0];
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const Box q = load_box(queries, qi);
    unsigned long long cand = 0, hits = 0;
    auto mark = [&](int t) { atomicOr(bitmap + (t >> 5), 1u << (t & 31)); };
    for (int64_t it = gw; it < nitems; it += nw) {
        int2 r = items[it];
        r.x &= ~kAllHit; /* every point is tested here, all-hit items included */
        if (lane == 0) cand += (unsigned long long)(r.y - r.x);
        const int head_end = min(r.y, (r.x + 3) & ~3);
        const int vb = head_end, ve = head_end + ((r.y - head_end) & ~3);
        for (int i = r.x + lane; i < head_end; i += 32)
            if (in_box(q, __ldg(X + i), __ldg(Y + i))) {
                mark(__ldg(tid + i));
                hits++;
            }
        for (int i = ve + lane; i < r.y; i += 32)
            if (in_box(q, __ldg(X + i), __ldg(Y + i))) {
                mark(__ldg(tid + i));
                hits++;
            }
        const float4* X4 = reinterpret_cast<const float4*>(X + vb);
        const float4* Y4 = reinterpret_cast<const float4*>(Y + vb);
        const int4* T4 = reinterpret_cast<const int4*>(tid + vb);
        const int nv = (ve - vb) >> 2;
        int carry = -1;
        for (int k0 = 0; k0 < nv; k0 += 32) {
            const int k = k0 + lane;
            int t0 = -1, t1 = -1, t2 = -1, t3 = -1;
            if (k < nv) {
                const float4 x = __ldg(X4 + k), y = __ldg(Y4 + k);
                const bool h0 = in_box(q, x.x, y.x), h1 = in_box(q, x.y, y.y);
                const bool h2 = in_box(q, x.z, y.z), h3 = in_box(q, x.w, y.w);
                if (h0 | h1 | h2 | h3) {
                    const int4 tt = __ldg(T4 + k);
                    t0 = h0 ? tt.x : -1;
                    t1 = h1 ? tt.y : -1;
                    t2 = h2 ? tt.z : -1;
                    t3 = h3 ? tt.w : -1;
                    hits += (unsigned long long)(h0 + h1 + h2 + h3);
                }
            }
            /* one mark per run of hits of one trajectory */
            int prev = __shfl_up_sync(FULL, t3, 1);
            if (lane == 0) prev = carry;
            carry = __shfl_sync(FULL, t3, 31);
            if (t0 >= 0 && t0 != prev) mark(t0);
            if (t1 >= 0 && t1 != t0) mark(t1);
            if (t2 >= 0 && t2 != t1) mark(t2);
            if (t3 >= 0 && t3 != t2) mark(t3);
        }
    }
    if (work) {
        unsigned long long w = 8ull * cand + 4ull * hits;
        for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(FULL, w, o);
        if (lane == 0 && w) atomicAdd(work, w);
    }
}

/* Plain execution, step 3 (one CTA of kPlainSub threads): the bitmap's ids in ascending order
 * go to out_tid[off[qi]..] and off[qi + 1] = off[qi] + count; the words are cleared for the next
 * query. When the ids do not fit `capacity`, nothing is written and trunc[0] is set; the offsets
 * keep counting. */
__global__ void __launch_bounds__(kPlainSub) k_plain_emit(int qi, uint32_t* bitmap, int words, int64_t* off,
                                                          int32_t* out_tid, int64_t capacity, int32_t* trunc) {
    dep_wait();
    __shared__ int wsum[kPlainSub / 32 + 1];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int per = (words + kPlainSub - 1) / kPlainSub;
    const int w0 = min(words, t * per), w1 = min(words, w0 + per);
    int c = 0;
    for (int w = w0; w < w1; w++) c += __popc(bitmap[w]);
    int x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (t == 0) {
        int run = 0;
        for (int w = 0; w < kPlainSub / 32; w++) {
            const int v = wsum[w];
            wsum[w] = run;
            run += v;
        }
        wsum[kPlainSub / 32] = run;
    }
    __syncthreads();
    const int64_t base = qi == 0 ? 0 : off[qi];
    const int64_t total = wsum[kPlainSub / 32];
    __syncthreads(); /* every thread has read off[qi] before it is rewritten below (qi == 0) */
    if (t == 0) {
        if (qi == 0) off[0] = 0;
        off[qi + 1] = base + total;
        if (base + total > capacity) *trunc = 1;
    }
    const bool write = base + total <= capacity;
    int64_t o = base + wsum[warp] + x - c;
    for (int w = w0; w < w1; w++) {
        uint32_t v = bitmap[w];
        if (!v) continue;
        bitmap[w] = 0u;
        if (!write) continue;
        while (v) {
            const int b = __ffs(v) - 1;
            v &= v - 1;
            out_tid[o++] = w * 32 + b;
        }
    }
}

/* ---------------------------------------------------------------- block helpers */
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

/* exclusive block scan of one int per thread; kThreads threads */
__device__ int block_scan_excl(int v, int* total, int* sh /* kThreads/32 + 1 */) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int w = 0; w < kThreads / 32; w++) {
            int t = sh[w];
            sh[w] = run;
            run += t;
        }
        sh[kThreads / 32] = run;
    }
    __syncthreads();
    int r = sh[warp] + x - v;
    *total = sh[kThreads / 32];
    __syncthreads();
    return r;
}

/* Tests the points [b, e) against q, calling hit(i) for every point inside. The aligned body
 * is read as float4 pairs (four x and four y per thread per step). */
template <class Hit>
__device__ __forceinline__ void scan_range(const float* __restrict__ X, const float* __restrict__ Y, int b, int e,
                                           const Box& q, Hit hit) {
    int head_end = min(e, (b + 3) & ~3);
    for (int i = b + (int)threadIdx.x; i < head_end; i += blockDim.x)
        if (in_box(q, __ldg(X + i), __ldg(Y + i))) hit(i);
    int vb = head_end, ve = head_end + ((e - head_end) & ~3);
    const float4* X4 = reinterpret_cast<const float4*>(X + vb);
    const float4* Y4 = reinterpret_cast<const float4*>(Y + vb);
    int nv = (ve - vb) >> 2;
    for (int k = threadIdx.x; k < nv; k += blockDim.x) {
        float4 x = __ldg(X4 + k), y = __ldg(Y4 + k);
        int i = vb + 4 * k;
        if (in_box(q, x.x, y.x)) hit(i);
        if (in_box(q, x.y, y.y)) hit(i + 1);
        if (in_box(q, x.z, y.z)) hit(i + 2);
        if (in_box(q, x.w, y.w)) hit(i + 3);
    }
    for (int i = ve + (int)threadIdx.x; i < e; i += blockDim.x)
        if (in_box(q, __ldg(X + i), __ldg(Y + i))) hit(i);
}

/* ---------------------------------------------------------------- id sets, bitmap form */
/* One CTA per query (grid-stride over the queries, or over qlist): a bitmap of n+1 trajectory
 * bits in shared memory (or in a per-CTA global slice when it does not fit), set by every
 * candidate hit, then emitted in ascending id order into the arena. Exact for any result
 * size; its fixed cost is proportional to n, so it serves the queries the hash form below
 * cannot hold. */
__global__ void __launch_bounds__(kThreads) k_range_ids(const gat_mbb* queries, int nq, const int64_t* ioff,
                                                        const int2* items, const float* X, const float* Y,
                                                        const int32_t* tid, int words, uint32_t* gbitmap,
                                                        uint32_t* arena, int64_t cap, unsigned long long* cursor,
                                                        int64_t* segbase, int64_t* segcnt, unsigned long long* work,
                                                        const int* qlist, int ioff_by_pos) {
    dep_wait();
    extern __shared__ uint32_t smem_bm[];
    __shared__ int sh[kThreads / 32 + 1];
    __shared__ unsigned long long base_sh;
    uint32_t* bm = gbitmap ? gbitmap + (size_t)blockIdx.x * words : smem_bm;
    int per = (words + kThreads - 1) / kThreads;
    unsigned long long my_work = 0; /* added once at exit */
    for (int j = blockIdx.x; j < nq; j += gridDim.x) {
        const int qi = qlist ? qlist[j] : j;
        for (int w = threadIdx.x; w < words; w += blockDim.x) bm[w] = 0u;
        __syncthreads();
        Box q = load_box(queries, qi);
        unsigned long long cand = 0, hits = 0;
        const int64_t ib = (int64_t)(ioff_by_pos ? j : qi) * kSub;
        for (int64_t it = ioff[ib]; it < ioff[ib + kSub]; it++) {
            int2 r = items[it];
            r.x &= ~kAllHit; /* every point is tested here, all-hit items included */
            cand += (unsigned long long)(r.y - r.x);
            scan_range(X, Y, r.x, r.y, q, [&](int i) {
                int t = __ldg(tid + i);
                atomicOr(&bm[t >> 5], 1u << (t & 31));
                hits++;
            });
        }
        /* algorithmic bytes: x and y of every candidate point, the id of every hit */
        my_work += (threadIdx.x == 0 ? 8ull * cand : 0ull) + 4ull * hits;
        __syncthreads();
        int w0 = threadIdx.x * per, w1 = min(words, w0 + per);
        int c = 0;
        for (int w = w0; w < w1; w++) c += __popc(bm[w]);
        int total;
        int pre = block_scan_excl(c, &total, sh);
        if (threadIdx.x == 0) {
            base_sh = atomicAdd(cursor, (unsigned long long)total);
            segcnt[qi] = total;
            segbase[qi] = (int64_t)base_sh;
        }
        __syncthreads();
        int64_t base = (int64_t)base_sh;
        if (base + total <= cap) {
            int64_t o = base + pre;
            for (int w = w0; w < w1; w++) {
                uint32_t v = bm[w];
                while (v) {
                    int b = __ffs(v) - 1;
                    v &= v - 1;
                    arena[o++] = (uint32_t)(w * 32 + b);
                }
            }
        }
        __syncthreads();
    }
    if (work) {
        for (int o = 16; o > 0; o >>= 1) my_work += __shfl_down_sync(0xffffffffu, my_work, o);
        if ((threadIdx.x & 31) == 0 && my_work) atomicAdd(work, my_work);
    }
}

/* ---------------------------------------------------------------- locality order */
/* A batch's queries are scanned in the order of the index position of (about) their first
 * candidate point, bucketed: queries that start near each other in the index's point order
 * (Morton-cell order for the Grid, row-major cells for FSG, KD-leaf order for STIG) read
 * overlapping point ranges, and the CTAs working at one time then share those ranges in L2
 * instead of each fetching them from HBM. The order only changes which CTA scans a query and
 * when; every query's result lands in its own slot, so results are the same. */
constexpr int kOrderBuckets = 1 << 16;
constexpr int kOrderMin = 256; /* smaller batches keep the given order */

/* The key of a query: the index position of the leaf (block, cell) reached by descending from
 * the root into the first child the query intersects, the first candidate of the traversal or
 * close to it; a key only orders queries, so an approximation costs nothing but locality. */
template <int KIND>
__device__ int64_t order_key(const GridDev& g, const StigDev& s, const FsgDev& f, const MortonDev& m, const Box& q) {
    if (KIND == GAT_INDEX_GRID) {
        int nd = 0;
        for (int guard = 0; guard < 64; guard++) {
            const int ch = g.node_child[nd];
            if (ch < 0) break;
            int next = -1;
            for (int c = 0; c < 4 && next < 0; c++) {
                const float4 b = g.node_mbb[ch + c];
                if (box_intersect(q, Box{b.x, b.y, b.z, b.w})) next = ch + c;
            }
            if (next < 0) break;
            nd = next;
        }
        return g.node_pbeg[nd];
    }
    if (KIND == GAT_INDEX_MORTON) {
        int level = 0;
        uint32_t id = 0;
        while (level < m.total_level && !morton_leaf(m, level, id)) {
            int next = -1;
            for (int c = 0; c < 4 && next < 0; c++)
                if (box_intersect(q, morton_box(m, level + 1, (id << 2) + c))) next = c;
            if (next < 0) break;
            id = (id << 2) + (uint32_t)next;
            level++;
        }
        return __ldg(m.cbeg + id * (1u << (2 * (m.total_level - level))));
    }
    if (KIND == GAT_INDEX_STIG) {
        int nd = 0;
        for (int guard = 0; guard < 64 && !s.kind[nd]; guard++) {
            const float lo = s.dim[nd] == 0 ? q.xmin : q.ymin;
            nd = !(lo > s.median[nd]) ? s.left[nd] : s.right[nd];
        }
        return s.kind[nd] ? s.lo[nd] : 0;
    }
    /* FSG: the first cell of the candidate rectangle's first row, clamped to the grid */
    const int g1 = (int)__fdiv_rn(__fsub_rn(q.xmin, f.rxmin), f.cell);
    const int g3 = (int)__fdiv_rn(__fsub_rn(f.rymax, q.ymax), f.cell);
    long long c = (long long)max(g1, 0) + (long long)max(g3, 0) * f.nx;
    if (c > f.cellnum - 1) c = f.cellnum - 1;
    return c < 0 ? 0 : f.cbeg[c];
}

template <int KIND>
__global__ void k_order_keys(GridDev g, StigDev s, FsgDev f, MortonDev m, const gat_mbb* queries, int nq, int64_t npoints,
                             unsigned long long* __restrict__ hist, int* __restrict__ bucket) {
    dep_wait();
    const int qi = blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= nq) return;
    const int64_t key = order_key<KIND>(g, s, f, m, load_box(queries, qi));
    const int b = (int)min((long long)kOrderBuckets - 1, (long long)key * (kOrderBuckets - 1) / (npoints + 1));
    bucket[qi] = b;
    atomicAdd(&hist[b], 1ull);
}

__global__ void k_order_scatter(int nq, const int* __restrict__ bucket, unsigned long long* __restrict__ base,
                                int* __restrict__ order) {
    const int qi = blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= nq) return;
    order[atomicAdd(&base[bucket[qi]], 1ull)] = qi;
}

/* Split of a batch by size: the queries of `order` (or 0..nq-1) with at most `cut` candidate items
 * first, the others after, each part in its order (a stable partition by a scan of the flags) */
__global__ void k_small_flags(int nq, const int* __restrict__ order, const int64_t* __restrict__ ioff, int cut,
                              int64_t* flags) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nq) return;
    const int q = order ? order[j] : j;
    flags[j] = ioff[(int64_t)(q + 1) * kSub] - ioff[(int64_t)q * kSub] <= cut ? 1 : 0;
}
__global__ void k_split_scatter(int nq, const int* __restrict__ order, const int64_t* __restrict__ flags,
                                const int64_t* __restrict__ pos, int* out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nq) return;
    const int q = order ? order[j] : j;
    out[flags[j] ? pos[j] : pos[nq] + (j - pos[j])] = q;
}

/* ---------------------------------------------------------------- id sets, hash form */
/* Queries are taken from a counter by persistent CTAs (the next query's index is fetched while
 * the current one finishes). The CTA's warps take the query's candidate items from a
 * shared-memory counter, scan each with 128-bit loads of x / y / tid (MBB::pInBox) and insert
 * the trajectory id of every hit that starts a run (the previous point is not a hit of the same
 * trajectory: a trajectory's points in one cell are contiguous in every index order) into an
 * open-addressing set in shared memory; a successful insert also appends the id to a list, so
 * the query's m distinct ids are known without scanning the set. The list is sorted (each warp
 * sorts runs of 32 ids in registers, then every id's rank is its position in its run plus its
 * lower bound in every other run; long lists merge the sorted runs pairwise) and written to the
 * arena at the rank; the set is cleared by probing each listed id again. A query whose distinct
 * ids exceed half the set's slots goes on the overflow list for the bitmap kernel; the result is
 * the same set either way. Two shapes: 256 threads with a 8192-slot set, or 128 threads with a
 * 4096-slot set (twice the queries in flight per SM, half the warps meeting at each barrier);
 * run_batch picks one per batch-size class by timing both on the first batch. */
/* A set of 2^HB slots holds up to 2^(HB-1) ids (load factor <= 1/2): 48 KB of shared memory per
 * CTA for HB = 13 (256 threads), 24 KB for HB = 12 (128 threads). */
constexpr int kRankSortMax = 512; /* lists up to this length are sorted by run ranks */
constexpr int kSmallItems = 16;   /* shape 3: queries with at most this many items are scanned one per warp */

template <int HB>
__device__ __forceinline__ unsigned hs_slot(int t) { return ((unsigned)t * 2654435761u) >> (32 - HB); }

/* inserts t; a new id is appended to list (count: ids inserted; ovf: the list or a probe ran out) */
template <int HB>
__device__ __forceinline__ void hs_insert(int* tab, int* list, int t, int* count, int* ovf) {
    unsigned h = hs_slot<HB>(t);
    for (int p = 0; p < 64; p++) {
        int v = tab[h];
        if (v == t) return;
        if (v == -1) {
            v = atomicCAS(&tab[h], -1, t);
            if (v == -1) {
                const int pos = atomicAdd(count, 1);
                if (pos < (1 << (HB - 1)))
                    list[pos] = t;
                else
                    *ovf = 1;
                return;
            }
            if (v == t) return;
        }
        h = (h + 1) & ((1u << HB) - 1);
    }
    *ovf = 1;
}

/* empties the slot holding t (t is in the set) */
template <int HB>
__device__ __forceinline__ void hs_erase(int* tab, int t) {
    unsigned h = hs_slot<HB>(t);
    for (int p = 0; p < (1 << HB); p++) {
        if (tab[h] == t) {
            tab[h] = -1;
            return;
        }
        h = (h + 1) & ((1u << HB) - 1);
    }
}

/* Inserts those of a lane's 4 ids that start a run (differ from the previous point's id; -1 =
 * not a hit). Most steps start no run (a trajectory's points in a cell are consecutive), so the
 * warp tests once whether any lane has one instead of branching on each of the four. Called by
 * all lanes of the warp. */
template <int HB>
__device__ __forceinline__ void insert_runs(int* tab, int* list, int prev, int t0, int t1, int t2, int t3, int* count,
                                            int* ovf) {
    const bool n0 = t0 >= 0 && t0 != prev, n1 = t1 >= 0 && t1 != t0;
    const bool n2 = t2 >= 0 && t2 != t1, n3 = t3 >= 0 && t3 != t2;
    if (!__any_sync(0xffffffffu, n0 | n1 | n2 | n3)) return;
    if (n0) hs_insert<HB>(tab, list, t0, count, ovf);
    if (n1) hs_insert<HB>(tab, list, t1, count, ovf);
    if (n2) hs_insert<HB>(tab, list, t2, count, ovf);
    if (n3) hs_insert<HB>(tab, list, t3, count, ovf);
}

/* ascending sort of the 32 values of a warp (one per lane), bitonic network over shuffles */
__device__ __forceinline__ int warp_sort32(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const int o = __shfl_xor_sync(0xffffffffu, v, j);
            const bool up = (lane & k) == 0;
            const bool lower = (lane & j) == 0;
            v = (lower == up) ? min(v, o) : max(v, o);
        }
    return v;
}

/* number of the 32 ascending values run[0..32) below x: a binary search over the first 31
 * (it leaves lo = how many of them are below x), then the last */
__device__ __forceinline__ int lower_bound32(const int* run, int x) {
    int lo = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1)
        if (run[lo + step - 1] < x) lo += step;
    return lo + (run[31] < x ? 1 : 0);
}

/* One candidate item scanned by one warp: the ids of its points in q that start a run of equal
 * ids go into the set `tab` (appended to `list`; count / ovf as hs_insert). An all-hit item
 * (bit 31 of its start) has every point in q, so only its ids are read. cand / hits / allp add
 * the item's tested points, hits and all-hit points (lane 0 counts the item sizes). */
template <int HB>
__device__ __forceinline__ void scan_item(int2 r, const Box& q, const float* __restrict__ X, const float* __restrict__ Y,
                                          const int32_t* __restrict__ tid, int* tab, int* list, int* count, int* ovf,
                                          unsigned long long& cand, unsigned long long& hits, unsigned long long& allp) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const bool all = r.x < 0;
    r.x &= ~kAllHit;
    const int head_end = min(r.y, (r.x + 3) & ~3);
    const int vb = head_end, ve = head_end + ((r.y - head_end) & ~3);
    if (all) {
        /* every point of the item is a hit: only the ids are read, and the first id of
         * each run of equal ids is inserted (head and tail points always) */
        if (lane == 0) allp += (unsigned long long)(r.y - r.x);
        for (int i = r.x + lane; i < head_end; i += 32) hs_insert<HB>(tab, list, __ldg(tid + i), count, ovf);
        for (int i = ve + lane; i < r.y; i += 32) hs_insert<HB>(tab, list, __ldg(tid + i), count, ovf);
        const int4* T4 = reinterpret_cast<const int4*>(tid + vb);
        const int nv = (ve - vb) >> 2;
        int carry = -1;
        int4 nt = make_int4(-1, -1, -1, -1);
        if (lane < nv) nt = __ldg(T4 + lane);
        for (int k0 = 0; k0 < nv; k0 += 32) {
            const int kk = k0 + lane;
            int4 tt = nt;
            if (kk + 32 < nv) nt = __ldg(T4 + kk + 32);
            if (kk >= nv) tt = make_int4(-1, -1, -1, -1);
            int prev = __shfl_up_sync(FULL, tt.w, 1);
            if (lane == 0) prev = carry;
            carry = __shfl_sync(FULL, tt.w, 31);
            insert_runs<HB>(tab, list, prev, tt.x, tt.y, tt.z, tt.w, count, ovf);
        }
        return;
    }
    if (lane == 0) cand += (unsigned long long)(r.y - r.x);
    /* unaligned head and tail points: plain inserts */
    for (int i = r.x + lane; i < head_end; i += 32)
        if (in_box(q, __ldg(X + i), __ldg(Y + i))) {
            hs_insert<HB>(tab, list, __ldg(tid + i), count, ovf);
            hits++;
        }
    for (int i = ve + lane; i < r.y; i += 32)
        if (in_box(q, __ldg(X + i), __ldg(Y + i))) {
            hs_insert<HB>(tab, list, __ldg(tid + i), count, ovf);
            hits++;
        }
    const float4* X4 = reinterpret_cast<const float4*>(X + vb);
    const float4* Y4 = reinterpret_cast<const float4*>(Y + vb);
    const int4* T4 = reinterpret_cast<const int4*>(tid + vb);
    const int nv = (ve - vb) >> 2;
    int carry = -1; /* tid of the last point of the previous step if it was a hit */
    /* one step tests 4 points per lane; the next step's x, y and ids are loaded before the
     * current step is tested (the ids unconditionally: most candidates are hits, and a
     * load issued only after the test put the whole L2 latency on every step) */
    float4 nx = make_float4(0.f, 0.f, 0.f, 0.f), ny = nx;
    int4 nt = make_int4(-1, -1, -1, -1);
    if (lane < nv) {
        nx = __ldg(X4 + lane);
        ny = __ldg(Y4 + lane);
        nt = __ldg(T4 + lane);
    }
    for (int k0 = 0; k0 < nv; k0 += 32) {
        const int kk = k0 + lane;
        const float4 x = nx, y = ny;
        const int4 tt = nt;
        if (kk + 32 < nv) {
            nx = __ldg(X4 + kk + 32);
            ny = __ldg(Y4 + kk + 32);
            nt = __ldg(T4 + kk + 32);
        }
        int t0 = -1, t1 = -1, t2 = -1, t3 = -1;
        if (kk < nv) {
            const bool h0 = in_box(q, x.x, y.x), h1 = in_box(q, x.y, y.y);
            const bool h2 = in_box(q, x.z, y.z), h3 = in_box(q, x.w, y.w);
            t0 = h0 ? tt.x : -1;
            t1 = h1 ? tt.y : -1;
            t2 = h2 ? tt.z : -1;
            t3 = h3 ? tt.w : -1;
            hits += (unsigned long long)(h0 + h1 + h2 + h3);
        }
        int prev = __shfl_up_sync(FULL, t3, 1);
        if (lane == 0) prev = carry;
        carry = __shfl_sync(FULL, t3, 31);
        insert_runs<HB>(tab, list, prev, t0, t1, t2, t3, count, ovf);
    }
}

template <int NT, int HB>
__global__ void __launch_bounds__(NT, 1024 / NT) k_range_hash(const gat_mbb* queries, int nq, const int64_t* ioff,
                                                           const int2* items, const float* __restrict__ X,
                                                           const float* __restrict__ Y, const int32_t* __restrict__ tid,
                                                           uint32_t* arena, int64_t cap, unsigned long long* ctr,
                                                           int64_t* segbase, int64_t* segcnt, int* ovf_list,
                                                           unsigned long long* work, const int* __restrict__ order,
                                                           const int* __restrict__ small, int ns) {
    constexpr int kHashSize = 1 << HB;
    dep_wait();
    extern __shared__ int hs_smem[];
    int* tab = hs_smem;             /* kHashSize */
    int* buf = hs_smem + kHashSize; /* kHashSize / 2 ids in insertion order */
    __shared__ int cnt_sh, ovf_sh, q_sh, next_sh, item_sh;
    __shared__ unsigned long long base_sh;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned FULL = 0xffffffffu;
    for (int i = threadIdx.x; i < kHashSize; i += blockDim.x) tab[i] = -1;
    /* ctr: [0] arena cursor, [1] work bytes, [2] query counter, [3] overflow count, [4] counter of
     * the small queries (warp mode) */
    /* the next query of the list order[0..nq) (or 0..nq-1), -1 past its end */
    auto fetch = [&]() {
        const int j = (int)atomicAdd(&ctr[2], 1ull);
        return j >= nq ? -1 : (order ? order[j] : j);
    };
    if (threadIdx.x == 0) {
        next_sh = fetch();
        cnt_sh = 0;
        ovf_sh = 0;
        item_sh = 0;
    }
    unsigned long long my_work = 0; /* algorithmic bytes of this thread, added once at exit */
    for (;;) {
        __syncthreads(); /* the set and list are clear, the next query is known */
        const int qi = next_sh;
        if (qi < 0) break;
        const Box q = load_box(queries, qi);
        const int64_t i0 = ioff[(int64_t)qi * kSub], i1 = ioff[(int64_t)(qi + 1) * kSub];
        unsigned long long cand = 0, hits = 0, allp = 0;
        for (;;) {
            int k = 0;
            if (lane == 0) k = atomicAdd(&item_sh, 1);
            k = __shfl_sync(FULL, k, 0);
            const int64_t it = i0 + k;
            /* stop once every item is taken or the set has overflowed (warp-uniform reads) */
            if (it >= i1 || __shfl_sync(FULL, *(volatile int*)&ovf_sh, 0)) break;
            scan_item<HB>(items[it], q, X, Y, tid, tab, buf, &cnt_sh, &ovf_sh, cand, hits, allp);
        }
        /* algorithmic bytes: x and y of every tested point, the id of every hit, the id of every
         * point of an all-hit item */
        my_work += 8ull * cand + 4ull * hits + 4ull * allp;
        __syncthreads(); /* every insert is done */
        const int m = cnt_sh;
        const bool overflow = ovf_sh != 0;
        if (threadIdx.x == 0) {
            if (overflow) {
                const int o = (int)atomicAdd(&ctr[3], 1ull);
                ovf_list[o] = qi;
                segcnt[qi] = 0;
                segbase[qi] = 0;
            } else {
                base_sh = atomicAdd(&ctr[0], (unsigned long long)m);
                segcnt[qi] = m;
                segbase[qi] = (int64_t)base_sh;
            }
            next_sh = fetch();
        }
        __syncthreads(); /* the arena base and the next query are known */
        const int64_t base = (int64_t)base_sh;
        const bool write = !overflow && base + m <= cap;
        if (overflow) {
            for (int i = threadIdx.x; i < kHashSize; i += blockDim.x) tab[i] = -1;
        } else if (m <= kRankSortMax) {
            /* runs of 32 sorted in registers (padded with INT_MAX), written back in place */
            const int runs = (m + 31) >> 5;
            for (int c = warp; c < runs; c += NT / 32) {
                const int i = 32 * c + lane;
                const int v = warp_sort32(i < m ? buf[i] : INT_MAX);
                __syncwarp();
                buf[i] = v;
            }
            __syncthreads();
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                const int x = buf[i], own = i >> 5;
                int rank = i & 31;
                for (int c = 0; c < runs; c++)
                    if (c != own) rank += lower_bound32(buf + 32 * c, x);
                if (write) arena[base + rank] = (uint32_t)x;
                hs_erase<HB>(tab, x);
            }
        } else {
            /* long lists: the set is cleared, runs of 32 are sorted by the warps, then merged in
             * pairs: an id's place in the merged run is its place in its own run plus the number
             * of ids below it in the partner run (a binary search; the ids are distinct), ping-
             * ponging between the list and the set's first slots, which are cleared again at the
             * end. log2(m / 32) rounds, one barrier each. */
            for (int i = threadIdx.x; i < m; i += blockDim.x) hs_erase<HB>(tab, buf[i]);
            const int runs = (m + 31) >> 5;
            for (int c = warp; c < runs; c += NT / 32) {
                const int i = 32 * c + lane;
                const int v = warp_sort32(i < m ? buf[i] : INT_MAX);
                __syncwarp();
                if (i < m) buf[i] = v;
            }
            __syncthreads();
            int* src = buf;
            int* dst = tab;
            for (int L = 32; L < m; L <<= 1) {
                for (int i = threadIdx.x; i < m; i += blockDim.x) {
                    const int x = src[i];
                    const int start = i & ~(2 * L - 1);
                    const int mid = min(start + L, m), end = min(start + 2 * L, m);
                    const bool in_a = i < mid;
                    int lo = in_a ? mid : start;
                    int len = in_a ? end - mid : mid - start;
                    const int first = lo;
                    while (len > 0) {
                        const int half = len >> 1;
                        if (src[lo + half] < x) {
                            lo += half + 1;
                            len -= half + 1;
                        } else {
                            len = half;
                        }
                    }
                    dst[start + (i - (in_a ? start : mid)) + (lo - first)] = x;
                }
                __syncthreads();
                int* t = src;
                src = dst;
                dst = t;
            }
            for (int i = threadIdx.x; i < m; i += blockDim.x) {
                const int v = src[i];
                if (write) arena[base + i] = (uint32_t)v;
                tab[i] = -1; /* the same thread read slot i above when the result is in the set */
            }
        }
        if (threadIdx.x == 0) {
            cnt_sh = 0;
            ovf_sh = 0;
            item_sh = 0;
        }
    }
    /* Warp mode: the small queries small[0..ns), one per warp, each with a set of 2^WB slots of
     * its own (the warp's share of the block's shared memory, all clear after the block mode) and
     * no block barrier; the id list is sorted by the warp (runs of 32, then run ranks). A query
     * with more distinct ids than its set holds goes on the overflow list for the bitmap kernel. */
    if (ns > 0) {
        constexpr int kWarps = NT / 32;
        constexpr int WB = HB - (kWarps == 8 ? 3 : kWarps == 4 ? 2 : 1);
        __shared__ int wcnt[kWarps], wovf[kWarps];
        int* wtab = hs_smem + warp * (1 << WB);
        int* wlist = hs_smem + kHashSize + warp * (1 << (WB - 1));
        if (lane == 0) {
            wcnt[warp] = 0;
            wovf[warp] = 0;
        }
        __syncwarp();
        for (;;) {
            int j = 0;
            if (lane == 0) j = (int)atomicAdd(&ctr[4], 1ull);
            j = __shfl_sync(FULL, j, 0);
            if (j >= ns) break;
            const int qi = small[j];
            const Box q = load_box(queries, qi);
            const int64_t i0 = ioff[(int64_t)qi * kSub], i1 = ioff[(int64_t)(qi + 1) * kSub];
            unsigned long long cand = 0, hits = 0, allp = 0;
            for (int64_t it = i0; it < i1; it++) {
                __syncwarp();
                if (__shfl_sync(FULL, *(volatile int*)&wovf[warp], 0)) break;
                scan_item<WB>(items[it], q, X, Y, tid, wtab, wlist, &wcnt[warp], &wovf[warp], cand, hits, allp);
            }
            my_work += 8ull * cand + 4ull * hits + 4ull * allp;
            __syncwarp();
            const int m = wcnt[warp];
            if (wovf[warp]) {
                if (lane == 0) {
                    const int o = (int)atomicAdd(&ctr[3], 1ull);
                    ovf_list[o] = qi;
                    segcnt[qi] = 0;
                    segbase[qi] = 0;
                }
                for (int i = lane; i < (1 << WB); i += 32) wtab[i] = -1;
            } else {
                const int runs = (m + 31) >> 5;
                for (int c = 0; c < runs; c++) {
                    const int i = 32 * c + lane;
                    const int v = warp_sort32(i < m ? wlist[i] : INT_MAX);
                    __syncwarp();
                    wlist[i] = v;
                }
                unsigned long long b = 0;
                if (lane == 0) {
                    b = atomicAdd(&ctr[0], (unsigned long long)m);
                    segcnt[qi] = m;
                    segbase[qi] = (int64_t)b;
                }
                const int64_t base = (int64_t)__shfl_sync(FULL, b, 0);
                const bool write = base + m <= cap;
                __syncwarp();
                for (int i = lane; i < m; i += 32) {
                    const int x = wlist[i], own = i >> 5;
                    int rank = i & 31;
                    for (int c = 0; c < runs; c++)
                        if (c != own) rank += lower_bound32(wlist + 32 * c, x);
                    if (write) arena[base + rank] = (uint32_t)x;
                    hs_erase<WB>(wtab, x);
                }
            }
            __syncwarp();
            if (lane == 0) {
                wcnt[warp] = 0;
                wovf[warp] = 0;
            }
            __syncwarp();
        }
    }
    if (work) {
        for (int o = 16; o > 0; o >>= 1) my_work += __shfl_down_sync(FULL, my_work, o);
        if (lane == 0 && my_work) atomicAdd(work, my_work);
    }
}

/* ---------------------------------------------------------------- point lists */
/* One CTA per query: count hits, reserve 2*count arena entries, compact the hit keys
 * ((tid << pidx_bits) | pidx) with ballots, sort them with a stable LSD radix sort over the
 * key's significant bits, drop duplicates (a STIG point can sit in two leaves). */
__global__ void __launch_bounds__(kThreads) k_range_points(const gat_mbb* queries, int nq, const int64_t* ioff,
                                                           const int2* items, const float* X, const float* Y,
                                                           const uint32_t* key, int key_bits, uint32_t* arena,
                                                           int64_t cap, unsigned long long* cursor,
                                                           int64_t* segbase, int64_t* segcnt) {
    __shared__ int sh[kThreads / 32 + 1];
    __shared__ int hist[256];
    __shared__ int wcount[kThreads / 32][257];
    __shared__ int running[256];
    __shared__ unsigned long long base_sh;
    __shared__ int wtot[kThreads / 32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int qi = blockIdx.x; qi < nq; qi += gridDim.x) {
        Box q = load_box(queries, qi);
        /* pass 1: count */
        int c = 0;
        for (int64_t it = ioff[(int64_t)qi * kSub]; it < ioff[(int64_t)(qi + 1) * kSub]; it++) {
            int2 r = items[it];
            r.x &= ~kAllHit; /* every point is tested here, all-hit items included */
            scan_range(X, Y, r.x, r.y, q, [&](int) { c++; });
        }
        int total;
        block_scan_excl(c, &total, sh);
        if (threadIdx.x == 0) base_sh = atomicAdd(cursor, 2ull * (unsigned long long)total);
        __syncthreads();
        int64_t base = (int64_t)base_sh;
        if (base + 2 * (int64_t)total > cap) {
            if (threadIdx.x == 0) {
                segcnt[qi] = total;
                segbase[qi] = base;
            }
            __syncthreads();
            continue;
        }
        uint32_t* A = arena + base;
        uint32_t* B = A + total;
        /* pass 2: compact keys in item order, tile by tile (kThreads points per tile) */
        int written = 0;
        for (int64_t it = ioff[(int64_t)qi * kSub]; it < ioff[(int64_t)(qi + 1) * kSub]; it++) {
            int2 r = items[it];
            r.x &= ~kAllHit;
            for (int t0 = r.x; t0 < r.y; t0 += kThreads) {
                int i = t0 + threadIdx.x;
                bool h = i < r.y && in_box(q, __ldg(X + i), __ldg(Y + i));
                unsigned bal = __ballot_sync(0xffffffffu, h);
                if (lane == 0) wtot[warp] = __popc(bal);
                __syncthreads();
                int wb = 0, tt = 0;
                for (int w = 0; w < kThreads / 32; w++) {
                    if (w < warp) wb += wtot[w];
                    tt += wtot[w];
                }
                if (h) A[written + wb + __popc(bal & lanemask_lt())] = __ldg(key + i);
                written += tt;
                __syncthreads();
            }
        }
        /* stable LSD radix sort, 8 bits per pass */
        int passes = (key_bits + 7) / 8;
        uint32_t* src = A;
        uint32_t* dst = B;
        for (int p = 0; p < passes; p++) {
            int shift = 8 * p;
            for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[d] = 0;
            __syncthreads();
            for (int i = threadIdx.x; i < total; i += blockDim.x) atomicAdd(&hist[(src[i] >> shift) & 255], 1);
            __syncthreads();
            if (threadIdx.x == 0) {
                int run = 0;
                for (int d = 0; d < 256; d++) {
                    running[d] = run;
                    run += hist[d];
                }
            }
            for (int d = threadIdx.x; d < 257; d += blockDim.x)
                for (int w = 0; w < kThreads / 32; w++) wcount[w][d] = 0;
            __syncthreads();
            for (int t0 = 0; t0 < total; t0 += kThreads) {
                int i = t0 + threadIdx.x;
                bool valid = i < total;
                uint32_t k = valid ? src[i] : 0u;
                int d = valid ? (int)((k >> shift) & 255) : 256;
                unsigned peers = __match_any_sync(0xffffffffu, d);
                int rank = __popc(peers & lanemask_lt());
                if (rank == 0) wcount[warp][d] = __popc(peers);
                __syncthreads();
                for (int dd = threadIdx.x; dd < 256; dd += blockDim.x) {
                    int run = running[dd];
                    for (int w = 0; w < kThreads / 32; w++) {
                        int t = wcount[w][dd];
                        wcount[w][dd] = run;
                        run += t;
                    }
                    running[dd] = run;
                }
                __syncthreads();
                if (valid) dst[wcount[warp][d] + rank] = k;
                __syncthreads();
                for (int dd = threadIdx.x; dd < 257; dd += blockDim.x)
                    for (int w = 0; w < kThreads / 32; w++) wcount[w][dd] = 0;
                __syncthreads();
            }
            uint32_t* t = src;
            src = dst;
            dst = t;
        }
        /* unique: sorted keys in src, compacted into dst */
        int uniq = 0;
        for (int t0 = 0; t0 < total; t0 += kThreads) {
            int i = t0 + threadIdx.x;
            bool keep = i < total && (i == 0 || src[i] != src[i - 1]);
            unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) wtot[warp] = __popc(bal);
            __syncthreads();
            int wb = 0, tt = 0;
            for (int w = 0; w < kThreads / 32; w++) {
                if (w < warp) wb += wtot[w];
                tt += wtot[w];
            }
            if (keep) dst[uniq + wb + __popc(bal & lanemask_lt())] = src[i];
            uniq += tt;
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            segcnt[qi] = uniq;
            segbase[qi] = base + (dst == A ? 0 : total);
        }
        __syncthreads();
    }
}

/* ---------------------------------------------------------------- gather */
__global__ void k_gather(int nq, const int64_t* segbase, const int64_t* segcnt, const int64_t* off,
                         const uint32_t* arena, int mode, int pidx_bits, int32_t* out_tid, int32_t* out_pidx) {
    for (int qi = blockIdx.x; qi < nq; qi += gridDim.x) {
        int64_t b = segbase[qi], n = segcnt[qi], o = off[qi];
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            uint32_t k = arena[b + i];
            if (mode == GAT_RESULT_IDS) {
                out_tid[o + i] = (int32_t)k;
            } else {
                out_tid[o + i] = (int32_t)(k >> pidx_bits);
                if (out_pidx) out_pidx[o + i] = (int32_t)(k & ((1u << pidx_bits) - 1u));
            }
        }
    }
}

int key_bits_of(const gat_index* ix) {
    int b = 1;
    while (b < 32 && ((int64_t)ix->db->n << ix->pidx_bits) >= ((int64_t)1 << b)) b++;
    return b;
}

/* Candidate items of queries 0..nq-1, or of the nq queries listed in device array qlist (their
 * offsets then by list position): a count pass, a scan of the counts, a pass writing the items.
 * Leaves ioff (kSub offsets per query, nq * kSub + 1 entries) and items in scratch. */
int build_items(gat_ctx* ctx, const gat_index* ix, const gat_mbb* d_q, int nq, const int* qlist, int64_t** ioff_out,
                int2** items_out) {
    cudaStream_t s = ctx->stream;
    int st = GAT_OK;
    const int64_t nsub = (int64_t)nq * kSub;
    int64_t* icnt = (int64_t*)scratch(ctx, S_RANGE_ICNT, (nsub + 1) * sizeof(int64_t), &st);
    int64_t* ioff = icnt ? (int64_t*)scratch(ctx, S_RANGE_IOFF, (nsub + 1) * sizeof(int64_t), &st) : nullptr;
    if (!ioff) return st;
    const int tb = 128, gb = (int)((nsub + tb - 1) / tb);
    auto launch = [&](const int64_t* off, int64_t* cnt, int2* items) {
        switch (ix->kind) {
            case GAT_INDEX_GRID:
                k_items<GAT_INDEX_GRID><<<gb, tb, 0, s>>>(ix->grid, ix->stig, ix->fsg, ix->morton, d_q, nq, qlist, off, cnt,
                                                          items, ctx->d_flag);
                break;
            case GAT_INDEX_STIG:
                k_items<GAT_INDEX_STIG><<<gb, tb, 0, s>>>(ix->grid, ix->stig, ix->fsg, ix->morton, d_q, nq, qlist, off, cnt,
                                                          items, ctx->d_flag);
                break;
            case GAT_INDEX_MORTON:
                k_items<GAT_INDEX_MORTON><<<gb, tb, 0, s>>>(ix->grid, ix->stig, ix->fsg, ix->morton, d_q, nq, qlist, off,
                                                            cnt, items, ctx->d_flag);
                break;
            default:
                k_items<GAT_INDEX_FSG><<<gb, tb, 0, s>>>(ix->grid, ix->stig, ix->fsg, ix->morton, d_q, nq, qlist, off, cnt,
                                                         items, ctx->d_flag);
        }
        count_launch(ctx);
    };
    if (ix->kind != GAT_INDEX_FSG && !qlist) {
        /* task list (above): flags, their scan, the list; counts, their scan, the items. The
         * list and counts are sized for every (query, sub-thread), so only the item total is
         * read back. */
        int64_t* tpos = (int64_t*)scratch(ctx, S_RANGE_TPOS, (nsub + 1) * sizeof(int64_t), &st);
        char* tb_ = tpos ? (char*)scratch(ctx, S_RANGE_TASK, (size_t)nsub * 4 + 2 * (size_t)(nsub + 1) * 8 + 16, &st)
                         : nullptr;
        if (!tb_) return st;
        int64_t* tcnt = reinterpret_cast<int64_t*>(tb_);
        int64_t* toff = tcnt + (nsub + 1);
        int32_t* tasks = reinterpret_cast<int32_t*>(toff + (nsub + 1));
        switch (ix->kind) {
            case GAT_INDEX_GRID:
                k_task_flags<GAT_INDEX_GRID><<<gb, tb, 0, s>>>(ix->grid, ix->stig, ix->morton, d_q, nq, icnt);
                break;
            case GAT_INDEX_STIG:
                k_task_flags<GAT_INDEX_STIG><<<gb, tb, 0, s>>>(ix->grid, ix->stig, ix->morton, d_q, nq, icnt);
                break;
            default:
                k_task_flags<GAT_INDEX_MORTON><<<gb, tb, 0, s>>>(ix->grid, ix->stig, ix->morton, d_q, nq, icnt);
        }
        if ((st = scan_i64(ctx, icnt, tpos, nsub)) != GAT_OK) return st;
        const int lg = (int)std::max<int64_t>(1, std::min<int64_t>((nsub + 255) / 256, (int64_t)ctx->sm_count * 16));
        k_task_list<<<lg, 256, 0, s>>>(nsub, icnt, tpos, tasks);
        GAT_CUDA_TRY(ctx, cudaMemsetAsync(tcnt, 0, (size_t)(nsub + 1) * 8, s), "range");
        auto walk = [&](const int64_t* off, int64_t* cnt, int2* items) {
            switch (ix->kind) {
                case GAT_INDEX_GRID:
                    k_task_walk<GAT_INDEX_GRID><<<lg, 128, 0, s>>>(ix->grid, ix->stig, ix->fsg, ix->morton, d_q, tasks,
                                                                   tpos + nsub, off, cnt, items, ctx->d_flag);
                    break;
                case GAT_INDEX_STIG:
                    k_task_walk<GAT_INDEX_STIG><<<lg, 128, 0, s>>>(ix->grid, ix->stig, ix->fsg, ix->morton, d_q, tasks,
                                                                   tpos + nsub, off, cnt, items, ctx->d_flag);
                    break;
                default:
                    k_task_walk<GAT_INDEX_MORTON><<<lg, 128, 0, s>>>(ix->grid, ix->stig, ix->fsg, ix->morton, d_q, tasks,
                                                                     tpos + nsub, off, cnt, items, ctx->d_flag);
            }
        };
        walk(nullptr, tcnt, nullptr);
        if ((st = scan_i64(ctx, tcnt, toff, nsub)) != GAT_OK) return st;
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_pinned, toff + nsub, sizeof(int64_t), cudaMemcpyDeviceToHost, s), "range");
        GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "range");
        const int64_t nitems = ctx->h_pinned[0];
        int2* items = (int2*)scratch(ctx, S_RANGE_ITEMS, (nitems + 1) * sizeof(int2), &st);
        if (!items) return st;
        walk(toff, nullptr, items);
        k_task_qoff<<<(nq + 256) / 256, 256, 0, s>>>(nq, tpos, toff, ioff);
        count_launch(ctx, 5);
        GAT_CUDA_TRY(ctx, cudaGetLastError(), "range candidates launch");
        *ioff_out = ioff;
        *items_out = items;
        return GAT_OK;
    }
    launch(nullptr, icnt, nullptr);
    if ((st = scan_i64(ctx, icnt, ioff, nsub)) != GAT_OK) return st;
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_pinned, ioff + nsub, sizeof(int64_t), cudaMemcpyDeviceToHost, s), "range");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "range");
    const int64_t nitems = ctx->h_pinned[0];
    int2* items = (int2*)scratch(ctx, S_RANGE_ITEMS, (nitems + 1) * sizeof(int2), &st);
    if (!items) return st;
    launch(ioff, nullptr, items);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "range candidates launch");
    *ioff_out = ioff;
    *items_out = items;
    return GAT_OK;
}

/* Locality order of a batch (k_order_keys): the query indices bucketed by their order key. */
int locality_order(gat_ctx* ctx, const gat_index* ix, const gat_mbb* d_q, int nq, int** order_out) {
    cudaStream_t s = ctx->stream;
    int st = GAT_OK;
    /* [order nq | bucket nq | hist kOrderBuckets + 1 (u64, 8-byte aligned; the scan writes the
     * total into the last entry)] */
    const size_t qwords = ((size_t)2 * nq + 1) & ~(size_t)1;
    int* ob = (int*)scratch(ctx, S_RANGE_ORDER, qwords * sizeof(int) + (size_t)(kOrderBuckets + 1) * 8, &st);
    if (!ob) return st;
    int* bucket = ob + nq;
    auto* hist = reinterpret_cast<unsigned long long*>(ob + qwords);
    (void)launch_dep(ctx, k_zero_words, dim3(64), dim3(256), 0, s, reinterpret_cast<int*>(hist), 2 * kOrderBuckets);
    const int grid = (nq + 255) / 256;
    switch (ix->kind) {
        case GAT_INDEX_GRID:
            k_order_keys<GAT_INDEX_GRID><<<grid, 256, 0, s>>>(ix->grid, ix->stig, ix->fsg, ix->morton, d_q, nq, ix->npoints,
                                                                hist, bucket);
            break;
        case GAT_INDEX_STIG:
            k_order_keys<GAT_INDEX_STIG><<<grid, 256, 0, s>>>(ix->grid, ix->stig, ix->fsg, ix->morton, d_q, nq, ix->npoints,
                                                                hist, bucket);
            break;
        case GAT_INDEX_MORTON:
            k_order_keys<GAT_INDEX_MORTON><<<grid, 256, 0, s>>>(ix->grid, ix->stig, ix->fsg, ix->morton, d_q, nq,
                                                                  ix->npoints, hist, bucket);
            break;
        default:
            k_order_keys<GAT_INDEX_FSG><<<grid, 256, 0, s>>>(ix->grid, ix->stig, ix->fsg, ix->morton, d_q, nq, ix->npoints,
                                                               hist, bucket);
    }
    if ((st = scan_i64(ctx, reinterpret_cast<int64_t*>(hist), reinterpret_cast<int64_t*>(hist), kOrderBuckets)) != GAT_OK)
        return st;
    k_order_scatter<<<grid, 256, 0, s>>>(nq, bucket, hist, ob);
    count_launch(ctx, 3);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "range order");
    *order_out = ob;
    return GAT_OK;
}

/* Runs the pipeline for queries d_q[0..nq) and leaves per-query (segbase, segcnt) in scratch.
 * Returns the total result count in *total.
 * Candidate items first (k_items); id sets then take one launch of the hash kernel in the
 * batch's locality order, and queries whose ids exceed its set go through the bitmap kernel;
 * point lists take the point-list kernel. */
int run_batch(gat_ctx* ctx, const gat_index* ix, const gat_mbb* d_q, int nq, int mode, int64_t* d_off_out,
              int64_t* total) {
    cudaStream_t s = ctx->stream;
    int st = GAT_OK;
    int64_t* segbase = (int64_t*)scratch(ctx, S_RANGE_SEGBASE, (nq + 1) * sizeof(int64_t), &st);
    int64_t* segcnt = (int64_t*)scratch(ctx, S_RANGE_SEGCNT, (nq + 1) * sizeof(int64_t), &st);
    unsigned long long* cursor = (unsigned long long*)scratch(ctx, S_RANGE_CURSOR, 64, &st);
    int* ovf_list = (int*)scratch(ctx, S_RANGE_OVF, (size_t)(nq + 1) * sizeof(int), &st);
    if (!segbase || !segcnt || !cursor || !ovf_list) return st;
    const int words = (ix->db->n + 1 + 31) / 32;
    const size_t smem_bm = (size_t)words * 4;
    const bool bm_in_smem = smem_bm <= 200 * 1024;
    const bool ids = mode == GAT_RESULT_IDS;
    int64_t* ioff = nullptr;
    int2* items = nullptr;
    int* order = nullptr;
    int grid = 1;
    if ((st = build_items(ctx, ix, d_q, nq, nullptr, &ioff, &items)) != GAT_OK) return st;
    if ((st = check_device_flag(ctx, "range candidates")) != GAT_OK) return st;
    /* the hash kernel's two shapes (256 threads / 8192 slots, 128 threads / 4096 slots) */
    int hgrid[3] = {0, 0, 0}, hper[3] = {0, 0, 0};
    size_t hsmem[3] = {0, (size_t)(8192 + 4096) * sizeof(int), (size_t)(4096 + 2048) * sizeof(int)};
    /* shape 3: the batch split by size, queries with more than kSmallItems candidate items in
     * 256-thread block mode and the others one per warp (split[0..ns) small, [ns, nq) large) */
    int* split = nullptr;
    int ns = -1;
    auto make_split = [&]() -> int {
        if (ns >= 0) return GAT_OK;
        int st2 = GAT_OK;
        int64_t* fl = (int64_t*)scratch(ctx, S_RANGE_TPOS, (size_t)2 * (nq + 1) * sizeof(int64_t), &st2);
        split = fl ? (int*)scratch(ctx, S_RANGE_TASK, (size_t)(nq + 1) * sizeof(int), &st2) : nullptr;
        if (!split) return st2;
        int64_t* pos = fl + (nq + 1);
        k_small_flags<<<(nq + 255) / 256, 256, 0, s>>>(nq, order, ioff, kSmallItems, fl);
        count_launch(ctx);
        if ((st2 = scan_i64(ctx, fl, pos, nq)) != GAT_OK) return st2;
        k_split_scatter<<<(nq + 255) / 256, 256, 0, s>>>(nq, order, fl, pos, split);
        count_launch(ctx);
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_pinned + 8, pos + nq, sizeof(int64_t), cudaMemcpyDeviceToHost, s), "range");
        GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "range");
        ns = (int)ctx->h_pinned[8];
        return GAT_OK;
    };
    int shape = ctx->range_shape;
    uint64_t tune_key = 0;
    gat_ctx* tab = ctx->root ? ctx->root : ctx;
    if (ids) {
        if (nq >= kOrderMin && (st = locality_order(ctx, ix, d_q, nq, &order)) != GAT_OK) return st;
        allow_smem(k_range_hash<256, 13>, hsmem[1]);
        allow_smem(k_range_hash<128, 12>, hsmem[2]);
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_range_hash<256, 13>, 256, hsmem[1]);
        hgrid[1] = std::max(1, std::min(nq, std::max(1, per_sm) * ctx->sm_count));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_range_hash<128, 12>, 128, hsmem[2]);
        hgrid[2] = std::max(1, std::min(nq, std::max(1, per_sm) * ctx->sm_count));
        hper[1] = hgrid[1];
        hper[2] = hgrid[2];
        if (shape == 0) {
            uint64_t lg = 0;
            while (lg < 40 && ((int64_t)1 << lg) < nq) lg++;
            tune_key = ((uint64_t)ix->kind << 8) | lg;
            std::lock_guard<std::mutex> lk(tab->tune_mu);
            auto hit = tab->range_tune.find(tune_key);
            if (hit != tab->range_tune.end()) shape = hit->second;
        }
    } else {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_range_points, kThreads, 0);
        grid = std::max(1, std::min(nq, std::max(1, per_sm) * ctx->sm_count));
    }
    const int key_bits = key_bits_of(ix);
    /* result arena: start from a size guess and grow once if the cursor overshoots */
    int64_t cap = std::max<int64_t>(1 << 20, (int64_t)nq * 256);
    for (int attempt = 0; attempt < 2; attempt++) {
        uint32_t* arena = (uint32_t*)scratch(ctx, S_RANGE_ARENA, (size_t)cap * 4, &st);
        if (!arena) return st;
        cap = (int64_t)(ctx->slot_bytes[S_RANGE_ARENA] / 4);
        /* cursor: [0] arena entries, [1] work bytes, [2] query counter, [3] overflowed queries */
        /* one shape over the query list lst[0..n) (lst null: 0..n-1), and the small queries
         * sm[0..n_sm) in warp mode after it */
        auto hash_run = [&](int sh, const int* lst, int n, const int* sm, int n_sm, unsigned long long* work) {
            const int g = std::max(1, std::min(n + n_sm, hper[sh == 2 ? 2 : 1]));
            if (sh == 2)
                k_range_hash<128, 12><<<g, 128, hsmem[2], s>>>(d_q, n, ioff, items, ix->d_x, ix->d_y, ix->d_tid, arena, cap,
                                                               cursor, segbase, segcnt, ovf_list, work, lst, sm, n_sm);
            else
                k_range_hash<256, 13><<<g, 256, hsmem[1], s>>>(d_q, n, ioff, items, ix->d_x, ix->d_y, ix->d_tid, arena, cap,
                                                               cursor, segbase, segcnt, ovf_list, work, lst, sm, n_sm);
            count_launch(ctx);
        };
        auto hash_launch = [&](int sh, unsigned long long* work) {
            cudaError_t e = cudaMemsetAsync(cursor, 0, 5 * sizeof(unsigned long long), s);
            if (e != cudaSuccess) return e;
            if (sh == 3)
                /* the large queries in block mode, then the small ones one per warp */
                hash_run(1, split + ns, nq - ns, split, ns, work);
            else
                hash_run(sh, order, nq, nullptr, 0, work);
            return cudaGetLastError();
        };
        /* the queries the hash kernel handed on (more distinct ids than its set holds) in the
         * bitmap form; leaves the cursor's [0] arena entries and [1] work bytes in h_pinned */
        auto bitmap_pass = [&](unsigned long long* wk, bool timed) -> int {
            GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_pinned, cursor, 4 * sizeof(int64_t), cudaMemcpyDeviceToHost, s), "range");
            GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "range scan");
            const int64_t n_ovf = ctx->h_pinned[3];
            if (n_ovf <= 0) return GAT_OK;
            int per_sm = 0, st2 = GAT_OK;
            if (bm_in_smem) allow_smem(k_range_ids, smem_bm);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_range_ids, kThreads, bm_in_smem ? smem_bm : 0);
            const int g2 = (int)std::max<int64_t>(1, std::min<int64_t>(n_ovf, (int64_t)std::max(1, per_sm) * ctx->sm_count));
            uint32_t* gbm = nullptr;
            if (!bm_in_smem) {
                gbm = (uint32_t*)scratch(ctx, S_RANGE_ARENA2, (size_t)g2 * words * 4, &st2);
                if (!gbm) return st2;
            }
            if (timed) timed_begin(ctx, GAT_KERNEL_RANGE_SCAN);
            k_range_ids<<<g2, kThreads, bm_in_smem ? smem_bm : 0, s>>>(d_q, (int)n_ovf, ioff, items, ix->d_x, ix->d_y,
                                                                      ix->d_tid, words, gbm, arena, cap, cursor, segbase,
                                                                      segcnt, wk, ovf_list, 0);
            if (timed) timed_end(ctx, GAT_KERNEL_RANGE_SCAN, 0.0);
            count_launch(ctx);
            GAT_CUDA_TRY(ctx, cudaGetLastError(), "range scan launch");
            GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_pinned, cursor, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s), "range");
            GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "range scan");
            return GAT_OK;
        };
        if (ids && (shape == 0 || shape == 3) && (st = make_split()) != GAT_OK) return st;
        if (ids && shape == 0) {
            /* first batch of its class: time the three shapes on it twice each, in rotation (the
             * first runs meet cold caches), each with the bitmap pass for the queries its set
             * hands on (the smaller set hands on more), and keep the best (the later run below
             * overwrites every output) */
            constexpr int kShapes = 3, kRuns = 2 * kShapes;
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            float best[kShapes + 1] = {1e30f, 1e30f, 1e30f, 1e30f};
            bool ok = cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
            for (int r = 0; r < kRuns && ok; r++) {
                const int sh = 1 + r % kShapes;
                ok = cudaEventRecord(e0, s) == cudaSuccess && hash_launch(sh, nullptr) == cudaSuccess;
                if (ok && (st = bitmap_pass(nullptr, false)) != GAT_OK) break;
                float ms = 0.f;
                ok = ok && cudaEventRecord(e1, s) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
                     cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
                best[sh] = std::min(best[sh], ms);
            }
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            if (st != GAT_OK) return st;
            if (!ok) return cuda_fail(ctx, cudaGetLastError(), "range shape tuning");
            shape = 1;
            for (int sh = 2; sh <= kShapes; sh++)
                if (best[sh] < best[shape]) shape = sh;
            std::lock_guard<std::mutex> lk(tab->tune_mu);
            tab->range_tune[tune_key] = shape;
        }
        unsigned long long* work = ctx->timing ? cursor + 1 : nullptr;
        timed_begin(ctx, GAT_KERNEL_RANGE_SCAN);
        if (ids) {
            GAT_CUDA_TRY(ctx, hash_launch(shape, work), "range scan launch");
        } else {
            GAT_CUDA_TRY(ctx, cudaMemsetAsync(cursor, 0, 4 * sizeof(unsigned long long), s), "range");
            k_range_points<<<grid, kThreads, 0, s>>>(d_q, nq, ioff, items, ix->d_x, ix->d_y, ix->d_key, key_bits, arena,
                                                     cap, cursor, segbase, segcnt);
            count_launch(ctx);
        }
        timed_end(ctx, GAT_KERNEL_RANGE_SCAN, 0.0);
        GAT_CUDA_TRY(ctx, cudaGetLastError(), "range scan launch");
        if (ids) {
            if ((st = bitmap_pass(work, true)) != GAT_OK) return st;
        } else {
            GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_pinned, cursor, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s), "range");
            GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "range scan");
        }
        const int64_t used = ctx->h_pinned[0];
        if (used <= cap) {
            if (ctx->timing) timed_add_work(ctx, GAT_KERNEL_RANGE_SCAN, (double)ctx->h_pinned[1]);
            break;
        }
        if (attempt == 1) return fail(ctx, GAT_ERR_OOM, "range: result arena overflow");
        cap = used;
    }
    if ((st = scan_i64(ctx, segcnt, d_off_out, nq)) != GAT_OK) return st;
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_pinned, d_off_out + nq, sizeof(int64_t), cudaMemcpyDeviceToHost, s), "range");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "range");
    *total = ctx->h_pinned[0];
    return GAT_OK;
}

int run_gather(gat_ctx* ctx, const gat_index* ix, int nq, int mode, const int64_t* d_off, int32_t* d_tid,
               int32_t* d_pidx) {
    int st = GAT_OK;
    int64_t* segbase = (int64_t*)scratch(ctx, S_RANGE_SEGBASE, (nq + 1) * sizeof(int64_t), &st);
    int64_t* segcnt = (int64_t*)scratch(ctx, S_RANGE_SEGCNT, (nq + 1) * sizeof(int64_t), &st);
    uint32_t* arena = (uint32_t*)ctx->slot_ptr[S_RANGE_ARENA];
    int grid = std::max(1, std::min(nq, ctx->sm_count * 8));
    k_gather<<<grid, kThreads, 0, ctx->stream>>>(nq, segbase, segcnt, d_off, arena, mode, ix->pidx_bits, d_tid, d_pidx);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "range gather launch");
    return GAT_OK;
}


/* Plain execution of id-set queries: per query three dependent launches (items, scan, emit),
 * every buffer sized for any single query before the first launch (items by the index's
 * candidate-range bound, the id bitmap by the set's trajectory count), so nothing waits on the
 * host between queries; one synchronisation at the end reads the total and the status. */
int run_plain_ids(gat_ctx* ctx, const gat_index* ix, const gat_mbb* d_q, int nq, int64_t* d_off, int32_t* d_tid,
                  int64_t capacity, int64_t* needed) {
    cudaStream_t s = ctx->stream;
    int st = GAT_OK;
    /* items of one query: every candidate range (a leaf, a block, or a row of cells) yields its
     * points in chunks of kChunk - 3 or more points, plus one partial chunk */
    const int64_t ranges = ix->kind == GAT_INDEX_FSG ? (int64_t)ix->fsg.ny + 2 : std::max<int64_t>(ix->leaves, 1);
    const int64_t item_cap = 2 * ranges + ix->npoints / (kChunk - 4) + 2 * kPlainSub + 16;
    const int words = (ix->db->n + 1 + 31) / 32;
    int64_t* ioff = (int64_t*)scratch(ctx, S_RANGE_IOFF, 2 * sizeof(int64_t), &st);
    int2* items = (int2*)scratch(ctx, S_RANGE_ITEMS, (size_t)(item_cap + 1) * sizeof(int2), &st);
    uint32_t* bitmap = (uint32_t*)scratch(ctx, S_RANGE_ARENA2, (size_t)words * 4, &st);
    /* cursor: [0] truncation word, [1] work of the whole call */
    unsigned long long* cursor = (unsigned long long*)scratch(ctx, S_RANGE_CURSOR, 64, &st);
    if (!ioff || !items || !bitmap || !cursor) return st;
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(bitmap, 0, (size_t)words * 4, s), "range");
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(cursor, 0, 64, s), "range");
    int32_t* trunc = reinterpret_cast<int32_t*>(cursor);
    unsigned long long* work = ctx->timing ? cursor + 1 : nullptr;
    auto items_kernel = ix->kind == GAT_INDEX_GRID     ? k_plain_items<GAT_INDEX_GRID>
                        : ix->kind == GAT_INDEX_STIG   ? k_plain_items<GAT_INDEX_STIG>
                        : ix->kind == GAT_INDEX_MORTON ? k_plain_items<GAT_INDEX_MORTON>
                                                       : k_plain_items<GAT_INDEX_FSG>;
    const int scan_grid = ctx->sm_count;
    for (int qi = 0; qi < nq; qi++) {
        cudaError_t e = launch_dep(ctx, items_kernel, dim3(1), dim3(kPlainSub), 0, s, ix->grid, ix->stig, ix->fsg,
                                   ix->morton, d_q, qi, ioff, items, item_cap, ctx->d_flag);
        timed_begin(ctx, GAT_KERNEL_RANGE_SCAN);
        if (e == cudaSuccess)
            e = launch_dep(ctx, k_plain_scan, dim3(scan_grid), dim3(kThreads), 0, s, d_q, qi, (const int64_t*)ioff,
                           (const int2*)items, (const float*)ix->d_x, (const float*)ix->d_y, (const int32_t*)ix->d_tid,
                           bitmap, work);
        timed_end(ctx, GAT_KERNEL_RANGE_SCAN, 0.0);
        if (e == cudaSuccess)
            e = launch_dep(ctx, k_plain_emit, dim3(1), dim3(kPlainSub), 0, s, qi, bitmap, words, d_off, d_tid, capacity,
                           trunc);
        count_launch(ctx, 3);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "range plain launch");
    }
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_pinned, d_off + nq, sizeof(int64_t), cudaMemcpyDeviceToHost, s), "range");
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_pinned + 1, cursor, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s), "range");
    if ((st = check_device_flag(ctx, "range candidates")) != GAT_OK) return st;
    *needed = ctx->h_pinned[0];
    if (ctx->timing) timed_add_work(ctx, GAT_KERNEL_RANGE_SCAN, (double)ctx->h_pinned[2]);
    if ((int32_t)ctx->h_pinned[1] != 0) return fail(ctx, GAT_ERR_TRUNCATED, "range: output capacity too small");
    return GAT_OK;
}

/* Device-side entry shared by the host and device APIs. Offsets, tids and pidx go to device
 * buffers with the given capacity; needed receives the total. */
int range_dev(gat_ctx* ctx, const gat_index* ix, const gat_mbb* d_q, int nq, int mode, int exec, int64_t* d_off,
              int32_t* d_tid, int32_t* d_pidx, int64_t capacity, int64_t* needed) {
    if (mode == GAT_RESULT_POINTS && ix->pidx_bits < 0)
        return fail(ctx, GAT_ERR_ARG, "range: trajectory ids and point indices do not fit a 32-bit key");
    if (nq == 0) {
        GAT_CUDA_TRY(ctx, cudaMemsetAsync(d_off, 0, sizeof(int64_t), ctx->stream), "range");
        *needed = 0;
        return gat_ctx_sync(ctx);
    }
    int st;
    if (exec == GAT_EXEC_BATCHED) {
        int64_t total = 0;
        if ((st = run_batch(ctx, ix, d_q, nq, mode, d_off, &total)) != GAT_OK) return st;
        *needed = total;
        if (total > capacity) return fail(ctx, GAT_ERR_TRUNCATED, "range: output capacity too small");
        if ((st = run_gather(ctx, ix, nq, mode, d_off, d_tid, d_pidx)) != GAT_OK) return st;
        return gat_ctx_sync(ctx);
    }
    if (mode == GAT_RESULT_IDS) return run_plain_ids(ctx, ix, d_q, nq, d_off, d_tid, capacity, needed);
    /* plain point lists: one query per pipeline run */
    int64_t done = 0;
    int64_t* off1 = (int64_t*)scratch(ctx, S_RANGE_OFF, 2 * sizeof(int64_t), &st);
    if (!off1) return st;
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(d_off, 0, sizeof(int64_t), ctx->stream), "range");
    bool truncated = false;
    for (int qi = 0; qi < nq; qi++) {
        int64_t total = 0;
        if ((st = run_batch(ctx, ix, d_q + qi, 1, mode, off1, &total)) != GAT_OK) return st;
        if (!truncated && done + total <= capacity) {
            if ((st = run_gather(ctx, ix, 1, mode, off1, d_tid + done, d_pidx ? d_pidx + done : nullptr)) != GAT_OK)
                return st;
        } else {
            truncated = true;
        }
        done += total;
        ctx->h_pinned[1] = done;
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(d_off + qi + 1, ctx->h_pinned + 1, sizeof(int64_t), cudaMemcpyHostToDevice, ctx->stream), "range");
        GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "range");
    }
    *needed = done;
    if (truncated) return fail(ctx, GAT_ERR_TRUNCATED, "range: output capacity too small");
    return GAT_OK;
}

}  // namespace
}  // namespace gat

using namespace gat;

extern "C" {

int gat_range_query_dev(gat_ctx* ctx, const gat_index* ix, const gat_mbb* d_queries, int nq, int result_kind, int exec,
                        int64_t* d_offsets, int32_t* d_tid, int32_t* d_pidx, int64_t capacity, int64_t* needed) {
    if (!ctx || !ix || nq < 0 || (nq > 0 && (!d_queries || !d_tid)) || !d_offsets || !needed ||
        (result_kind != GAT_RESULT_IDS && result_kind != GAT_RESULT_POINTS) ||
        (exec != GAT_EXEC_PLAIN && exec != GAT_EXEC_BATCHED))
        return fail(ctx, GAT_ERR_ARG, "gat_range_query_dev: bad arguments");
    if (!same_owner(ix->ctx, ctx)) return fail(ctx, GAT_ERR_STATE, "gat_range_query_dev: index from another context");
    if (int rq = require_device(ctx, "gat_range_query_dev")) return rq;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return range_dev(ctx, ix, d_queries, nq, result_kind, exec, d_offsets, d_tid, d_pidx, capacity, needed);
}

int gat_range_query(gat_ctx* ctx, const gat_index* ix, const gat_mbb* queries, int nq, int result_kind, int exec,
                    int64_t* offsets, int32_t* out_tid, int32_t* out_pidx, int64_t capacity, int64_t* needed) {
    if (!ctx || !ix || nq < 0 || (nq > 0 && !queries) || !offsets || !needed || capacity < 0 ||
        (capacity > 0 && !out_tid) || (result_kind == GAT_RESULT_POINTS && capacity > 0 && !out_pidx) ||
        (result_kind != GAT_RESULT_IDS && result_kind != GAT_RESULT_POINTS) ||
        (exec != GAT_EXEC_PLAIN && exec != GAT_EXEC_BATCHED))
        return fail(ctx, GAT_ERR_ARG, "gat_range_query: bad arguments");
    if (!same_owner(ix->ctx, ctx)) return fail(ctx, GAT_ERR_STATE, "gat_range_query: index from another context");
    if (int rq = require_device(ctx, "gat_range_query")) return rq;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    int st = GAT_OK;
    gat_mbb* dq = (gat_mbb*)scratch(ctx, S_RANGE_Q, (size_t)(nq + 1) * sizeof(gat_mbb), &st);
    if (!dq) return st;
    if (nq > 0) GAT_CUDA_TRY(ctx, cudaMemcpyAsync(dq, queries, nq * sizeof(gat_mbb), cudaMemcpyHostToDevice, s), "range H2D");
    /* outputs land in device scratch first, sized to the host capacity */
    int64_t dcap = std::max<int64_t>(capacity, 1);
    int32_t* dt = (int32_t*)scratch(ctx, S_RANGE_OUT_T, (size_t)dcap * 4, &st);
    int32_t* dp = result_kind == GAT_RESULT_POINTS ? (int32_t*)scratch(ctx, S_RANGE_OUT_P, (size_t)dcap * 4, &st) : nullptr;
    int64_t* csr = (int64_t*)scratch(ctx, S_RANGE_CSR, (size_t)(nq + 2) * sizeof(int64_t), &st);
    if (!dt || !csr || (result_kind == GAT_RESULT_POINTS && !dp)) return st;
    int64_t need = 0;
    st = range_dev(ctx, ix, dq, nq, result_kind, exec, csr, dt, dp, capacity, &need);
    *needed = need;
    if (st == GAT_OK || st == GAT_ERR_TRUNCATED)
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(offsets, csr, (size_t)(nq + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s), "range D2H");
    if (st == GAT_OK && need > 0) {
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(out_tid, dt, (size_t)need * 4, cudaMemcpyDeviceToHost, s), "range D2H");
        if (result_kind == GAT_RESULT_POINTS)
            GAT_CUDA_TRY(ctx, cudaMemcpyAsync(out_pidx, dp, (size_t)need * 4, cudaMemcpyDeviceToHost, s), "range D2H");
    }
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "range");
    return st;
}

}  // extern "C"
