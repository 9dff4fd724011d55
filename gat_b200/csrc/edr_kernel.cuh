/* The EDR wavefront kernel, shared by the pair API (edr.cu) and the top-k walk (topk.cu).
 *
 * Recurrence (Grid::SimilarityExecuter, Grid.cpp:1274-1306): with m = D[r-1][c-1] + subcost,
 * u = D[r-1][c] + 1, l = D[r][c-1] + 1, the reference takes m when m is below both others,
 * else l when l is below both others, else u. That is min(m, u, l) except when m == l, where
 * it is u (also when u is larger); the kernel evaluates exactly that. subcost is 0 when
 * |x1 - x2| < eps and |y1 - y2| < eps with float differences compared in double
 * (Grid.cpp:1281); the kernel compares the float |difference| with u_eps, the smallest float
 * not below eps, which is the same predicate. Orientation: rows are the query when the
 * candidate is at least as long, else the candidate (Grid.cpp:1234-1247).
 *
 * Mapping: a warp works on row tiles of 32*R rows. Lane L owns R consecutive rows of the tile
 * and handles column j = s - L at step s, so a step advances 32*R cells of one anti-diagonal
 * band. The value below a lane's last row moves to the next lane with one shuffle per step;
 * columns are staged 32 at a time in per-warp shared memory that every lane reads; a tile hands
 * its bottom row to the next tile through a carry row in global memory (L2-resident).
 * Everything is int32 arithmetic plus two float subtractions and two compares per cell.
 *
 * Two kernels: k_edr (one warp per pair, its tiles in sequence; used by the allocation-free
 * entry point) and k_edr_tiles (row tiles as work items, longest pairs first, consecutive
 * tiles of a pair pipelined across warps; every other caller).
 */
#pragma once
#include <algorithm>

#include "internal.h"
#include "launch.cuh"

namespace gat {
namespace edr {

constexpr int kWarps = 8; /* k_edr (one warp per pair) */
constexpr int kTileWarps = 8; /* k_edr_tiles (2-warp CTAs measured no better on small launches) */
constexpr int kBig = 1 << 29; /* above any distance; up + 1 never overflows against it */

/* Pair source over (a_off, a_len, b_off, b_len) arrays; results to out[p]. A pair with a side
 * outside 1..lim gets -1, raises GAT_ERR_ARG in the status word and runs as an empty problem
 * whose result goes to the sink word (flag + 1). */
struct SoaPairs {
    int npairs;
    const int* d_npairs;
    const int64_t* a_off;
    const int32_t* a_len;
    const int64_t* b_off;
    const int32_t* b_len;
    const float2* A;
    const float2* B;
    int32_t* out;
    int lim;
    int32_t* flag;
    static constexpr int kKind = 0;
    __device__ int count() const { return d_npairs ? *d_npairs : npairs; }
    __device__ void get(int p, const float2*& a, int& la, const float2*& b, int& lb, int32_t*& o) const {
        la = a_len[p];
        lb = b_len[p];
        if (la < 1 || lb < 1 || la > lim || lb > lim) {
            out[p] = -1;
            atomicCAS(flag, 0, GAT_ERR_ARG);
            a = A;
            b = B;
            la = lb = 0;
            o = flag + 1;
            return;
        }
        a = A + a_off[p];
        b = B + b_off[p];
        o = out + p;
    }
};

template <int R, class Src>
__global__ void __launch_bounds__(kWarps * 32) k_edr(Src src, float u, int* __restrict__ carry, int carry_stride,
                                                     unsigned* __restrict__ work, unsigned long long* __restrict__ cells) {
    __shared__ float2 bring[kWarps][64];
    __shared__ int cring[kWarps][64];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gw = blockIdx.x * kWarps + wib;
    int* cbuf0 = carry + (size_t)gw * 2 * carry_stride;
    int* cbuf1 = cbuf0 + carry_stride;
    const int n = src.count();
    for (;;) {
        unsigned p = 0;
        if (lane == 0) p = atomicAdd(work, 1u);
        p = __shfl_sync(FULL, p, 0);
        if ((int)p >= n) break;
        const float2 *pa, *pb;
        int la, lb;
        int32_t* outp;
        src.get((int)p, pa, la, pb, lb, outp);
        const float2* rows;
        const float2* cols;
        int len1, len2;
        if (lb >= la) {
            rows = pa;
            cols = pb;
            len1 = la;
            len2 = lb;
        } else {
            rows = pb;
            cols = pa;
            len1 = lb;
            len2 = la;
        }
        int result;
        if (len1 == 0 || len2 == 0) {
            result = len1 + len2;
        } else {
            constexpr int kTile = 32 * R;
            const int ntiles = (len1 + kTile - 1) / kTile;
            const int last_row = len1 - 1;
            result = 0;
            for (int t = 0; t < ntiles; t++) {
                const int* cin = (t & 1) ? cbuf1 : cbuf0;
                int* cout = (t & 1) ? cbuf0 : cbuf1;
                const bool write_carry = t + 1 < ntiles;
                const int r0 = t * kTile + lane * R;
                float ax[R], ay[R];
                int left[R];
#pragma unroll
                for (int i = 0; i < R; i++) {
                    int r = r0 + i;
                    if (r < len1) {
                        float2 v = rows[r];
                        ax[i] = v.x;
                        ay[i] = v.y;
                    } else {
                        ax[i] = __int_as_float(0x7f800000); /* +inf never matches */
                        ay[i] = ax[i];
                    }
                    left[i] = r + 1; /* D[r+1][0] */
                }
                const bool owns_last = (last_row >= r0) && (last_row < r0 + R);
                const int last_i = last_row - r0;
                int diag_in = r0; /* D[r0][0] */
                int bottom = 0;
                const int steps = len2 + 31;
                for (int s = 0; s < steps; s++) {
                    if ((s & 31) == 0) {
                        __syncwarp();
                        int c = s + lane;
                        if (c < len2) {
                            bring[wib][c & 63] = cols[c];
                            cring[wib][c & 63] = t == 0 ? c + 1 : cin[c + 1];
                        }
                        __syncwarp();
                    }
                    const int from_above = __shfl_up_sync(FULL, bottom, 1);
                    const int j = s - lane;
                    if (j >= 0 && j < len2) {
                        const float2 b = bring[wib][j & 63];
                        const int upf = lane == 0 ? cring[wib][j & 63] : from_above;
                        /* Everything except the carry from the row above depends only on the
                         * previous column: with m = diag + subcost and l = left + 1, the
                         * reference's choice equals min(up + 1, mml) where mml = min(m, l),
                         * or +inf when m == l (then it takes up + 1 whatever the others are).
                         * The chain down the lane's rows is then one add-min per cell. */
                        int mml[R];
#pragma unroll
                        for (int i = 0; i < R; i++) {
                            const bool match = (fabsf(__fsub_rn(ax[i], b.x)) < u) & (fabsf(__fsub_rn(ay[i], b.y)) < u);
                            const int m = (i == 0 ? diag_in : left[i - 1]) + (match ? 0 : 1);
                            const int l = left[i] + 1;
                            mml[i] = (m == l) ? kBig : min(m, l);
                        }
                        int up = upf;
#pragma unroll
                        for (int i = 0; i < R; i++) {
                            up = __viaddmin_s32(up, 1, mml[i]);
                            left[i] = up;
                        }
                        bottom = up;
                        diag_in = upf;
                        if (write_carry && lane == 31) cout[j + 1] = bottom;
                        if (owns_last && j == len2 - 1) {
#pragma unroll
                            for (int i = 0; i < R; i++)
                                if (i == last_i) result = left[i];
                        }
                    }
                }
                __syncwarp();
            }
            /* the owner of the last row holds the answer */
            const int owner = (last_row % (32 * R)) / R;
            result = __shfl_sync(FULL, result, owner);
        }
        if (lane == 0) {
            *outp = result;
            if (cells) atomicAdd(cells, (unsigned long long)len1 * (unsigned long long)len2);
        }
    }
}

/* ================================================================ tiled, load-balanced form
 * Work items are row tiles. A pair whose rows span T >= 2 tiles contributes T items and its
 * tiles run on different warps, pipelined: tile t consumes the bottom row of tile t-1 through a
 * carry row in L2 while tile t-1 is still producing it. Pairs with one tile, and multi-tile
 * pairs beyond the cooperative pool, are one item that a single warp walks tile by tile with
 * its own carry rows.
 *
 * Carry words: each column's carry value is one 64-bit word, tag << 16 | (uint16) value, with
 * tag = launch epoch << 8 | producing tile (mod 256). The consumer polls the words it needs and
 * accepts a word whose tag is the one it expects, so the hand-over needs neither a progress
 * flag nor a memory fence: a 64-bit store is seen whole or not at all. Values are the
 * column-shifted distances E = D - c, which lie in [-16384, 16384] and fit 16 bits; epochs
 * come from a per-context device counter and only grow (2^40 launches before a repeat), and carry buffers are zeroed when allocated, so a
 * stale word never carries the expected tag. A tile rewrites the buffer its predecessor read
 * (double buffering per pair) only for columns that predecessor has already consumed.
 *
 * Schedule (longest first): a count pass puts every pair in one of kClasses duration classes
 * (half-octaves of the pair's critical path in column steps: len2 + 32 (T - 1) when its tiles
 * are pipelined, T (len2 + 31) on one warp) and a write pass lays the items out class by
 * class, longest class first, a pair's tiles consecutive. Warps take items in that order from
 * one counter, so the long pairs start first and the short ones fill in behind them.
 *
 * Waits are bounded: after kSpinLimit polls the warp raises GAT_ERR_TIMEOUT in the status word
 * and abandons the pair (its result becomes -1). The producer of the tile a warp waits for
 * took the preceding item from the same counter, so it is already running. */
constexpr int kSpinLimit = 1 << 22;
constexpr int kClasses = 48;
/* counter block: [0] item counter, [1] cooperative slots taken, [2] total items,
 * [4, 4 + kClasses) items per class, [4 + kClasses, 4 + 2 kClasses) class cursors, then the
 * launch's epoch (64-bit, 8-byte aligned) */
constexpr int kCtrEpoch = 4 + 2 * kClasses;
constexpr int kCtrWords = kCtrEpoch + 2;
typedef unsigned long long carry_t;

constexpr int kEdrCarveoutPct = 100; /* preferred shared-memory share of the SM for k_edr_tiles (launch_tiles) */

struct TileCtl {
    const int4* items; /* (pair, tile or -1 for a whole pair on one warp, cooperative slot, tiles) */
    const int* total;
    carry_t* pair_carry; /* cooperative slot s: rows pair_carry + s * 2 * stride */
    carry_t* warp_carry; /* per-warp double carry rows for single-warp pairs */
    int stride;
    const unsigned long long* epoch; /* written by the schedule's write pass */
    int32_t* flag;
    int spin_limit;  /* polls before a carry wait gives up (kSpinLimit) */
    int stall_pair;  /* tests of the bounded wait: this pair's first pipelined tile writes no carries (-1: none) */
};

/* The carry word is the only datum exchanged, so neither access needs to order other memory
 * operations (no "memory" clobber: the step loop's shared-memory loads may move across them);
 * volatile keeps every poll a fresh load. */
__device__ __forceinline__ carry_t ld_carry(const carry_t* p) {
    carry_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void st_carry(carry_t* p, carry_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v));
}

/* floor(2 log2(d)) for d >= 1, clamped to the class range */
__device__ __forceinline__ int duration_class(long long d) {
    if (d < 1) d = 1;
    const int e = 63 - __clzll(d);
    const int half = (d * d >= (1LL << (2 * e + 1))) ? 1 : 0;
    return min(2 * e + half, kClasses - 1);
}

template <int R, bool COL, class Src>
__global__ void k_sched_count(Src src, int cap, int coop_cap, int* __restrict__ ctr, int2* __restrict__ meta) {
    dep_wait();
    __shared__ int hist[kClasses];
    for (int i = threadIdx.x; i < kClasses; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const int n = min(src.count(), cap);
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float2 *a, *b;
        int la, lb;
        int32_t* o;
        src.get(p, a, la, b, lb, o);
        const int len1 = min(la, lb), len2 = max(la, lb);
        const int nlane = COL ? len2 : len1, nstep = COL ? len1 : len2;
        const int T = nlane <= 0 ? 1 : (nlane + 32 * R - 1) / (32 * R);
        int slot = -1, items = 1;
        if (T >= 2) {
            const int sl = atomicAdd(&ctr[1], 1);
            if (sl < coop_cap) {
                slot = sl;
                items = T;
            }
        }
        const long long dur = slot >= 0 ? (long long)nstep + 32LL * (T - 1) : (long long)T * (nstep + 31);
        const int c = duration_class(dur);
        atomicAdd(&hist[c], items);
        meta[p] = make_int2(slot, (c << 16) | items);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kClasses; i += blockDim.x)
        if (hist[i]) atomicAdd(&ctr[4 + i], hist[i]);
}

template <class Src>
__global__ void k_sched_write(Src src, int cap, int* __restrict__ ctr, const int2* __restrict__ meta,
                              int4* __restrict__ items, unsigned long long* __restrict__ epochs) {
    dep_wait();
    __shared__ int off[kClasses];
    __shared__ int lcnt[kClasses];
    __shared__ int lbase[kClasses];
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int c = kClasses - 1; c >= 0; c--) {
            off[c] = acc;
            acc += ctr[4 + c];
        }
        if (blockIdx.x == 0) {
            ctr[2] = acc;
            /* a fresh epoch per launch from the context's device counter, so launches replayed
             * from a CUDA graph never reuse a tag */
            *reinterpret_cast<unsigned long long*>(ctr + kCtrEpoch) = atomicAdd(epochs, 1ull) + 1ull;
        }
    }
    const int n = min(src.count(), cap);
    /* block-sized chunks (uniform trip count over the block) so the local counters reset */
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        for (int i = threadIdx.x; i < kClasses; i += blockDim.x) lcnt[i] = 0;
        __syncthreads();
        const int p = base + threadIdx.x;
        int c = 0, nit = 0, loc = 0, slot = -1;
        if (p < n) {
            const int2 m = meta[p];
            slot = m.x;
            c = m.y >> 16;
            nit = m.y & 0xffff;
            loc = atomicAdd(&lcnt[c], nit);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < kClasses; i += blockDim.x)
            if (lcnt[i]) lbase[i] = atomicAdd(&ctr[4 + kClasses + i], lcnt[i]);
        __syncthreads();
        if (p < n) {
            const int pos = off[c] + lbase[c] + loc;
            if (slot < 0)
                items[pos] = make_int4(p, -1, -1, 1);
            else
                for (int t = 0; t < nit; t++) items[pos + t] = make_int4(p, t, slot, nit);
        }
        __syncthreads();
    }
}

/* Match mask of one cell: -1 when |x1 - x2| < u and |y1 - y2| < u (float differences, no
 * contraction), else 0. */
__device__ __forceinline__ int match_mask(float ax, float ay, float2 b, float u) {
    const float dx = __fsub_rn(ax, b.x), dy = __fsub_rn(ay, b.y);
    int m;
    asm("{\n\t.reg .pred p;\n\t.reg .f32 t0, t1;\n\t"
        "abs.f32 t0, %1;\n\tabs.f32 t1, %2;\n\t"
        "setp.lt.f32 p, t0, %3;\n\t"
        "set.lt.and.s32.f32 %0, t1, %3, p;\n\t}"
        : "=r"(m)
        : "f"(dx), "f"(dy), "f"(u));
    return m;
}

/* One wavefront step of a lane's R rows at column c (DP column index). Values are held shifted
 * by their column: E[r][c] = D[r][c] - c. The reference's three operands at (r, c) become, in
 * column c's shift, m = E[r-1][c-1] + (match ? -1 : 0), l = E[r][c-1] and u = E[r-1][c] + 1;
 * a common shift keeps every comparison, so the choice min(u, mml), mml = min(m, l) or +inf
 * when m == l, is taken on shifted values unchanged. State per row i: Lp[i] = E[r0+i+1][c-1];
 * diag0 = E[r0][c-1]; up0 = E[r0][c] (the value above the lane's first row). */
template <int R>
__device__ __forceinline__ int wf_step(const float (&ax)[R], const float (&ay)[R], int (&Lp)[R], int& diag0, float2 b,
                                       int up0, float u) {
    int mml[R];
#pragma unroll
    for (int i = 0; i < R; i++) {
        const int m = (i == 0 ? diag0 : Lp[i - 1]) + match_mask(ax[i], ay[i], b, u);
        mml[i] = (m == Lp[i]) ? kBig : min(m, Lp[i]);
    }
    int up = up0;
#pragma unroll
    for (int i = 0; i < R; i++) {
        up = __viaddmin_s32(up, 1, mml[i]);
        Lp[i] = up;
    }
    diag0 = up0;
    return up;
}

/* Column-tile form of the same recurrence: a lane owns R consecutive DP columns and a step
 * advances one DP row r. Values are held shifted by their row: F[r][c] = D[r][c] - r, so in
 * row r's shift u = F[r-1][c] needs no add, m = F[r-1][c-1] + (match ? -1 : 0) and
 * l = F[r][c-1] + 1, whose chain runs along the lane's columns: with mm1 = m - 1 and
 * prev = F[r][c-1], m == l exactly when mm1 == prev, min(m, l) = min(mm1, prev) + 1, and the
 * cell is u when they are equal, else min(u, min(m, l)). State per column j: F[j] =
 * F[r-1][c_j] on entry, F[r][c_j] on exit; diag0 = F[r-1][c_0 - 1]; left = F[r][c_0 - 1] (the
 * value to the left of the lane's first column). Same interface as wf_step. */
template <int R>
__device__ __forceinline__ int cf_step(const float (&bx)[R], const float (&by)[R], int (&F)[R], int& diag0, float2 a,
                                       int left, float u) {
    int prev = left;
    int diag = diag0;
#pragma unroll
    for (int j = 0; j < R; j++) {
        const int up = F[j];
        const int mm1 = diag + match_mask(bx[j], by[j], a, u) - 1;
        const int mn = min(mm1, prev);
        const int d = (mm1 == prev) ? up : __viaddmin_s32(mn, 1, up);
        diag = up;
        F[j] = d;
        prev = d;
    }
    diag0 = left;
    return prev;
}

/* One row tile of one pair (rows r0 = t * 32R ...). cin: the carry words of tile t-1's bottom
 * row (nullptr for t == 0), accepted with tag tag_in; cout: this tile's bottom row for tile t+1
 * (nullptr for the last tile), written with tag tag_out. Returns false when a wait gave up.
 * The owner lane of the pair's last row leaves the distance in `result`.
 *
 * Columns move through a per-warp window of 64 points in shared memory: at the start of the
 * chunk of columns [s0, s0 + 32) the window holds columns s0 - 32 .. s0 + 31, so lane L reads
 * column s0 + k - L of step k at window index 32 + k - L (a per-lane base plus a constant).
 * The next chunk's points and carry words are loaded one chunk early. Chunks where every
 * lane's column is inside the pair skip the bounds test. */
/* COL: the column-tile form (cf_step); rows / cols / len1 / len2 then name the lane side
 * (columns) and the step side (rows), the carry runs along the tile's last column, and the
 * result is F + len2 (the step side's length), exactly as the row form's E + len2. */
template <int R, bool COL = false>
__device__ __forceinline__ bool edr_tile(const float2* __restrict__ rows, const float2* __restrict__ cols, int len1,
                                         int len2, int t, const carry_t* cin, carry_t* cout, carry_t tag_in,
                                         carry_t tag_out, float u, float2* sb, int* sc, int& result,
                                         int spin_limit) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const bool lane0 = lane == 0;
    const bool writer = cout != nullptr && lane == 31;
    constexpr int kTile = 32 * R;
    const int r0 = t * kTile + lane * R;
    float ax[R], ay[R];
    int Lp[R];
#pragma unroll
    for (int i = 0; i < R; i++) {
        const int r = r0 + i;
        if (r < len1) {
            const float2 v = rows[r];
            ax[i] = v.x;
            ay[i] = v.y;
        } else {
            ax[i] = __int_as_float(0x7f800000); /* +inf never matches */
            ay[i] = ax[i];
        }
        Lp[i] = r + 1; /* E[r+1][0] = D[r+1][0] */
    }
    int diag0 = r0; /* E[r0][0] */
    int bottom = 0;
    const float2* pb = sb + 32 - lane;
    const int steps = len2 + 31;
    const carry_t tag_hi = tag_out << 16;
    /* prefetched inputs of the next chunk: column point and carry word of column s0 + lane */
    float2 nb = make_float2(0.f, 0.f);
    carry_t nw = 0;
    bool nw_ok = false;
    if (lane < len2) {
        nb = cols[lane];
        if (cin) {
            nw = ld_carry(cin + lane + 1);
            nw_ok = (nw >> 16) == tag_in;
        }
    }
    for (int s0 = 0; s0 < steps; s0 += 32) {
        const int c = s0 + lane;
        if (s0 < len2) {
            int cv = 0; /* E[0][c+1] = D[0][c+1] - (c+1) for the first tile */
            if (cin) {
                bool ok = c >= len2 || nw_ok;
                for (int polls = 0;; polls++) {
                    if (!ok) {
                        nw = ld_carry(cin + c + 1);
                        ok = (nw >> 16) == tag_in;
                    }
                    if (__all_sync(FULL, ok)) break;
                    if (polls >= spin_limit) return false;
                    if (polls >= 16) __nanosleep(64); /* each poll is an L2 round trip already */
                }
                cv = (int)(short)(nw & 0xffffu);
            }
            __syncwarp();
            sb[lane] = sb[32 + lane];
            sb[32 + lane] = nb;
            sc[lane] = cv;
            __syncwarp();
            /* next chunk */
            const int cn = c + 32;
            nw_ok = false;
            if (cn < len2) {
                nb = cols[cn];
                if (cin) {
                    nw = ld_carry(cin + cn + 1);
                    nw_ok = (nw >> 16) == tag_in;
                }
            }
        } else {
            __syncwarp();
            sb[lane] = sb[32 + lane];
            __syncwarp();
        }
        if (s0 >= 32 && s0 + 32 <= len2) {
            /* every lane's column s0 + k - lane lies in [1, len2) */
#pragma unroll 8
            for (int k = 0; k < 32; k++) {
                const int from_above = __shfl_up_sync(FULL, bottom, 1);
                const int up0 = lane0 ? sc[k] : from_above;
                bottom = COL ? cf_step<R>(ax, ay, Lp, diag0, pb[k], up0, u) : wf_step<R>(ax, ay, Lp, diag0, pb[k], up0, u);
                if (writer) st_carry(cout + (s0 + k - 30), tag_hi | (carry_t)(unsigned short)bottom);
            }
        } else {
            const int kend = min(32, steps - s0);
            for (int k = 0; k < kend; k++) {
                const int from_above = __shfl_up_sync(FULL, bottom, 1);
                const int j = s0 + k - lane;
                if (j >= 0 && j < len2) {
                    const int up0 = lane0 ? sc[k] : from_above;
                    bottom = COL ? cf_step<R>(ax, ay, Lp, diag0, pb[k], up0, u)
                                 : wf_step<R>(ax, ay, Lp, diag0, pb[k], up0, u);
                    if (writer) st_carry(cout + (j + 1), tag_hi | (carry_t)(unsigned short)bottom);
                }
            }
        }
    }
    const int last_i = len1 - 1 - r0;
    if (last_i >= 0 && last_i < R) {
#pragma unroll
        for (int i = 0; i < R; i++)
            if (i == last_i) result = Lp[i] + len2; /* D = E + column */
    }
    __syncwarp();
    return true;
}

template <int R, bool COL, class Src>
__global__ void __launch_bounds__(kTileWarps * 32, R == 2 ? 4 : 3) k_edr_tiles(Src src, float u, TileCtl ctl, unsigned* __restrict__ work,
                                                           unsigned long long* __restrict__ cells) {
    dep_wait();
    __shared__ float2 bring[kTileWarps][64];
    __shared__ int cring[kTileWarps][32];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gw = blockIdx.x * kTileWarps + wib;
    carry_t* wc0 = ctl.warp_carry + (size_t)gw * 2 * ctl.stride;
    carry_t* wc1 = wc0 + ctl.stride;
    const carry_t ep = *ctl.epoch << 8;
    const unsigned total = (unsigned)*ctl.total;
    for (;;) {
        unsigned idx = 0;
        if (lane == 0) idx = atomicAdd(work, 1u);
        idx = __shfl_sync(FULL, idx, 0);
        if (idx >= total) break;
        const int4 it = ctl.items[idx];
        const int p = it.x, t = it.y;
        const float2 *pa, *pb;
        int la, lb;
        int32_t* outp;
        src.get(p, pa, la, pb, lb, outp);
        const float2 *rows, *cols;
        int len1, len2;
        if (lb >= la) {
            rows = pa;
            cols = pb;
            len1 = la;
            len2 = lb;
        } else {
            rows = pb;
            cols = pa;
            len1 = lb;
            len2 = la;
        }
        if (len1 == 0 || len2 == 0) {
            if (lane == 0) *outp = len1 + len2;
            continue;
        }
        /* lane side and step side: rows / columns for row tiles, columns / rows for column tiles */
        const float2* lpts = COL ? cols : rows;
        const float2* spts = COL ? rows : cols;
        const int nlane = COL ? len2 : len1, nstep = COL ? len1 : len2;
        constexpr int kTile = 32 * R;
        const int T = (nlane + kTile - 1) / kTile;
        int result = 0;
        bool ok = true, finished = false;
        if (t < 0) {
            for (int tt = 0; tt < T && ok; tt++)
                ok = edr_tile<R, COL>(lpts, spts, nlane, nstep, tt, tt > 0 ? ((tt - 1) & 1 ? wc1 : wc0) : nullptr,
                                      tt + 1 < T ? ((tt & 1) ? wc1 : wc0) : nullptr, ep | ((tt - 1) & 0xff),
                                      ep | (tt & 0xff), u, bring[wib], cring[wib], result, ctl.spin_limit);
            finished = true;
        } else {
            carry_t* pc = ctl.pair_carry + (size_t)it.z * 2 * ctl.stride;
            const bool stalled = p == ctl.stall_pair && t == 0;
            ok = edr_tile<R, COL>(lpts, spts, nlane, nstep, t, t > 0 ? pc + ((t - 1) & 1) * ctl.stride : nullptr,
                                  t + 1 < T && !stalled ? pc + (t & 1) * ctl.stride : nullptr, ep | ((t - 1) & 0xff),
                                  ep | (t & 0xff), u, bring[wib], cring[wib], result, ctl.spin_limit);
            finished = t == T - 1;
        }
        if (!ok) {
            if (lane == 0) {
                atomicCAS(ctl.flag, 0, GAT_ERR_TIMEOUT);
                *outp = -1;
            }
            continue;
        }
        if (finished) {
            const int owner = ((nlane - 1) % kTile) / R;
            result = __shfl_sync(FULL, result, owner);
            if (lane == 0) {
                *outp = result;
                if (cells) atomicAdd(cells, (unsigned long long)len1 * (unsigned long long)len2);
            }
        }
    }
}

/* Host side: schedule (count, write) -> tiled kernel. cap is the number of pairs (exact for
 * host-known lists, an upper bound for device-counted ones); max_rows / max_cols bound the
 * shorter / longer side of every pair. ev0/ev1, when given, bracket the tile kernel. */
template <int R, bool COL, class Src>
int launch_tiles(gat_ctx* ctx, const Src& src, int64_t cap, int max_rows, int max_cols, float u,
                 unsigned long long* cells, cudaEvent_t ev0 = nullptr, cudaEvent_t ev1 = nullptr) {
    int st = GAT_OK;
    cudaStream_t s = ctx->stream;
    int per_sm = 0;
    /* An SM's split between L1 and shared memory changes only while no block is resident on it.
     * With the default (no preference) the persistent grid's blocks, which need 5 KB, leave their
     * SMs at a small shared-memory split for the whole launch, and a kernel of another stream that
     * needs more (the range scan's 48 KB blocks) could not start on any of them until the grid
     * ended: range batches beside a long top-k round waited for it (16 rectangles, 1.1 ms alone:
     * 10.5 ms median beside 18 ms EDR launches that left half the SMs free; 2.5 ms with the
     * largest split). The tile kernel reads its points once and uses little L1. */
    prefer_split(reinterpret_cast<const void*>(k_edr_tiles<R, COL, Src>), ctx->device, kEdrCarveoutPct);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_edr_tiles<R, COL, Src>, kTileWarps * 32, 0);
    /* a serving lane leaves sm_reserve SMs free of this persistent grid for other streams */
    const int grid = std::max(1, ctx->sm_count - ctx->sm_reserve) * (per_sm > 0 ? per_sm : 1);
    /* carry rows run along the step side; tiles are cut along the lane side */
    const int max_lane = COL ? max_cols : max_rows, max_step = COL ? max_rows : max_cols;
    const int stride = max_step + 2;
    const int maxT = max_lane <= 0 ? 1 : (max_lane + 32 * R - 1) / (32 * R);
    const size_t budget = (size_t)512 << 20; /* cooperative carry rows */
    int64_t coop = (int64_t)(budget / ((size_t)2 * stride * sizeof(carry_t)));
    if (coop > cap) coop = cap;
    if (maxT < 2) coop = 0;
    const int64_t item_cap = cap + coop * (maxT - 1);
    if (item_cap >= (int64_t)1 << 31) return fail(ctx, GAT_ERR_ARG, "edr: too many work items in one launch");
    int* ctr = (int*)scratch(ctx, S_EDR_COUNTERS, kCtrWords * sizeof(int), &st);
    int2* meta = (int2*)scratch(ctx, S_EDR_META, (size_t)cap * sizeof(int2), &st);
    int4* items = (int4*)scratch(ctx, S_EDR_ITEMS, (size_t)item_cap * sizeof(int4), &st);
    carry_t* pcarry =
        coop > 0 ? (carry_t*)scratch_zeroed(ctx, S_EDR_PCARRY, (size_t)coop * 2 * stride * sizeof(carry_t), &st) : nullptr;
    carry_t* wcarry = (carry_t*)scratch_zeroed(ctx, S_EDR_CARRY, (size_t)grid * kTileWarps * 2 * stride * sizeof(carry_t), &st);
    if (!ctr || !meta || !items || !wcarry || (coop > 0 && !pcarry)) return st;
    (void)launch_dep(ctx, k_zero_words, dim3(1), dim3(256), 0, s, ctr, (int)kCtrWords);
    const int pgrid = (int)std::max<int64_t>(1, std::min<int64_t>((cap + 255) / 256, (int64_t)ctx->sm_count * 8));
    (void)launch_dep(ctx, k_sched_count<R, COL, Src>, dim3(pgrid), dim3(256), 0, s, src, (int)cap, (int)coop, ctr, meta);
    count_launch(ctx);
    (void)launch_dep(ctx, k_sched_write<Src>, dim3(pgrid), dim3(256), 0, s, src, (int)cap, ctr, meta, items, edr_epochs(ctx));
    count_launch(ctx);
    /* the stall knob (tests of the bounded wait) also shortens the wait to ~2^12 polls */
    const int stall = ctx->test_stall_pair - 1;
    TileCtl ctl{items, ctr + 2, pcarry, wcarry, stride, reinterpret_cast<const unsigned long long*>(ctr + kCtrEpoch),
                ctx->d_flag, stall >= 0 ? (1 << 12) : kSpinLimit, stall};
    /* serving lanes: after the previous EDR grid of any sibling lane (not inside a capture, whose
     * graph cannot wait on an event recorded outside it) */
    std::unique_lock<std::mutex> chain;
    if (ctx->edr_chain) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(s, &cs);
        if (cs == cudaStreamCaptureStatusNone) {
            chain = std::unique_lock<std::mutex>(ctx->edr_chain->mu);
            GAT_CUDA_TRY(ctx, cudaStreamWaitEvent(s, ctx->edr_chain->ev, 0), "edr chain");
        }
    }
    timed_begin(ctx, GAT_KERNEL_EDR);
    if (ev0) cudaEventRecord(ev0, s);
    (void)launch_dep(ctx, k_edr_tiles<R, COL, Src>, dim3(grid), dim3(kTileWarps * 32), 0, s, src, u, ctl, reinterpret_cast<unsigned*>(ctr), cells);
    if (ev1) cudaEventRecord(ev1, s);
    timed_end(ctx, GAT_KERNEL_EDR, 0.0);
    if (chain.owns_lock()) GAT_CUDA_TRY(ctx, cudaEventRecord(ctx->edr_chain->ev, s), "edr chain");
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "edr launch");
    return GAT_OK;
}

/* Tile shapes: rows (or columns) per lane 2, 4, 8, in row or column form. shape = R | COL << 4 */
constexpr int kShapeCol = 16;

template <class Src>
int launch_shape(gat_ctx* ctx, int shape, const Src& src, int64_t cap, int max_rows, int max_cols, float u,
                 unsigned long long* cells, cudaEvent_t ev0 = nullptr, cudaEvent_t ev1 = nullptr) {
    switch (shape) {
        case 2: return launch_tiles<2, false, Src>(ctx, src, cap, max_rows, max_cols, u, cells, ev0, ev1);
        case 4: return launch_tiles<4, false, Src>(ctx, src, cap, max_rows, max_cols, u, cells, ev0, ev1);
        case 8: return launch_tiles<8, false, Src>(ctx, src, cap, max_rows, max_cols, u, cells, ev0, ev1);
        case 2 | kShapeCol: return launch_tiles<2, true, Src>(ctx, src, cap, max_rows, max_cols, u, cells, ev0, ev1);
        case 8 | kShapeCol: return launch_tiles<8, true, Src>(ctx, src, cap, max_rows, max_cols, u, cells, ev0, ev1);
        default: return launch_tiles<4, true, Src>(ctx, src, cap, max_rows, max_cols, u, cells, ev0, ev1);
    }
}

inline uint64_t ceil_log2(int64_t v) {
    uint64_t e = 0;
    while (e < 62 && ((int64_t)1 << e) < v) e++;
    return e;
}

/* EDR over a pair source with the context's tile shape. Rows per lane (GAT_TUNE_EDR_ROWS) and
 * form (GAT_TUNE_EDR_FORM) are fixed by the knobs or autotuned: the first launch of a shape
 * class times the open candidates on this launch's own pairs (every candidate writes the same
 * results; the cell counter is fed once) and records the fastest; later launches of the class
 * use it. */
template <class Src>
int edr_launch(gat_ctx* ctx, const Src& src, int64_t cap, int max_rows, int max_cols, float u,
               unsigned long long* cells) {
    if (cap <= 0) return GAT_OK;
    int cand[6], nc = 0;
    for (int form = 0; form < 2; form++) {
        if (ctx->edr_form && ctx->edr_form != form + 1) continue;
        for (int r : {4, 8, 2}) {
            if (ctx->edr_rows && ctx->edr_rows != r) continue;
            cand[nc++] = r | (form ? kShapeCol : 0);
        }
    }
    if (nc == 1) return launch_shape(ctx, cand[0], src, cap, max_rows, max_cols, u, cells);
    const uint64_t key = ((uint64_t)Src::kKind << 60) | ((uint64_t)(ctx->edr_rows | ctx->edr_form << 4) << 52) |
                         (ceil_log2(cap) << 40) | (ceil_log2(max_rows) << 20) | ceil_log2(max_cols);
    /* worker contexts share their parent's table (one tuning per shape class per device) */
    gat_ctx* tab = ctx->root ? ctx->root : ctx;
    {
        std::lock_guard<std::mutex> lk(tab->tune_mu);
        auto hit = tab->edr_tune.find(key);
        if (hit != tab->edr_tune.end()) {
            const int shape = hit->second;
            return launch_shape(ctx, shape, src, cap, max_rows, max_cols, u, cells);
        }
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        cudaGetLastError();
        return launch_shape(ctx, cand[0], src, cap, max_rows, max_cols, u, cells);
    }
    int best = cand[0], st = GAT_OK;
    float best_ms = 0.f;
    for (int i = 0; i < nc && st == GAT_OK; i++) {
        st = launch_shape(ctx, cand[i], src, cap, max_rows, max_cols, u, i == 0 ? cells : nullptr, e0, e1);
        if (st != GAT_OK) break;
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            st = cuda_fail(ctx, cudaGetLastError(), "edr autotune");
            break;
        }
        if (i == 0 || ms < best_ms) {
            best_ms = ms;
            best = cand[i];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st == GAT_OK) {
        std::lock_guard<std::mutex> lk(tab->tune_mu);
        tab->edr_tune[key] = best;
    }
    return st;
}

}  // namespace edr
}  // namespace gat
