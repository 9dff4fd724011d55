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
 * Mapping: one warp per pair (persistent, pairs taken from an atomic counter). Lane L owns R
 * consecutive rows of a 32*R-row tile and handles column j = s - L at step s, so a step
 * advances 32*R cells of one anti-diagonal band. The value below a lane's last row moves to
 * the next lane with one shuffle per step; columns are staged 32 at a time in a per-warp
 * shared-memory ring that every lane reads; tiles of 32*R rows run one after another and
 * hand their bottom row to the next tile through a double-buffered carry row in global
 * memory (L2-resident). Everything is int32 arithmetic plus two float subtractions per cell.
 */
#pragma once
#include <algorithm>

#include "internal.h"

namespace gat {
namespace edr {

constexpr int kWarps = 8;
constexpr int kBig = 1 << 29; /* above any distance; up + 1 never overflows against it */

/* Pair source over (a_off, a_len, b_off, b_len) arrays; results to out[p]. */
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
    __device__ int count() const { return d_npairs ? *d_npairs : npairs; }
    __device__ void get(int p, const float2*& a, int& la, const float2*& b, int& lb, int32_t*& o) const {
        a = A + a_off[p];
        la = a_len[p];
        b = B + b_off[p];
        lb = b_len[p];
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
 * carry row in L2 as tile t-1 publishes it, 32 columns at a time (release/acquire on a
 * per-tile progress word). Pairs with one tile, and pairs beyond the cooperative pool, are one
 * item that a single warp walks tile by tile with its own carry rows. Waits are bounded:
 * after kSpinLimit polls the warp raises GAT_ERR_TIMEOUT in the status word and abandons the
 * pair (its result becomes -1). Every warp of the persistent grid is resident and items are
 * taken in increasing order, so the producer of any tile a warp waits for is already running. */
constexpr int kSpinLimit = 1 << 22;

struct TileCtl {
    const int64_t* item_pre; /* exclusive prefix of items per pair, item_pre[count] = total */
    int* prog;               /* progress word per cooperative item (zeroed per launch) */
    int* pair_carry;         /* cooperative pair p: rows pair_carry + p * 2 * stride */
    int coop_cap;            /* pairs with index >= coop_cap run on one warp */
    int* warp_carry;         /* per-warp double carry rows for single-warp pairs */
    int stride;
    int32_t* flag;
};

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <int R, class Src>
__global__ void k_edr_prep(Src src, int cap, int coop_cap, int64_t* items) {
    const int n = src.count();
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < cap; p += gridDim.x * blockDim.x) {
        int64_t it = 0;
        if (p < n) {
            const float2 *a, *b;
            int la, lb;
            int32_t* o;
            src.get(p, a, la, b, lb, o);
            int len1 = min(la, lb);
            int T = len1 <= 0 ? 1 : (len1 + 32 * R - 1) / (32 * R);
            it = (T >= 2 && p < coop_cap) ? T : 1;
        }
        items[p] = it;
    }
}

/* One row tile of one pair (rows r0 = t * 32R ...). cin: the bottom row of tile t-1
 * (nullptr for t == 0), cout: this tile's bottom row for tile t+1 (nullptr for the last tile);
 * prog_in/prog_out: progress words when the neighbouring tile runs on another warp. Returns
 * false when a wait gave up. The owner lane of the pair's last row leaves the distance in
 * `result`. */
template <int R>
__device__ __forceinline__ bool edr_tile(const float2* __restrict__ rows, const float2* __restrict__ cols, int len1,
                                         int len2, int t, const int* cin, int* cout, const int* prog_in,
                                         int* prog_out, float u, float2* bring, int* cring, int& result) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    constexpr int kTile = 32 * R;
    const int last_row = len1 - 1;
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
            if (prog_in && s < len2) {
                int ok = 1;
                if (lane == 0) {
                    const int need = min(s + 32, len2);
                    int polls = 0;
                    while (ld_acquire(prog_in) < need) {
                        if (++polls > kSpinLimit) {
                            ok = 0;
                            break;
                        }
                        __nanosleep(64);
                    }
                }
                if (!__shfl_sync(FULL, ok, 0)) return false;
            }
            int c = s + lane;
            if (c < len2) {
                bring[c & 63] = cols[c];
                cring[c & 63] = cin ? __ldcg(cin + c + 1) : c + 1;
            }
            __syncwarp();
        }
        const int from_above = __shfl_up_sync(FULL, bottom, 1);
        const int j = s - lane;
        if (j >= 0 && j < len2) {
            const float2 b = bring[j & 63];
            const int upf = lane == 0 ? cring[j & 63] : from_above;
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
            if (cout && lane == 31) {
                cout[j + 1] = bottom;
                if (prog_out && (((j + 1) & 31) == 0 || j + 1 == len2)) st_release(prog_out, j + 1);
            }
            if (owns_last && j == len2 - 1) {
#pragma unroll
                for (int i = 0; i < R; i++)
                    if (i == last_i) result = left[i];
            }
        }
    }
    __syncwarp();
    return true;
}

template <int R, class Src>
__global__ void __launch_bounds__(kWarps * 32) k_edr_tiles(Src src, float u, TileCtl ctl, unsigned* __restrict__ work,
                                                           unsigned long long* __restrict__ cells) {
    __shared__ float2 bring[kWarps][64];
    __shared__ int cring[kWarps][64];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gw = blockIdx.x * kWarps + wib;
    int* wc0 = ctl.warp_carry + (size_t)gw * 2 * ctl.stride;
    int* wc1 = wc0 + ctl.stride;
    const int n = src.count();
    /* without an item prefix every pair is one item (no pair spans two tiles) */
    const int64_t total = ctl.item_pre ? ctl.item_pre[n] : (int64_t)n;
    for (;;) {
        unsigned item = 0;
        if (lane == 0) item = atomicAdd(work, 1u);
        item = __shfl_sync(FULL, item, 0);
        if ((int64_t)item >= total) break;
        int p = (int)item, t0 = 0, nitems = 1;
        if (ctl.item_pre) {
            int lo = 0, hi = n - 1; /* last pair whose first item is <= item */
            while (lo < hi) {
                int mid = (lo + hi + 1) >> 1;
                if (ctl.item_pre[mid] <= (int64_t)item)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            p = lo;
            t0 = (int)((int64_t)item - ctl.item_pre[p]);
            nitems = (int)(ctl.item_pre[p + 1] - ctl.item_pre[p]);
        }
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
        constexpr int kTile = 32 * R;
        const int T = (len1 + kTile - 1) / kTile;
        int result = 0;
        bool ok = true, finished = false;
        if (nitems == 1) {
            for (int t = 0; t < T && ok; t++)
                ok = edr_tile<R>(rows, cols, len1, len2, t, t > 0 ? ((t - 1) & 1 ? wc1 : wc0) : nullptr,
                                 t + 1 < T ? ((t & 1) ? wc1 : wc0) : nullptr, nullptr, nullptr, u, bring[wib], cring[wib],
                                 result);
            finished = true;
        } else {
            const int t = t0;
            int* pc = ctl.pair_carry + (size_t)p * 2 * ctl.stride;
            const int64_t base = ctl.item_pre ? ctl.item_pre[p] : p;
            ok = edr_tile<R>(rows, cols, len1, len2, t, t > 0 ? pc + ((t - 1) & 1) * ctl.stride : nullptr,
                             t + 1 < T ? pc + (t & 1) * ctl.stride : nullptr, t > 0 ? ctl.prog + base + t - 1 : nullptr,
                             t + 1 < T ? ctl.prog + base + t : nullptr, u, bring[wib], cring[wib], result);
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
            const int owner = ((len1 - 1) % kTile) / R;
            result = __shfl_sync(FULL, result, owner);
            if (lane == 0) {
                *outp = result;
                if (cells) atomicAdd(cells, (unsigned long long)len1 * (unsigned long long)len2);
            }
        }
    }
}

/* Host side: prep (items per pair) -> scan -> tiled kernel. cap bounds the pair count (exact
 * for host-known lists, an upper bound for device-counted ones); max_rows / max_cols bound the
 * shorter / longer side of every pair. */
template <int R, class Src>
int launch_tiles(gat_ctx* ctx, const Src& src, int64_t cap, int max_rows, int max_cols, float u,
                 unsigned long long* cells) {
    int st = GAT_OK;
    cudaStream_t s = ctx->stream;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_edr_tiles<R, Src>, kWarps * 32, 0);
    const int grid = ctx->sm_count * (per_sm > 0 ? per_sm : 1);
    const int stride = max_cols + 2;
    const int maxT = max_rows <= 0 ? 1 : (max_rows + 32 * R - 1) / (32 * R);
    const size_t budget = (size_t)512 << 20; /* cooperative carry rows */
    int64_t coop = (int64_t)(budget / ((size_t)2 * stride * sizeof(int)));
    if (coop > cap) coop = cap;
    if (maxT < 2) coop = 0;
    int64_t* items = coop > 0 ? (int64_t*)scratch(ctx, S_EDR_ITEMS, (size_t)(cap + 1) * 8, &st) : nullptr;
    int* prog = coop > 0 ? (int*)scratch(ctx, S_EDR_PROG, (size_t)coop * maxT * 4, &st) : nullptr;
    int* pcarry = coop > 0 ? (int*)scratch(ctx, S_EDR_PCARRY, (size_t)coop * 2 * stride * 4, &st) : nullptr;
    int* wcarry = (int*)scratch(ctx, S_EDR_CARRY, (size_t)grid * kWarps * 2 * stride * 4, &st);
    unsigned* work = (unsigned*)scratch(ctx, S_EDR_COUNTERS, 64, &st);
    if (!wcarry || !work || (coop > 0 && (!items || !prog || !pcarry))) return st;
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(work, 0, sizeof(unsigned), s), "edr");
    if (coop > 0) {
        /* items per pair and their prefix; skipped when no pair spans two tiles */
        GAT_CUDA_TRY(ctx, cudaMemsetAsync(prog, 0, (size_t)coop * maxT * 4, s), "edr");
        int pgrid = (int)std::min<int64_t>((cap + 255) / 256, (int64_t)ctx->sm_count * 16);
        k_edr_prep<R, Src><<<pgrid > 0 ? pgrid : 1, 256, 0, s>>>(src, (int)cap, (int)coop, items);
        count_launch(ctx);
        if ((st = scan_i64(ctx, items, items, cap)) != GAT_OK) return st;
    }
    TileCtl ctl{items, prog, pcarry, (int)coop, wcarry, stride, ctx->d_flag};
    timed_begin(ctx, GAT_KERNEL_EDR);
    k_edr_tiles<R, Src><<<grid, kWarps * 32, 0, s>>>(src, u, ctl, work, cells);
    timed_end(ctx, GAT_KERNEL_EDR, 0.0);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "edr launch");
    return GAT_OK;
}

template <class Src>
int edr_launch(gat_ctx* ctx, const Src& src, int64_t cap, int max_rows, int max_cols, float u,
               unsigned long long* cells) {
    if (cap <= 0) return GAT_OK;
    return max_rows <= 128 ? launch_tiles<4, Src>(ctx, src, cap, max_rows, max_cols, u, cells)
                           : launch_tiles<8, Src>(ctx, src, cap, max_rows, max_cols, u, cells);
}

}  // namespace edr
}  // namespace gat
