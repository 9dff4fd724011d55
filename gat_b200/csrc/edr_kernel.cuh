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


}  // namespace edr
}  // namespace gat
