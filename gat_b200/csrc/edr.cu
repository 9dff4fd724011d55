/* EDR distance of (query, candidate) pairs: an anti-diagonal wavefront inside one warp.
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
#include <algorithm>

#include "internal.h"

namespace gat {
namespace {

constexpr int kWarps = 8;

template <int R>
__global__ void __launch_bounds__(kWarps * 32) k_edr(int npairs, const int* __restrict__ d_npairs,
                                                     const int64_t* __restrict__ a_off, const int32_t* __restrict__ a_len,
                                                     const int64_t* __restrict__ b_off, const int32_t* __restrict__ b_len,
                                                     const float2* __restrict__ A, const float2* __restrict__ B, float u,
                                                     int32_t* __restrict__ out, int* __restrict__ carry, int carry_stride,
                                                     unsigned* __restrict__ work, unsigned long long* __restrict__ cells) {
    __shared__ float2 bring[kWarps][64];
    __shared__ int cring[kWarps][64];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gw = blockIdx.x * kWarps + wib;
    int* cbuf0 = carry + (size_t)gw * 2 * carry_stride;
    int* cbuf1 = cbuf0 + carry_stride;
    const int n = d_npairs ? *d_npairs : npairs;
    for (;;) {
        unsigned p = 0;
        if (lane == 0) p = atomicAdd(work, 1u);
        p = __shfl_sync(FULL, p, 0);
        if ((int)p >= n) break;
        const int la = a_len[p], lb = b_len[p];
        const float2* rows;
        const float2* cols;
        int len1, len2;
        if (lb >= la) {
            rows = A + a_off[p];
            cols = B + b_off[p];
            len1 = la;
            len2 = lb;
        } else {
            rows = B + b_off[p];
            cols = A + a_off[p];
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
                        int up = upf, diag = diag_in;
#pragma unroll
                        for (int i = 0; i < R; i++) {
                            const bool match = (fabsf(__fsub_rn(ax[i], b.x)) < u) & (fabsf(__fsub_rn(ay[i], b.y)) < u);
                            const int m = diag + (match ? 0 : 1);
                            const int uu = up + 1;
                            const int l = left[i] + 1;
                            const int d = (m == l) ? uu : min(m, min(uu, l));
                            diag = left[i];
                            left[i] = d;
                            up = d;
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
            out[p] = result;
            if (cells) atomicAdd(cells, (unsigned long long)len1 * (unsigned long long)len2);
        }
    }
}

}  // namespace

/* Launch over pairs given as (a_off, a_len, b_off, b_len) arrays. max_cols bounds the longer
 * side of every pair (sizes the carry rows); rows_hint picks the tile height. */
int edr_launch_soa(gat_ctx* ctx, int npairs, const int* d_npairs, const int64_t* a_off, const int32_t* a_len,
                   const int64_t* b_off, const int32_t* b_len, int rows_hint, int max_cols, const float2* A,
                   const float2* B, float u, int32_t* d_out, unsigned long long* d_cells) {
    if (npairs <= 0 && !d_npairs) return GAT_OK;
    int st = GAT_OK;
    const int R = rows_hint <= 128 ? 4 : 8;
    int per_sm = 0;
    if (R == 4)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_edr<4>, kWarps * 32, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_edr<8>, kWarps * 32, 0);
    per_sm = std::max(1, per_sm);
    int grid = ctx->sm_count * per_sm;
    if (!d_npairs) grid = std::max(1, std::min(grid, (npairs + kWarps - 1) / kWarps));
    int stride = max_cols + 2;
    int* carry = (int*)scratch(ctx, S_EDR_CARRY, (size_t)grid * kWarps * 2 * stride * sizeof(int), &st);
    unsigned* work = (unsigned*)scratch(ctx, S_EDR_COUNTERS, 64, &st);
    if (!carry || !work) return st;
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(work, 0, sizeof(unsigned), ctx->stream), "edr");
    timed_begin(ctx, GAT_KERNEL_EDR);
    if (R == 4)
        k_edr<4><<<grid, kWarps * 32, 0, ctx->stream>>>(npairs, d_npairs, a_off, a_len, b_off, b_len, A, B, u, d_out,
                                                        carry, stride, work, d_cells);
    else
        k_edr<8><<<grid, kWarps * 32, 0, ctx->stream>>>(npairs, d_npairs, a_off, a_len, b_off, b_len, A, B, u, d_out,
                                                        carry, stride, work, d_cells);
    timed_end(ctx, GAT_KERNEL_EDR, 0.0);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "edr launch");
    return GAT_OK;
}

}  // namespace gat

using namespace gat;

namespace {
int check_lengths(gat_ctx* ctx, int npairs, const int32_t* a, const int32_t* b, int* max_rows, int* max_cols) {
    int mr = 0, mc = 0;
    for (int i = 0; i < npairs; i++) {
        if (a[i] < 1 || b[i] < 1 || a[i] > GAT_EDR_MAX_LEN || b[i] > GAT_EDR_MAX_LEN)
            return fail(ctx, GAT_ERR_ARG, "edr: trajectory length outside 1..GAT_EDR_MAX_LEN");
        mr = std::max(mr, std::min(a[i], b[i]));
        mc = std::max(mc, std::max(a[i], b[i]));
    }
    *max_rows = mr;
    *max_cols = mc;
    return GAT_OK;
}
}  // namespace

extern "C" {

int gat_edr_pairs(gat_ctx* ctx, int npairs, const int32_t* q_len, const int64_t* q_off, const float* q_xy,
                  int64_t q_points, const int32_t* c_len, const int64_t* c_off, const float* c_xy, int64_t c_points,
                  double eps, int32_t* out) {
    if (!ctx || npairs < 0 || (npairs > 0 && (!q_len || !q_off || !q_xy || !c_len || !c_off || !c_xy || !out)) ||
        !(eps > 0) || q_points < 0 || c_points < 0)
        return fail(ctx, GAT_ERR_ARG, "gat_edr_pairs: bad arguments");
    if (npairs == 0) return GAT_OK;
    int mr, mc, st;
    if ((st = check_lengths(ctx, npairs, q_len, c_len, &mr, &mc)) != GAT_OK) return st;
    for (int i = 0; i < npairs; i++)
        if (q_off[i] < 0 || q_off[i] + q_len[i] > q_points || c_off[i] < 0 || c_off[i] + c_len[i] > c_points)
            return fail(ctx, GAT_ERR_ARG, "gat_edr_pairs: pair points out of range");
    if (int rq = require_device(ctx, "gat_edr_pairs")) return rq;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    /* one staging buffer: [a_off | b_off | a_len | b_len | out | A | B] */
    size_t n8 = (size_t)npairs * 8, n4 = (size_t)npairs * 4;
    size_t a_bytes = (size_t)q_points * 8, b_bytes = (size_t)c_points * 8;
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t total = up(n8) * 2 + up(n4) * 3 + up(a_bytes) + up(b_bytes);
    char* buf = (char*)scratch(ctx, S_EDR_IO, total, &st);
    if (!buf) return st;
    char* p = buf;
    int64_t* d_aoff = (int64_t*)p; p += up(n8);
    int64_t* d_boff = (int64_t*)p; p += up(n8);
    int32_t* d_alen = (int32_t*)p; p += up(n4);
    int32_t* d_blen = (int32_t*)p; p += up(n4);
    int32_t* d_out = (int32_t*)p; p += up(n4);
    float2* d_a = (float2*)p; p += up(a_bytes);
    float2* d_b = (float2*)p;
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(d_aoff, q_off, n8, cudaMemcpyHostToDevice, s), "edr H2D");
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(d_boff, c_off, n8, cudaMemcpyHostToDevice, s), "edr H2D");
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(d_alen, q_len, n4, cudaMemcpyHostToDevice, s), "edr H2D");
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(d_blen, c_len, n4, cudaMemcpyHostToDevice, s), "edr H2D");
    if (a_bytes) GAT_CUDA_TRY(ctx, cudaMemcpyAsync(d_a, q_xy, a_bytes, cudaMemcpyHostToDevice, s), "edr H2D");
    if (b_bytes) GAT_CUDA_TRY(ctx, cudaMemcpyAsync(d_b, c_xy, b_bytes, cudaMemcpyHostToDevice, s), "edr H2D");
    if ((st = edr_launch_soa(ctx, npairs, nullptr, d_aoff, d_alen, d_boff, d_blen, mr, mc, d_a, d_b,
                             match_threshold(eps), d_out, nullptr)) != GAT_OK)
        return st;
    double cells = 0;
    for (int i = 0; i < npairs; i++) cells += (double)q_len[i] * (double)c_len[i];
    timed_add_work(ctx, GAT_KERNEL_EDR, cells);
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(out, d_out, n4, cudaMemcpyDeviceToHost, s), "edr D2H");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "edr");
    return GAT_OK;
}

int gat_edr_pairs_dev(gat_ctx* ctx, int npairs, const int32_t* d_q_len, const int64_t* d_q_off, const float* d_q_xy,
                      const int32_t* d_c_len, const int64_t* d_c_off, const float* d_c_xy, double eps, int32_t* d_out) {
    if (!ctx || npairs < 0 || (npairs > 0 && (!d_q_len || !d_q_off || !d_q_xy || !d_c_len || !d_c_off || !d_c_xy || !d_out)) ||
        !(eps > 0))
        return fail(ctx, GAT_ERR_ARG, "gat_edr_pairs_dev: bad arguments");
    if (npairs == 0) return GAT_OK;
    if (int rq = require_device(ctx, "gat_edr_pairs_dev")) return rq;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    /* lengths are device-resident; the carry rows are sized for the longest supported side */
    int st = edr_launch_soa(ctx, npairs, nullptr, d_q_off, d_q_len, d_c_off, d_c_len, GAT_EDR_MAX_LEN, GAT_EDR_MAX_LEN,
                            (const float2*)d_q_xy, (const float2*)d_c_xy, match_threshold(eps), d_out, nullptr);
    if (st != GAT_OK) return st;
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "edr");
    return GAT_OK;
}

}  // extern "C"
