/* EDR of (query, candidate) pair lists: the C ABI entry points over the wavefront kernel of
 * edr_kernel.cuh. */
#include <algorithm>

#include "edr_kernel.cuh"
#include "internal.h"

namespace gat {
using edr::SoaPairs;

/* Launch over pairs given as (a_off, a_len, b_off, b_len) arrays. max_rows / max_cols bound
 * the shorter / longer side of every pair. */
int edr_launch_soa(gat_ctx* ctx, int npairs, const int* d_npairs, const int64_t* a_off, const int32_t* a_len,
                   const int64_t* b_off, const int32_t* b_len, int max_rows, int max_cols, const float2* A,
                   const float2* B, float u, int32_t* d_out, unsigned long long* d_cells) {
    if (npairs <= 0) return GAT_OK;
    SoaPairs src{npairs, d_npairs, a_off, a_len, b_off, b_len, A, B, d_out, std::max(max_rows, max_cols), ctx->d_flag};
    return edr::edr_launch(ctx, src, npairs, max_rows, max_cols, u, d_cells);
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
    if ((st = check_device_flag(ctx, "edr")) != GAT_OK) return st;
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
    return check_device_flag(ctx, "edr");
}

}  // extern "C"
