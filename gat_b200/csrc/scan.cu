/* Device-wide exclusive scan of int64 counts (CSR offsets for range items and results). */
#include "internal.h"
#include "launch.cuh"

namespace gat {

__global__ void k_zero_words(int* p, int n) {
    dep_wait();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 0;
}
namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 4; /* per thread */
constexpr int kScanTile = kScanThreads * kScanItems;

/* block-wide exclusive scan of one value per thread; returns the block total in *total */
__device__ int64_t block_exclusive_scan(int64_t v, int64_t* total) {
    __shared__ int64_t warp_sums[kScanThreads / 32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int64_t s = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kScanThreads / 32) warp_sums[lane] = s; /* inclusive */
    }
    __syncthreads();
    int64_t base = warp == 0 ? 0 : warp_sums[warp - 1];
    *total = warp_sums[kScanThreads / 32 - 1];
    __syncthreads();
    return base + x - v;
}

/* out[i] = exclusive prefix of in within the tile; block_sums[b] = tile total */
__global__ void k_scan_tiles(const int64_t* in, int64_t* out, int64_t n, int64_t* block_sums) {
    dep_wait();
    int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int64_t v[kScanItems];
    int64_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    int64_t total;
    int64_t pre = block_exclusive_scan(s, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) out[base + k] = pre;
        pre += v[k];
    }
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void k_scan_add(int64_t* out, int64_t n, const int64_t* block_prefix) {
    dep_wait();
    int64_t base = (int64_t)blockIdx.x * kScanTile;
    int64_t add = block_prefix[blockIdx.x];
    for (int k = threadIdx.x; k < kScanTile; k += blockDim.x)
        if (base + k < n) out[base + k] += add;
}

__global__ void k_scan_total(int64_t* out, int64_t n, const int64_t* in_last, const int64_t* out_last_before) {
    dep_wait();
    /* out[n] = out[n-1] + in[n-1], with both read before out[n-1] changes (captured values) */
    if (threadIdx.x == 0 && blockIdx.x == 0) out[n] = *out_last_before + *in_last;
}

}  // namespace

/* Recursive tile scan. in and out may alias; out must hold n + 1 entries. */
int scan_i64(gat_ctx* ctx, const int64_t* in, int64_t* out, int64_t n) {
    cudaStream_t s = ctx->stream;
    if (n <= 0) {
        (void)launch_dep(ctx, k_zero_words, dim3(1), dim3(32), 0, s, reinterpret_cast<int*>(out), 2);
        return GAT_OK;
    }
    /* levels of block sums: level l holds ceil(n_l / tile) values */
    std::vector<int64_t> level_n;
    int64_t m = n;
    size_t words = 2; /* [0] = last input, [1] = last exclusive output */
    while (m > 1) {
        int64_t b = (m + kScanTile - 1) / kScanTile;
        level_n.push_back(b);
        words += (size_t)b + 1;
        m = b;
    }
    int st = GAT_OK;
    int64_t* tmp = (int64_t*)scratch(ctx, S_SCAN_TMP, words * sizeof(int64_t), &st);
    if (!tmp) return st;
    int64_t* last_in = tmp;
    int64_t* last_out = tmp + 1;
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(last_in, in + (n - 1), sizeof(int64_t), cudaMemcpyDeviceToDevice, s), "scan");
    /* pass down */
    const int64_t* cur_in = in;
    int64_t* cur_out = out;
    int64_t cur_n = n;
    int64_t* next = tmp + 2;
    std::vector<std::pair<int64_t*, int64_t>> outs;
    for (size_t l = 0; l <= level_n.size(); l++) {
        int64_t blocks = (cur_n + kScanTile - 1) / kScanTile;
        int64_t* sums = next;
        next += blocks + 1;
        (void)launch_dep(ctx, k_scan_tiles, dim3((unsigned)blocks), dim3(kScanThreads), 0, s, cur_in, cur_out, cur_n, sums);
        count_launch(ctx);
        outs.push_back({cur_out, cur_n});
        if (blocks == 1) break;
        cur_in = sums;
        cur_out = sums; /* scanned in place at the next level */
        cur_n = blocks;
    }
    /* pass up: add scanned block sums of level l+1 into level l */
    for (int l = (int)outs.size() - 2; l >= 0; l--) {
        int64_t blocks = (outs[l].second + kScanTile - 1) / kScanTile;
        (void)launch_dep(ctx, k_scan_add, dim3((unsigned)blocks), dim3(kScanThreads), 0, s, outs[l].first, outs[l].second, outs[l + 1].first);
        count_launch(ctx);
    }
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(last_out, out + (n - 1), sizeof(int64_t), cudaMemcpyDeviceToDevice, s), "scan");
    (void)launch_dep(ctx, k_scan_total, dim3(1), dim3(32), 0, s, out, n, last_in, last_out);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "scan launch");
    return GAT_OK;
}

}  // namespace gat
