/* Merging per-shard top-k lists into the global top-k, for a trajectory set split across GPUs by
 * contiguous id ranges (each shard holds trajectories lo..hi-1 and reports global ids).
 *
 * The reference splits queries, not the set, between its two GPUs (Grid.cpp:1758-2332); a set
 * split needs one exchange of k (distance, id) pairs per query and shard, then this merge.
 * Each shard's list is sorted by (distance, id), the canonical order of gat_topk, and holds that
 * shard's k best; the global k best are among their union, so the k smallest (distance, id)
 * keys of the union are exactly the unsharded result. Entries with id < 0 (a shard with fewer
 * than k trajectories) are padding: they sort last and are emitted as (-1, -1), as gat_topk
 * emits them. */
#include <algorithm>

#include "internal.h"

namespace gat {
namespace {

constexpr int kMergeThreads = 256;
constexpr int kMergeMax = 8192; /* nparts x k entries one block sorts in shared memory */

__device__ __forceinline__ unsigned long long merge_key(int32_t id, int32_t dist) {
    return id < 0 ? ~0ull : ((unsigned long long)(uint32_t)dist << 32) | (uint32_t)id;
}

/* one block per query: the nparts x k entries sorted in shared memory (bitonic), first k out */
__global__ void __launch_bounds__(kMergeThreads) k_topk_merge(int nq, int k, int nparts, const int32_t* __restrict__ ids,
                                                             const int32_t* __restrict__ dist, int32_t* out_ids,
                                                             int32_t* out_dist) {
    extern __shared__ unsigned long long keys[];
    const int q = blockIdx.x;
    const int m = nparts * k;
    int p2 = 1;
    while (p2 < m) p2 <<= 1;
    for (int i = threadIdx.x; i < p2; i += blockDim.x) {
        unsigned long long key = ~0ull;
        if (i < m) {
            const int part = i / k, j = i - part * k;
            const size_t at = ((size_t)part * nq + q) * k + j;
            key = merge_key(ids[at], dist[at]);
        }
        keys[i] = key;
    }
    __syncthreads();
    for (int kk = 2; kk <= p2; kk <<= 1)
        for (int j = kk >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < p2; i += blockDim.x) {
                const int ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long a = keys[i], b = keys[ixj];
                    const bool up = (i & kk) == 0;
                    if ((a > b) == up) {
                        keys[i] = b;
                        keys[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const unsigned long long key = keys[i];
        const bool pad = key == ~0ull;
        out_ids[(size_t)q * k + i] = pad ? -1 : (int32_t)(key & 0xffffffffull);
        out_dist[(size_t)q * k + i] = pad ? -1 : (int32_t)(key >> 32);
    }
}

bool merge_args_ok(int nq, int k, int nparts) {
    return nq >= 0 && k >= 1 && k <= 1024 && nparts >= 1 && (int64_t)nparts * k <= kMergeMax;
}

}  // namespace
}  // namespace gat

using namespace gat;

extern "C" {

int gat_topk_merge(int nq, int k, int nparts, const int32_t* ids, const int32_t* dist, int32_t* out_ids,
                   int32_t* out_dist) {
    if (!merge_args_ok(nq, k, nparts) || (nq > 0 && (!ids || !dist || !out_ids || !out_dist))) return GAT_ERR_ARG;
    std::vector<unsigned long long> keys((size_t)nparts * k);
    for (int q = 0; q < nq; q++) {
        for (int p = 0; p < nparts; p++)
            for (int j = 0; j < k; j++) {
                const size_t at = ((size_t)p * nq + q) * k + j;
                keys[(size_t)p * k + j] =
                    ids[at] < 0 ? ~0ull : ((unsigned long long)(uint32_t)dist[at] << 32) | (uint32_t)ids[at];
            }
        std::partial_sort(keys.begin(), keys.begin() + k, keys.end());
        for (int j = 0; j < k; j++) {
            const bool pad = keys[(size_t)j] == ~0ull;
            out_ids[(size_t)q * k + j] = pad ? -1 : (int32_t)(keys[(size_t)j] & 0xffffffffull);
            out_dist[(size_t)q * k + j] = pad ? -1 : (int32_t)(keys[(size_t)j] >> 32);
        }
    }
    return GAT_OK;
}

int gat_topk_merge_dev(gat_ctx* ctx, int nq, int k, int nparts, const int32_t* d_ids, const int32_t* d_dist,
                       int32_t* d_out_ids, int32_t* d_out_dist) {
    if (!ctx || !merge_args_ok(nq, k, nparts) || (nq > 0 && (!d_ids || !d_dist || !d_out_ids || !d_out_dist)))
        return fail(ctx, GAT_ERR_ARG, "gat_topk_merge_dev: bad arguments (nparts x k at most 8192)");
    if (nq == 0) return GAT_OK;
    if (int rq = require_device(ctx, "gat_topk_merge_dev")) return rq;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    int p2 = 1;
    while (p2 < nparts * k) p2 <<= 1;
    const size_t smem = (size_t)p2 * 8;
    allow_smem(k_topk_merge, smem);
    k_topk_merge<<<nq, kMergeThreads, smem, ctx->stream>>>(nq, k, nparts, d_ids, d_dist, d_out_ids, d_out_dist);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "gat_topk_merge_dev");
    return GAT_OK;
}

}  // extern "C"
