/* EDR of (query, candidate) pairs without any allocation: gat_edr_pairs_dev_noalloc.
 *
 * Some callers cannot call cudaMalloc at all: code running inside a CUDA-graph capture they do
 * not own, allocators that forbid it, or host programs that have to keep a fixed device
 * footprint. The regular entry points take their working memory from the context's scratch
 * arena, which grows with cudaMalloc. This one needs no context: the caller passes a stream and
 * device arrays, and the kernel's only working memory (the carry rows that hand the bottom row
 * of one 256-row tile to the next, plus a work counter) lives in the file-scope device array
 * below. Its size is fixed: kMaxLen points per trajectory side, kWarps resident warps.
 *
 * With CUDA's lazy module loading (the default), the first call on a device loads this file's
 * module there, and that reserves the array on that device until the process exits; later calls
 * allocate nothing. Every call uses the same array: calls that overlap on the GPU (on different
 * streams, or from several host threads) race on it and must be serialised by the caller. The
 * work counter is cleared at the start of each call; the carry rows need no clearing (each tile
 * reads only rows its predecessor wrote in the same call).
 */
#include <mutex>

#include "edr_kernel.cuh"
#include "gat_b200.h"

namespace gat {
namespace {

constexpr int kMaxLen = GAT_EDR_NOALLOC_MAX_LEN;
constexpr int kRowsPerLane = 8;
constexpr int kBlocks = 64;
constexpr int kNoAllocWarps = kBlocks * edr::kWarps;
constexpr int kStride = kMaxLen + 2;
constexpr size_t kCarryInts = (size_t)kNoAllocWarps * 2 * kStride;
/* tail words: [0] work counter, [1] sink for rejected pairs, [2..3] a dummy point */
constexpr size_t kTailInts = 64;

static __device__ __align__(256) int g_noalloc_scratch[kCarryInts + kTailInts];

/* Pair source over the caller's arrays. A pair with a side outside 1..max_len gets -1 and is
 * replaced by a 1 x 1 problem on a dummy point whose result goes to the sink word, so the
 * carry rows are never indexed past their fixed size. */
struct NoAllocPairs {
    int npairs;
    int max_len;
    const int64_t* a_off;
    const int32_t* a_len;
    const int64_t* b_off;
    const int32_t* b_len;
    const float2* A;
    const float2* B;
    int32_t* out;
    __device__ int count() const { return npairs; }
    __device__ void get(int p, const float2*& a, int& la, const float2*& b, int& lb, int32_t*& o) const {
        la = a_len[p];
        lb = b_len[p];
        if (la < 1 || lb < 1 || la > max_len || lb > max_len) {
            out[p] = -1;
            a = b = reinterpret_cast<const float2*>(&g_noalloc_scratch[kCarryInts + 2]);
            la = lb = 1;
            o = &g_noalloc_scratch[kCarryInts + 1];
            return;
        }
        a = A + a_off[p];
        b = B + b_off[p];
        o = out + p;
    }
};

std::mutex g_setup_mu;
int* g_scratch_addr[64] = {nullptr};

/* Device address of the scratch array on the current device. Host code cannot use the array's
 * name as an address (it names a host-side shadow), so the address comes from
 * cudaGetSymbolAddress with the device current. Outside a stream capture it is looked up again
 * on every call (cheap), so the address stays right after a cudaDeviceReset or a re-created
 * primary context; inside a capture the address of the last call outside one is used, and a
 * device that has never seen such a call gets GAT_ERR_STATE. */
int scratch_address(cudaStream_t s, int** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return GAT_ERR_CUDA;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
        cudaGetLastError();
        return GAT_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (cs == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return GAT_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<int*>(p);
    }
    if (!g_scratch_addr[dev]) return GAT_ERR_STATE;
    *out = g_scratch_addr[dev];
    return GAT_OK;
}

}  // namespace
}  // namespace gat

using namespace gat;

extern "C" int gat_edr_pairs_dev_noalloc(void* stream, int npairs, int max_len, const int32_t* d_q_len,
                                         const int64_t* d_q_off, const float* d_q_xy, const int32_t* d_c_len,
                                         const int64_t* d_c_off, const float* d_c_xy, double eps, int32_t* d_out) {
    if (npairs < 0 || !(eps > 0)) return GAT_ERR_ARG;
    if (max_len < 1 || max_len > kMaxLen) return GAT_ERR_ARG; /* beyond the fixed scratch */
    if (npairs == 0) return GAT_OK;
    if (!d_q_len || !d_q_off || !d_q_xy || !d_c_len || !d_c_off || !d_c_xy || !d_out) return GAT_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int* scratch = nullptr;
    int rc = scratch_address(s, &scratch);
    if (rc != GAT_OK) return rc;
    unsigned* work = reinterpret_cast<unsigned*>(scratch + kCarryInts);
    if (cudaMemsetAsync(work, 0, sizeof(unsigned), s) != cudaSuccess) {
        cudaGetLastError();
        return GAT_ERR_CUDA;
    }
    NoAllocPairs src{npairs,
                     max_len,
                     d_q_off,
                     d_q_len,
                     d_c_off,
                     d_c_len,
                     reinterpret_cast<const float2*>(d_q_xy),
                     reinterpret_cast<const float2*>(d_c_xy),
                     d_out};
    edr::k_edr<kRowsPerLane, NoAllocPairs><<<kBlocks, edr::kWarps * 32, 0, s>>>(src, match_threshold(eps), scratch,
                                                                               kStride, work, nullptr);
    if (cudaGetLastError() != cudaSuccess) return GAT_ERR_CUDA;
    return GAT_OK;
}
