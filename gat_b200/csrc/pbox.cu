/* Point boxes: the exact bounding box of the points under each quadtree node of a Grid, or in
 * each leaf of a STIG, from the index's own point arrays (min / max of the float coordinates;
 * a NaN coordinate makes the box NaN, which no containment test passes). When a box lies inside
 * a query rectangle under MBB::pInBox's inclusive comparisons, every point of that range is a
 * hit, so the scan can take the range's trajectory ids without testing a coordinate (range.cu).
 * The boxes depend only on the built arrays, so both builders and a loaded snapshot get the
 * same ones; they are not part of the snapshot format. */
#include <algorithm>

#include "internal.h"

namespace gat {
namespace {

__device__ __forceinline__ float4 empty_box() {
    return make_float4(__int_as_float(0x7f800000), __int_as_float(0x7f800000), __int_as_float(0xff800000),
                       __int_as_float(0xff800000));
}

__device__ __forceinline__ bool box_nan(const float4& b) { return b.x != b.x || b.y != b.y || b.z != b.z || b.w != b.w; }

/* union of two boxes; NaN if either is */
__device__ __forceinline__ float4 box_union(const float4& a, const float4& b) {
    if (box_nan(a) || box_nan(b)) return make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, 0.f);
    return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w));
}

/* a warp per node: the box of points [beg, end) for the nodes `take` selects, else the empty box */
template <class Range>
__global__ void k_node_points_box(int nnodes, Range range, const float* __restrict__ X, const float* __restrict__ Y,
                                  float4* out) {
    const int lane = threadIdx.x & 31;
    const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t nd = w0; nd < nnodes; nd += nw) {
        int b = 0, e = 0;
        float4 box = empty_box();
        if (range((int)nd, b, e)) {
            bool nan = false;
            for (int i = b + lane; i < e; i += 32) {
                const float x = X[i], y = Y[i];
                nan |= (x != x) || (y != y);
                box.x = fminf(box.x, x);
                box.y = fminf(box.y, y);
                box.z = fmaxf(box.z, x);
                box.w = fmaxf(box.w, y);
            }
            for (int o = 16; o > 0; o >>= 1) {
                box.x = fminf(box.x, __shfl_xor_sync(0xffffffffu, box.x, o));
                box.y = fminf(box.y, __shfl_xor_sync(0xffffffffu, box.y, o));
                box.z = fmaxf(box.z, __shfl_xor_sync(0xffffffffu, box.z, o));
                box.w = fmaxf(box.w, __shfl_xor_sync(0xffffffffu, box.w, o));
            }
            if (__any_sync(0xffffffffu, nan)) box = make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, 0.f);
        }
        if (lane == 0) out[nd] = box;
    }
}

/* Grid leaves: node_child < 0, points [pbeg, pend) */
struct GridLeaves {
    const int32_t* child;
    const int32_t* pbeg;
    const int32_t* pend;
    __device__ bool operator()(int nd, int& b, int& e) const {
        if (child[nd] >= 0) return false;
        b = pbeg[nd];
        e = pend[nd];
        return true;
    }
};

/* STIG leaves: kind 1, points [lo, hi] */
struct StigLeaves {
    const int32_t* kind;
    const int32_t* lo;
    const int32_t* hi;
    __device__ bool operator()(int nd, int& b, int& e) const {
        if (!kind[nd]) return false;
        b = lo[nd];
        e = hi[nd] + 1;
        return true;
    }
};

/* one round of internal Grid nodes from their four children; after as many rounds as the tree
 * has levels every internal node holds the union of its leaves (a round reads either a child's
 * value before or after that round's update, and both only grow towards the final box) */
__global__ void k_inner_boxes(int nnodes, const int32_t* __restrict__ child, float4* box) {
    for (int64_t nd = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; nd < nnodes; nd += (int64_t)gridDim.x * blockDim.x) {
        const int c = child[nd];
        if (c < 0) continue;
        float4 u = box_union(box_union(box[c], box[c + 1]), box_union(box[c + 2], box[c + 3]));
        box[nd] = u;
    }
}

int blocks_for(const gat_ctx* ctx, int64_t threads) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((threads + 255) / 256, (int64_t)ctx->sm_count * 16));
}

}  // namespace

int index_point_boxes(gat_index* ix) {
    gat_ctx* ctx = ix->ctx;
    if (ctx->device < 0 || (ix->kind != GAT_INDEX_GRID && ix->kind != GAT_INDEX_STIG)) return GAT_OK;
    const int nn = ix->kind == GAT_INDEX_GRID ? ix->grid.nnodes : ix->stig.nnodes;
    if (nn <= 0) return GAT_OK;
    cudaStream_t s = ctx->stream;
    if (ix->d_pbox) {
        cudaStreamSynchronize(s);
        cudaFree(ix->d_pbox);
        ix->d_pbox = nullptr;
    }
    GAT_CUDA_TRY(ctx, cudaMalloc(&ix->d_pbox, (size_t)nn * sizeof(float4)), "point boxes");
    ix->device_bytes += (size_t)nn * sizeof(float4);
    const int wb = blocks_for(ctx, (int64_t)nn * 32);
    if (ix->kind == GAT_INDEX_GRID) {
        const GridDev& g = ix->grid;
        k_node_points_box<<<wb, 256, 0, s>>>(nn, GridLeaves{g.node_child, g.node_pbeg, g.node_pend}, ix->d_x, ix->d_y,
                                             ix->d_pbox);
        for (int r = 0; r <= g.total_level + 1; r++) k_inner_boxes<<<blocks_for(ctx, nn), 256, 0, s>>>(nn, g.node_child, ix->d_pbox);
        count_launch(ctx, g.total_level + 3);
        ix->grid.node_pbox = ix->d_pbox;
    } else {
        const StigDev& d = ix->stig;
        k_node_points_box<<<wb, 256, 0, s>>>(nn, StigLeaves{d.kind, d.lo, d.hi}, ix->d_x, ix->d_y, ix->d_pbox);
        count_launch(ctx);
        ix->stig.pbox = ix->d_pbox;
    }
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "point boxes");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "point boxes");
    return GAT_OK;
}

}  // namespace gat
