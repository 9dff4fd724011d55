/* MortonGrid (MortonGrid.h:27, MortonGrid.cpp): the GT-quadtree kept as an implicit tree.
 *
 * The reference's MortonGrid holds the same cells, point order and quadtree as the Grid, but
 * without node objects: a bitmap marks the leaves by node id (level, id), bit
 * (4^level - 1) / 3 + id (findIdxInBitmap, MortonGrid.cpp:8-13), and a node's box is computed
 * from its first and last Morton cells when the walk needs it (generateMBBfromNode,
 * MortonGrid.cpp:261-265). Both builders take a node as a leaf under the same rule (fewer than
 * MAXPOINTINNODE points, or the last level: Grid.cpp:58-94, MortonGrid.cpp:238-259), so the leaves
 * are the Grid's and so are the query results; what differs is how the candidate stage walks the
 * tree (computed boxes and bitmap probes instead of node loads).
 *
 * The device build reads a built Grid: the first point of every Morton cell from the Grid's
 * point order (each point's cell in the Grid builder's float expressions; the points are in cell
 * order), and the leaf bitmap from the Grid's breadth-first node arrays (a node's (level, id)
 * from its path of child positions up to the root). The Grid's point arrays are shared, not
 * copied. */
#include <algorithm>

#include "cells.cuh"
#include "internal.h"

namespace gat {
namespace {

constexpr int kMaxMortonLevel = 13; /* 4^13 cells; stack entries pack (id << 4) | level */

int grid_blocks(const gat_ctx* ctx, int64_t n) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)ctx->sm_count * 16));
}

/* cbeg[c] = the first point (in the Grid's order) whose cell is at least c, c = 0..ncells */
__global__ void k_cell_starts(int64_t P, const float* __restrict__ X, const float* __restrict__ Y, CellParams cp,
                              int64_t ncells, int32_t* cbeg) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= P; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = i < P ? point_cell(cp, __ldg(X + i), __ldg(Y + i)) : ncells;
        const int64_t prev = i > 0 ? point_cell(cp, __ldg(X + i - 1), __ldg(Y + i - 1)) : -1;
        for (int64_t k = prev + 1; k <= c; k++) cbeg[k] = (int32_t)i;
    }
}

/* parent of every node of the breadth-first tree (children of j at child[j] .. child[j] + 3) */
__global__ void k_parents(int nnodes, const int32_t* __restrict__ child, int32_t* parent) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nnodes; j += gridDim.x * blockDim.x) {
        if (j == 0) parent[0] = -1;
        const int ch = child[j];
        if (ch >= 0)
            for (int c = 0; c < 4; c++) parent[ch + c] = j;
    }
}

/* every leaf's bit at (4^level - 1) / 3 + id: its id digits are its child positions on the path
 * from the root (UL, UR, DL, DR = 0..3, MortonGrid.cpp:249-254) */
__global__ void k_leaf_bits(int nnodes, const int32_t* __restrict__ child, const int32_t* __restrict__ parent,
                            uint32_t* bits) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nnodes; j += gridDim.x * blockDim.x) {
        if (child[j] >= 0) continue;
        int level = 0;
        uint64_t id = 0, mul = 1;
        for (int k = j; parent[k] >= 0; k = parent[k]) {
            id += (uint64_t)(k - child[parent[k]]) * mul;
            mul <<= 2;
            level++;
        }
        const uint64_t idx = (((uint64_t)1 << (2 * level)) - 1) / 3 + id;
        atomicOr(bits + (idx >> 5), 1u << (idx & 31));
    }
}

}  // namespace
}  // namespace gat

using namespace gat;

extern "C" {

int gat_morton_grid_build(gat_ctx* ctx, const gat_index* grid, gat_index** out) {
    if (!ctx || !grid || !out) return fail(ctx, GAT_ERR_ARG, "gat_morton_grid_build: bad arguments");
    if (grid->kind != GAT_INDEX_GRID) return fail(ctx, GAT_ERR_ARG, "gat_morton_grid_build: not a Grid index");
    if (!same_owner(grid->ctx, ctx)) return fail(ctx, GAT_ERR_STATE, "gat_morton_grid_build: index from another context");
    if (int rq = require_device(ctx, "gat_morton_grid_build")) return rq;
    const GridDev& g = grid->grid;
    if (g.total_level > kMaxMortonLevel || g.total_level < 0)
        return fail(ctx, GAT_ERR_ARG, "gat_morton_grid_build: more than 4^13 cells");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    gat_index* ix = new gat_index();
    ix->ctx = ctx;
    ix->db = grid->db;
    ix->kind = GAT_INDEX_MORTON;
    ix->base = grid;
    ix->npoints = grid->npoints;
    ix->pidx_bits = grid->pidx_bits;
    ix->d_x = grid->d_x;
    ix->d_y = grid->d_y;
    ix->d_key = grid->d_key;
    ix->d_tid = grid->d_tid;
    ix->leaves = grid->leaves;
    ix->nodes = grid->nodes;
    ix->grid = g;
    int st = GAT_OK;
    const int64_t ncells = (int64_t)g.axis * g.axis;
    const uint64_t nbits = (((uint64_t)1 << (2 * (g.total_level + 1))) - 1) / 3;
    const size_t words = (size_t)((nbits + 31) / 32);
    auto* cbeg = (int32_t*)index_alloc(ix, (size_t)(ncells + 1) * sizeof(int32_t), &st);
    auto* bits = cbeg ? (uint32_t*)index_alloc(ix, words * sizeof(uint32_t), &st) : nullptr;
    int32_t* parent = nullptr;
    if (bits && cudaMalloc(&parent, (size_t)std::max(1, g.nnodes) * sizeof(int32_t)) != cudaSuccess) {
        cudaGetLastError();
        st = fail(ctx, GAT_ERR_OOM, "gat_morton_grid_build: allocation");
    }
    if (st != GAT_OK) {
        gat_index_destroy(ix);
        return st;
    }
    ix->morton = MortonDev{g.rxmin, g.rymax, g.cell, g.total_level, bits, cbeg};
    CellParams cp{g.rxmin, g.rymax, g.cell, 1, g.axis, 0, 0, g.vparam};
    cudaError_t e = cudaMemsetAsync(bits, 0, words * sizeof(uint32_t), s);
    if (e == cudaSuccess) {
        k_cell_starts<<<grid_blocks(ctx, ix->npoints + 1), 256, 0, s>>>(ix->npoints, ix->d_x, ix->d_y, cp, ncells, cbeg);
        k_parents<<<grid_blocks(ctx, g.nnodes), 256, 0, s>>>(g.nnodes, g.node_child, parent);
        k_leaf_bits<<<grid_blocks(ctx, g.nnodes), 256, 0, s>>>(g.nnodes, g.node_child, parent, bits);
        count_launch(ctx, 3);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(parent);
    if (e != cudaSuccess) {
        st = cuda_fail(ctx, e, "gat_morton_grid_build");
        gat_index_destroy(ix);
        return st;
    }
    *out = ix;
    return GAT_OK;
}

int gat_morton_grid_leaves(gat_ctx* ctx, const gat_index* ix, int32_t* level, int32_t* id, int64_t capacity,
                           int64_t* count) {
    if (!ctx || !ix || !count || capacity < 0 || (capacity > 0 && (!level || !id)))
        return fail(ctx, GAT_ERR_ARG, "gat_morton_grid_leaves: bad arguments");
    if (ix->kind != GAT_INDEX_MORTON) return fail(ctx, GAT_ERR_ARG, "gat_morton_grid_leaves: not a MortonGrid");
    if (!same_owner(ix->ctx, ctx)) return fail(ctx, GAT_ERR_STATE, "gat_morton_grid_leaves: index from another context");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    const int L = ix->morton.total_level;
    const uint64_t nbits = (((uint64_t)1 << (2 * (L + 1))) - 1) / 3;
    std::vector<uint32_t> bits((size_t)((nbits + 31) / 32));
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(bits.data(), ix->morton.leaf, bits.size() * 4, cudaMemcpyDeviceToHost, ctx->stream),
                 "gat_morton_grid_leaves");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "gat_morton_grid_leaves");
    int64_t n = 0;
    int lv = 0;
    uint64_t first = 0, next = 1; /* bits [first, next) belong to level lv */
    for (uint64_t b = 0; b < nbits; b++) {
        while (b >= next) {
            lv++;
            first = next;
            next += (uint64_t)1 << (2 * lv);
        }
        if (!((bits[b >> 5] >> (b & 31)) & 1u)) continue;
        if (n < capacity) {
            level[n] = lv;
            id[n] = (int32_t)(b - first);
        }
        n++;
    }
    *count = n;
    return n > capacity ? fail(ctx, GAT_ERR_TRUNCATED, "gat_morton_grid_leaves: capacity too small") : GAT_OK;
}

}  // extern "C"
