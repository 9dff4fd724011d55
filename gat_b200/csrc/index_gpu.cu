/* Device placement of index points for the Grid and FSG builders (the layouts of
 * Grid::addDatasetToGrid, Grid.cpp:210-316, and FSG::addDatasetToGrid, FSG.cpp:95-143).
 *
 * Both indexes order points by cell, trajectories ascending within a cell and points in
 * trajectory order within a trajectory: a stable sort by cell of the set's points taken in
 * trajectory order. The device computes every point's cell with the builders' float expressions
 * (IEEE single subtract and divide, truncation toward zero), sorts (cell, original position)
 * pairs with a stable LSD radix sort, gathers x / y / trajectory / key in that order, and finds
 * the cell boundaries by binary search over the sorted cells. For the Grid it also forms the
 * frequency vectors: 64-bit (trajectory, virtual cell) keys sorted and run-length counted give
 * each trajectory's (virtual cell, count) list in ascending cell order, which is what merging
 * the runs' (cell >> vparam, count) pairs per trajectory yields (Grid.cpp:152-166).
 *
 * The quadtree stays on the host: it is a walk over the cell boundaries only.
 * The sorts and the run-length encoding are CUB's (the CUDA toolkit's header library); an index
 * build runs once per trajectory set and is not on the query path. */
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_run_length_encode.cuh>

#include "internal.h"

namespace gat {
namespace {

struct CellParams {
    float rxmin, rymax, cell;
    int morton; /* 1: Grid (Morton id on an axis x axis grid), 0: FSG (row-major nx x ny) */
    int axis, nx, ny, vparam;
};

__device__ __forceinline__ uint32_t spread_bits(uint32_t v) {
    v &= 0xFFFF;
    v = (v | (v << 8)) & 0x00FF00FF;
    v = (v | (v << 4)) & 0x0F0F0F0F;
    v = (v | (v << 2)) & 0x33333333;
    v = (v | (v << 1)) & 0x55555555;
    return v;
}

/* float -> int truncation as the host's (int) cast gives it for every value that can land in a
 * grid; NaN and values beyond the int range are reported as outside (the host's conversion of
 * those yields INT_MIN, a negative row or column, hence also outside) */
__device__ __forceinline__ bool trunc_int(float v, int* out) {
    if (!(v > -2147483648.0f && v < 2147483648.0f)) return false;
    *out = __float2int_rz(v);
    return true;
}

/* Grid::WhichCellPointIn (Grid.cpp:202-208) / FSG::WhichCellPointIn (FSG.cpp:88-93); -1 outside */
__device__ __forceinline__ int point_cell(const CellParams& p, float lon, float lat) {
    int row, col;
    if (!trunc_int(__fdiv_rn(__fsub_rn(p.rymax, lat), p.cell), &row)) return -1;
    if (!trunc_int(__fdiv_rn(__fsub_rn(lon, p.rxmin), p.cell), &col)) return -1;
    if (p.morton) {
        if (row < 0 || col < 0 || row >= p.axis || col >= p.axis) return -1;
        return (int)(spread_bits((uint32_t)col) | (spread_bits((uint32_t)row) << 1));
    }
    if (row < 0 || col < 0 || row >= p.ny || col >= p.nx) return -1;
    return row * p.nx + col;
}

/* per point (trajectory order): cell, position, trajectory, point index within the trajectory,
 * and for the Grid the frequency-vector key (trajectory << 32 | cell >> vparam) */
__global__ void k_point_cells(int64_t P, int n, const int64_t* __restrict__ off, const float2* __restrict__ xy,
                              CellParams p, uint32_t* cell, int32_t* pos, int32_t* tid, int32_t* pidx,
                              unsigned long long* fvkey, int32_t* flag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < P; i += (int64_t)gridDim.x * blockDim.x) {
        /* the largest t with off[t] <= i is the trajectory holding point i (off[1] = 0; an empty
         * trajectory shares its successor's offset and so is never the largest) */
        int lo = 1, hi = n;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (off[mid] <= i)
                lo = mid;
            else
                hi = mid - 1;
        }
        const float2 v = xy[i];
        int c = point_cell(p, v.x, v.y);
        if (c < 0) {
            atomicCAS(flag, 0, GAT_ERR_ARG);
            c = 0;
        }
        cell[i] = (uint32_t)c;
        pos[i] = (int32_t)i;
        tid[i] = lo;
        pidx[i] = (int32_t)(i - off[lo]);
        if (fvkey) fvkey[i] = ((unsigned long long)(unsigned)lo << 32) | (unsigned)(c >> p.vparam);
    }
}

/* index-order arrays from the sorted positions; key = tid << pidx_bits | pidx, or 0 when the
 * pair does not fit 32 bits (pidx_bits < 0) */
__global__ void k_gather_points(int64_t P, const int32_t* __restrict__ order, const float2* __restrict__ xy,
                                const int32_t* __restrict__ tid_in, const int32_t* __restrict__ pidx_in, float* x,
                                float* y, int32_t* tid, int32_t* pidx, uint32_t* key, int pidx_bits) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < P; i += (int64_t)gridDim.x * blockDim.x) {
        const int s = order[i];
        const float2 v = xy[s];
        x[i] = v.x;
        y[i] = v.y;
        const int t = tid_in[s], k = pidx_in[s];
        tid[i] = t;
        pidx[i] = k;
        key[i] = pidx_bits >= 0 ? ((uint32_t)t << pidx_bits) | (uint32_t)k : 0u;
    }
}

/* cb[c] = the first sorted position whose cell is >= c, for c = 0..ncells */
__global__ void k_cell_bounds(int64_t P, int64_t ncells, const uint32_t* __restrict__ cells, int64_t* cb) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c <= ncells; c += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = P;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((int64_t)cells[mid] < c)
                lo = mid + 1;
            else
                hi = mid;
        }
        cb[c] = lo;
    }
}

/* temporaries of one build, freed on every exit */
struct Temps {
    std::vector<void*> ptrs;
    cudaError_t err = cudaSuccess;
    ~Temps() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    T* get(size_t n) {
        if (err != cudaSuccess) return nullptr;
        void* p = nullptr;
        err = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
        if (err != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
};

int bits_to_hold(int64_t v) {
    int b = 1;
    while (b < 62 && (int64_t(1) << b) <= v) b++;
    return b;
}

int grid_size(const gat_ctx* ctx, int64_t work) {
    const int64_t want = (work + 255) / 256;
    return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)std::max(1, ctx->sm_count) * 8));
}

}  // namespace

int device_place(gat_index* ix, const DevicePlaceArgs& a, std::vector<int64_t>& cb, DeviceFv* fv) {
    gat_ctx* ctx = ix->ctx;
    const gat_db* db = ix->db;
    cudaStream_t s = ctx->stream;
    const int64_t P = db->npoints;
    const int n = db->n;
    if (P >= ((int64_t)1 << 31) - 1) return fail(ctx, GAT_ERR_ARG, std::string(a.what) + ": more than 2^31 - 2 points");
    Temps tmp;
    uint32_t* cells = tmp.get<uint32_t>(P);
    uint32_t* cells_s = tmp.get<uint32_t>(P);
    int32_t* pos = tmp.get<int32_t>(P);
    int32_t* order = tmp.get<int32_t>(P);
    int32_t* tid0 = tmp.get<int32_t>(P);
    int32_t* pidx0 = tmp.get<int32_t>(P);
    int32_t* pidx1 = tmp.get<int32_t>(P);
    int64_t* d_cb = tmp.get<int64_t>((size_t)a.ncells + 1);
    unsigned long long* fvk = fv ? tmp.get<unsigned long long>(P) : nullptr;
    if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
    CellParams cp{a.rxmin, a.rymax, a.cell, a.morton ? 1 : 0, a.axis, a.nx, a.ny, a.vparam};
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_flag, 0, sizeof(int32_t), s), "index build");
    if (P > 0) {
        k_point_cells<<<grid_size(ctx, P), 256, 0, s>>>(P, n, db->d_off, db->d_xy, cp, cells, pos, tid0, pidx0, fvk,
                                                        ctx->d_flag);
        count_launch(ctx);
    }
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "index build (cells)");
    if (check_device_flag(ctx, "index build") != GAT_OK)
        return fail(ctx, GAT_ERR_ARG, std::string(a.what) + ": a point lies outside the grid range");
    /* stable sort of (cell, position) */
    const int end_bit = bits_to_hold(a.ncells);
    size_t tbytes = 0;
    GAT_CUDA_TRY(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tbytes, cells, cells_s, pos, order, (int)P, 0, end_bit, s),
                 "index build sort");
    void* tstore = tmp.get<char>(tbytes);
    if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
    if (P > 0) {
        GAT_CUDA_TRY(ctx, cub::DeviceRadixSort::SortPairs(tstore, tbytes, cells, cells_s, pos, order, (int)P, 0, end_bit, s),
                     "index build sort");
        count_launch(ctx, 2 * ((end_bit + 7) / 8) + 1);
    }
    /* index-order arrays, allocated in the host builder's upload order (x, y, tid, key) with its
     * one element of padding, zeroed */
    const int tid_bits = bits_to_hold(n);
    int pidx_bits = bits_to_hold(std::max(1, db->maxlen - 1));
    if (tid_bits + pidx_bits > 32) pidx_bits = -1; /* point-level results unavailable for this set */
    ix->pidx_bits = pidx_bits;
    ix->npoints = P;
    int st = GAT_OK;
    const size_t pb = (size_t)(P + 1) * 4;
    float* dx = (float*)index_alloc(ix, pb, &st);
    float* dy = dx ? (float*)index_alloc(ix, pb, &st) : nullptr;
    int32_t* dt = dy ? (int32_t*)index_alloc(ix, pb, &st) : nullptr;
    uint32_t* dk = dt ? (uint32_t*)index_alloc(ix, pb, &st) : nullptr;
    if (!dk) return st;
    ix->d_x = dx;
    ix->d_y = dy;
    ix->d_tid = dt;
    ix->d_key = dk;
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(dx + P, 0, 4, s), "index build");
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(dy + P, 0, 4, s), "index build");
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(dt + P, 0, 4, s), "index build");
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(dk + P, 0, 4, s), "index build");
    if (P > 0) {
        k_gather_points<<<grid_size(ctx, P), 256, 0, s>>>(P, order, db->d_xy, tid0, pidx0, dx, dy, dt, pidx1, dk, pidx_bits);
        count_launch(ctx);
    }
    k_cell_bounds<<<grid_size(ctx, a.ncells + 1), 256, 0, s>>>(P, a.ncells, cells_s, d_cb);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "index build (gather)");
    /* host copies: gat_index_points, snapshots and the quadtree walk read them */
    ix->h_x.resize(P);
    ix->h_y.resize(P);
    ix->h_tid.resize(P);
    ix->h_pidx.resize(P);
    cb.resize((size_t)a.ncells + 1);
    if (P > 0) {
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ix->h_x.data(), dx, P * 4, cudaMemcpyDeviceToHost, s), "index build");
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ix->h_y.data(), dy, P * 4, cudaMemcpyDeviceToHost, s), "index build");
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ix->h_tid.data(), dt, P * 4, cudaMemcpyDeviceToHost, s), "index build");
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ix->h_pidx.data(), pidx1, P * 4, cudaMemcpyDeviceToHost, s), "index build");
    }
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(cb.data(), d_cb, cb.size() * 8, cudaMemcpyDeviceToHost, s), "index build");
    if (fv) {
        fv->off.assign((size_t)n + 2, 0);
        fv->cell.clear();
        fv->cnt.clear();
        fv->max_nnz = 0;
        if (P > 0) {
            unsigned long long* fvk_s = tmp.get<unsigned long long>(P);
            unsigned long long* uk = tmp.get<unsigned long long>(P);
            int32_t* cnt = tmp.get<int32_t>(P);
            int32_t* nruns = tmp.get<int32_t>(1);
            if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
            /* keys hold the trajectory above bit 32 and the virtual cell below it */
            const int kbits = 32 + bits_to_hold(n);
            size_t b1 = 0, b2 = 0;
            GAT_CUDA_TRY(ctx, cub::DeviceRadixSort::SortKeys(nullptr, b1, fvk, fvk_s, (int)P, 0, kbits, s), "index build fv");
            GAT_CUDA_TRY(ctx, cub::DeviceRunLengthEncode::Encode(nullptr, b2, fvk_s, uk, cnt, nruns, (int)P, s),
                         "index build fv");
            void* t2 = tmp.get<char>(std::max(b1, b2));
            if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
            GAT_CUDA_TRY(ctx, cub::DeviceRadixSort::SortKeys(t2, b1, fvk, fvk_s, (int)P, 0, kbits, s), "index build fv");
            GAT_CUDA_TRY(ctx, cub::DeviceRunLengthEncode::Encode(t2, b2, fvk_s, uk, cnt, nruns, (int)P, s), "index build fv");
            count_launch(ctx, 2 * ((kbits + 7) / 8) + 3);
            int32_t R = 0;
            GAT_CUDA_TRY(ctx, cudaMemcpyAsync(&R, nruns, 4, cudaMemcpyDeviceToHost, s), "index build");
            GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "index build");
            std::vector<unsigned long long> hk((size_t)R);
            fv->cnt.resize((size_t)R);
            if (R > 0) {
                GAT_CUDA_TRY(ctx, cudaMemcpyAsync(hk.data(), uk, (size_t)R * 8, cudaMemcpyDeviceToHost, s), "index build");
                GAT_CUDA_TRY(ctx, cudaMemcpyAsync(fv->cnt.data(), cnt, (size_t)R * 4, cudaMemcpyDeviceToHost, s),
                             "index build");
            }
            GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "index build");
            fv->cell.resize((size_t)R);
            for (int32_t r = 0; r < R; r++) {
                fv->cell[(size_t)r] = (int32_t)(hk[(size_t)r] & 0xffffffffull);
                fv->off[(size_t)(hk[(size_t)r] >> 32) + 1]++;
            }
            for (int t = 0; t <= n; t++) {
                fv->max_nnz = std::max<int>(fv->max_nnz, (int)fv->off[(size_t)t + 1]);
                fv->off[(size_t)t + 1] += fv->off[(size_t)t];
            }
        }
    }
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "index build");
    return GAT_OK;
}

}  // namespace gat
