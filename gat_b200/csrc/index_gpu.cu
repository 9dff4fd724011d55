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
 * Only the cell boundaries travel to the host, where the quadtree is a walk over them; the host
 * copies of the points are downloaded when first asked for (gat_index_points, snapshots).
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
 * pair does not fit 32 bits (pidx_bits < 0; the point index then goes to pidx) */
__global__ void k_gather_points(int64_t P, const int32_t* __restrict__ order, const float2* __restrict__ xy,
                                const int32_t* __restrict__ tid_in, const int32_t* __restrict__ pidx_in, float* x,
                                float* y, int32_t* tid, uint32_t* key, int32_t* pidx, int pidx_bits) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < P; i += (int64_t)gridDim.x * blockDim.x) {
        const int s = order[i];
        const float2 v = xy[s];
        x[i] = v.x;
        y[i] = v.y;
        const int t = tid_in[s], k = pidx_in[s];
        tid[i] = t;
        key[i] = pidx_bits >= 0 ? ((uint32_t)t << pidx_bits) | (uint32_t)k : 0u;
        if (pidx) pidx[i] = k;
    }
}

/* bound[j] = the first position p in the sorted keys with keys[p] >= j << shift, j = 0..m */
template <class K>
__global__ void k_bounds(int64_t P, int64_t m, const K* __restrict__ keys, int shift, int64_t* bound) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j <= m; j += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long want = (unsigned long long)j << shift;
        int64_t lo = 0, hi = P;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((unsigned long long)keys[mid] < want)
                lo = mid + 1;
            else
                hi = mid;
        }
        bound[j] = lo;
    }
}

/* frequency-vector cells: the low half of each (trajectory, virtual cell) run key */
__global__ void k_fv_cells(int64_t R, const unsigned long long* __restrict__ runs, int32_t* cell) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < R; r += (int64_t)gridDim.x * blockDim.x)
        cell[r] = (int32_t)(runs[r] & 0xffffffffull);
}

/* device allocations of one build, freed with it */
struct Temps {
    std::vector<void*> ptrs;
    cudaError_t err = cudaSuccess;
    Temps() = default;
    Temps(const Temps&) = delete;
    Temps& operator=(const Temps&) = delete;
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

/* the Grid's sorted, counted (trajectory, virtual cell) runs between device_place and device_fv */
struct DeviceFvRuns {
    Temps tmp;
    unsigned long long* runs = nullptr;
    int32_t* cnt = nullptr;
    int32_t* nruns = nullptr;
};
void DeviceFvRunsFree::operator()(DeviceFvRuns* r) const { delete r; }

int device_place(gat_index* ix, const DevicePlaceArgs& a, std::vector<int64_t>& cb, DeviceFvHandle* fv) {
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
    if (pidx_bits < 0) GAT_CUDA_TRY(ctx, cudaMalloc(&ix->d_pidx, std::max<size_t>((size_t)P, 1) * 4), "index build");
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(dx + P, 0, 4, s), "index build");
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(dy + P, 0, 4, s), "index build");
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(dt + P, 0, 4, s), "index build");
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(dk + P, 0, 4, s), "index build");
    if (P > 0) {
        k_gather_points<<<grid_size(ctx, P), 256, 0, s>>>(P, order, db->d_xy, tid0, pidx0, dx, dy, dt, dk, ix->d_pidx,
                                                          pidx_bits);
        count_launch(ctx);
    }
    k_bounds<uint32_t><<<grid_size(ctx, a.ncells + 1), 256, 0, s>>>(P, a.ncells, cells_s, 0, d_cb);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "index build (gather)");
    cb.resize((size_t)a.ncells + 1);
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(cb.data(), d_cb, cb.size() * 8, cudaMemcpyDeviceToHost, s), "index build");
    ix->host_pending = true;
    if (fv) {
        /* (trajectory, virtual cell) keys sorted and run-length counted; kept for device_fv */
        DeviceFvHandle r(new DeviceFvRuns());
        unsigned long long* fvk_s = r->tmp.get<unsigned long long>(P);
        r->runs = r->tmp.get<unsigned long long>(P);
        r->cnt = r->tmp.get<int32_t>(P + 1);
        r->nruns = r->tmp.get<int32_t>(1);
        if (r->tmp.err != cudaSuccess) return cuda_fail(ctx, r->tmp.err, "index build (device temporaries)");
        GAT_CUDA_TRY(ctx, cudaMemsetAsync(r->nruns, 0, 4, s), "index build fv");
        if (P > 0) {
            /* keys hold the trajectory above bit 32 and the virtual cell below it */
            const int kbits = 32 + bits_to_hold(n);
            size_t b1 = 0, b2 = 0;
            GAT_CUDA_TRY(ctx, cub::DeviceRadixSort::SortKeys(nullptr, b1, fvk, fvk_s, (int)P, 0, kbits, s), "index build fv");
            GAT_CUDA_TRY(ctx, cub::DeviceRunLengthEncode::Encode(nullptr, b2, fvk_s, r->runs, r->cnt, r->nruns, (int)P, s),
                         "index build fv");
            void* t2 = tmp.get<char>(std::max(b1, b2));
            if (tmp.err != cudaSuccess) return cuda_fail(ctx, tmp.err, "index build (device temporaries)");
            GAT_CUDA_TRY(ctx, cub::DeviceRadixSort::SortKeys(t2, b1, fvk, fvk_s, (int)P, 0, kbits, s), "index build fv");
            GAT_CUDA_TRY(ctx, cub::DeviceRunLengthEncode::Encode(t2, b2, fvk_s, r->runs, r->cnt, r->nruns, (int)P, s),
                         "index build fv");
            count_launch(ctx, 2 * ((kbits + 7) / 8) + 3);
        }
        *fv = std::move(r);
    }
    /* the temporaries are freed on return: wait for the work that reads them */
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "index build");
    return GAT_OK;
}

int device_fv(gat_index* ix, DeviceFvRuns* fv) {
    gat_ctx* ctx = ix->ctx;
    cudaStream_t s = ctx->stream;
    const int n = ix->db->n;
    int32_t R = 0;
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(&R, fv->nruns, 4, cudaMemcpyDeviceToHost, s), "index build fv");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "index build fv");
    /* sizes and order of the host builder's uploads: fv_off [n+2], fv_cell [R], fv_cnt [R], each
     * with one zeroed element of padding */
    int st = GAT_OK;
    int64_t* off = (int64_t*)index_alloc(ix, (size_t)(n + 3) * 8, &st);
    int32_t* cell = off ? (int32_t*)index_alloc(ix, (size_t)(R + 1) * 4, &st) : nullptr;
    int32_t* cnt = cell ? (int32_t*)index_alloc(ix, (size_t)(R + 1) * 4, &st) : nullptr;
    if (!cnt) return st;
    ix->d_fv_off = off;
    ix->d_fv_cell = cell;
    ix->d_fv_cnt = cnt;
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(off + n + 2, 0, 8, s), "index build fv");
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(cell + R, 0, 4, s), "index build fv");
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(cnt + R, 0, 4, s), "index build fv");
    if (R > 0) {
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(cnt, fv->cnt, (size_t)R * 4, cudaMemcpyDeviceToDevice, s), "index build fv");
        k_fv_cells<<<grid_size(ctx, R), 256, 0, s>>>(R, fv->runs, cell);
        count_launch(ctx);
    }
    /* off[t] = entries of trajectories below t: the first run whose key is >= t << 32 */
    k_bounds<unsigned long long><<<grid_size(ctx, n + 2), 256, 0, s>>>(R, n + 1, fv->runs, 32, off);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "index build fv");
    std::vector<int64_t> h((size_t)n + 2);
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), off, h.size() * 8, cudaMemcpyDeviceToHost, s), "index build fv");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "index build fv");
    int mx = 0;
    for (int t = 0; t <= n; t++) mx = std::max<int>(mx, (int)(h[(size_t)t + 1] - h[(size_t)t]));
    ix->fv_max_nnz = mx;
    ix->fv_entries = R;
    return GAT_OK;
}

int index_points_device(const gat_index* ix, float* x, float* y, int32_t* tid, int32_t* pidx) {
    gat_ctx* ctx = ix->ctx;
    const int64_t P = ix->npoints;
    if (P == 0) return GAT_OK;
    cudaSetDevice(ctx->device);
    const size_t b = (size_t)P * 4;
    if (x) GAT_CUDA_TRY(ctx, cudaMemcpy(x, ix->d_x, b, cudaMemcpyDeviceToHost), "index points");
    if (y) GAT_CUDA_TRY(ctx, cudaMemcpy(y, ix->d_y, b, cudaMemcpyDeviceToHost), "index points");
    if (tid) GAT_CUDA_TRY(ctx, cudaMemcpy(tid, ix->d_tid, b, cudaMemcpyDeviceToHost), "index points");
    if (pidx && ix->pidx_bits >= 0) {
        /* the point index is the key's low pidx_bits bits */
        GAT_CUDA_TRY(ctx, cudaMemcpy(pidx, ix->d_key, b, cudaMemcpyDeviceToHost), "index points");
        const uint32_t mask = (uint32_t)((1ull << ix->pidx_bits) - 1);
        for (int64_t i = 0; i < P; i++) pidx[i] = (int32_t)((uint32_t)pidx[i] & mask);
    } else if (pidx) {
        GAT_CUDA_TRY(ctx, cudaMemcpy(pidx, ix->d_pidx, b, cudaMemcpyDeviceToHost), "index points");
    }
    return GAT_OK;
}

int index_host_copies(gat_index* ix) {
    std::lock_guard<std::mutex> lk(ix->host_mu);
    if (!ix->host_pending) return GAT_OK;
    const size_t P = (size_t)ix->npoints;
    std::vector<float> x(P), y(P);
    std::vector<int32_t> tid(P), pidx(P);
    if (int st = index_points_device(ix, x.data(), y.data(), tid.data(), pidx.data())) return st;
    ix->h_x.swap(x);
    ix->h_y.swap(y);
    ix->h_tid.swap(tid);
    ix->h_pidx.swap(pidx);
    ix->host_pending = false;
    return GAT_OK;
}

}  // namespace gat
