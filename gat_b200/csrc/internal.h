/* Internal types of libgat_b200: context, device-resident trajectory set and indexes.
 *
 * Device layout (all arrays in HBM, owned by the handle):
 *   trajectory set : xy[P] float2 in trajectory order (trajectory t at off[t] .. off[t+1]),
 *                    len[n+1] (len[0] = 0), off[n+2]
 *   index points   : x[P], y[P] float SoA in the index's point order (Morton-cell order for
 *                    the Grid, the STIG leaf order, row-major cell order for FSG), key[P] =
 *                    (tid << pidx_bits) | point index within trajectory, tid[P]
 *   Grid tree      : breadth-first node arrays, children of node i at child[i] .. child[i]+3,
 *                    child = -1 for leaves, leaf point range [pbeg, pend)
 *   STIG tree      : node arrays (leaf flag, split dim, median, children, leaf range + MBB)
 *   FSG            : per-cell point range, cells along x/y
 *   FVTable        : CSR over trajectory ids: fv_off[n+2], (vcell, count) entries sorted by vcell
 */
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "gat_b200.h"

namespace gat {

/* ---------------------------------------------------------------- device structs */
struct GridDev {
    float rxmin, rymin, rxmax, rymax; /* grid range (the Grid's MBB) */
    float cell;
    int axis, cellnum, total_level, vparam;
    int nnodes;
    const float4* node_mbb;
    const int32_t* node_child;
    const int32_t* node_pbeg;
    const int32_t* node_pend;
    const float4* node_pbox; /* exact box of each node's points (index_point_boxes; null: none) */
};

struct StigDev {
    int nnodes;
    const int32_t* kind;   /* 1 leaf, 0 internal */
    const int32_t* dim;    /* depth % 2 */
    const float* median;
    const int32_t* left;
    const int32_t* right;
    const int32_t* lo;     /* leaf: inclusive range */
    const int32_t* hi;
    const float4* mbb;     /* leaf MBB */
    const float4* pbox;    /* exact box of each leaf's points (index_point_boxes; null: none) */
};

struct FsgDev {
    float rxmin, rymin, rxmax, rymax;
    float cell;
    int nx, ny, cellnum;
    const int32_t* cbeg; /* point range of cell c: [cbeg[c], cend[c]) */
    const int32_t* cend;
};

/* MortonGrid (MortonGrid.h:22-40): the Grid's quadtree as an implicit tree. Node (level, id)
 * covers the Morton cells [id * 4^(L - level), (id + 1) * 4^(L - level)); it is a leaf when bit
 * (4^level - 1) / 3 + id of `leaf` is set (findIdxInBitmap, MortonGrid.cpp:8-13); its points are
 * [cbeg[first cell], cbeg[last cell + 1]) of the Grid's point order. */
struct MortonDev {
    float rxmin, rymax, cell;
    int total_level;
    const uint32_t* leaf;
    const int32_t* cbeg;
};

/* One EDR problem: query side (a) and candidate side (b), offsets into two point arrays. */
struct EdrPair {
    int64_t a_off;
    int64_t b_off;
    int32_t a_len;
    int32_t b_len;
};

}  // namespace gat

/* ---------------------------------------------------------------- handles */
struct EdrChain;

struct gat_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    std::mutex mu;           /* serialises calls on one context */
    int64_t launches = 0;
    /* scratch arena: slot -> device buffer, grown on demand, freed with the context */
    std::vector<void*> slot_ptr;
    std::vector<size_t> slot_bytes;
    std::vector<char> slot_fresh; /* allocated since the last scratch_zeroed clear */
    int32_t* d_flag = nullptr; /* [0] device status written by kernels (0 = ok), [1] sink word,
                                  [4..5] EDR launch epochs (64-bit counter) */
    /* optional per-kernel-class event timing (gat_ctx_set_timing) */
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pending[GAT_KERNEL_CLASSES];
    std::vector<cudaEvent_t> ev_free;
    double t_ms[GAT_KERNEL_CLASSES] = {0, 0, 0};
    int64_t t_launches[GAT_KERNEL_CLASSES] = {0, 0, 0};
    double t_work[GAT_KERNEL_CLASSES] = {0, 0, 0};
    int64_t* h_pinned = nullptr; /* pinned host words for small D2H reads */
    void* h_stage = nullptr;     /* pinned staging for host arrays the library builds (host_stage) */
    size_t h_stage_bytes = 0;
    gat_ctx* root = nullptr; /* worker contexts: the context whose indexes they may use */
    /* EDR rows per lane: 0 = autotune per shape class (edr_tune), else fixed */
    int edr_rows = 0;
    int edr_form = 0; /* 0 = autotune, 1 = row tiles, 2 = column tiles */
    int topk_chunk = 0, topk_growth = 0; /* 0 = defaults */
    int index_build = 0;                 /* 0 = device when present, 1 = host, 2 = device */
    int dep_launch = 1;                  /* programmatic dependent launch on the query path */
    int test_stall_pair = 0;             /* GAT_TUNE_TEST_STALL_CARRY (tests of the bounded wait) */
    int sm_reserve = 0;                  /* SMs the persistent EDR kernel leaves to other streams (serving lanes) */
    int edr_reserve_pct = 0;             /* GAT_TUNE_EDR_RESERVE as set (sm_reserve = sm_count * pct / 100) */
    int serve_reserve = 0;               /* GAT_TUNE_SERVE_RESERVE: percent of the SMs a server's top-k lanes leave free */
    EdrChain* edr_chain = nullptr;       /* serving lanes: EDR grids of sibling lanes run one at a time */
    cudaMemPool_t build_pool = nullptr;  /* scratch slots and index-build temporaries, kept until gat_ctx_trim */
    std::map<uint64_t, int> edr_tune; /* worker contexts use their root's table */
    int range_shape = 0;               /* GAT_TUNE_RANGE_SHAPE: 0 = tuned per batch-size class, 1, 2 fixed */
    std::map<uint64_t, int> range_tune; /* (index kind, batch size class) -> hash kernel shape */
    std::mutex tune_mu;
    /* objects that hold device memory of this context's scratch or workers (cached CUDA graphs);
     * released first by gat_ctx_destroy and gat_ctx_trim */
    std::vector<std::pair<void*, void (*)(void*)>> owned;
};

/* The persistent EDR grids of a server's top-k lanes run one at a time: each launch waits for
 * the completion event of the previous one (of any lane) and records its own. A grid leaves free
 * CTA slots for the range lane only while no second grid is resident to fill them. */
struct EdrChain {
    std::mutex mu;
    cudaEvent_t ev = nullptr;
};

struct gat_db {
    gat_ctx* ctx = nullptr;
    int n = 0;
    int64_t npoints = 0;
    int maxlen = 0;
    std::vector<int32_t> h_len;  /* [n+1], h_len[0] = 0 */
    std::vector<int64_t> h_off;  /* [n+2] */
    std::vector<float> h_x, h_y; /* trajectory order; on a device context downloaded on first use */
    bool host_pending = false;
    std::mutex host_mu;
    int32_t* d_len = nullptr;
    int64_t* d_off = nullptr;
    float2* d_xy = nullptr;
};

struct gat_index {
    gat_ctx* ctx = nullptr;
    const gat_db* db = nullptr;
    int kind = 0;
    int64_t npoints = 0;
    int pidx_bits = 0;
    size_t device_bytes = 0;
    std::vector<void*> allocs;        /* device arrays in upload order (index snapshots rely on it) */
    std::vector<size_t> alloc_bytes;
    /* points in index order */
    float* d_x = nullptr;
    float* d_y = nullptr;
    uint32_t* d_key = nullptr;
    int32_t* d_tid = nullptr;
    /* host copies kept for gat_index_points, snapshots and the tree walks of the builders; an
     * index placed on the device downloads them on first use (host_pending, under host_mu) */
    std::vector<int32_t> h_tid, h_pidx;
    std::vector<float> h_x, h_y;
    bool host_pending = false;
    std::mutex host_mu;
    int32_t* d_pidx = nullptr; /* device-placed index whose point index does not fit the key */
    float4* d_pbox = nullptr;  /* derived, not saved in snapshots: GridDev::node_pbox / StigDev::pbox */
    int64_t leaves = 0, nodes = 0;
    gat::GridDev grid{};
    gat::StigDev stig{};
    gat::FsgDev fsg{};
    gat::MortonDev morton{};
    const gat_index* base = nullptr; /* MortonGrid: the Grid whose point arrays it reads */
    /* Grid FVTable (CSR over tids 0..n) */
    int64_t* d_fv_off = nullptr;
    int32_t* d_fv_cell = nullptr;
    int32_t* d_fv_cnt = nullptr;
    int fv_max_nnz = 0;
    int64_t fv_entries = 0;
};

/* ---------------------------------------------------------------- helpers (context.cpp) */
namespace gat {

int fail(gat_ctx* ctx, int code, const std::string& msg);
int cuda_fail(gat_ctx* ctx, cudaError_t e, const char* what);
/* device scratch slot of at least `bytes` bytes; contents undefined */
void* scratch(gat_ctx* ctx, int slot, size_t bytes, int* status);
/* releases the context's owned objects (cached graphs and their workers) */
void release_owned(gat_ctx* ctx);
/* same, but a slot that was (re)allocated is cleared to zero (on the context stream) first */
void* scratch_zeroed(gat_ctx* ctx, int slot, size_t bytes, int* status);
/* cudaMalloc tracked by an index (freed by gat_index_destroy) */
void* index_alloc(gat_index* ix, size_t bytes, int* status);
template <class T>
T* index_upload(gat_index* ix, const std::vector<T>& v, int* status) {
    T* p = (T*)index_alloc(ix, v.size() * sizeof(T) + sizeof(T), status);
    if (!p) return nullptr;
    cudaError_t e = v.empty() ? cudaSuccess : cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(p + v.size(), 0, sizeof(T)); /* the padding element */
    if (e != cudaSuccess) {
        *status = cuda_fail(ix->ctx, e, "upload");
        return nullptr;
    }
    return p;
}
/* pinned host staging of at least `bytes` bytes, owned by the context (one user at a time: the
 * caller's copies from it must finish before the next call) */
void* host_stage(gat_ctx* ctx, size_t bytes, int* status);
/* Derives the exact box of the points under every quadtree node (Grid) or STIG leaf, so that the
 * range walks can mark candidate ranges whose every point is a hit (pbox.cu). Called after a
 * Grid or STIG is built or loaded on a device context; a no-op for other kinds. */
int index_point_boxes(gat_index* ix);
/* reads and clears the device status word; returns GAT_OK or the code a kernel stored */
int check_device_flag(gat_ctx* ctx, const char* what);
inline void count_launch(gat_ctx* ctx, int n = 1) { ctx->launches += n; }
/* brackets one launch of a timed kernel class (no-ops unless timing is on) */
void timed_begin(gat_ctx* ctx, int cls);
void timed_end(gat_ctx* ctx, int cls, double work);
/* device-side work counter for classes whose work is only known on the device (EDR cells) */
void timed_add_work(gat_ctx* ctx, int cls, double work);

/* the context's stream-ordered memory pool (scratch slots, index-build temporaries; it keeps
 * freed memory until gat_ctx_trim); null when the device has no memory pools (index_gpu.cu) */
cudaMemPool_t build_pool(gat_ctx* ctx);
/* returns every scratch slot and waits for the context's stream */
void free_slots(gat_ctx* ctx);
/* replaces the context's (still unused) stream by one of the device's greatest priority */
int ctx_use_priority_stream(gat_ctx* ctx);
/* GAT_ERR_STATE for a host-only context (device -1) */
int require_device(gat_ctx* ctx, const char* what);
/* Opts a kernel into `bytes` of dynamic shared memory when that (plus the kernel's few KB of
 * static shared memory) could exceed the 48 KB default. */
template <class K>
inline void allow_smem(K kernel, size_t bytes) {
    if (bytes > 40 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}
/* true when `user` may run queries on objects created through `owner` (the same context, or
 * worker contexts of one parent) */
bool same_owner(const gat_ctx* owner, const gat_ctx* user);

/* the context's device counter of tiled-EDR launches (tags carry words) */
inline unsigned long long* edr_epochs(gat_ctx* ctx) { return reinterpret_cast<unsigned long long*>(ctx->d_flag + 4); }
/* smallest float >= eps (the reference compares |float diff| < (double)EPSILON) */
float match_threshold(double eps);

/* scratch slot ids */
enum Slot {
    S_SCAN_TMP = 0,
    S_RANGE_Q,
    S_RANGE_ICNT,
    S_RANGE_IOFF,
    S_RANGE_ITEMS,
    S_RANGE_SEGBASE,
    S_RANGE_SEGCNT,
    S_RANGE_ARENA,
    S_RANGE_ARENA2,
    S_RANGE_OFF,
    S_RANGE_OUT_T,
    S_RANGE_OUT_P,
    S_RANGE_CURSOR,
    S_RANGE_OVF,
    S_RANGE_CSR,
    S_RANGE_ORDER,
    S_RANGE_TPOS,
    S_RANGE_TASK,
    S_EDR_PAIRS,
    S_EDR_CARRY,
    S_EDR_COUNTERS,
    S_EDR_IO,
    S_EDR_ITEMS,
    S_EDR_PCARRY,
    S_EDR_META,
    S_TOPK_GSTAGE,
    S_TOPK_QFV,
    S_TOPK_LB,
    S_TOPK_PAIRS,
    S_TOPK_DIST,
    S_TOPK_QSTATE,
    S_TOPK_SEG,
    S_TOPK_IO,
    S_TOPK_OUT,
    S_TOPK_NEAR,
    S_COUNT
};

/* ---------------------------------------------------------------- launchers (.cu) */
/* exclusive scan of n int64 counts into out[0..n] (out[n] = total); in may alias out */
int scan_i64(gat_ctx* ctx, const int64_t* in, int64_t* out, int64_t n);
/* EDR of pairs (a_off, a_len, b_off, b_len) over point arrays A and B; the count is read
 * from d_npairs when non-NULL, else npairs (edr.cu) */
int edr_launch_soa(gat_ctx* ctx, int npairs, const int* d_npairs, const int64_t* a_off, const int32_t* a_len,
                   const int64_t* b_off, const int32_t* b_len, int rows_hint, int max_cols, const float2* A,
                   const float2* B, float u, int32_t* d_out, unsigned long long* d_cells);

/* Device builds of a Grid or FSG index (index_gpu.cu): points, cell boundaries, quadtree and
 * frequency vectors computed in HBM, allocated in the host builder's order; the host copies of
 * the points are downloaded on first use. */
struct DevicePlaceArgs {
    const char* what; /* the API call, for error messages */
    bool morton;      /* Grid (Morton ids on axis x axis) or FSG (row-major nx x ny) */
    float rxmin, rymax, cell;
    int axis, nx, ny, vparam;
    int64_t ncells;
};
int device_build_grid(gat_index* ix, const DevicePlaceArgs& a, int total_level, int leaf_cap);
int device_build_fsg(gat_index* ix, const DevicePlaceArgs& a);
/* uploads lon / lat (host, trajectory order) into d_xy as interleaved (lon, lat) pairs */
int upload_set_points(gat_ctx* ctx, const float* lon, const float* lat, int64_t P, float2* d_xy);
/* downloads the host copies (h_x, h_y) of a device trajectory set (no-op when present) */
int db_host_copies(const gat_db* db);
/* downloads the host copies of a device-placed index (no-op otherwise) */
int index_host_copies(gat_index* ix);
/* gat_index_points for a device-placed index without host copies: device arrays straight into
 * the caller's buffers (any may be NULL); the caller holds ix->host_mu */
int index_points_device(const gat_index* ix, float* x, float* y, int32_t* tid, int32_t* pidx);

}  // namespace gat

#define GAT_CUDA_TRY(ctx, expr, what)                    \
    do {                                                 \
        cudaError_t e__ = (expr);                        \
        if (e__ != cudaSuccess) return gat::cuda_fail((ctx), e__, (what)); \
    } while (0)
