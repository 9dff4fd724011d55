/* Context, error reporting, device scratch arena and the device-resident trajectory set. */
#include <cmath>
#include <cstring>
#include <limits>

#include "internal.h"

namespace gat {

int fail(gat_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(gat_ctx* ctx, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError(); /* clear sticky-free errors so later calls can proceed */
    return fail(ctx, e == cudaErrorMemoryAllocation ? GAT_ERR_OOM : GAT_ERR_CUDA, m);
}

void release_owned(gat_ctx* ctx) {
    for (auto& o : ctx->owned) o.second(o.first);
    ctx->owned.clear();
}

void* scratch(gat_ctx* ctx, int slot, size_t bytes, int* status) {
    if (bytes == 0) bytes = 256;
    if (ctx->slot_bytes[slot] >= bytes) return ctx->slot_ptr[slot];
    if (ctx->device >= 0) {
        /* a slot cannot move while a CUDA graph is being captured from this context */
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(ctx->stream, &cs);
        if (cs != cudaStreamCaptureStatusNone) {
            *status = fail(ctx, GAT_ERR_STATE, "scratch growth during graph capture");
            return nullptr;
        }
    }
    /* Slots live in the context's stream-ordered pool: growing one frees and allocates in the
     * stream's order, with no device-wide synchronisation (cudaFree would wait for the kernels of
     * every stream, so one context's growth would stall the others: the serving lanes) */
    cudaMemPool_t pool = ctx->device >= 0 ? build_pool(ctx) : nullptr;
    auto release = [&](void* q) {
        if (pool) {
            cudaFreeAsync(q, ctx->stream);
        } else {
            cudaStreamSynchronize(ctx->stream);
            cudaFree(q);
        }
    };
    auto take = [&](void** q, size_t b) {
        return pool ? cudaMallocFromPoolAsync(q, b, pool, ctx->stream) : cudaMalloc(q, b);
    };
    if (ctx->slot_ptr[slot]) {
        release(ctx->slot_ptr[slot]);
        ctx->slot_ptr[slot] = nullptr;
        ctx->slot_bytes[slot] = 0;
    }
    size_t grow = bytes + bytes / 4;
    void* p = nullptr;
    cudaError_t e = take(&p, grow);
    if (e != cudaSuccess) {
        cudaGetLastError();
        e = take(&p, bytes);
        grow = bytes;
    }
    if (e != cudaSuccess) {
        *status = cuda_fail(ctx, e, "scratch allocation");
        return nullptr;
    }
    ctx->slot_ptr[slot] = p;
    ctx->slot_bytes[slot] = grow;
    ctx->slot_fresh[slot] = 1;
    return p;
}

/* returns every scratch slot (to the context's pool when it has one) and waits for the stream */
void free_slots(gat_ctx* ctx) {
    for (size_t i = 0; i < ctx->slot_ptr.size(); i++) {
        if (ctx->slot_ptr[i]) {
            if (ctx->build_pool)
                cudaFreeAsync(ctx->slot_ptr[i], ctx->stream);
            else
                cudaFree(ctx->slot_ptr[i]);
        }
        ctx->slot_ptr[i] = nullptr;
        ctx->slot_bytes[i] = 0;
    }
    cudaStreamSynchronize(ctx->stream);
}

void* host_stage(gat_ctx* ctx, size_t bytes, int* status) {
    if (bytes <= ctx->h_stage_bytes) return ctx->h_stage;
    const size_t had = ctx->h_stage_bytes;
    if (ctx->h_stage) {
        /* an earlier copy may still read it */
        cudaStreamSynchronize(ctx->stream);
        cudaFreeHost(ctx->h_stage);
        ctx->h_stage = nullptr;
        ctx->h_stage_bytes = 0;
    }
    const size_t nb = std::max<size_t>(std::max<size_t>(bytes, 2 * had), (size_t)64 << 10); /* grows by doubling */
    void* p = nullptr;
    cudaError_t e = cudaMallocHost(&p, nb);
    if (e != cudaSuccess) {
        *status = cuda_fail(ctx, e, "pinned staging");
        return nullptr;
    }
    ctx->h_stage = p;
    ctx->h_stage_bytes = nb;
    return p;
}

void* scratch_zeroed(gat_ctx* ctx, int slot, size_t bytes, int* status) {
    void* p = scratch(ctx, slot, bytes, status);
    if (p && ctx->slot_fresh[slot]) {
        cudaError_t e = cudaMemsetAsync(p, 0, ctx->slot_bytes[slot], ctx->stream);
        if (e != cudaSuccess) {
            *status = cuda_fail(ctx, e, "scratch clear");
            return nullptr;
        }
        ctx->slot_fresh[slot] = 0;
    }
    return p;
}

void* index_alloc(gat_index* ix, size_t bytes, int* status) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        *status = cuda_fail(ix->ctx, e, "index allocation");
        return nullptr;
    }
    ix->allocs.push_back(p);
    ix->alloc_bytes.push_back(bytes ? bytes : 16);
    ix->device_bytes += bytes;
    return p;
}

int check_device_flag(gat_ctx* ctx, const char* what) {
    /* read into the context's pinned words: a copy to pageable memory goes through the driver's
     * shared staging buffer and can wait behind other streams' pageable copies */
    int32_t* hf = reinterpret_cast<int32_t*>(ctx->h_pinned + 63);
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(hf, ctx->d_flag, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream), what);
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), what);
    const int32_t flag = *hf;
    if (flag == 0) return GAT_OK;
    cudaMemsetAsync(ctx->d_flag, 0, sizeof(int32_t), ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return fail(ctx, flag, std::string(what) + ": device reported status " + std::to_string(flag));
}

int ctx_use_priority_stream(gat_ctx* ctx) {
    if (!ctx || ctx->device < 0) return GAT_OK;
    int least = 0, greatest = 0;
    cudaStream_t s = nullptr;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, greatest);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "priority stream");
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    ctx->stream = s;
    return GAT_OK;
}

bool same_owner(const gat_ctx* owner, const gat_ctx* user) {
    const gat_ctx* a = owner->root ? owner->root : owner;
    const gat_ctx* b = user->root ? user->root : user;
    return a == b;
}

int require_device(gat_ctx* ctx, const char* what) {
    if (ctx && ctx->device < 0) return fail(ctx, GAT_ERR_STATE, std::string(what) + ": host-only context has no device");
    return GAT_OK;
}

static cudaEvent_t take_event(gat_ctx* ctx) {
    if (!ctx->ev_free.empty()) {
        cudaEvent_t e = ctx->ev_free.back();
        ctx->ev_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void timed_begin(gat_ctx* ctx, int cls) {
    if (!ctx->timing) return;
    cudaEvent_t a = take_event(ctx), b = take_event(ctx);
    cudaEventRecord(a, ctx->stream);
    ctx->ev_pending[cls].push_back({a, b});
}

void timed_end(gat_ctx* ctx, int cls, double work) {
    if (!ctx->timing || ctx->ev_pending[cls].empty()) return;
    cudaEventRecord(ctx->ev_pending[cls].back().second, ctx->stream);
    ctx->t_launches[cls]++;
    ctx->t_work[cls] += work;
}

void timed_add_work(gat_ctx* ctx, int cls, double work) {
    if (ctx->timing) ctx->t_work[cls] += work;
}

static void drain_events(gat_ctx* ctx) {
    for (int c = 0; c < GAT_KERNEL_CLASSES; c++) {
        for (auto& pr : ctx->ev_pending[c]) {
            float ms = 0.f;
            cudaEventSynchronize(pr.second);
            if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) ctx->t_ms[c] += ms;
            ctx->ev_free.push_back(pr.first);
            ctx->ev_free.push_back(pr.second);
        }
        ctx->ev_pending[c].clear();
    }
    cudaGetLastError();
}

float match_threshold(double eps) {
    float u = (float)eps;
    if ((double)u < eps) u = std::nextafter(u, std::numeric_limits<float>::infinity());
    return u;
}

}  // namespace gat

using namespace gat;

extern "C" {

int gat_ctx_create(int device, gat_ctx** out) {
    if (!out) return GAT_ERR_ARG;
    *out = nullptr;
    if (device == -1) {
        /* host-only context: builds index layouts without a GPU (for inspection and tests);
         * every call that needs the device returns GAT_ERR_STATE */
        gat_ctx* c = new gat_ctx();
        c->device = -1;
        c->slot_ptr.assign(S_COUNT, nullptr);
        c->slot_bytes.assign(S_COUNT, 0);
    c->slot_fresh.assign(S_COUNT, 0);
        *out = c;
        return GAT_OK;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return GAT_ERR_CUDA;
    }
    gat_ctx* c = new gat_ctx();
    c->device = device;
    c->slot_ptr.assign(S_COUNT, nullptr);
    c->slot_bytes.assign(S_COUNT, 0);
    c->slot_fresh.assign(S_COUNT, 0);
    if ((e = cudaSetDevice(device)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMalloc(&c->d_flag, 16 * sizeof(int32_t))) != cudaSuccess ||
        (e = cudaMemset(c->d_flag, 0, 16 * sizeof(int32_t))) != cudaSuccess ||
        (e = cudaMallocHost(&c->h_pinned, 64 * sizeof(int64_t))) != cudaSuccess) {
        cudaGetLastError();
        gat_ctx_destroy(c);
        return e == cudaErrorMemoryAllocation ? GAT_ERR_OOM : GAT_ERR_CUDA;
    }
    *out = c;
    return GAT_OK;
}

int gat_ctx_create_worker(gat_ctx* parent, gat_ctx** out) {
    if (!parent || !out) return GAT_ERR_ARG;
    int rc = gat_ctx_create(parent->device < 0 ? -1 : parent->device, out);
    if (rc != GAT_OK) return rc;
    (*out)->root = parent->root ? parent->root : parent;
    return GAT_OK;
}

int gat_ctx_trim(gat_ctx* ctx) {
    if (!ctx) return GAT_ERR_ARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (ctx->device < 0) return GAT_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    release_owned(ctx);
    free_slots(ctx);
    if (ctx->build_pool) cudaMemPoolTrimTo(ctx->build_pool, 0);
    return GAT_OK;
}

void gat_ctx_destroy(gat_ctx* ctx) {
    if (!ctx) return;
    if (ctx->device < 0) {
        delete ctx;
        return;
    }
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    release_owned(ctx);
    drain_events(ctx);
    for (cudaEvent_t e : ctx->ev_free) cudaEventDestroy(e);
    free_slots(ctx);
    if (ctx->build_pool) cudaMemPoolDestroy(ctx->build_pool);
    if (ctx->d_flag) cudaFree(ctx->d_flag);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* gat_last_error(const gat_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

void* gat_ctx_stream(gat_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int gat_ctx_sync(gat_ctx* ctx) {
    if (!ctx) return GAT_ERR_ARG;
    if (ctx->device < 0) return GAT_OK;
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
    return GAT_OK;
}

int64_t gat_ctx_launches(const gat_ctx* ctx) { return ctx ? ctx->launches : 0; }

int gat_ctx_set_timing(gat_ctx* ctx, int on) {
    if (!ctx) return GAT_ERR_ARG;
    if (int rq = require_device(ctx, "gat_ctx_set_timing")) return rq;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaStreamSynchronize(ctx->stream);
    drain_events(ctx);
    for (int c = 0; c < GAT_KERNEL_CLASSES; c++) {
        ctx->t_ms[c] = 0;
        ctx->t_launches[c] = 0;
        ctx->t_work[c] = 0;
    }
    ctx->timing = on != 0;
    return GAT_OK;
}

int gat_ctx_kernel_stats(gat_ctx* ctx, int cls, double* ms, int64_t* launches, double* work) {
    if (!ctx || cls < 0 || cls >= GAT_KERNEL_CLASSES) return GAT_ERR_ARG;
    if (int rq = require_device(ctx, "gat_ctx_kernel_stats")) return rq;
    std::lock_guard<std::mutex> lk(ctx->mu);
    drain_events(ctx);
    if (ms) *ms = ctx->t_ms[cls];
    if (launches) *launches = ctx->t_launches[cls];
    if (work) *work = ctx->t_work[cls];
    return GAT_OK;
}

int gat_ctx_set_tuning(gat_ctx* ctx, int knob, int value) {
    if (!ctx) return GAT_ERR_ARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (knob == GAT_TUNE_EDR_FORM) {
        if (value < 0 || value > 2) return fail(ctx, GAT_ERR_ARG, "gat_ctx_set_tuning: EDR form must be 0, 1 or 2");
        ctx->edr_form = value;
        std::lock_guard<std::mutex> tk(ctx->tune_mu);
        ctx->edr_tune.clear();
        return GAT_OK;
    }
    if (knob == GAT_TUNE_TOPK_CHUNK) {
        if (value < 0 || value > (1 << 24)) return fail(ctx, GAT_ERR_ARG, "gat_ctx_set_tuning: chunk outside 0..2^24");
        ctx->topk_chunk = value;
        return GAT_OK;
    }
    if (knob == GAT_TUNE_TOPK_GROWTH) {
        if (value < 0 || value == 1 || value > 64) return fail(ctx, GAT_ERR_ARG, "gat_ctx_set_tuning: growth must be 0 or 2..64");
        ctx->topk_growth = value;
        return GAT_OK;
    }
    if (knob == GAT_TUNE_INDEX_BUILD) {
        if (value < 0 || value > 2) return fail(ctx, GAT_ERR_ARG, "gat_ctx_set_tuning: index build must be 0, 1 or 2");
        ctx->index_build = value;
        return GAT_OK;
    }
    if (knob == GAT_TUNE_DEP_LAUNCH) {
        if (value < 0 || value > 1) return fail(ctx, GAT_ERR_ARG, "gat_ctx_set_tuning: dependent launch must be 0 or 1");
        ctx->dep_launch = value;
        return GAT_OK;
    }
    if (knob == GAT_TUNE_TEST_STALL_CARRY) {
        if (value < 0) return fail(ctx, GAT_ERR_ARG, "gat_ctx_set_tuning: stall pair must be >= 0");
        ctx->test_stall_pair = value;
        return GAT_OK;
    }
    if (knob == GAT_TUNE_RANGE_SHAPE) {
        if (value < 0 || value > 3) return fail(ctx, GAT_ERR_ARG, "gat_ctx_set_tuning: range shape must be 0..3");
        ctx->range_shape = value;
        std::lock_guard<std::mutex> tk(ctx->tune_mu);
        ctx->range_tune.clear();
        return GAT_OK;
    }
    if (knob == GAT_TUNE_EDR_RESERVE) {
        if (value < 0 || value > 90) return fail(ctx, GAT_ERR_ARG, "gat_ctx_set_tuning: EDR reserve must be 0..90");
        ctx->sm_reserve = ctx->sm_count * value / 100;
        ctx->edr_reserve_pct = value;
        return GAT_OK;
    }
    if (knob == GAT_TUNE_SERVE_RESERVE) {
        if (value < 0 || value > 90) return fail(ctx, GAT_ERR_ARG, "gat_ctx_set_tuning: serve reserve must be 0..90");
        ctx->serve_reserve = value;
        return GAT_OK;
    }
    if (knob != GAT_TUNE_EDR_ROWS) return fail(ctx, GAT_ERR_ARG, "gat_ctx_set_tuning: unknown knob");
    if (value != 0 && value != 2 && value != 4 && value != 8)
        return fail(ctx, GAT_ERR_ARG, "gat_ctx_set_tuning: EDR rows per lane must be 0 (autotune), 2, 4 or 8");
    ctx->edr_rows = value;
    std::lock_guard<std::mutex> tk(ctx->tune_mu);
    ctx->edr_tune.clear();
    return GAT_OK;
}

int gat_ctx_get_tuning(gat_ctx* ctx, int knob, int* value) {
    if (!ctx || !value) return GAT_ERR_ARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (knob == GAT_TUNE_EDR_ROWS)
        *value = ctx->edr_rows;
    else if (knob == GAT_TUNE_EDR_TUNED) {
        std::lock_guard<std::mutex> tk(ctx->tune_mu);
        *value = (int)ctx->edr_tune.size();
    }
    else if (knob == GAT_TUNE_TOPK_CHUNK)
        *value = ctx->topk_chunk;
    else if (knob == GAT_TUNE_EDR_FORM)
        *value = ctx->edr_form;
    else if (knob == GAT_TUNE_TOPK_GROWTH)
        *value = ctx->topk_growth;
    else if (knob == GAT_TUNE_INDEX_BUILD)
        *value = ctx->index_build;
    else if (knob == GAT_TUNE_TEST_STALL_CARRY)
        *value = ctx->test_stall_pair;
    else if (knob == GAT_TUNE_DEP_LAUNCH)
        *value = ctx->dep_launch;
    else if (knob == GAT_TUNE_SERVE_RESERVE)
        *value = ctx->serve_reserve;
    else if (knob == GAT_TUNE_RANGE_SHAPE)
        *value = ctx->range_shape;
    else if (knob == GAT_TUNE_EDR_RESERVE)
        *value = ctx->edr_reserve_pct;
    else
        return fail(ctx, GAT_ERR_ARG, "gat_ctx_get_tuning: unknown knob");
    return GAT_OK;
}

int64_t gat_ctx_scratch_bytes(const gat_ctx* ctx) {
    if (!ctx) return 0;
    int64_t s = 0;
    if (ctx->build_pool) {
        /* the pool holds the scratch slots and the kept index-build temporaries */
        uint64_t held = 0;
        if (cudaMemPoolGetAttribute(ctx->build_pool, cudaMemPoolAttrReservedMemCurrent, &held) == cudaSuccess)
            s = (int64_t)held;
        return s;
    }
    for (size_t b : ctx->slot_bytes) s += (int64_t)b;
    return s;
}

int gat_db_create(gat_ctx* ctx, int n, const int32_t* lengths, const float* lon, const float* lat,
                  gat_db** out) {
    if (!ctx || !out || n < 0 || (n > 0 && (!lengths || !lon || !lat))) return fail(ctx, GAT_ERR_ARG, "gat_db_create: bad arguments");
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (ctx->device >= 0) cudaSetDevice(ctx->device);
    gat_db* db = new gat_db();
    db->ctx = ctx;
    db->n = n;
    db->h_len.assign(n + 1, 0);
    db->h_off.assign(n + 2, 0);
    for (int t = 1; t <= n; t++) {
        if (lengths[t - 1] < 0) {
            delete db;
            return fail(ctx, GAT_ERR_ARG, "gat_db_create: negative length");
        }
        db->h_len[t] = lengths[t - 1];
        db->h_off[t + 1] = db->h_off[t] + lengths[t - 1];
        if (lengths[t - 1] > db->maxlen) db->maxlen = lengths[t - 1];
    }
    db->npoints = db->h_off[n + 1];
    if (ctx->device < 0) {
        db->h_x.assign(lon, lon + db->npoints);
        db->h_y.assign(lat, lat + db->npoints);
        *out = db;
        return GAT_OK;
    }
    /* the host copies of the points are downloaded when a host builder or a snapshot needs them */
    db->host_pending = true;
    cudaError_t e;
    if ((e = cudaMalloc(&db->d_len, (n + 1) * sizeof(int32_t))) != cudaSuccess ||
        (e = cudaMalloc(&db->d_off, (n + 2) * sizeof(int64_t))) != cudaSuccess ||
        (e = cudaMalloc(&db->d_xy, (db->npoints + 1) * sizeof(float2))) != cudaSuccess ||
        (e = cudaMemcpy(db->d_len, db->h_len.data(), (n + 1) * sizeof(int32_t), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(db->d_off, db->h_off.data(), (n + 2) * sizeof(int64_t), cudaMemcpyHostToDevice)) != cudaSuccess) {
        int rc = cuda_fail(ctx, e, "gat_db_create");
        gat_db_destroy(db);
        return rc;
    }
    if (int rc = upload_set_points(ctx, lon, lat, db->npoints, db->d_xy)) {
        gat_db_destroy(db);
        return rc;
    }
    *out = db;
    return GAT_OK;
}

void gat_db_destroy(gat_db* db) {
    if (!db) return;
    if (db->ctx->device < 0) {
        delete db;
        return;
    }
    cudaSetDevice(db->ctx->device);
    cudaStreamSynchronize(db->ctx->stream);
    cudaFree(db->d_len);
    cudaFree(db->d_off);
    cudaFree(db->d_xy);
    delete db;
}

int gat_db_info(const gat_db* db, int64_t info[4]) {
    if (!db || !info) return GAT_ERR_ARG;
    info[0] = db->n;
    info[1] = db->npoints;
    info[2] = db->maxlen;
    info[3] = 0;
    return GAT_OK;
}

void gat_index_destroy(gat_index* ix) {
    if (!ix) return;
    if (ix->ctx->device < 0) {
        delete ix;
        return;
    }
    cudaSetDevice(ix->ctx->device);
    cudaStreamSynchronize(ix->ctx->stream);
    for (void* p : ix->allocs) cudaFree(p);
    if (ix->d_pidx) cudaFree(ix->d_pidx);
    if (ix->d_pbox) cudaFree(ix->d_pbox);
    delete ix;
}

int gat_index_info(const gat_index* ix, int64_t info[8]) {
    if (!ix || !info) return GAT_ERR_ARG;
    for (int i = 0; i < 8; i++) info[i] = 0;
    info[0] = ix->kind;
    info[1] = ix->npoints;
    info[2] = ix->leaves;
    info[3] = ix->nodes;
    if (ix->kind == GAT_INDEX_GRID || ix->kind == GAT_INDEX_MORTON) info[4] = info[5] = ix->grid.axis;
    if (ix->kind == GAT_INDEX_FSG) {
        info[4] = ix->fsg.nx;
        info[5] = ix->fsg.ny;
    }
    info[6] = (int64_t)ix->device_bytes;
    return GAT_OK;
}

int gat_index_points(gat_ctx* ctx, const gat_index* ix, int64_t n, float* x, float* y, int32_t* tid,
                     int32_t* pidx) {
    if (!ctx || !ix || n != ix->npoints) return fail(ctx, GAT_ERR_ARG, "gat_index_points: size mismatch");
    if (ix->kind == GAT_INDEX_MORTON) return gat_index_points(ctx, ix->base, n, x, y, tid, pidx); /* the Grid's order */
    {
        /* a device-placed index whose host copies were never asked for: read the device arrays */
        std::lock_guard<std::mutex> lk(const_cast<gat_index*>(ix)->host_mu);
        if (ix->host_pending) return index_points_device(ix, x, y, tid, pidx);
    }
    size_t b = (size_t)n * 4;
    if (x) memcpy(x, ix->h_x.data(), b);
    if (y) memcpy(y, ix->h_y.data(), b);
    if (tid) memcpy(tid, ix->h_tid.data(), b);
    if (pidx) memcpy(pidx, ix->h_pidx.data(), b);
    return GAT_OK;
}

}  // extern "C"
