/* Serving loop: continuous batching of range and top-k requests over device-resident indexes.
 *
 * The reference has no serving layer; its harness runs one batch per call (SystemTest.cpp).
 * Here requests arrive one at a time from any host thread. A scheduler thread forms batches as
 * soon as a lane is free: it takes the queue whose head request is oldest (range requests
 * grouped by index and result kind, top-k requests grouped by eps and run at the largest k of
 * the batch, each request keeping its own first k, which the canonical (distance, id) order
 * makes exact), and admits the batch only while the estimated device bytes of all admitted
 * batches stay within the budget. Each lane is a worker context (own stream, scratch arena and
 * host thread), so batches of different lanes overlap on the device, and requests that arrive
 * while others run join the next batch that a free lane and the budget allow. A request whose
 * estimate alone exceeds the budget fails with GAT_ERR_OOM. Per request the loop records
 * arrival, admission and completion times (ns since the server started).
 *
 * Estimates: range requests reserve 1 KB plus 16 bytes per expected result entry (a running
 * mean of the index's observed result sizes); top-k requests reserve 32 bytes per trajectory
 * of the set (lower bounds, candidate order, distances) plus 64 KB. After a batch, a lane
 * whose scratch arena exceeds its share of the budget (budget / lanes) frees it.
 *
 * Head-of-line blocking: a top-k batch runs for milliseconds, a range batch for well under one.
 * With two or more lanes, lane 0 runs range batches only, on a stream of the device's greatest
 * priority, so a range request never waits behind top-k work for a lane; the other lanes leave
 * an eighth of the SMs free of their persistent EDR grids, so the range kernels also find SMs
 * while top-k work runs (a persistent grid holds its SMs until it ends); and a top-k batch stops
 * growing once its queries hold kTopkBatchPoints points (its DP work grows with them), so one
 * batch of long queries cannot hold a lane for long. */
#include <algorithm>
#include <chrono>
#include <climits>
#include <condition_variable>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

#include "internal.h"

using namespace gat;

namespace {

enum { REQ_RANGE = 0, REQ_TOPK = 1 };
constexpr int64_t kTopkBatchPoints = 8192; /* query points per top-k batch (at least one request) */

struct Request {
    int64_t id = 0;
    int kind = REQ_RANGE;
    int index_kind = 0, result_kind = 0;
    gat_mbb box{};
    std::vector<float> lon, lat;
    int k = 0;
    double eps = 0;
    int64_t reserve = 0;
    int status = -1; /* -1 while pending */
    std::vector<int32_t> tid, pidx;   /* range result */
    std::vector<int32_t> ids, dist;   /* top-k result */
    int64_t t[3] = {0, 0, 0};          /* arrival, admission, completion */
};

/* Pinned host buffers of a lane. A copy between pageable host memory and the device goes
 * through the driver's staging buffer shared by all streams, so a lane whose copy waits for a
 * long top-k batch on its own stream held every other lane's copies back (range batches then
 * took as long as the top-k batch running beside them); copies from and to pinned memory are
 * plain DMA on the lane's own stream. Grown by doubling, freed with the server. */
struct PinnedArena {
    char* p = nullptr;
    size_t bytes = 0;
    std::vector<char> fallback; /* a context without a device (queries then fail anyway) */
    char* get(size_t b) {
        if (b <= bytes) return p;
        const size_t had = bytes;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        const size_t nb = std::max<size_t>(std::max<size_t>(b, 2 * had), (size_t)4 << 20);
        void* q = nullptr;
        if (cudaMallocHost(&q, nb) != cudaSuccess) {
            cudaGetLastError();
            fallback.resize(b);
            return fallback.data();
        }
        p = (char*)q;
        bytes = nb;
        return p;
    }
    ~PinnedArena() {
        if (p) cudaFreeHost(p);
    }
};
inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

struct Batch {
    int kind = REQ_RANGE;
    int index_kind = 0, result_kind = 0;
    std::vector<Request*> reqs;
    int64_t reserve = 0;
};

}  // namespace

struct gat_server {
    gat_ctx* ctx = nullptr;
    EdrChain chain; /* the top-k lanes' EDR grids, one at a time */
    const gat_index* ix[3] = {nullptr, nullptr, nullptr};
    gat_server_config cfg{};
    std::vector<gat_ctx*> lanes;
    std::vector<std::thread> workers;
    std::thread scheduler;
    std::mutex mu;
    std::condition_variable cv_sched, cv_lane, cv_done;
    std::deque<Request*> q_range[3][2];
    std::deque<Request*> q_topk;
    std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
    std::vector<Batch*> lane_batch;
    int64_t next_id = 0;
    int64_t reserved = 0;
    /* a free lane for a batch of this kind, or -1: with two or more lanes, lane 0 takes range
     * batches only (and is preferred for them) */
    int lane_for(int kind) const {
        const int L = (int)lane_batch.size();
        if (L < 2) return lane_batch[0] ? -1 : 0;
        if (kind == REQ_RANGE && !lane_batch[0]) return 0;
        for (int i = 1; i < L; i++)
            if (!lane_batch[i]) return i;
        return -1;
    }
    bool stopping = false, lanes_stop = false;
    double hits_mean[3] = {4096, 4096, 4096};
    int64_t stats[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    int64_t now() const {
        return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count();
    }
    bool pending() const {
        if (!q_topk.empty()) return true;
        for (auto& a : q_range)
            for (auto& q : a)
                if (!q.empty()) return true;
        return false;
    }
    int free_lane() const {
        for (size_t i = 0; i < lane_batch.size(); i++)
            if (!lane_batch[i]) return (int)i;
        return -1;
    }
    bool idle() const {
        for (Batch* b : lane_batch)
            if (b) return false;
        return true;
    }
    int64_t range_reserve(int ik, int rk) const {
        return 1024 + (int64_t)(hits_mean[ik] * (rk == GAT_RESULT_POINTS ? 16.0 : 8.0)) * 2;
    }
    int64_t topk_reserve() const {
        const int n = ix[GAT_INDEX_GRID] ? ix[GAT_INDEX_GRID]->db->n : 0;
        return (int64_t)n * 32 + (64 << 10);
    }
    void finish(Request* r, int status) {
        r->status = status;
        r->t[2] = now();
        stats[1]++;
        if (status != GAT_OK) stats[7]++;
    }
    /* Pops the next batch (lock held). Returns nullptr when nothing fits the budget now. */
    Batch* form_batch() {
        std::deque<Request*>* best = nullptr;
        int64_t best_t = INT64_MAX;
        if (!q_topk.empty() && lane_for(REQ_TOPK) >= 0) {
            best = &q_topk;
            best_t = q_topk.front()->t[0];
        }
        for (auto& a : q_range)
            for (auto& q : a)
                if (!q.empty() && q.front()->t[0] < best_t) {
                    best = &q;
                    best_t = q.front()->t[0];
                }
        if (!best) return nullptr;
        Request* head = best->front();
        const int limit = head->kind == REQ_TOPK ? cfg.max_topk_batch : cfg.max_range_batch;
        auto* b = new Batch();
        b->kind = head->kind;
        b->index_kind = head->index_kind;
        b->result_kind = head->result_kind;
        int64_t points = 0;
        for (auto it = best->begin(); it != best->end() && (int)b->reqs.size() < limit;) {
            Request* r = *it;
            if (r->kind == REQ_TOPK && r->eps != head->eps) {
                ++it;
                continue;
            }
            if (r->kind == REQ_TOPK) {
                if (!b->reqs.empty() && points + (int64_t)r->lon.size() > kTopkBatchPoints) break;
                points += (int64_t)r->lon.size();
            }
            if (reserved + b->reserve + r->reserve > cfg.budget_bytes) {
                if (r->reserve > cfg.budget_bytes) { /* can never fit */
                    finish(r, GAT_ERR_OOM);
                    it = best->erase(it);
                    cv_done.notify_all();
                    continue;
                }
                break;
            }
            b->reserve += r->reserve;
            b->reqs.push_back(r);
            it = best->erase(it);
        }
        if (b->reqs.empty()) {
            delete b;
            return nullptr;
        }
        return b;
    }

    void run_scheduler() {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv_sched.wait(lk, [&] { return (pending() && free_lane() >= 0) || (stopping && !pending()); });
            if (stopping && !pending()) break;
            Batch* b = form_batch();
            if (!b) {
                /* the head does not fit next to the admitted batches: wait for a completion */
                if (!idle()) cv_sched.wait(lk);
                continue;
            }
            const int lane = lane_for(b->kind);
            const int64_t t = now();
            for (Request* r : b->reqs) r->t[1] = t;
            reserved += b->reserve;
            stats[5] = std::max(stats[5], reserved);
            stats[6] = std::max<int64_t>(stats[6], (int64_t)b->reqs.size());
            stats[2]++;
            stats[b->kind == REQ_TOPK ? 4 : 3]++;
            lane_batch[lane] = b;
            cv_lane.notify_all();
        }
        /* drained: stop the lanes once they are idle */
        cv_sched.wait(lk, [&] { return idle(); });
        lanes_stop = true;
        cv_lane.notify_all();
    }

    void run_range(gat_ctx* w, PinnedArena& pa, Batch* b) {
        const int n = (int)b->reqs.size();
        int64_t cap = std::max<int64_t>(1024, (int64_t)(hits_mean[b->index_kind] * n * 1.5)), need = 0;
        const bool pts = b->result_kind == GAT_RESULT_POINTS;
        gat_mbb* q = nullptr;
        int64_t* off = nullptr;
        int32_t *tid = nullptr, *pidx = nullptr;
        int rc = GAT_OK;
        for (int attempt = 0; attempt < 2; attempt++) {
            /* [queries | offsets | ids | point indexes] in the lane's pinned buffer */
            const size_t bq = align256((size_t)n * sizeof(gat_mbb)), bo = align256((size_t)(n + 1) * 8);
            const size_t bt = align256((size_t)cap * 4);
            char* base = pa.get(bq + bo + bt + (pts ? bt : 0));
            q = reinterpret_cast<gat_mbb*>(base);
            off = reinterpret_cast<int64_t*>(base + bq);
            tid = reinterpret_cast<int32_t*>(base + bq + bo);
            pidx = pts ? reinterpret_cast<int32_t*>(base + bq + bo + bt) : nullptr;
            for (int i = 0; i < n; i++) q[i] = b->reqs[i]->box;
            rc = gat_range_query(w, ix[b->index_kind], q, n, b->result_kind, GAT_EXEC_BATCHED, off, tid, pidx, cap, &need);
            if (rc != GAT_ERR_TRUNCATED) break;
            cap = need;
        }
        std::lock_guard<std::mutex> lk(mu);
        for (int i = 0; i < n; i++) {
            Request* r = b->reqs[i];
            if (rc == GAT_OK) {
                r->tid.assign(tid + off[i], tid + off[i + 1]);
                if (pts) r->pidx.assign(pidx + off[i], pidx + off[i + 1]);
            }
            finish(r, rc);
        }
        if (rc == GAT_OK && n > 0)
            hits_mean[b->index_kind] = 0.8 * hits_mean[b->index_kind] + 0.2 * std::max(1.0, (double)off[n] / n);
    }

    void run_topk(gat_ctx* w, PinnedArena& pa, Batch* b) {
        const int n = (int)b->reqs.size();
        int kmax = 0;
        size_t points = 0;
        for (Request* r : b->reqs) {
            kmax = std::max(kmax, r->k);
            points += r->lon.size();
        }
        /* [lengths | lon | lat | ids | distances] in the lane's pinned buffer */
        const size_t bl = align256((size_t)n * 4), bp = align256(points * 4), br = align256((size_t)n * kmax * 4);
        char* base = pa.get(bl + 2 * bp + 2 * br);
        int32_t* len = reinterpret_cast<int32_t*>(base);
        float* lon = reinterpret_cast<float*>(base + bl);
        float* lat = reinterpret_cast<float*>(base + bl + bp);
        int32_t* ids = reinterpret_cast<int32_t*>(base + bl + 2 * bp);
        int32_t* dist = reinterpret_cast<int32_t*>(base + bl + 2 * bp + br);
        size_t at = 0;
        for (int i = 0; i < n; i++) {
            Request* r = b->reqs[i];
            len[i] = (int32_t)r->lon.size();
            std::copy(r->lon.begin(), r->lon.end(), lon + at);
            std::copy(r->lat.begin(), r->lat.end(), lat + at);
            at += r->lon.size();
        }
        int rc = gat_topk(w, ix[GAT_INDEX_GRID], n, len, lon, lat, kmax, b->reqs[0]->eps, GAT_EXEC_BATCHED, ids, dist,
                          nullptr);
        std::lock_guard<std::mutex> lk(mu);
        for (int i = 0; i < n; i++) {
            Request* r = b->reqs[i];
            if (rc == GAT_OK) {
                r->ids.assign(ids + (size_t)i * kmax, ids + (size_t)i * kmax + r->k);
                r->dist.assign(dist + (size_t)i * kmax, dist + (size_t)i * kmax + r->k);
            }
            finish(r, rc);
        }
    }

    void run_lane(int i) {
        gat_ctx* w = lanes[i];
        if (w->device >= 0) cudaSetDevice(w->device);
        PinnedArena pa;
        for (;;) {
            Batch* b = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_lane.wait(lk, [&] { return lane_batch[i] != nullptr || lanes_stop; });
                if (!lane_batch[i]) break;
                b = lane_batch[i];
            }
            if (b->kind == REQ_TOPK)
                run_topk(w, pa, b);
            else
                run_range(w, pa, b);
            if (gat_ctx_scratch_bytes(w) > cfg.budget_bytes / (int64_t)lanes.size()) gat_ctx_trim(w);
            std::lock_guard<std::mutex> lk(mu);
            reserved -= b->reserve;
            lane_batch[i] = nullptr;
            delete b;
            cv_done.notify_all();
            cv_sched.notify_all();
        }
    }
};

namespace {
Request* find(gat_server* s, int64_t id) {
    auto it = s->reqs.find(id);
    return it == s->reqs.end() ? nullptr : it->second.get();
}
}  // namespace

extern "C" {

int gat_server_create(gat_ctx* ctx, const gat_index* grid, const gat_index* stig, const gat_index* fsg,
                      const gat_server_config* cfg, gat_server** out) {
    if (!ctx || !out || (!grid && !stig && !fsg)) return GAT_ERR_ARG;
    *out = nullptr;
    const gat_index* ixs[3] = {grid, stig, fsg};
    for (int k = 0; k < 3; k++)
        if (ixs[k] && (ixs[k]->kind != k || !same_owner(ixs[k]->ctx, ctx)))
            return fail(ctx, GAT_ERR_ARG, "gat_server_create: index kind or owner mismatch");
    gat_server_config c{4, (int64_t)40 << 30, 4096, 32};
    if (cfg) c = *cfg;
    if (c.lanes < 1 || c.lanes > 64 || c.budget_bytes <= 0 || c.max_range_batch < 1 || c.max_topk_batch < 1)
        return fail(ctx, GAT_ERR_ARG, "gat_server_create: bad configuration");
    auto* s = new gat_server();
    s->ctx = ctx;
    for (int k = 0; k < 3; k++) s->ix[k] = ixs[k];
    s->cfg = c;
    for (int i = 0; i < c.lanes; i++) {
        gat_ctx* w = nullptr;
        int rc = gat_ctx_create_worker(ctx, &w);
        if (rc != GAT_OK) {
            for (gat_ctx* x : s->lanes) gat_ctx_destroy(x);
            if (s->chain.ev) cudaEventDestroy(s->chain.ev);
            delete s;
            return fail(ctx, rc, "gat_server_create: worker context");
        }
        /* lane 0 takes range batches on a high-priority stream; the others leave SMs to it and
         * run their EDR grids one at a time */
        if (c.lanes >= 2) {
            if (i == 0) {
                rc = ctx_use_priority_stream(w);
            } else {
                const int pct = ctx->serve_reserve > 0 ? ctx->serve_reserve : 12;
                w->sm_reserve = std::max(1, w->sm_count * pct / 100);
                w->edr_reserve_pct = pct;
                if (w->device >= 0) {
                    if (!s->chain.ev && cudaEventCreateWithFlags(&s->chain.ev, cudaEventDisableTiming) != cudaSuccess) {
                        cudaGetLastError();
                        rc = GAT_ERR_CUDA;
                    }
                    w->edr_chain = &s->chain;
                }
            }
        }
        s->lanes.push_back(w);
        if (rc != GAT_OK) {
            for (gat_ctx* x : s->lanes) gat_ctx_destroy(x);
            if (s->chain.ev) cudaEventDestroy(s->chain.ev);
            delete s;
            return fail(ctx, rc, "gat_server_create: lane stream");
        }
    }
    s->lane_batch.assign((size_t)c.lanes, nullptr);
    for (int i = 0; i < c.lanes; i++) s->workers.emplace_back([s, i] { s->run_lane(i); });
    s->scheduler = std::thread([s] { s->run_scheduler(); });
    *out = s;
    return GAT_OK;
}

void gat_server_destroy(gat_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_sched.notify_all();
    s->scheduler.join();
    for (auto& t : s->workers) t.join();
    for (gat_ctx* w : s->lanes) gat_ctx_destroy(w);
    if (s->chain.ev) cudaEventDestroy(s->chain.ev);
    delete s;
}

int gat_server_submit_range(gat_server* s, int index_kind, gat_mbb box, int result_kind, int64_t* id) {
    if (!s || !id || index_kind < 0 || index_kind > 2 || !s->ix[index_kind] ||
        (result_kind != GAT_RESULT_IDS && result_kind != GAT_RESULT_POINTS))
        return GAT_ERR_ARG;
    auto r = std::make_unique<Request>();
    r->kind = REQ_RANGE;
    r->index_kind = index_kind;
    r->result_kind = result_kind;
    r->box = box;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) return GAT_ERR_STATE;
        r->id = s->next_id++;
        r->t[0] = s->now();
        r->reserve = s->range_reserve(index_kind, result_kind);
        *id = r->id;
        s->q_range[index_kind][result_kind].push_back(r.get());
        s->reqs[r->id] = std::move(r);
        s->stats[0]++;
    }
    s->cv_sched.notify_all();
    return GAT_OK;
}

int gat_server_submit_topk(gat_server* s, int q_len, const float* lon, const float* lat, int k, double eps,
                           int64_t* id) {
    if (!s || !id || q_len < 1 || q_len > GAT_EDR_MAX_LEN || !lon || !lat || k < 1 || !(eps > 0) ||
        !s->ix[GAT_INDEX_GRID])
        return GAT_ERR_ARG;
    if (k > s->ix[GAT_INDEX_GRID]->db->n) return GAT_ERR_ARG;
    auto r = std::make_unique<Request>();
    r->kind = REQ_TOPK;
    r->lon.assign(lon, lon + q_len);
    r->lat.assign(lat, lat + q_len);
    r->k = k;
    r->eps = eps;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) return GAT_ERR_STATE;
        r->id = s->next_id++;
        r->t[0] = s->now();
        r->reserve = s->topk_reserve();
        *id = r->id;
        s->q_topk.push_back(r.get());
        s->reqs[r->id] = std::move(r);
        s->stats[0]++;
    }
    s->cv_sched.notify_all();
    return GAT_OK;
}

int gat_server_wait(gat_server* s, int64_t id, int timeout_ms, int* req_status) {
    if (!s) return GAT_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    Request* r = find(s, id);
    if (!r) return GAT_ERR_ARG;
    auto done = [&] { return r->status != -1; };
    if (timeout_ms < 0)
        s->cv_done.wait(lk, done);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done))
        return GAT_ERR_TIMEOUT;
    if (req_status) *req_status = r->status;
    return GAT_OK;
}

int gat_server_range_result(gat_server* s, int64_t id, int32_t* tids, int32_t* pidx, int64_t capacity,
                            int64_t* count) {
    if (!s || !count) return GAT_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    Request* r = find(s, id);
    if (!r || r->kind != REQ_RANGE) return GAT_ERR_ARG;
    if (r->status == -1) return GAT_ERR_STATE;
    if (r->status != GAT_OK) return r->status;
    *count = (int64_t)r->tid.size();
    if (capacity < *count) return GAT_ERR_TRUNCATED;
    if (tids) std::copy(r->tid.begin(), r->tid.end(), tids);
    if (pidx && r->result_kind == GAT_RESULT_POINTS) std::copy(r->pidx.begin(), r->pidx.end(), pidx);
    return GAT_OK;
}

int gat_server_topk_result(gat_server* s, int64_t id, int32_t* ids, int32_t* dist, int capacity) {
    if (!s) return GAT_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    Request* r = find(s, id);
    if (!r || r->kind != REQ_TOPK) return GAT_ERR_ARG;
    if (r->status == -1) return GAT_ERR_STATE;
    if (r->status != GAT_OK) return r->status;
    if (capacity < r->k) return GAT_ERR_TRUNCATED;
    if (ids) std::copy(r->ids.begin(), r->ids.end(), ids);
    if (dist) std::copy(r->dist.begin(), r->dist.end(), dist);
    return GAT_OK;
}

int gat_server_request_times(gat_server* s, int64_t id, int64_t t[3]) {
    if (!s || !t) return GAT_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    Request* r = find(s, id);
    if (!r) return GAT_ERR_ARG;
    for (int i = 0; i < 3; i++) t[i] = r->t[i];
    return GAT_OK;
}

int gat_server_release(gat_server* s, int64_t id) {
    if (!s) return GAT_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    Request* r = find(s, id);
    if (!r) return GAT_ERR_ARG;
    if (r->status == -1) return GAT_ERR_STATE;
    s->reqs.erase(id);
    return GAT_OK;
}

int gat_server_stats(gat_server* s, int64_t out[8]) {
    if (!s || !out) return GAT_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    for (int i = 0; i < 8; i++) out[i] = s->stats[i];
    return GAT_OK;
}

}  // extern "C"
