/* Index snapshots: a built index written to a file and loaded back without rebuilding (a
 * serving process restarts in the time it takes to read and upload the arrays instead of
 * sorting the set again). The file holds the index's parameters, every device array in the
 * order the builder uploaded it, the point-index array the host keeps, and a hash of the
 * trajectory set it was built over; loading checks the hash against the given set.
 *
 * Layout (little-endian, this build's struct layouts):
 *   "GATIDX01" | u32 version | i32 kind | i32 n | i64 npoints | i32 maxlen | u64 set hash |
 *   i32 pidx_bits | i64 leaves | i64 nodes | i32 fv_max_nnz | i64 fv_entries |
 *   GridDev | StigDev | FsgDev (raw; their pointers are replaced on load) |
 *   u32 arrays | (u64 bytes, bytes)* | u64 pidx count | pidx | u64 checksum of all preceding bytes */
#include <cstdio>
#include <cstring>
#include <thread>

#include "internal.h"

using namespace gat;

namespace {

constexpr char kMagic[8] = {'G', 'A', 'T', 'I', 'D', 'X', '0', '1'};
constexpr uint32_t kVersion = 1;

uint64_t mix(uint64_t h, uint64_t v) {
    h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
    return h * 0xff51afd7ed558ccdull;
}

uint64_t hash_bytes(const void* p, size_t n, uint64_t h) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t v;
        memcpy(&v, b + i, 8);
        h = mix(h, v);
    }
    uint64_t tail = 0;
    if (i < n) memcpy(&tail, b + i, n - i);
    return mix(h, tail ^ (uint64_t)n);
}

/* the trajectory set's content: lengths and coordinates, hashed in 8 parallel slices */
uint64_t set_hash(const gat_db* db) {
    uint64_t h = hash_bytes(db->h_len.data(), db->h_len.size() * 4, 0x5ca1ab1eull ^ (uint64_t)db->n);
    const size_t np = db->h_x.size();
    constexpr int kParts = 8;
    uint64_t part[kParts] = {};
    std::vector<std::thread> th;
    for (int k = 0; k < kParts; k++)
        th.emplace_back([&, k] {
            const size_t a = np * k / kParts, b = np * (k + 1) / kParts;
            uint64_t x = hash_bytes(db->h_x.data() + a, (b - a) * 4, 0x1234 + k);
            part[k] = hash_bytes(db->h_y.data() + a, (b - a) * 4, x);
        });
    for (auto& t : th) t.join();
    for (int k = 0; k < kParts; k++) h = mix(h, part[k]);
    return h;
}

/* the device pointer fields of an index in upload order */
std::vector<void**> fields(gat_index* ix) {
    std::vector<void**> f = {(void**)&ix->d_x, (void**)&ix->d_y, (void**)&ix->d_tid, (void**)&ix->d_key};
    if (ix->kind == GAT_INDEX_GRID) {
        GridDev& g = ix->grid;
        for (void** p : {(void**)&g.node_mbb, (void**)&g.node_child, (void**)&g.node_pbeg, (void**)&g.node_pend,
                         (void**)&ix->d_fv_off, (void**)&ix->d_fv_cell, (void**)&ix->d_fv_cnt})
            f.push_back(p);
    } else if (ix->kind == GAT_INDEX_STIG) {
        StigDev& d = ix->stig;
        for (void** p : {(void**)&d.kind, (void**)&d.dim, (void**)&d.median, (void**)&d.left, (void**)&d.right,
                         (void**)&d.lo, (void**)&d.hi, (void**)&d.mbb})
            f.push_back(p);
    } else {
        for (void** p : {(void**)&ix->fsg.cbeg, (void**)&ix->fsg.cend}) f.push_back(p);
    }
    return f;
}

struct Out {
    FILE* f;
    uint64_t h = 0x0ddba11ull;
    bool ok = true;
    void put(const void* p, size_t n) {
        if (!ok || n == 0) return;
        ok = fwrite(p, 1, n, f) == n;
        h = hash_bytes(p, n, h);
    }
    template <class T>
    void val(const T& v) {
        put(&v, sizeof(T));
    }
};

struct In {
    FILE* f;
    uint64_t h = 0x0ddba11ull;
    bool ok = true;
    void get(void* p, size_t n) {
        if (!ok || n == 0) return;
        ok = fread(p, 1, n, f) == n;
        if (ok) h = hash_bytes(p, n, h);
    }
    template <class T>
    T val() {
        T v{};
        get(&v, sizeof(T));
        return v;
    }
};

}  // namespace

extern "C" {

int gat_index_save(gat_ctx* ctx, const gat_index* index, const char* path) {
    if (!ctx || !index || !path) return fail(ctx, GAT_ERR_ARG, "gat_index_save: bad arguments");
    if (int rq = require_device(ctx, "gat_index_save")) return rq;
    if (!same_owner(index->ctx, ctx)) return fail(ctx, GAT_ERR_STATE, "gat_index_save: index from another context");
    if (index->kind == GAT_INDEX_MORTON)
        return fail(ctx, GAT_ERR_ARG, "gat_index_save: a MortonGrid is not saved; save its Grid and rebuild it");
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    gat_index* ix = const_cast<gat_index*>(index);
    if (ix->allocs.size() != fields(ix).size())
        return fail(ctx, GAT_ERR_STATE, "gat_index_save: the index's arrays do not match its kind");
    if (int st = index_host_copies(ix)) return st;
    if (int st = db_host_copies(ix->db)) return st;
    FILE* f = fopen(path, "wb");
    if (!f) return fail(ctx, GAT_ERR_ARG, std::string("gat_index_save: cannot open ") + path);
    Out o{f};
    const gat_db* db = ix->db;
    o.put(kMagic, 8);
    o.val(kVersion);
    o.val<int32_t>(ix->kind);
    o.val<int32_t>(db->n);
    o.val<int64_t>(ix->npoints);
    o.val<int32_t>(db->maxlen);
    o.val<uint64_t>(set_hash(db));
    o.val<int32_t>(ix->pidx_bits);
    o.val<int64_t>(ix->leaves);
    o.val<int64_t>(ix->nodes);
    o.val<int32_t>(ix->fv_max_nnz);
    o.val<int64_t>(ix->fv_entries);
    o.val(ix->grid);
    o.val(ix->stig);
    o.val(ix->fsg);
    o.val<uint32_t>((uint32_t)ix->allocs.size());
    std::vector<char> buf;
    int st = GAT_OK;
    for (size_t i = 0; i < ix->allocs.size() && o.ok; i++) {
        buf.resize(ix->alloc_bytes[i]);
        cudaError_t e = cudaMemcpy(buf.data(), ix->allocs[i], buf.size(), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            st = cuda_fail(ctx, e, "gat_index_save");
            break;
        }
        o.val<uint64_t>(buf.size());
        o.put(buf.data(), buf.size());
    }
    o.val<uint64_t>(ix->h_pidx.size());
    o.put(ix->h_pidx.data(), ix->h_pidx.size() * 4);
    const uint64_t sum = o.h;
    if (o.ok) o.ok = fwrite(&sum, 8, 1, f) == 1;
    const bool closed = fclose(f) == 0;
    if (st != GAT_OK) return st;
    if (!o.ok || !closed) return fail(ctx, GAT_ERR_ARG, std::string("gat_index_save: write failed: ") + path);
    return GAT_OK;
}

int gat_index_load(gat_ctx* ctx, const gat_db* db, const char* path, gat_index** out) {
    if (!ctx || !db || !path || !out) return fail(ctx, GAT_ERR_ARG, "gat_index_load: bad arguments");
    if (db->ctx != ctx) return fail(ctx, GAT_ERR_STATE, "gat_index_load: trajectory set from another context");
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (ctx->device >= 0) cudaSetDevice(ctx->device);
    if (int st = db_host_copies(db)) return st;
    FILE* f = fopen(path, "rb");
    if (!f) return fail(ctx, GAT_ERR_ARG, std::string("gat_index_load: cannot open ") + path);
    In in{f};
    auto bad = [&](const char* why) {
        fclose(f);
        return fail(ctx, GAT_ERR_ARG, std::string("gat_index_load: ") + why);
    };
    char magic[8];
    in.get(magic, 8);
    if (!in.ok || memcmp(magic, kMagic, 8) != 0 || in.val<uint32_t>() != kVersion) return bad("not an index snapshot");
    gat_index* ix = new gat_index();
    ix->ctx = ctx;
    ix->db = db;
    ix->kind = in.val<int32_t>();
    const int32_t n = in.val<int32_t>();
    ix->npoints = in.val<int64_t>();
    const int32_t maxlen = in.val<int32_t>();
    const uint64_t hash = in.val<uint64_t>();
    if (!in.ok || ix->kind < 0 || ix->kind > 2 || n != db->n || ix->npoints != db->npoints || maxlen != db->maxlen ||
        hash != set_hash(db)) {
        delete ix;
        return bad("the snapshot was taken over another trajectory set");
    }
    ix->pidx_bits = in.val<int32_t>();
    ix->leaves = in.val<int64_t>();
    ix->nodes = in.val<int64_t>();
    ix->fv_max_nnz = in.val<int32_t>();
    ix->fv_entries = in.val<int64_t>();
    ix->grid = in.val<GridDev>();
    ix->stig = in.val<StigDev>();
    ix->fsg = in.val<FsgDev>();
    /* derived arrays are recomputed below, never read from the file */
    ix->grid.node_pbox = nullptr;
    ix->stig.pbox = nullptr;
    std::vector<void**> fl = fields(ix);
    if (in.val<uint32_t>() != fl.size() || !in.ok) {
        delete ix;
        return bad("array count does not match the index kind");
    }
    std::vector<std::vector<char>> host(fl.size());
    for (size_t i = 0; i < fl.size() && in.ok; i++) {
        const uint64_t bytes = in.val<uint64_t>();
        if (!in.ok || bytes > ((uint64_t)1 << 40)) {
            in.ok = false;
            break;
        }
        host[i].resize(bytes);
        in.get(host[i].data(), bytes);
    }
    const uint64_t np = in.val<uint64_t>();
    if (in.ok && np == (uint64_t)ix->npoints) {
        ix->h_pidx.resize(np);
        in.get(ix->h_pidx.data(), np * 4);
    } else {
        in.ok = false;
    }
    const uint64_t want = in.h;
    uint64_t sum = 0;
    const bool sum_ok = in.ok && fread(&sum, 8, 1, f) == 1 && sum == want;
    fclose(f);
    const size_t pts = (size_t)ix->npoints;
    if (!sum_ok || host[0].size() < pts * 4 || host[1].size() < pts * 4 || host[2].size() < pts * 4) {
        delete ix;
        return fail(ctx, GAT_ERR_ARG, "gat_index_load: truncated or corrupted snapshot");
    }
    /* host copies the queries and gat_index_points use */
    ix->h_x.assign((const float*)host[0].data(), (const float*)host[0].data() + pts);
    ix->h_y.assign((const float*)host[1].data(), (const float*)host[1].data() + pts);
    ix->h_tid.assign((const int32_t*)host[2].data(), (const int32_t*)host[2].data() + pts);
    if (ctx->device >= 0) {
        for (size_t i = 0; i < fl.size(); i++) {
            int st = GAT_OK;
            void* p = index_alloc(ix, host[i].size(), &st);
            if (!p) {
                gat_index_destroy(ix);
                return st;
            }
            cudaError_t e = cudaMemcpy(p, host[i].data(), host[i].size(), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                gat_index_destroy(ix);
                return cuda_fail(ctx, e, "gat_index_load");
            }
            *fl[i] = p;
        }
        if (int st = index_point_boxes(ix)) {
            gat_index_destroy(ix);
            return st;
        }
    }
    *out = ix;
    return GAT_OK;
}

}  // extern "C"
