/* C++ host layer over the C ABI of gat_b200.h: the reference's harness classes (SystemTest.h,
 * Grid.h, STIG.h, FSG.h, MBB.h, Trajectory.h, SamplePoint.h) with their names and argument
 * meaning, so a GAT host program switches by changing includes and the namespace. Header-only;
 * link against libgat_b200.so. Every call goes through the C ABI.
 *
 *   gat::Context ctx(0);
 *   gat::Grid g(ctx, gat::MBB(121, 30.7, 122, 31.7), 0.0025f, 2);
 *   g.addDatasetToGrid(tradb, n);               // tradb[1..n], as the reference's (Grid.cpp:218)
 *   gat::STIG stig(ctx);  stig.initial(10240, 2, tradb, n);
 *   gat::FSG fsg(ctx, gat::MBB(121, 30.7, 122, 31.7), 0.01f);  fsg.addDatasetToGrid(tradb, n);
 *   gat::SystemTest st(tradb, &g, &stig, &fsg);
 *   st.rangeQueryTest(gat::MBB(121.4, 31.0, 121.5, 31.1), 1000);
 *   st.similarityQueryTest(47, 16, 32);         // README form: query = trajectory 47
 *
 * Differences from the reference: results are returned (lastRange / lastTopk) rather than only
 * timed; top-k ids come sorted by (distance, id) with their distances; one GPU (the context's).
 * Constructors throw gat::Error when the library refuses; query methods return its status. */
#ifndef GAT_B200_HPP
#define GAT_B200_HPP

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "gat_b200.h"

namespace gat {

class Error : public std::runtime_error {
public:
    Error(int status, const std::string& what) : std::runtime_error(what), status(status) {}
    int status;
};

/* MBB.h:2-13: same fields in the same order (layout-compatible with gat_mbb). */
struct MBB {
    float xmin = 0.f, ymin = 0.f, xmax = 0.f, ymax = 0.f;
    MBB() = default;
    MBB(float val_xmin, float val_ymin, float val_xmax, float val_ymax)
        : xmin(val_xmin), ymin(val_ymin), xmax(val_xmax), ymax(val_ymax) {}
    /* MBB::pInBox (MBB.cpp:21-26): inclusive on every side */
    bool pInBox(float x, float y) const { return x <= xmax && x >= xmin && y <= ymax && y >= ymin; }
    gat_mbb c() const { return gat_mbb{xmin, ymin, xmax, ymax}; }
};

/* SamplePoint.h:5-20 */
struct SamplePoint {
    float lon = 0.f, lat = 0.f;
    int time = 0, tid = 0;
    SamplePoint() = default;
    SamplePoint(float lon1, float lat1, int time1, int tid1) : lon(lon1), lat(lat1), time(time1), tid(tid1) {}
};

/* Trajectory.h:8-29 (points and length; the reader's bookkeeping fields are not needed) */
struct Trajectory {
    int tid = 0;
    std::vector<SamplePoint> points;
    int length = 0;
    Trajectory() = default;
    explicit Trajectory(int tid_) : tid(tid_) {}
    int addSamplePoints(float lon, float lat, int time) {
        points.emplace_back(lon, lat, time, tid);
        length = (int)points.size();
        return 0;
    }
};

inline void check(gat_ctx* ctx, int rc, const char* what) {
    if (rc != GAT_OK) {
        const char* m = ctx ? gat_last_error(ctx) : nullptr;
        throw Error(rc, std::string(what) + ": " + (m ? m : "failed"));
    }
}

/* One device (device < 0: host-only, index layouts without a GPU). */
class Context {
public:
    explicit Context(int device = 0) {
        int rc = gat_ctx_create(device, &h);
        if (rc != GAT_OK) throw Error(rc, "gat_ctx_create failed");
    }
    ~Context() {
        if (h) gat_ctx_destroy(h);
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    /* tuning knobs (GAT_TUNE_*); results never depend on them */
    void setTuning(int knob, int value) {
        int rc = gat_ctx_set_tuning(h, knob, value);
        if (rc != GAT_OK) throw Error(rc, gat_last_error(h));
    }
    int tuning(int knob) const {
        int v = 0;
        int rc = gat_ctx_get_tuning(h, knob, &v);
        if (rc != GAT_OK) throw Error(rc, gat_last_error(h));
        return v;
    }
    /* returns the scratch arena and kept index-build temporaries to the device */
    void trim() {
        int rc = gat_ctx_trim(h);
        if (rc != GAT_OK) throw Error(rc, gat_last_error(h));
    }
    gat_ctx* h = nullptr;
};

/* The trajectory set tradb[1..n] (tradb[0] unused), uploaded once and shared by indexes. */
class TrajectorySet {
public:
    TrajectorySet(Context& ctx, const Trajectory* db, int traNum) : ctx_(ctx) {
        std::vector<int32_t> len(traNum);
        std::vector<float> lon, lat;
        for (int t = 1; t <= traNum; t++) {
            len[t - 1] = (int32_t)db[t].points.size();
            for (const SamplePoint& p : db[t].points) {
                lon.push_back(p.lon);
                lat.push_back(p.lat);
            }
        }
        check(ctx.h, gat_db_create(ctx.h, traNum, len.data(), lon.data(), lat.data(), &h), "gat_db_create");
    }
    ~TrajectorySet() {
        if (h) gat_db_destroy(h);
    }
    TrajectorySet(const TrajectorySet&) = delete;
    TrajectorySet& operator=(const TrajectorySet&) = delete;
    gat_db* h = nullptr;

private:
    Context& ctx_;
};

class Index {
public:
    virtual ~Index() {
        if (h) gat_index_destroy(h);
        delete db_;
    }
    Index(const Index&) = delete;
    Index& operator=(const Index&) = delete;
    gat_index* h = nullptr;
    Context& ctx;
    int kind;

protected:
    Index(Context& c, int k) : ctx(c), kind(k) {}
    void set_db(const Trajectory* db, int traNum) {
        delete db_;
        db_ = nullptr;
        db_ = new TrajectorySet(ctx, db, traNum);
    }
    TrajectorySet* db_ = nullptr;
};

/* Grid.h:39 Grid(range, cell_size, VITURAL_CELL_PARAM) + addDatasetToGrid (Grid.h:42): the
 * GT-quadtree (leaves below leafCap points, MAXPOINTINNODE) with the FVTable for top-k. */
class Grid : public Index {
public:
    Grid(Context& c, const MBB& mbb, float val_cell_size, int VITURAL_CELL_PARAM = 2, int leafCap = 512)
        : Index(c, GAT_INDEX_GRID), range(mbb), cell_size(val_cell_size), vparam(VITURAL_CELL_PARAM), leaf_cap(leafCap) {}
    int addDatasetToGrid(const Trajectory* db, int traNum) {
        set_db(db, traNum);
        return gat_grid_build(ctx.h, db_->h, range.c(), cell_size, vparam, leaf_cap, &h);
    }
    MBB range;
    float cell_size;
    int vparam, leaf_cap;
};

/* STIG.h:57 initial(blockSize, dim, data, trajNum) (dim is 2: x/y kd-tree) */
class STIG : public Index {
public:
    explicit STIG(Context& c) : Index(c, GAT_INDEX_STIG) {}
    int initial(int blockSize, int dim, const Trajectory* data, int trajNum) {
        if (dim != 2) return GAT_ERR_ARG;
        set_db(data, trajNum);
        return gat_stig_build(ctx.h, db_->h, blockSize, &h);
    }
};

/* FSG.h:35 FSG(range, cell_size) + addDatasetToGrid (FSG.h:38) */
class FSG : public Index {
public:
    FSG(Context& c, const MBB& mbb, float val_cell_size) : Index(c, GAT_INDEX_FSG), range(mbb), cell_size(val_cell_size) {}
    int addDatasetToGrid(const Trajectory* db, int traNum) {
        set_db(db, traNum);
        return gat_fsg_build(ctx.h, db_->h, range.c(), cell_size, &h);
    }
    MBB range;
    float cell_size;
};

/* MortonGrid.h:46 MortonGrid(range, cell_size, VITURAL_CELL_PARAM) + addDatasetToGrid: the Grid's
 * cells and point order with the quadtree kept as a leaf bitmap over implicit node ids
 * (gat_morton_grid_build over a Grid it owns). */
class MortonGrid : public Index {
public:
    MortonGrid(Context& c, const MBB& mbb, float val_cell_size, int VITURAL_CELL_PARAM = 2, int leafCap = 512)
        : Index(c, GAT_INDEX_MORTON), grid(c, mbb, val_cell_size, VITURAL_CELL_PARAM, leafCap) {}
    ~MortonGrid() override {
        if (h) gat_index_destroy(h); /* before its Grid */
        h = nullptr;
    }
    int addDatasetToGrid(const Trajectory* db, int traNum) {
        int rc = grid.addDatasetToGrid(db, traNum);
        return rc != GAT_OK ? rc : gat_morton_grid_build(ctx.h, grid.h, &h);
    }
    Grid grid;
};

/* PreProcess::readTraFromFormatedFile (PreProcess.cpp:224-315): the formatted trajectory file
 * into tradb[1..n] (tradb[0] empty, as the reference's global table) and the file's box. */
inline int readTrajectoryFile(const char* path, std::vector<Trajectory>& tradb, MBB* range = nullptr) {
    int n = 0;
    int64_t points = 0;
    float box[4] = {0, 0, 0, 0};
    int rc = gat_traj_file_info(path, &n, &points, box);
    if (rc != GAT_OK) return rc;
    std::vector<int32_t> len((size_t)n), times((size_t)points);
    std::vector<float> lon((size_t)points), lat((size_t)points);
    rc = gat_traj_file_read(path, n, points, len.data(), lon.data(), lat.data(), times.data());
    if (rc != GAT_OK) return rc;
    tradb.assign((size_t)n + 1, Trajectory());
    size_t o = 0;
    for (int t = 1; t <= n; t++) {
        tradb[(size_t)t].tid = t;
        for (int i = 0; i < len[(size_t)t - 1]; i++, o++) tradb[(size_t)t].addSamplePoints(lon[o], lat[o], times[o]);
    }
    if (range) *range = MBB(box[0], box[1], box[2], box[3]);
    return GAT_OK;
}

/* PreProcess::writeTraDataToFile (PreProcess.cpp:203-222) of tradb[1..n]. */
inline int writeTrajectoryFile(const char* path, const Trajectory* tradb, int n, const MBB& range) {
    std::vector<int32_t> len((size_t)n), times;
    std::vector<float> lon, lat;
    for (int t = 1; t <= n; t++) {
        len[(size_t)t - 1] = (int32_t)tradb[t].points.size();
        for (const SamplePoint& p : tradb[t].points) {
            lon.push_back(p.lon);
            lat.push_back(p.lat);
            times.push_back(p.time);
        }
    }
    const float box[4] = {range.xmin, range.ymin, range.xmax, range.ymax};
    return gat_traj_file_write(path, n, len.data(), lon.data(), lat.data(), times.data(), box);
}

/* Per query: offsets[q] .. offsets[q+1] into tids (and pidx for point results). */
struct RangeResult {
    std::vector<int64_t> offsets;
    std::vector<int32_t> tids, pidx;
    int nq() const { return offsets.empty() ? 0 : (int)offsets.size() - 1; }
};

/* Per query k (id, distance) pairs sorted by (distance, id). */
struct TopkResult {
    int nq = 0, k = 0;
    std::vector<int32_t> ids, dist;
    int64_t stats[4] = {0, 0, 0, 0};
};

/* Range query over any index; grows the result buffer to the needed size. */
inline int range_query(const Index& ix, const MBB* q, int nq, int kind, int exec, RangeResult& out) {
    out.offsets.assign((size_t)nq + 1, 0);
    int64_t cap = std::max<int64_t>(1024, (int64_t)nq * 64), need = 0;
    for (int attempt = 0; attempt < 2; attempt++) {
        out.tids.resize((size_t)cap);
        out.pidx.resize(kind == GAT_RESULT_POINTS ? (size_t)cap : 0);
        static_assert(sizeof(MBB) == sizeof(gat_mbb), "MBB layout");
        int rc = gat_range_query(ix.ctx.h, ix.h, reinterpret_cast<const gat_mbb*>(q), nq, kind, exec, out.offsets.data(),
                                 out.tids.data(), kind == GAT_RESULT_POINTS ? out.pidx.data() : nullptr, cap, &need);
        if (rc == GAT_ERR_TRUNCATED && attempt == 0) {
            cap = need;
            continue;
        }
        if (rc != GAT_OK) return rc;
        out.tids.resize((size_t)need);
        if (kind == GAT_RESULT_POINTS) out.pidx.resize((size_t)need);
        return GAT_OK;
    }
    return GAT_ERR_TRUNCATED;
}

/* SystemTest.h:13-35. rangeQueryNum copies of one MBB per call, as the reference's harness does
 * (SystemTest.cpp:31-33); the batch forms take arrays. */
class SystemTest {
public:
    SystemTest() = default;
    SystemTest(const Trajectory* tradb_, Grid* g_, STIG* stig_, FSG* fsg_, MortonGrid* mgrid_ = nullptr)
        : tradb(tradb_), g(g_), stig(stig_), fsg(fsg_), mgrid(mgrid_) {}

    const Trajectory* tradb = nullptr;
    Grid* g = nullptr;
    STIG* stig = nullptr;
    FSG* fsg = nullptr;
    MortonGrid* mgrid = nullptr;
    MBB rangeQueryMBB;
    int rangeQueryNum = 0;
    int similarityScale = 0;
    int similarityKValue = 0;
    double epsilon = 0.005; /* EPSILON, ConstDefine.h:28 */
    int exec = GAT_EXEC_BATCHED;
    bool verbose = true;
    RangeResult lastRange;
    TopkResult lastTopk;
    double lastMs = 0.0;

    int rangeQueryTest(MBB mbb, int num) { return repeat_range(g, "", mbb, num); }
    int STIGrangeQueryTest(MBB mbb, int num) { return repeat_range(stig, " STIG", mbb, num); }
    int FSGrangeQueryTest(MBB mbb, int num) { return repeat_range(fsg, " FSG", mbb, num); }
    /* SystemTest.h:29. The reference's rangeQueryBatchGPUWithoutMorton (Grid.cpp:544-662) walks
     * the Grid's Morton-ordered points through per-block segment lists that pretend to be
     * row-major; every segment starts at offset 0 of its block (the offset it pushes is never
     * advanced, Grid.cpp:818-827), so it rescans each block's first points and its results are
     * not the Grid's. There is no correct answer of its own to reproduce; this runs the
     * GT-quadtree path. */
    int rangeQueryTestWithoutMorton(MBB mbb, int num) { return repeat_range(g, " (without Morton)", mbb, num); }
    /* SystemTest.h:33 (SystemTest.cpp:386-425): the MortonGrid's implicit-tree walk; its id sets
     * are the Grid's. Without a MortonGrid the Grid answers. */
    int MortonGridRangeQueryTest(MBB mbb, int num) {
        return repeat_range(mgrid ? static_cast<Index*>(mgrid) : static_cast<Index*>(g), " Morton Grid", mbb, num);
    }

    /* SystemTest.h:30: similarityScale copies of t against the grid's set */
    int similarityQueryTest(const Trajectory& t, int scale, int k) {
        std::vector<Trajectory> q((size_t)scale, t);
        similarityScale = scale;
        similarityKValue = k;
        return similarityQueryBatch(q.data(), scale, k, lastTopk);
    }
    /* README.md:30 form: the query is trajectory queryTrajNo of the set */
    int similarityQueryTest(int queryTrajNo, int scale, int k) {
        if (!tradb || queryTrajNo < 1) return GAT_ERR_ARG;
        return similarityQueryTest(tradb[queryTrajNo], scale, k);
    }

    /* batch forms */
    int rangeQueryBatch(Index* ix, const MBB* q, int nq, int kind, RangeResult& out) {
        if (!ix || !ix->h) return GAT_ERR_STATE;
        auto t0 = std::chrono::steady_clock::now();
        int rc = range_query(*ix, q, nq, kind, exec, out);
        lastMs = ms_since(t0);
        return rc;
    }
    int similarityQueryBatch(const Trajectory* q, int nq, int k, TopkResult& out) {
        if (!g || !g->h) return GAT_ERR_STATE;
        std::vector<int32_t> len((size_t)nq);
        std::vector<float> lon, lat;
        for (int i = 0; i < nq; i++) {
            len[(size_t)i] = (int32_t)q[i].points.size();
            for (const SamplePoint& p : q[i].points) {
                lon.push_back(p.lon);
                lat.push_back(p.lat);
            }
        }
        out.nq = nq;
        out.k = k;
        out.ids.assign((size_t)nq * k, 0);
        out.dist.assign((size_t)nq * k, 0);
        if (verbose) printf("one GPU similarity @ k=%d and #query=%d:\n", k, nq);
        auto t0 = std::chrono::steady_clock::now();
        int rc = gat_topk(g->ctx.h, g->h, nq, len.data(), lon.data(), lat.data(), k, epsilon, exec, out.ids.data(),
                          out.dist.data(), out.stats);
        lastMs = ms_since(t0);
        if (verbose && rc == GAT_OK) printf("GPU Time of similarity:%fms\n", lastMs);
        return rc;
    }

private:
    static double ms_since(std::chrono::steady_clock::time_point t0) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    int repeat_range(Index* ix, const char* name, MBB mbb, int num) {
        rangeQueryMBB = mbb;
        rangeQueryNum = num;
        std::vector<MBB> q((size_t)num, mbb);
        if (verbose) printf("single GPU%s range query #query=%d:\n", name, num);
        int rc = rangeQueryBatch(ix, q.data(), num, GAT_RESULT_IDS, lastRange);
        if (verbose && rc == GAT_OK) printf("Single GPU Time%s:%fms\n", name, lastMs);
        return rc;
    }
};

}  // namespace gat

#endif /* GAT_B200_HPP */
