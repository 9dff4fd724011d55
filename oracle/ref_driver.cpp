/* Test-infrastructure driver around the reference's own CPU code.
 *
 * oracle/Makefile compiles the reference's sources (Grid.cpp, FVTable.cpp, STIG.cpp, FSG.cpp,
 * MBB.cpp, Cell.cpp, Trajectory.cpp, SamplePoint.cpp, QueryResult.cpp) where they lie, links
 * them with this file, and writes the executable to oracle/_ref/gatref. Nothing here is part of
 * the product: tests use it to pin the restated oracle (oracle/oracle.cpp) and to write golden
 * fixtures, and bench.py times it as the CPU baseline of the reference.
 *
 * Input files use one small binary format, written by oracle/pyoracle.py:
 *   data file    : "GATD", int32 n_traj, int64 n_points, int32 lengths[n_traj],
 *                  float lon[n_points], float lat[n_points]   (trajectory ids are 1..n_traj)
 *   query file   : "GATQ", int32 n, float[n][4] (xmin, ymin, xmax, ymax)
 *   pair file    : "GATP", int32 n, int32 lenA[n], int32 lenB[n], float A[sum lenA][2],
 *                  float B[sum lenB][2]        (x = lon, y = lat)
 *   id file      : "GATI", int32 n, int32 ids[n]
 * Output is a sequence of named arrays (int32 name length, name, char dtype, int64 count, data),
 * read by oracle/pyoracle.py.
 *
 * Two facts of the reference are handled here rather than patched in its sources:
 *  - FVTable::formPriorityQueue (FVTable.cpp:141-152, 171-183) erases the std::map node that its
 *    loop iterator points at and then increments that iterator. glibc's free() writes its
 *    bookkeeping into the freed node, after which the increment follows a garbage pointer and a
 *    plain -O2 build crashes. This driver replaces the global operator delete with a per-thread
 *    FIFO quarantine (freed blocks are released 4096 frees later), which leaves the erased node
 *    intact exactly like AddressSanitizer's quarantine does, without the sanitizer's cost. The
 *    iteration order the reference then produces is the one an ASan build produces.
 *  - The GPU handler functions declared in cudaKernel.h are referenced by the GPU query paths
 *    of Grid/STIG/FSG/FVTable but never reached by the CPU calls made here; they are defined
 *    below as stubs that abort, so kernel.cu is not needed.
 */
#include <map>
#include "PreProcess.h"
#include <Grid.h>
#include <STIG.h>
#include <FSG.h>
#include <CalcInAxis.h>

#include "datagen.h"

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

Trajectory* tradb = nullptr;
/* globals PreProcess.cpp refers to (defined in the reference's main.cpp, not linked here) */
std::map<std::string, tidLinkTable*> vidTotid;
std::map<std::string, tidLinkTable*>::iterator iter;
std::string baseDate;
int DaysBetween2Date(std::string, std::string) { return 0; }
void* baseAddrGPU = nullptr;
double gat_ref_epsilon = 0.005;
int gat_ref_leaf_cap = 20000;

/* ---------------------------------------------------------------- deferred free */
#ifndef GATREF_NO_QUARANTINE
namespace {
struct Quarantine {
    static const size_t kSlots = 4096;
    void* slot[kSlots];
    size_t pos = 0;
    Quarantine() { memset(slot, 0, sizeof(slot)); }
    ~Quarantine() {
        for (size_t i = 0; i < kSlots; i++) free(slot[i]);
    }
    void put(void* p) {
        void* old = slot[pos];
        slot[pos] = p;
        pos = (pos + 1) % kSlots;
        free(old);
    }
};
thread_local Quarantine tl_quarantine;
}  // namespace
void operator delete(void* p) noexcept {
    if (p) tl_quarantine.put(p);
}
void operator delete(void* p, size_t) noexcept {
    if (p) tl_quarantine.put(p);
}
void operator delete[](void* p) noexcept {
    if (p) tl_quarantine.put(p);
}
void operator delete[](void* p, size_t) noexcept {
    if (p) tl_quarantine.put(p);
}
#endif

/* ---------------------------------------------------------------- GPU handler stubs */
static void gpu_stub(const char* name) {
    fprintf(stderr, "gatref: GPU path %s is not part of the CPU oracle\n", name);
    abort();
}
int cudaRangeQueryHandler(int*, int*, int*, int, float, float, float, float, Point*&, int&, Point*,
                          Point*&) {
    gpu_stub("cudaRangeQueryHandler");
    return 0;
}
int putCellDataSetIntoGPU(Point*, Point*&, int) {
    gpu_stub("putCellDataSetIntoGPU");
    return 0;
}
int handleEDRdistance(SPoint*, SPoint**, int, int, int*, int*) {
    gpu_stub("handleEDRdistance");
    return 0;
}
void CUDAwarmUp() { gpu_stub("CUDAwarmUp"); }
int cudaRangeQueryTestHandler(RangeQueryStateTable*, int, uint8_t*, int, int, cudaStream_t) {
    gpu_stub("cudaRangeQueryTestHandler");
    return 0;
}
int EDRDistance_Batch_Handler(int, TaskInfoTableForSimilarity*, SPoint*, int*, SPoint**, int*, int*,
                              int*, cudaStream_t*) {
    gpu_stub("EDRDistance_Batch_Handler");
    return 0;
}
int Similarity_Pruning_Handler(intPair*, intPair*, intPair*, intPair*, intPair*, int, int, int, int,
                               int, int, int, short*, cudaStream_t) {
    gpu_stub("Similarity_Pruning_Handler");
    return 0;
}
int cudaRangeQuerySTIGHandler(RangeQueryStateTable*, int, uint8_t*, int, int, cudaStream_t) {
    gpu_stub("cudaRangeQuerySTIGHandler");
    return 0;
}
int cudaRangeQueryTestHandlerNonMorton(RangeQueryStateTable*, int, uint8_t*, int, int, cudaStream_t,
                                       int*, int*, int*, int*) {
    gpu_stub("cudaRangeQueryTestHandlerNonMorton");
    return 0;
}

/* ---------------------------------------------------------------- I/O */
namespace {

[[noreturn]] void die(const char* msg) {
    fprintf(stderr, "gatref: %s\n", msg);
    exit(2);
}

struct Reader {
    FILE* f;
    explicit Reader(const char* path) : f(fopen(path, "rb")) {
        if (!f) die("cannot open input");
    }
    ~Reader() { fclose(f); }
    void magic(const char* m) {
        char buf[4];
        if (fread(buf, 1, 4, f) != 4 || memcmp(buf, m, 4) != 0) die("bad magic");
    }
    template <class T>
    T get() {
        T v;
        if (fread(&v, sizeof(T), 1, f) != 1) die("short read");
        return v;
    }
    template <class T>
    void vec(std::vector<T>& v, size_t n) {
        v.resize(n);
        if (n && fread(v.data(), sizeof(T), n, f) != n) die("short read");
    }
};

struct Writer {
    FILE* f;
    explicit Writer(const char* path) : f(fopen(path, "wb")) {
        if (!f) die("cannot open output");
    }
    ~Writer() { fclose(f); }
    void arr(const char* name, char dtype, const void* p, int64_t count, size_t elsize) {
        int32_t nl = (int32_t)strlen(name);
        fwrite(&nl, 4, 1, f);
        fwrite(name, 1, nl, f);
        fwrite(&dtype, 1, 1, f);
        fwrite(&count, 8, 1, f);
        if (count) fwrite(p, elsize, (size_t)count, f);
    }
    void i32(const char* n, const std::vector<int32_t>& v) { arr(n, 'i', v.data(), v.size(), 4); }
    void i64(const char* n, const std::vector<int64_t>& v) { arr(n, 'l', v.data(), v.size(), 8); }
    void f32(const char* n, const std::vector<float>& v) { arr(n, 'f', v.data(), v.size(), 4); }
    void f64(const char* n, const std::vector<double>& v) { arr(n, 'd', v.data(), v.size(), 8); }
};

struct Data {
    int n = 0;
    std::vector<int32_t> len;
    std::vector<float> lon, lat;
};

Data read_data(const char* path) {
    Reader r(path);
    r.magic("GATD");
    Data d;
    d.n = r.get<int32_t>();
    int64_t np = r.get<int64_t>();
    r.vec(d.len, d.n);
    r.vec(d.lon, np);
    r.vec(d.lat, np);
    return d;
}

/* Fills the reference's global trajectory table (ids start at 1, main.cpp:116-121). */
void load_tradb(const Data& d) {
    tradb = new Trajectory[d.n + 1];
    int64_t off = 0;
    for (int i = 1; i <= d.n; i++) {
        Trajectory& t = tradb[i];
        t.tid = i;
        t.length = d.len[i - 1];
        t.points.reserve(t.length);
        for (int j = 0; j < t.length; j++, off++)
            t.points.push_back(SamplePoint(d.lon[off], d.lat[off], 0, i));
    }
}

std::vector<MBB> read_queries(const char* path) {
    Reader r(path);
    r.magic("GATQ");
    int n = r.get<int32_t>();
    std::vector<float> raw;
    r.vec(raw, (size_t)n * 4);
    std::vector<MBB> q(n);
    for (int i = 0; i < n; i++) q[i] = MBB(raw[4 * i], raw[4 * i + 1], raw[4 * i + 2], raw[4 * i + 3]);
    return q;
}

std::vector<int32_t> read_ids(const char* path) {
    Reader r(path);
    r.magic("GATI");
    int n = r.get<int32_t>();
    std::vector<int32_t> v;
    r.vec(v, n);
    return v;
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

/* ID sets from vector<bool> result tables as CSR (sorted by construction). */
void write_id_sets(Writer& w, const std::vector<CPURangeQueryResult>& res, int ntraj) {
    std::vector<int64_t> off(1, 0);
    std::vector<int32_t> ids;
    for (const auto& r : res) {
        for (int t = 0; t <= ntraj && t < (int)r.size(); t++)
            if (r[t]) ids.push_back(t);
        off.push_back((int64_t)ids.size());
    }
    w.i64("id_off", off);
    w.i32("ids", ids);
}

/* Depth-first (UL, UR, DL, DR) listing of the quadtree (Grid.cpp:58-94). */
void walk_quadtree(QuadtreeNode* n, std::vector<int32_t>& node_id, std::vector<int32_t>& level,
                   std::vector<int32_t>& npts, std::vector<int32_t>& leaf, std::vector<float>& mbb) {
    node_id.push_back(n->NodeID);
    level.push_back(n->level);
    npts.push_back(n->numPoints);
    leaf.push_back(n->isLeaf ? 1 : 0);
    mbb.push_back(n->mbb.xmin);
    mbb.push_back(n->mbb.ymin);
    mbb.push_back(n->mbb.xmax);
    mbb.push_back(n->mbb.ymax);
    if (!n->isLeaf) {
        walk_quadtree(n->UL, node_id, level, npts, leaf, mbb);
        walk_quadtree(n->UR, node_id, level, npts, leaf, mbb);
        walk_quadtree(n->DL, node_id, level, npts, leaf, mbb);
        walk_quadtree(n->DR, node_id, level, npts, leaf, mbb);
    }
}

Grid* build_grid(const Data& d, float cell, float bx0, float by0, float bx1, float by1) {
    Grid* g = new Grid(MBB(bx0, by0, bx1, by1), cell, 2);
    g->addDatasetToGrid(tradb, d.n);
    return g;
}

/* gtq DATA QUERIES OUT cell leafcap bx0 by0 bx1 by1 layout(0/1) threads
 * threads: 0 -> Grid::rangeQueryBatch on one core (Grid.cpp:341)
 *         -1 -> Grid::rangeQueryBatchMultiThread, the reference's fixed 16 threads (Grid.cpp:407)
 *          T -> T threads, each calling Grid::rangeQueryBatch on a contiguous slice of queries */
int cmd_gtq(int argc, char** argv) {
    if (argc < 12) die("usage: gtq DATA QUERIES OUT cell leafcap bx0 by0 bx1 by1 layout threads");
    Data d = read_data(argv[2]);
    std::vector<MBB> q = read_queries(argv[3]);
    Writer w(argv[4]);
    float cell = (float)atof(argv[5]);
    gat_ref_leaf_cap = atoi(argv[6]);
    int layout = atoi(argv[11]);
    int threads = argc > 12 ? atoi(argv[12]) : 0;
    load_tradb(d);
    double t0 = now_s();
    Grid* g = build_grid(d, cell, (float)atof(argv[7]), (float)atof(argv[8]), (float)atof(argv[9]),
                         (float)atof(argv[10]));
    double t_build = now_s() - t0;
    int nq = (int)q.size();
    std::vector<CPURangeQueryResult> res(nq);
    t0 = now_s();
    if (nq > 0) {
        if (threads == 0) {
            g->rangeQueryBatch(q.data(), nq, res.data(), nullptr);
        } else if (threads < 0) {
            g->rangeQueryBatchMultiThread(q.data(), nq, res.data(), nullptr);
        } else {
            std::vector<std::thread> th;
            int per = (nq + threads - 1) / threads;
            for (int s = 0; s < nq; s += per) {
                int c = std::min(per, nq - s);
                th.emplace_back([g, &q, &res, s, c]() { g->rangeQueryBatch(&q[s], c, &res[s], nullptr); });
            }
            for (auto& t : th) t.join();
        }
    }
    double t_query = now_s() - t0;
    write_id_sets(w, res, d.n);
    w.f64("t_build", {t_build});
    w.f64("t_query", {t_query});
    if (layout) {
        std::vector<int32_t> meta = {g->cellNum_axis, g->cellnum, g->totalPointNum, g->nodeNum};
        w.i32("meta", meta);
        std::vector<float> px(g->totalPointNum), py(g->totalPointNum);
        std::vector<int32_t> pt(g->totalPointNum);
        for (int i = 0; i < g->totalPointNum; i++) {
            px[i] = g->allPoints[i].x;
            py[i] = g->allPoints[i].y;
            pt[i] = g->allPoints[i].tID;
        }
        w.f32("px", px);
        w.f32("py", py);
        w.i32("ptid", pt);
        std::vector<int32_t> cs(g->cellnum), ce(g->cellnum);
        std::vector<float> cm;
        for (int c = 0; c < g->cellnum; c++) {
            cs[c] = g->cellPtr[c].pointRangeStart;
            ce[c] = g->cellPtr[c].pointRangeEnd;
            cm.push_back(g->cellPtr[c].mbb.xmin);
            cm.push_back(g->cellPtr[c].mbb.ymin);
            cm.push_back(g->cellPtr[c].mbb.xmax);
            cm.push_back(g->cellPtr[c].mbb.ymax);
        }
        w.i32("cell_start", cs);
        w.i32("cell_end", ce);
        w.f32("cell_mbb", cm);
        std::vector<int32_t> nid, lvl, npts, leaf;
        std::vector<float> nmbb;
        walk_quadtree(g->root, nid, lvl, npts, leaf, nmbb);
        w.i32("node_id", nid);
        w.i32("node_level", lvl);
        w.i32("node_npts", npts);
        w.i32("node_leaf", leaf);
        w.f32("node_mbb", nmbb);
        /* candidate leaves per query, in traversal order (Grid.cpp:428-446) */
        std::vector<int64_t> coff(1, 0);
        std::vector<int32_t> cid, clvl;
        for (int i = 0; i < nq; i++) {
            std::vector<QuadtreeNode*> cells;
            g->findMatchNodeInQuadTree(g->root, q[i], &cells);
            for (auto* n : cells) {
                cid.push_back(n->NodeID);
                clvl.push_back(n->level);
            }
            coff.push_back((int64_t)cid.size());
        }
        w.i64("cand_off", coff);
        w.i32("cand_node", cid);
        w.i32("cand_level", clvl);
        /* cell-run table of every trajectory (Grid.cpp:189-196, 264-288) */
        std::vector<int64_t> roff(1, 0);
        std::vector<int32_t> rcell, rstart, rcount;
        for (int t = 1; t <= d.n; t++) {
            const cellBasedTraj& cb = g->cellBasedTrajectory[t];
            for (int r = 0; r < cb.length; r++) {
                rcell.push_back(cb.cellNo[r]);
                rstart.push_back(cb.startIdx[r]);
                rcount.push_back(cb.numOfPointInCell[r]);
            }
            roff.push_back((int64_t)rcell.size());
        }
        w.i64("run_off", roff);
        w.i32("run_cell", rcell);
        w.i32("run_start", rstart);
        w.i32("run_count", rcount);
        /* frequency vectors (virtual cell -> count), FVTable.cpp:18-30 */
        std::vector<int64_t> foff(1, 0);
        std::vector<int32_t> fcell, fcnt;
        for (int t = 0; t <= d.n; t++) {
            for (auto& kv : g->freqVectors.FreqVector[t]) {
                fcell.push_back(kv.first);
                fcnt.push_back(kv.second);
            }
            foff.push_back((int64_t)fcell.size());
        }
        w.i64("fv_off", foff);
        w.i32("fv_cell", fcell);
        w.i32("fv_count", fcnt);
    }
    return 0;
}

void walk_stig(STIG* s, void* node, bool is_leaf, std::vector<int32_t>& lr, std::vector<float>& mbb,
               std::vector<int32_t>& depth, std::vector<int32_t>& kind, std::vector<float>& med) {
    if (is_leaf) {
        LeafNode* l = (LeafNode*)node;
        kind.push_back(1);
        depth.push_back(l->depth);
        lr.push_back(l->leftRange);
        lr.push_back(l->rightRange);
        mbb.push_back(l->boundingBox.xmin);
        mbb.push_back(l->boundingBox.ymin);
        mbb.push_back(l->boundingBox.xmax);
        mbb.push_back(l->boundingBox.ymax);
        med.push_back(0.f);
        return;
    }
    InternalNode* in = (InternalNode*)node;
    kind.push_back(0);
    depth.push_back(in->depth);
    lr.push_back(-1);
    lr.push_back(-1);
    for (int i = 0; i < 4; i++) mbb.push_back(0.f);
    med.push_back(in->medium);
    walk_stig(s, in->left, in->leftIsLeaf, lr, mbb, depth, kind, med);
    walk_stig(s, in->right, in->rightIsLeaf, lr, mbb, depth, kind, med);
}

/* stig DATA QUERIES OUT blocksize layout(0/1)
 * STIG has no CPU query path; candidate blocks come from STIG::searchTree (STIG.cpp:179) and
 * the ID set applies the inclusive MBB::pInBox to every point of those blocks. */
int cmd_stig(int argc, char** argv) {
    if (argc < 7) die("usage: stig DATA QUERIES OUT blocksize layout");
    Data d = read_data(argv[2]);
    std::vector<MBB> q = read_queries(argv[3]);
    Writer w(argv[4]);
    int bs = atoi(argv[5]);
    int layout = atoi(argv[6]);
    load_tradb(d);
    double t0 = now_s();
    STIG* s = new STIG();
    s->initial(bs, 2, tradb, d.n);
    double t_build = now_s() - t0;
    std::vector<int64_t> boff(1, 0), ioff(1, 0);
    std::vector<int32_t> blk, ids;
    std::vector<char> mark(d.n + 1);
    for (size_t i = 0; i < q.size(); i++) {
        std::vector<STIGBlock> b;
        s->searchTree(q[i], &b);
        std::fill(mark.begin(), mark.end(), 0);
        for (auto& x : b) {
            blk.push_back(x.startIdx);
            blk.push_back(x.endIdx);
            for (int p = x.startIdx; p <= x.endIdx; p++)
                if (q[i].pInBox(s->allPoints[p].x, s->allPoints[p].y)) mark[s->allPoints[p].tID] = 1;
        }
        for (int t = 0; t <= d.n; t++)
            if (mark[t]) ids.push_back(t);
        boff.push_back((int64_t)blk.size() / 2);
        ioff.push_back((int64_t)ids.size());
    }
    w.i64("blk_off", boff);
    w.i32("blk", blk);
    w.i64("id_off", ioff);
    w.i32("ids", ids);
    w.f64("t_build", {t_build});
    if (layout) {
        std::vector<float> px, py;
        std::vector<int32_t> pt;
        for (auto& p : s->allPoints) {
            px.push_back(p.x);
            py.push_back(p.y);
            pt.push_back(p.tID);
        }
        w.f32("px", px);
        w.f32("py", py);
        w.i32("ptid", pt);
        std::vector<int32_t> lr, depth, kind;
        std::vector<float> mbb, med;
        walk_stig(s, s->root, s->totalPointsNum <= s->blockSize, lr, mbb, depth, kind, med);
        w.i32("node_lr", lr);
        w.f32("node_mbb", mbb);
        w.i32("node_depth", depth);
        w.i32("node_kind", kind);
        w.f32("node_median", med);
    }
    return 0;
}

/* fsg DATA OUT cell bx0 by0 bx1 by1 : layout of FSG::addDatasetToGrid (FSG.cpp:95-143). The
 * reference's FSG query path exists only on the GPU (FSG.cpp:145), so no query is run here. */
int cmd_fsg(int argc, char** argv) {
    if (argc < 9) die("usage: fsg DATA OUT cell bx0 by0 bx1 by1");
    Data d = read_data(argv[2]);
    Writer w(argv[3]);
    load_tradb(d);
    double t0 = now_s();
    FSG* f = new FSG(MBB((float)atof(argv[5]), (float)atof(argv[6]), (float)atof(argv[7]),
                         (float)atof(argv[8])),
                     (float)atof(argv[4]));
    f->addDatasetToGrid(tradb, d.n);
    double t_build = now_s() - t0;
    std::vector<int32_t> meta = {f->cell_num_x, f->cell_num_y, f->cellnum, f->totalPointNum};
    w.i32("meta", meta);
    w.f64("t_build", {t_build});
    std::vector<float> px, py;
    std::vector<int32_t> pt, cs, ce;
    for (int i = 0; i < f->totalPointNum; i++) {
        px.push_back(f->allPoints[i].x);
        py.push_back(f->allPoints[i].y);
        pt.push_back(f->allPoints[i].tID);
    }
    for (int c = 0; c < f->cellnum; c++) {
        cs.push_back(f->cellPtr[c].pointRangeStart);
        ce.push_back(f->cellPtr[c].pointRangeEnd);
    }
    w.f32("px", px);
    w.f32("py", py);
    w.i32("ptid", pt);
    w.i32("cell_start", cs);
    w.i32("cell_end", ce);
    return 0;
}

/* edr PAIRS OUT eps threads : Grid::SimilarityExecuter (Grid.cpp:1222) per (A = query,
 * B = candidate) pair; threads > 1 partitions the pairs into contiguous slices. */
int cmd_edr(int argc, char** argv) {
    if (argc < 5) die("usage: edr PAIRS OUT eps [threads]");
    Reader r(argv[2]);
    r.magic("GATP");
    int n = r.get<int32_t>();
    std::vector<int32_t> la, lb;
    r.vec(la, n);
    r.vec(lb, n);
    int64_t sa = 0, sb = 0;
    for (int i = 0; i < n; i++) {
        sa += la[i];
        sb += lb[i];
    }
    std::vector<float> a, b;
    r.vec(a, sa * 2);
    r.vec(b, sb * 2);
    Writer w(argv[3]);
    gat_ref_epsilon = atof(argv[4]);
    int threads = argc > 5 ? atoi(argv[5]) : 1;
    if (threads < 1) threads = 1;
    std::vector<SPoint> A(sa), B(sb);
    for (int64_t i = 0; i < sa; i++) A[i] = SPoint{a[2 * i], a[2 * i + 1], 0};
    for (int64_t i = 0; i < sb; i++) B[i] = SPoint{b[2 * i], b[2 * i + 1], 0};
    std::vector<int64_t> oa(n + 1, 0), ob(n + 1, 0);
    for (int i = 0; i < n; i++) {
        oa[i + 1] = oa[i] + la[i];
        ob[i + 1] = ob[i] + lb[i];
    }
    std::vector<int32_t> dist(n);
    double t0 = now_s();
    auto work = [&](int s, int e) {
        Grid g;
        for (int i = s; i < e; i++) {
            SPoint* cand = &B[ob[i]];
            int lc = lb[i];
            int res = 0;
            g.SimilarityExecuter(&A[oa[i]], &cand, la[i], &lc, 1, &res);
            dist[i] = res;
        }
    };
    if (threads == 1) {
        work(0, n);
    } else {
        std::vector<std::thread> th;
        std::atomic<int> next(0);
        for (int t = 0; t < threads; t++)
            th.emplace_back([&]() {
                for (;;) {
                    int s = next.fetch_add(16);
                    if (s >= n) break;
                    work(s, std::min(n, s + 16));
                }
            });
        for (auto& t : th) t.join();
    }
    double t = now_s() - t0;
    w.i32("dist", dist);
    w.f64("t_query", {t});
    return 0;
}

/* rangebench OUT n len_lo len_hi seed nq side_lo side_hi cell leafcap bx0 by0 bx1 by1 per_step steps threads
 * The batched range workload timed through the reference's own CPU query: n random walks with
 * lengths uniform in [len_lo, len_hi] and nq rectangles with log-uniform sides in
 * [side_lo, side_hi], generated with seed by oracle/datagen.cpp (the library's streams, so the
 * arrays equal the GPU run's); the reference's Grid (Grid::Grid + addDatasetToGrid) over them;
 * then `steps` steps. Step s takes the rectangles s, s + stride, s + 2 stride, ... (per_step of
 * them, stride = nq / per_step, so every step is a different sample spread over the whole
 * query set) and runs them on `threads` threads, each calling Grid::rangeQueryBatch
 * (Grid.cpp:341-405) on a contiguous slice. Writes the per-step seconds, the build seconds, the
 * number of ids per step and the id sets of step 0 (its rectangle indices in q_index). */
int cmd_rangebench(int argc, char** argv) {
    if (argc < 19) die("usage: rangebench OUT n len_lo len_hi seed nq side_lo side_hi cell leafcap bx0 by0 bx1 by1 per_step steps threads");
    Writer w(argv[2]);
    const int n = atoi(argv[3]), len_lo = atoi(argv[4]), len_hi = atoi(argv[5]);
    const uint64_t seed = (uint64_t)atoll(argv[6]);
    const int nq = atoi(argv[7]);
    const double side_lo = atof(argv[8]), side_hi = atof(argv[9]);
    const float cell = (float)atof(argv[10]);
    gat_ref_leaf_cap = atoi(argv[11]);
    const float box[4] = {(float)atof(argv[12]), (float)atof(argv[13]), (float)atof(argv[14]), (float)atof(argv[15])};
    const int per_step = atoi(argv[16]), steps = atoi(argv[17]);
    const int threads = std::max(1, atoi(argv[18]));
    if (n < 1 || nq < 1 || per_step < 1 || per_step > nq || steps < 1) die("rangebench: bad sizes");
    const int stride = nq / per_step;
    if (steps > stride) die("rangebench: more steps than distinct samples");
    Data d;
    d.n = n;
    d.len.resize(n);
    orc_gen_lengths(n, ORC_LEN_UNIFORM, 0.0, 0.0, len_lo, len_hi, seed, d.len.data());
    int64_t np = 0;
    for (int v : d.len) np += v;
    d.lon.resize(np);
    d.lat.resize(np);
    orc_gen_walks(n, d.len.data(), box, 1e-4, seed, d.lon.data(), d.lat.data());
    std::vector<float> q4((size_t)nq * 4);
    orc_gen_boxes(nq, ORC_SIDE_LOGUNIFORM, side_lo, side_hi, box, seed, q4.data());
    load_tradb(d);
    std::vector<float>().swap(d.lon);
    std::vector<float>().swap(d.lat);
    double t0 = now_s();
    Grid* g = build_grid(d, cell, box[0], box[1], box[2], box[3]);
    const double t_build = now_s() - t0;
    std::vector<double> t_step;
    std::vector<int64_t> ids_step, id_off(1, 0);
    std::vector<int32_t> ids0, qidx0;
    for (int s = 0; s < steps; s++) {
        std::vector<MBB> q(per_step);
        for (int j = 0; j < per_step; j++) {
            const float* b = &q4[(size_t)(s + (int64_t)j * stride) * 4];
            q[j] = MBB(b[0], b[1], b[2], b[3]);
        }
        std::vector<CPURangeQueryResult> res(per_step);
        t0 = now_s();
        std::vector<std::thread> th;
        const int per = (per_step + threads - 1) / threads;
        for (int b = 0; b < per_step; b += per) {
            const int c = std::min(per, per_step - b);
            th.emplace_back([g, &q, &res, b, c]() { g->rangeQueryBatch(&q[b], c, &res[b], nullptr); });
        }
        for (auto& t : th) t.join();
        t_step.push_back(now_s() - t0);
        int64_t cnt = 0;
        for (int j = 0; j < per_step; j++) {
            const CPURangeQueryResult& r = res[j];
            for (int t = 0; t <= n && t < (int)r.size(); t++)
                if (r[t]) {
                    cnt++;
                    if (s == 0) ids0.push_back(t);
                }
            if (s == 0) {
                id_off.push_back((int64_t)ids0.size());
                qidx0.push_back(s + j * stride);
            }
        }
        ids_step.push_back(cnt);
    }
    w.f64("t_build", {t_build});
    w.f64("t_step", t_step);
    w.i64("ids_step", ids_step);
    w.i64("id_off", id_off);
    w.i32("ids", ids0);
    w.i32("q_index", qidx0);
    std::vector<int64_t> meta = {n, np, nq, per_step, stride, threads};
    w.i64("meta", meta);
    return 0;
}

/* Query frequency vector exactly as Grid::SimilarityQueryBatch builds it (Grid.cpp:860-877). */
std::map<int, int> query_fv(Grid* g, const Trajectory& t) {
    std::map<int, int> fv;
    for (int p = 0; p < t.length; p++) {
        int cellid = g->WhichCellPointIn(SamplePoint(t.points[p].lon, t.points[p].lat, 1, 1));
        int v = cellid >> g->VITURAL_CELL_PARAM;
        auto it = fv.find(v);
        if (it == fv.end())
            fv.insert(std::pair<int, int>(v, 1));
        else
            fv[v] = fv[v] + 1;
    }
    return fv;
}

/* fvlb DATA QIDS OUT cell bx0 by0 bx1 by1 : FVTable::formPriorityQueue (FVTable.cpp:77) for
 * each query trajectory; every queue entry is popped and stored as lb[q][tid]. */
int cmd_fvlb(int argc, char** argv) {
    if (argc < 10) die("usage: fvlb DATA QIDS OUT cell bx0 by0 bx1 by1");
    Data d = read_data(argv[2]);
    std::vector<int32_t> qids = read_ids(argv[3]);
    Writer w(argv[4]);
    load_tradb(d);
    Grid* g = build_grid(d, (float)atof(argv[5]), (float)atof(argv[6]), (float)atof(argv[7]),
                         (float)atof(argv[8]), (float)atof(argv[9]));
    std::vector<int32_t> lb((size_t)qids.size() * (d.n + 1), -1);
    for (size_t qi = 0; qi < qids.size(); qi++) {
        std::map<int, int> fv = query_fv(g, tradb[qids[qi]]);
        std::priority_queue<FDwithID, std::vector<FDwithID>, cmp> pq;
        g->freqVectors.formPriorityQueue(&pq, &fv);
        while (!pq.empty()) {
            lb[qi * (d.n + 1) + pq.top().traID] = pq.top().FD;
            pq.pop();
        }
    }
    w.i32("lb", lb);
    return 0;
}

/* topk DATA QIDS OUT cell k eps bx0 by0 bx1 by1 [reps] : Grid::SimilarityQueryBatchCPUParallel
 * (Grid.cpp:1133) with query j = tradb[qid[j]], the README's similarityQueryTest(queryTrajNo,..)
 * form. Output ids are in the reference's order (worst first, Grid.cpp:1202-1209); the EDR of
 * each returned id is recomputed with Grid::SimilarityExecuter so distance multisets can be
 * compared. */
int cmd_topk(int argc, char** argv) {
    if (argc < 12) die("usage: topk DATA QIDS OUT cell k eps bx0 by0 bx1 by1");
    Data d = read_data(argv[2]);
    std::vector<int32_t> qids = read_ids(argv[3]);
    Writer w(argv[4]);
    float cell = (float)atof(argv[5]);
    int k = atoi(argv[6]);
    gat_ref_epsilon = atof(argv[7]);
    load_tradb(d);
    double t0 = now_s();
    Grid* g = build_grid(d, cell, (float)atof(argv[8]), (float)atof(argv[9]), (float)atof(argv[10]),
                         (float)atof(argv[11]));
    double t_build = now_s() - t0;
    int nq = (int)qids.size();
    Trajectory* qTra = new Trajectory[nq];
    for (int j = 0; j < nq; j++) qTra[j] = tradb[qids[j]];
    std::vector<int32_t> out((size_t)nq * k);
    /* the reference prints phase timings on stdout; keep stdout clean for callers */
    fflush(stdout);
    FILE* saved = stdout;
    stdout = fopen("/dev/null", "w");
    std::streambuf* old = std::cout.rdbuf(nullptr);
    int reps = argc > 12 ? std::max(1, atoi(argv[12])) : 1;
    std::vector<double> t_reps;
    for (int r = 0; r < reps; r++) {
        t0 = now_s();
        g->SimilarityQueryBatchCPUParallel(qTra, nq, out.data(), k);
        t_reps.push_back(now_s() - t0);
    }
    double t_query = t_reps.back();
    std::cout.rdbuf(old);
    fclose(stdout);
    stdout = saved;
    std::vector<int32_t> dist(out.size());
    for (int j = 0; j < nq; j++) {
        const Trajectory& q = tradb[qids[j]];
        std::vector<SPoint> qa(q.length);
        for (int p = 0; p < q.length; p++) qa[p] = SPoint{q.points[p].lon, q.points[p].lat, q.tid};
        for (int i = 0; i < k; i++) {
            const Trajectory& c = tradb[out[(size_t)j * k + i]];
            std::vector<SPoint> ca(c.length);
            for (int p = 0; p < c.length; p++) ca[p] = SPoint{c.points[p].lon, c.points[p].lat, c.tid};
            SPoint* cp = ca.data();
            int lc = c.length, res = 0;
            g->SimilarityExecuter(qa.data(), &cp, q.length, &lc, 1, &res);
            dist[(size_t)j * k + i] = res;
        }
    }
    w.i32("ids", out);
    w.i32("dist", dist);
    w.f64("t_build", {t_build});
    w.f64("t_query", {t_query});
    w.f64("t_reps", t_reps);
    return 0;
}

/* nbr IDS OUT vcells : FVTable::findNeighbor (FVTable.cpp:53-75) for every cell id in IDS, and
 * getIdxFromXY (Grid.cpp:25-54) over the grid [-2, 9] x [-2, 9], including the negative
 * coordinates findNeighbor produces at the grid edge. */
int cmd_nbr(int argc, char** argv) {
    if (argc < 5) die("usage: nbr IDS OUT vcells");
    std::vector<int32_t> cells = read_ids(argv[2]);
    Writer w(argv[3]);
    FVTable fv;
    fv.initFVTable(1, atoi(argv[4]));
    std::vector<int32_t> out;
    for (int c : cells) {
        int nb[8];
        fv.findNeighbor(c, nb);
        out.insert(out.end(), nb, nb + 8);
    }
    w.i32("nbr", out);
    std::vector<int32_t> grid;
    for (int x = -2; x <= 9; x++)
        for (int y = -2; y <= 9; y++) grid.push_back(getIdxFromXY(x, y));
    w.i32("idx_grid", grid);
    return 0;
}

}  // namespace

/* wfile DATA OUT xmin ymin xmax ymax: PreProcess::writeTraDataToFile (PreProcess.cpp:203-222)
 * over the trajectories of DATA (point times 0) */
int cmd_wfile(int argc, char** argv) {
    if (argc < 8) die("usage: gatref wfile DATA OUT xmin ymin xmax ymax");
    Data d = read_data(argv[2]);
    load_tradb(d);
    PreProcess pp;
    pp.maxTid = d.n;
    pp.xmin = (float)atof(argv[4]);
    pp.ymin = (float)atof(argv[5]);
    pp.xmax = (float)atof(argv[6]);
    pp.ymax = (float)atof(argv[7]);
    pp.writeTraDataToFile(argv[3]);
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 2) die("usage: gatref {gtq|stig|fsg|edr|rangebench|fvlb|topk|nbr|wfile} ...");
    std::string c = argv[1];
    if (c == "gtq") return cmd_gtq(argc, argv);
    if (c == "stig") return cmd_stig(argc, argv);
    if (c == "fsg") return cmd_fsg(argc, argv);
    if (c == "edr") return cmd_edr(argc, argv);
    if (c == "rangebench") return cmd_rangebench(argc, argv);
    if (c == "fvlb") return cmd_fvlb(argc, argv);
    if (c == "topk") return cmd_topk(argc, argv);
    if (c == "nbr") return cmd_nbr(argc, argv);
    if (c == "wfile") return cmd_wfile(argc, argv);
    die("unknown command");
}
