/* CPU restatement of the reference's hot-path algorithms. TEST INFRASTRUCTURE ONLY.
 *
 * Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker;
 * never linked into or called by the product. Parity of this restatement with the reference
 * is pinned by tests/test_oracle_vs_reference.py (against the reference's own code compiled by
 * oracle/Makefile into oracle/_ref/gatref) and by tests/test_golden.py (committed fixtures).
 *
 * Build: g++ -std=c++17 -O2 -ffp-contract=off (oracle/Makefile). Float expressions are written
 * in the reference's order and types so that x86-64 SSE rounding matches it bit for bit. */
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <thread>
#include <vector>

namespace {

struct Box {
    float xmin, ymin, xmax, ymax;
    /* MBB::pInBox (MBB.cpp:21-26): inclusive on all four sides */
    bool in(float x, float y) const { return x <= xmax && x >= xmin && y <= ymax && y >= ymin; }
};

/* BoxIntersect (MBB.cpp:28-73): 0 when disjoint or only touching, else 1/2/3. */
int box_intersect(const Box& a1, const Box& b1) {
    Box a, b;
    bool swapped = false;
    if (a1.xmin < b1.xmin) {
        a = a1;
        b = b1;
    } else if (a1.xmin == b1.xmin) {
        if (a1.xmax > b1.xmax) {
            a = a1;
            b = b1;
        } else {
            b = a1;
            a = b1;
            swapped = true;
        }
    } else {
        b = a1;
        a = b1;
        swapped = true;
    }
    if (b.xmin >= a.xmax) return 0;
    if (b.ymax <= a.ymin) return 0;
    if (b.ymin >= a.ymax) return 0;
    if (a.in(b.xmin, b.ymin) && a.in(b.xmin, b.ymax) && a.in(b.xmax, b.ymin) && a.in(b.xmax, b.ymax))
        return swapped ? 3 : 2;
    return 1;
}

/* Bit length as getIdxFromXY computes it (Grid.cpp:27-37): int(log2(v)) + 1, with v == 0 -> 1.
 * For v < 0 the reference takes log2 of a negative number; the NaN converts to INT_MIN on
 * x86-64 (cvttsd2si), so the length is INT_MIN + 1. */
int idx_len(int v) {
    if (v == 0) return 1;
    if (v < 0) return INT_MIN + 1;
    return (int)std::log2((double)v) + 1;
}

/* getIdxFromXY (Grid.cpp:25-54): Morton interleave, x on odd positions starting at bit 0.
 * When both coordinates are negative the loop bound 2*max(lenx, leny) is negative in the
 * compiled reference (g++ -O2 does not wrap it), so the loop does not run and the id is 0;
 * pinned against the compiled reference by tests/test_oracle_vs_reference.py. */
int morton(int x, int y) {
    int lx = idx_len(x), ly = idx_len(y);
    long long lim = 2LL * std::max(lx, ly);
    int result = 0, xbit = 1, ybit = 1;
    for (int i = 1; i <= lim; i++) {
        if ((i & 1) == 1) {
            result += ((x >> (xbit - 1)) & 1) * (1 << (i - 1));
            xbit++;
        } else {
            result += ((y >> (ybit - 1)) & 1) * (1 << (i - 1));
            ybit++;
        }
    }
    return result;
}

struct Traj {
    int n = 0;
    std::vector<int32_t> len;
    std::vector<int64_t> off; /* off[t] = first point of trajectory t (1-based), off[n+1] = total */
    std::vector<float> x, y;
    void load(int n_, const int32_t* l, const float* lon, const float* lat) {
        n = n_;
        len.assign(n + 1, 0);
        off.assign(n + 2, 0);
        for (int t = 1; t <= n; t++) {
            len[t] = l[t - 1];
            off[t + 1] = off[t] + len[t];
        }
        x.assign(lon, lon + off[n + 1]);
        y.assign(lat, lat + off[n + 1]);
    }
};

struct Run {
    int tid, start, count; /* start is the point index within the trajectory */
};

/* Splits a trajectory into maximal runs of consecutive points in the same cell, the runs
 * Grid::addTrajectoryIntoCell emits (Grid.cpp:128-199; FSG.cpp:30-86 for FSG). */
template <class CellOf>
void trajectory_runs(const Traj& T, int tid, CellOf cell_of, std::vector<std::pair<int, Run>>& out) {
    int L = T.len[tid];
    if (L == 0) return;
    int64_t o = T.off[tid];
    int last = cell_of(T.x[o], T.y[o]);
    int last_start = 0;
    for (int i = 1; i < L; i++) {
        int c = cell_of(T.x[o + i], T.y[o + i]);
        if (c != last) {
            out.push_back({last, Run{tid, last_start, i - last_start}});
            last = c;
            last_start = i;
        }
    }
    out.push_back({last, Run{tid, last_start, L - last_start}});
}

}  // namespace

/* ================================================================ GT-quadtree */
struct orc_grid {
    Traj T;
    Box range;
    float cell;
    int vparam, leaf_cap;
    int axis, cellnum, total_level;
    std::vector<Box> cell_mbb;
    std::vector<int32_t> cstart, cend; /* inclusive point ranges, end = start - 1 when empty */
    std::vector<float> px, py;
    std::vector<int32_t> ptid, ppidx;
    struct Node {
        int id, level, npts;
        bool leaf;
        Box mbb;
        int child[4];
    };
    std::vector<Node> nodes; /* depth-first order, root at 0 */
    std::vector<std::map<int, int>> fv;

    int cell_of(float lon, float lat) const {
        /* Grid::WhichCellPointIn (Grid.cpp:202-208) */
        int row = (int)((range.ymax - lat) / cell);
        int col = (int)((lon - range.xmin) / cell);
        return morton(col, row);
    }
    int build_node(int level, int id) {
        /* Grid::buildQuadTree (Grid.cpp:58-94) */
        int span = (int)std::pow(4, total_level - level);
        int first = id * span, last = (id + 1) * span - 1;
        int pts = 0;
        for (int i = first; i <= last; i++) pts += cend[i] - cstart[i] + 1;
        Node nd;
        nd.id = id;
        nd.level = level;
        nd.npts = pts;
        nd.mbb = Box{cell_mbb[first].xmin, cell_mbb[last].ymin, cell_mbb[last].xmax, cell_mbb[first].ymax};
        nd.leaf = (pts < leaf_cap) || (level == total_level);
        int me = (int)nodes.size();
        nodes.push_back(nd);
        if (!nd.leaf) {
            for (int c = 0; c < 4; c++) {
                int ch = build_node(level + 1, (id << 2) + c);
                nodes[me].child[c] = ch;
            }
        }
        return me;
    }
    void candidates(int ni, const Box& q, std::vector<int>& out) const {
        /* Grid::findMatchNodeInQuadTree (Grid.cpp:428-446): leaves are taken without a test;
         * children of inner nodes are entered when BoxIntersect(query, child) != 0. */
        const Node& nd = nodes[ni];
        if (nd.leaf) {
            out.push_back(ni);
            return;
        }
        for (int c = 0; c < 4; c++)
            if (box_intersect(q, nodes[nd.child[c]].mbb)) candidates(nd.child[c], q, out);
    }
};

extern "C" orc_grid* orc_grid_build(int n, const int32_t* lengths, const float* lon, const float* lat,
                                    const float box[4], float cell, int vparam, int leaf_cap) {
    orc_grid* g = new orc_grid();
    g->T.load(n, lengths, lon, lat);
    g->range = Box{box[0], box[1], box[2], box[3]};
    g->cell = cell;
    g->vparam = vparam;
    g->leaf_cap = leaf_cap;
    /* Grid::Grid (Grid.cpp:97-124) */
    int dx = (int)((g->range.xmax - g->range.xmin) / cell) + 1;
    int dy = (int)((g->range.ymax - g->range.ymin) / cell) + 1;
    int mv = std::max(dx, dy);
    g->axis = mv >> (int(std::log2(mv))) << (int(std::log2(mv)) + 1);
    g->cellnum = g->axis * g->axis;
    g->total_level = int(std::log2(g->cellnum) / std::log2(4));
    g->cell_mbb.resize(g->cellnum);
    for (int i = 0; i < g->axis; i++)
        for (int j = 0; j < g->axis; j++)
            g->cell_mbb[morton(j, i)] =
                Box{g->range.xmin + cell * j, g->range.ymax - cell * (i + 1), g->range.xmin + cell * (j + 1),
                    g->range.ymax - cell * (i)};
    /* runs per trajectory, appended to cells in trajectory-id order (Grid.cpp:210-226) */
    std::vector<std::vector<Run>> cell_runs(g->cellnum);
    g->fv.assign(n + 1, {});
    std::vector<std::pair<int, Run>> runs;
    for (int t = 1; t <= n; t++) {
        runs.clear();
        trajectory_runs(g->T, t, [g](float a, float b) { return g->cell_of(a, b); }, runs);
        for (auto& r : runs) {
            cell_runs[r.first].push_back(r.second);
            g->fv[t][r.first >> vparam] += r.second.count; /* FVTable::addPointToFVTable */
        }
    }
    /* cell-contiguous point array (Grid.cpp:238-261) */
    g->cstart.resize(g->cellnum);
    g->cend.resize(g->cellnum);
    int pc = 0;
    for (int c = 0; c < g->cellnum; c++) {
        g->cstart[c] = pc;
        for (auto& r : cell_runs[c]) {
            int64_t o = g->T.off[r.tid];
            for (int k = r.start; k < r.start + r.count; k++) {
                g->px.push_back(g->T.x[o + k]);
                g->py.push_back(g->T.y[o + k]);
                g->ptid.push_back(r.tid);
                g->ppidx.push_back(k);
                pc++;
            }
        }
        g->cend[c] = pc - 1;
    }
    g->build_node(0, 0);
    return g;
}

extern "C" void orc_grid_free(orc_grid* g) { delete g; }

extern "C" void orc_grid_meta(const orc_grid* g, int32_t meta[6]) {
    int leaves = 0;
    for (auto& nd : g->nodes) leaves += nd.leaf;
    meta[0] = g->axis;
    meta[1] = g->cellnum;
    meta[2] = (int32_t)g->px.size();
    meta[3] = g->total_level;
    meta[4] = leaves;
    meta[5] = (int32_t)g->nodes.size();
}

extern "C" void orc_grid_points(const orc_grid* g, float* x, float* y, int32_t* tid, int32_t* pidx) {
    size_t n = g->px.size();
    memcpy(x, g->px.data(), n * 4);
    memcpy(y, g->py.data(), n * 4);
    memcpy(tid, g->ptid.data(), n * 4);
    memcpy(pidx, g->ppidx.data(), n * 4);
}

extern "C" void orc_grid_cells(const orc_grid* g, int32_t* start, int32_t* end, float* mbb4) {
    for (int c = 0; c < g->cellnum; c++) {
        start[c] = g->cstart[c];
        end[c] = g->cend[c];
        mbb4[4 * c + 0] = g->cell_mbb[c].xmin;
        mbb4[4 * c + 1] = g->cell_mbb[c].ymin;
        mbb4[4 * c + 2] = g->cell_mbb[c].xmax;
        mbb4[4 * c + 3] = g->cell_mbb[c].ymax;
    }
}

extern "C" void orc_grid_nodes(const orc_grid* g, int32_t* id, int32_t* level, int32_t* npts,
                               int32_t* leaf, float* mbb4) {
    for (size_t i = 0; i < g->nodes.size(); i++) {
        const auto& nd = g->nodes[i];
        id[i] = nd.id;
        level[i] = nd.level;
        npts[i] = nd.npts;
        leaf[i] = nd.leaf;
        mbb4[4 * i + 0] = nd.mbb.xmin;
        mbb4[4 * i + 1] = nd.mbb.ymin;
        mbb4[4 * i + 2] = nd.mbb.xmax;
        mbb4[4 * i + 3] = nd.mbb.ymax;
    }
}

extern "C" int64_t orc_grid_fv(const orc_grid* g, int64_t* off, int32_t* cell, int32_t* count) {
    int64_t k = 0;
    if (off) off[0] = 0;
    for (int t = 0; t <= g->T.n; t++) {
        for (auto& kv : g->fv[t]) {
            if (cell) {
                cell[k] = kv.first;
                count[k] = kv.second;
            }
            k++;
        }
        if (off) off[t + 1] = k;
    }
    return k;
}

namespace {
/* Writes per-query results from a predicate over candidate point ranges. */
template <class ForEachCandidate>
void range_collect(int nq, const float* q4, int mode, int64_t* counts, int32_t* out_a,
                   int32_t* out_b, ForEachCandidate each) {
    int64_t w = 0;
    for (int qi = 0; qi < nq; qi++) {
        Box q{q4[4 * qi], q4[4 * qi + 1], q4[4 * qi + 2], q4[4 * qi + 3]};
        std::vector<std::pair<int32_t, int32_t>> hits;
        each(q, [&](int tid, int pidx) { hits.push_back({tid, mode == 0 ? 0 : pidx}); });
        std::sort(hits.begin(), hits.end());
        hits.erase(std::unique(hits.begin(), hits.end()), hits.end());
        counts[qi] = (int64_t)hits.size();
        if (out_a) {
            for (auto& h : hits) {
                out_a[w] = h.first;
                if (mode == 1 && out_b) out_b[w] = h.second;
                w++;
            }
        }
    }
}
}  // namespace

extern "C" void orc_grid_range(const orc_grid* g, const float* q4, int nq, int mode, int64_t* counts,
                               int32_t* out_a, int32_t* out_b) {
    /* Grid::rangeQueryBatch (Grid.cpp:341-405): every point of every cell of every candidate
     * leaf is tested with MBB::pInBox. */
    range_collect(nq, q4, mode, counts, out_a, out_b, [g](const Box& q, auto emit) {
        std::vector<int> leaves;
        g->candidates(0, q, leaves);
        for (int li : leaves) {
            const auto& nd = g->nodes[li];
            int span = (int)std::pow(4, g->total_level - nd.level);
            int first = nd.id * span, last = (nd.id + 1) * span - 1;
            for (int c = first; c <= last; c++)
                for (int i = g->cstart[c]; i <= g->cend[c]; i++)
                    if (q.in(g->px[i], g->py[i])) emit(g->ptid[i], g->ppidx[i]);
        }
    });
}

extern "C" int orc_grid_candidates(const orc_grid* g, const float q4[4], int32_t* node_id,
                                   int32_t* level) {
    std::vector<int> leaves;
    g->candidates(0, Box{q4[0], q4[1], q4[2], q4[3]}, leaves);
    for (size_t i = 0; i < leaves.size(); i++) {
        if (node_id) node_id[i] = g->nodes[leaves[i]].id;
        if (level) level[i] = g->nodes[leaves[i]].level;
    }
    return (int)leaves.size();
}

/* ================================================================ STIG */
struct orc_stig {
    struct P {
        float x, y;
        int32_t tid, pidx;
    };
    std::vector<P> pts;
    int block;
    struct Node {
        bool leaf;
        int depth;
        float median;
        int l, r;   /* leaf: inclusive range */
        Box mbb;    /* leaf only */
        int left, right;
    };
    std::vector<Node> nodes;
    bool root_leaf;

    static bool cmp_x(const P& a, const P& b) { return a.x < b.x; }
    static bool cmp_y(const P& a, const P& b) { return a.y < b.y; }

    Node make_leaf(int depth, int s, int e) const {
        /* STIG::createIndex(LeafNode*) (STIG.cpp:71-93) */
        float xmin = 999, xmax = -999, ymin = 999, ymax = -999;
        for (int i = s; i <= e; i++) {
            if (pts[i].x < xmin) xmin = pts[i].x;
            if (pts[i].x > xmax) xmax = pts[i].x;
            if (pts[i].y < ymin) ymin = pts[i].y;
            if (pts[i].y > ymax) ymax = pts[i].y;
        }
        Node nd{};
        nd.leaf = true;
        nd.depth = depth;
        nd.l = s;
        nd.r = e;
        nd.mbb = Box{xmin, ymin, xmax, ymax};
        return nd;
    }
    /* The subtree over [s, e] as a node list in depth-first order (its root first), children
     * as indices into the list.
     * STIG::createIndex(InternalNode*) (STIG.cpp:96-168): std::sort over [s, e), the last
     * element excluded; left child [s, m] as a leaf or [s, m-1] as an inner node, right [m, e].
     * A left leaf [s, m] shares index m with the right subtree, so its MBB is taken before the
     * right subtree sorts, as in the reference; an inner left child [s, m-1] is disjoint from
     * [m, e], so the two are built on separate threads for the first `spawn` levels. Every
     * std::sort call sees the same range and contents as in the sequential order, so the
     * result is the same. */
    std::vector<Node> make_internal(int depth, int s, int e, int spawn) {
        if (depth % 2 == 0)
            std::sort(&pts[s], &pts[e], cmp_x);
        else
            std::sort(&pts[s], &pts[e], cmp_y);
        const int m = (s + e) / 2;
        Node nd{};
        nd.leaf = false;
        nd.depth = depth;
        nd.median = depth % 2 == 0 ? pts[m].x : pts[m].y;
        std::vector<Node> lt, rt;
        std::thread worker;
        if (m - s <= block)
            lt.push_back(make_leaf(depth + 1, s, m));
        else if (spawn > 0)
            worker = std::thread([&, spawn]() { lt = make_internal(depth + 1, s, m - 1, spawn - 1); });
        else
            lt = make_internal(depth + 1, s, m - 1, 0);
        if (e - m + 1 <= block)
            rt.push_back(make_leaf(depth + 1, m, e));
        else
            rt = make_internal(depth + 1, m, e, spawn > 0 ? spawn - 1 : 0);
        if (worker.joinable()) worker.join();
        std::vector<Node> out;
        out.reserve(1 + lt.size() + rt.size());
        nd.left = 1;
        nd.right = 1 + (int)lt.size();
        out.push_back(nd);
        for (const auto* part : {&lt, &rt}) {
            const int base = (int)out.size();
            for (Node c : *part) {
                if (!c.leaf) {
                    c.left += base;
                    c.right += base;
                }
                out.push_back(c);
            }
        }
        return out;
    }
    static bool slab(float amin, float amax, float bmin, float bmax) {
        /* STIG::intersectBlock (STIG.cpp:340-347) */
        if (amax < bmin) return false;
        if (amin > bmax) return false;
        return true;
    }
    void search(int ni, const Box& q, std::vector<std::pair<int, int>>& out) const {
        /* STIG::searchNode (STIG.cpp:201-252) */
        const Node& nd = nodes[ni];
        if (nd.leaf) {
            if (box_intersect(nd.mbb, q)) out.push_back({nd.l, nd.r});
            return;
        }
        float lo = nd.depth % 2 == 0 ? q.xmin : q.ymin;
        float hi = nd.depth % 2 == 0 ? q.xmax : q.ymax;
        if (slab(lo, hi, 0, nd.median)) search(nd.left, q, out);
        if (slab(lo, hi, nd.median, 180)) search(nd.right, q, out);
    }
    void leaves(int ni, std::vector<int>& out) const {
        if (nodes[ni].leaf) {
            out.push_back(ni);
            return;
        }
        leaves(nodes[ni].left, out);
        leaves(nodes[ni].right, out);
    }
};

extern "C" orc_stig* orc_stig_build(int n, const int32_t* lengths, const float* lon, const float* lat,
                                    int block_size) {
    if (block_size < 2) return nullptr; /* STIG.cpp:120-130 recurses without end below 2 */
    orc_stig* s = new orc_stig();
    s->block = block_size;
    /* STIG::initial (STIG.cpp:35-66): points in trajectory order */
    int64_t o = 0;
    for (int t = 1; t <= n; t++)
        for (int j = 0; j < lengths[t - 1]; j++, o++) s->pts.push_back({lon[o], lat[o], t, j});
    int total = (int)s->pts.size();
    s->root_leaf = total <= block_size;
    if (s->root_leaf)
        s->nodes.push_back(s->make_leaf(0, 0, total - 1));
    else
        s->nodes = s->make_internal(0, 0, total - 1, 5);
    return s;
}

extern "C" void orc_stig_free(orc_stig* s) { delete s; }
extern "C" int64_t orc_stig_npoints(const orc_stig* s) { return (int64_t)s->pts.size(); }

extern "C" void orc_stig_points(const orc_stig* s, float* x, float* y, int32_t* tid, int32_t* pidx) {
    for (size_t i = 0; i < s->pts.size(); i++) {
        x[i] = s->pts[i].x;
        y[i] = s->pts[i].y;
        tid[i] = s->pts[i].tid;
        pidx[i] = s->pts[i].pidx;
    }
}

extern "C" int orc_stig_leaves(const orc_stig* s, int32_t* lr, float* mbb4) {
    std::vector<int> lv;
    s->leaves(0, lv);
    for (size_t i = 0; i < lv.size(); i++) {
        const auto& nd = s->nodes[lv[i]];
        if (lr) {
            lr[2 * i] = nd.l;
            lr[2 * i + 1] = nd.r;
        }
        if (mbb4) {
            mbb4[4 * i] = nd.mbb.xmin;
            mbb4[4 * i + 1] = nd.mbb.ymin;
            mbb4[4 * i + 2] = nd.mbb.xmax;
            mbb4[4 * i + 3] = nd.mbb.ymax;
        }
    }
    return (int)lv.size();
}

extern "C" int orc_stig_candidates(const orc_stig* s, const float q4[4], int32_t* blocks) {
    std::vector<std::pair<int, int>> out;
    s->search(0, Box{q4[0], q4[1], q4[2], q4[3]}, out);
    for (size_t i = 0; blocks && i < out.size(); i++) {
        blocks[2 * i] = out[i].first;
        blocks[2 * i + 1] = out[i].second;
    }
    return (int)out.size();
}

extern "C" void orc_stig_range(const orc_stig* s, const float* q4, int nq, int mode, int64_t* counts,
                               int32_t* out_a, int32_t* out_b) {
    range_collect(nq, q4, mode, counts, out_a, out_b, [s](const Box& q, auto emit) {
        std::vector<std::pair<int, int>> blocks;
        s->search(0, q, blocks);
        for (auto& b : blocks)
            for (int i = b.first; i <= b.second; i++)
                if (q.in(s->pts[i].x, s->pts[i].y)) emit(s->pts[i].tid, s->pts[i].pidx);
    });
}

/* ================================================================ FSG */
struct orc_fsg {
    Traj T;
    Box range;
    float cell;
    int nx, ny, cellnum;
    std::vector<int32_t> cstart, cend;
    std::vector<float> px, py;
    std::vector<int32_t> ptid, ppidx;
    int cell_of(float lon, float lat) const {
        /* FSG::WhichCellPointIn (FSG.cpp:88-93) */
        int row = (int)((range.ymax - lat) / cell);
        int col = (int)((lon - range.xmin) / cell);
        return row * nx + col;
    }
    void candidates(const Box& q, std::vector<int>& out) const {
        /* FSG::rangeQueryBatchGPU candidate cells (FSG.cpp:183-262): the border ring first,
         * then the interior cells. Indices are not clamped to the grid by the reference. */
        int m = nx;
        int g1 = (int)((q.xmin - range.xmin) / cell);
        int g2 = (int)((q.xmax - range.xmin) / cell);
        int g3 = (int)((range.ymax - q.ymax) / cell);
        int g4 = (int)((range.ymax - q.ymin) / cell);
        int a = g1 + g3 * m, b = g2 + g3 * m, c = g1 + g4 * m, d = g2 + g4 * m;
        for (int i = a; i <= b; i++) out.push_back(i);
        if (g4 - g3 >= 1)
            for (int i = c; i <= d; i++) out.push_back(i);
        if (g4 - g3 >= 2) {
            for (int i = a + m; i <= a + (g4 - g3 - 1) * m; i += m) out.push_back(i);
            if (g2 > g1)
                for (int i = b + m; i <= b + (g4 - g3 - 1) * m; i += m) out.push_back(i);
        }
        if (b >= a + 2 && c >= a + 2 * m)
            for (int i = a + 1; i <= b - 1; i++)
                for (int j = 1; j <= g4 - g3 - 1; j++) out.push_back(i + j * m);
    }
};

extern "C" orc_fsg* orc_fsg_build(int n, const int32_t* lengths, const float* lon, const float* lat,
                                  const float box[4], float cell) {
    orc_fsg* f = new orc_fsg();
    f->T.load(n, lengths, lon, lat);
    f->range = Box{box[0], box[1], box[2], box[3]};
    f->cell = cell;
    /* FSG::FSG (FSG.cpp:7-28) */
    f->nx = (int)((f->range.xmax - f->range.xmin) / cell) + 1;
    f->ny = (int)((f->range.ymax - f->range.ymin) / cell) + 1;
    f->cellnum = f->nx * f->ny;
    std::vector<std::vector<Run>> cell_runs(f->cellnum);
    std::vector<std::pair<int, Run>> runs;
    for (int t = 1; t <= n; t++) {
        runs.clear();
        trajectory_runs(f->T, t, [f](float a, float b) { return f->cell_of(a, b); }, runs);
        for (auto& r : runs) cell_runs[r.first].push_back(r.second);
    }
    f->cstart.resize(f->cellnum);
    f->cend.resize(f->cellnum);
    int pc = 0;
    for (int c = 0; c < f->cellnum; c++) {
        f->cstart[c] = pc;
        for (auto& r : cell_runs[c]) {
            int64_t o = f->T.off[r.tid];
            for (int k = r.start; k < r.start + r.count; k++) {
                f->px.push_back(f->T.x[o + k]);
                f->py.push_back(f->T.y[o + k]);
                f->ptid.push_back(r.tid);
                f->ppidx.push_back(k);
                pc++;
            }
        }
        f->cend[c] = pc - 1;
    }
    return f;
}

extern "C" void orc_fsg_free(orc_fsg* f) { delete f; }
extern "C" void orc_fsg_meta(const orc_fsg* f, int32_t meta[4]) {
    meta[0] = f->nx;
    meta[1] = f->ny;
    meta[2] = f->cellnum;
    meta[3] = (int32_t)f->px.size();
}
extern "C" void orc_fsg_points(const orc_fsg* f, float* x, float* y, int32_t* tid, int32_t* pidx) {
    size_t n = f->px.size();
    memcpy(x, f->px.data(), n * 4);
    memcpy(y, f->py.data(), n * 4);
    memcpy(tid, f->ptid.data(), n * 4);
    memcpy(pidx, f->ppidx.data(), n * 4);
}
extern "C" void orc_fsg_cells(const orc_fsg* f, int32_t* start, int32_t* end) {
    for (int c = 0; c < f->cellnum; c++) {
        start[c] = f->cstart[c];
        end[c] = f->cend[c];
    }
}
extern "C" int orc_fsg_candidates(const orc_fsg* f, const float q4[4], int32_t* cells) {
    std::vector<int> out;
    f->candidates(Box{q4[0], q4[1], q4[2], q4[3]}, out);
    for (size_t i = 0; cells && i < out.size(); i++) cells[i] = out[i];
    return (int)out.size();
}
extern "C" void orc_fsg_range(const orc_fsg* f, const float* q4, int nq, int mode, int64_t* counts,
                              int32_t* out_a, int32_t* out_b) {
    /* Cells whose index falls outside [0, cellnum) are skipped: the reference reads its cell
     * array out of bounds there (undefined behaviour), and no point lies in such a cell. */
    range_collect(nq, q4, mode, counts, out_a, out_b, [f](const Box& q, auto emit) {
        std::vector<int> cells;
        f->candidates(q, cells);
        for (int c : cells) {
            if (c < 0 || c >= f->cellnum) continue;
            for (int i = f->cstart[c]; i <= f->cend[c]; i++)
                if (q.in(f->px[i], f->py[i])) emit(f->ptid[i], f->ppidx[i]);
        }
    });
}

/* ================================================================ EDR */
extern "C" int32_t orc_edr(const float* a, int la, const float* b, int lb, double eps) {
    /* Grid::SimilarityExecuter (Grid.cpp:1222-1318). The query is tra1 (rows) when the
     * candidate is at least as long, else the candidate is. */
    const float *t1, *t2;
    int l1, l2;
    if (lb >= la) {
        t1 = a;
        t2 = b;
        l1 = la;
        l2 = lb;
    } else {
        t1 = b;
        t2 = a;
        l1 = lb;
        l2 = la;
    }
    std::vector<int> prev(l2 + 1), cur(l2 + 1);
    for (int c = 0; c <= l2; c++) prev[c] = c;
    for (int r = 1; r <= l1; r++) {
        cur[0] = r;
        float px = t1[2 * (r - 1)], py = t1[2 * (r - 1) + 1];
        for (int c = 1; c <= l2; c++) {
            float qx = t2[2 * (c - 1)], qy = t2[2 * (c - 1) + 1];
            /* fabs of the float difference, compared in double against EPSILON (Grid.cpp:1281) */
            bool match = ((double)std::fabs(px - qx) < eps) && ((double)std::fabs(py - qy) < eps);
            int subcost = match ? 0 : 1;
            int m = prev[c - 1] + subcost;
            int u = prev[c] + 1;
            int l = cur[c - 1] + 1;
            /* Grid.cpp:1297-1300 */
            bool c1 = (m < u) && (m < l);
            bool c2 = (l < u) && (l < m);
            cur[c] = c1 * m + c2 * l + !(c1 || c2) * u;
        }
        std::swap(prev, cur);
    }
    return prev[l2];
}

extern "C" void orc_edr_batch(int npairs, const int32_t* la, const int64_t* oa, const float* a,
                              const int32_t* lb, const int64_t* ob, const float* b, double eps,
                              int threads, int32_t* out) {
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            int i = next.fetch_add(1);
            if (i >= npairs) break;
            out[i] = orc_edr(a + 2 * oa[i], la[i], b + 2 * ob[i], lb[i], eps);
        }
    };
    if (threads <= 1) {
        work();
        return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < threads; t++) th.emplace_back(work);
    for (auto& t : th) t.join();
}

/* ================================================================ FV lower bound */
extern "C" void orc_fv_neighbors(int vcell_count, int cell, int32_t out[8]) {
    /* FVTable::findNeighbor (FVTable.cpp:53-75) */
    int x = 0, y = 0;
    int bits = int(std::log2(vcell_count));
    for (int bit = 0; bit <= bits - 1; bit++) {
        if (bit % 2 == 0)
            x += ((cell >> bit) & 1) * (1 << (bit / 2));
        else
            y += ((cell >> bit) & 1) * (1 << (bit / 2));
    }
    int cnt = 0;
    for (int xx = x - 1; xx <= x + 1; xx++)
        for (int yy = y - 1; yy <= y + 1; yy++)
            if (xx != x || yy != y) out[cnt++] = morton(xx, yy);
}

namespace {
/* FVTable::formPriorityQueue body for one trajectory (FVTable.cpp:81-202). The reference
 * increments a std::map iterator after erasing its node (undefined behaviour); this
 * restatement visits every key present when each pass starts, in ascending order, once. */
int fv_lb_one(const std::map<int, int>& db, const std::map<int, int>& q, int vcells) {
    std::map<int, int> pos, neg;
    for (auto& kv : db) {
        auto it = q.find(kv.first);
        if (it == q.end()) {
            pos.insert({kv.first, kv.second});
        } else {
            int d = kv.second - it->second;
            if (d > 0)
                pos.insert({kv.first, d});
            else if (d < 0)
                neg.insert({kv.first, -d});
        }
    }
    for (auto& kv : q) {
        if (db.count(kv.first)) continue;
        int d = -kv.second;
        if (d > 0)
            pos.insert({kv.first, d});
        else if (d < 0)
            neg.insert({kv.first, -d});
    }
    std::vector<int> keys;
    for (auto& kv : pos) keys.push_back(kv.first);
    for (int cid : keys) {
        auto self = pos.find(cid);
        if (self == pos.end()) continue;
        int pv = self->second; /* never refreshed inside the neighbour loop (FVTable.cpp:132) */
        int32_t nb[8];
        orc_fv_neighbors(vcells, cid, nb);
        for (int i = 0; i < 8; i++) {
            auto it = neg.find(nb[i]);
            if (it == neg.end()) continue;
            int nv = it->second;
            if (pv > nv) {
                pos[cid] = pv - nv;
                neg.erase(nb[i]);
            } else if (pv == nv) {
                pos.erase(cid);
                neg.erase(nb[i]);
                break;
            } else {
                neg[nb[i]] = nv - pv;
                pos.erase(cid);
                break;
            }
        }
    }
    keys.clear();
    for (auto& kv : neg) keys.push_back(kv.first);
    for (int cid : keys) {
        auto self = neg.find(cid);
        if (self == neg.end()) continue;
        int nv = self->second;
        int32_t nb[8];
        orc_fv_neighbors(vcells, cid, nb);
        for (int i = 0; i < 8; i++) {
            auto it = pos.find(nb[i]);
            if (it == pos.end()) continue;
            int pv = it->second;
            if (nv > pv) {
                neg[cid] = nv - pv;
                pos.erase(nb[i]);
            } else if (pv == nv) {
                neg.erase(cid);
                pos.erase(nb[i]);
                break;
            } else {
                pos[nb[i]] = pv - nv;
                neg.erase(cid);
                break;
            }
        }
    }
    int sp = 0, sn = 0;
    for (auto& kv : pos) sp += kv.second;
    for (auto& kv : neg) sn += kv.second;
    return std::max(sp, sn);
}
}  // namespace

extern "C" int orc_grid_query_fv(const orc_grid* g, const float* lon, const float* lat, int len,
                                 int32_t* cell, int32_t* count) {
    std::map<int, int> fv;
    for (int p = 0; p < len; p++) fv[g->cell_of(lon[p], lat[p]) >> g->vparam] += 1;
    int k = 0;
    for (auto& kv : fv) {
        if (cell) {
            cell[k] = kv.first;
            count[k] = kv.second;
        }
        k++;
    }
    return k;
}

extern "C" void orc_grid_fv_lb(const orc_grid* g, int qnnz, const int32_t* qcell, const int32_t* qcount,
                               int32_t* lb) {
    std::map<int, int> q;
    for (int i = 0; i < qnnz; i++) q[qcell[i]] = qcount[i];
    /* FVTable::initFVTable is given cellnum >> 2 virtual cells (Grid.cpp:214) */
    int vcells = g->cellnum >> 2;
    lb[0] = 0;
    for (int t = 1; t <= g->T.n; t++) lb[t] = fv_lb_one(g->fv[t], q, vcells);
}

/* ================================================================ top-k */
extern "C" void orc_grid_topk(const orc_grid* g, const float* qlon, const float* qlat, int qlen, int k,
                              double eps, int pruned, int threads, int32_t* ids, int32_t* dist,
                              int64_t* evaluated) {
    int n = g->T.n;
    std::vector<float> qa(2 * qlen);
    for (int i = 0; i < qlen; i++) {
        qa[2 * i] = qlon[i];
        qa[2 * i + 1] = qlat[i];
    }
    auto edr_of = [&](int t) {
        std::vector<float> c(2 * g->T.len[t]);
        int64_t o = g->T.off[t];
        for (int i = 0; i < g->T.len[t]; i++) {
            c[2 * i] = g->T.x[o + i];
            c[2 * i + 1] = g->T.y[o + i];
        }
        return orc_edr(qa.data(), qlen, c.data(), g->T.len[t], eps);
    };
    std::vector<std::pair<int, int>> best; /* (dist, id) */
    int64_t evals = 0;
    if (!pruned) {
        std::vector<int> d(n + 1);
        std::atomic<int> next(1);
        auto work = [&]() {
            for (;;) {
                int t = next.fetch_add(1);
                if (t > n) break;
                d[t] = edr_of(t);
            }
        };
        std::vector<std::thread> th;
        for (int i = 0; i < std::max(1, threads); i++) th.emplace_back(work);
        for (auto& t : th) t.join();
        for (int t = 1; t <= n; t++) best.push_back({d[t], t});
        evals = n;
    } else {
        /* Pruned walk in two phases, exact for (distance, id) order whenever the bound holds:
         * (1) evaluate candidates in ascending lower-bound order while the bound is below the
         *     current k-th distance W (the reference's loop condition, Grid.cpp:917);
         * (2) candidates whose bound equals W can still tie at W; walk them in ascending id
         *     order and stop once k results with ids below the next candidate are known. */
        std::vector<int32_t> qc(qlen + 1), qn(qlen + 1);
        int nnz = orc_grid_query_fv(g, qlon, qlat, qlen, qc.data(), qn.data());
        std::vector<int32_t> lb(n + 1);
        orc_grid_fv_lb(g, nnz, qc.data(), qn.data(), lb.data());
        std::vector<std::pair<int, int>> order;
        for (int t = 1; t <= n; t++) order.push_back({lb[t], t});
        std::sort(order.begin(), order.end());
        auto kth = [&]() {
            std::vector<std::pair<int, int>> tmp = best;
            std::nth_element(tmp.begin(), tmp.begin() + (k - 1), tmp.end());
            return tmp[k - 1].first;
        };
        size_t i = 0;
        for (; i < order.size(); i++) {
            if ((int)best.size() >= k && order[i].first >= kth()) break;
            best.push_back({edr_of(order[i].second), order[i].second});
            evals++;
        }
        if ((int)best.size() >= k) {
            int W = kth();
            for (; i < order.size() && order[i].first == W; i++) {
                int below = 0; /* results that sort before (W, this id) */
                for (auto& b : best)
                    if (b.first < W || (b.first == W && b.second < order[i].second)) below++;
                if (below >= k) break;
                best.push_back({edr_of(order[i].second), order[i].second});
                evals++;
            }
        }
    }
    std::sort(best.begin(), best.end());
    for (int i = 0; i < k; i++) {
        ids[i] = i < (int)best.size() ? best[i].second : -1;
        dist[i] = i < (int)best.size() ? best[i].first : -1;
    }
    if (evaluated) *evaluated = evals;
}
