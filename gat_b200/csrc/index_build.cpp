/* Builders of the three range indexes, in the reference's exact layouts, uploaded to HBM.
 *
 * The builders reproduce the reference's float arithmetic (cell assignment, cell and node MBBs)
 * with the same expressions in the same types and no FP contraction, so every point lands in
 * the same cell and every node gets the same MBB as in the reference. The work is organised
 * differently: runs are produced per trajectory in parallel and placed with a stable counting
 * sort by cell, which yields the reference's order (cells ascending, trajectories ascending
 * within a cell, runs in trajectory order) without its per-cell linked lists. On a context with
 * a device the Grid and FSG builds run there instead (index_gpu.cu), with the same result.
 */
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <thread>
#include <unordered_map>

#include "internal.h"

namespace gat {
namespace {

unsigned host_threads() { return std::max(1u, std::min(32u, std::thread::hardware_concurrency())); }

template <class F>
void parallel_chunks(int64_t n, F f) {
    unsigned hw = host_threads();
    if (n < 8192 || hw == 1) {
        f(0, n, 0);
        return;
    }
    std::vector<std::thread> th;
    int64_t per = (n + hw - 1) / hw;
    for (unsigned t = 0; t < hw; t++) {
        int64_t s = t * per, e = std::min(n, s + per);
        if (s >= e) break;
        th.emplace_back([=]() { f(s, e, (int)t); });
    }
    for (auto& x : th) x.join();
}

/* Morton id of non-negative (x, y): x bits on even positions starting at bit 0, the id
 * getIdxFromXY (Grid.cpp:25-54) computes for in-grid cells. */
inline uint32_t spread(uint32_t v) {
    v &= 0xFFFF;
    v = (v | (v << 8)) & 0x00FF00FF;
    v = (v | (v << 4)) & 0x0F0F0F0F;
    v = (v | (v << 2)) & 0x33333333;
    v = (v | (v << 1)) & 0x55555555;
    return v;
}
inline uint32_t compact(uint32_t v) {
    v &= 0x55555555;
    v = (v | (v >> 1)) & 0x33333333;
    v = (v | (v >> 2)) & 0x0F0F0F0F;
    v = (v | (v >> 4)) & 0x00FF00FF;
    v = (v | (v >> 8)) & 0x0000FFFF;
    return v;
}
inline int morton(int x, int y) { return (int)(spread((uint32_t)x) | (spread((uint32_t)y) << 1)); }

int bits_for(int64_t v) {
    int b = 1;
    while (b < 62 && (int64_t(1) << b) <= v) b++;
    return b;
}

struct RunSet {
    /* runs in trajectory order: cell, trajectory, first point index, point count */
    std::vector<int32_t> cell, tid, start, count;
    std::vector<int64_t> traj_first; /* first run of trajectory t (1-based), size n+2 */
};

/* Maximal runs of consecutive points in one cell per trajectory (Grid.cpp:128-199,
 * FSG.cpp:30-86). cell_of returns -1 for a point outside the grid. */
int make_runs(const gat_db* db, const std::function<int(float, float)>& cell_of, RunSet& rs) {
    int n = db->n;
    std::vector<int64_t> nruns(n + 2, 0);
    std::atomic<int> bad(0);
    parallel_chunks(n, [&](int64_t s, int64_t e, int) {
        for (int64_t i = s; i < e; i++) {
            int t = (int)i + 1;
            int64_t o = db->h_off[t];
            int L = db->h_len[t];
            int cnt = 0, last = INT_MIN;
            for (int k = 0; k < L; k++) {
                int c = cell_of(db->h_x[o + k], db->h_y[o + k]);
                if (c < 0) bad = 1;
                if (c != last) cnt++;
                last = c;
            }
            nruns[t + 1] = cnt;
        }
    });
    if (bad) return GAT_ERR_ARG;
    for (int t = 1; t <= n; t++) nruns[t + 1] += nruns[t];
    rs.traj_first = nruns;
    int64_t R = nruns[n + 1];
    rs.cell.resize(R);
    rs.tid.resize(R);
    rs.start.resize(R);
    rs.count.resize(R);
    parallel_chunks(n, [&](int64_t s, int64_t e, int) {
        for (int64_t i = s; i < e; i++) {
            int t = (int)i + 1;
            int64_t o = db->h_off[t], w = nruns[t];
            int L = db->h_len[t];
            int last = INT_MIN, st = 0;
            for (int k = 0; k < L; k++) {
                int c = cell_of(db->h_x[o + k], db->h_y[o + k]);
                if (c != last) {
                    if (k > 0) {
                        rs.cell[w] = last;
                        rs.tid[w] = t;
                        rs.start[w] = st;
                        rs.count[w] = k - st;
                        w++;
                    }
                    last = c;
                    st = k;
                }
            }
            if (L > 0) {
                rs.cell[w] = last;
                rs.tid[w] = t;
                rs.start[w] = st;
                rs.count[w] = L - st;
            }
        }
    });
    return GAT_OK;
}

/* Stable counting sort of the runs by cell, then the cell-contiguous point arrays:
 * cell_beg[c] .. cell_beg[c+1] holds cell c's points (Grid.cpp:238-261). */
void place_points(const gat_db* db, const RunSet& rs, int ncells, gat_index* ix, std::vector<int64_t>& cell_beg) {
    int64_t R = (int64_t)rs.cell.size();
    unsigned hw = host_threads();
    if (R < 65536) hw = 1;
    int64_t per = (R + hw - 1) / std::max<int64_t>(1, hw);
    /* per-thread point counts per cell over contiguous run ranges */
    std::vector<std::vector<int64_t>> hist(hw, std::vector<int64_t>(ncells, 0));
    {
        std::vector<std::thread> th;
        for (unsigned t = 0; t < hw; t++)
            th.emplace_back([&, t]() {
                int64_t s = t * per, e = std::min(R, s + per);
                for (int64_t r = s; r < e; r++) hist[t][rs.cell[r]] += rs.count[r];
            });
        for (auto& x : th) x.join();
    }
    cell_beg.assign(ncells + 1, 0);
    for (int c = 0; c < ncells; c++) {
        int64_t tot = 0;
        for (unsigned t = 0; t < hw; t++) tot += hist[t][c];
        cell_beg[c + 1] = cell_beg[c] + tot;
    }
    /* each thread's write cursor per cell = cell start + points of earlier threads */
    for (int c = 0; c < ncells; c++) {
        int64_t cur = cell_beg[c];
        for (unsigned t = 0; t < hw; t++) {
            int64_t h = hist[t][c];
            hist[t][c] = cur;
            cur += h;
        }
    }
    int64_t P = cell_beg[ncells];
    ix->npoints = P;
    ix->h_x.resize(P);
    ix->h_y.resize(P);
    ix->h_tid.resize(P);
    ix->h_pidx.resize(P);
    std::vector<std::thread> th;
    for (unsigned t = 0; t < hw; t++)
        th.emplace_back([&, t]() {
            int64_t s = t * per, e = std::min(R, s + per);
            for (int64_t r = s; r < e; r++) {
                int64_t w = hist[t][rs.cell[r]];
                int tid = rs.tid[r];
                int64_t o = db->h_off[tid] + rs.start[r];
                for (int k = 0; k < rs.count[r]; k++) {
                    ix->h_x[w + k] = db->h_x[o + k];
                    ix->h_y[w + k] = db->h_y[o + k];
                    ix->h_tid[w + k] = tid;
                    ix->h_pidx[w + k] = rs.start[r] + k;
                }
                hist[t][rs.cell[r]] = w + rs.count[r];
            }
        });
    for (auto& x : th) x.join();
}

/* Uploads the index-order point arrays (x, y, tid, key). */
int upload_points(gat_index* ix) {
    int st = GAT_OK;
    if (ix->ctx->device < 0) return GAT_OK; /* host-only context: layout only */
    const gat_db* db = ix->db;
    int tid_bits = bits_for(db->n);
    ix->pidx_bits = bits_for(std::max(1, db->maxlen - 1));
    std::vector<uint32_t> key(ix->npoints);
    bool fits = tid_bits + ix->pidx_bits <= 32;
    for (int64_t i = 0; i < ix->npoints; i++)
        key[i] = fits ? ((uint32_t)ix->h_tid[i] << ix->pidx_bits) | (uint32_t)ix->h_pidx[i] : 0u;
    if (!fits) ix->pidx_bits = -1; /* point-level results unavailable for this set */
    if (!(ix->d_x = index_upload(ix, ix->h_x, &st))) return st;
    if (!(ix->d_y = index_upload(ix, ix->h_y, &st))) return st;
    if (!(ix->d_tid = index_upload(ix, ix->h_tid, &st))) return st;
    if (!(ix->d_key = index_upload(ix, key, &st))) return st;
    return GAT_OK;
}

/* Whether points are placed on the device (GAT_TUNE_INDEX_BUILD); GAT_ERR_STATE when the device
 * is asked for on a host-only context. */
int use_device(gat_index* ix, const char* what, bool* dev) {
    const gat_ctx* ctx = ix->ctx;
    if (ctx->index_build == 2 && ctx->device < 0)
        return fail(ix->ctx, GAT_ERR_STATE, std::string(what) + ": device build asked for on a host-only context");
    *dev = ctx->device >= 0 && ctx->index_build != 1;
    return GAT_OK;
}

/* Host placement for the Grid: runs, the stable counting sort by cell and the frequency vectors
 * over virtual cells cell >> vparam (Grid.cpp:152-166; FVTable.cpp:18-30). cb stays empty when a
 * point lies outside the grid. */
template <class CellOf>
void host_place_grid(gat_index* ix, const CellOf& cell_of, int vparam, std::vector<int64_t>& cb,
                     std::vector<int64_t>& fv_off, std::vector<int32_t>& fv_cell, std::vector<int32_t>& fv_cnt) {
    const gat_db* db = ix->db;
    RunSet rs;
    if (make_runs(db, cell_of, rs) != GAT_OK) return;
    place_points(db, rs, ix->grid.cellnum, ix, cb);
    int n = db->n;
    fv_off.assign(n + 2, 0);
    std::vector<std::vector<std::pair<int32_t, int32_t>>> fv_tmp(n + 1);
    parallel_chunks(n, [&](int64_t s, int64_t e, int) {
        for (int64_t i = s; i < e; i++) {
            int t = (int)i + 1;
            auto& v = fv_tmp[t];
            for (int64_t r = rs.traj_first[t]; r < rs.traj_first[t + 1]; r++) v.push_back({rs.cell[r] >> vparam, rs.count[r]});
            std::sort(v.begin(), v.end(), [](auto& a, auto& b) { return a.first < b.first; });
            size_t w = 0;
            for (size_t k = 0; k < v.size(); k++) {
                if (w > 0 && v[w - 1].first == v[k].first)
                    v[w - 1].second += v[k].second;
                else
                    v[w++] = v[k];
            }
            v.resize(w);
        }
    });
    int maxnnz = 0;
    for (int t = 0; t <= n; t++) {
        fv_off[t + 1] = fv_off[t] + (int64_t)fv_tmp[t].size();
        maxnnz = std::max(maxnnz, (int)fv_tmp[t].size());
    }
    ix->fv_max_nnz = maxnnz;
    ix->fv_entries = fv_off[n + 1];
    fv_cell.resize(fv_off[n + 1]);
    fv_cnt.resize(fv_off[n + 1]);
    for (int t = 0; t <= n; t++)
        for (size_t k = 0; k < fv_tmp[t].size(); k++) {
            fv_cell[fv_off[t] + k] = fv_tmp[t][k].first;
            fv_cnt[fv_off[t] + k] = fv_tmp[t][k].second;
        }
}

}  // namespace

/* ================================================================ Grid (GT-quadtree) */
static int build_grid(gat_index* ix, gat_mbb range, float cell, int vparam, int leaf_cap) {
    GridDev& g = ix->grid;
    g.rxmin = range.xmin;
    g.rymin = range.ymin;
    g.rxmax = range.xmax;
    g.rymax = range.ymax;
    g.cell = cell;
    g.vparam = vparam;
    /* Grid::Grid (Grid.cpp:104-109) */
    int dx = (int)((range.xmax - range.xmin) / cell) + 1;
    int dy = (int)((range.ymax - range.ymin) / cell) + 1;
    int mv = std::max(dx, dy);
    if (mv <= 0 || mv > (1 << 14)) return fail(ix->ctx, GAT_ERR_ARG, "gat_grid_build: grid larger than 2^15 cells per axis");
    g.axis = mv >> (int(std::log2(mv))) << (int(std::log2(mv)) + 1);
    g.cellnum = g.axis * g.axis;
    g.total_level = int(std::log2(g.cellnum) / std::log2(4));
    const int axis = g.axis;
    /* Grid::WhichCellPointIn (Grid.cpp:202-208); -1 outside the grid */
    auto cell_of = [range, cell, axis](float lon, float lat) -> int {
        int row = (int)((range.ymax - lat) / cell);
        int col = (int)((lon - range.xmin) / cell);
        if (row < 0 || col < 0 || row >= axis || col >= axis) return -1;
        return morton(col, row);
    };
    bool dev = false;
    if (int st = use_device(ix, "gat_grid_build", &dev)) return st;
    if (dev) {
        /* points, quadtree and frequency vectors built in HBM (index_gpu.cu) */
        DevicePlaceArgs a{"gat_grid_build", true, range.xmin, range.ymax, cell, axis, 0, 0, vparam, g.cellnum};
        return device_build_grid(ix, a, g.total_level, leaf_cap);
    }
    if (int st = db_host_copies(ix->db)) return st;
    std::vector<int64_t> cb;
    std::vector<int64_t> fv_off;
    std::vector<int32_t> fv_cell, fv_cnt;
    host_place_grid(ix, cell_of, vparam, cb, fv_off, fv_cell, fv_cnt);
    if (cb.empty()) return fail(ix->ctx, GAT_ERR_ARG, "gat_grid_build: a point lies outside the grid range");
    /* quadtree, breadth first (Grid::buildQuadTree, Grid.cpp:58-94) */
    auto cell_box = [&](int c) {
        int col = (int)compact((uint32_t)c), row = (int)compact((uint32_t)c >> 1);
        /* Grid.cpp:121 */
        return make_float4(range.xmin + cell * col, range.ymax - cell * (row + 1), range.xmin + cell * (col + 1),
                           range.ymax - cell * (row));
    };
    std::vector<float4> nmbb;
    std::vector<int32_t> nchild, npbeg, npend;
    struct Q {
        int level, id;
    };
    std::vector<Q> queue;
    queue.push_back({0, 0});
    int64_t leaves = 0;
    for (size_t qi = 0; qi < queue.size(); qi++) {
        Q q = queue[qi];
        int64_t span = 1;
        for (int l = q.level; l < g.total_level; l++) span *= 4;
        int64_t first = (int64_t)q.id * span, last = first + span - 1;
        int64_t pts = cb[last + 1] - cb[first];
        float4 a = cell_box((int)first), b = cell_box((int)last);
        nmbb.push_back(make_float4(a.x, b.y, b.z, a.w));
        npbeg.push_back((int32_t)cb[first]);
        npend.push_back((int32_t)cb[last + 1]);
        bool leaf = (pts < leaf_cap) || (q.level == g.total_level);
        if (leaf) {
            nchild.push_back(-1);
            leaves++;
        } else {
            nchild.push_back((int32_t)queue.size());
            for (int c = 0; c < 4; c++) queue.push_back({q.level + 1, (q.id << 2) + c});
        }
    }
    g.nnodes = (int)queue.size();
    ix->nodes = g.nnodes;
    ix->leaves = leaves;

    int st = upload_points(ix);
    if (st != GAT_OK || ix->ctx->device < 0) return st;
    if (!(g.node_mbb = index_upload(ix, nmbb, &st))) return st;
    if (!(g.node_child = index_upload(ix, nchild, &st))) return st;
    if (!(g.node_pbeg = index_upload(ix, npbeg, &st))) return st;
    if (!(g.node_pend = index_upload(ix, npend, &st))) return st;
    if (!(ix->d_fv_off = index_upload(ix, fv_off, &st))) return st;
    if (!(ix->d_fv_cell = index_upload(ix, fv_cell, &st))) return st;
    if (!(ix->d_fv_cnt = index_upload(ix, fv_cnt, &st))) return st;
    return GAT_OK;
}

/* ================================================================ STIG */
namespace {
struct SP {
    float x, y;
    int32_t tid, pidx;
};
/* STIG.cpp:27-33 */
bool sp_cmp_x(const SP& a, const SP& b) { return a.x < b.x; }
bool sp_cmp_y(const SP& a, const SP& b) { return a.y < b.y; }

struct SNode {
    bool leaf = false;
    int depth = 0;
    float median = 0;
    int lo = 0, hi = 0;
    float4 mbb{};
    std::unique_ptr<SNode> left, right;
};

struct StigBuilder {
    std::vector<SP>& p;
    int block;
    explicit StigBuilder(std::vector<SP>& pts, int b) : p(pts), block(b) {}

    void leaf(SNode* nd, int depth, int s, int e) {
        /* STIG::createIndex(LeafNode*) (STIG.cpp:71-93) */
        nd->leaf = true;
        nd->depth = depth;
        nd->lo = s;
        nd->hi = e;
        float xmin = 999, xmax = -999, ymin = 999, ymax = -999;
        for (int i = s; i <= e; i++) {
            if (p[i].x < xmin) xmin = p[i].x;
            if (p[i].x > xmax) xmax = p[i].x;
            if (p[i].y < ymin) ymin = p[i].y;
            if (p[i].y > ymax) ymax = p[i].y;
        }
        nd->mbb = make_float4(xmin, ymin, xmax, ymax);
    }
    /* STIG::createIndex(InternalNode*) (STIG.cpp:96-168). Subtrees touch disjoint ranges
     * except that a left leaf [s, m] shares index m with the right subtree [m, e]; the left
     * leaf's MBB is taken before the right subtree is built, as in the reference. Disjoint
     * subtrees are built on separate threads near the root. */
    void internal(SNode* nd, int depth, int s, int e, int spawn) {
        nd->depth = depth;
        if (depth % 2 == 0)
            std::sort(&p[s], &p[e], sp_cmp_x);
        else
            std::sort(&p[s], &p[e], sp_cmp_y);
        int m = (s + e) / 2;
        nd->median = depth % 2 == 0 ? p[m].x : p[m].y;
        nd->left.reset(new SNode());
        nd->right.reset(new SNode());
        bool left_leaf = m - s <= block;
        bool right_leaf = e - m + 1 <= block;
        std::thread lt;
        if (left_leaf) {
            leaf(nd->left.get(), depth + 1, s, m);
        } else if (spawn > 0) {
            SNode* l = nd->left.get();
            lt = std::thread([this, l, depth, s, m, spawn]() { internal(l, depth + 1, s, m - 1, spawn - 1); });
        } else {
            internal(nd->left.get(), depth + 1, s, m - 1, 0);
        }
        if (right_leaf)
            leaf(nd->right.get(), depth + 1, m, e);
        else
            internal(nd->right.get(), depth + 1, m, e, spawn > 0 ? spawn - 1 : 0);
        if (lt.joinable()) lt.join();
    }
};

void flatten(const SNode* nd, std::vector<const SNode*>& order) {
    order.push_back(nd);
    if (!nd->leaf) {
        flatten(nd->left.get(), order);
        flatten(nd->right.get(), order);
    }
}
}  // namespace

static int build_stig(gat_index* ix, int block) {
    const gat_db* db = ix->db;
    if (int st = db_host_copies(db)) return st;
    /* STIG::initial (STIG.cpp:35-66): points in trajectory order */
    std::vector<SP> pts(db->npoints);
    for (int t = 1; t <= db->n; t++)
        for (int k = 0; k < db->h_len[t]; k++) {
            int64_t o = db->h_off[t] + k;
            pts[o] = SP{db->h_x[o], db->h_y[o], t, k};
        }
    int total = (int)pts.size();
    if (total == 0) return fail(ix->ctx, GAT_ERR_ARG, "gat_stig_build: empty trajectory set");
    SNode root;
    StigBuilder b(pts, block);
    if (total <= block)
        b.leaf(&root, 0, 0, total - 1);
    else
        b.internal(&root, 0, 0, total - 1, 5);
    std::vector<const SNode*> order;
    flatten(&root, order);
    std::vector<int32_t> kind, dim, left, right, lo, hi;
    std::vector<float> median;
    std::vector<float4> mbb;
    /* children indices in the depth-first order */
    std::unordered_map<const SNode*, int> index_of;
    for (size_t i = 0; i < order.size(); i++) index_of[order[i]] = (int)i;
    int64_t leaves = 0;
    for (const SNode* s : order) {
        kind.push_back(s->leaf ? 1 : 0);
        dim.push_back(s->depth % 2);
        median.push_back(s->median);
        left.push_back(s->leaf ? -1 : index_of[s->left.get()]);
        right.push_back(s->leaf ? -1 : index_of[s->right.get()]);
        lo.push_back(s->lo);
        hi.push_back(s->hi);
        mbb.push_back(s->mbb);
        leaves += s->leaf;
    }
    ix->leaves = leaves;
    ix->nodes = (int64_t)order.size();
    ix->npoints = total;
    ix->h_x.resize(total);
    ix->h_y.resize(total);
    ix->h_tid.resize(total);
    ix->h_pidx.resize(total);
    for (int i = 0; i < total; i++) {
        ix->h_x[i] = pts[i].x;
        ix->h_y[i] = pts[i].y;
        ix->h_tid[i] = pts[i].tid;
        ix->h_pidx[i] = pts[i].pidx;
    }
    int st = upload_points(ix);
    if (st != GAT_OK || ix->ctx->device < 0) return st;
    StigDev& d = ix->stig;
    d.nnodes = (int)order.size();
    if (!(d.kind = index_upload(ix, kind, &st))) return st;
    if (!(d.dim = index_upload(ix, dim, &st))) return st;
    if (!(d.median = index_upload(ix, median, &st))) return st;
    if (!(d.left = index_upload(ix, left, &st))) return st;
    if (!(d.right = index_upload(ix, right, &st))) return st;
    if (!(d.lo = index_upload(ix, lo, &st))) return st;
    if (!(d.hi = index_upload(ix, hi, &st))) return st;
    if (!(d.mbb = index_upload(ix, mbb, &st))) return st;
    return GAT_OK;
}

/* ================================================================ FSG */
static int build_fsg(gat_index* ix, gat_mbb range, float cell) {
    FsgDev& f = ix->fsg;
    f.rxmin = range.xmin;
    f.rymin = range.ymin;
    f.rxmax = range.xmax;
    f.rymax = range.ymax;
    f.cell = cell;
    /* FSG::FSG (FSG.cpp:11-13) */
    f.nx = (int)((range.xmax - range.xmin) / cell) + 1;
    f.ny = (int)((range.ymax - range.ymin) / cell) + 1;
    if (f.nx <= 0 || f.ny <= 0 || (int64_t)f.nx * f.ny > (int64_t)1 << 30)
        return fail(ix->ctx, GAT_ERR_ARG, "gat_fsg_build: bad grid size");
    f.cellnum = f.nx * f.ny;
    const int nx = f.nx, ny = f.ny;
    /* FSG::WhichCellPointIn (FSG.cpp:88-93); -1 outside the grid */
    auto cell_of = [range, cell, nx, ny](float lon, float lat) -> int {
        int row = (int)((range.ymax - lat) / cell);
        int col = (int)((lon - range.xmin) / cell);
        if (row < 0 || col < 0 || row >= ny || col >= nx) return -1;
        return row * nx + col;
    };
    bool dev = false;
    if (int st = use_device(ix, "gat_fsg_build", &dev)) return st;
    if (dev) {
        /* points and cell ranges built in HBM (index_gpu.cu) */
        DevicePlaceArgs a{"gat_fsg_build", false, range.xmin, range.ymax, cell, 0, nx, ny, 0, f.cellnum};
        return device_build_fsg(ix, a);
    }
    if (int st = db_host_copies(ix->db)) return st;
    std::vector<int64_t> cb;
    RunSet rs;
    if (make_runs(ix->db, cell_of, rs) != GAT_OK)
        return fail(ix->ctx, GAT_ERR_ARG, "gat_fsg_build: a point lies outside the grid range");
    place_points(ix->db, rs, f.cellnum, ix, cb);
    std::vector<int32_t> cbeg(f.cellnum), cend(f.cellnum);
    for (int c = 0; c < f.cellnum; c++) {
        cbeg[c] = (int32_t)cb[c];
        cend[c] = (int32_t)cb[c + 1];
    }
    ix->leaves = f.cellnum;
    int st = upload_points(ix);
    if (st != GAT_OK || ix->ctx->device < 0) return st;
    if (!(f.cbeg = index_upload(ix, cbeg, &st))) return st;
    if (!(f.cend = index_upload(ix, cend, &st))) return st;
    return GAT_OK;
}

}  // namespace gat

using namespace gat;

static int finish_build(gat_ctx* ctx, gat_index* ix, int st, gat_index** out) {
    if (st == GAT_OK) st = index_point_boxes(ix);
    if (st != GAT_OK) {
        gat_index_destroy(ix);
        return st;
    }
    *out = ix;
    return GAT_OK;
}

extern "C" {

int gat_grid_build(gat_ctx* ctx, const gat_db* db, gat_mbb range, float cell_size, int virtual_cell_param,
                   int leaf_cap, gat_index** out) {
    if (!ctx || !db || !out || !(cell_size > 0) || leaf_cap < 1 || virtual_cell_param < 0 || virtual_cell_param > 16 ||
        !(range.xmax > range.xmin) || !(range.ymax > range.ymin))
        return fail(ctx, GAT_ERR_ARG, "gat_grid_build: bad arguments");
    if (db->ctx != ctx) return fail(ctx, GAT_ERR_STATE, "gat_grid_build: trajectory set from another context");
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (ctx->device >= 0) cudaSetDevice(ctx->device);
    gat_index* ix = new gat_index();
    ix->ctx = ctx;
    ix->db = db;
    ix->kind = GAT_INDEX_GRID;
    return finish_build(ctx, ix, build_grid(ix, range, cell_size, virtual_cell_param, leaf_cap), out);
}

int gat_stig_build(gat_ctx* ctx, const gat_db* db, int block_size, gat_index** out) {
    /* block sizes below 2 make STIG::createIndex recurse without end: a two-point range splits
     * into a one-point left leaf and a right child equal to itself (STIG.cpp:120-130) */
    if (!ctx || !db || !out || block_size < 2) return fail(ctx, GAT_ERR_ARG, "gat_stig_build: block size must be at least 2");
    if (db->ctx != ctx) return fail(ctx, GAT_ERR_STATE, "gat_stig_build: trajectory set from another context");
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (ctx->device >= 0) cudaSetDevice(ctx->device);
    gat_index* ix = new gat_index();
    ix->ctx = ctx;
    ix->db = db;
    ix->kind = GAT_INDEX_STIG;
    return finish_build(ctx, ix, build_stig(ix, block_size), out);
}

int gat_fsg_build(gat_ctx* ctx, const gat_db* db, gat_mbb range, float cell_size, gat_index** out) {
    if (!ctx || !db || !out || !(cell_size > 0) || !(range.xmax > range.xmin) || !(range.ymax > range.ymin))
        return fail(ctx, GAT_ERR_ARG, "gat_fsg_build: bad arguments");
    if (db->ctx != ctx) return fail(ctx, GAT_ERR_STATE, "gat_fsg_build: trajectory set from another context");
    std::lock_guard<std::mutex> lk(ctx->mu);
    if (ctx->device >= 0) cudaSetDevice(ctx->device);
    gat_index* ix = new gat_index();
    ix->ctx = ctx;
    ix->db = db;
    ix->kind = GAT_INDEX_FSG;
    return finish_build(ctx, ix, build_fsg(ix, range, cell_size), out);
}

}  // extern "C"
