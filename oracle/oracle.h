/* CPU restatement of the reference's hot-path algorithms. TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library, and
 * only as the checker or the timed CPU baseline; the product (gat_b200/) never links it.
 *
 * Every function restates one reference routine with plain loops and cites the reference
 * file:line it follows. Pinning: tests/test_oracle_vs_reference.py checks this restatement
 * against the reference's own code compiled from its sources (oracle/_ref/gatref) on seeded
 * inputs, and tests/test_golden.py against the committed golden fixtures that gatref wrote.
 *
 * Conventions: trajectory ids are 1..n (the reference's tradb starts at 1, main.cpp:116-121);
 * lengths[i] and the concatenated lon/lat arrays describe trajectory i+1. Every output array is
 * caller-allocated; calls that produce variable-size output take a NULL output pointer first to
 * report sizes. */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_grid orc_grid; /* GT-quadtree index (Grid.cpp) + FVTable */
typedef struct orc_stig orc_stig; /* STIG KD-tree index (STIG.cpp) */
typedef struct orc_fsg orc_fsg;   /* FSG flat grid (FSG.cpp) */

/* ---- GT-quadtree (Grid.cpp:97-316) ---- */
orc_grid* orc_grid_build(int n, const int32_t* lengths, const float* lon, const float* lat,
                         const float box[4], float cell, int vparam, int leaf_cap);
void orc_grid_free(orc_grid* g);
/* meta: axis, cellnum, total points, total levels, leaves, nodes */
void orc_grid_meta(const orc_grid* g, int32_t meta[6]);
/* points in cell order: x, y, tid, point index within its trajectory */
void orc_grid_points(const orc_grid* g, float* x, float* y, int32_t* tid, int32_t* pidx);
void orc_grid_cells(const orc_grid* g, int32_t* start, int32_t* end, float* mbb4);
/* nodes in depth-first (UL, UR, DL, DR) order: id, level, npts, leaf, mbb */
void orc_grid_nodes(const orc_grid* g, int32_t* id, int32_t* level, int32_t* npts, int32_t* leaf,
                    float* mbb4);
/* frequency vectors: sizes (off has n+2 entries, trajectory 0 is empty) or contents */
int64_t orc_grid_fv(const orc_grid* g, int64_t* off, int32_t* cell, int32_t* count);
/* range query, Grid::rangeQueryBatch (Grid.cpp:341-405). mode 0: sorted trajectory-id sets;
 * mode 1: sorted (tid, pidx) point hits. counts[q] always written; out_a (ids / tids) and
 * out_b (pidx) written when non-NULL, sized by the counts. */
void orc_grid_range(const orc_grid* g, const float* q4, int nq, int mode, int64_t* counts,
                    int32_t* out_a, int32_t* out_b);
/* candidate leaves of a query in traversal order (Grid.cpp:428-446): node ids and levels */
int orc_grid_candidates(const orc_grid* g, const float q4[4], int32_t* node_id, int32_t* level);

/* ---- STIG (STIG.cpp:35-252) ---- */
orc_stig* orc_stig_build(int n, const int32_t* lengths, const float* lon, const float* lat,
                         int block_size);
void orc_stig_free(orc_stig* s);
int64_t orc_stig_npoints(const orc_stig* s);
void orc_stig_points(const orc_stig* s, float* x, float* y, int32_t* tid, int32_t* pidx);
/* leaves in depth-first order: [left, right] inclusive ranges and MBBs; returns count */
int orc_stig_leaves(const orc_stig* s, int32_t* lr, float* mbb4);
/* candidate blocks of a query (STIG::searchTree), [start, end] pairs; returns count */
int orc_stig_candidates(const orc_stig* s, const float q4[4], int32_t* blocks);
void orc_stig_range(const orc_stig* s, const float* q4, int nq, int mode, int64_t* counts,
                    int32_t* out_a, int32_t* out_b);

/* ---- FSG (FSG.cpp:7-393) ---- */
orc_fsg* orc_fsg_build(int n, const int32_t* lengths, const float* lon, const float* lat,
                       const float box[4], float cell);
void orc_fsg_free(orc_fsg* f);
void orc_fsg_meta(const orc_fsg* f, int32_t meta[4]);
void orc_fsg_points(const orc_fsg* f, float* x, float* y, int32_t* tid, int32_t* pidx);
void orc_fsg_cells(const orc_fsg* f, int32_t* start, int32_t* end);
/* candidate cells of a query (FSG.cpp:183-262): border cells then interior cells; returns count */
int orc_fsg_candidates(const orc_fsg* f, const float q4[4], int32_t* cells);
void orc_fsg_range(const orc_fsg* f, const float* q4, int nq, int mode, int64_t* counts,
                   int32_t* out_a, int32_t* out_b);

/* ---- EDR (Grid.cpp:1222-1318) ---- */
/* a = query, b = candidate, points interleaved (x, y); eps as the reference's double EPSILON */
int32_t orc_edr(const float* a, int la, const float* b, int lb, double eps);
void orc_edr_batch(int npairs, const int32_t* la, const int64_t* oa, const float* a,
                   const int32_t* lb, const int64_t* ob, const float* b, double eps, int threads,
                   int32_t* out);

/* ---- FV lower bound (FVTable.cpp:53-207) ---- */
/* neighbour keys of a virtual cell exactly as FVTable::findNeighbor + getIdxFromXY compute them
 * on x86-64 g++ (negative coordinates included) */
void orc_fv_neighbors(int vcell_count, int cell, int32_t out[8]);
/* query frequency vector from query points (Grid.cpp:860-877): returns nnz, fills cell/count
 * when non-NULL (sorted by cell) */
int orc_grid_query_fv(const orc_grid* g, const float* lon, const float* lat, int len,
                      int32_t* cell, int32_t* count);
/* lb[t] for t = 0..n (lb[0] unused) */
void orc_grid_fv_lb(const orc_grid* g, int qnnz, const int32_t* qcell, const int32_t* qcount,
                    int32_t* lb);

/* ---- top-k (Grid.cpp:852-1220) ---- */
/* canonical top-k by (EDR asc, id asc) over every trajectory, query given by its points.
 * pruned != 0 walks candidates in lower-bound order and stops once the next bound exceeds the
 * current k-th distance (same result when the bound holds); evaluated[0] receives the number
 * of EDR evaluations. */
void orc_grid_topk(const orc_grid* g, const float* qlon, const float* qlat, int qlen, int k,
                   double eps, int pruned, int threads, int32_t* ids, int32_t* dist,
                   int64_t* evaluated);

#ifdef __cplusplus
}
#endif
