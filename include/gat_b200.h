/* gat_b200: trajectory range and EDR top-k queries on one NVIDIA B200 (sm_100a).
 *
 * C ABI of the library gat_b200/libgat_b200.so. Every entry point returns a gat_status; on
 * failure gat_last_error(ctx) holds a message. Nothing aborts the process.
 *
 * Handles are opaque and owned by the library (destroy indexes, then trajectory sets, then the
 * context they were made on): a gat_db holds a trajectory set resident in
 * device memory, a gat_index holds one of the reference's three range indexes (GT-quadtree
 * "Grid" with its FVTable, STIG, FSG) in the reference's exact layout, resident in device
 * memory (Grid and FSG are built on the device by default, STIG on the host). Host output buffers are owned by the caller; calls whose output
 * size is data-dependent take a capacity and report the size needed (GAT_ERR_TRUNCATED when
 * it did not fit, with nothing written beyond the capacity).
 *
 * Trajectory ids are 1..n, as in the reference (tradb[1..], main.cpp:116-121): lengths[i] and
 * the concatenated lon/lat arrays describe trajectory i+1. Coordinates are float32.
 *
 * Reference interfaces replaced (file:line in the reference):
 *   cudaRangeQueryTestHandler        cudaKernel.h:21  -> gat_range_query (GAT_INDEX_GRID, FSG)
 *   cudaRangeQuerySTIGHandler        cudaKernel.h:28  -> gat_range_query (GAT_INDEX_STIG)
 *   EDRDistance_Batch_Handler        cudaKernel.h:24  -> gat_edr_pairs
 *   Similarity_Pruning_Handler       cudaKernel.h:26  -> gat_fv_lower_bounds
 *   Grid::SimilarityQueryBatchOnGPU  Grid.h:65        -> gat_topk
 *   Grid::Grid + addDatasetToGrid    Grid.h:39,42     -> gat_grid_build
 *   STIG::initial                    STIG.h:57        -> gat_stig_build
 *   FSG::FSG + addDatasetToGrid      FSG.h:35,38      -> gat_fsg_build
 *   PreProcess::readTraFromFormatedFile / writeTraDataToFile
 *                                    PreProcess.cpp:203-315 -> gat_traj_file_read / _write
 * Additions without a counterpart: index snapshots, the serving loop, the top-k merge of sets
 * sharded across GPUs, tuning knobs, and an allocation-free EDR entry point.
 */
#ifndef GAT_B200_H
#define GAT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GAT_OK = 0,
    GAT_ERR_ARG = 1,       /* invalid argument (size, pointer, out-of-grid point, ...) */
    GAT_ERR_OOM = 2,       /* device or host allocation failed */
    GAT_ERR_CUDA = 3,      /* CUDA runtime error */
    GAT_ERR_TRUNCATED = 4, /* output larger than the capacity given; *needed holds the size */
    GAT_ERR_TIMEOUT = 5,   /* a bounded device-side wait gave up */
    GAT_ERR_STATE = 6      /* handle used with the wrong context or kind */
} gat_status;

typedef struct gat_ctx gat_ctx;
typedef struct gat_db gat_db;
typedef struct gat_index gat_index;

/* MBB.h:5 field order */
typedef struct {
    float xmin, ymin, xmax, ymax;
} gat_mbb;

enum { GAT_INDEX_GRID = 0, GAT_INDEX_STIG = 1, GAT_INDEX_FSG = 2, GAT_INDEX_MORTON = 3 };
/* GAT_RESULT_IDS: per query, the sorted set of trajectory ids with at least one point in the
 * box (the reference's vector<bool> result row, QueryResult.h:4).
 * GAT_RESULT_POINTS: per query, the sorted (trajectory id, point index) pairs in the box. */
enum { GAT_RESULT_IDS = 0, GAT_RESULT_POINTS = 1 };
/* GAT_EXEC_PLAIN: one query per launch sequence. GAT_EXEC_BATCHED: all queries in one. */
enum { GAT_EXEC_PLAIN = 0, GAT_EXEC_BATCHED = 1 };

/* ---------------------------------------------------------------- context */
/* Creates a context bound to a CUDA device with its own stream. device = -1 creates a
 * host-only context: trajectory sets and indexes are built on the host (layout inspection via
 * gat_index_points / gat_index_info) and every call that needs a GPU returns GAT_ERR_STATE. */
int gat_ctx_create(int device, gat_ctx** out);
void gat_ctx_destroy(gat_ctx* ctx);
const char* gat_last_error(const gat_ctx* ctx);
/* A worker context (no counterpart in the reference): same device as parent, its own stream,
 * scratch arena and lock, and it may run queries on the trajectory sets and indexes created
 * through the parent, so several host threads can drive one device concurrently. Destroy
 * workers before their parent. */
int gat_ctx_create_worker(gat_ctx* parent, gat_ctx** out);
/* Frees the context's scratch arena and the index-build temporaries it keeps for reuse (both
 * grow again on demand). */
int gat_ctx_trim(gat_ctx* ctx);
/* The cudaStream_t all work of the context is issued on (for event timing by callers). */
void* gat_ctx_stream(gat_ctx* ctx);
int gat_ctx_sync(gat_ctx* ctx);
/* Kernel launches issued by the context since creation (all of them are this library's). */
int64_t gat_ctx_launches(const gat_ctx* ctx);
/* Device bytes currently held by the context's scratch arena and index-build temporaries. */
int64_t gat_ctx_scratch_bytes(const gat_ctx* ctx);
/* Per-kernel timing: when on, launches of the kernel classes below are bracketed by CUDA
 * events on the context stream; gat_ctx_kernel_stats returns their summed device time (ms),
 * launch count and algorithmic work (DP cells for EDR, bytes for the others) since the last
 * reset. Turning timing on resets the counters. */
enum { GAT_KERNEL_EDR = 0, GAT_KERNEL_BOUNDS = 1, GAT_KERNEL_RANGE_SCAN = 2, GAT_KERNEL_INDEX_BUILD = 3,
       GAT_KERNEL_CLASSES = 4 };
int gat_ctx_set_timing(gat_ctx* ctx, int on);
int gat_ctx_kernel_stats(gat_ctx* ctx, int kernel_class, double* ms, int64_t* launches, double* work);
/* Tuning knobs (no counterpart in the reference, which has fixed launch shapes).
 * GAT_TUNE_EDR_ROWS: rows each lane of the EDR wavefront owns (tile height = 32 x rows).
 *   0 (default) = autotune: the first launch of each shape class (pair count, longest shorter
 *   side and longest longer side, each rounded up to a power of two) times 2, 4 and 8 rows
 *   per lane on the caller's own data and keeps the fastest for that class; results are the
 *   same for every choice. 2, 4 or 8 fixes the value. Setting the knob clears the tuned table.
 * gat_ctx_get_tuning(GAT_TUNE_EDR_ROWS) returns the knob; GAT_TUNE_EDR_TUNED returns the
 * number of tuned shape classes.
 * GAT_TUNE_EDR_FORM: 0 (default) = autotune, 1 = row tiles (lanes own rows of the shorter
 *   side, steps walk the longer side), 2 = column tiles (lanes own columns, steps walk the
 *   shorter side: a shorter critical path for pairs of uneven length). Same results.
 * GAT_TUNE_TOPK_CHUNK / GAT_TUNE_TOPK_GROWTH: candidates a query evaluates in the first round
 *   of the top-k walk, and the factor each later round grows by (0 = defaults: a first round of
 *   1280 for up to 4 queries per batch and 128 for larger batches, never below 8k or 4k;
 *   growth 2). Results never depend on them; they trade rounds against surplus evaluations.
 * GAT_TUNE_INDEX_BUILD: where gat_grid_build and gat_fsg_build place the points. 0 (default) =
 *   on the device for a context with one, 1 = on the host, 2 = on the device (GAT_ERR_STATE on a
 *   host-only context). Both give the same index, array for array; STIG is always built on the
 *   host (its median splits follow std::sort's order among equal coordinates).
 * GAT_TUNE_DEP_LAUNCH: 1 (default) launches the kernels of the top-k and EDR paths as
 *   programmatic dependent launches (each kernel is set up while the one before it drains; the
 *   order of their work is unchanged), 0 launches them plainly. Same results.
 * GAT_TUNE_TEST_STALL_CARRY: for tests of the bounded wait between pipelined EDR tiles, never
 *   for production. v > 0 makes the first tile of pair v - 1 of every later pipelined launch
 *   skip its carry stores and shortens each wait to about 4096 polls, so the next tile of that
 *   pair gives up: the pair gets -1, the call returns GAT_ERR_TIMEOUT, every other pair keeps
 *   its exact distance and the context stays usable. 0 (default) turns it off.
 * GAT_TUNE_SERVE_RESERVE: read by gat_server_create from the context it is given: the percent of
 *   the SMs (1..90) that the persistent EDR grids of the server's top-k lanes leave free for its
 *   range lane; 0 (default) = 12. Same results.
 * GAT_TUNE_RANGE_SHAPE: block shape of the batched range scan for trajectory-id sets. 0 (default)
 *   = autotune: the first batch of each (index kind, batch size rounded up to a power of two)
 *   class times the shapes on its own queries and keeps the fastest; 1 = 256 threads per CTA
 *   with an 8192-slot id set, 2 = 128 threads with a 4096-slot set, 3 = the batch split by size
 *   (queries with more than 16 candidate items on shape 1, the others one per warp with a
 *   1024-slot set and no block barrier, in the same launch). Same results.
 *   Setting the knob clears the tuned table.
 * GAT_TUNE_EDR_RESERVE: percent of the SMs (0..90) that this context's persistent EDR grid
 *   leaves to other streams (0, the default, takes them all). Same results. */
enum { GAT_TUNE_EDR_ROWS = 1, GAT_TUNE_EDR_TUNED = 2, GAT_TUNE_TOPK_CHUNK = 3, GAT_TUNE_TOPK_GROWTH = 4,
       GAT_TUNE_EDR_FORM = 5, GAT_TUNE_INDEX_BUILD = 6, GAT_TUNE_DEP_LAUNCH = 7, GAT_TUNE_TEST_STALL_CARRY = 8,
       GAT_TUNE_SERVE_RESERVE = 9, GAT_TUNE_RANGE_SHAPE = 10, GAT_TUNE_EDR_RESERVE = 11 };
int gat_ctx_set_tuning(gat_ctx* ctx, int knob, int value);
int gat_ctx_get_tuning(gat_ctx* ctx, int knob, int* value);

/* ---------------------------------------------------------------- trajectory set */
int gat_db_create(gat_ctx* ctx, int n, const int32_t* lengths, const float* lon, const float* lat,
                  gat_db** out);
void gat_db_destroy(gat_db* db);
/* info[0] = n, info[1] = total points, info[2] = longest trajectory */
int gat_db_info(const gat_db* db, int64_t info[4]);

/* ---------------------------------------------------------------- indexes */
/* Grid::Grid(range, cell_size, virtual_cell_param) + addDatasetToGrid (Grid.cpp:97-316):
 * Morton cells, cell-contiguous points, quadtree with leaves below leaf_cap points
 * (MAXPOINTINNODE, ConstDefine.h:32), and the FVTable over virtual cells cell >> param. */
int gat_grid_build(gat_ctx* ctx, const gat_db* db, gat_mbb range, float cell_size,
                   int virtual_cell_param, int leaf_cap, gat_index** out);
/* STIG::initial(block_size, 2, ...) (STIG.cpp:35-168); block_size >= 2 (smaller sizes make the
 * reference's recursion endless) */
int gat_stig_build(gat_ctx* ctx, const gat_db* db, int block_size, gat_index** out);
/* FSG::FSG(range, cell_size) + addDatasetToGrid (FSG.cpp:7-143) */
int gat_fsg_build(gat_ctx* ctx, const gat_db* db, gat_mbb range, float cell_size, gat_index** out);
/* MortonGrid (MortonGrid.h:27, MortonGrid::buildQuadTree MortonGrid.cpp:238-259): the same
 * quadtree as `grid`, kept as an implicit tree (a leaf bitmap over node ids (level, id) plus the
 * first point of every Morton cell) and walked by computing each node's box from its corner
 * cells (MortonGrid::generateMBBfromNode, MortonGrid.cpp:261-265) instead of reading stored node
 * boxes. It answers gat_range_query (MortonGrid::rangeQueryBatch, MortonGrid.cpp:268-312) with
 * the Grid's results and reads the Grid's point arrays: destroy it before the Grid. Not part of
 * index snapshots (rebuild it from a loaded Grid). Grids of more than 4^13 cells give GAT_ERR_ARG. */
int gat_morton_grid_build(gat_ctx* ctx, const gat_index* grid, gat_index** out);
/* The MortonGrid's leaves as (level, id) pairs in bitmap order; *count receives their number
 * (GAT_ERR_TRUNCATED when capacity is smaller). */
int gat_morton_grid_leaves(gat_ctx* ctx, const gat_index* morton, int32_t* level, int32_t* id, int64_t capacity,
                           int64_t* count);
void gat_index_destroy(gat_index* index);
/* info[0] = kind, [1] = points, [2] = leaves / blocks / cells, [3] = nodes, [4] = axis or
 * cells along x, [5] = cells along y, [6] = device bytes */
int gat_index_info(const gat_index* index, int64_t info[8]);
/* Copies the index's point order back: x, y, trajectory id, point index within trajectory
 * (any pointer may be NULL). n must equal info[1]. */
int gat_index_points(gat_ctx* ctx, const gat_index* index, int64_t n, float* x, float* y,
                     int32_t* tid, int32_t* pidx);

/* Index snapshots (no counterpart in the reference): gat_index_save writes a built index (any
 * kind) to a file; gat_index_load rebuilds it on a context from that file and the trajectory set
 * it was built over, without sorting the set again. The file records a hash of the set's
 * lengths and coordinates; a different set, a truncated or corrupted file, or a file of another
 * build gives GAT_ERR_ARG. Saving needs a device context. */
int gat_index_save(gat_ctx* ctx, const gat_index* index, const char* path);
int gat_index_load(gat_ctx* ctx, const gat_db* db, const char* path, gat_index** out);

/* ---------------------------------------------------------------- range query */
/* Per query, the result set in the reference's inclusive MBB::pInBox semantics (MBB.cpp:21)
 * over the index's candidate leaves / blocks / cells. offsets has nq + 1 entries (CSR);
 * out_tid receives trajectory ids, out_pidx point indices (GAT_RESULT_POINTS only; may be
 * NULL for GAT_RESULT_IDS). capacity counts entries of out_tid. */
int gat_range_query(gat_ctx* ctx, const gat_index* index, const gat_mbb* queries, int nq,
                    int result_kind, int exec, int64_t* offsets, int32_t* out_tid,
                    int32_t* out_pidx, int64_t capacity, int64_t* needed);
/* Same with every array in device memory (queries, offsets, out_tid, out_pidx); needed is a
 * host pointer. Work is enqueued on the context stream; the call returns after the result
 * size is known. */
int gat_range_query_dev(gat_ctx* ctx, const gat_index* index, const gat_mbb* d_queries, int nq,
                        int result_kind, int exec, int64_t* d_offsets, int32_t* d_tid,
                        int32_t* d_pidx, int64_t capacity, int64_t* needed);

/* ---------------------------------------------------------------- EDR */
/* EDR of (query, candidate) pairs with the reference's recurrence (Grid.cpp:1274-1306) and
 * match test |dx| < eps && |dy| < eps evaluated as float differences compared in double.
 * Points are interleaved (x, y); pair i uses q_xy[2*q_off[i] ...] for q_len[i] points and
 * c_xy[2*c_off[i] ...] for c_len[i] points. Lengths must be 1..GAT_EDR_MAX_LEN. */
#define GAT_EDR_MAX_LEN 16384
int gat_edr_pairs(gat_ctx* ctx, int npairs, const int32_t* q_len, const int64_t* q_off,
                  const float* q_xy, int64_t q_points, const int32_t* c_len,
                  const int64_t* c_off, const float* c_xy, int64_t c_points, double eps,
                  int32_t* out);
/* Same, device arrays. A pair with a side outside 1..GAT_EDR_MAX_LEN gets -1 and the call
 * returns GAT_ERR_ARG. */
int gat_edr_pairs_dev(gat_ctx* ctx, int npairs, const int32_t* d_q_len, const int64_t* d_q_off,
                      const float* d_q_xy, const int32_t* d_c_len, const int64_t* d_c_off,
                      const float* d_c_xy, double eps, int32_t* d_out);
/* gat_edr_pairs_dev without any allocation (no counterpart in the reference). For callers that
 * cannot call cudaMalloc: code running inside a CUDA-graph capture that someone else owns (an
 * allocation there fails or ends up in their graph), runtimes and allocators that forbid device
 * allocations, and programs that must keep a fixed device footprint. There is no context: the
 * caller passes a stream and device arrays. The kernel's working memory is a file-scope device
 * array of fixed size (16.8 MB), which bounds every trajectory side to GAT_EDR_NOALLOC_MAX_LEN
 * points: max_len (the longest side the caller passes, a host value) above it returns
 * GAT_ERR_ARG, and a pair whose side exceeds max_len gets -1. With CUDA's default lazy module
 * loading, the first call on each device loads the module holding the array, which reserves the
 * 16.8 MB there until the process exits: make that first call outside any capture or
 * no-allocation region; later calls allocate nothing. A call outside a capture looks the
 * array's address up again, so a cudaDeviceReset between calls is harmless; a call inside a
 * capture uses the address of the last call outside one (GAT_ERR_STATE before any).
 * Asynchronous on `stream`; calls that overlap on the GPU share the array and race, so the
 * caller serialises them. */
#define GAT_EDR_NOALLOC_MAX_LEN 4096
int gat_edr_pairs_dev_noalloc(void* stream, int npairs, int max_len, const int32_t* d_q_len,
                              const int64_t* d_q_off, const float* d_q_xy, const int32_t* d_c_len,
                              const int64_t* d_c_off, const float* d_c_xy, double eps,
                              int32_t* d_out);

/* ---------------------------------------------------------------- top-k similarity */
/* FVTable::formPriorityQueue lower bounds (FVTable.cpp:77-207) of every trajectory of the
 * grid's set against each query: out[q * (n + 1) + t], t = 0..n (t = 0 unused). */
int gat_fv_lower_bounds(gat_ctx* ctx, const gat_index* grid, int nq, const int32_t* q_len,
                        const float* q_lon, const float* q_lat, int32_t* out);
/* The k trajectories of the grid's set with the smallest EDR to each query, sorted by
 * (distance, trajectory id). Candidates are evaluated in frequency-vector lower-bound order
 * and pruned once the bound exceeds the current k-th distance (Grid.cpp:852-1019), so the
 * result equals the exhaustive one. stats (may be NULL): [0] EDR pairs evaluated, [1] DP
 * cells evaluated, [2] launches issued. */
int gat_topk(gat_ctx* ctx, const gat_index* grid, int nq, const int32_t* q_len,
             const float* q_lon, const float* q_lat, int k, double eps, int exec,
             int32_t* out_ids, int32_t* out_dist, int64_t* stats);
/* Same with query points and outputs in device memory: d_q_off[nq+1] point offsets. */
int gat_topk_dev(gat_ctx* ctx, const gat_index* grid, int nq, const int32_t* d_q_len,
                 const int64_t* d_q_off, const float* d_q_xy, int max_q_len, int k, double eps,
                 int exec, int32_t* d_ids, int32_t* d_dist, int64_t* stats);

/* ---------------------------------------------------------------- sharded sets (no counterpart in the reference,
 * whose two-GPU mode splits the queries, Grid.cpp:1758-2332) */
/* A trajectory set split across GPUs by contiguous id ranges answers top-k as the merge of each
 * shard's gat_topk (ids made global by adding the shard's first id - 1): the k smallest
 * (distance, id) of the union, equal to the unsharded result. Inputs are [nparts][nq][k], each
 * list sorted by (distance, id); id -1 marks padding (a shard with fewer than k trajectories)
 * and is emitted as (-1, -1). nparts x k must not exceed 8192. gat_topk_merge runs on host
 * buffers; gat_topk_merge_dev on device buffers (for example after an all-gather), on the
 * context's stream. */
int gat_topk_merge(int nq, int k, int nparts, const int32_t* ids, const int32_t* dist, int32_t* out_ids,
                   int32_t* out_dist);
int gat_topk_merge_dev(gat_ctx* ctx, int nq, int k, int nparts, const int32_t* d_ids, const int32_t* d_dist,
                       int32_t* d_out_ids, int32_t* d_out_dist);

/* ---------------------------------------------------------------- serving (no counterpart in the reference) */
/* A request loop over device-resident indexes with continuous batching: requests are submitted
 * one at a time from any thread; a scheduler thread forms a batch whenever one of `lanes`
 * worker contexts is free, from the queue whose head request is oldest (range requests grouped
 * by index and result kind, top-k requests by eps), and admits it only while the estimated
 * device bytes of all admitted batches stay within budget_bytes. Batches of different lanes
 * overlap on the device. With two or more lanes, lane 0 runs range batches only, on a stream of
 * the greatest priority, and the other lanes' persistent EDR grids leave an eighth of the SMs
 * free, so range requests never wait behind top-k work; a top-k batch stops growing at 8192
 * query points. Results equal those of the same request run alone. */
typedef struct gat_server gat_server;
typedef struct {
    int lanes;            /* worker contexts (streams) running batches concurrently; default 4 */
    int64_t budget_bytes; /* device bytes for admitted batches' results and scratch; default 40 GiB */
    int max_range_batch;  /* range requests per batch; default 4096 */
    int max_topk_batch;   /* top-k requests per batch; default 32 */
} gat_server_config;
/* cfg may be NULL (defaults). Any index may be NULL except that range requests need the index
 * they name and top-k requests need the grid. */
int gat_server_create(gat_ctx* ctx, const gat_index* grid, const gat_index* stig, const gat_index* fsg,
                      const gat_server_config* cfg, gat_server** out);
/* Finishes every submitted request, then stops the threads and frees everything. */
void gat_server_destroy(gat_server* server);
int gat_server_submit_range(gat_server* server, int index_kind, gat_mbb box, int result_kind, int64_t* id);
int gat_server_submit_topk(gat_server* server, int q_len, const float* lon, const float* lat, int k,
                           double eps, int64_t* id);
/* Waits for a request (timeout_ms < 0: no limit; GAT_ERR_TIMEOUT when it runs out); the
 * request's own status goes to *req_status (GAT_ERR_OOM when it can never fit the budget). */
int gat_server_wait(gat_server* server, int64_t id, int timeout_ms, int* req_status);
/* Result of a finished range request: *count entries (GAT_ERR_TRUNCATED when capacity is
 * smaller); pidx only for GAT_RESULT_POINTS requests. */
int gat_server_range_result(gat_server* server, int64_t id, int32_t* tids, int32_t* pidx, int64_t capacity,
                            int64_t* count);
/* Result of a finished top-k request: k ids and distances sorted by (distance, id). */
int gat_server_topk_result(gat_server* server, int64_t id, int32_t* ids, int32_t* dist, int capacity);
/* Arrival, admission and completion times of a request, ns since the server started. */
int gat_server_request_times(gat_server* server, int64_t id, int64_t t[3]);
/* Forgets a finished request and its result. */
int gat_server_release(gat_server* server, int64_t id);
/* [0] submitted, [1] completed, [2] batches, [3] range batches, [4] top-k batches,
 * [5] peak admitted bytes, [6] largest batch, [7] failed requests */
int gat_server_stats(gat_server* server, int64_t stats[8]);

/* ---------------------------------------------------------------- trajectory files */
/* The reference's formatted trajectory file (PreProcess.cpp:203-315): the count, the box
 * (xmin,ymin,xmax,ymax), a line of lengths, then per trajectory one "lat,lon,tid,time;" record
 * per point. No context needed. gat_traj_file_info reads the three header lines: n, the total
 * number of points and the box (box may be NULL). gat_traj_file_read fills caller arrays sized
 * by those counts (GAT_ERR_TRUNCATED when n or points do not match the file; times may be NULL).
 * gat_traj_file_write writes the reference writer's bytes (times NULL writes 0; a point's tid
 * field is its trajectory's number). Malformed files and unopenable paths give GAT_ERR_ARG. */
int gat_traj_file_info(const char* path, int* n, int64_t* points, float box[4]);
int gat_traj_file_read(const char* path, int n, int64_t points, int32_t* lengths, float* lon, float* lat,
                       int32_t* times);
int gat_traj_file_write(const char* path, int n, const int32_t* lengths, const float* lon, const float* lat,
                        const int32_t* times, const float box[4]);

/* ---------------------------------------------------------------- synthetic inputs */
enum { GAT_LEN_UNIFORM = 0, GAT_LEN_LOGNORMAL = 1, GAT_LEN_LOGUNIFORM = 2 };
enum { GAT_SIDE_FIXED = 0, GAT_SIDE_LOGUNIFORM = 1 };
/* n lengths: uniform integers in [lo, hi]; round(exp(N(p0, p1))) clipped to [lo, hi]; or
 * round(log-uniform(lo, hi)). */
int gat_gen_lengths(int n, int kind, double p0, double p1, int lo, int hi, uint64_t seed,
                    int32_t* out);
/* Clamped random walks in box: start uniform, N(0, step) increments per axis. */
int gat_gen_walks(int n, const int32_t* lengths, const float box[4], double step, uint64_t seed,
                  float* lon, float* lat);
/* Query rectangles with centres uniform in box; side s0 (GAT_SIDE_FIXED) or log-uniform in
 * [s0, s1] per axis. out4 = (xmin, ymin, xmax, ymax) per rectangle. */
int gat_gen_boxes(int n, int kind, double s0, double s1, const float box[4], uint64_t seed,
                  float* out4);
/* k distinct ids from 1..n */
int gat_gen_sample_ids(int k, int n, uint64_t seed, int32_t* out);
/* EDR pairs: A a random walk, B A's path resampled to B's length plus N(0, jitter) noise. */
int gat_gen_pairs(int n, const int32_t* len_a, const int32_t* len_b, const float box[4],
                  double step, double jitter, uint64_t seed, float* a_xy, float* b_xy);

#ifdef __cplusplus
}
#endif
#endif /* GAT_B200_H */
