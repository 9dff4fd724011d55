/* EDR top-k similarity with frequency-vector lower-bound pruning.
 *
 * Per batch of queries (device-resident; every step is a kernel over all queries of the batch):
 *   1. query frequency vectors: cell of every query point (Grid::WhichCellPointIn,
 *      Grid.cpp:202-208) shifted to its virtual cell, counted per cell (Grid.cpp:860-877)
 *   2. lower bounds: FVTable::formPriorityQueue's per-trajectory bound (FVTable.cpp:81-202):
 *      signed difference of the two frequency vectors, greedy cancellation of positive cells
 *      against negative 8-neighbour cells and back, bound = max(sum+, sum-)
 *   3. round 1: the K1 candidates with the smallest (bound, id)
 *      round 2: the remaining candidates whose bound is below the k-th distance W1 of round 1
 *      The reference evaluates candidates in bound order until the bound reaches the current
 *      k-th distance (Grid.cpp:917); after round 2 every candidate with bound below the k-th
 *      distance has been evaluated, so the k smallest distances are final.
 *   4. ties: candidates whose bound equals the k-th distance W may tie at W; they are taken in
 *      ascending id order until the k-th (distance, id) slot is decided, giving the canonical
 *      order (distance ascending, lower trajectory id first) exactly.
 *   5. selection of the k smallest (distance, id) pairs.
 * EDR pairs of every round run through the warp-wavefront kernel (edr.cu).
 */
#include <algorithm>
#include <climits>

#include "internal.h"

namespace gat {
namespace {

constexpr int kT = 256;
constexpr int kMaxRounds = 24;
constexpr int kMaxFv = 128; /* merged frequency-vector entries per (query, trajectory) */

/* per-query state words: the walk position (bound, id) of the last candidate taken, the
 * chunk end chosen for the current round, the k-th distance, the done flag */
enum { QS_POS_LB = 0, QS_POS_ID, QS_END_LB, QS_END_ID, QS_W, QS_DONE, QS_EVAL, QS_WORDS };

/* (bound, id) strictly after (plb, pid) in the walk order */
__device__ __forceinline__ bool after(int v, int t, int plb, int pid) { return v > plb || (v == plb && t > pid); }
/* (bound, id) at or before (elb, eid) */
__device__ __forceinline__ bool upto(int v, int t, int elb, int eid) { return v < elb || (v == elb && t <= eid); }

/* ---------------------------------------------------------------- reference cell ids */
/* getIdxFromXY (Grid.cpp:25-54) as the x86-64 build evaluates it, negative inputs included:
 * the bit length of a negative value is INT_MIN + 1 (log2 of a negative number converted to
 * int), and when both inputs are negative the loop does not run. */
__device__ __forceinline__ int ref_len(int v) {
    if (v == 0) return 1;
    if (v < 0) return INT_MIN + 1;
    return 32 - __clz(v);
}
__device__ int ref_morton(int x, int y) {
    int lx = ref_len(x), ly = ref_len(y);
    long long lim = 2LL * max(lx, ly);
    int result = 0, xbit = 1, ybit = 1;
    for (int i = 1; i <= lim; i++) {
        if (i & 1) {
            result += ((x >> (xbit - 1)) & 1) * (1 << (i - 1));
            xbit++;
        } else {
            result += ((y >> (ybit - 1)) & 1) * (1 << (i - 1));
            ybit++;
        }
    }
    return result;
}

/* Grid::WhichCellPointIn (Grid.cpp:202-208) */
__device__ __forceinline__ int cell_of(const GridDev& g, float lon, float lat) {
    int row = (int)__fdiv_rn(__fsub_rn(g.rymax, lat), g.cell);
    int col = (int)__fdiv_rn(__fsub_rn(lon, g.rxmin), g.cell);
    return ref_morton(col, row);
}

/* ---------------------------------------------------------------- 1. query FV */
/* one CTA per query: virtual cell of each point, bitonic sort in shared memory, run lengths.
 * qfv rows have stride `stride` (>= longest query); nnz in qfv_n. */
__global__ void k_query_fv(GridDev g, int nq, const int32_t* q_len, const int64_t* q_off, const float2* Q,
                           int stride, int pow2, int32_t* qfv_cell, int32_t* qfv_cnt, int32_t* qfv_n) {
    extern __shared__ int sk[];
    for (int qi = blockIdx.x; qi < nq; qi += gridDim.x) {
        int L = q_len[qi];
        int64_t o = q_off[qi];
        for (int i = threadIdx.x; i < pow2; i += blockDim.x)
            sk[i] = i < L ? (cell_of(g, Q[o + i].x, Q[o + i].y) >> g.vparam) : INT_MAX;
        __syncthreads();
        for (int k = 2; k <= pow2; k <<= 1)
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < pow2; i += blockDim.x) {
                    int ixj = i ^ j;
                    if (ixj > i) {
                        int a = sk[i], b = sk[ixj];
                        bool up = (i & k) == 0;
                        if ((a > b) == up) {
                            sk[i] = b;
                            sk[ixj] = a;
                        }
                    }
                }
                __syncthreads();
            }
        if (threadIdx.x == 0) {
            int w = 0;
            for (int i = 0; i < L; i++) {
                if (w > 0 && qfv_cell[(size_t)qi * stride + w - 1] == sk[i]) {
                    qfv_cnt[(size_t)qi * stride + w - 1]++;
                } else {
                    qfv_cell[(size_t)qi * stride + w] = sk[i];
                    qfv_cnt[(size_t)qi * stride + w] = 1;
                    w++;
                }
            }
            qfv_n[qi] = w;
        }
        __syncthreads();
    }
}

/* ---------------------------------------------------------------- 2. lower bounds */
/* FVTable::findNeighbor (FVTable.cpp:53-75): x from even bits, y from odd bits of the
 * virtual cell id over log2(vcells) bits, neighbours in order xx = x-1..x+1, yy = y-1..y+1. */
__device__ __forceinline__ void fv_neighbors(int cell, int bits, int nb[8]) {
    int x = 0, y = 0;
    for (int bit = 0; bit < bits; bit++) {
        if ((bit & 1) == 0)
            x += ((cell >> bit) & 1) << (bit >> 1);
        else
            y += ((cell >> bit) & 1) << (bit >> 1);
    }
    int c = 0;
    for (int xx = x - 1; xx <= x + 1; xx++)
        for (int yy = y - 1; yy <= y + 1; yy++)
            if (xx != x || yy != y) nb[c++] = ref_morton(xx, yy);
}

__device__ __forceinline__ int find_key(const int* key, int n, int k) {
    int lo = 0, hi = n - 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        int v = key[mid];
        if (v == k) return mid;
        if (v < k)
            lo = mid + 1;
        else
            hi = mid - 1;
    }
    return -1;
}

/* one thread per (query, trajectory). The merged vector holds every cell of either vector
 * with value db - query (0 = absent). Pass 1 visits the positive cells in ascending order,
 * pass 2 the negative ones (FVTable.cpp:129-187); the reference increments a map iterator
 * after erasing its node, this visits each key present when the pass starts once. */
__global__ void __launch_bounds__(kT) k_lower_bounds(int n, int nq, const int64_t* __restrict__ fv_off,
                                                     const int32_t* __restrict__ fv_cell,
                                                     const int32_t* __restrict__ fv_cnt, const int32_t* qfv_cell,
                                                     const int32_t* qfv_cnt, const int32_t* qfv_n, int stride,
                                                     int vbits, int32_t* lb, int32_t* flag) {
    extern __shared__ int sq[];
    int qi = blockIdx.y;
    int qn = qfv_n[qi];
    int* qc = sq;
    int* qv = sq + stride;
    for (int i = threadIdx.x; i < qn; i += blockDim.x) {
        qc[i] = qfv_cell[(size_t)qi * stride + i];
        qv[i] = qfv_cnt[(size_t)qi * stride + i];
    }
    __syncthreads();
    int t = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (t > n) return;
    int64_t b = fv_off[t], e = fv_off[t + 1];
    int key[kMaxFv], val[kMaxFv];
    int m = 0, i = 0;
    int64_t j = b;
    bool overflow = false;
    /* merge (both sorted by cell): db - query */
    while (i < qn || j < e) {
        int kc, kv;
        if (j < e && (i >= qn || fv_cell[j] < qc[i])) {
            kc = fv_cell[j];
            kv = fv_cnt[j];
            j++;
        } else if (i < qn && (j >= e || qc[i] < fv_cell[j])) {
            kc = qc[i];
            kv = -qv[i];
            i++;
        } else {
            kc = qc[i];
            kv = fv_cnt[j] - qv[i];
            i++;
            j++;
        }
        if (m >= kMaxFv) {
            overflow = true;
            break;
        }
        key[m] = kc;
        val[m] = kv;
        m++;
    }
    if (overflow) {
        atomicCAS(flag, 0, GAT_ERR_ARG);
        lb[(size_t)qi * (n + 1) + t] = 0;
        return;
    }
    int nb[8];
    for (int a = 0; a < m; a++) {
        int pv = val[a];
        if (pv <= 0) continue;
        fv_neighbors(key[a], vbits, nb);
        for (int s = 0; s < 8; s++) {
            int f = find_key(key, m, nb[s]);
            if (f < 0 || val[f] >= 0) continue;
            int nv = -val[f];
            if (pv > nv) {
                val[a] = pv - nv;
                val[f] = 0;
            } else if (pv == nv) {
                val[a] = 0;
                val[f] = 0;
                break;
            } else {
                val[f] = -(nv - pv);
                val[a] = 0;
                break;
            }
        }
    }
    for (int a = 0; a < m; a++) {
        if (val[a] >= 0) continue;
        int nv = -val[a];
        fv_neighbors(key[a], vbits, nb);
        for (int s = 0; s < 8; s++) {
            int f = find_key(key, m, nb[s]);
            if (f < 0 || val[f] <= 0) continue;
            int pv = val[f];
            if (nv > pv) {
                val[a] = -(nv - pv);
                val[f] = 0;
            } else if (pv == nv) {
                val[a] = 0;
                val[f] = 0;
                break;
            } else {
                val[f] = pv - nv;
                val[a] = 0;
                break;
            }
        }
    }
    int sp = 0, sn = 0;
    for (int a = 0; a < m; a++) {
        if (val[a] > 0) sp += val[a];
        if (val[a] < 0) sn -= val[a];
    }
    lb[(size_t)qi * (n + 1) + t] = max(sp, sn);
}

/* ---------------------------------------------------------------- 3. the walk */
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__global__ void k_walk_init(int nq, int32_t* qs) {
    int qi = blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= nq) return;
    int32_t* s = qs + (size_t)qi * QS_WORDS;
    s[QS_POS_LB] = -1;
    s[QS_POS_ID] = 0;
    s[QS_END_LB] = -1;
    s[QS_END_ID] = 0;
    s[QS_W] = INT_MAX;
    s[QS_DONE] = 0;
    s[QS_EVAL] = 0;
}

/* Chooses the end (elb, eid) of the next chunk: the `chunk` candidates that follow the walk
 * position in (bound, id) order, among bounds <= W (larger bounds can never be needed). A
 * histogram over bound values finds elb; an ordered scan of the ids with bound elb finds eid. */
__global__ void k_walk_select(int n, const int32_t* lb, int chunk, int bins, int32_t* qs) {
    extern __shared__ int hist[];
    __shared__ int sh_elb, sh_need, sh_eid, sh_seen;
    __shared__ int wtot[kT / 32];
    int qi = blockIdx.x;
    int32_t* s = qs + (size_t)qi * QS_WORDS;
    if (s[QS_DONE]) return;
    const int plb = s[QS_POS_LB], pid = s[QS_POS_ID], W = s[QS_W];
    for (int i = threadIdx.x; i < bins; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const int32_t* row = lb + (size_t)qi * (n + 1);
    for (int t = 1 + threadIdx.x; t <= n; t += blockDim.x) {
        int v = row[t];
        if (v <= W && after(v, t, plb, pid)) atomicAdd(&hist[min(v, bins - 1)], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0, v = -1, need = 0;
        for (int i = max(plb, 0); i < bins; i++) {
            if (hist[i] == 0) continue;
            v = i;
            if (run + hist[i] >= chunk) {
                need = chunk - run;
                break;
            }
            run += hist[i];
            need = -1; /* the whole bucket fits */
        }
        sh_elb = v;
        sh_need = need;
        sh_eid = v < 0 ? 0 : n;
        sh_seen = 0;
    }
    __syncthreads();
    const int elb = sh_elb, need = sh_need;
    if (elb >= 0 && need > 0) {
        int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int t0 = 1; t0 <= n; t0 += blockDim.x) {
            int t = t0 + threadIdx.x;
            bool h = t <= n && row[t] == elb && after(elb, t, plb, pid);
            unsigned bal = __ballot_sync(0xffffffffu, h);
            if (lane == 0) wtot[warp] = __popc(bal);
            __syncthreads();
            int wb = 0, tt = 0;
            for (int w = 0; w < kT / 32; w++) {
                if (w < warp) wb += wtot[w];
                tt += wtot[w];
            }
            int seen = sh_seen;
            int rank = seen + wb + __popc(bal & lanemask_lt());
            if (h && rank == need - 1) sh_eid = t;
            __syncthreads();
            if (threadIdx.x == 0) sh_seen = seen + tt;
            __syncthreads();
            if (sh_seen >= need) break;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (elb < 0) {
            s[QS_DONE] = 1; /* nothing left below W */
        } else {
            s[QS_END_LB] = elb;
            s[QS_END_ID] = sh_eid;
        }
    }
}

/* Appends the query's chunk (walk position, chunk end] as EDR pairs and advances the walk. */
__global__ void __launch_bounds__(kT) k_walk_compact(int n, const int32_t* lb, int32_t* qs, const int32_t* q_len,
                                                     const int64_t* q_off, const int32_t* db_len,
                                                     const int64_t* db_off, int64_t cap, unsigned long long* cursor,
                                                     int32_t* pq, int32_t* pt, int64_t* aoff, int32_t* alen,
                                                     int64_t* boff, int32_t* blen, int64_t* seg_base, int64_t* seg_cnt) {
    __shared__ int wtot[kT / 32];
    __shared__ int sh_total;
    __shared__ unsigned long long sh_base;
    int qi = blockIdx.x;
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t* s = qs + (size_t)qi * QS_WORDS;
    const bool active = !s[QS_DONE];
    const int plb = s[QS_POS_LB], pid = s[QS_POS_ID], elb = s[QS_END_LB], eid = s[QS_END_ID];
    const int32_t* row = lb + (size_t)qi * (n + 1);
    auto pick = [&](int t) -> bool {
        int v = row[t];
        return after(v, t, plb, pid) && upto(v, t, elb, eid);
    };
    int c = 0;
    if (active)
        for (int t = 1 + threadIdx.x; t <= n; t += blockDim.x) c += pick(t);
    if (threadIdx.x == 0) sh_total = 0;
    __syncthreads();
    atomicAdd(&sh_total, c);
    __syncthreads();
    const int total = sh_total;
    if (threadIdx.x == 0) sh_base = atomicAdd(cursor, (unsigned long long)total);
    __syncthreads();
    const int64_t base = (int64_t)sh_base;
    const bool fits = base + total <= cap;
    int written = 0;
    if (active && fits && total > 0) {
        for (int t0 = 1; t0 <= n; t0 += blockDim.x) {
            int t = t0 + threadIdx.x;
            bool h = t <= n && pick(t);
            unsigned bal = __ballot_sync(0xffffffffu, h);
            if (lane == 0) wtot[warp] = __popc(bal);
            __syncthreads();
            int wb = 0, tt = 0;
            for (int w = 0; w < kT / 32; w++) {
                if (w < warp) wb += wtot[w];
                tt += wtot[w];
            }
            if (h) {
                int64_t o = base + written + wb + __popc(bal & lanemask_lt());
                pq[o] = qi;
                pt[o] = t;
                aoff[o] = q_off[qi];
                alen[o] = q_len[qi];
                boff[o] = db_off[t];
                blen[o] = db_len[t];
            }
            written += tt;
            __syncthreads();
            if (written >= total) break;
        }
    }
    if (threadIdx.x == 0) {
        seg_base[qi] = base;
        seg_cnt[qi] = active ? (fits ? total : -1) : 0;
        if (active && fits) {
            s[QS_POS_LB] = elb;
            s[QS_POS_ID] = eid;
        }
    }
}

/* ---------------------------------------------------------------- 4. k-th distance, stop rule */
/* W = k-th smallest evaluated distance (INT_MAX while fewer than k). */
__global__ void k_kth(int nrounds, const int64_t* seg_base, const int64_t* seg_cnt, int nq, const int32_t* dist,
                      int k, int bins, int32_t* qs) {
    extern __shared__ int hist[];
    int qi = blockIdx.x;
    int32_t* s = qs + (size_t)qi * QS_WORDS;
    if (s[QS_DONE]) return;
    for (int i = threadIdx.x; i < bins; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    int64_t nev = 0;
    for (int r = 0; r < nrounds; r++) {
        int64_t b = seg_base[(size_t)r * nq + qi], c = seg_cnt[(size_t)r * nq + qi];
        if (c <= 0) continue;
        nev += c;
        for (int64_t i = threadIdx.x; i < c; i += blockDim.x) atomicAdd(&hist[min(dist[b + i], bins - 1)], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0, W = INT_MAX;
        for (int i = 0; i < bins; i++) {
            if (run + hist[i] >= k) {
                W = i;
                break;
            }
            run += hist[i];
        }
        s[QS_W] = W;
        s[QS_EVAL] = (int)nev;
    }
}

/* Stop rule, with (nlb, nid) the first candidate after the walk position: done when there is
 * none with bound <= W, or when nlb == W and k evaluated pairs already sort before (W, nid).
 * While nlb < W the walk must go on: a candidate with a smaller bound may be closer. */
__global__ void k_walk_check(int n, const int32_t* lb, int nrounds, const int64_t* seg_base, const int64_t* seg_cnt,
                             int nq, const int32_t* dist, const int32_t* pt, int k, int32_t* qs, int* pending) {
    __shared__ unsigned long long sh_next;
    __shared__ int cnt;
    int qi = blockIdx.x;
    int32_t* s = qs + (size_t)qi * QS_WORDS;
    if (s[QS_DONE]) return;
    const int W = s[QS_W], plb = s[QS_POS_LB], pid = s[QS_POS_ID];
    if (threadIdx.x == 0) {
        sh_next = ~0ull;
        cnt = 0;
    }
    __syncthreads();
    const int32_t* row = lb + (size_t)qi * (n + 1);
    unsigned long long best = ~0ull;
    for (int t = 1 + threadIdx.x; t <= n; t += blockDim.x) {
        int v = row[t];
        if (v <= W && after(v, t, plb, pid)) {
            unsigned long long key = ((unsigned long long)(unsigned)v << 32) | (unsigned)t;
            if (key < best) best = key;
        }
    }
    if (best != ~0ull) atomicMin(&sh_next, best);
    __syncthreads();
    const unsigned long long nx = sh_next;
    bool done;
    if (nx == ~0ull) {
        done = true;
    } else {
        int nlb = (int)(nx >> 32), nid = (int)(nx & 0xffffffffu);
        if (nlb < W) {
            done = false;
        } else {
            for (int r = 0; r < nrounds; r++) {
                int64_t b = seg_base[(size_t)r * nq + qi], c = seg_cnt[(size_t)r * nq + qi];
                for (int64_t i = threadIdx.x; i < c; i += blockDim.x) {
                    int d = dist[b + i];
                    if (d < W || (d == W && pt[b + i] < nid)) atomicAdd(&cnt, 1);
                }
            }
            __syncthreads();
            done = cnt >= k;
        }
    }
    if (threadIdx.x == 0) {
        s[QS_DONE] = done ? 1 : 0;
        if (!done) atomicAdd(pending, 1);
    }
}

/* ---------------------------------------------------------------- 5. selection */
/* k smallest (distance, id): the LT pairs below W sorted, then the k - LT smallest ids at W
 * (a bitmap over ids in shared memory or a per-CTA global slice). */
__global__ void k_final(int nrounds, const int64_t* seg_base, const int64_t* seg_cnt, int nq, const int32_t* dist,
                        const int32_t* pt, int k, int words, uint32_t* gbitmap, const int32_t* qs, int32_t* out_ids,
                        int32_t* out_dist) {
    extern __shared__ uint32_t bm_s[];
    __shared__ unsigned long long lt_keys[1024];
    __shared__ int lt_n;
    __shared__ int warp_cnt[kT / 32 + 1];
    int qi = blockIdx.x;
    uint32_t* bm = gbitmap ? gbitmap + (size_t)blockIdx.x * words : bm_s;
    const int32_t* s = qs + (size_t)qi * QS_WORDS;
    int W = s[QS_W];
    for (int w = threadIdx.x; w < words; w += blockDim.x) bm[w] = 0;
    if (threadIdx.x == 0) lt_n = 0;
    __syncthreads();
    for (int r = 0; r < nrounds; r++) {
        int64_t b = seg_base[(size_t)r * nq + qi], c = seg_cnt[(size_t)r * nq + qi];
        for (int64_t i = threadIdx.x; i < c; i += blockDim.x) {
            int d = dist[b + i], id = pt[b + i];
            if (d < W) {
                int slot = atomicAdd(&lt_n, 1);
                if (slot < 1024) lt_keys[slot] = ((unsigned long long)(unsigned)d << 32) | (unsigned)id;
            } else if (d == W) {
                atomicOr(&bm[id >> 5], 1u << (id & 31));
            }
        }
    }
    __syncthreads();
    int nlt = min(lt_n, 1024);
    /* sort the (few) pairs below W */
    int p2 = 1;
    while (p2 < nlt) p2 <<= 1;
    for (int i = nlt + threadIdx.x; i < p2; i += blockDim.x) lt_keys[i] = ~0ull;
    __syncthreads();
    for (int kk = 2; kk <= p2; kk <<= 1)
        for (int j = kk >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < p2; i += blockDim.x) {
                int ixj = i ^ j;
                if (ixj > i) {
                    unsigned long long a = lt_keys[i], bb = lt_keys[ixj];
                    bool up = (i & kk) == 0;
                    if ((a > bb) == up) {
                        lt_keys[i] = bb;
                        lt_keys[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    int emit = min(nlt, k);
    for (int i = threadIdx.x; i < emit; i += blockDim.x) {
        out_ids[(size_t)qi * k + i] = (int32_t)(lt_keys[i] & 0xffffffffu);
        out_dist[(size_t)qi * k + i] = (int32_t)(lt_keys[i] >> 32);
    }
    /* the k - emit smallest ids at distance W, in ascending order */
    int need = k - emit;
    int per = (words + kT - 1) / kT;
    int w0 = threadIdx.x * per, w1 = min(words, w0 + per);
    int c = 0;
    for (int w = w0; w < w1; w++) c += __popc(bm[w]);
    /* exclusive scan over threads */
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = c;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_cnt[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int w = 0; w < kT / 32; w++) {
            int t = warp_cnt[w];
            warp_cnt[w] = run;
            run += t;
        }
        warp_cnt[kT / 32] = run;
    }
    __syncthreads();
    const int last_warp_incl = warp_cnt[kT / 32] - warp_cnt[kT / 32 - 1];
    int pre = warp_cnt[warp] + x - c;
    for (int w = w0; w < w1 && pre < need; w++) {
        uint32_t v = bm[w];
        while (v && pre < need) {
            int bit = __ffs(v) - 1;
            v &= v - 1;
            out_ids[(size_t)qi * k + emit + pre] = w * 32 + bit;
            out_dist[(size_t)qi * k + emit + pre] = W;
            pre++;
        }
    }
    /* fewer than k candidates in the whole set: pad with -1 */
    if (threadIdx.x == 0) {
        int ties = warp_cnt[kT / 32 - 1] + last_warp_incl;
        int have = emit + min(ties, need);
        for (int i = have; i < k; i++) {
            out_ids[(size_t)qi * k + i] = -1;
            out_dist[(size_t)qi * k + i] = -1;
        }
    }
}

struct PairBufs {
    int32_t *pq, *pt, *alen, *blen, *dist;
    int64_t *aoff, *boff;
    int64_t cap;
};

size_t pair_bytes(int64_t cap) { return (size_t)cap * (4 * 5 + 8 * 2) + 7 * 256; }
int64_t pair_cap(size_t bytes) { return bytes < 7 * 256 ? 0 : (int64_t)((bytes - 7 * 256) / (4 * 5 + 8 * 2)); }

void carve_pairs(char* base, int64_t c, PairBufs& o) {
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    char* p = base;
    o.pq = (int32_t*)p; p += up((size_t)c * 4);
    o.pt = (int32_t*)p; p += up((size_t)c * 4);
    o.alen = (int32_t*)p; p += up((size_t)c * 4);
    o.blen = (int32_t*)p; p += up((size_t)c * 4);
    o.dist = (int32_t*)p; p += up((size_t)c * 4);
    o.aoff = (int64_t*)p; p += up((size_t)c * 8);
    o.boff = (int64_t*)p;
    o.cap = c;
}

/* grows the pair arrays (scratch slot S_TOPK_PAIRS), preserving the first `keep` entries */
int ensure_pairs(gat_ctx* ctx, PairBufs& P, int64_t need, int64_t keep) {
    if (need <= P.cap) return GAT_OK;
    int64_t cap = std::max<int64_t>(need, P.cap * 2);
    void* nb = nullptr;
    cudaError_t e = cudaMalloc(&nb, pair_bytes(cap));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "top-k pair buffer");
    PairBufs N;
    carve_pairs((char*)nb, cap, N);
    cudaStream_t s = ctx->stream;
    if (P.cap > 0 && keep > 0) {
        cudaMemcpyAsync(N.pq, P.pq, keep * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(N.pt, P.pt, keep * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(N.alen, P.alen, keep * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(N.blen, P.blen, keep * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(N.dist, P.dist, keep * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(N.aoff, P.aoff, keep * 8, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(N.boff, P.boff, keep * 8, cudaMemcpyDeviceToDevice, s);
    }
    if (ctx->slot_ptr[S_TOPK_PAIRS]) {
        cudaStreamSynchronize(s);
        cudaFree(ctx->slot_ptr[S_TOPK_PAIRS]);
    }
    ctx->slot_ptr[S_TOPK_PAIRS] = nb;
    ctx->slot_bytes[S_TOPK_PAIRS] = pair_bytes(cap);
    P = N;
    return GAT_OK;
}

int read_word(gat_ctx* ctx, const void* d, int64_t* v) {
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_pinned, d, 8, cudaMemcpyDeviceToHost, ctx->stream), "top-k");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "top-k");
    *v = ctx->h_pinned[0];
    return GAT_OK;
}

/* the whole pipeline for queries [0, nq) of the given device arrays */
int topk_batch(gat_ctx* ctx, const gat_index* g, int nq, const int32_t* d_q_len, const int64_t* d_q_off,
               const float2* d_q_xy, int max_q_len, int k, float u, int32_t* d_ids, int32_t* d_dist, int64_t* stats) {
    cudaStream_t s = ctx->stream;
    const gat_db* db = g->db;
    int n = db->n;
    int st = GAT_OK;
    int stride = std::max(1, max_q_len);
    int pow2 = 1;
    while (pow2 < max_q_len) pow2 <<= 1;
    /* query FVs */
    size_t fvb = (size_t)nq * stride * 4;
    char* qfv = (char*)scratch(ctx, S_TOPK_QFV, fvb * 2 + (size_t)nq * 4 + 1024, &st);
    if (!qfv) return st;
    int32_t* qfv_cell = (int32_t*)qfv;
    int32_t* qfv_cnt = (int32_t*)(qfv + fvb);
    int32_t* qfv_n = (int32_t*)(qfv + 2 * fvb);
    size_t smem_fv = (size_t)pow2 * 4;
    if (smem_fv > 48 * 1024) cudaFuncSetAttribute(k_query_fv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_fv);
    k_query_fv<<<std::min(nq, ctx->sm_count * 4), 512, smem_fv, s>>>(g->grid, nq, d_q_len, d_q_off, d_q_xy, stride, pow2,
                                                                      qfv_cell, qfv_cnt, qfv_n);
    count_launch(ctx);
    /* lower bounds */
    int32_t* lb = (int32_t*)scratch(ctx, S_TOPK_LB, (size_t)nq * (n + 1) * 4, &st);
    if (!lb) return st;
    int vbits = (int)std::log2((double)(g->grid.cellnum >> 2));
    size_t smem_lb = (size_t)stride * 8;
    if (smem_lb > 48 * 1024) cudaFuncSetAttribute(k_lower_bounds, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_lb);
    dim3 lgrid((n + kT - 1) / kT, nq);
    timed_begin(ctx, GAT_KERNEL_BOUNDS);
    k_lower_bounds<<<lgrid, kT, smem_lb, s>>>(n, nq, g->d_fv_off, g->d_fv_cell, g->d_fv_cnt, qfv_cell, qfv_cnt, qfv_n, stride,
                                             vbits, lb, ctx->d_flag);
    /* algorithmic bytes: every trajectory's FV (8 B per entry + 8 B offset) and its bound (4 B)
     * per query */
    timed_end(ctx, GAT_KERNEL_BOUNDS, (double)nq * ((double)g->fv_entries * 8.0 + (double)n * 12.0));
    count_launch(ctx);
    if (stats && stats[3] == -1) { /* bounds only */
        return check_device_flag(ctx, "frequency-vector bounds");
    }
    /* per-query state + segments */
    int32_t* qs = (int32_t*)scratch(ctx, S_TOPK_QSTATE, (size_t)nq * QS_WORDS * 4 + 256, &st);
    int64_t* seg = (int64_t*)scratch(ctx, S_TOPK_SEG, (size_t)kMaxRounds * nq * 2 * 8 + 256, &st);
    unsigned long long* cursor = (unsigned long long*)scratch(ctx, S_TOPK_IO, 256, &st);
    if (!qs || !seg || !cursor) return st;
    int64_t* seg_base = seg;
    int64_t* seg_cnt = seg + (size_t)kMaxRounds * nq;
    unsigned long long* cells = cursor + 1;
    int* pending = (int*)(cursor + 2);
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(cursor, 0, 64, s), "top-k");
    int bins_lb = std::max(max_q_len, db->maxlen) + 2;
    int bins_d = max_q_len + db->maxlen + 2;
    size_t smem_lbh = (size_t)bins_lb * 4, smem_dh = (size_t)bins_d * 4;
    if (smem_dh > 48 * 1024) cudaFuncSetAttribute(k_kth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_dh);
    k_walk_init<<<(nq + 127) / 128, 128, 0, s>>>(nq, qs);
    count_launch(ctx);
    if (smem_lbh > 48 * 1024) cudaFuncSetAttribute(k_walk_select, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_lbh);

    PairBufs P{};
    if (ctx->slot_ptr[S_TOPK_PAIRS]) carve_pairs((char*)ctx->slot_ptr[S_TOPK_PAIRS], pair_cap(ctx->slot_bytes[S_TOPK_PAIRS]), P);
    int chunk = std::max(4 * k, 128);
    if ((st = ensure_pairs(ctx, P, std::max<int64_t>((int64_t)nq * chunk * 2, 1 << 16), 0)) != GAT_OK) return st;

    int rounds = 0;
    int64_t used = 0;
    int rows_hint = std::min(max_q_len, db->maxlen);
    int max_cols = std::max(max_q_len, db->maxlen);
    int words = (n + 1 + 31) / 32;
    /* the walk: each round takes the next `chunk` candidates of every unfinished query in
     * (bound, id) order, evaluates them, updates W and applies the stop rule; chunks grow
     * geometrically so a query needs O(log) rounds */
    for (;;) {
        if (rounds >= kMaxRounds) return fail(ctx, GAT_ERR_STATE, "top-k: candidate walk did not finish");
        k_walk_select<<<nq, kT, smem_lbh, s>>>(n, lb, chunk, bins_lb, qs);
        count_launch(ctx);
        bool done_round = false;
        for (int attempt = 0; attempt < 2 && !done_round; attempt++) {
            k_walk_compact<<<nq, kT, 0, s>>>(n, lb, qs, d_q_len, d_q_off, db->d_len, db->d_off, P.cap, cursor, P.pq, P.pt,
                                             P.aoff, P.alen, P.boff, P.blen, seg_base + (size_t)rounds * nq,
                                             seg_cnt + (size_t)rounds * nq);
            count_launch(ctx);
            int64_t cur = 0;
            if ((st = read_word(ctx, cursor, &cur)) != GAT_OK) return st;
            if (cur <= P.cap) {
                int np = (int)(cur - used);
                if (np > 0 && (st = edr_launch_soa(ctx, np, nullptr, P.aoff + used, P.alen + used, P.boff + used,
                                                   P.blen + used, rows_hint, max_cols, d_q_xy, db->d_xy, u,
                                                   P.dist + used, cells)) != GAT_OK)
                    return st;
                used = cur;
                done_round = true;
            } else {
                /* overflow: grow, rewind the cursor, redo the compaction (the walk position only
                 * advances when a query's chunk fitted) */
                if ((st = ensure_pairs(ctx, P, cur, used)) != GAT_OK) return st;
                ctx->h_pinned[2] = used;
                GAT_CUDA_TRY(ctx, cudaMemcpyAsync(cursor, ctx->h_pinned + 2, 8, cudaMemcpyHostToDevice, s), "top-k");
            }
        }
        if (!done_round) return fail(ctx, GAT_ERR_OOM, "top-k: pair buffer overflow");
        rounds++;
        k_kth<<<nq, kT, smem_dh, s>>>(rounds, seg_base, seg_cnt, nq, P.dist, k, bins_d, qs);
        count_launch(ctx);
        GAT_CUDA_TRY(ctx, cudaMemsetAsync(pending, 0, 4, s), "top-k");
        k_walk_check<<<nq, kT, 0, s>>>(n, lb, rounds, seg_base, seg_cnt, nq, P.dist, P.pt, k, qs, pending);
        count_launch(ctx);
        int64_t pend = 0;
        if ((st = read_word(ctx, cursor + 2, &pend)) != GAT_OK) return st;
        if ((pend & 0xffffffff) == 0) break;
        chunk = (int)std::min<int64_t>((int64_t)chunk * 2, 1 << 20);
    }
    /* selection */
    uint32_t* gbm = nullptr;
    size_t smem_final = (size_t)words * 4;
    if (smem_final > 160 * 1024) {
        gbm = (uint32_t*)scratch(ctx, S_TOPK_DIST, (size_t)nq * words * 4, &st);
        if (!gbm) return st;
        smem_final = 0;
    } else if (smem_final > 32 * 1024) {
        cudaFuncSetAttribute(k_final, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_final);
    }
    k_final<<<nq, kT, smem_final, s>>>(rounds, seg_base, seg_cnt, nq, P.dist, P.pt, k, words, gbm, qs, d_ids, d_dist);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "top-k launch");
    if ((st = check_device_flag(ctx, "top-k")) != GAT_OK) return st;
    if (stats || ctx->timing) {
        int64_t c = 0;
        if ((st = read_word(ctx, cells, &c)) != GAT_OK) return st;
        timed_add_work(ctx, GAT_KERNEL_EDR, (double)c);
        if (stats) {
            stats[0] += used;
            stats[1] += c;
        }
    }
    return GAT_OK;
}

int topk_dev(gat_ctx* ctx, const gat_index* g, int nq, const int32_t* d_q_len, const int64_t* d_q_off,
             const float2* d_q_xy, int max_q_len, int k, double eps, int exec, int32_t* d_ids, int32_t* d_dist,
             int64_t* stats) {
    float u = match_threshold(eps);
    int64_t l0 = ctx->launches;
    int64_t local[4] = {0, 0, 0, 0};
    int st = GAT_OK;
    if (exec == GAT_EXEC_BATCHED) {
        /* batches bounded so the bound matrix stays below ~4 GiB */
        int64_t per = std::max<int64_t>(1, ((int64_t)1 << 30) / std::max(1, g->db->n + 1));
        for (int q0 = 0; q0 < nq && st == GAT_OK; q0 += (int)per) {
            int c = (int)std::min<int64_t>(per, nq - q0);
            st = topk_batch(ctx, g, c, d_q_len + q0, d_q_off + q0, d_q_xy, max_q_len, k, u, d_ids + (size_t)q0 * k,
                            d_dist + (size_t)q0 * k, local);
        }
    } else {
        for (int qi = 0; qi < nq && st == GAT_OK; qi++)
            st = topk_batch(ctx, g, 1, d_q_len + qi, d_q_off + qi, d_q_xy, max_q_len, k, u, d_ids + (size_t)qi * k,
                            d_dist + (size_t)qi * k, local);
    }
    if (st != GAT_OK) return st;
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "top-k");
    if (stats) {
        stats[0] = local[0];
        stats[1] = local[1];
        stats[2] = ctx->launches - l0;
    }
    return GAT_OK;
}

int check_grid(gat_ctx* ctx, const gat_index* g) {
    if (!g || g->kind != GAT_INDEX_GRID) return fail(ctx, GAT_ERR_STATE, "top-k needs a Grid index (it holds the FVTable)");
    if (g->ctx != ctx) return fail(ctx, GAT_ERR_STATE, "index from another context");
    return GAT_OK;
}

struct HostQueries {
    int64_t total = 0;
    int maxlen = 0;
    std::vector<int64_t> off;
};

int prep_host_queries(gat_ctx* ctx, int nq, const int32_t* q_len, HostQueries& h) {
    h.off.assign(nq + 1, 0);
    for (int i = 0; i < nq; i++) {
        if (q_len[i] < 1 || q_len[i] > GAT_EDR_MAX_LEN) return fail(ctx, GAT_ERR_ARG, "top-k: query length outside 1..GAT_EDR_MAX_LEN");
        h.off[i + 1] = h.off[i] + q_len[i];
        h.maxlen = std::max(h.maxlen, q_len[i]);
    }
    h.total = h.off[nq];
    return GAT_OK;
}

__global__ void k_interleave(const float* lon, const float* lat, int64_t n, float2* xy) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        xy[i] = make_float2(lon[i], lat[i]);
}

/* copies host queries to device scratch: [len | off | lon | lat | xy]; lon/lat are copied
 * from the caller's buffers as they are (pinned buffers copy at full link speed) and
 * interleaved on the device */
int upload_queries(gat_ctx* ctx, int nq, const int32_t* q_len, const float* lon, const float* lat, const HostQueries& h,
                   int32_t** dl, int64_t** doff, float2** dxy) {
    int st = GAT_OK;
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t b_len = up((size_t)nq * 4), b_off = up((size_t)(nq + 1) * 8), b_f = up((size_t)h.total * 4);
    char* p = (char*)scratch(ctx, S_EDR_IO, b_len + b_off + 2 * b_f + 2 * b_f, &st);
    if (!p) return st;
    *dl = (int32_t*)p;
    *doff = (int64_t*)(p + b_len);
    float* dlon = (float*)(p + b_len + b_off);
    float* dlat = (float*)(p + b_len + b_off + b_f);
    *dxy = (float2*)(p + b_len + b_off + 2 * b_f);
    cudaStream_t s = ctx->stream;
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(*dl, q_len, (size_t)nq * 4, cudaMemcpyHostToDevice, s), "top-k H2D");
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(*doff, h.off.data(), (size_t)(nq + 1) * 8, cudaMemcpyHostToDevice, s), "top-k H2D");
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(dlon, lon, (size_t)h.total * 4, cudaMemcpyHostToDevice, s), "top-k H2D");
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(dlat, lat, (size_t)h.total * 4, cudaMemcpyHostToDevice, s), "top-k H2D");
    int grid = (int)std::min<int64_t>(ctx->sm_count * 8, (h.total + 255) / 256 + 1);
    k_interleave<<<grid, 256, 0, s>>>(dlon, dlat, h.total, *dxy);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "top-k H2D");
    return GAT_OK;
}

}  // namespace
}  // namespace gat

using namespace gat;

extern "C" {

int gat_topk_dev(gat_ctx* ctx, const gat_index* grid, int nq, const int32_t* d_q_len, const int64_t* d_q_off,
                 const float* d_q_xy, int max_q_len, int k, double eps, int exec, int32_t* d_ids, int32_t* d_dist,
                 int64_t* stats) {
    if (!ctx || nq < 0 || k < 1 || k > 1024 || !(eps > 0) || max_q_len < 1 || max_q_len > GAT_EDR_MAX_LEN ||
        (nq > 0 && (!d_q_len || !d_q_off || !d_q_xy || !d_ids || !d_dist)))
        return fail(ctx, GAT_ERR_ARG, "gat_topk_dev: bad arguments");
    int st = check_grid(ctx, grid);
    if (st != GAT_OK) return st;
    if (nq == 0) return GAT_OK;
    if (int rq = require_device(ctx, "gat_topk_dev")) return rq;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    return topk_dev(ctx, grid, nq, d_q_len, d_q_off, (const float2*)d_q_xy, max_q_len, k, eps, exec, d_ids, d_dist, stats);
}

int gat_topk(gat_ctx* ctx, const gat_index* grid, int nq, const int32_t* q_len, const float* q_lon, const float* q_lat,
             int k, double eps, int exec, int32_t* out_ids, int32_t* out_dist, int64_t* stats) {
    if (!ctx || nq < 0 || k < 1 || k > 1024 || !(eps > 0) || (exec != GAT_EXEC_PLAIN && exec != GAT_EXEC_BATCHED) ||
        (nq > 0 && (!q_len || !q_lon || !q_lat || !out_ids || !out_dist)))
        return fail(ctx, GAT_ERR_ARG, "gat_topk: bad arguments");
    int st = check_grid(ctx, grid);
    if (st != GAT_OK) return st;
    if (nq == 0) return GAT_OK;
    if (int rq = require_device(ctx, "gat_topk")) return rq;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    HostQueries h;
    if ((st = prep_host_queries(ctx, nq, q_len, h)) != GAT_OK) return st;
    int32_t* dl;
    int64_t* doff;
    float2* dxy;
    if ((st = upload_queries(ctx, nq, q_len, q_lon, q_lat, h, &dl, &doff, &dxy)) != GAT_OK) return st;
    int32_t* dres = (int32_t*)scratch(ctx, S_TOPK_OUT, (size_t)nq * k * 8 + 16, &st);
    if (!dres) return st;
    st = topk_dev(ctx, grid, nq, dl, doff, dxy, h.maxlen, k, eps, exec, dres, dres + (size_t)nq * k, stats);
    if (st == GAT_OK) {
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(out_ids, dres, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, ctx->stream), "top-k D2H");
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(out_dist, dres + (size_t)nq * k, (size_t)nq * k * 4, cudaMemcpyDeviceToHost, ctx->stream), "top-k D2H");
    }
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "top-k D2H");
    return st;
}

int gat_fv_lower_bounds(gat_ctx* ctx, const gat_index* grid, int nq, const int32_t* q_len, const float* q_lon,
                        const float* q_lat, int32_t* out) {
    if (!ctx || nq < 0 || (nq > 0 && (!q_len || !q_lon || !q_lat || !out))) return fail(ctx, GAT_ERR_ARG, "gat_fv_lower_bounds: bad arguments");
    int st = check_grid(ctx, grid);
    if (st != GAT_OK) return st;
    if (nq == 0) return GAT_OK;
    if (int rq = require_device(ctx, "gat_fv_lower_bounds")) return rq;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    HostQueries h;
    if ((st = prep_host_queries(ctx, nq, q_len, h)) != GAT_OK) return st;
    int32_t* dl;
    int64_t* doff;
    float2* dxy;
    if ((st = upload_queries(ctx, nq, q_len, q_lon, q_lat, h, &dl, &doff, &dxy)) != GAT_OK) return st;
    int64_t stats[4] = {0, 0, 0, -1}; /* bounds only */
    st = topk_batch(ctx, grid, nq, dl, doff, dxy, h.maxlen, 1, match_threshold(1e-9), nullptr, nullptr, stats);
    if (st != GAT_OK) return st;
    int n = grid->db->n;
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(out, ctx->slot_ptr[S_TOPK_LB], (size_t)nq * (n + 1) * 4, cudaMemcpyDeviceToHost, ctx->stream), "bounds D2H");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "bounds");
    return GAT_OK;
}

}  // extern "C"
