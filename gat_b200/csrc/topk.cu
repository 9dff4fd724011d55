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

#include "edr_kernel.cuh"
#include "internal.h"
#include "launch.cuh"

namespace gat {
namespace {

constexpr int kT = 256;
constexpr int kMaxFv = 128; /* merged frequency-vector entries per (query, trajectory) */

/* ---------------------------------------------------------------- reference cell ids */
/* getIdxFromXY (Grid.cpp:25-54) as the x86-64 build evaluates it, negative inputs included:
 * the bit length of a negative value is INT_MIN + 1 (log2 of a negative number converted to
 * int), and when both inputs are negative the loop does not run. */
__device__ __forceinline__ int ref_len(int v) {
    if (v == 0) return 1;
    if (v < 0) return INT_MIN + 1;
    return 32 - __clz(v);
}
__device__ __forceinline__ uint32_t spread16(uint32_t v) {
    v &= 0xFFFF;
    v = (v | (v << 8)) & 0x00FF00FF;
    v = (v | (v << 4)) & 0x0F0F0F0F;
    v = (v | (v << 2)) & 0x33333333;
    v = (v | (v << 1)) & 0x55555555;
    return v;
}
/* Closed form of that loop: it interleaves the low L bits of x and y, L = the larger bit
 * length (a negative input's length never wins), and yields 0 when both are negative. */
__device__ __forceinline__ int ref_morton(int x, int y) {
    if (x < 0 && y < 0) return 0;
    int L = max(x < 0 ? 0 : ref_len(x), y < 0 ? 0 : ref_len(y));
    uint32_t m = L >= 16 ? 0xFFFFu : ((1u << L) - 1u);
    return (int)(spread16((uint32_t)x & m) | (spread16((uint32_t)y & m) << 1));
}

/* Grid::WhichCellPointIn (Grid.cpp:202-208) */
__device__ __forceinline__ int cell_of(const GridDev& g, float lon, float lat) {
    int row = (int)__fdiv_rn(__fsub_rn(g.rymax, lat), g.cell);
    int col = (int)__fdiv_rn(__fsub_rn(lon, g.rxmin), g.cell);
    return ref_morton(col, row);
}

/* ---------------------------------------------------------------- 1. query FV */
/* one CTA per query: virtual cell of each point, then runs of equal consecutive cells
 * (a trajectory stays in a cell for many points), then the few runs sorted and merged.
 * qfv rows have stride `stride` (>= longest query); nnz in qfv_n. */
__global__ void k_query_fv(GridDev g, int nq, const int32_t* q_len, const int64_t* q_off, const float2* Q,
                           int stride, int pow2, int32_t* qfv_cell, int32_t* qfv_cnt, int32_t* qfv_n) {
    dep_wait();
    extern __shared__ unsigned long long rkey[]; /* pow2 run keys (cell << 32 | count), then pow2 cells */
    int* sk = reinterpret_cast<int*>(rkey + pow2);
    __shared__ int wsum[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int qi = blockIdx.x; qi < nq; qi += gridDim.x) {
        const int L = q_len[qi];
        const int64_t o = q_off[qi];
        for (int i = threadIdx.x; i < L; i += blockDim.x) sk[i] = cell_of(g, Q[o + i].x, Q[o + i].y) >> g.vparam;
        __syncthreads();
        /* run heads, compacted in order (L <= pow2 <= blockDim.x * chunks) */
        int base = 0;
        for (int c0 = 0; c0 < L; c0 += blockDim.x) {
            int i = c0 + threadIdx.x;
            bool head = i < L && (i == 0 || sk[i] != sk[i - 1]);
            unsigned bal = __ballot_sync(0xffffffffu, head);
            if (lane == 0) wsum[warp] = __popc(bal);
            __syncthreads();
            int wb = 0, tot = 0;
            for (int w = 0; w < nw; w++) {
                if (w < warp) wb += wsum[w];
                tot += wsum[w];
            }
            unsigned lt;
            asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
            if (head) {
                int r = base + wb + __popc(bal & lt);
                int e = i + 1;
                while (e < L && sk[e] == sk[i]) e++;
                rkey[r] = ((unsigned long long)(unsigned)sk[i] << 32) | (unsigned)(e - i);
            }
            base += tot;
            __syncthreads();
        }
        /* sort the runs by cell (bitonic over 64-bit (cell, count) keys in the run area),
         * then one thread merges equal cells; runs are few, the sort is short */
        const int R = base;
        int p2 = 1;
        while (p2 < R) p2 <<= 1;
        for (int a = R + threadIdx.x; a < p2; a += blockDim.x) rkey[a] = ~0ull;
        __syncthreads();
        for (int kk = 2; kk <= p2; kk <<= 1)
            for (int j = kk >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < p2; i += blockDim.x) {
                    int ixj = i ^ j;
                    if (ixj > i) {
                        unsigned long long a = rkey[i], b = rkey[ixj];
                        if ((a > b) == ((i & kk) == 0)) {
                            rkey[i] = b;
                            rkey[ixj] = a;
                        }
                    }
                }
                __syncthreads();
            }
        if (threadIdx.x == 0) {
            int w = 0;
            int32_t* oc = qfv_cell + (size_t)qi * stride;
            int32_t* on = qfv_cnt + (size_t)qi * stride;
            for (int a = 0; a < R; a++) {
                int cell = (int)(rkey[a] >> 32), cnt = (int)(rkey[a] & 0xffffffffu);
                if (w > 0 && oc[w - 1] == cell) {
                    on[w - 1] += cnt;
                } else {
                    oc[w] = cell;
                    on[w] = cnt;
                    w++;
                }
            }
            qfv_n[qi] = w;
        }
        __syncthreads();
    }
}

/* ---------------------------------------------------------------- 2. lower bounds */
/* Virtual cells that can change a trajectory's bound: the query's cells (shared cells), the
 * neighbour keys of the query's cells (pass 2 of FVTable.cpp:160-187 finds trajectory cells
 * there) and the cells whose own neighbour keys hit a query cell (pass 1, FVTable.cpp:129-156).
 * Away from the grid border the neighbour relation is symmetric, so the last set only needs
 * checking for border cells. A trajectory with no cell in the set has bound
 * max(its length, query length). */
__global__ void k_near_bitmap(int nq, int vbits, const int32_t* qfv_cell, const int32_t* qfv_n, int stride, int words,
                              uint32_t* near);

/* ---------------------------------------------------------------- 2b. bound kernel */
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

__device__ __forceinline__ bool in_qfv(const int32_t* qc, int qn, int c) {
    int lo = 0, hi = qn - 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        if (qc[mid] == c) return true;
        if (qc[mid] < c)
            lo = mid + 1;
        else
            hi = mid - 1;
    }
    return false;
}

__device__ __forceinline__ void set_bit(uint32_t* bm, int words, int c) {
    if (c >= 0 && (c >> 5) < words) atomicOr(&bm[c >> 5], 1u << (c & 31));
}

__global__ void k_near_bitmap(int nq, int vbits, const int32_t* qfv_cell, const int32_t* qfv_n, int stride, int words,
                              uint32_t* near) {
    dep_wait();
    int qi = blockIdx.x;
    uint32_t* bm = near + (size_t)qi * words;
    for (int w = threadIdx.x; w < words; w += blockDim.x) bm[w] = 0;
    __syncthreads();
    const int qn = qfv_n[qi];
    const int32_t* qc = qfv_cell + (size_t)qi * stride;
    int nb[8];
    for (int i = threadIdx.x; i < qn; i += blockDim.x) {
        set_bit(bm, words, qc[i]);
        fv_neighbors(qc[i], vbits, nb);
        for (int k = 0; k < 8; k++) set_bit(bm, words, nb[k]);
    }
    /* border cells (virtual x or y equal to 0 or side - 1): at x == 0 / y == 0 findNeighbor's
     * keys come from getIdxFromXY(-1, .); at the far border they can equal the id of a query
     * point beyond the grid, whose own neighbours are decoded from its low bits only */
    const int side = 1 << (vbits / 2);
    for (int e = threadIdx.x; e < 4 * side; e += blockDim.x) {
        int k4 = e / side, r = e % side;
        int x = k4 == 0 ? 0 : k4 == 1 ? side - 1 : r;
        int y = k4 == 0 || k4 == 1 ? r : (k4 == 2 ? 0 : side - 1);
        int c = 0;
        for (int bit = 0; bit < vbits / 2; bit++) c |= (((x >> bit) & 1) << (2 * bit)) | (((y >> bit) & 1) << (2 * bit + 1));
        fv_neighbors(c, vbits, nb);
        for (int k = 0; k < 8; k++)
            if (in_qfv(qc, qn, nb[k])) {
                set_bit(bm, words, c);
                break;
            }
    }
}

/* one thread per (query, trajectory). The merged vector holds every cell of either vector
 * with value db - query (0 = absent). Pass 1 visits the positive cells in ascending order,
 * pass 2 the negative ones (FVTable.cpp:129-187); the reference increments a map iterator
 * after erasing its node, this visits each key present when the pass starts once. */
__global__ void __launch_bounds__(kT) k_lower_bounds(int n, int nq, const int64_t* __restrict__ fv_off,
                                                     const int32_t* __restrict__ fv_cell,
                                                     const int32_t* __restrict__ fv_cnt, const int32_t* qfv_cell,
                                                     const int32_t* qfv_cnt, const int32_t* qfv_n, int stride,
                                                     int vbits, const uint32_t* __restrict__ near, int words,
                                                     const int32_t* __restrict__ q_len, int32_t* lb, int32_t* flag) {
    dep_wait();
    extern __shared__ int sq[];
    int qi = blockIdx.y;
    int qn = qfv_n[qi];
    const int qlen = q_len[qi];
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
    {
        const uint32_t* bm = near + (size_t)qi * words;
        bool touches = false;
        int tlen = 0;
        for (int64_t j = b; j < e; j++) {
            int c = fv_cell[j];
            tlen += fv_cnt[j];
            if ((c >> 5) < words && ((__ldg(bm + (c >> 5)) >> (c & 31)) & 1u)) touches = true;
        }
        if (!touches) {
            lb[(size_t)qi * (n + 1) + t] = max(tlen, qlen);
            return;
        }
    }
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

/* ---------------------------------------------------------------- 3. candidate order */
/* Stable counting sort of every query's candidates by bound: tiles of kSortTile ids count
 * their bounds (per-tile histograms laid out bound-major, tile-minor), one exclusive scan over
 * all queries turns them into output positions, and one warp per tile scatters its ids in id
 * order, so equal bounds keep ascending ids: the order is (bound, id). */
constexpr int kSortTile = 2048;

__global__ void k_sort_hist(int n, const int32_t* lb, int bins, int ntile, int64_t* H) {
    dep_wait();
    extern __shared__ int hist[];
    int tile = blockIdx.x, qi = blockIdx.y;
    for (int i = threadIdx.x; i < bins; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const int32_t* row = lb + (size_t)qi * (n + 1);
    int t0 = 1 + tile * kSortTile, t1 = min(n, (tile + 1) * kSortTile);
    for (int t = t0 + threadIdx.x; t <= t1; t += blockDim.x) atomicAdd(&hist[min(row[t], bins - 1)], 1);
    __syncthreads();
    for (int v = threadIdx.x; v < bins; v += blockDim.x) H[((size_t)qi * bins + v) * ntile + tile] = hist[v];
}

/* one warp per (tile, query); the tile's running output offset per bound lives in shared
 * memory (loaded from the scanned histograms), the warp walks its ids in order 32 at a time */
__global__ void __launch_bounds__(32) k_sort_scatter(int n, const int32_t* lb, int bins, int ntile, const int64_t* H,
                                                     int32_t* cand, int32_t* slb) {
    dep_wait();
    extern __shared__ long long run[];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x;
    const int tile = blockIdx.x, qi = blockIdx.y;
    for (int v = lane; v < bins; v += 32) run[v] = H[((size_t)qi * bins + v) * ntile + tile];
    __syncwarp();
    const int32_t* row = lb + (size_t)qi * (n + 1);
    const int t0 = 1 + tile * kSortTile, t1 = min(n, (tile + 1) * kSortTile);
    unsigned lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    for (int b = t0; b <= t1; b += 32) {
        const int t = b + lane;
        const int raw = t <= t1 ? row[t] : -1;
        const int v = raw < 0 ? -1 : min(raw, bins - 1);
        const unsigned peers = __match_any_sync(FULL, v);
        const int leader = __ffs(peers) - 1;
        const int rank = __popc(peers & lt);
        long long base = 0;
        if (v >= 0 && lane == leader) {
            base = run[v];
            run[v] = base + __popc(peers);
        }
        base = __shfl_sync(FULL, base, leader);
        if (v >= 0) {
            const int64_t pos = base + rank; /* global position; query qi's slice starts at qi * n */
            cand[pos] = t;
            slb[pos] = raw;
        }
        __syncwarp();
    }
}

/* ---------------------------------------------------------------- 4. the walk */
/* per-query walk state */
enum { WS_END = 0, WS_START, WS_CHUNK, WS_W, WS_DONE, WS_WORDS };

__global__ void k_walk_init(int nq, int chunk, int32_t* ws) {
    dep_wait();
    int qi = blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= nq) return;
    int32_t* s = ws + (size_t)qi * WS_WORDS;
    s[WS_END] = 0;
    s[WS_START] = 0;
    s[WS_CHUNK] = chunk;
    s[WS_W] = INT_MAX;
    s[WS_DONE] = 0;
}

/* One CTA: each unfinished query extends its evaluated prefix [0, end) of the (bound, id)
 * order by up to `chunk` candidates whose bound is at most W; the new slices are numbered
 * consecutively over the queries (wprefix) for the EDR kernel. */
__global__ void k_walk_plan(int n, int nq, const int32_t* slb, int32_t* ws, int* wprefix) {
    dep_wait();
    __shared__ int warp_sum[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int q0 = 0; q0 < nq; q0 += blockDim.x) {
        int qi = q0 + threadIdx.x;
        int cnt = 0;
        if (qi < nq) {
            int32_t* s = ws + (size_t)qi * WS_WORDS;
            int end = s[WS_END];
            s[WS_START] = end;
            if (!s[WS_DONE]) {
                int e = (int)min((long long)n, (long long)end + s[WS_CHUNK]);
                /* candidates with a bound above W can never be needed */
                int W = s[WS_W];
                const int32_t* row = slb + (size_t)qi * n;
                if (e > end && row[e - 1] > W) {
                    int lo = end, hi = e - 1; /* first index in [end, e) with bound > W */
                    while (lo < hi) {
                        int mid = (lo + hi) >> 1;
                        if (row[mid] > W)
                            hi = mid;
                        else
                            lo = mid + 1;
                    }
                    e = lo;
                }
                cnt = e - end;
                s[WS_END] = e;
            }
        }
        int x = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sum[warp] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            int run = 0;
            for (int w = 0; w < nw; w++) {
                int t = warp_sum[w];
                warp_sum[w] = run;
                run += t;
            }
        }
        __syncthreads();
        if (qi < nq) wprefix[qi] = carry + warp_sum[warp] + x - cnt;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += warp_sum[warp] + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) wprefix[nq] = carry;
}

/* EDR pairs of the current round: work item w belongs to the query whose wprefix range holds
 * it, and is candidate start + (w - wprefix[q]) of that query's order. */
struct WalkPairs {
    int n, nq;
    const int* wprefix;
    const int32_t* ws;
    const int32_t* cand;
    const int32_t* q_len;
    const int64_t* q_off;
    const float2* Q;
    const int32_t* db_len;
    const int64_t* db_off;
    const float2* DB;
    int32_t* sdist;
    static constexpr int kKind = 1;
    __device__ int count() const { return wprefix[nq]; }
    __device__ void get(int w, const float2*& a, int& la, const float2*& b, int& lb, int32_t*& o) const {
        int lo = 0, hi = nq - 1; /* last q with wprefix[q] <= w */
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (wprefix[mid] <= w)
                lo = mid;
            else
                hi = mid - 1;
        }
        int q = lo;
        size_t idx = (size_t)q * n + ws[(size_t)q * WS_WORDS + WS_START] + (w - wprefix[q]);
        int t = cand[idx];
        a = Q + q_off[q];
        la = q_len[q];
        b = DB + db_off[t];
        lb = db_len[t];
        o = sdist + idx;
    }
};

/* Per query: W = k-th smallest distance over the evaluated prefix, then the stop rule with
 * (nlb, nid) the next candidate: done at the end of the order, when nlb > W, or when nlb == W
 * and k evaluated pairs already sort before (W, nid). While nlb < W the walk goes on: a
 * candidate with a smaller bound may still be closer. */
__global__ void k_walk_kth(int n, int k, int bins, int growth, const int32_t* slb, const int32_t* cand,
                           const int32_t* sdist, int32_t* ws) {
    dep_wait();
    extern __shared__ int hist[];
    __shared__ int sh_W, cnt;
    __shared__ int warp_tot[kT / 32];
    int qi = blockIdx.x;
    int32_t* s = ws + (size_t)qi * WS_WORDS;
    if (s[WS_DONE]) return;
    const int end = s[WS_END];
    const int32_t* dist = sdist + (size_t)qi * n;
    for (int i = threadIdx.x; i < bins; i += blockDim.x) hist[i] = 0;
    if (threadIdx.x == 0) {
        cnt = 0;
        sh_W = INT_MAX;
    }
    __syncthreads();
    /* histogram of the evaluated distances, four loads in flight per thread (a negative
     * distance marks a pair whose wait gave up; the call then fails, it is not counted) */
    for (int i0 = threadIdx.x; i0 < end; i0 += 4 * blockDim.x) {
        int d[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int i = i0 + u * blockDim.x;
            d[u] = i < end ? dist[i] : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
            if (d[u] >= 0) atomicAdd(&hist[min(d[u], bins - 1)], 1);
    }
    __syncthreads();
    /* W = the first bin where the running count reaches k: each thread sums a slice of bins,
     * a block-wide scan gives the slice's starting count, and the one thread whose slice
     * crosses k walks it */
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const int per = (bins + blockDim.x - 1) / blockDim.x;
        const int b0 = min(bins, threadIdx.x * per), b1 = min(bins, b0 + per);
        int local = 0;
        for (int b = b0; b < b1; b++) local += hist[b];
        int incl = local;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        int before = incl - local;
        for (int w = 0; w < warp; w++) before += warp_tot[w];
        if (before < k && before + local >= k) {
            int run = before;
            for (int b = b0; b < b1; b++) {
                if (run + hist[b] >= k) {
                    sh_W = b;
                    break;
                }
                run += hist[b];
            }
        }
    }
    __syncthreads();
    const int W = sh_W;
    bool done;
    if (end >= n) {
        done = true;
    } else {
        int nlb = slb[(size_t)qi * n + end];
        if (nlb < W) {
            done = false;
        } else if (nlb > W) {
            done = true;
        } else {
            int nid = cand[(size_t)qi * n + end];
            const int32_t* ids = cand + (size_t)qi * n;
            int c = 0;
            for (int i = threadIdx.x; i < end; i += blockDim.x) {
                int d = dist[i];
                c += (d < W || (d == W && ids[i] < nid));
            }
            atomicAdd(&cnt, c);
            __syncthreads();
            done = cnt >= k;
        }
    }
    if (threadIdx.x == 0) {
        s[WS_W] = W;
        s[WS_DONE] = done ? 1 : 0;
        s[WS_CHUNK] = (int)min((long long)growth * s[WS_CHUNK], 1LL << 30);
    }
}

/* ---------------------------------------------------------------- 5. selection */
/* k smallest (distance, id) over the evaluated prefix: the pairs below W sorted, then the
 * smallest ids at W (a bitmap over ids in shared memory or a per-CTA global slice). */
__global__ void k_final(int n, int k, int words, uint32_t* gbitmap, const int32_t* cand, const int32_t* sdist,
                        const int32_t* ws, int32_t* out_ids, int32_t* out_dist, int32_t* flag,
                        unsigned long long* pairs) {
    dep_wait();
    extern __shared__ uint32_t bm_s[];
    __shared__ unsigned long long lt_keys[1024];
    __shared__ int lt_n;
    __shared__ int warp_cnt[kT / 32 + 1];
    int qi = blockIdx.x;
    uint32_t* bm = gbitmap ? gbitmap + (size_t)blockIdx.x * words : bm_s;
    const int32_t* s = ws + (size_t)qi * WS_WORDS;
    if (threadIdx.x == 0 && !s[WS_DONE]) atomicCAS(flag, 0, GAT_ERR_STATE);
    const int W = s[WS_W], end = s[WS_END];
    if (threadIdx.x == 0) atomicAdd(pairs, (unsigned long long)end); /* pairs evaluated */
    const int32_t* dist = sdist + (size_t)qi * n;
    const int32_t* ids = cand + (size_t)qi * n;
    for (int w = threadIdx.x; w < words; w += blockDim.x) bm[w] = 0;
    if (threadIdx.x == 0) lt_n = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < end; i += blockDim.x) {
        int d = dist[i], id = ids[i];
        if (d < W) {
            int slot = atomicAdd(&lt_n, 1);
            if (slot < 1024) lt_keys[slot] = ((unsigned long long)(unsigned)d << 32) | (unsigned)id;
        } else if (d == W) {
            atomicOr(&bm[id >> 5], 1u << (id & 31));
        }
    }
    __syncthreads();
    int nlt = min(lt_n, 1024);
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
    int need = k - emit;
    int per = (words + kT - 1) / kT;
    int w0 = threadIdx.x * per, w1 = min(words, w0 + per);
    int c = 0;
    for (int w = w0; w < w1; w++) c += __popc(bm[w]);
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
    if (threadIdx.x == 0) {
        int have = emit + min(warp_cnt[kT / 32], need);
        for (int i = have; i < k; i++) {
            out_ids[(size_t)qi * k + i] = -1;
            out_dist[(size_t)qi * k + i] = -1;
        }
    }
}

/* device bytes topk_batch needs per query (sorted candidates, bounds, distances, histograms) */
size_t topk_bytes_per_query(int n, int bins) {
    int ntile = (n + kSortTile - 1) / kSortTile;
    return (size_t)(n + 1) * 4 + (size_t)n * 12 + (size_t)bins * ntile * 8 + 64;
}

/* State of one batch between its phases (pointers into the context's scratch). */
struct TopkRun {
    const gat_index* g = nullptr;
    int nq = 0, n = 0, k = 0, max_q_len = 0;
    float u = 0.f;
    int32_t* lb = nullptr;
    int32_t *cand = nullptr, *slb = nullptr, *sdist = nullptr, *ws = nullptr;
    int* wprefix = nullptr;
    bool lone = false;
    int chunk0 = 0, growth = 0, rounds = 0;
    int bins_d = 0;
    size_t smem_d = 0;
    int rows_hint = 0, max_cols = 0;
    WalkPairs src{};
};

/* Phase 1: query frequency vectors, lower bounds, candidate order, walk state. */
int topk_pre(gat_ctx* ctx, const gat_index* g, int nq, const int32_t* d_q_len, const int64_t* d_q_off,
             const float2* d_q_xy, int max_q_len, int k, float u, int64_t* stats, TopkRun& R) {
    cudaStream_t s = ctx->stream;
    const gat_db* db = g->db;
    int n = db->n;
    int st = GAT_OK;
    R.g = g;
    R.nq = nq;
    R.n = n;
    R.k = k;
    R.u = u;
    R.max_q_len = max_q_len;
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
    size_t smem_fv = (size_t)pow2 * 12;
    allow_smem(k_query_fv, smem_fv);
    (void)launch_dep(ctx, k_query_fv, dim3(std::min(nq, ctx->sm_count * 4)), dim3(512), smem_fv, s, g->grid, nq, d_q_len, d_q_off, d_q_xy, stride, pow2,
                                                                      qfv_cell, qfv_cnt, qfv_n);
    count_launch(ctx);
    /* lower bounds */
    int32_t* lb = (int32_t*)scratch(ctx, S_TOPK_LB, (size_t)nq * (n + 1) * 4, &st);
    if (!lb) return st;
    R.lb = lb;
    int vbits = (int)std::log2((double)(g->grid.cellnum >> 2));
    int nwords = ((1 << vbits) + 31) / 32;
    uint32_t* near = (uint32_t*)scratch(ctx, S_TOPK_NEAR, (size_t)nq * nwords * 4 + 64, &st);
    if (!near) return st;
    (void)launch_dep(ctx, k_near_bitmap, dim3(nq), dim3(kT), 0, s, nq, vbits, qfv_cell, qfv_n, stride, nwords, near);
    count_launch(ctx);
    size_t smem_lb = (size_t)stride * 8;
    allow_smem(k_lower_bounds, smem_lb);
    dim3 lgrid((n + kT - 1) / kT, nq);
    timed_begin(ctx, GAT_KERNEL_BOUNDS);
    (void)launch_dep(ctx, k_lower_bounds, dim3(lgrid), dim3(kT), smem_lb, s, n, nq, g->d_fv_off, g->d_fv_cell, g->d_fv_cnt, qfv_cell, qfv_cnt, qfv_n, stride,
                                             vbits, near, nwords, d_q_len, lb, ctx->d_flag);
    /* algorithmic bytes: every trajectory's FV (8 B per entry + 8 B offset) and its bound (4 B)
     * per query */
    timed_end(ctx, GAT_KERNEL_BOUNDS, (double)nq * ((double)g->fv_entries * 8.0 + (double)n * 12.0));
    count_launch(ctx);
    if (stats && stats[3] == -1) return GAT_OK; /* bounds only */
    /* candidate order */
    int bins_lb = std::max(max_q_len, db->maxlen) + 2;
    int ntile = (n + kSortTile - 1) / kSortTile;
    int64_t* H = (int64_t*)scratch(ctx, S_TOPK_SEG, (size_t)nq * bins_lb * ntile * 8 + 64, &st);
    char* sorted = (char*)scratch(ctx, S_TOPK_PAIRS, (size_t)nq * n * 12 + 1024, &st);
    int32_t* ws = (int32_t*)scratch(ctx, S_TOPK_QSTATE, (size_t)nq * WS_WORDS * 4 + (size_t)(nq + 1) * 4 + 256, &st);
    if (!H || !sorted || !ws) return st;
    R.cand = (int32_t*)sorted;
    R.slb = R.cand + (size_t)nq * n;
    R.sdist = R.slb + (size_t)nq * n;
    R.ws = ws;
    R.wprefix = (int*)(ws + (size_t)nq * WS_WORDS);
    size_t smem_h = (size_t)bins_lb * 4;
    allow_smem(k_sort_hist, smem_h);
    (void)launch_dep(ctx, k_sort_hist, dim3(dim3(ntile, nq)), dim3(kT), smem_h, s, n, lb, bins_lb, ntile, H);
    count_launch(ctx);
    if ((st = scan_i64(ctx, H, H, (int64_t)nq * bins_lb * ntile)) != GAT_OK) return st;
    size_t smem_run = (size_t)bins_lb * 8;
    allow_smem(k_sort_scatter, smem_run);
    (void)launch_dep(ctx, k_sort_scatter, dim3(dim3(ntile, nq)), dim3(32), smem_run, s, n, lb, bins_lb, ntile, H, R.cand, R.slb);
    count_launch(ctx);
    /* the walk: a finished query costs nothing in later rounds and `rounds` covers the whole
     * order with growing chunks. A lone query leaves most of the GPU idle in a small round, so
     * it starts with a larger chunk; every walk doubles its chunk per round, which keeps the
     * surplus evaluations of the last round small. On the C2 set (100k walks, k = 32), first
     * rounds of 768 / 1024 / 1280 / 1536 candidates with doubling ran 3.21k / 3.29k / 3.40k /
     * 3.28k queries per second, quadrupling from 1024 2.9k. */
    R.lone = nq <= 4;
    R.chunk0 = ctx->topk_chunk ? ctx->topk_chunk : (R.lone ? 1280 : 128);
    R.chunk0 = std::max(R.chunk0, R.lone ? 8 * k : 4 * k);
    R.growth = ctx->topk_growth ? ctx->topk_growth : 2;
    R.rounds = 1;
    for (int64_t cover = R.chunk0, c = R.chunk0; cover < n; R.rounds++) {
        c *= R.growth;
        cover += c;
    }
    R.rounds += 1;
    (void)launch_dep(ctx, k_walk_init, dim3((nq + 127) / 128), dim3(128), 0, s, nq, R.chunk0, ws);
    count_launch(ctx);
    R.bins_d = max_q_len + db->maxlen + 2;
    R.smem_d = (size_t)R.bins_d * 4;
    allow_smem(k_walk_kth, R.smem_d);
    R.rows_hint = std::min(max_q_len, db->maxlen);
    R.max_cols = std::max(max_q_len, db->maxlen);
    R.src = WalkPairs{n, nq, R.wprefix, ws, R.cand, d_q_len, d_q_off, d_q_xy, db->d_len, db->d_off, db->d_xy, R.sdist};
    return GAT_OK;
}

/* Phase 2a: each unfinished query extends its evaluated prefix (pair numbering in wprefix). */
void topk_plan(gat_ctx* ctx, const TopkRun& R) {
    (void)launch_dep(ctx, k_walk_plan, dim3(1), dim3(1024), 0, ctx->stream, R.n, R.nq, R.slb, R.ws, R.wprefix);
    count_launch(ctx);
}

/* Phase 2b: EDR of the planned pairs (at most npairs), then the k-th distance and stop rule. */
int topk_round(gat_ctx* ctx, const TopkRun& R, int64_t npairs, unsigned long long* cells) {
    int st = edr::edr_launch(ctx, R.src, npairs, R.rows_hint, R.max_cols, R.u, cells);
    if (st != GAT_OK) return st;
    (void)launch_dep(ctx, k_walk_kth, dim3(R.nq), dim3(kT), R.smem_d, ctx->stream, R.n, R.k, R.bins_d, R.growth, R.slb, R.cand, R.sdist, R.ws);
    count_launch(ctx);
    return GAT_OK;
}

/* Phase 3: the k smallest (distance, id) pairs per query. */
int topk_post(gat_ctx* ctx, const TopkRun& R, int32_t* d_ids, int32_t* d_dist, unsigned long long* pairs) {
    int st = GAT_OK;
    int words = (R.n + 1 + 31) / 32;
    uint32_t* gbm = nullptr;
    size_t smem_final = (size_t)words * 4;
    if (smem_final > 160 * 1024) {
        gbm = (uint32_t*)scratch(ctx, S_TOPK_DIST, (size_t)R.nq * words * 4, &st);
        if (!gbm) return st;
        smem_final = 0;
    } else {
        allow_smem(k_final, smem_final);
    }
    (void)launch_dep(ctx, k_final, dim3(R.nq), dim3(kT), smem_final, ctx->stream, R.n, R.k, words, gbm, R.cand, R.sdist, R.ws, d_ids, d_dist, ctx->d_flag,
                                                   pairs);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "top-k launch");
    return GAT_OK;
}

/* The whole pipeline for queries [0, nq) of the given device arrays. acc: device counters
 * [0] DP cells, [1] pairs evaluated, accumulated over calls; status and counters are read by
 * the caller once per API call. */
int topk_batch(gat_ctx* ctx, const gat_index* g, int nq, const int32_t* d_q_len, const int64_t* d_q_off,
               const float2* d_q_xy, int max_q_len, int k, float u, int32_t* d_ids, int32_t* d_dist, int64_t* stats,
               unsigned long long* acc) {
    TopkRun R;
    int st = topk_pre(ctx, g, nq, d_q_len, d_q_off, d_q_xy, max_q_len, k, u, stats, R);
    if (st != GAT_OK) return st;
    if (stats && stats[3] == -1) return check_device_flag(ctx, "frequency-vector bounds");
    /* A lone query's first rounds are launched without a host round trip, sized by their upper
     * bound (each query extends by at most its chunk; a finished query adds no pairs and the
     * kernels of an empty round exit at once). Later rounds, and every round of a batch, read
     * the exact pair count first; it is zero once no query can extend (every query at the end
     * of its order or with its next bound above W). */
    /* with per-kernel timing on, rounds follow the exact sizes, as the query graph's loop does */
    const int blind_rounds = (R.lone && !ctx->timing) ? 2 : 0;
    int64_t chunk_r = R.chunk0;
    for (int r = 0; r < R.rounds; r++) {
        topk_plan(ctx, R);
        int64_t npairs = std::min<int64_t>((int64_t)nq * chunk_r, (int64_t)nq * R.n);
        if (r >= blind_rounds) {
            int32_t* cnt = reinterpret_cast<int32_t*>(ctx->h_pinned + 4);
            GAT_CUDA_TRY(ctx, cudaMemcpyAsync(cnt, R.wprefix + nq, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream),
                         "top-k");
            GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "top-k");
            npairs = *cnt;
            if (npairs == 0) break;
        }
        if ((st = topk_round(ctx, R, npairs, acc)) != GAT_OK) return st;
        chunk_r = std::min<int64_t>(chunk_r * R.growth, (int64_t)1 << 30);
    }
    return topk_post(ctx, R, d_ids, d_dist, acc + 1);
}

/* ---------------------------------------------------------------- lone queries as a CUDA graph */
/* One query of the plain form is a chain of ~20 small launches with data-dependent rounds.
 * Launched one by one from the host, the chain waits on launch latency and on a host read of
 * each round's size. Instead the whole chain of one query is a CUDA graph: a stage kernel takes
 * the next query index from a device counter and copies that query into fixed buffers; the
 * bound / order kernels follow; the walk rounds sit in a conditional while node whose
 * condition the last kernel of each round sets from the query's done flag; the selection and
 * an unstage kernel write the k results to the caller's arrays. The host launches the graph
 * once per query with no synchronisation in between. Every buffer the graph touches belongs
 * to a worker context used by nothing else, sized by a first, uncaptured run of the same
 * kernels, so no pointer in the graph moves. EDR rounds are sized for the whole set (empty
 * slots cost nothing) and use a fixed tile height (no host-side tuning inside a graph). */
struct StageDesc {
    const int32_t* q_len;
    const int64_t* q_off;
    const float2* q_xy;
    int32_t* ids;
    int32_t* dist;
    int nq;
    int max_len;
};

__global__ void k_stage(const StageDesc* d, int* next, int* cur, int32_t* len1, int64_t* off1, float2* xy1,
                        int32_t* flag) {
    dep_wait();
    __shared__ int qi_s, len_s;
    __shared__ long long off_s;
    if (threadIdx.x == 0) {
        const int qi = atomicAdd(next, 1);
        int L = 1;
        long long o = 0;
        if (qi < d->nq) {
            L = d->q_len[qi];
            o = d->q_off[qi];
            if (L < 1 || L > d->max_len) {
                atomicCAS(flag, 0, GAT_ERR_ARG); /* the longest query was understated */
                L = min(max(L, 1), d->max_len);
            }
        }
        *cur = qi;
        qi_s = qi;
        len_s = L;
        off_s = o;
        len1[0] = L;
        off1[0] = 0;
        off1[1] = L;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < len_s; i += blockDim.x)
        xy1[i] = qi_s < d->nq ? d->q_xy[off_s + i] : make_float2(0.f, 0.f);
}

__global__ void k_unstage(const StageDesc* d, const int* cur, const int32_t* ids1, const int32_t* dist1, int k) {
    dep_wait();
    const int qi = *cur;
    if (qi >= d->nq) return;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        d->ids[(size_t)qi * k + i] = ids1[i];
        d->dist[(size_t)qi * k + i] = dist1[i];
    }
}

/* ends the round loop once the query is done; a bound on the rounds guards the loop */
__global__ void k_loop_cond(const int32_t* ws, int* iter, int maxit, int32_t* flag, unsigned long long* rounds,
                            cudaGraphConditionalHandle h) {
    dep_wait();
    const int it = ++(*iter);
    atomicAdd(rounds, 1ull);
    bool more = ws[WS_DONE] == 0;
    if (more && it >= maxit) {
        atomicCAS(flag, 0, GAT_ERR_STATE);
        more = false;
    }
    cudaGraphSetConditional(h, more ? 1u : 0u);
}

struct LoneGraph {
    const gat_index* g = nullptr;
    int max_q_len = 0, k = 0;
    float u = 0.f;
    int chunk = 0, growth = 0, rows = 0, form = 0, dep = 1; /* the context's knobs when the graph was built */
    gat_ctx* w = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev = nullptr;
    int64_t launches_fixed = 0, launches_round = 0; /* per replay: outside / inside the loop */
    StageDesc* d_desc = nullptr;
    int *d_next = nullptr, *d_cur = nullptr, *d_iter = nullptr;
    int32_t* len1 = nullptr;
    int64_t* off1 = nullptr;
    float2* xy1 = nullptr;
    int32_t *ids1 = nullptr, *dist1 = nullptr;
    unsigned long long* acc = nullptr; /* [0] cells, [1] pairs, [2] rounds */
};

void lone_graph_free(void* p) {
    auto* L = static_cast<LoneGraph*>(p);
    if (L->exec) cudaGraphExecDestroy(L->exec);
    if (L->graph) cudaGraphDestroy(L->graph);
    if (L->ev) cudaEventDestroy(L->ev);
    if (L->w) gat_ctx_destroy(L->w);
    delete L;
}

constexpr int kLoneGraphCache = 2;
constexpr int kLoneRows = 4; /* 128-point tiles: the best of 2/4/8 on one query's pairs (a few hundred points) */
constexpr int kLoneForm = 1; /* row tiles: column tiles measured slower on one query's pairs (many short tiles) */

int lone_graph_get(gat_ctx* ctx, const gat_index* g, int max_q_len, int k, float u, LoneGraph** out) {
    for (auto& o : ctx->owned)
        if (o.second == lone_graph_free) {
            auto* L = static_cast<LoneGraph*>(o.first);
            if (L->g == g && L->max_q_len == max_q_len && L->k == k && L->u == u && L->chunk == ctx->topk_chunk &&
                L->growth == ctx->topk_growth && L->rows == ctx->edr_rows && L->form == ctx->edr_form &&
                L->dep == ctx->dep_launch) {
                *out = L;
                return GAT_OK;
            }
        }
    int n_graphs = 0;
    for (auto& o : ctx->owned) n_graphs += o.second == lone_graph_free;
    if (n_graphs >= kLoneGraphCache) {
        for (auto it = ctx->owned.begin(); it != ctx->owned.end(); ++it)
            if (it->second == lone_graph_free) {
                lone_graph_free(it->first);
                ctx->owned.erase(it);
                break;
            }
    }
    auto* L = new LoneGraph();
    L->g = g;
    L->max_q_len = max_q_len;
    L->k = k;
    L->u = u;
    int st = gat_ctx_create_worker(ctx, &L->w);
    if (st != GAT_OK) {
        delete L;
        return fail(ctx, st, "top-k: worker context for the query graph");
    }
    L->chunk = ctx->topk_chunk;
    L->growth = ctx->topk_growth;
    L->rows = ctx->edr_rows;
    L->form = ctx->edr_form;
    L->dep = ctx->dep_launch;
    L->w->edr_rows = ctx->edr_rows ? ctx->edr_rows : kLoneRows;
    L->w->edr_form = ctx->edr_form ? ctx->edr_form : kLoneForm;
    L->w->topk_chunk = ctx->topk_chunk;
    L->w->topk_growth = ctx->topk_growth;
    L->w->dep_launch = ctx->dep_launch;
    if (cudaEventCreateWithFlags(&L->ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        lone_graph_free(L);
        return fail(ctx, GAT_ERR_CUDA, "top-k: event");
    }
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t b_desc = up(sizeof(StageDesc)), b_ctr = 256, b_len = 256, b_off = 256;
    const size_t b_xy = up((size_t)max_q_len * sizeof(float2)), b_out = up((size_t)k * 4);
    char* p = (char*)scratch(L->w, S_TOPK_GSTAGE, b_desc + b_ctr + b_len + b_off + b_xy + 2 * b_out, &st);
    L->acc = (unsigned long long*)scratch(L->w, S_TOPK_IO, 256, &st);
    if (!p || !L->acc) {
        lone_graph_free(L);
        return fail(ctx, GAT_ERR_OOM, "top-k: query graph buffers");
    }
    L->d_desc = (StageDesc*)p;
    p += b_desc;
    L->d_next = (int*)p;
    L->d_cur = L->d_next + 1;
    L->d_iter = L->d_next + 2;
    p += b_ctr;
    L->len1 = (int32_t*)p;
    p += b_len;
    L->off1 = (int64_t*)p;
    p += b_off;
    L->xy1 = (float2*)p;
    p += b_xy;
    L->ids1 = (int32_t*)p;
    L->dist1 = (int32_t*)(p + b_out);
    ctx->owned.emplace_back(L, lone_graph_free);
    *out = L;
    return GAT_OK;
}

/* the kernels of one query before / inside / after the round loop, on the worker's stream */
int lone_pre(LoneGraph* L, TopkRun& R) {
    gat_ctx* w = L->w;
    (void)launch_dep(w, k_stage, dim3(1), dim3(256), 0, w->stream, L->d_desc, L->d_next, L->d_cur, L->len1, L->off1, L->xy1, w->d_flag);
    count_launch(w);
    (void)launch_dep(w, k_zero_words, dim3(1), dim3(32), 0, w->stream, L->d_iter, 1);
    return topk_pre(w, L->g, 1, L->len1, L->off1, L->xy1, L->max_q_len, L->k, L->u, nullptr, R);
}

int lone_round(LoneGraph* L, const TopkRun& R, const cudaGraphConditionalHandle* h) {
    gat_ctx* w = L->w;
    topk_plan(w, R);
    int st = topk_round(w, R, R.n, L->acc);
    if (st != GAT_OK) return st;
    if (h) {
        (void)launch_dep(w, k_loop_cond, dim3(1), dim3(1), 0, w->stream, R.ws, L->d_iter, R.rounds + 1, w->d_flag, L->acc + 2, *h);
        count_launch(w);
    }
    return GAT_OK;
}

int lone_post(LoneGraph* L, const TopkRun& R) {
    gat_ctx* w = L->w;
    int st = topk_post(w, R, L->ids1, L->dist1, L->acc + 1);
    if (st != GAT_OK) return st;
    (void)launch_dep(w, k_unstage, dim3(1), dim3(256), 0, w->stream, L->d_desc, L->d_cur, L->ids1, L->dist1, L->k);
    count_launch(w);
    return GAT_OK;
}

/* The first query of a new graph runs uncaptured (this sizes every scratch slot), then the
 * graph is captured: pre and post as child graphs, the rounds as the body of a while node. */
int lone_build(LoneGraph* L) {
    gat_ctx* w = L->w;
    cudaStream_t s = w->stream;
    TopkRun R;
    int st = lone_pre(L, R);
    if (st != GAT_OK) return st;
    for (int r = 0; r < R.rounds; r++) {
        if ((st = lone_round(L, R, nullptr)) != GAT_OK) return st;
        int32_t* done = reinterpret_cast<int32_t*>(w->h_pinned + 4);
        GAT_CUDA_TRY(w, cudaMemcpyAsync(done, R.ws + WS_DONE, 4, cudaMemcpyDeviceToHost, s), "top-k");
        GAT_CUDA_TRY(w, cudaStreamSynchronize(s), "top-k");
        if (*done) break;
    }
    if ((st = lone_post(L, R)) != GAT_OK) return st;
    GAT_CUDA_TRY(w, cudaStreamSynchronize(s), "top-k");
    GAT_CUDA_TRY(w, cudaGetLastError(), "top-k");

    cudaGraph_t gpre = nullptr, gpost = nullptr, G = nullptr;
    auto cleanup = [&]() {
        if (gpre) cudaGraphDestroy(gpre);
        if (gpost) cudaGraphDestroy(gpost);
        if (G) cudaGraphDestroy(G);
        cudaGetLastError();
    };
    auto capture = [&](cudaGraph_t* out, auto&& fn) -> int {
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return cuda_fail(w, cudaGetLastError(), "capture");
        int rc = fn();
        cudaGraph_t gr = nullptr;
        cudaError_t e = cudaStreamEndCapture(s, &gr);
        if (rc != GAT_OK) {
            if (gr) cudaGraphDestroy(gr);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(w, e, "capture");
        *out = gr;
        return GAT_OK;
    };
    int64_t l0 = w->launches;
    TopkRun RC;
    if ((st = capture(&gpre, [&] { return lone_pre(L, RC); })) != GAT_OK) return cleanup(), st;
    const int64_t l1 = w->launches;
    if ((st = capture(&gpost, [&] { return lone_post(L, RC); })) != GAT_OK) return cleanup(), st;
    const int64_t l2 = w->launches;
    if (cudaGraphCreate(&G, 0) != cudaSuccess) return cleanup(), cuda_fail(w, cudaGetLastError(), "graph");
    cudaGraphNode_t npre = nullptr, nloop = nullptr, npost = nullptr;
    cudaGraphConditionalHandle h;
    if (cudaGraphAddChildGraphNode(&npre, G, nullptr, 0, gpre) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&h, G, 1, cudaGraphCondAssignDefault) != cudaSuccess)
        return cleanup(), cuda_fail(w, cudaGetLastError(), "graph");
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if (cudaGraphAddNode(&nloop, G, &npre, 1, &cp) != cudaSuccess) return cleanup(), cuda_fail(w, cudaGetLastError(), "graph");
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return cleanup(), cuda_fail(w, cudaGetLastError(), "graph");
    const int64_t l3 = w->launches;
    st = lone_round(L, RC, &h);
    const int64_t l4 = w->launches;
    cudaGraph_t body_out = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &body_out);
    if (st != GAT_OK) return cleanup(), st;
    if (e != cudaSuccess) return cleanup(), cuda_fail(w, e, "graph");
    if (cudaGraphAddChildGraphNode(&npost, G, &nloop, 1, gpost) != cudaSuccess ||
        cudaGraphInstantiate(&L->exec, G, 0) != cudaSuccess)
        return cleanup(), cuda_fail(w, cudaGetLastError(), "graph instantiate");
    cudaGraphDestroy(gpre);
    cudaGraphDestroy(gpost);
    gpre = gpost = nullptr;
    L->graph = G;
    L->launches_fixed = (l1 - l0) + (l2 - l1);
    L->launches_round = l4 - l3;
    w->launches = l0; /* captured launches run at replay time; counted there */
    return GAT_OK;
}

/* Plain form through the query graph: queries [0, nq), one graph launch each. */
int topk_plain_graph(gat_ctx* ctx, const gat_index* g, int nq, const int32_t* d_q_len, const int64_t* d_q_off,
                     const float2* d_q_xy, int max_q_len, int k, float u, int32_t* d_ids, int32_t* d_dist, int64_t* stats) {
    LoneGraph* L = nullptr;
    int st = lone_graph_get(ctx, g, max_q_len, k, u, &L);
    if (st != GAT_OK) return st;
    gat_ctx* w = L->w;
    cudaStream_t s = w->stream;
    /* the worker's stream starts after the caller's work on the context stream */
    GAT_CUDA_TRY(ctx, cudaEventRecord(L->ev, ctx->stream), "top-k");
    GAT_CUDA_TRY(ctx, cudaStreamWaitEvent(s, L->ev, 0), "top-k");
    StageDesc* hd = reinterpret_cast<StageDesc*>(w->h_pinned);
    *hd = StageDesc{d_q_len, d_q_off, d_q_xy, d_ids, d_dist, nq, max_q_len};
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(L->d_desc, hd, sizeof(StageDesc), cudaMemcpyHostToDevice, s), "top-k");
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(L->d_next, 0, sizeof(int), s), "top-k");
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(L->acc, 0, 3 * sizeof(unsigned long long), s), "top-k");
    const int64_t lw0 = w->launches;
    int first = 0;
    if (!L->exec) {
        if ((st = lone_build(L)) != GAT_OK) {
            /* leave no half-built graph behind; the error names the failing step */
            std::string msg = w->err;
            for (auto it = ctx->owned.begin(); it != ctx->owned.end(); ++it)
                if (it->first == L) {
                    ctx->owned.erase(it);
                    break;
                }
            lone_graph_free(L);
            return fail(ctx, st, "top-k graph: " + msg);
        }
        first = 1;
    }
    for (int q = first; q < nq; q++) GAT_CUDA_TRY(ctx, cudaGraphLaunch(L->exec, s), "top-k graph launch");
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(w->h_pinned + 8, L->acc, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s),
                 "top-k");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "top-k");
    if ((st = check_device_flag(w, "top-k")) != GAT_OK) return fail(ctx, st, w->err);
    const int64_t rounds = w->h_pinned[10];
    ctx->launches += (w->launches - lw0) + (int64_t)(nq - first) * L->launches_fixed + rounds * L->launches_round;
    if (stats) {
        stats[0] = w->h_pinned[9];
        stats[1] = w->h_pinned[8];
        stats[2] = 0;
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
    unsigned long long* acc = (unsigned long long*)scratch(ctx, S_TOPK_IO, 256, &st);
    if (!acc) return st;
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(acc, 0, 2 * sizeof(unsigned long long), ctx->stream), "top-k");
    if (exec == GAT_EXEC_BATCHED) {
        /* query batches sized so the per-batch candidate arrays stay below ~8 GiB */
        int bins = std::max(max_q_len, g->db->maxlen) + 2;
        int64_t per = std::max<int64_t>(1, ((int64_t)8 << 30) / (int64_t)topk_bytes_per_query(g->db->n, bins));
        for (int q0 = 0; q0 < nq && st == GAT_OK; q0 += (int)per) {
            int c = (int)std::min<int64_t>(per, nq - q0);
            st = topk_batch(ctx, g, c, d_q_len + q0, d_q_off + q0, d_q_xy, max_q_len, k, u, d_ids + (size_t)q0 * k,
                            d_dist + (size_t)q0 * k, local, acc);
        }
    } else if (!ctx->timing) {
        /* plain form: one query per launch of the query graph */
        st = topk_plain_graph(ctx, g, nq, d_q_len, d_q_off, d_q_xy, max_q_len, k, u, d_ids, d_dist, stats);
        if (st == GAT_OK && stats) stats[2] = ctx->launches - l0;
        return st;
    } else {
        /* plain form with per-kernel timing: the same kernels launched one by one */
        for (int qi = 0; qi < nq && st == GAT_OK; qi++)
            st = topk_batch(ctx, g, 1, d_q_len + qi, d_q_off + qi, d_q_xy, max_q_len, k, u, d_ids + (size_t)qi * k,
                            d_dist + (size_t)qi * k, local, acc);
    }
    if (st != GAT_OK) return st;
    /* one read for the whole call: counters, then the device status word */
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_pinned + 6, acc, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                      ctx->stream), "top-k");
    if ((st = check_device_flag(ctx, "top-k")) != GAT_OK) return st;
    timed_add_work(ctx, GAT_KERNEL_EDR, (double)ctx->h_pinned[6]);
    if (stats) {
        stats[0] = ctx->h_pinned[7];
        stats[1] = ctx->h_pinned[6];
        stats[2] = ctx->launches - l0;
    }
    return GAT_OK;
}

int check_grid(gat_ctx* ctx, const gat_index* g) {
    if (!g || g->kind != GAT_INDEX_GRID) return fail(ctx, GAT_ERR_STATE, "top-k needs a Grid index (it holds the FVTable)");
    if (!same_owner(g->ctx, ctx)) return fail(ctx, GAT_ERR_STATE, "index from another context");
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
    /* the offsets are built here: copied from pinned staging, not from pageable memory */
    int64_t* hoff = (int64_t*)host_stage(ctx, (size_t)(nq + 1) * 8, &st);
    if (!hoff) return st;
    std::copy(h.off.begin(), h.off.begin() + (nq + 1), hoff);
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(*doff, hoff, (size_t)(nq + 1) * 8, cudaMemcpyHostToDevice, s), "top-k H2D");
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
    st = topk_batch(ctx, grid, nq, dl, doff, dxy, h.maxlen, 1, match_threshold(1e-9), nullptr, nullptr, stats, nullptr);
    if (st != GAT_OK) return st;
    int n = grid->db->n;
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(out, ctx->slot_ptr[S_TOPK_LB], (size_t)nq * (n + 1) * 4, cudaMemcpyDeviceToHost, ctx->stream), "bounds D2H");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "bounds");
    return GAT_OK;
}

}  // extern "C"
