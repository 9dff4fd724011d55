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
    extern __shared__ int hist[];
    __shared__ int sh_W, cnt;
    int qi = blockIdx.x;
    int32_t* s = ws + (size_t)qi * WS_WORDS;
    if (s[WS_DONE]) return;
    const int end = s[WS_END];
    const int32_t* dist = sdist + (size_t)qi * n;
    for (int i = threadIdx.x; i < bins; i += blockDim.x) hist[i] = 0;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < end; i += blockDim.x) atomicAdd(&hist[min(dist[i], bins - 1)], 1);
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
        sh_W = W;
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
                        const int32_t* ws, int32_t* out_ids, int32_t* out_dist, int32_t* flag) {
    extern __shared__ uint32_t bm_s[];
    __shared__ unsigned long long lt_keys[1024];
    __shared__ int lt_n;
    __shared__ int warp_cnt[kT / 32 + 1];
    int qi = blockIdx.x;
    uint32_t* bm = gbitmap ? gbitmap + (size_t)blockIdx.x * words : bm_s;
    const int32_t* s = ws + (size_t)qi * WS_WORDS;
    if (threadIdx.x == 0 && !s[WS_DONE]) atomicCAS(flag, 0, GAT_ERR_STATE);
    const int W = s[WS_W], end = s[WS_END];
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

int read_word(gat_ctx* ctx, const void* d, int64_t* v) {
    GAT_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_pinned, d, 8, cudaMemcpyDeviceToHost, ctx->stream), "top-k");
    GAT_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "top-k");
    *v = ctx->h_pinned[0];
    return GAT_OK;
}

/* device bytes topk_batch needs per query (sorted candidates, bounds, distances, histograms) */
size_t topk_bytes_per_query(int n, int bins) {
    int ntile = (n + kSortTile - 1) / kSortTile;
    return (size_t)(n + 1) * 4 + (size_t)n * 12 + (size_t)bins * ntile * 8 + 64;
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
    size_t smem_fv = (size_t)pow2 * 12;
    allow_smem(k_query_fv, smem_fv);
    k_query_fv<<<std::min(nq, ctx->sm_count * 4), 512, smem_fv, s>>>(g->grid, nq, d_q_len, d_q_off, d_q_xy, stride, pow2,
                                                                      qfv_cell, qfv_cnt, qfv_n);
    count_launch(ctx);
    /* lower bounds */
    int32_t* lb = (int32_t*)scratch(ctx, S_TOPK_LB, (size_t)nq * (n + 1) * 4, &st);
    if (!lb) return st;
    int vbits = (int)std::log2((double)(g->grid.cellnum >> 2));
    int nwords = ((1 << vbits) + 31) / 32;
    uint32_t* near = (uint32_t*)scratch(ctx, S_TOPK_NEAR, (size_t)nq * nwords * 4 + 64, &st);
    if (!near) return st;
    k_near_bitmap<<<nq, kT, 0, s>>>(nq, vbits, qfv_cell, qfv_n, stride, nwords, near);
    count_launch(ctx);
    size_t smem_lb = (size_t)stride * 8;
    allow_smem(k_lower_bounds, smem_lb);
    dim3 lgrid((n + kT - 1) / kT, nq);
    timed_begin(ctx, GAT_KERNEL_BOUNDS);
    k_lower_bounds<<<lgrid, kT, smem_lb, s>>>(n, nq, g->d_fv_off, g->d_fv_cell, g->d_fv_cnt, qfv_cell, qfv_cnt, qfv_n, stride,
                                             vbits, near, nwords, d_q_len, lb, ctx->d_flag);
    /* algorithmic bytes: every trajectory's FV (8 B per entry + 8 B offset) and its bound (4 B)
     * per query */
    timed_end(ctx, GAT_KERNEL_BOUNDS, (double)nq * ((double)g->fv_entries * 8.0 + (double)n * 12.0));
    count_launch(ctx);
    if (stats && stats[3] == -1) { /* bounds only */
        return check_device_flag(ctx, "frequency-vector bounds");
    }
    /* candidate order */
    int bins_lb = std::max(max_q_len, db->maxlen) + 2;
    int ntile = (n + kSortTile - 1) / kSortTile;
    int64_t* H = (int64_t*)scratch(ctx, S_TOPK_SEG, (size_t)nq * bins_lb * ntile * 8 + 64, &st);
    char* sorted = (char*)scratch(ctx, S_TOPK_PAIRS, (size_t)nq * n * 12 + 1024, &st);
    int32_t* ws = (int32_t*)scratch(ctx, S_TOPK_QSTATE, (size_t)nq * WS_WORDS * 4 + (size_t)(nq + 1) * 4 + 256, &st);
    unsigned long long* cells = (unsigned long long*)scratch(ctx, S_TOPK_IO, 256, &st);
    if (!H || !sorted || !ws || !cells) return st;
    int32_t* cand = (int32_t*)sorted;
    int32_t* slb = cand + (size_t)nq * n;
    int32_t* sdist = slb + (size_t)nq * n;
    int* wprefix = (int*)(ws + (size_t)nq * WS_WORDS);
    size_t smem_h = (size_t)bins_lb * 4;
    allow_smem(k_sort_hist, smem_h);
    k_sort_hist<<<dim3(ntile, nq), kT, smem_h, s>>>(n, lb, bins_lb, ntile, H);
    count_launch(ctx);
    if ((st = scan_i64(ctx, H, H, (int64_t)nq * bins_lb * ntile)) != GAT_OK) return st;
    size_t smem_run = (size_t)bins_lb * 8;
    allow_smem(k_sort_scatter, smem_run);
    k_sort_scatter<<<dim3(ntile, nq), 32, smem_run, s>>>(n, lb, bins_lb, ntile, H, cand, slb);
    count_launch(ctx);
    /* the walk: a finished query costs nothing in later rounds, `rounds` covers the whole
     * order with growing chunks, and the loop ends early once no query extends */
    /* a lone query leaves most of the GPU idle in a small round, so it starts with a larger
     * chunk and grows faster; a batch keeps rounds tight to limit surplus evaluations */
    const bool lone = nq <= 4;
    int chunk0 = lone ? std::max(8 * k, 1024) : std::max(4 * k, 128);
    int growth = lone ? 4 : 2;
    int rounds = 1;
    for (int64_t cover = chunk0, c = chunk0; cover < n; rounds++) {
        c *= growth;
        cover += c;
    }
    rounds += 1;
    GAT_CUDA_TRY(ctx, cudaMemsetAsync(cells, 0, 8, s), "top-k");
    k_walk_init<<<(nq + 127) / 128, 128, 0, s>>>(nq, chunk0, ws);
    count_launch(ctx);
    int bins_d = max_q_len + db->maxlen + 2;
    size_t smem_d = (size_t)bins_d * 4;
    allow_smem(k_walk_kth, smem_d);
    int rows_hint = std::min(max_q_len, db->maxlen);
    int max_cols = std::max(max_q_len, db->maxlen);
    WalkPairs src{n, nq, wprefix, ws, cand, d_q_len, d_q_off, d_q_xy, db->d_len, db->d_off, db->d_xy, sdist};
    for (int r = 0; r < rounds; r++) {
        k_walk_plan<<<1, 1024, 0, s>>>(n, nq, slb, ws, wprefix);
        count_launch(ctx);
        /* the round's pair count sizes the EDR launch exactly; it is zero once no query can
         * extend (every query at the end of its order or with its next bound above W) */
        int32_t* cnt = reinterpret_cast<int32_t*>(ctx->h_pinned + 4);
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(cnt, wprefix + nq, sizeof(int32_t), cudaMemcpyDeviceToHost, s), "top-k");
        GAT_CUDA_TRY(ctx, cudaStreamSynchronize(s), "top-k");
        const int64_t npairs = *cnt;
        if (npairs == 0) break;
        if ((st = edr::edr_launch(ctx, src, npairs, rows_hint, max_cols, u, cells)) != GAT_OK) return st;
        k_walk_kth<<<nq, kT, smem_d, s>>>(n, k, bins_d, growth, slb, cand, sdist, ws);
        count_launch(ctx);
    }
    /* selection */
    int words = (n + 1 + 31) / 32;
    uint32_t* gbm = nullptr;
    size_t smem_final = (size_t)words * 4;
    if (smem_final > 160 * 1024) {
        gbm = (uint32_t*)scratch(ctx, S_TOPK_DIST, (size_t)nq * words * 4, &st);
        if (!gbm) return st;
        smem_final = 0;
    } else {
        allow_smem(k_final, smem_final);
    }
    k_final<<<nq, kT, smem_final, s>>>(n, k, words, gbm, cand, sdist, ws, d_ids, d_dist, ctx->d_flag);
    count_launch(ctx);
    GAT_CUDA_TRY(ctx, cudaGetLastError(), "top-k launch");
    if (stats || ctx->timing) {
        /* pairs evaluated = sum of the evaluated prefixes */
        std::vector<int32_t> h((size_t)nq * WS_WORDS);
        GAT_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), ws, h.size() * 4, cudaMemcpyDeviceToHost, s), "top-k");
        int64_t c = 0;
        if ((st = read_word(ctx, cells, &c)) != GAT_OK) return st;
        timed_add_work(ctx, GAT_KERNEL_EDR, (double)c);
        if (stats) {
            for (int q = 0; q < nq; q++) stats[0] += h[(size_t)q * WS_WORDS + WS_END];
            stats[1] += c;
        }
    }
    return check_device_flag(ctx, "top-k");
}

int topk_dev(gat_ctx* ctx, const gat_index* g, int nq, const int32_t* d_q_len, const int64_t* d_q_off,
             const float2* d_q_xy, int max_q_len, int k, double eps, int exec, int32_t* d_ids, int32_t* d_dist,
             int64_t* stats) {
    float u = match_threshold(eps);
    int64_t l0 = ctx->launches;
    int64_t local[4] = {0, 0, 0, 0};
    int st = GAT_OK;
    if (exec == GAT_EXEC_BATCHED) {
        /* query batches sized so the per-batch candidate arrays stay below ~8 GiB */
        int bins = std::max(max_q_len, g->db->maxlen) + 2;
        int64_t per = std::max<int64_t>(1, ((int64_t)8 << 30) / (int64_t)topk_bytes_per_query(g->db->n, bins));
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
