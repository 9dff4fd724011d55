/* Seeded synthetic inputs: random-walk trajectories, query rectangles, EDR pair sets.
 *
 * The reference loads a taxi trajectory file that is not available (main.cpp:121); every
 * workload here is generated instead. Each trajectory, rectangle and pair draws from its own
 * SplitMix64 stream keyed by (seed, purpose, index), so the output does not depend on the
 * number of host threads used to produce it. Positions are accumulated in double and stored
 * as float32 (the reference's SamplePoint holds floats, SamplePoint.h:11-12). */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "gat_b200.h"

namespace {

inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t s;
    bool has_spare = false;
    double spare = 0.0;
    Rng(uint64_t seed, uint64_t purpose, uint64_t index)
        : s(mix64(seed * 0x9E3779B97F4A7C15ULL ^ mix64(purpose + 0x632BE59BD9B4E019ULL) ^
                  mix64(index * 0xD1B54A32D192ED03ULL + 1))) {}
    uint64_t next() {
        s += 0x9E3779B97F4A7C15ULL;
        return mix64(s);
    }
    /* uniform in [0, 1) with 53 random bits */
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    /* standard normal, Box-Muller */
    double normal() {
        if (has_spare) {
            has_spare = false;
            return spare;
        }
        double u1 = uniform(), u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        double r = std::sqrt(-2.0 * std::log(u1));
        double t = 6.283185307179586 * u2;
        spare = r * std::sin(t);
        has_spare = true;
        return r * std::cos(t);
    }
};

enum : uint64_t { P_LEN = 1, P_WALK = 2, P_BOX = 3, P_SAMPLE = 4, P_PAIR = 5 };

template <class F>
void parallel_for(int64_t n, F f) {
    unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 4096 || hw == 1) {
        for (int64_t i = 0; i < n; i++) f(i);
        return;
    }
    std::vector<std::thread> th;
    int64_t per = (n + hw - 1) / hw;
    for (unsigned t = 0; t < hw; t++) {
        int64_t s = t * per, e = std::min(n, s + per);
        if (s >= e) break;
        th.emplace_back([=]() {
            for (int64_t i = s; i < e; i++) f(i);
        });
    }
    for (auto& x : th) x.join();
}

inline double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

int draw_length(Rng& r, int kind, double p0, double p1, int lo, int hi) {
    double v;
    switch (kind) {
        case GAT_LEN_UNIFORM:
            return lo + (int)std::floor(r.uniform() * (double)(hi - lo + 1));
        case GAT_LEN_LOGNORMAL:
            v = std::exp(p0 + p1 * r.normal());
            break;
        case GAT_LEN_LOGUNIFORM:
            v = std::exp(std::log((double)lo) + r.uniform() * (std::log((double)hi) - std::log((double)lo)));
            break;
        default:
            return lo;
    }
    long iv = std::lround(v);
    return (int)std::min<long>(hi, std::max<long>(lo, iv));
}

/* One clamped random walk: start uniform in the box, N(0, step) per axis per step. */
void walk(Rng& r, int len, const float box[4], double step, float* lon, float* lat) {
    double x = box[0] + r.uniform() * (double)(box[2] - box[0]);
    double y = box[1] + r.uniform() * (double)(box[3] - box[1]);
    for (int i = 0; i < len; i++) {
        if (i > 0) {
            x = clampd(x + step * r.normal(), box[0], box[2]);
            y = clampd(y + step * r.normal(), box[1], box[3]);
        }
        lon[i] = (float)x;
        lat[i] = (float)y;
    }
}

}  // namespace

extern "C" {

int gat_gen_lengths(int n, int kind, double p0, double p1, int lo, int hi, uint64_t seed, int32_t* out) {
    if (n < 0 || lo < 1 || hi < lo || !out) return GAT_ERR_ARG;
    parallel_for(n, [&](int64_t i) {
        Rng r(seed, P_LEN, (uint64_t)i);
        out[i] = draw_length(r, kind, p0, p1, lo, hi);
    });
    return GAT_OK;
}

int gat_gen_walks(int n, const int32_t* lengths, const float box[4], double step, uint64_t seed,
                  float* lon, float* lat) {
    if (n < 0 || !lengths || !lon || !lat) return GAT_ERR_ARG;
    std::vector<int64_t> off(n + 1, 0);
    for (int i = 0; i < n; i++) off[i + 1] = off[i] + lengths[i];
    parallel_for(n, [&](int64_t i) {
        Rng r(seed, P_WALK, (uint64_t)i);
        walk(r, lengths[i], box, step, lon + off[i], lat + off[i]);
    });
    return GAT_OK;
}

int gat_gen_boxes(int n, int kind, double s0, double s1, const float box[4], uint64_t seed, float* out4) {
    if (n < 0 || !out4 || s0 <= 0) return GAT_ERR_ARG;
    parallel_for(n, [&](int64_t i) {
        Rng r(seed, P_BOX, (uint64_t)i);
        double cx = box[0] + r.uniform() * (double)(box[2] - box[0]);
        double cy = box[1] + r.uniform() * (double)(box[3] - box[1]);
        double w = s0, h = s0;
        if (kind == GAT_SIDE_LOGUNIFORM) {
            w = std::exp(std::log(s0) + r.uniform() * (std::log(s1) - std::log(s0)));
            h = std::exp(std::log(s0) + r.uniform() * (std::log(s1) - std::log(s0)));
        }
        out4[4 * i + 0] = (float)(cx - 0.5 * w);
        out4[4 * i + 1] = (float)(cy - 0.5 * h);
        out4[4 * i + 2] = (float)(cx + 0.5 * w);
        out4[4 * i + 3] = (float)(cy + 0.5 * h);
    });
    return GAT_OK;
}

int gat_gen_sample_ids(int k, int n, uint64_t seed, int32_t* out) {
    /* k distinct ids from 1..n, in draw order (partial Fisher-Yates) */
    if (k < 0 || k > n || !out) return GAT_ERR_ARG;
    std::vector<int32_t> v(n);
    for (int i = 0; i < n; i++) v[i] = i + 1;
    Rng r(seed, P_SAMPLE, 0);
    for (int i = 0; i < k; i++) {
        int j = i + (int)(r.uniform() * (double)(n - i));
        if (j >= n) j = n - 1;
        std::swap(v[i], v[j]);
        out[i] = v[i];
    }
    return GAT_OK;
}

int gat_gen_pairs(int n, const int32_t* len_a, const int32_t* len_b, const float box[4], double step,
                  double jitter, uint64_t seed, float* a_xy, float* b_xy) {
    /* Pair i: A is a clamped random walk; B follows A's path resampled to B's length, with
     * N(0, jitter) noise per coordinate, so that points of the two match within eps often. */
    if (n < 0 || !len_a || !len_b || !a_xy || !b_xy) return GAT_ERR_ARG;
    std::vector<int64_t> oa(n + 1, 0), ob(n + 1, 0);
    for (int i = 0; i < n; i++) {
        oa[i + 1] = oa[i] + len_a[i];
        ob[i + 1] = ob[i] + len_b[i];
    }
    parallel_for(n, [&](int64_t i) {
        Rng r(seed, P_PAIR, (uint64_t)i);
        int la = len_a[i], lb = len_b[i];
        std::vector<float> x(la), y(la);
        walk(r, la, box, step, x.data(), y.data());
        float* A = a_xy + 2 * oa[i];
        float* B = b_xy + 2 * ob[i];
        for (int j = 0; j < la; j++) {
            A[2 * j] = x[j];
            A[2 * j + 1] = y[j];
        }
        for (int j = 0; j < lb; j++) {
            int s = (int)(((int64_t)j * la) / lb);
            B[2 * j] = (float)clampd((double)x[s] + jitter * r.normal(), box[0], box[2]);
            B[2 * j + 1] = (float)clampd((double)y[s] + jitter * r.normal(), box[1], box[3]);
        }
    });
    return GAT_OK;
}

}  // extern "C"
