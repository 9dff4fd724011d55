/* Seeded synthetic workloads for the test oracles and the CPU baseline. TEST INFRASTRUCTURE ONLY.
 *
 * The reference measures on a taxi trajectory file that is not available (main.cpp:121), so every
 * workload is generated. This file produces exactly the arrays the library's generator produces
 * (same streams, same arithmetic; tests/test_datagen.py compares them array for array), so that
 * the CPU baseline of the reference and the oracle can build their inputs without loading the
 * library: the compiled reference (oracle/_ref/gatref) links this file, and oracle/liboracle.so
 * exports it to Python.
 *
 * Streams: every trajectory, rectangle, length and pair draws from its own SplitMix64 sequence
 * keyed by (seed, purpose, index), so the output does not depend on the thread count. Uniforms
 * take the top 53 bits; normals come from the Box-Muller transform in pairs (cosine first, the
 * sine kept for the next draw). Positions accumulate in double and are stored as float32. */
#include "datagen.h"

#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

namespace {

constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ULL;

uint64_t finalize(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

enum Purpose : uint64_t { kLengths = 1, kWalk = 2, kRect = 3, kSample = 4, kPair = 5 };

class Stream {
   public:
    Stream(uint64_t seed, uint64_t purpose, uint64_t index) {
        state_ = finalize(seed * kGolden ^ finalize(purpose + 0x632BE59BD9B4E019ULL) ^
                          finalize(index * 0xD1B54A32D192ED03ULL + 1));
    }
    double uniform() {
        state_ += kGolden;
        return (double)(finalize(state_) >> 11) * (1.0 / 9007199254740992.0);
    }
    double normal() {
        if (spare_ok_) {
            spare_ok_ = false;
            return spare_;
        }
        double a = uniform();
        const double b = uniform();
        if (a < 1e-300) a = 1e-300;
        const double radius = std::sqrt(-2.0 * std::log(a));
        const double angle = 6.283185307179586 * b;
        spare_ = radius * std::sin(angle);
        spare_ok_ = true;
        return radius * std::cos(angle);
    }

   private:
    uint64_t state_;
    double spare_ = 0.0;
    bool spare_ok_ = false;
};

/* f(i) for i in [0, n) on up to 32 host threads (contiguous slices) */
template <class F>
void each(int64_t n, F f) {
    const int64_t hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 4096 || hw == 1) {
        for (int64_t i = 0; i < n; i++) f(i);
        return;
    }
    std::vector<std::thread> pool;
    const int64_t per = (n + hw - 1) / hw;
    for (int64_t s = 0; s < n; s += per)
        pool.emplace_back([=]() {
            for (int64_t i = s; i < std::min(n, s + per); i++) f(i);
        });
    for (auto& t : pool) t.join();
}

double clamp(double v, double lo, double hi) { return std::min(hi, std::max(lo, v)); }

int one_length(Stream& r, int kind, double p0, double p1, int lo, int hi) {
    if (kind == ORC_LEN_UNIFORM) return lo + (int)std::floor(r.uniform() * (double)(hi - lo + 1));
    double v;
    if (kind == ORC_LEN_LOGNORMAL)
        v = std::exp(p0 + p1 * r.normal());
    else if (kind == ORC_LEN_LOGUNIFORM)
        v = std::exp(std::log((double)lo) + r.uniform() * (std::log((double)hi) - std::log((double)lo)));
    else
        return lo;
    return (int)std::min<long>(hi, std::max<long>(lo, std::lround(v)));
}

/* a clamped walk: start uniform in the box, then N(0, step) per axis per point */
void one_walk(Stream& r, int len, const float box[4], double step, float* lon, float* lat) {
    double x = box[0] + r.uniform() * (double)(box[2] - box[0]);
    double y = box[1] + r.uniform() * (double)(box[3] - box[1]);
    for (int i = 0; i < len; i++) {
        if (i > 0) {
            x = clamp(x + step * r.normal(), box[0], box[2]);
            y = clamp(y + step * r.normal(), box[1], box[3]);
        }
        lon[i] = (float)x;
        lat[i] = (float)y;
    }
}

std::vector<int64_t> prefix(int n, const int32_t* len) {
    std::vector<int64_t> off(n + 1, 0);
    for (int i = 0; i < n; i++) off[i + 1] = off[i] + len[i];
    return off;
}

}  // namespace

extern "C" {

void orc_gen_lengths(int n, int kind, double p0, double p1, int lo, int hi, uint64_t seed, int32_t* out) {
    each(n, [&](int64_t i) {
        Stream r(seed, kLengths, (uint64_t)i);
        out[i] = one_length(r, kind, p0, p1, lo, hi);
    });
}

void orc_gen_walks(int n, const int32_t* lengths, const float box[4], double step, uint64_t seed, float* lon,
                   float* lat) {
    const std::vector<int64_t> off = prefix(n, lengths);
    each(n, [&](int64_t i) {
        Stream r(seed, kWalk, (uint64_t)i);
        one_walk(r, lengths[i], box, step, lon + off[i], lat + off[i]);
    });
}

void orc_gen_boxes(int n, int kind, double s0, double s1, const float box[4], uint64_t seed, float* out4) {
    each(n, [&](int64_t i) {
        Stream r(seed, kRect, (uint64_t)i);
        const double cx = box[0] + r.uniform() * (double)(box[2] - box[0]);
        const double cy = box[1] + r.uniform() * (double)(box[3] - box[1]);
        double w = s0, h = s0;
        if (kind == ORC_SIDE_LOGUNIFORM) {
            w = std::exp(std::log(s0) + r.uniform() * (std::log(s1) - std::log(s0)));
            h = std::exp(std::log(s0) + r.uniform() * (std::log(s1) - std::log(s0)));
        }
        float* o = out4 + 4 * i;
        o[0] = (float)(cx - 0.5 * w);
        o[1] = (float)(cy - 0.5 * h);
        o[2] = (float)(cx + 0.5 * w);
        o[3] = (float)(cy + 0.5 * h);
    });
}

void orc_gen_sample_ids(int k, int n, uint64_t seed, int32_t* out) {
    std::vector<int32_t> ids(n);
    for (int i = 0; i < n; i++) ids[i] = i + 1;
    Stream r(seed, kSample, 0);
    for (int i = 0; i < k; i++) {
        const int j = std::min(n - 1, i + (int)(r.uniform() * (double)(n - i)));
        std::swap(ids[i], ids[j]);
        out[i] = ids[i];
    }
}

void orc_gen_pairs(int n, const int32_t* len_a, const int32_t* len_b, const float box[4], double step, double jitter,
                   uint64_t seed, float* a_xy, float* b_xy) {
    const std::vector<int64_t> oa = prefix(n, len_a), ob = prefix(n, len_b);
    each(n, [&](int64_t i) {
        Stream r(seed, kPair, (uint64_t)i);
        const int la = len_a[i], lb = len_b[i];
        std::vector<float> x(la), y(la);
        one_walk(r, la, box, step, x.data(), y.data());
        float* A = a_xy + 2 * oa[i];
        float* B = b_xy + 2 * ob[i];
        for (int j = 0; j < la; j++) {
            A[2 * j] = x[j];
            A[2 * j + 1] = y[j];
        }
        /* B follows A's path resampled to B's length, with N(0, jitter) noise per coordinate */
        for (int j = 0; j < lb; j++) {
            const int s = (int)(((int64_t)j * la) / lb);
            B[2 * j] = (float)clamp((double)x[s] + jitter * r.normal(), box[0], box[2]);
            B[2 * j + 1] = (float)clamp((double)y[s] + jitter * r.normal(), box[1], box[3]);
        }
    });
}

}  // extern "C"
