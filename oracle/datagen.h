/* Seeded synthetic workloads (oracle/datagen.cpp). TEST INFRASTRUCTURE ONLY: the same arrays as
 * the library's generator, produced without loading the library. */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_LEN_UNIFORM = 0, ORC_LEN_LOGNORMAL = 1, ORC_LEN_LOGUNIFORM = 2 };
enum { ORC_SIDE_FIXED = 0, ORC_SIDE_LOGUNIFORM = 1 };

/* n lengths: uniform integers in [lo, hi], round(exp(N(p0, p1))) or round(log-uniform(lo, hi)),
 * clipped to [lo, hi] */
void orc_gen_lengths(int n, int kind, double p0, double p1, int lo, int hi, uint64_t seed, int32_t* out);
/* clamped random walks in box (xmin, ymin, xmax, ymax): start uniform, N(0, step) increments */
void orc_gen_walks(int n, const int32_t* lengths, const float box[4], double step, uint64_t seed, float* lon,
                   float* lat);
/* rectangles with centres uniform in box, side s0 or log-uniform in [s0, s1] per axis */
void orc_gen_boxes(int n, int kind, double s0, double s1, const float box[4], uint64_t seed, float* out4);
/* k distinct ids of 1..n in draw order */
void orc_gen_sample_ids(int k, int n, uint64_t seed, int32_t* out);
/* EDR pairs: A a walk, B A's path resampled to B's length plus N(0, jitter) noise */
void orc_gen_pairs(int n, const int32_t* len_a, const int32_t* len_b, const float box[4], double step, double jitter,
                   uint64_t seed, float* a_xy, float* b_xy);

#ifdef __cplusplus
}
#endif
