/*
 * qaf_init.h — the seeded initial-condition generator shared by every party
 * that must start from bit-identical fields: the CUDA library, the FP64 host
 * oracle, the driver around the reference's own CUDA build, and the Python
 * tests (which restate the same arithmetic in numpy).
 *
 * The reference reads its initial Q tensor from CSV files or fills it with
 * libc rand() (InertialFriction/friction/friction.cu:21-41, :164-185); neither
 * is reproducible across machines, so every workload here is seeded instead.
 *
 * Generator: SplitMix64. The k-th draw (k = 0, 1, ...) of a stream seeded with
 * `seed` is mix(seed + (k + 1) * 0x9E3779B97F4A7C15), where mix is the
 * SplitMix64 finaliser. It is turned into a double in [0, 1) from its top 53
 * bits, then mapped to [lo, hi) as lo + (hi - lo) * u.
 *
 * The "random Q" initial state draws N*N values for r1 = Q11 in the physical
 * order i + j*N (x fastest, the reference's layout), then N*N values for
 * r2 = Q12 from the same stream; omega is zero.
 *
 * The "coupled" initial state is the smooth one of the reference's coupled
 * runs (UnitTest/TimeIntegration/couple/couple.cu:4-35): omega = 0,
 * r1 = 0.2 (sin^2(x+y) - 1/2) + amp u, r2 = 0.2 sin(x+y) cos(x+y) + amp u',
 * x = i lx/nx, y = j ly/ny, with u, u' ~ U(0, 1) from this stream (draws
 * i + j nx and nx ny + i + j nx) in place of rand()/RAND_MAX; amp = 1e-3
 * there.
 */
#ifndef QAF_INIT_H
#define QAF_INIT_H

#include <math.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

static inline uint64_t qaf_splitmix64_at(uint64_t seed, uint64_t k) {
    uint64_t z = seed + (k + 1u) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline double qaf_uniform_at(uint64_t seed, uint64_t k, double lo, double hi) {
    double u = (double)(qaf_splitmix64_at(seed, k) >> 11) * (1.0 / 9007199254740992.0);
    return lo + (hi - lo) * u;
}

/* Fill out[0..n) with draws first..first+n-1 of the stream, mapped to [lo, hi). */
static inline void qaf_fill_uniform(uint64_t seed, uint64_t first, double lo, double hi,
                                    double* out, size_t n) {
    for (size_t i = 0; i < n; ++i) out[i] = qaf_uniform_at(seed, first + i, lo, hi);
}

/* Random-Q initial state on an nx*ny grid: r1 ~ U(lo,hi), r2 ~ U(lo,hi), w = 0.
 * Any output pointer may be NULL. */
static inline void qaf_random_q_init(uint64_t seed, int nx, int ny, double lo, double hi,
                                     double* w, double* r1, double* r2) {
    size_t n = (size_t)nx * (size_t)ny;
    if (w) for (size_t i = 0; i < n; ++i) w[i] = 0.0;
    if (r1) qaf_fill_uniform(seed, 0, lo, hi, r1, n);
    if (r2) qaf_fill_uniform(seed, n, lo, hi, r2, n);
}

/* Coupled-run initial state (see the header comment). Any output pointer may be NULL. */
static inline void qaf_couple_init(uint64_t seed, int nx, int ny, double lx, double ly, double amp,
                                   double* w, double* r1, double* r2) {
    size_t n = (size_t)nx * (size_t)ny;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            size_t k = (size_t)i + (size_t)j * (size_t)nx;
            double s = sin(i * (lx / nx) + j * (ly / ny)), c = cos(i * (lx / nx) + j * (ly / ny));
            if (w) w[k] = 0.0;
            if (r1) r1[k] = 0.2 * (s * s - 0.5) + amp * qaf_uniform_at(seed, k, 0.0, 1.0);
            if (r2) r2[k] = 0.2 * s * c + amp * qaf_uniform_at(seed, n + k, 0.0, 1.0);
        }
}

#ifdef __cplusplus
}
#endif
#endif /* QAF_INIT_H */
