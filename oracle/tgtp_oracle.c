/*
 * TEST INFRASTRUCTURE ONLY — the CPU oracle (see tgtp_oracle.h).  Never linked into the product.
 *
 * Build: make -C oracle restatement  (gcc -std=c11 -O2 -ffp-contract=off: ISO C evaluation of every
 * float expression in its own type, no FMA contraction, matching the reference built at -O2).
 */
#define _POSIX_C_SOURCE 200809L
#include "tgtp_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define RWRATIO 25 /* src/aesc.h:17 */

/* MurmurHash3 fmix32, src/aesc.h:31-41 and src/rw_experiment_saba.cpp:44-51. */
static inline uint32_t fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

/* SplitMix32 (16/15/15), src/aesc.h:23-30 and src/rw_experiment_saba.cpp:54-61. */
static inline uint32_t splitmix32(uint32_t* state) {
    *state += 0x9e3779b9u;
    uint32_t z = *state;
    z = (z ^ (z >> 16)) * 0x21f0aaadu;
    z = (z ^ (z >> 15)) * 0x735a2d97u;
    return z ^ (z >> 15);
}

/* std::max / std::min on doubles and reals: (a < b) ? b : a and (b < a) ? b : a. */
static inline double max_d(double a, double b) { return a < b ? b : a; }
#define MAXR(a, b) ((a) < (b) ? (b) : (a))
#define MINR(a, b) ((b) < (a) ? (b) : (a))

/* double -> int32 as x86-64 cvttsd2si does it: out-of-range and NaN give INT32_MIN. */
static inline int x86_f64_to_i32(double t) {
    if (!(t > -2147483649.0 && t < 2147483648.0)) return INT32_MIN;
    return (int)t;
}

/* std::lower_bound over adj[lo, hi) */
static inline uint64_t lower_bound_u32(const uint32_t* adj, uint64_t lo, uint64_t hi, uint32_t key) {
    while (lo < hi) {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (adj[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

/*
 * SABA one-way walk counter, src/rw_experiment_saba.cpp:65-145, with integer counters.  Lane j of
 * the bouquet starting at walk ii gets the grid seed (ii + j + 1) * floor((2^32-1)/W) (:71-79);
 * the primary phase hashes the current vertex and keeps the high 32 bits of r * degree (:83-115),
 * the whole bouquet falls back to SplitMix32 % degree once any lane's secret is zero (:117-143).
 */
static void saba_source(const uint32_t* idx, const uint32_t* adj, uint32_t src, uint32_t len_walk,
                        uint32_t n_walk, uint64_t* cnt) {
    if (n_walk == 0) return;
    const uint32_t grid_step = UINT32_MAX / n_walk;
    for (uint64_t ii = 0; ii < n_walk; ii += 8) {
        uint32_t cur[8], secret[8], state[8];
        for (int j = 0; j < 8; ++j) {
            cur[j] = src;
            secret[j] = ((uint32_t)ii + (uint32_t)(j + 1)) * grid_step;
            state[j] = secret[j];
        }
        uint32_t len = 0;
        for (; len < len_walk; len++) {
            int any_zero = 0;
            for (int j = 0; j < 8; ++j) any_zero |= secret[j] == 0;
            if (any_zero) break;
            for (int j = 0; j < 8; ++j) {
                const uint32_t d = idx[cur[j] + 1] - idx[cur[j]];
                const uint32_t r = secret[j] ^ fmix32(cur[j]);
                const uint32_t k = (uint32_t)(((uint64_t)r * d) >> 32);
                cur[j] = adj[idx[cur[j]] + k];
                secret[j] *= d;
                cnt[cur[j]]++;
            }
        }
        for (; len < len_walk; len++) {
            for (int j = 0; j < 8; ++j) {
                const uint32_t r = splitmix32(&state[j]);
                const uint32_t d = idx[cur[j] + 1] - idx[cur[j]];
                cur[j] = adj[idx[cur[j]] + r % d];
                cnt[cur[j]]++;
            }
        }
    }
}

int oracle_saba(const uint32_t* idx, const uint32_t* adj, uint64_t n, uint32_t depth,
                uint32_t n_walks, uint64_t* counters, int threads) {
    if (n_walks % 8 != 0) return -1;
    memset(counters, 0, sizeof(uint64_t) * n);
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
    {
        uint64_t* local = (uint64_t*)calloc(n, sizeof(uint64_t));
#pragma omp for schedule(dynamic, 256)
        for (long long src = 0; src < (long long)n; ++src) {
            if (idx[src + 1] == idx[src]) continue;
            saba_source(idx, adj, (uint32_t)src, depth, n_walks, local);
        }
#pragma omp critical
        for (uint64_t v = 0; v < n; ++v) counters[v] += local[v];
        free(local);
    }
    return 0;
}

/*
 * std::mt19937, restated from Matsumoto & Nishimura, "Mersenne Twister: a 623-dimensionally
 * equidistributed uniform pseudo-random number generator" (ACM TOMACS 8(1), 1998), with the C++
 * standard's seeding (x_0 = seed, x_i = 1812433253 * (x_{i-1} ^ (x_{i-1} >> 30)) + i) and its
 * tempering.  The reference's MT19937 walk runners draw from it (src/rw_experiment.cpp:39-47,
 * src/rw_experiment_simd.cpp:54-59).
 */
typedef struct {
    uint32_t x[624];
    int next;
} mt19937_state;

static void mt19937_seed(mt19937_state* s, uint32_t seed) {
    s->x[0] = seed;
    for (uint32_t i = 1; i < 624; ++i) s->x[i] = 1812433253u * (s->x[i - 1] ^ (s->x[i - 1] >> 30)) + i;
    s->next = 624;
}

static uint32_t mt19937_draw(mt19937_state* s) {
    if (s->next >= 624) {
        for (int i = 0; i < 624; ++i) {
            const uint32_t y = (s->x[i] & 0x80000000u) | (s->x[(i + 1) % 624] & 0x7fffffffu);
            s->x[i] = s->x[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        s->next = 0;
    }
    uint32_t y = s->x[s->next++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

uint32_t oracle_mt19937_nth(uint32_t seed, uint64_t k) {
    mt19937_state s;
    mt19937_seed(&s, seed);
    uint32_t y = 0;
    for (uint64_t i = 0; i < k; ++i) y = mt19937_draw(&s);
    return y;
}

/*
 * The reference's MT19937 walk baselines with integer counters: every source with a neighbour
 * reseeds the generator with 42 + src (src/rw_experiment.cpp:110) and makes n_walks walks of
 * exactly depth hops, each hop k = draw % degree(cur) (:39-47).  simd = 0: walk-major order (the
 * scalar runner); simd = 1: bouquets of 8 walks stepping together, the 8 draws of a hop taken in
 * lane order (src/rw_experiment_simd.cpp:44-83, n_walks a multiple of 8).  counters[v] = visits
 * of v (start vertices not counted).
 */
int oracle_mt_walks(const uint32_t* idx, const uint32_t* adj, uint64_t n, uint32_t depth,
                    uint32_t n_walks, int simd, uint64_t* counters, int threads) {
    if (simd && n_walks % 8 != 0) return -1;
    memset(counters, 0, sizeof(uint64_t) * n);
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
    {
        uint64_t* local = (uint64_t*)calloc(n, sizeof(uint64_t));
        mt19937_state rng;
#pragma omp for schedule(dynamic, 256)
        for (long long src = 0; src < (long long)n; ++src) {
            if (idx[src + 1] == idx[src]) continue;
            mt19937_seed(&rng, 42u + (uint32_t)src);
            if (!simd) {
                for (uint32_t i = 0; i < n_walks; ++i) {
                    uint32_t cur = (uint32_t)src;
                    for (uint32_t len = 0; len < depth; ++len) {
                        const uint32_t k = mt19937_draw(&rng) % (idx[cur + 1] - idx[cur]);
                        cur = adj[idx[cur] + k];
                        local[cur]++;
                    }
                }
            } else {
                for (uint32_t ii = 0; ii < n_walks; ii += 8) {
                    uint32_t cur[8];
                    for (int l = 0; l < 8; ++l) cur[l] = (uint32_t)src;
                    for (uint32_t len = 0; len < depth; ++len) {
                        uint32_t r[8];
                        for (int l = 0; l < 8; ++l) r[l] = mt19937_draw(&rng);
                        for (int l = 0; l < 8; ++l)
                            cur[l] = adj[idx[cur[l]] + r[l] % (idx[cur[l] + 1] - idx[cur[l]])];
                        for (int l = 0; l < 8; ++l) local[cur[l]]++;
                    }
                }
            }
        }
#pragma omp critical
        for (uint64_t v = 0; v < n; ++v) counters[v] += local[v];
        free(local);
    }
    return 0;
}

/* k-th largest value (1-based, counting multiplicity) by quickselect; destroys a[]. */
#define DEFINE_KTH(T, NAME)                                                              \
    static T NAME(T* a, uint64_t size, uint64_t k) {                                     \
        if (k == 0 || size == 0) return 0;                                               \
        int64_t lo = 0, hi = (int64_t)size - 1;                                          \
        const int64_t want = (int64_t)k - 1; /* index in descending order */             \
        while (lo < hi) {                                                                \
            const T pivot = a[lo + (hi - lo) / 2];                                       \
            int64_t i = lo, j = hi;                                                      \
            while (i <= j) {                                                             \
                while (a[i] > pivot) i++;                                                \
                while (a[j] < pivot) j--;                                                \
                if (i <= j) {                                                            \
                    T t = a[i]; a[i] = a[j]; a[j] = t;                                   \
                    i++;                                                                 \
                    j--;                                                                 \
                }                                                                        \
            }                                                                            \
            /* now a[lo..j] >= pivot >= a[i..hi] and a[j+1..i-1] == pivot */            \
            if (want <= j) hi = j;                                                       \
            else if (want >= i) lo = i;                                                  \
            else return a[want];                                                         \
        }                                                                                \
        return a[want];                                                                  \
    }
DEFINE_KTH(float, kth_largest_f32)
DEFINE_KTH(double, kth_largest_f64)

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)

/* ---- the reference's own arithmetic: FP32 residuals and eigenvectors ---- */
#define REAL float
#define VEC float
#define FN(name) CAT(name, _f32)
#include "tgtp_oracle_body.inc"
#undef REAL
#undef VEC
#undef FN

/* ---- plain FP64 form ---- */
#define REAL double
#define VEC double
#define FN(name) CAT(name, _f64)
#define SPLIT_SUMS 1
#include "tgtp_oracle_body.inc"
#undef REAL
#undef VEC
#undef FN

float oracle_walk2_f32(const uint32_t* idx, const uint32_t* adj, uint32_t src, uint32_t v,
                       uint64_t num_walk, uint32_t len_walk, const float* pvec) {
    uint64_t fb = 0;
    return walk2_f32(idx, adj, src, v, num_walk, len_walk, pvec, &fb);
}

/*
 * sorted_eigens_<omega>.txt parser with the reference's semantics (src/aesc.h:51-64): omega rows of
 * "lambda x_0 .. x_{n-1}" stored vertex-major, each eigenvector token parsed straight to float
 * (istream >> float is strtof, not strtod-then-round) and, for the FP64 form, to double.
 */
int oracle_parse_eigens(const char* path, uint64_t n, int omega, double* values, float* vec_f32,
                        double* vec_f64) {
    FILE* f = fopen(path, "rb");
    if (!f) return -1;
    fseek(f, 0, SEEK_END);
    long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    char* buf = (char*)malloc((size_t)size + 1);
    if (!buf || fread(buf, 1, (size_t)size, f) != (size_t)size) {
        fclose(f);
        free(buf);
        return -1;
    }
    fclose(f);
    buf[size] = 0;
    char* p = buf;
    int rc = 0;
    for (int i = 0; i < omega && rc == 0; ++i) {
        char* end;
        values[i] = strtod(p, &end);
        if (end == p || !isfinite(values[i])) { rc = -2; break; }
        p = end;
        for (uint64_t j = 0; j < n; ++j) {
            char* e1;
            char* e2;
            const float xf = strtof(p, &e1);
            const double xd = strtod(p, &e2);
            if (e1 == p || !isfinite(xf) || !isfinite(xd)) { rc = -2; break; }
            if (vec_f32) vec_f32[j * (uint64_t)omega + i] = xf;
            if (vec_f64) vec_f64[j * (uint64_t)omega + i] = xd;
            p = e2;
        }
    }
    free(buf);
    return rc;
}
