/*
 * TEST INFRASTRUCTURE ONLY — the CPU oracle.  Nothing in the product (tgtp_b200/, include/) links,
 * loads or calls this; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg do,
 * and only as the checker.
 *
 * A plain-C restatement of the reference's hot path:
 *   - SABA one-way walk counter        src/rw_experiment_saba.cpp:65-145 (integer counters)
 *   - MT19937 walk baselines           src/rw_experiment.cpp:34-47, rw_experiment_simd.cpp:44-83
 *   - calculate_taus / get_tau /
 *     get_delta / get_upsilon          src/aesc.h:129-216
 *   - tgtp_baseline (push, stop test,
 *     edge max, chi, 2-way walks,
 *     symmetrisation)                  src/aesc.h:218-551
 * in two precisions: the reference's own FP32 arithmetic (bit-exact with the reference built at
 * -O2) and the plain FP64 form (every float of the reference held in double).
 *
 * Parity pin: tests/test_oracle_golden.py compares this against golden vectors produced by the
 * reference compiled from its own sources (oracle/Makefile, tests/golden/make_golden.py).
 */
#ifndef TGTP_ORACLE_H
#define TGTP_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint64_t push_rounds;        /* sum over sources of the final ell            */
    uint64_t push_vertices;      /* frontier vertices drained by diffuse         */
    uint64_t push_traversals;    /* adjacency entries visited by diffuse         */
    uint64_t walk_edges;         /* CSR slots that ran the 2-way walk            */
    uint64_t walk_count;         /* sum of nr over those slots                   */
    uint64_t walk_hops;          /* sum of nr * rest_ell (pairs of hops)         */
    uint64_t fallback_bouquets;  /* bouquets that entered the SplitMix32 phase   */
    uint64_t tau_iterations;     /* get_delta evaluations in calculate_taus      */
} oracle_stats;

/* SABA counters: counters[v] = visits of v over all sources (start vertex not counted). */
int oracle_saba(const uint32_t* idx, const uint32_t* adj, uint64_t n, uint32_t depth,
                uint32_t n_walks, uint64_t* counters, int threads);

/* The k-th draw (1-based) of std::mt19937 seeded with `seed` (known answer: seed 5489, k 10000
 * gives 4123659995, the C++ standard's check value). */
uint32_t oracle_mt19937_nth(uint32_t seed, uint64_t k);

/* MT19937 walk baselines src/rw_experiment.cpp:34-47 (simd = 0) and
 * src/rw_experiment_simd.cpp:44-83 (simd = 1), integer counters; -1 if simd and n_walks % 8. */
int oracle_mt_walks(const uint32_t* idx, const uint32_t* adj, uint64_t n, uint32_t depth,
                    uint32_t n_walks, int simd, uint64_t* counters, int threads);

/* Per-CSR-slot walk-length bound tau (src/aesc.h:164-216), epsilon = eps/2 as the caller passes. */
int oracle_taus_f32(const uint32_t* idx, const uint32_t* adj, uint64_t n, const double* values,
                    const float* vectors, int omega, double eps, int* taus, oracle_stats* st,
                    int threads);
int oracle_taus_f64(const uint32_t* idx, const uint32_t* adj, uint64_t n, const double* values,
                    const double* vectors, int omega, double eps, int* taus, oracle_stats* st,
                    int threads);

/*
 * Full tgtp(): scores[m] (symmetric, float32, CSR order).  Optional outputs (may be NULL):
 *   taus[m], ell[n] (push rounds per source), presym[m] (scores before symmetrisation),
 *   nr[m] (walk count per slot, 0 when no walk ran).
 * vectors are vertex-major: vectors[v*omega + i].
 */
int oracle_tgtp_f32(const uint32_t* idx, const uint32_t* adj, uint64_t n, const double* values,
                    const float* vectors, int omega, double eps, double delta, int gamma,
                    float* scores, int* taus, int* ell, float* presym, uint64_t* nr,
                    oracle_stats* st, int threads);
int oracle_tgtp_f64(const uint32_t* idx, const uint32_t* adj, uint64_t n, const double* values,
                    const double* vectors, int omega, double eps, double delta, int gamma,
                    float* scores, int* taus, int* ell, double* presym, uint64_t* nr,
                    oracle_stats* st, int threads);

/* sorted_eigens_<omega>.txt -> values[omega], vectors vertex-major (either pointer may be NULL). */
int oracle_parse_eigens(const char* path, uint64_t n, int omega, double* values, float* vec_f32,
                        double* vec_f64);

/* 2-way walk estimator for one (src, v) pair with a caller-given residual vector. */
float oracle_walk2_f32(const uint32_t* idx, const uint32_t* adj, uint32_t src, uint32_t v,
                       uint64_t num_walk, uint32_t len_walk, const float* pvec);

#ifdef __cplusplus
}
#endif
#endif
