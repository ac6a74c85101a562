/*
 * Test infrastructure only: force-included (-include) when the reference's
 * own sources are compiled into oracle/_ref/ as the CPU checker.
 *
 * The reference calls one Intel SVML intrinsic, _mm256_rem_epu32
 * (src/aesc.h:353-354, src/rw_experiment_saba.cpp:125), which GCC does not
 * provide.  Its documented meaning is the lane-wise unsigned 32-bit remainder
 * a % b over eight lanes; this is a plain scalar statement of that meaning.
 */
#ifndef TGTP_ORACLE_SHIM_H
#define TGTP_ORACLE_SHIM_H
#include <immintrin.h>
#include <stdint.h>

static inline __m256i _mm256_rem_epu32(__m256i a, __m256i b) {
    uint32_t x[8] __attribute__((aligned(32)));
    uint32_t y[8] __attribute__((aligned(32)));
    _mm256_store_si256((__m256i*)x, a);
    _mm256_store_si256((__m256i*)y, b);
    for (int lane = 0; lane < 8; ++lane) x[lane] = x[lane] % y[lane];
    return _mm256_load_si256((const __m256i*)x);
}
#endif
