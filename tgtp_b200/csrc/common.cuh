// Device-side building blocks shared by the SABA and AESC kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tgtp {

constexpr unsigned kFullMask = 0xffffffffu;

// MurmurHash3 fmix32: the vertex hash of the primary SABA phase
// (src/aesc.h:31-41, src/rw_experiment_saba.cpp:44-51).
__host__ __device__ __forceinline__ uint32_t fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// SplitMix32 with the 16/15/15 mixer: the fallback generator (src/aesc.h:23-30).
__host__ __device__ __forceinline__ uint32_t splitmix32(uint32_t& state) {
    state += 0x9e3779b9u;
    uint32_t z = state;
    z = (z ^ (z >> 16)) * 0x21f0aaadu;
    z = (z ^ (z >> 15)) * 0x735a2d97u;
    return z ^ (z >> 15);
}

// Correctly rounded arithmetic that the compiler never contracts into FMA, in both precisions.
// The reference is compiled under ISO C++ (no contraction); every operation of the parity forms
// goes through these so that each rounding happens where the reference's does.
__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }

template <class R> __device__ __forceinline__ R from_u64(uint64_t x);
template <> __device__ __forceinline__ float from_u64<float>(uint64_t x) { return __ull2float_rn(x); }
template <> __device__ __forceinline__ double from_u64<double>(uint64_t x) { return __ull2double_rn(x); }
template <class R> __device__ __forceinline__ R from_f64(double x);
template <> __device__ __forceinline__ float from_f64<float>(double x) { return __double2float_rn(x); }
template <> __device__ __forceinline__ double from_f64<double>(double x) { return x; }

// std::max / std::min as the reference calls them: (a < b) ? b : a and (b < a) ? b : a.
template <class T> __device__ __forceinline__ T std_max(T a, T b) { return a < b ? b : a; }
template <class T> __device__ __forceinline__ T std_min(T a, T b) { return b < a ? b : a; }

// double -> int32 with the x86-64 cvttsd2si result for out-of-range values and NaN (INT32_MIN),
// which is what the reference's implicit conversion produces on its target.
__device__ __forceinline__ int x86_f64_to_i32(double t) {
    if (!(t > -2147483649.0 && t < 2147483648.0)) return (int)0x80000000;
    return (int)t;
}

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* __restrict__ a, uint32_t lo,
                                                    uint32_t hi, uint32_t key) {
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (__ldg(a + mid) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

}  // namespace tgtp
