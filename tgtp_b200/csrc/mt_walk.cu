// The reference's MT19937 walk baselines on sm_100a with exact uint32 visit counters:
//   scalar  src/rw_experiment.cpp:34-47      walk i, hop j takes draw i * depth + j
//   simd    src/rw_experiment_simd.cpp:44-83 bouquet b (walks 8b .. 8b+7) steps together; hop j
//                                            of lane l takes draw 8 b depth + 8 j + l
// from every vertex with a neighbour, with std::mt19937 reseeded to 42 + src per source
// (src/rw_experiment.cpp:110) and k = draw % degree(cur) per hop.  They are the comparison rows of
// the walk experiment (not the SABA walk): same counters as the reference's routines, integer
// instead of float.
//
// Layout.  One warp per source (grid-stride over the sources).  The generator is the Mersenne
// Twister of Matsumoto & Nishimura (ACM TOMACS 8(1), 1998) with the C++ standard's seeding.  Its
// 624-word state lives in shared memory as a ring of two generations: generation t (t = 0 the
// seeded state, t >= 1 the state after t regenerations, whose tempered words are draws
// 624 (t-1) .. 624 t - 1) sits in half t & 1.  Generation t + 1 is built from t into the other
// half by the 32 lanes together: word i needs old words i and i + 1 and either old word i + 397
// (i < 227) or new word i - 227 -- at least 227 places back, so 32 consecutive words never depend
// on one another.  The lanes walk side by side, one walk each (scalar) or one bouquet per 8 lanes
// (simd), so that the draws one hop of all active lanes takes span at most 624 consecutive numbers:
// they then lie in the two generations the ring holds.
#include <algorithm>

#include "common.cuh"
#include "internal.hpp"

namespace tgtp {
namespace {

constexpr uint32_t kMtWords = 624;
constexpr uint32_t kMtShift = 397;
constexpr int kMtThreads = 256;
constexpr int kMtWarps = kMtThreads / 32;

__device__ __forceinline__ uint32_t mt_temper(uint32_t y) {
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

// Generation 0 (the seeding recurrence is sequential: lane 0 alone).
__device__ __forceinline__ void mt_seed(uint32_t* ring, uint32_t seed, uint32_t lane) {
    __syncwarp();
    if (lane == 0) {
        uint32_t x = seed;
        ring[0] = x;
        for (uint32_t i = 1; i < kMtWords; ++i) {
            x = 1812433253u * (x ^ (x >> 30)) + i;
            ring[i] = x;
        }
    }
    __syncwarp();
}

// Generation t + 1 from generation t, all lanes of the warp.
__device__ __forceinline__ void mt_regenerate(uint32_t* ring, uint32_t t, uint32_t lane) {
    const uint32_t* o = ring + (t & 1u) * kMtWords;
    uint32_t* w = ring + ((t + 1u) & 1u) * kMtWords;
    for (uint32_t c = 0; c < kMtWords; c += 32) {
        const uint32_t i = c + lane;
        if (i < kMtWords) {
            const uint32_t nx = i + 1 < kMtWords ? o[i + 1] : w[0];
            const uint32_t y = (o[i] & 0x80000000u) | (nx & 0x7fffffffu);
            const uint32_t far = i + kMtShift < kMtWords ? o[i + kMtShift] : w[i + kMtShift - kMtWords];
            w[i] = far ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        __syncwarp();
    }
}

template <bool SIMD>
__global__ void __launch_bounds__(kMtThreads)
mt_walk_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ adj, uint64_t n,
               uint32_t depth, uint32_t n_walks, uint32_t* __restrict__ cnt) {
    __shared__ uint32_t s_ring[kMtWarps][2 * kMtWords];
    const uint32_t lane = threadIdx.x & 31;
    uint32_t* ring = s_ring[threadIdx.x >> 5];
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    // a group is one walk (scalar) or one bouquet of 8 walks (simd); it takes `per` draws a hop
    const uint32_t per = SIMD ? 8u : 1u;
    const uint64_t gdraws = uint64_t(per) * depth;  // draws of one group's whole walk
    const uint32_t groups = n_walks / per;
    // groups side by side: the draws of one hop span (G - 1) * gdraws + per <= 624 numbers
    uint32_t G = SIMD ? 4u : 32u;
    if (gdraws > 0 && (kMtWords - per) / gdraws + 1 < G) G = uint32_t((kMtWords - per) / gdraws + 1);
    const uint32_t grp = SIMD ? lane >> 3 : lane, sub = SIMD ? lane & 7u : 0u;
    for (uint64_t src = warp; src < n; src += nwarps) {
        if (__ldg(idx + src + 1) == __ldg(idx + src)) continue;  // isolated (warp-uniform)
        mt_seed(ring, 42u + uint32_t(src), lane);
        uint64_t gen = 0;  // newest generation in the ring (the one before it sits in the other half)
        for (uint32_t g0 = 0; g0 < groups; g0 += G) {
            const uint32_t gact = min(G, groups - g0);
            const bool active = grp < gact;
            const uint64_t base = (uint64_t(g0) + grp) * gdraws + sub;
            const uint64_t top = (uint64_t(g0) + gact - 1) * gdraws + (per - 1);
            uint32_t cur = uint32_t(src);
            for (uint32_t j = 0; j < depth; ++j) {
                // the hop's largest draw decides the newest generation needed (warp-uniform); its
                // smallest is less than 624 before, so within the generation before
                const uint64_t kmax = top + uint64_t(j) * per;
                while (gen < kmax / kMtWords + 1) {
                    mt_regenerate(ring, uint32_t(gen), lane);
                    ++gen;
                }
                if (active) {
                    const uint64_t k = base + uint64_t(j) * per;
                    const uint32_t t = uint32_t(k / kMtWords) + 1u;
                    const uint32_t r = mt_temper(ring[(t & 1u) * kMtWords + uint32_t(k % kMtWords)]);
                    const uint32_t rb = __ldg(idx + cur);
                    const uint32_t d = __ldg(idx + cur + 1) - rb;
                    cur = __ldg(adj + rb + r % d);
                    atomicAdd(cnt + cur, 1u);
                }
            }
        }
    }
}

}  // namespace

void mt_walk_run(tgtp_graph* g, uint32_t depth, uint32_t n_walks, bool simd,
                 uint32_t* device_counters) {
    cudaStream_t s = g->stream;
    g->sums.reserve(4 * sizeof(unsigned long long));
    TGTP_CUDA(cudaMemsetAsync(device_counters, 0, sizeof(uint32_t) * g->n, s));
    TGTP_CUDA(cudaMemsetAsync(g->sums.ptr, 0, 4 * sizeof(unsigned long long), s));
    if (n_walks == 0 || depth == 0 || g->n == 0) return;
    const void* kern = simd ? reinterpret_cast<const void*>(mt_walk_kernel<true>)
                            : reinterpret_cast<const void*>(mt_walk_kernel<false>);
    int per_sm = 0;
    TGTP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kMtThreads, 0));
    uint64_t blocks = uint64_t(g->num_sms) * std::max(per_sm, 1);
    blocks = std::min<uint64_t>(blocks, (g->n + kMtWarps - 1) / kMtWarps);
    ScopedKernel k(g->prof, s, "mt_walk");
    if (simd)
        mt_walk_kernel<true><<<unsigned(blocks), kMtThreads, 0, s>>>(
            g->idx.as<uint32_t>(), g->adj.as<uint32_t>(), g->n, depth, n_walks, device_counters);
    else
        mt_walk_kernel<false><<<unsigned(blocks), kMtThreads, 0, s>>>(
            g->idx.as<uint32_t>(), g->adj.as<uint32_t>(), g->n, depth, n_walks, device_counters);
    TGTP_LAUNCH_CHECK("mt_walk_kernel");
}

}  // namespace tgtp
