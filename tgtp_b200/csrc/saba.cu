// SABA walk counter on sm_100a: the one-way sampling-aware walk of src/rw_experiment_saba.cpp:65-145
// with exact uint32 visit counters.
//
// Layout and mapping.  The reference's unit is an 8-lane bouquet: lane j of the bouquet that starts
// at walk ii carries the ordered-grid seed (ii + j + 1) * floor((2^32-1)/W).  Here a warp runs four
// bouquets side by side (lanes 8g..8g+7 = bouquet g), so the "any lane's secret is zero" test of the
// reference (:83-85) is one warp ballot masked to the bouquet's byte.  Every bouquet makes exactly
// `depth` hops, so the work is uniform and each warp takes a contiguous, equal share of the
// n * W/8 bouquets; consecutive bouquets share their start row, which stays in L1.
//
// Per hop a lane loads idx[cur], idx[cur+1] and adj[idx[cur] + k] (the dependent chain) and bumps
// one counter with a fire-and-forget atomic that is off that chain.  Counters of vertex ids below
// `hot` live in shared memory per block (hubs have low ids in the power-law generators, and every
// id is hot when n is small) and are flushed once at the end; the rest go to L2 atomics.
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "internal.hpp"

namespace tgtp {
namespace {

constexpr int kSabaThreads = 512;
constexpr uint32_t kSabaHotCap = 12288;  // 48 KiB of shared counters per block

__global__ void __launch_bounds__(kSabaThreads)
saba_walk_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ adj,
                 uint32_t depth, uint32_t bouquets_per_src, uint32_t grid_step,
                 uint64_t total_bouquets, uint32_t* __restrict__ counters, uint32_t hot,
                 unsigned long long* __restrict__ fallback_total) {
    extern __shared__ uint32_t s_cnt[];
    for (uint32_t i = threadIdx.x; i < hot; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();

    const uint32_t lane = threadIdx.x & 31;
    const uint32_t j = lane & 7;
    const uint32_t grp = lane >> 3;
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;

    // Contiguous share of bouquets for this warp, rounded to groups of four.
    const uint64_t groups = (total_bouquets + 3) / 4;
    const uint64_t g_lo = groups * warp / nwarps;
    const uint64_t g_hi = groups * (warp + 1) / nwarps;

    uint64_t b = g_lo * 4 + grp;  // this group's bouquet
    uint32_t src = uint32_t(b / bouquets_per_src);
    uint32_t bq = uint32_t(b - uint64_t(src) * bouquets_per_src);
    uint32_t fallbacks = 0;

    for (uint64_t gi = g_lo; gi < g_hi; ++gi) {
        bool active = b < total_bouquets;
        uint32_t beg = 0, d = 0, cur = src;
        if (active) {
            beg = __ldg(idx + src);
            d = __ldg(idx + src + 1) - beg;
            active = d != 0;  // isolated sources are skipped (src/rw_experiment_saba.cpp:197-198)
        }
        uint32_t secret = (bq * 8u + j + 1u) * grid_step;
        uint32_t state = secret;
        bool primary = true;
        for (uint32_t len = 0; len < depth; ++len) {
            const unsigned zero = __ballot_sync(kFullMask, active && primary && secret == 0u);
            if ((zero >> (grp * 8)) & 0xffu) primary = false;
            if (active) {
                uint32_t k;
                if (primary) {
                    k = __umulhi(secret ^ fmix32(cur), d);
                    secret *= d;
                } else {
                    k = splitmix32(state) % d;
                }
                cur = __ldg(adj + beg + k);
                beg = __ldg(idx + cur);
                d = __ldg(idx + cur + 1) - beg;
                if (cur < hot) atomicAdd(s_cnt + cur, 1u);
                else atomicAdd(counters + cur, 1u);
            }
        }
        if (active && !primary && j == 0) ++fallbacks;
        // advance this group by four bouquets
        b += 4;
        bq += 4;
        while (bq >= bouquets_per_src) {
            bq -= bouquets_per_src;
            ++src;
        }
    }

    __syncthreads();
    for (uint32_t i = threadIdx.x; i < hot; i += blockDim.x) {
        const uint32_t c = s_cnt[i];
        if (c) atomicAdd(counters + i, c);
    }
    // fallback statistics
    uint32_t f = fallbacks;
#pragma unroll
    for (int o = 16; o; o >>= 1) f += __shfl_xor_sync(kFullMask, f, o);
    if (lane == 0 && f) atomicAdd(fallback_total, (unsigned long long)f);
}

// ---- walk graph renumbered by degree ---------------------------------------------------------------
// A walk visits a vertex in proportion to its degree, so the counters that take most increments
// belong to the highest-degree vertices.  saba_count renumbers the vertices by degree (highest
// first, ties by id) into a walk copy of the graph: row p holds the neighbours of vertex orig(p) in
// their original order, renumbered, and info[p] = (row start, degree, orig(p), 0) is one 16-byte
// load per hop.  The hash of the primary phase and the neighbour index k are taken on the original
// ids and orders, so every trajectory is the reference's; the counters of the first `hot` numbers
// live in shared memory, and the per-number counters are scattered back to the original ids at the
// end.
__global__ void saba_iota_kernel(uint32_t* __restrict__ ids, uint64_t n) {
    for (uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
         v += uint64_t(gridDim.x) * blockDim.x)
        ids[v] = uint32_t(v);
}

__global__ void saba_info_kernel(const uint32_t* __restrict__ order, const uint32_t* __restrict__ sdeg,
                                 const uint32_t* __restrict__ beg, uint64_t n,
                                 uint4* __restrict__ info, uint32_t* __restrict__ inv) {
    for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
         p += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t old = order[p];
        info[p] = make_uint4(beg[p], sdeg[p], old, 0u);
        inv[old] = uint32_t(p);
    }
}

__global__ void saba_adj_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ adj,
                                const uint32_t* __restrict__ row_of,
                                const uint32_t* __restrict__ inv, const uint4* __restrict__ info,
                                uint64_t m, uint32_t* __restrict__ adjp) {
    for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < m;
         q += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t old = row_of[q];
        const uint32_t p = inv[old];
        adjp[info[p].x + (uint32_t(q) - idx[old])] = inv[adj[q]];
    }
}

__global__ void saba_scatter_kernel(const uint32_t* __restrict__ cnt, const uint4* __restrict__ info,
                                    uint64_t n, uint32_t* __restrict__ counters) {
    for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < n;
         p += uint64_t(gridDim.x) * blockDim.x)
        counters[info[p].z] = cnt[p];
}

// The walk on the renumbered graph.  Each lane carries WPL walkers (bouquets 4w + g of the warp's
// step, g = lane / 8) whose hops are interleaved, so WPL independent load chains are in flight per
// lane.  A warp takes a contiguous, equal share of the steps (4 WPL bouquets each).
// The row records of the first `hot_rec` numbers (the highest degrees, which take most hops: on
// R-MAT scale 18 the top 2,048 / 4,096 vertices hold 38 % / 52 % of the degree mass) are copied
// into shared memory, so a hop that lands there makes one random L1/L2 load instead of two.
// Shared memory: hot_rec 12-byte records (three arrays), then `hot` 4-byte counters
// (hot_rec <= hot <= n).
template <int WPL>
__global__ void __launch_bounds__(kSabaThreads)
saba_walk_perm_kernel(const uint4* __restrict__ info, const uint32_t* __restrict__ adjp,
                      uint32_t depth, uint32_t bouquets_per_src, uint32_t grid_step,
                      uint64_t total_bouquets, uint32_t* __restrict__ cnt, uint32_t hot,
                      uint32_t hot_rec, unsigned long long* __restrict__ fallback_total) {
    // the records as three arrays (row start, degree, original id: 12 bytes a vertex), then the
    // counters
    extern __shared__ uint32_t s_words[];
    uint32_t* s_beg = s_words;
    uint32_t* s_deg = s_beg + hot_rec;
    uint32_t* s_org = s_deg + hot_rec;
    uint32_t* s_cnt = s_org + hot_rec;
    for (uint32_t i = threadIdx.x; i < hot_rec; i += blockDim.x) {
        const uint4 r = __ldg(info + i);
        s_beg[i] = r.x;
        s_deg[i] = r.y;
        s_org[i] = r.z;
    }
    for (uint32_t i = threadIdx.x; i < hot; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();

    const uint32_t lane = threadIdx.x & 31, j = lane & 7, grp = lane >> 3;
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    constexpr uint32_t SB = 4 * WPL;  // bouquets per warp step
    const uint64_t steps = (total_bouquets + SB - 1) / SB;
    const uint64_t s_lo = steps * warp / nwarps, s_hi = steps * (warp + 1) / nwarps;

    uint32_t src[WPL], bq[WPL];
#pragma unroll
    for (int w = 0; w < WPL; ++w) {
        const uint64_t b = s_lo * SB + uint32_t(w) * 4 + grp;
        src[w] = uint32_t(b / bouquets_per_src);
        bq[w] = uint32_t(b - uint64_t(src[w]) * bouquets_per_src);
    }
    uint32_t fallbacks = 0;
    for (uint64_t st = s_lo; st < s_hi; ++st) {
        bool active[WPL], primary[WPL];
        uint32_t beg[WPL], d[WPL], orig[WPL], secret[WPL], state[WPL];
#pragma unroll
        for (int w = 0; w < WPL; ++w) {
            const uint64_t b = st * SB + uint32_t(w) * 4 + grp;
            active[w] = b < total_bouquets;
            beg[w] = d[w] = orig[w] = 0;
            if (active[w]) {
                const uint4 r = __ldg(info + src[w]);
                beg[w] = r.x;
                d[w] = r.y;
                orig[w] = r.z;
                active[w] = r.y != 0;  // isolated sources are skipped (:197-198)
            }
            secret[w] = (bq[w] * 8u + j + 1u) * grid_step;
            state[w] = secret[w];
            primary[w] = true;
        }
        for (uint32_t len = 0; len < depth; ++len) {
            uint32_t nxt[WPL];
#pragma unroll
            for (int w = 0; w < WPL; ++w) {
                const unsigned zero =
                    __ballot_sync(kFullMask, active[w] && primary[w] && secret[w] == 0u);
                if ((zero >> (grp * 8)) & 0xffu) primary[w] = false;
            }
#pragma unroll
            for (int w = 0; w < WPL; ++w) {
                nxt[w] = 0;
                if (active[w]) {
                    uint32_t k;
                    if (primary[w]) {
                        k = __umulhi(secret[w] ^ fmix32(orig[w]), d[w]);
                        secret[w] *= d[w];
                    } else {
                        k = splitmix32(state[w]) % d[w];
                    }
                    nxt[w] = __ldg(adjp + beg[w] + k);
                }
            }
#pragma unroll
            for (int w = 0; w < WPL; ++w) {
                if (active[w]) {
                    if (nxt[w] < hot_rec) {
                        beg[w] = s_beg[nxt[w]];
                        d[w] = s_deg[nxt[w]];
                        orig[w] = s_org[nxt[w]];
                    } else {
                        const uint4 r = __ldg(info + nxt[w]);
                        beg[w] = r.x;
                        d[w] = r.y;
                        orig[w] = r.z;
                    }
                    if (nxt[w] < hot) atomicAdd(s_cnt + nxt[w], 1u);
                    else atomicAdd(cnt + nxt[w], 1u);
                }
            }
        }
#pragma unroll
        for (int w = 0; w < WPL; ++w) {
            if (active[w] && !primary[w] && j == 0) ++fallbacks;
            bq[w] += SB;
            while (bq[w] >= bouquets_per_src) {
                bq[w] -= bouquets_per_src;
                ++src[w];
            }
        }
    }

    __syncthreads();
    for (uint32_t i = threadIdx.x; i < hot; i += blockDim.x) {
        const uint32_t c = s_cnt[i];
        if (c) atomicAdd(cnt + i, c);
    }
    uint32_t f = fallbacks;
#pragma unroll
    for (int o = 16; o; o >>= 1) f += __shfl_xor_sync(kFullMask, f, o);
    if (lane == 0 && f) atomicAdd(fallback_total, (unsigned long long)f);
}

// ---- walk copy with the next row inlined in each slot ------------------------------------------------
// A hop of saba_walk_perm_kernel makes two dependent random loads: the chosen slot (the next vertex
// p) and then p's 16-byte row record.  In this copy, slot q of the renumbered adjacency holds the
// record of the vertex it points to: (row start, degree, fmix32(original id), p).  A hop is then one
// dependent 16-byte load; the counter update (p) stays off the dependent chain.  The copy takes
// 16 bytes per slot (4 x the plain renumbered adjacency).
__global__ void saba_adj16_kernel(const uint32_t* __restrict__ adjp, const uint4* __restrict__ info,
                                  uint64_t m, uint4* __restrict__ adj16) {
    for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < m;
         q += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t p = adjp[q];
        const uint4 r = info[p];
        adj16[q] = make_uint4(r.x, r.y, fmix32(r.z), p);
    }
}

// The walk over the inlined copy: trajectories, hashes and fallbacks exactly as
// saba_walk_perm_kernel (the hash of the primary phase is read precomputed from the slot).
template <int WPL>
__global__ void __launch_bounds__(kSabaThreads)
saba_walk_inline_kernel(const uint4* __restrict__ info, const uint4* __restrict__ adj16,
                        uint32_t depth, uint32_t bouquets_per_src, uint32_t grid_step,
                        uint64_t total_bouquets, uint32_t* __restrict__ cnt, uint32_t hot,
                        unsigned long long* __restrict__ fallback_total) {
    extern __shared__ uint32_t s_cnt[];
    for (uint32_t i = threadIdx.x; i < hot; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();

    const uint32_t lane = threadIdx.x & 31, j = lane & 7, grp = lane >> 3;
    const uint64_t warp = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    constexpr uint32_t SB = 4 * WPL;  // bouquets per warp step
    const uint64_t steps = (total_bouquets + SB - 1) / SB;
    const uint64_t s_lo = steps * warp / nwarps, s_hi = steps * (warp + 1) / nwarps;

    uint32_t src[WPL], bq[WPL];
#pragma unroll
    for (int w = 0; w < WPL; ++w) {
        const uint64_t b = s_lo * SB + uint32_t(w) * 4 + grp;
        src[w] = uint32_t(b / bouquets_per_src);
        bq[w] = uint32_t(b - uint64_t(src[w]) * bouquets_per_src);
    }
    uint32_t fallbacks = 0;
    for (uint64_t st = s_lo; st < s_hi; ++st) {
        bool active[WPL], primary[WPL];
        uint32_t beg[WPL], d[WPL], hsh[WPL], secret[WPL], state[WPL];
#pragma unroll
        for (int w = 0; w < WPL; ++w) {
            const uint64_t b = st * SB + uint32_t(w) * 4 + grp;
            active[w] = b < total_bouquets;
            beg[w] = d[w] = hsh[w] = 0;
            if (active[w]) {
                const uint4 r = __ldg(info + src[w]);
                beg[w] = r.x;
                d[w] = r.y;
                hsh[w] = fmix32(r.z);
                active[w] = r.y != 0;  // isolated sources are skipped (:197-198)
            }
            secret[w] = (bq[w] * 8u + j + 1u) * grid_step;
            state[w] = secret[w];
            primary[w] = true;
        }
        for (uint32_t len = 0; len < depth; ++len) {
#pragma unroll
            for (int w = 0; w < WPL; ++w) {
                const unsigned zero =
                    __ballot_sync(kFullMask, active[w] && primary[w] && secret[w] == 0u);
                if ((zero >> (grp * 8)) & 0xffu) primary[w] = false;
            }
#pragma unroll
            for (int w = 0; w < WPL; ++w) {
                if (active[w]) {
                    uint32_t k;
                    if (primary[w]) {
                        k = __umulhi(secret[w] ^ hsh[w], d[w]);
                        secret[w] *= d[w];
                    } else {
                        k = splitmix32(state[w]) % d[w];
                    }
                    const uint4 e = __ldg(adj16 + beg[w] + k);
                    beg[w] = e.x;
                    d[w] = e.y;
                    hsh[w] = e.z;
                    if (e.w < hot) atomicAdd(s_cnt + e.w, 1u);
                    else atomicAdd(cnt + e.w, 1u);
                }
            }
        }
#pragma unroll
        for (int w = 0; w < WPL; ++w) {
            if (active[w] && !primary[w] && j == 0) ++fallbacks;
            bq[w] += SB;
            while (bq[w] >= bouquets_per_src) {
                bq[w] -= bouquets_per_src;
                ++src[w];
            }
        }
    }

    __syncthreads();
    for (uint32_t i = threadIdx.x; i < hot; i += blockDim.x) {
        const uint32_t c = s_cnt[i];
        if (c) atomicAdd(cnt + i, c);
    }
    uint32_t f = fallbacks;
#pragma unroll
    for (int o = 16; o; o >>= 1) f += __shfl_xor_sync(kFullMask, f, o);
    if (lane == 0 && f) atomicAdd(fallback_total, (unsigned long long)f);
}

// visit_count = sum c[v], checksum = sum (v+1) c[v], both exact in 64 bits.
__global__ void saba_sums_kernel(const uint32_t* __restrict__ c, uint64_t n,
                                 unsigned long long* __restrict__ out) {
    unsigned long long s0 = 0, s1 = 0;
    for (uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
         v += uint64_t(gridDim.x) * blockDim.x) {
        const unsigned long long x = c[v];
        s0 += x;
        s1 += x * (v + 1);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        s0 += __shfl_xor_sync(kFullMask, s0, o);
        s1 += __shfl_xor_sync(kFullMask, s1, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out + 0, s0);
        atomicAdd(out + 1, s1);
    }
}

}  // namespace

// Builds the degree-renumbered walk copy of the graph once per handle.
void saba_prepare(tgtp_graph* g) {
    if (g->saba_ready) return;
    cudaStream_t s = g->stream;
    const uint64_t n = g->n, m = g->m;
    if (n > uint64_t(INT32_MAX) || m > uint64_t(UINT32_MAX))
        fail(TGTP_ERR_UNSUPPORTED, "graph too large for the walk counter");
    g->saba_info.reserve(sizeof(uint4) * (n + 1));
    g->saba_adj.reserve(sizeof(uint32_t) * (m + 1));
    DeviceBuffer ids, order, sdeg, beg, inv, tmp;
    ids.reserve(sizeof(uint32_t) * (n + 1));
    order.reserve(sizeof(uint32_t) * (n + 1));
    sdeg.reserve(sizeof(uint32_t) * (n + 1));
    beg.reserve(sizeof(uint32_t) * (n + 1));
    inv.reserve(sizeof(uint32_t) * (n + 1));
    const unsigned nb = unsigned(std::min<uint64_t>((n + 255) / 256, 8u * g->num_sms));
    saba_iota_kernel<<<nb ? nb : 1, 256, 0, s>>>(ids.as<uint32_t>(), n);
    TGTP_LAUNCH_CHECK("saba_iota_kernel");
    size_t t1 = 0, t2 = 0;
    TGTP_CUDA(cub::DeviceRadixSort::SortPairsDescending(
        nullptr, t1, g->deg.as<uint32_t>(), sdeg.as<uint32_t>(), ids.as<uint32_t>(),
        order.as<uint32_t>(), int(n), 0, 32, s));
    TGTP_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t2, sdeg.as<uint32_t>(), beg.as<uint32_t>(),
                                            int(n), s));
    tmp.reserve(std::max(t1, t2));
    TGTP_CUDA(cub::DeviceRadixSort::SortPairsDescending(
        tmp.ptr, t1, g->deg.as<uint32_t>(), sdeg.as<uint32_t>(), ids.as<uint32_t>(),
        order.as<uint32_t>(), int(n), 0, 32, s));
    TGTP_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, t2, sdeg.as<uint32_t>(), beg.as<uint32_t>(),
                                            int(n), s));
    saba_info_kernel<<<nb ? nb : 1, 256, 0, s>>>(order.as<uint32_t>(), sdeg.as<uint32_t>(),
                                                 beg.as<uint32_t>(), n, g->saba_info.as<uint4>(),
                                                 inv.as<uint32_t>());
    TGTP_LAUNCH_CHECK("saba_info_kernel");
    if (m) {
        const unsigned mb = unsigned(std::min<uint64_t>((m + 255) / 256, 8u * g->num_sms));
        saba_adj_kernel<<<mb, 256, 0, s>>>(g->idx.as<uint32_t>(), g->adj.as<uint32_t>(),
                                           g->row_of.as<uint32_t>(), inv.as<uint32_t>(),
                                           g->saba_info.as<uint4>(), m, g->saba_adj.as<uint32_t>());
        TGTP_LAUNCH_CHECK("saba_adj_kernel");
    }
    TGTP_CUDA(cudaStreamSynchronize(s));  // the temporaries go back to the cache
    g->saba_ready = true;
}

// Whether saba_count walks the inlined copy (one dependent 16-byte load per hop) or the plain
// renumbered copy (two): the tuned choice (saba_tune), else TGTP_SABA_INLINE=0/1, else the inlined
// copy while its 16 bytes per slot stay within 48 MB.  Walks are random, so the copies are read
// from L2: on the 4,039-vertex graph (2.8 MB inlined) the inlined copy measured 1.5x the plain
// one; on R-MAT scale 18 (122 MB inlined against 33 MB plain, beside a 126 MB L2) it measured
// 0.8x, the inlined copy no longer fitting.  saba_tune may still try it up to 2 GiB.
bool saba_inline_fits(const tgtp_graph* g) { return g->m * sizeof(uint4) <= (size_t(2) << 30); }

bool saba_use_inline(const tgtp_graph* g) {
    if (g->saba_choice) return (g->saba_choice & 0x100) != 0;
    if (const char* e = std::getenv("TGTP_SABA_INLINE")) return std::atoi(e) != 0;
    return g->m * sizeof(uint4) <= size_t(48) << 20;
}

// Row records of the plain walk copy kept in shared memory (the highest-degree numbers): the tuned
// choice (saba_tune: 1,024 x bits 12-14 of the choice), else TGTP_SABA_HOT_REC, else 4,096.
// Shared memory and L1 share 256 KB per SM: with the default 12,288 counters, 4,096 records of
// 12 bytes make a 96 KB block, two of which leave 60 KB of L1 for the walk copy.  On R-MAT scale 18
// (D 5 / 10 / 15, W 2,048 / 16,384): 3,072 records (as 16-byte records, the same block size)
// measured 1.09-1.11x 2,048 and 1.06-1.28x no records with one walker per lane; 4,096 12-byte
// records 1.03-1.04x 3,072; any split that left under 32 KB of L1 (three 72 KB blocks, or two of
// 102-104 KB) lost about a third.
uint32_t saba_hot_records(const tgtp_graph* g) {
    if (g->saba_choice) return 1024u * ((g->saba_choice >> 12) & 7u);
    if (const char* e = std::getenv("TGTP_SABA_HOT_REC"))
        return uint32_t(std::max(0, std::min(std::atoi(e), 8192)));
    return 4096u;
}

void saba_prepare_inline(tgtp_graph* g) {
    if (g->saba_inline_ready) return;
    saba_prepare(g);
    cudaStream_t s = g->stream;
    g->saba_adj16.reserve(sizeof(uint4) * (g->m + 1));
    if (g->m) {
        const unsigned mb = unsigned(std::min<uint64_t>((g->m + 255) / 256, 8u * g->num_sms));
        saba_adj16_kernel<<<mb, 256, 0, s>>>(g->saba_adj.as<uint32_t>(), g->saba_info.as<uint4>(),
                                             g->m, g->saba_adj16.as<uint4>());
        TGTP_LAUNCH_CHECK("saba_adj16_kernel");
    }
    g->saba_inline_ready = true;
}

template <int WPL>
void saba_launch(tgtp_graph* g, uint32_t depth, uint32_t bps, uint32_t grid_step, uint64_t total,
                 uint32_t* cnt, unsigned long long* fb) {
    cudaStream_t s = g->stream;
    uint32_t cap = kSabaHotCap;
    if (const char* e = std::getenv("TGTP_SABA_HOT")) cap = uint32_t(std::atoi(e));
    cap = std::max<uint32_t>(1024u, std::min<uint32_t>(cap, 53248u));
    const uint32_t hot = uint32_t(g->n < cap ? g->n : cap);
    const bool inl = saba_use_inline(g);
    const uint32_t hot_rec = inl ? 0u : std::min(hot, saba_hot_records(g));
    const size_t smem = sizeof(uint32_t) * (hot + 3 * size_t(hot_rec));
    if (inl) saba_prepare_inline(g);
    const void* kern = inl ? reinterpret_cast<const void*>(saba_walk_inline_kernel<WPL>)
                           : reinterpret_cast<const void*>(saba_walk_perm_kernel<WPL>);
    TGTP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int per_sm = 0;
    TGTP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSabaThreads, smem));
    if (per_sm < 1) per_sm = 1;
    uint64_t blocks = uint64_t(g->num_sms) * per_sm;
    const uint64_t need = (total + 4 * WPL - 1) / (4 * WPL) / (kSabaThreads / 32) + 1;
    if (blocks > need) blocks = need;
    ScopedKernel k(g->prof, s, "saba_walk");
    if (inl) {
        saba_walk_inline_kernel<WPL><<<unsigned(blocks), kSabaThreads, smem, s>>>(
            g->saba_info.as<uint4>(), g->saba_adj16.as<uint4>(), depth, bps, grid_step, total,
            cnt, hot, fb);
        TGTP_LAUNCH_CHECK("saba_walk_inline_kernel");
    } else {
        saba_walk_perm_kernel<WPL><<<unsigned(blocks), kSabaThreads, smem, s>>>(
            g->saba_info.as<uint4>(), g->saba_adj.as<uint32_t>(), depth, bps, grid_step, total,
            cnt, hot, hot_rec, fb);
        TGTP_LAUNCH_CHECK("saba_walk_perm_kernel");
    }
}

void saba_run(tgtp_graph* g, uint32_t depth, uint32_t n_walks, uint32_t* device_counters) {
    cudaStream_t s = g->stream;
    g->sums.reserve(4 * sizeof(unsigned long long));
    auto* sums = g->sums.as<unsigned long long>();
    TGTP_CUDA(cudaMemsetAsync(device_counters, 0, sizeof(uint32_t) * g->n, s));
    TGTP_CUDA(cudaMemsetAsync(sums, 0, 4 * sizeof(unsigned long long), s));
    if (n_walks == 0 || depth == 0) return;
    saba_prepare(g);
    const uint32_t bouquets_per_src = n_walks / 8;
    const uint32_t grid_step = UINT32_MAX / n_walks;
    const uint64_t total = g->n * uint64_t(bouquets_per_src);
    g->saba_cnt.reserve(sizeof(uint32_t) * (g->n + 1));
    auto* cnt = g->saba_cnt.as<uint32_t>();
    TGTP_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * g->n, s));
    // walkers per lane: the tuned choice, else TGTP_SABA_WPL, else 1 over the inlined copy and 2
    // over the plain one (its two dependent loads per hop want more chains in flight)
    int wpl = saba_use_inline(g) ? 1 : 2;
    if (g->saba_choice) wpl = g->saba_choice & 0xff;
    else if (const char* e = std::getenv("TGTP_SABA_WPL")) wpl = std::atoi(e);
    switch (wpl) {
        case 2: saba_launch<2>(g, depth, bouquets_per_src, grid_step, total, cnt, sums + 2); break;
        case 4: saba_launch<4>(g, depth, bouquets_per_src, grid_step, total, cnt, sums + 2); break;
        default: saba_launch<1>(g, depth, bouquets_per_src, grid_step, total, cnt, sums + 2); break;
    }
    {
        ScopedKernel k(g->prof, s, "saba_scatter");
        const unsigned nb = unsigned(std::min<uint64_t>((g->n + 255) / 256, 8u * g->num_sms));
        saba_scatter_kernel<<<nb ? nb : 1, 256, 0, s>>>(cnt, g->saba_info.as<uint4>(), g->n,
                                                        device_counters);
        TGTP_LAUNCH_CHECK("saba_scatter_kernel");
    }
}

int saba_tune(tgtp_graph* g, uint32_t depth, uint32_t n_walks, int trials) {
    std::vector<uint16_t> cand;
    for (int wpl : {1, 2, 4}) {
        if (saba_inline_fits(g)) cand.push_back(uint16_t(0x100 | wpl));
        // plain copy: no hot records, or 3,072 / 4,096 of them in shared memory
        for (int code : {0, 3, 4}) cand.push_back(uint16_t((code << 12) | wpl));
    }
    g->counters.reserve(sizeof(uint32_t) * (g->n + 1));
    auto* c = g->counters.as<uint32_t>();
    cudaEvent_t e0, e1;
    TGTP_CUDA(cudaEventCreate(&e0));
    TGTP_CUDA(cudaEventCreate(&e1));
    const bool prof = g->prof.enabled;
    g->prof.enabled = false;
    float best = 0;
    uint16_t pick = 0;
    try {
        for (uint16_t ch : cand) {
            g->saba_choice = ch;
            saba_run(g, depth, n_walks, c);  // warm-up (and the walk copy of this layout)
            float t = 0;
            for (int i = 0; i < std::max(trials, 1); ++i) {
                TGTP_CUDA(cudaEventRecord(e0, g->stream));
                saba_run(g, depth, n_walks, c);
                TGTP_CUDA(cudaEventRecord(e1, g->stream));
                TGTP_CUDA(cudaEventSynchronize(e1));
                float ms = 0;
                TGTP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                t = i == 0 ? ms : std::min(t, ms);
            }
            if (!pick || t < best) {
                best = t;
                pick = ch;
            }
        }
    } catch (...) {
        g->saba_choice = 0;
        g->prof.enabled = prof;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    g->saba_choice = pick;
    g->prof.enabled = prof;
    TGTP_CUDA(cudaEventDestroy(e0));
    TGTP_CUDA(cudaEventDestroy(e1));
    return pick;
}

void saba_summarize(tgtp_graph* g, const uint32_t* device_counters, uint64_t* host_sums3) {
    cudaStream_t s = g->stream;
    auto* sums = g->sums.as<unsigned long long>();
    {
        ScopedKernel k(g->prof, s, "saba_sums");
        const unsigned blocks = unsigned(std::min<uint64_t>((g->n + 255) / 256, 4u * g->num_sms));
        saba_sums_kernel<<<blocks ? blocks : 1, 256, 0, s>>>(device_counters, g->n, sums);
        TGTP_LAUNCH_CHECK("saba_sums_kernel");
    }
    unsigned long long h[3];
    TGTP_CUDA(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, s));
    TGTP_CUDA(cudaStreamSynchronize(s));
    host_sums3[0] = h[0];
    host_sums3[1] = h[1];
    host_sums3[2] = h[2];
}

}  // namespace tgtp

// ---- walk counter that allocates nothing -------------------------------------------------------
//
// Some callers cannot allocate device memory when they want the walk summary: a process whose
// device memory is owned by another allocator (a framework arena or a fixed budget that a stray
// cudaMalloc would overrun), or a latency-critical loop where cudaMalloc/cudaFree would synchronise
// the whole device.  saba_count_static serves them: the caller passes the CSR already on the device
// and receives the summary the walk runner prints; the per-vertex counters and the three sums live
// in the fixed array below, which every GPU that loads this library holds until the process exits.
namespace tgtp {
namespace {

// Largest vertex count saba_count_static accepts (16 MiB of uint32 counters).
constexpr uint64_t kStaticSabaMaxVertices = uint64_t(1) << 22;
// Words 0..7: four uint64 sums (visit count, checksum, fallback bouquets, active vertices);
// word 8: the CSR check's flags (kBad* below); counters start at word 64 (byte 256).
constexpr uint64_t kStaticSabaHeaderWords = 64;
constexpr uint64_t kStaticSabaFlagWord = 8;
enum : uint32_t { kBadOffsets = 1u, kBadNeighbour = 2u, kDeadEnd = 4u };

__device__ __align__(256) uint32_t g_static_saba_scratch[kStaticSabaHeaderWords + kStaticSabaMaxVertices];

// Device address of the scratch array on the current device.  It is looked up on every call
// (cudaGetSymbolAddress allocates nothing and is cheap), so a new primary context after a
// cudaDeviceReset never sees a stale address.
void* static_scratch(int device, int* num_sms) {
    void* p = nullptr;
    TGTP_CUDA(cudaGetSymbolAddress(&p, g_static_saba_scratch));
    TGTP_CUDA(cudaDeviceGetAttribute(num_sms, cudaDevAttrMultiProcessorCount, device));
    return p;
}

// The caller's CSR is checked before any walk: offsets start at 0 and never decrease, every
// neighbour id is below n, and every neighbour has a nonzero degree (a walk that reached a vertex
// without neighbours would pick adj[idx[cur] + (r % 0)]).  Offsets are checked by one pass; the
// neighbour pass reads adj[0 .. idx[n]) only, the slots the CSR declares.  Violations set flag bits
// in the scratch header; the host reads them back and refuses the call.
__global__ void static_check_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ adj,
                                    uint64_t n, uint32_t* __restrict__ flags,
                                    unsigned long long* __restrict__ active) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t t0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    uint32_t bad = 0;
    unsigned long long a = 0;
    if (t0 == 0 && idx[0] != 0u) bad |= kBadOffsets;
    for (uint64_t v = t0; v < n; v += stride) {
        const uint32_t b = idx[v], e = idx[v + 1];
        if (e < b) bad |= kBadOffsets;
        a += e != b;
    }
    const uint64_t m = idx[n];
    for (uint64_t q = t0; q < m; q += stride) {
        const uint32_t u = adj[q];
        if (uint64_t(u) >= n) bad |= kBadNeighbour;
        else if (idx[u + 1] == idx[u]) bad |= kDeadEnd;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        a += __shfl_xor_sync(kFullMask, a, o);
        bad |= __shfl_xor_sync(kFullMask, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (a) atomicAdd(active, a);
        if (bad) atomicOr(flags, bad);
    }
}

}  // namespace
}  // namespace tgtp

extern "C" tgtp_status saba_count_static(const uint32_t* device_idx, const uint32_t* device_adj,
                                         uint64_t n, uint32_t depth, uint32_t n_walks,
                                         void* cuda_stream, saba_result* out) {
    using namespace tgtp;
    return guarded([&] {
        if (!device_idx || !device_adj || !out) fail(TGTP_ERR_INVALID_ARGUMENT, "null argument");
        if (n == 0) fail(TGTP_ERR_INVALID_ARGUMENT, "empty graph");
        if (n > kStaticSabaMaxVertices)
            fail(TGTP_ERR_INVALID_ARGUMENT,
                 "saba_count_static accepts at most 4194304 vertices (its counters are a fixed "
                 "16 MiB device array); use saba_count for larger graphs");
        if (n_walks % 8 != 0)
            fail(TGTP_ERR_INVALID_ARGUMENT,
                 "n_walks must be a multiple of 8 within the 32-bit grid domain");
        int device = 0;
        TGTP_CUDA(cudaGetDevice(&device));
        int num_sms = 0;
        auto* base = static_cast<uint32_t*>(static_scratch(device, &num_sms));
        auto* sums = reinterpret_cast<unsigned long long*>(base);
        uint32_t* counters = base + kStaticSabaHeaderWords;
        cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
        // the array keeps the previous call's contents: start from zero
        TGTP_CUDA(cudaMemsetAsync(base, 0, sizeof(uint32_t) * (kStaticSabaHeaderWords + n), s));
        static_check_kernel<<<unsigned(std::min<uint64_t>((n + 255) / 256, 4u * num_sms)), 256, 0, s>>>(
            device_idx, device_adj, n, base + kStaticSabaFlagWord, sums + 3);
        TGTP_LAUNCH_CHECK("static_check_kernel");
        uint32_t flags = 0;
        TGTP_CUDA(cudaMemcpyAsync(&flags, base + kStaticSabaFlagWord, sizeof(flags),
                                  cudaMemcpyDeviceToHost, s));
        TGTP_CUDA(cudaStreamSynchronize(s));
        if (flags & kBadOffsets)
            fail(TGTP_ERR_INVALID_ARGUMENT, "CSR offsets must start at 0 and never decrease");
        if (flags & kBadNeighbour)
            fail(TGTP_ERR_INVALID_ARGUMENT, "CSR neighbour id out of range (must be below n)");
        if (flags & kDeadEnd)
            fail(TGTP_ERR_INVALID_ARGUMENT,
                 "CSR has an edge into a vertex without neighbours (a walk could not leave it)");
        if (n_walks && depth) {
            const uint32_t bouquets_per_src = n_walks / 8;
            const uint32_t grid_step = UINT32_MAX / n_walks;
            const uint64_t total = n * uint64_t(bouquets_per_src);
            const uint32_t hot = uint32_t(n < kSabaHotCap ? n : kSabaHotCap);
            const size_t smem = sizeof(uint32_t) * hot;
            TGTP_CUDA(cudaFuncSetAttribute(saba_walk_kernel,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(sizeof(uint32_t) * kSabaHotCap)));
            int per_sm = 0;
            TGTP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, saba_walk_kernel,
                                                                    kSabaThreads, smem));
            if (per_sm < 1) per_sm = 1;
            uint64_t blocks = uint64_t(num_sms) * per_sm;
            const uint64_t need = (total + 3) / 4 / (kSabaThreads / 32) + 1;
            if (blocks > need) blocks = need;
            saba_walk_kernel<<<unsigned(blocks), kSabaThreads, smem, s>>>(
                device_idx, device_adj, depth, bouquets_per_src, grid_step, total, counters, hot,
                sums + 2);
            TGTP_LAUNCH_CHECK("saba_walk_kernel");
        }
        const unsigned blocks = unsigned(std::min<uint64_t>((n + 255) / 256, 4u * num_sms));
        saba_sums_kernel<<<blocks ? blocks : 1, 256, 0, s>>>(counters, n, sums);
        TGTP_LAUNCH_CHECK("saba_sums_kernel");
        unsigned long long h[4];
        TGTP_CUDA(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, s));
        TGTP_CUDA(cudaStreamSynchronize(s));
        out->visit_count = h[0];
        out->checksum = h[1];
        out->fallback_bouquets = h[2];
        const unsigned __int128 expect = (unsigned __int128)h[3] * n_walks * depth;
        if ((unsigned __int128)h[0] != expect)
            fail(TGTP_ERR_OVERFLOW, "a uint32 visit counter overflowed");
    });
}
