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
#include <mutex>

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

void saba_run(tgtp_graph* g, uint32_t depth, uint32_t n_walks, uint32_t* device_counters) {
    cudaStream_t s = g->stream;
    g->sums.reserve(4 * sizeof(unsigned long long));
    auto* sums = g->sums.as<unsigned long long>();
    TGTP_CUDA(cudaMemsetAsync(device_counters, 0, sizeof(uint32_t) * g->n, s));
    TGTP_CUDA(cudaMemsetAsync(sums, 0, 4 * sizeof(unsigned long long), s));
    if (n_walks == 0 || depth == 0) return;
    const uint32_t bouquets_per_src = n_walks / 8;
    const uint32_t grid_step = UINT32_MAX / n_walks;
    const uint64_t total = g->n * uint64_t(bouquets_per_src);
    const uint32_t hot = uint32_t(g->n < kSabaHotCap ? g->n : kSabaHotCap);
    const size_t smem = sizeof(uint32_t) * hot;
    TGTP_CUDA(cudaFuncSetAttribute(saba_walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(sizeof(uint32_t) * kSabaHotCap)));
    int per_sm = 0;
    TGTP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, saba_walk_kernel,
                                                            kSabaThreads, smem));
    if (per_sm < 1) per_sm = 1;
    uint64_t blocks = uint64_t(g->num_sms) * per_sm;
    const uint64_t need = (total + 3) / 4 / (kSabaThreads / 32) + 1;  // one group-step per warp
    if (blocks > need) blocks = need;
    {
        ScopedKernel k(g->prof, s, "saba_walk");
        saba_walk_kernel<<<unsigned(blocks), kSabaThreads, smem, s>>>(
            g->idx.as<uint32_t>(), g->adj.as<uint32_t>(), depth, bouquets_per_src, grid_step, total,
            device_counters, hot, sums + 2);
        TGTP_LAUNCH_CHECK("saba_walk_kernel");
    }
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
// counters start at word 64 (byte 256).
constexpr uint64_t kStaticSabaHeaderWords = 64;

__device__ __align__(256) uint32_t g_static_saba_scratch[kStaticSabaHeaderWords + kStaticSabaMaxVertices];

constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
void* g_static_addr[kMaxDevices] = {};
int g_static_sms[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once per device.
void* static_scratch(int device, int* num_sms) {
    if (device < 0 || device >= kMaxDevices) fail(TGTP_ERR_UNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[device]) {
        void* p = nullptr;
        TGTP_CUDA(cudaGetSymbolAddress(&p, g_static_saba_scratch));
        int sms = 0;
        TGTP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        g_static_sms[device] = sms;
        g_static_addr[device] = p;
    }
    *num_sms = g_static_sms[device];
    return g_static_addr[device];
}

__global__ void static_active_kernel(const uint32_t* __restrict__ idx, uint64_t n,
                                     unsigned long long* __restrict__ active) {
    unsigned long long a = 0;
    for (uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
         v += uint64_t(gridDim.x) * blockDim.x)
        a += idx[v + 1] != idx[v];
#pragma unroll
    for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(kFullMask, a, o);
    if ((threadIdx.x & 31) == 0 && a) atomicAdd(active, a);
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
        static_active_kernel<<<unsigned(std::min<uint64_t>((n + 255) / 256, 4u * num_sms)), 256, 0, s>>>(
            device_idx, n, sums + 3);
        TGTP_LAUNCH_CHECK("static_active_kernel");
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
