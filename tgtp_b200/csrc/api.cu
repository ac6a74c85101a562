// C ABI of libtgtp_gpu (include/tgtp_gpu.h): graph/eigen upload, device-side preparation of the
// per-slot maps, the SABA entry points, profiling, and error reporting.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>

#include "common.cuh"
#include "internal.hpp"

namespace tgtp {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

// ---- device block cache and stream pool -----------------------------------------------------------
namespace {
std::mutex g_cache_mu;
std::map<std::pair<int, size_t>, std::vector<void*>> g_free_blocks;  // (device, class) -> blocks
std::map<int, std::vector<cudaStream_t>> g_free_streams;

size_t size_class(size_t bytes) {
    if (bytes <= (size_t(1) << 20)) {  // powers of two up to 1 MiB
        size_t c = 256;
        while (c < bytes) c <<= 1;
        return c;
    }
    const size_t g = size_t(2) << 20;  // 2 MiB steps above
    return (bytes + g - 1) / g * g;
}
}  // namespace

void* cache_alloc(size_t bytes, size_t* granted) {
    int dev = 0;
    TGTP_CUDA(cudaGetDevice(&dev));
    const size_t c = size_class(bytes);
    {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        auto it = g_free_blocks.find({dev, c});
        if (it != g_free_blocks.end() && !it->second.empty()) {
            void* p = it->second.back();
            it->second.pop_back();
            *granted = c;
            return p;
        }
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, c);
    if (e == cudaErrorMemoryAllocation) {  // give the cache back to the driver and retry once
        (void)cudaGetLastError();
        cache_trim();
        e = cudaMalloc(&p, c);
    }
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        fail(e == cudaErrorMemoryAllocation ? TGTP_ERR_OUT_OF_MEMORY : TGTP_ERR_CUDA,
             std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    *granted = c;
    return p;
}

// Set while a graph whose stream has been synchronised releases its buffers: no work can still use
// them, so the per-block device synchronisation is skipped.
thread_local bool g_release_quiet = false;

void cache_free(void* p, size_t granted) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        (!g_release_quiet && cudaDeviceSynchronize() != cudaSuccess)) {
        (void)cudaGetLastError();
        cudaFree(p);
        return;
    }
    std::lock_guard<std::mutex> lock(g_cache_mu);
    g_free_blocks[{dev, granted}].push_back(p);
}

void cache_trim() {
    std::lock_guard<std::mutex> lock(g_cache_mu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto& kv : g_free_blocks) {
        cudaSetDevice(kv.first.first);
        for (void* p : kv.second) cudaFree(p);
        kv.second.clear();
    }
    cudaSetDevice(cur);
}

cudaStream_t stream_acquire() {
    int dev = 0;
    TGTP_CUDA(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        auto& v = g_free_streams[dev];
        if (!v.empty()) {
            cudaStream_t s = v.back();
            v.pop_back();
            return s;
        }
    }
    cudaStream_t s = nullptr;
    TGTP_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return s;
}

void stream_release(cudaStream_t s) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
        (void)cudaGetLastError();
        cudaStreamDestroy(s);
        return;
    }
    std::lock_guard<std::mutex> lock(g_cache_mu);
    g_free_streams[dev].push_back(s);
}

// ---- profiler ------------------------------------------------------------------------------------
cudaEvent_t Profiler::take() {
    if (!pool_.empty()) {
        cudaEvent_t e = pool_.back();
        pool_.pop_back();
        return e;
    }
    cudaEvent_t e;
    TGTP_CUDA(cudaEventCreate(&e));
    return e;
}
void Profiler::begin(cudaStream_t s, const char* name) {
    open_ = take();
    open_name_ = name;
    TGTP_CUDA(cudaEventRecord(open_, s));
}
void Profiler::end(cudaStream_t s) {
    if (!open_) return;
    cudaEvent_t b = take();
    if (cudaEventRecord(b, s) != cudaSuccess) return;  // called from a destructor: never throw
    pending_.push_back({open_name_, open_, b});
    open_ = nullptr;
}
void Profiler::collect() {
    for (auto& p : pending_) {
        TGTP_CUDA(cudaEventSynchronize(p.b));
        float ms = 0;
        TGTP_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
        auto it = std::find_if(totals.begin(), totals.end(),
                               [&](const Entry& e) { return e.name == p.name; });
        if (it == totals.end()) {
            totals.push_back({p.name, 0, 0});
            it = totals.end() - 1;
        }
        it->launches += 1;
        it->total_ms += ms;
        pool_.push_back(p.a);
        pool_.push_back(p.b);
    }
    pending_.clear();
}
void Profiler::clear() {
    for (auto& p : pending_) {
        cudaEventSynchronize(p.b);
        pool_.push_back(p.a);
        pool_.push_back(p.b);
    }
    pending_.clear();
    totals.clear();
}
Profiler::~Profiler() {
    for (auto& p : pending_) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (auto e : pool_) cudaEventDestroy(e);
}

// ---- per-slot maps built on the device at upload -----------------------------------------------
namespace {

__global__ void degree_kernel(const uint32_t* __restrict__ idx, uint64_t n, uint32_t* __restrict__ deg) {
    for (uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
         v += uint64_t(gridDim.x) * blockDim.x)
        deg[v] = idx[v + 1] - idx[v];
}

// row_of[pos] = u with idx[u] <= pos < idx[u+1] (rows may be empty: take the last such u).
__global__ void row_of_kernel(const uint32_t* __restrict__ idx, uint64_t n, uint64_t m,
                              uint32_t* __restrict__ row_of) {
    for (uint64_t pos = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; pos < m;
         pos += uint64_t(gridDim.x) * blockDim.x) {
        uint64_t lo = 0, hi = n;  // largest u with idx[u] <= pos
        while (hi - lo > 1) {
            const uint64_t mid = (lo + hi) >> 1;
            if (idx[mid] <= pos) lo = mid;
            else hi = mid;
        }
        row_of[pos] = uint32_t(lo);
    }
}

// Per-slot checks of an uploaded CSR (after row_of, which needs only monotone offsets): neighbour
// ids below n (bit 0), rows sorted ascending (bit 1), a repeated neighbour (bit 2); and the degree
// summary (max, min, vertices with a nonzero degree).  info = {flags, max, min, active}.
__global__ void validate_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ adj,
                                const uint32_t* __restrict__ row_of, uint64_t n, uint64_t m,
                                unsigned* __restrict__ info) {
    unsigned flags = 0, mx = 0, mn = 0xffffffffu, act = 0;
    for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < m;
         q += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t a = adj[q];
        if (a >= n) flags |= 1u;
        else if (idx[a + 1] == idx[a]) flags |= 8u;  // a walk would stop at a vertex without neighbours
        if (q > idx[row_of[q]]) {
            const uint32_t b = adj[q - 1];
            if (a < b) flags |= 2u;
            if (a == b) flags |= 4u;
        }
    }
    for (uint64_t v = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; v < n;
         v += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t d = idx[v + 1] - idx[v];
        mx = max(mx, d);
        mn = min(mn, d);
        act += d != 0;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        flags |= __shfl_xor_sync(kFullMask, flags, o);
        mx = max(mx, __shfl_xor_sync(kFullMask, mx, o));
        mn = min(mn, __shfl_xor_sync(kFullMask, mn, o));
        act += __shfl_xor_sync(kFullMask, act, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (flags) atomicOr(info, flags);
        atomicMax(info + 1, mx);
        atomicMin(info + 2, mn);
        if (act) atomicAdd(info + 3, act);
    }
}

// rev[pos] = lower_bound(row v, u) for slot (u, v): the slot src/aesc.h:207-209 and :541-542 address.
// sym_src[q] = 1 + max{pos : rev[pos] == q}: the slot whose value lands in rev_preds[q] last
// (src/aesc.h:538-545 writes rows in order, so the largest pos wins).
__global__ void rev_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ adj,
                           const uint32_t* __restrict__ row_of, uint64_t m,
                           uint32_t* __restrict__ rev, uint32_t* __restrict__ sym_src) {
    for (uint64_t pos = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; pos < m;
         pos += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t u = row_of[pos], v = adj[pos];
        const uint32_t q = lower_bound_u32(adj, idx[v], idx[v + 1], u);
        rev[pos] = q;
        atomicMax(sym_src + q, uint32_t(pos + 1));
    }
}

// adjd[pos] = (neighbour, neighbour's degree): one coalesced 8-byte load per pushed slot instead of
// a load plus a dependent degree gather.
__global__ void adjd_kernel(const uint32_t* __restrict__ adj, const uint32_t* __restrict__ deg,
                            uint64_t m, uint2* __restrict__ adjd) {
    for (uint64_t pos = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; pos < m;
         pos += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t u = adj[pos];
        adjd[pos] = make_uint2(u, deg[u]);
    }
}

// forward slots (v >= u) are the tail of each sorted row; count them per row.
__global__ void forward_count_kernel(const uint32_t* __restrict__ idx,
                                     const uint32_t* __restrict__ adj, uint64_t n,
                                     uint32_t* __restrict__ cnt, uint32_t* __restrict__ lbp) {
    for (uint64_t u = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < n;
         u += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t lb = lower_bound_u32(adj, idx[u], idx[u + 1], uint32_t(u));
        cnt[u] = idx[u + 1] - lb;
        lbp[u] = lb;
    }
}

// Exclusive scan of cnt[0..n) in one block, chunk by chunk with a running carry; writes the total
// to cnt_total.  Runs once per upload.
__global__ void scan_kernel(uint32_t* __restrict__ cnt, uint64_t n, uint32_t* __restrict__ total) {
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint64_t base = 0; base < n; base += blockDim.x) {
        const uint64_t i = base + threadIdx.x;
        const uint32_t x = i < n ? cnt[i] : 0;
        uint32_t incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFullMask, incl, o);
            if (lane >= uint32_t(o)) incl += y;
        }
        if (lane == 31) warp_sums[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            const uint32_t nw = blockDim.x >> 5;
            uint32_t ws = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(kFullMask, ws, o);
                if (lane >= uint32_t(o)) ws += y;
            }
            if (lane < nw) warp_sums[lane] = ws;  // inclusive
        }
        __syncthreads();
        const uint32_t before = (wid ? warp_sums[wid - 1] : 0) + carry;
        if (i < n) cnt[i] = before + incl - x;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = before + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// One thread per slot: forward slot p = (u, v >= u) goes to off[u] + (p - lb[u]), with the edge's
// record (u, v, p, reverse slot of p) beside it for the tau kernels.
__global__ void forward_fill_kernel(const uint32_t* __restrict__ adj,
                                    const uint32_t* __restrict__ row_of,
                                    const uint32_t* __restrict__ rev, uint64_t m,
                                    const uint32_t* __restrict__ off,
                                    const uint32_t* __restrict__ lbp, uint32_t* __restrict__ fwd,
                                    uint4* __restrict__ fedge) {
    for (uint64_t p = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < m;
         p += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t u = row_of[p], v = adj[p];
        if (v < u) continue;
        const uint32_t e = off[u] + (uint32_t(p) - lbp[u]);
        fwd[e] = uint32_t(p);
        fedge[e] = make_uint4(u, v, uint32_t(p), rev[p]);
    }
}

// 1 + lambda_i, 1 - lambda_i and eigen_t_1 = lambda_i^2, lambda_i^4, ... by repeated
// multiplication (double, and its float cast), one thread per eigen index.
__global__ void eigen_tables_kernel(const double* __restrict__ values, uint32_t omega, int rows,
                                    double* __restrict__ onep, double* __restrict__ onem,
                                    double* __restrict__ tab, float* __restrict__ tabf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= omega) return;
    const double v = values[i];
    onep[i] = __dadd_rn(1.0, v);
    onem[i] = __dsub_rn(1.0, v);
    const double sq = __dmul_rn(v, v);
    double e = sq;
    for (int k = 0; k < rows; ++k) {
        tab[size_t(k) * omega + i] = e;
        tabf[size_t(k) * omega + i] = __double2float_rn(e);
        e = __dmul_rn(e, sq);
    }
}

__global__ void f64_to_storage_kernel(const double* __restrict__ in, uint64_t count,
                                      float* __restrict__ out_f32, __nv_bfloat16* __restrict__ out_bf16) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += uint64_t(gridDim.x) * blockDim.x) {
        if (out_f32) out_f32[i] = __double2float_rn(in[i]);
        if (out_bf16) out_bf16[i] = __double2bfloat16(in[i]);
    }
}
__global__ void f32_to_bf16_kernel(const float* __restrict__ in, uint64_t count,
                                   __nv_bfloat16* __restrict__ out) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += uint64_t(gridDim.x) * blockDim.x)
        out[i] = __float2bfloat16_rn(in[i]);
}

unsigned grid_for(uint64_t work, int num_sms) {
    const uint64_t b = (work + 255) / 256;
    const uint64_t cap = uint64_t(num_sms) * 8;
    return unsigned(std::max<uint64_t>(1, std::min(b, cap)));
}

}  // namespace

void graph_prepare(tgtp_graph* g) {
    cudaStream_t s = g->stream;
    const uint64_t n = g->n, m = g->m;
    auto* idx = g->idx.as<uint32_t>();
    auto* adj = g->adj.as<uint32_t>();
    g->deg.reserve(sizeof(uint32_t) * (n + 1));
    g->row_of.reserve(sizeof(uint32_t) * (m + 1));
    g->rev.reserve(sizeof(uint32_t) * (m + 1));
    g->sym_src.reserve(sizeof(uint32_t) * (m + 1));
    // first the maps that read neighbour ids only as values, the checks, the forward counts.  The
    // per-row scratch is the handle's (released with it), so returning does not wait for the
    // kernels after the checks: the caller's next call on the stream overlaps them (e.g. the
    // eigenvector copy)
    DeviceBuffer& cnt = g->prep_cnt;
    DeviceBuffer& lbp = g->prep_lbp;
    cnt.reserve(sizeof(uint32_t) * (n + 8));
    lbp.reserve(sizeof(uint32_t) * (n + 1));
    auto* c = cnt.as<uint32_t>();
    unsigned* info = c + n + 1;  // forward total, then {flags, max, min, active}
    const unsigned init[5] = {0u, 0u, 0u, 0xffffffffu, 0u};
    TGTP_CUDA(cudaMemcpyAsync(info, init, sizeof(init), cudaMemcpyHostToDevice, s));
    degree_kernel<<<grid_for(n, g->num_sms), 256, 0, s>>>(idx, n, g->deg.as<uint32_t>());
    TGTP_LAUNCH_CHECK("degree_kernel");
    if (m) {
        row_of_kernel<<<grid_for(m, g->num_sms), 256, 0, s>>>(idx, n, m, g->row_of.as<uint32_t>());
        TGTP_LAUNCH_CHECK("row_of_kernel");
    }
    validate_kernel<<<grid_for(std::max(n, m), g->num_sms), 256, 0, s>>>(
        idx, adj, g->row_of.as<uint32_t>(), n, m, info + 1);
    TGTP_LAUNCH_CHECK("validate_kernel");
    forward_count_kernel<<<grid_for(n, g->num_sms), 256, 0, s>>>(idx, adj, n, c,
                                                                 lbp.as<uint32_t>());
    TGTP_LAUNCH_CHECK("forward_count_kernel");
    scan_kernel<<<1, 1024, 0, s>>>(c, n, info);
    TGTP_LAUNCH_CHECK("scan_kernel");
    unsigned h[5] = {0, 0, 0, 0, 0};
    TGTP_CUDA(cudaMemcpyAsync(h, info, sizeof(h), cudaMemcpyDeviceToHost, s));
    TGTP_CUDA(cudaStreamSynchronize(s));
    if (h[1] & 1u) fail(TGTP_ERR_INVALID_ARGUMENT, "neighbour id out of range");
    if (h[1] & 2u) fail(TGTP_ERR_INVALID_ARGUMENT, "rows must be sorted");
    if (h[1] & 8u) fail(TGTP_ERR_INVALID_ARGUMENT, "an edge leads to a vertex without neighbours");
    g->has_multi_edges = (h[1] & 4u) != 0;
    g->max_degree = h[2];
    g->min_degree = h[3];
    g->num_active = h[4];
    const uint32_t total = h[0];
    // then the maps that index by neighbour id
    if (m) {
        TGTP_CUDA(cudaMemsetAsync(g->sym_src.ptr, 0, sizeof(uint32_t) * m, s));
        rev_kernel<<<grid_for(m, g->num_sms), 256, 0, s>>>(idx, adj, g->row_of.as<uint32_t>(), m,
                                                           g->rev.as<uint32_t>(),
                                                           g->sym_src.as<uint32_t>());
        TGTP_LAUNCH_CHECK("rev_kernel");
        g->adjd.reserve(sizeof(uint2) * (m + 1));
        adjd_kernel<<<grid_for(m, g->num_sms), 256, 0, s>>>(adj, g->deg.as<uint32_t>(), m,
                                                            g->adjd.as<uint2>());
        TGTP_LAUNCH_CHECK("adjd_kernel");
    }
    g->num_forward = total;
    g->forward.reserve(sizeof(uint32_t) * (total + 1));
    g->fedge.reserve(sizeof(uint4) * (total + 1));
    if (m)
        forward_fill_kernel<<<grid_for(m, g->num_sms), 256, 0, s>>>(
            adj, g->row_of.as<uint32_t>(), g->rev.as<uint32_t>(), m, c, lbp.as<uint32_t>(),
            g->forward.as<uint32_t>(), g->fedge.as<uint4>());
    TGTP_LAUNCH_CHECK("forward_fill_kernel");
}

}  // namespace tgtp

tgtp_graph::~tgtp_graph() {
    // the device buffers (members) are returned to the cache after this body, once the device
    // is idle; the stream goes back to the pool
    if (stream) cudaStreamSynchronize(stream);
    if (hint_event) cudaEventDestroy(hint_event);
    if (hint_host) cudaFreeHost(hint_host);
    if (own_stream) tgtp::stream_release(own_stream);
}

using namespace tgtp;

extern "C" {

const char* tgtp_last_error(void) { return g_last_error.c_str(); }
int tgtp_abi_version(void) { return TGTP_ABI_VERSION; }
void tgtp_host_free(void* p) { std::free(p); }

tgtp_status tgtp_graph_upload(const uint32_t* idx, const uint32_t* adj, uint64_t n, uint64_t m,
                              tgtp_graph** out) {
    return guarded([&] {
        if (!out) fail(TGTP_ERR_INVALID_ARGUMENT, "null output handle");
        *out = nullptr;
        if (!idx || (m && !adj)) fail(TGTP_ERR_INVALID_ARGUMENT, "null CSR pointer");
        if (n == 0) fail(TGTP_ERR_INVALID_ARGUMENT, "empty graph");
        if (n >= 0xffffffffull) fail(TGTP_ERR_INVALID_ARGUMENT, "vertex count exceeds uint32");
        if (m >= 0xffffffffull) fail(TGTP_ERR_INVALID_ARGUMENT, "graph exceeds CSR index capacity");
        if (idx[0] != 0 || idx[n] != m)
            fail(TGTP_ERR_INVALID_ARGUMENT, "row offsets must start at 0 and end at m");
        auto g = std::make_unique<tgtp_graph>();
        g->n = n;
        g->m = m;
        // monotone offsets here (the device maps rely on them); neighbour ranges, row order,
        // repeated neighbours and the degree summary are checked on the device (graph_prepare)
        for (uint64_t v = 0; v < n; ++v)
            if (idx[v + 1] < idx[v]) fail(TGTP_ERR_INVALID_ARGUMENT, "row offsets decrease");
        TGTP_CUDA(cudaGetDevice(&g->device));
        TGTP_CUDA(cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, g->device));
        g->own_stream = stream_acquire();
        g->stream = g->own_stream;
        g->idx.reserve(sizeof(uint32_t) * (n + 1));
        g->adj.reserve(sizeof(uint32_t) * (m + 1));
        TGTP_CUDA(cudaMemcpyAsync(g->idx.ptr, idx, sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice,
                                  g->stream));
        if (m)
            TGTP_CUDA(cudaMemcpyAsync(g->adj.ptr, adj, sizeof(uint32_t) * m, cudaMemcpyHostToDevice,
                                      g->stream));
        graph_prepare(g.get());
        *out = g.release();
    });
}

tgtp_status tgtp_graph_free(tgtp_graph* g) {
    return guarded([&] {
        if (!g) return;
        if (g->batch_refs > 0)
            fail(TGTP_ERR_INVALID_ARGUMENT, "this graph belongs to a live batch; free the batch first");
        // every use of the graph's buffers was ordered on its stream: one synchronisation of that
        // stream covers the release of all of them
        TGTP_CUDA(cudaStreamSynchronize(g->stream));
        g_release_quiet = true;
        delete g;
        g_release_quiet = false;
    });
}

tgtp_status tgtp_graph_set_stream(tgtp_graph* g, void* cuda_stream) {
    return guarded([&] {
        if (!g) fail(TGTP_ERR_INVALID_ARGUMENT, "null graph");
        TGTP_CUDA(cudaStreamSynchronize(g->stream));
        g->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : g->own_stream;
    });
}

void* tgtp_graph_stream(tgtp_graph* g) { return g ? static_cast<void*>(g->stream) : nullptr; }

tgtp_status tgtp_graph_info(const tgtp_graph* g, uint64_t* n, uint64_t* m) {
    return guarded([&] {
        if (!g) fail(TGTP_ERR_INVALID_ARGUMENT, "null graph");
        if (n) *n = g->n;
        if (m) *m = g->m;
    });
}

tgtp_status tgtp_eigens_upload(tgtp_graph* g, const double* values, const void* vectors,
                               uint32_t omega, int32_t dtype, int32_t store_dtype) {
    return guarded([&] {
        if (!g || !values || !vectors) fail(TGTP_ERR_INVALID_ARGUMENT, "null argument");
        if (g->batch_refs > 0)
            fail(TGTP_ERR_INVALID_ARGUMENT, "this graph belongs to a live batch; free the batch first");
        if (omega < 2 || omega > g->n)
            fail(TGTP_ERR_INVALID_ARGUMENT, "omega must be between 2 and vertex count");
        if (dtype != TGTP_VEC_F32 && dtype != TGTP_VEC_F64)
            fail(TGTP_ERR_INVALID_ARGUMENT, "host eigenvectors must be F32 or F64");
        if (store_dtype < TGTP_VEC_F32 || store_dtype > TGTP_VEC_BF16)
            fail(TGTP_ERR_INVALID_ARGUMENT, "unknown storage dtype");
        if (dtype == TGTP_VEC_F32 && store_dtype == TGTP_VEC_F64)
            fail(TGTP_ERR_INVALID_ARGUMENT, "F32 host data cannot be stored as F64");
        for (uint32_t i = 0; i < omega; ++i)
            if (!std::isfinite(values[i])) fail(TGTP_ERR_INVALID_ARGUMENT, "invalid eigenvalue");
        if (g->omega != omega) {
            g->has_f32 = g->has_f64 = g->has_bf16 = false;
        }
        cudaStream_t s = g->stream;
        const uint64_t count = g->n * uint64_t(omega);
        g->omega = omega;
        g->split_omega = 0;
        g->values.assign(values, values + omega);
        g->d_values.reserve(sizeof(double) * omega);
        TGTP_CUDA(cudaMemcpyAsync(g->d_values.ptr, values, sizeof(double) * omega,
                                  cudaMemcpyHostToDevice, s));
        // tau-bound tables: onep/onem per eigen index, and eigen_t_1 after k multiplications
        // (src/aesc.h:174-176, :190, :201-203), in the reference's exact sequence of roundings,
        // formed on the device from the uploaded values
        constexpr int kRows = 64;
        g->onep.reserve(sizeof(double) * omega);
        g->onem.reserve(sizeof(double) * omega);
        g->etab.reserve(sizeof(double) * kRows * omega);
        g->etab_f.reserve(sizeof(float) * kRows * omega);
        eigen_tables_kernel<<<(omega + 127) / 128, 128, 0, s>>>(
            g->d_values.as<double>(), omega, kRows, g->onep.as<double>(), g->onem.as<double>(),
            g->etab.as<double>(), g->etab_f.as<float>());
        TGTP_LAUNCH_CHECK("eigen_tables_kernel");
        const unsigned blocks = grid_for(count, g->num_sms);
        if (dtype == TGTP_VEC_F32) {
            g->vec_f32.reserve(sizeof(float) * count);
            TGTP_CUDA(cudaMemcpyAsync(g->vec_f32.ptr, vectors, sizeof(float) * count,
                                      cudaMemcpyHostToDevice, s));
            if (store_dtype == TGTP_VEC_BF16) {
                g->vec_bf16.reserve(sizeof(__nv_bfloat16) * count);
                f32_to_bf16_kernel<<<blocks, 256, 0, s>>>(g->vec_f32.as<float>(), count,
                                                          g->vec_bf16.as<__nv_bfloat16>());
                TGTP_LAUNCH_CHECK("f32_to_bf16_kernel");
                g->has_bf16 = true;
            } else {
                g->has_f32 = true;
            }
        } else {
            g->vec_f64.reserve(sizeof(double) * count);
            TGTP_CUDA(cudaMemcpyAsync(g->vec_f64.ptr, vectors, sizeof(double) * count,
                                      cudaMemcpyHostToDevice, s));
            if (store_dtype == TGTP_VEC_F64) {
                g->has_f64 = true;
            } else {
                float* f32 = nullptr;
                __nv_bfloat16* b16 = nullptr;
                if (store_dtype == TGTP_VEC_F32) {
                    g->vec_f32.reserve(sizeof(float) * count);
                    f32 = g->vec_f32.as<float>();
                    g->has_f32 = true;
                } else {
                    g->vec_bf16.reserve(sizeof(__nv_bfloat16) * count);
                    b16 = g->vec_bf16.as<__nv_bfloat16>();
                    g->has_bf16 = true;
                }
                f64_to_storage_kernel<<<blocks, 256, 0, s>>>(g->vec_f64.as<double>(), count, f32, b16);
                TGTP_LAUNCH_CHECK("f64_to_storage_kernel");
            }
        }
        TGTP_CUDA(cudaStreamSynchronize(s));
    });
}

tgtp_status saba_count_device(tgtp_graph* g, uint32_t depth, uint32_t n_walks,
                              uint32_t* device_counters) {
    return guarded([&] {
        if (!g || !device_counters) fail(TGTP_ERR_INVALID_ARGUMENT, "null argument");
        if (n_walks % 8 != 0)
            fail(TGTP_ERR_INVALID_ARGUMENT,
                 "n_walks must be a multiple of 8 within the 32-bit grid domain");
        saba_run(g, depth, n_walks, device_counters);
    });
}

tgtp_status saba_tune(tgtp_graph* g, uint32_t depth, uint32_t n_walks, int32_t trials,
                      int32_t* choice) {
    return guarded([&] {
        if (!g) fail(TGTP_ERR_INVALID_ARGUMENT, "null graph");
        if (n_walks % 8 != 0)
            fail(TGTP_ERR_INVALID_ARGUMENT,
                 "n_walks must be a multiple of 8 within the 32-bit grid domain");
        const int pick = tgtp::saba_tune(g, depth, n_walks, trials);
        if (choice) *choice = pick;
    });
}

tgtp_status saba_count(tgtp_graph* g, uint32_t depth, uint32_t n_walks, uint32_t* host_counters,
                       saba_result* out) {
    return guarded([&] {
        if (!g) fail(TGTP_ERR_INVALID_ARGUMENT, "null graph");
        if (n_walks % 8 != 0)
            fail(TGTP_ERR_INVALID_ARGUMENT,
                 "n_walks must be a multiple of 8 within the 32-bit grid domain");
        g->counters.reserve(sizeof(uint32_t) * (g->n + 1));
        auto* c = g->counters.as<uint32_t>();
        saba_run(g, depth, n_walks, c);
        uint64_t sums[3];
        saba_summarize(g, c, sums);
        if (host_counters)
            TGTP_CUDA(cudaMemcpy(host_counters, c, sizeof(uint32_t) * g->n, cudaMemcpyDeviceToHost));
        if (out) {
            out->visit_count = sums[0];
            out->checksum = sums[1];
            out->fallback_bouquets = sums[2];
        }
        // Every walk makes exactly `depth` hops, so a wrapped uint32 counter shows as a shortfall.
        const unsigned __int128 expect = (unsigned __int128)g->num_active * n_walks * depth;
        if ((unsigned __int128)sums[0] != expect)
            fail(TGTP_ERR_OVERFLOW, "a uint32 visit counter overflowed");
    });
}

tgtp_status mt_walk_count(tgtp_graph* g, uint32_t depth, uint32_t n_walks, int32_t simd,
                          uint32_t* host_counters, saba_result* out) {
    return guarded([&] {
        if (!g) fail(TGTP_ERR_INVALID_ARGUMENT, "null graph");
        if (simd && n_walks % 8 != 0) fail(TGTP_ERR_INVALID_ARGUMENT, "n_walks must be a multiple of 8");
        g->counters.reserve(sizeof(uint32_t) * (g->n + 1));
        auto* c = g->counters.as<uint32_t>();
        mt_walk_run(g, depth, n_walks, simd != 0, c);
        uint64_t sums[3];
        saba_summarize(g, c, sums);
        if (host_counters)
            TGTP_CUDA(cudaMemcpy(host_counters, c, sizeof(uint32_t) * g->n, cudaMemcpyDeviceToHost));
        if (out) {
            out->visit_count = sums[0];
            out->checksum = sums[1];
            out->fallback_bouquets = 0;
        }
        const unsigned __int128 expect = (unsigned __int128)g->num_active * n_walks * depth;
        if ((unsigned __int128)sums[0] != expect)
            fail(TGTP_ERR_OVERFLOW, "a uint32 visit counter overflowed");
    });
}

tgtp_status tgtp_release_cached_memory(void) {
    return guarded([&] { cache_trim(); });
}

tgtp_status tgtp_graph_set_profiling(tgtp_graph* g, int enable) {
    return guarded([&] {
        if (!g) fail(TGTP_ERR_INVALID_ARGUMENT, "null graph");
        g->prof.clear();
        g->prof.enabled = enable != 0;
    });
}

tgtp_status tgtp_graph_set_trace(tgtp_graph* g, int enable) {
    return guarded([&] {
        if (!g) fail(TGTP_ERR_INVALID_ARGUMENT, "null graph");
        g->trace_on = enable != 0;
        g->trace_valid = false;
    });
}

tgtp_status tgtp_graph_read_trace(tgtp_graph* g, uint32_t* host_walks, uint32_t* host_rounds) {
    return guarded([&] {
        if (!g) fail(TGTP_ERR_INVALID_ARGUMENT, "null graph");
        if (!g->trace_on || !g->trace_valid)
            fail(TGTP_ERR_INVALID_ARGUMENT, "no traced run on this handle");
        const auto* t = g->trace.as<uint32_t>();
        if (host_walks)
            TGTP_CUDA(cudaMemcpyAsync(host_walks, t, sizeof(uint32_t) * g->m, cudaMemcpyDeviceToHost,
                                      g->stream));
        if (host_rounds)
            TGTP_CUDA(cudaMemcpyAsync(host_rounds, t + g->m, sizeof(uint32_t) * g->n,
                                      cudaMemcpyDeviceToHost, g->stream));
        TGTP_CUDA(cudaStreamSynchronize(g->stream));
    });
}

tgtp_status tgtp_graph_kernel_stats(tgtp_graph* g, tgtp_kernel_stat* out, int32_t cap,
                                    int32_t* count) {
    return guarded([&] {
        if (!g) fail(TGTP_ERR_INVALID_ARGUMENT, "null graph");
        g->prof.collect();
        const auto& t = g->prof.totals;
        if (count) *count = int32_t(t.size());
        for (int32_t i = 0; i < cap && i < int32_t(t.size()); ++i) {
            std::snprintf(out[i].name, sizeof(out[i].name), "%s", t[i].name.c_str());
            out[i].launches = t[i].launches;
            out[i].total_ms = t[i].total_ms;
        }
    });
}

}  // extern "C"
