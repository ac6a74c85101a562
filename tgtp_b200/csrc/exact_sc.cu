// Exact spanning centrality of sampled edges on sm_100a: the quantity of src/exact_sc.cpp:24-49
// (and scripts/paper_accuracy.py:13-54), R(u, v) = (e_u - e_v)^T L^+ (e_u - e_v) on the simple
// undirected graph of the CSR (a repeated neighbour counts once, self-loops are ignored), for graphs
// beyond a dense factorisation.  It is the accuracy reference of the approximate scores: each
// sampled slot's resistance comes from Jacobi-preconditioned conjugate gradients on the graph
// Laplacian in FP64, 32 slots at a time as the 32 columns of an n x 32 block (one 256-byte row per
// vertex, lane j of a warp = column j).
//
// One iteration is four grid-wide passes (each a kernel, so every pass sees the previous one's
// results complete):
//   spmv     lp = L p (pull over the simple neighbours of each row) and the column sums of p * lp;
//   update   alpha = rz / (p . Lp); x += alpha p; r -= alpha lp; the column sums of r;
//   project  r -= mean(r) (b is orthogonal to the constant vector, and so is every exact residual;
//            this removes the rounding drift); the column sums of r * r / d (= r . z) and r * r;
//   direct   beta = rz_new / rz; p = r / d + beta p.
// A column whose residual norm has reached tol * ||b|| takes alpha = 0 from then on, so converged
// columns stop moving while the others continue.  Column sums are FP64 atomics over one partial
// per block, so their last bits may vary between runs; the iteration is a solver, not a parity
// path, and its results are checked against the dense oracle to 1e-9.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace tgtp {
namespace {

constexpr int kCols = 32;      // slots per batch (block columns)
constexpr int kScThreads = 256;
constexpr int kScWarps = kScThreads / 32;

// Column sums: every warp keeps its lane's partial (lane = column), the block adds its warps'
// partials in shared memory and lane j of warp 0 adds the block's total to out[j].
__device__ __forceinline__ void block_column_sum(double v, double* out) {
    __shared__ double part[kScWarps][kCols];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    part[w][lane] = v;
    __syncthreads();
    if (w == 0) {
        double s = 0;
#pragma unroll
        for (int k = 0; k < kScWarps; ++k) s += part[k][lane];
        if (s != 0.0) atomicAdd(out + lane, s);
    }
}

// Simple degree: neighbours other than the vertex itself, each distinct id once (rows are sorted).
__global__ void simple_degree_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ adj,
                                     uint32_t n, double* __restrict__ ds) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        uint32_t c = 0, prev = 0xffffffffu;
        for (uint32_t q = idx[u]; q < idx[u + 1]; ++q) {
            const uint32_t w = adj[q];
            if (w != u && w != prev) ++c;
            prev = w;
        }
        ds[u] = double(c);
    }
}

// Right-hand sides of one batch: column j is e_u - e_v for slot slots[j] (zero for padding columns
// and self-loop slots); r = b, p = z = b / d, rz = b . z, bb = b . b.  x, r, p are zero on entry.
__global__ void sc_init_kernel(const uint32_t* __restrict__ slots, uint32_t count,
                               const uint32_t* __restrict__ row_of, const uint32_t* __restrict__ adj,
                               const double* __restrict__ ds, double* __restrict__ r,
                               double* __restrict__ p, uint32_t* __restrict__ ends,
                               double* __restrict__ sums) {
    const uint32_t j = threadIdx.x;
    if (j >= kCols) return;
    double rz = 0, bb = 0;
    uint32_t u = 0xffffffffu, v = 0xffffffffu;
    if (j < count) {
        const uint32_t q = slots[j];
        u = row_of[q];
        v = adj[q];
        if (u != v) {
            r[size_t(u) * kCols + j] = 1.0;
            r[size_t(v) * kCols + j] = -1.0;
            p[size_t(u) * kCols + j] = 1.0 / ds[u];
            p[size_t(v) * kCols + j] = -1.0 / ds[v];
            rz = 1.0 / ds[u] + 1.0 / ds[v];
            bb = 2.0;
        }
    }
    ends[2 * j] = u;
    ends[2 * j + 1] = v;
    sums[0 * kCols + j] = rz;  // rz
    sums[1 * kCols + j] = bb;  // b . b
    sums[4 * kCols + j] = bb;  // r . r (so the first test sees an unconverged column)
}

// sums layout (kCols doubles each): 0 rz, 1 b.b, 2 p.Lp, 3 sum of r, 4 r.r, 5 rz_new, 6 (r.r)_new
__global__ void __launch_bounds__(kScThreads)
sc_spmv_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ adj, uint32_t n,
               const double* __restrict__ ds, const double* __restrict__ p,
               double* __restrict__ lp, double* __restrict__ sums) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    double dot = 0;
    for (uint32_t u = warp; u < n; u += nw) {
        const uint32_t b = __ldg(idx + u), e = __ldg(idx + u + 1);
        double acc = 0;
        uint32_t prev = 0xffffffffu;
        for (uint32_t c = b; c < e; c += 32) {
            const uint32_t w = c + lane < e ? __ldg(adj + c + lane) : 0xffffffffu;
            const uint32_t pw = __shfl_up_sync(kFullMask, w, 1);
            const uint32_t before = lane == 0 ? prev : pw;
            const bool keep = w != 0xffffffffu && w != u && w != before;
            unsigned live = __ballot_sync(kFullMask, keep);
            prev = __shfl_sync(kFullMask, w, 31);
            while (live) {
                const int l = __ffs(live) - 1;
                live &= live - 1;
                const uint32_t t = __shfl_sync(kFullMask, w, l);
                acc += p[size_t(t) * kCols + lane];
            }
        }
        const double pu = p[size_t(u) * kCols + lane];
        const double y = ds[u] * pu - acc;
        lp[size_t(u) * kCols + lane] = y;
        dot += pu * y;
    }
    block_column_sum(dot, sums + 2 * kCols);
}

__device__ __forceinline__ bool sc_converged(const double* sums, uint32_t j, double tol2) {
    return sums[4 * kCols + j] <= tol2 * sums[1 * kCols + j];
}

__global__ void __launch_bounds__(kScThreads)
sc_update_kernel(uint32_t n, const double* __restrict__ p, const double* __restrict__ lp,
                 double* __restrict__ x, double* __restrict__ r, double* __restrict__ sums,
                 double tol2) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const double rz = sums[0 * kCols + lane], plp = sums[2 * kCols + lane];
    const double alpha = (sc_converged(sums, lane, tol2) || !(plp > 0.0)) ? 0.0 : rz / plp;
    double rs = 0;
    for (uint32_t u = warp; u < n; u += nw) {
        const size_t o = size_t(u) * kCols + lane;
        x[o] += alpha * p[o];
        const double rv = r[o] - alpha * lp[o];
        r[o] = rv;
        rs += rv;
    }
    block_column_sum(rs, sums + 3 * kCols);
}

__global__ void __launch_bounds__(kScThreads)
sc_project_kernel(uint32_t n, const double* __restrict__ ds, double* __restrict__ r,
                  const double* sums_in, double* sums_out) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const double mean = sums_in[3 * kCols + lane] / double(n);
    double rz = 0, rr = 0;
    for (uint32_t u = warp; u < n; u += nw) {
        const size_t o = size_t(u) * kCols + lane;
        const double rv = r[o] - mean;
        r[o] = rv;
        const double d = ds[u];
        rz += d > 0.0 ? rv * rv / d : 0.0;  // a vertex with no simple neighbour keeps z = 0
        rr += rv * rv;
    }
    block_column_sum(rz, sums_out + 0);
    __syncthreads();
    block_column_sum(rr, sums_out + kCols);
}

__global__ void __launch_bounds__(kScThreads)
sc_direct_kernel(uint32_t n, const double* __restrict__ ds, const double* __restrict__ r,
                 double* __restrict__ p, const double* __restrict__ sums, double beta_guard) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const double rz = sums[0 * kCols + lane], rz_new = sums[5 * kCols + lane];
    const double beta = rz > beta_guard ? rz_new / rz : 0.0;
    for (uint32_t u = warp; u < n; u += nw) {
        const size_t o = size_t(u) * kCols + lane;
        const double d = ds[u];
        p[o] = (d > 0.0 ? r[o] / d : 0.0) + beta * p[o];
    }
}

// rz <- rz_new, r.r <- (r.r)_new, and the accumulators of the next iteration cleared.
__global__ void sc_roll_kernel(double* __restrict__ sums) {
    const uint32_t j = threadIdx.x;
    if (j >= kCols) return;
    sums[0 * kCols + j] = sums[5 * kCols + j];
    sums[4 * kCols + j] = sums[6 * kCols + j];
    sums[2 * kCols + j] = 0.0;
    sums[3 * kCols + j] = 0.0;
    sums[5 * kCols + j] = 0.0;
    sums[6 * kCols + j] = 0.0;
}

__global__ void sc_answer_kernel(const double* __restrict__ x, const uint32_t* __restrict__ ends,
                                 uint32_t count, double* __restrict__ out) {
    const uint32_t j = threadIdx.x;
    if (j >= count) return;
    const uint32_t u = ends[2 * j], v = ends[2 * j + 1];
    out[j] = u == v ? 0.0 : x[size_t(u) * kCols + j] - x[size_t(v) * kCols + j];
}

}  // namespace

void exact_sc_slots(tgtp_graph* g, const uint32_t* host_slots, uint32_t count, double tol,
                    uint32_t max_iter, double* host_out, uint32_t* host_iters) {
    if (count == 0) return;
    if (!(tol > 0) || max_iter == 0) fail(TGTP_ERR_INVALID_ARGUMENT, "require tol > 0 and max_iter > 0");
    for (uint32_t i = 0; i < count; ++i)
        if (host_slots[i] >= g->m) fail(TGTP_ERR_INVALID_ARGUMENT, "slot id out of range");
    cudaStream_t s = g->stream;
    const uint32_t n = uint32_t(g->n);
    const size_t blk = sizeof(double) * size_t(n) * kCols;
    DeviceBuffer ds, x, r, p, lp, sums, slots, ends, out;
    ds.reserve(sizeof(double) * n);
    x.reserve(blk);
    r.reserve(blk);
    p.reserve(blk);
    lp.reserve(blk);
    sums.reserve(sizeof(double) * kCols * 8);
    slots.reserve(sizeof(uint32_t) * kCols);
    ends.reserve(sizeof(uint32_t) * 2 * kCols);
    out.reserve(sizeof(double) * count);
    const unsigned dblocks = unsigned(std::min<uint64_t>((n + 255) / 256, 8u * g->num_sms));
    simple_degree_kernel<<<dblocks ? dblocks : 1, 256, 0, s>>>(g->idx.as<uint32_t>(),
                                                               g->adj.as<uint32_t>(), n,
                                                               ds.as<double>());
    TGTP_LAUNCH_CHECK("simple_degree_kernel");
    const unsigned grid = unsigned(std::max<uint64_t>(
        1, std::min<uint64_t>((uint64_t(n) + kScWarps - 1) / kScWarps, uint64_t(g->num_sms) * 8)));
    const double tol2 = tol * tol;
    auto* S = sums.as<double>();
    std::vector<double> hs(kCols * 8);
    for (uint32_t b0 = 0; b0 < count; b0 += kCols) {
        const uint32_t bc = std::min<uint32_t>(kCols, count - b0);
        TGTP_CUDA(cudaMemsetAsync(x.ptr, 0, blk, s));
        TGTP_CUDA(cudaMemsetAsync(r.ptr, 0, blk, s));
        TGTP_CUDA(cudaMemsetAsync(p.ptr, 0, blk, s));
        TGTP_CUDA(cudaMemsetAsync(S, 0, sizeof(double) * kCols * 8, s));
        TGTP_CUDA(cudaMemcpyAsync(slots.ptr, host_slots + b0, sizeof(uint32_t) * bc,
                                  cudaMemcpyHostToDevice, s));
        sc_init_kernel<<<1, kCols, 0, s>>>(slots.as<uint32_t>(), bc, g->row_of.as<uint32_t>(),
                                           g->adj.as<uint32_t>(), ds.as<double>(), r.as<double>(),
                                           p.as<double>(), ends.as<uint32_t>(), S);
        TGTP_LAUNCH_CHECK("sc_init_kernel");
        uint32_t it = 0;
        bool done = false;
        while (!done) {
            if (it >= max_iter)
                fail(TGTP_ERR_TIMEOUT, "conjugate gradients did not converge within max_iter");
            sc_spmv_kernel<<<grid, kScThreads, 0, s>>>(g->idx.as<uint32_t>(), g->adj.as<uint32_t>(),
                                                       n, ds.as<double>(), p.as<double>(),
                                                       lp.as<double>(), S);
            sc_update_kernel<<<grid, kScThreads, 0, s>>>(n, p.as<double>(), lp.as<double>(),
                                                         x.as<double>(), r.as<double>(), S, tol2);
            // rz_new and (r.r)_new go to sums 5 and 6
            sc_project_kernel<<<grid, kScThreads, 0, s>>>(n, ds.as<double>(), r.as<double>(), S,
                                                          S + 5 * kCols);
            sc_direct_kernel<<<grid, kScThreads, 0, s>>>(n, ds.as<double>(), r.as<double>(),
                                                         p.as<double>(), S, 1e-300);
            sc_roll_kernel<<<1, kCols, 0, s>>>(S);
            TGTP_LAUNCH_CHECK("exact spanning centrality iteration");
            ++it;
            if (it % 8 == 0 || it >= max_iter) {
                TGTP_CUDA(cudaMemcpyAsync(hs.data(), S, sizeof(double) * kCols * 8,
                                          cudaMemcpyDeviceToHost, s));
                TGTP_CUDA(cudaStreamSynchronize(s));
                done = true;
                for (uint32_t j = 0; j < kCols; ++j)
                    if (!(hs[4 * kCols + j] <= tol2 * hs[1 * kCols + j])) done = false;
            }
        }
        sc_answer_kernel<<<1, kCols, 0, s>>>(x.as<double>(), ends.as<uint32_t>(), bc,
                                             out.as<double>() + b0);
        TGTP_LAUNCH_CHECK("sc_answer_kernel");
        if (host_iters) host_iters[b0 / kCols] = it;
    }
    TGTP_CUDA(cudaMemcpyAsync(host_out, out.ptr, sizeof(double) * count, cudaMemcpyDeviceToHost, s));
    TGTP_CUDA(cudaStreamSynchronize(s));
}

}  // namespace tgtp

extern "C" tgtp_status tgtp_exact_sc_slots(tgtp_graph* g, const uint32_t* host_slots, uint32_t count,
                                           double tol, uint32_t max_iter, double* host_resistance,
                                           uint32_t* host_iterations) {
    using namespace tgtp;
    return guarded([&] {
        if (!g || (count && (!host_slots || !host_resistance)))
            fail(TGTP_ERR_INVALID_ARGUMENT, "null argument");
        exact_sc_slots(g, host_slots, count, tol, max_iter, host_resistance, host_iterations);
    });
}
