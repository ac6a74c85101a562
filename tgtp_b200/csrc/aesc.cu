// tgtp() on sm_100a: the TGT+ approximate edge spanning centrality of src/aesc.h:113-551.
//
// Stages (one launch each, all on the graph's stream):
//   1. tau_kernel         per undirected edge (u <= v): the omega-eigenvector walk-length bound
//                         (calculate_taus, :164-216), written to both CSR slots.
//   2. source_kernel      persistent warps, one source at a time per warp (dynamic queue):
//                         residual push rounds until the push/walk cost test stops them
//                         (:456-503), the top-gamma edge bound (:414-442), the per-edge chi and
//                         walk count (:392-412, :508-521) and the 2-way bouquet walks (:241-391),
//                         accumulating the source's CSR row of scores (:524-525).
//   3. symmetrize_kernel  score[q] = row[q] + row[reverse slot] (:532-550).
//
// The parity forms (FP32 = the reference's own arithmetic, FP64 = every float held in double)
// keep the reference's evaluation order wherever a rounding depends on it:
//   * the push of one source is sequential over its frontier, in discovery order; the lanes of the
//     warp share one frontier vertex's adjacency (distinct neighbours, so their updates commute);
//   * float sums run in the reference's order (tau dot products per edge in index order, walk
//     lanes per bouquet lane in bouquet order, the eight lanes summed 0..7);
//   * every operation is a correctly rounded intrinsic, never contracted into an FMA.
// Max/min/integer reductions are order-free and run across lanes.
#include <cuda_bf16.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <type_traits>

#include "common.cuh"
#include "internal.hpp"

namespace tgtp {
namespace {

constexpr int kTauThreads = 128;
constexpr int kSrcWarps = 4;
constexpr int kSrcThreads = kSrcWarps * 32;
constexpr int kTopK = 16;            // register top-k used for gamma <= 16
constexpr int kTauTableRows = 64;    // rows of the eigen_t_1 power table (api.cu)
constexpr uint64_t kMaxWalks = 0xffffffffull;  // nr beyond the 32-bit grid is not supported

enum : unsigned { kErrDeadline = 1u, kErrWalkCount = 2u };

enum StatIdx {
    kStPushRounds = 0, kStPushVertices, kStPushTraversals, kStWalkEdges, kStWalkCount,
    kStWalkHops, kStFallback, kStTauIters, kStTauAmbiguous, kStCount
};

struct TauConst {
    double one_m_l1sq, b1;  // 1 - lambda_1^2, log(1/|lambda_1|)
    double one_m_l2sq, b2;  // the same for lambda_{omega-1}
};

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// get_tau (src/aesc.h:129-135).  p1/p2 in the reference's parameter order (its callers pass
// (degree(u), degree(v)) into parameters named (dv, du)).  The 1 - lambda^2 and log(1/|lambda|)
// constants are formed on the host with the same libm as the reference.
template <class Real>
__device__ int get_tau(uint32_t p1, uint32_t p2, Real epsilon, double one_m_lam2, double b,
                       Real delta, Real upsilon, unsigned long long& ambiguous) {
    const Real ed = rsub(epsilon, delta);
    const Real eps_delta = double(ed) > 0.0 ? ed : epsilon;
    const double d1 = double(p1), d2 = double(p2);
    const double x = __dsub_rn(__dsub_rn(__dadd_rn(__ddiv_rn(1.0, d2), __ddiv_rn(1.0, d1)),
                                         __ddiv_rn(__ddiv_rn(2.0, d2), d1)),
                               double(upsilon));
    const double y = __ddiv_rn(__ddiv_rn(x, double(eps_delta)), one_m_lam2);
    const double a = log(std_max(y, 1.0));
    const double q = __dsub_rn(__ddiv_rn(a, b), 1.0);
    // A last-place difference between this log and the host's can only move ceil() when q sits
    // within rounding of an integer; count such edges so a caller can see that it never happens.
    if (a != 0.0 && fabs(q - rint(q)) <= 1e-12 * fmax(1.0, fabs(q))) ++ambiguous;
    const int tau = x86_f64_to_i32(std_max(ceil(q), 1.0));
    return tau % 2 == 0 ? int(tau + 1) : int(tau);
}

// eigen_t_1[i] cast to the form's real type after k multiplications by lambda_i^2.
template <class Real>
__device__ __forceinline__ Real etab_value(const Real* tab, const double* tabd, uint32_t stride,
                                           uint32_t k, uint32_t i) {
    if (k < uint32_t(kTauTableRows)) return __ldg(tab + size_t(k) * stride + i);
    double e = __ldg(tabd + size_t(kTauTableRows - 1) * stride + i);
    const double sq = __ldg(tabd + i);
    for (uint32_t r = kTauTableRows - 1; r < k; ++r) e = __dmul_rn(e, sq);
    return from_f64<Real>(e);
}

// ---- stage 1: tau per undirected edge ------------------------------------------------------------
template <class Real>
__global__ void __launch_bounds__(kTauThreads)
tau_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ adj,
           const uint32_t* __restrict__ row_of, const uint32_t* __restrict__ rev,
           const uint32_t* __restrict__ forward, uint64_t num_forward,
           const Real* __restrict__ vec, uint32_t stride, uint32_t omega,
           const double* __restrict__ onep, const double* __restrict__ onem,
           const Real* __restrict__ etab, const double* __restrict__ etabd, Real epsilon,
           uint64_t m, TauConst c, int* __restrict__ taus, unsigned long long* __restrict__ stats) {
    unsigned long long iters = 0, ambiguous = 0;
    const Real mreal = from_u64<Real>(m);
    for (uint64_t e = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; e < num_forward;
         e += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t pos = __ldg(forward + e);
        const uint32_t u = __ldg(row_of + pos), v = __ldg(adj + pos);
        const Real* uf = vec + size_t(u) * stride;
        const Real* vf = vec + size_t(v) * stride;
        const uint32_t du = __ldg(idx + u + 1) - __ldg(idx + u);
        const uint32_t dv = __ldg(idx + v + 1) - __ldg(idx + v);
        // get_upsilon (:151-162)
        Real ups = 0;
        for (uint32_t i = 1; i + 1 < omega; ++i) {
            const Real diff = rsub(__ldg(uf + i), __ldg(vf + i));
            ups = from_f64<Real>(__dadd_rn(double(ups), __dmul_rn(double(rmul(diff, diff)),
                                                                  __ldg(onep + i))));
        }
        ups = rdiv(ups, mreal);
        int tau = get_tau<Real>(du, dv, epsilon, c.one_m_l1sq, c.b1, Real(0), Real(0), ambiguous);
        int t = 1;
        for (uint32_t k = 0;; ++k) {
            // get_delta (:137-150) with eigen_t_1 = lambda^(2(k+1))
            Real del = 0;
            for (uint32_t i = 1; i + 1 < omega; ++i) {
                const Real diff = rsub(__ldg(uf + i), __ldg(vf + i));
                const Real et = etab_value<Real>(etab, etabd, stride, k, i);
                del = from_f64<Real>(__dadd_rn(double(del), __ddiv_rn(double(rmul(rmul(diff, diff), et)),
                                                                      __ldg(onem + i))));
            }
            del = rdiv(del, mreal);
            ++iters;
            const int tp = get_tau<Real>(du, dv, epsilon, c.one_m_l2sq, c.b2, del, ups, ambiguous);
            if (t <= tp && tp < tau) {
                tau = tp;
                t += 2;
            } else {
                break;
            }
        }
        taus[pos] = tau;
        taus[__ldg(rev + pos)] = tau;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        iters += __shfl_xor_sync(kFullMask, iters, o);
        ambiguous += __shfl_xor_sync(kFullMask, ambiguous, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (iters) atomicAdd(stats + kStTauIters, iters);
        if (ambiguous) atomicAdd(stats + kStTauAmbiguous, ambiguous);
    }
}

// ---- stage 2: per-source push, edge bound and walks -----------------------------------------------
struct WalkItem {
    uint32_t pos, v, len, pad;
    unsigned long long nr;
};

template <class Real>
struct SourceParams {
    const uint32_t* idx;
    const uint32_t* adj;
    const uint32_t* deg;
    uint32_t n;
    const int* taus;
    Real* preds;
    unsigned* work;       // [0] next source, [1] error flags
    uint32_t* qbuf;       // 2 * n per warp
    WalkItem* items;      // max_degree per warp
    Real* pvec_g;         // n per warp (global tier)
    uint32_t* vis_g;      // ceil(n/32) per warp (global tier)
    size_t smem_per_warp;
    uint32_t max_degree;
    double eps;
    double logmd;         // log(m / delta), formed on the host
    int gamma;
    int* ell_out;
    unsigned long long* stats;
    uint64_t budget_ns;   // device time budget; past it every warp stops and flags a timeout
};

template <class Real>
__device__ __forceinline__ Real warp_max(Real x) {
#pragma unroll
    for (int o = 16; o; o >>= 1) x = std_max(x, __shfl_xor_sync(kFullMask, x, o));
    return x;
}
template <class Real>
__device__ __forceinline__ Real warp_min(Real x) {
#pragma unroll
    for (int o = 16; o; o >>= 1) x = std_min(x, __shfl_xor_sync(kFullMask, x, o));
    return x;
}
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long x) {
#pragma unroll
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(kFullMask, x, o);
    return x;
}

__device__ __forceinline__ bool vis_test_set(uint32_t* vis, uint32_t u) {
    const uint32_t bit = 1u << (u & 31);
    return !(atomicOr(vis + (u >> 5), bit) & bit);
}

// The real_gamma-th largest residual of the frontier (counting multiplicity) and how many of the
// chosen values equal it.  gamma <= kTopK: one pass keeping a sorted top-k per lane, then a
// warp merge.  Larger gamma: one pass per distinct value from the top.
template <class Real>
__device__ void kth_largest(const uint32_t* q, uint32_t qs, const Real* pvec, int rg, Real& t,
                            int& n_eq_taken) {
    const int lane = threadIdx.x & 31;
    if (rg <= kTopK) {
        Real L[kTopK];
#pragma unroll
        for (int j = 0; j < kTopK; ++j) L[j] = Real(-INFINITY);
        for (uint32_t i = lane; i < qs; i += 32) {
            const Real x = pvec[q[i]];
            if (x > L[kTopK - 1]) {
#pragma unroll
                for (int j = kTopK - 1; j > 0; --j) {
                    const Real prev = L[j - 1];
                    L[j] = x > prev ? prev : (x > L[j] ? x : L[j]);
                }
                L[0] = x > L[0] ? x : L[0];
            }
        }
        Real last = Real(-INFINITY);
        int run = 0;
        for (int r = 0; r < rg; ++r) {
            const Real mx = warp_max(L[0]);
            const unsigned who = __ballot_sync(kFullMask, L[0] == mx);
            if (lane == __ffs(who) - 1) {
#pragma unroll
                for (int j = 0; j < kTopK - 1; ++j) L[j] = L[j + 1];
                L[kTopK - 1] = Real(-INFINITY);
            }
            run = (r > 0 && mx == last) ? run + 1 : 1;
            last = mx;
        }
        t = last;
        n_eq_taken = run;
        return;
    }
    Real thr = Real(INFINITY);
    int remaining = rg;
    while (true) {
        Real best = Real(-INFINITY);
        unsigned cnt = 0;
        for (uint32_t i = lane; i < qs; i += 32) {
            const Real x = pvec[q[i]];
            if (x < thr) {
                if (x > best) {
                    best = x;
                    cnt = 1;
                } else if (x == best) {
                    ++cnt;
                }
            }
        }
        const Real mx = warp_max(best);
        unsigned c = best == mx ? cnt : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(kFullMask, c, o);
        if (int(c) >= remaining) {
            t = mx;
            n_eq_taken = remaining;
            return;
        }
        remaining -= int(c);
        thr = mx;
    }
}

template <class Real, bool SMEM>
__global__ void __launch_bounds__(kSrcThreads)
source_kernel(SourceParams<Real> p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t wib = threadIdx.x >> 5;
    const uint64_t gw = uint64_t(blockIdx.x) * kSrcWarps + wib;
    const uint32_t n = p.n;
    const uint32_t nwords = (n + 31) / 32;
    Real* pvec;
    uint32_t* vis;
    if (SMEM) {
        unsigned char* base = smem + size_t(wib) * p.smem_per_warp;
        pvec = reinterpret_cast<Real*>(base);
        vis = reinterpret_cast<uint32_t*>(base + ((size_t(n) * sizeof(Real) + 15) & ~size_t(15)));
    } else {
        pvec = p.pvec_g + gw * size_t(n);
        vis = p.vis_g + gw * size_t(nwords);
    }
    for (uint32_t i = lane; i < n; i += 32) pvec[i] = Real(0);
    for (uint32_t i = lane; i < nwords; i += 32) vis[i] = 0;
    uint32_t* qa = p.qbuf + gw * 2 * size_t(n);
    uint32_t* qb = qa + n;
    WalkItem* items = p.items + gw * size_t(p.max_degree);
    const uint32_t* __restrict__ idx = p.idx;
    const uint32_t* __restrict__ adj = p.adj;
    const uint32_t* __restrict__ deg = p.deg;
    unsigned long long st_rounds = 0, st_pv = 0, st_tr = 0, st_we = 0, st_wc = 0, st_wh = 0,
                       st_fb = 0;
    const uint64_t deadline = globaltimer_ns() + p.budget_ns;
    __syncwarp();

    while (true) {
        unsigned k = 0;
        if (lane == 0) k = atomicAdd(p.work, 1u);
        k = __shfl_sync(kFullMask, k, 0);
        if (k >= n) break;
        if (globaltimer_ns() > deadline) {
            if (lane == 0) atomicOr(p.work + 1, kErrDeadline);
            break;
        }
        const uint32_t src = k;
        uint32_t* q = qa;
        uint32_t* qn = qb;
        const uint32_t rb = __ldg(idx + src), re = __ldg(idx + src + 1);
        const uint32_t dsi = re - rb;
        const Real ds = from_u64<Real>(dsi);
        const Real pinit = from_f64<Real>(__ddiv_rn(1.0, double(ds)));  // preds = 1.0 / ds
        for (uint32_t pos = rb + lane; pos < re; pos += 32) p.preds[pos] = pinit;
        if (lane == 0) {
            pvec[src] = Real(1);
            q[0] = src;
        }
        uint32_t qs = 1;
        int ell = 0;
        Real gmin, gmax;
        bool timed_out = false;
        __syncwarp();
        while (true) {
            // ---- diffuse (:218-239) ----
            // Frontier vertices are fetched 32 at a time (id and row bounds per lane) and handed
            // out by shuffle; their order of processing is the frontier order.
            uint32_t qns = 0;
            st_pv += qs;
            for (uint32_t i0 = 0; i0 < qs; i0 += 32) {
                uint32_t myv = 0, myb = 0, myd = 0;
                if (i0 + lane < qs) {
                    myv = q[i0 + lane];
                    myb = __ldg(idx + myv);
                    myd = __ldg(idx + myv + 1) - myb;
                }
                const uint32_t cnt = min(32u, qs - i0);
                // first adjacency chunk of the next vertex, loaded one step ahead
                uint32_t nu = 0, nd = 1;
                {
                    const uint32_t vb0 = __shfl_sync(kFullMask, myb, 0);
                    const uint32_t vd0 = __shfl_sync(kFullMask, myd, 0);
                    if (lane < vd0) {
                        nu = __ldg(adj + vb0 + lane);
                        nd = __ldg(deg + nu);
                    }
                }
                for (uint32_t t = 0; t < cnt; ++t) {
                    const uint32_t v = __shfl_sync(kFullMask, myv, t);
                    const uint32_t vb = __shfl_sync(kFullMask, myb, t);
                    const uint32_t vd = __shfl_sync(kFullMask, myd, t);
                    const uint32_t cu = nu, cd = nd;
                    if (t + 1 < cnt) {
                        const uint32_t vb1 = __shfl_sync(kFullMask, myb, t + 1);
                        const uint32_t vd1 = __shfl_sync(kFullMask, myd, t + 1);
                        if (lane < vd1) {
                            nu = __ldg(adj + vb1 + lane);
                            nd = __ldg(deg + nu);
                        }
                    }
                    const Real r = pvec[v];
                    __syncwarp();
                    if (lane == 0) pvec[v] = Real(0);
                    __syncwarp();
                    st_tr += vd;
                    for (uint32_t c = 0; c < vd; c += 32) {
                        const uint32_t e = c + lane;
                        const bool act = e < vd;
                        uint32_t u = 0, du = 1;
                        if (act) {
                            if (c == 0) {
                                u = cu;
                                du = cd;
                            } else {
                                u = __ldg(adj + vb + e);
                                du = __ldg(deg + u);
                            }
                        }
                        const bool fresh = act && vis_test_set(vis, u);
                        const unsigned bal = __ballot_sync(kFullMask, fresh);
                        if (fresh) qn[qns + __popc(bal & ((1u << lane) - 1u))] = u;
                        qns += __popc(bal);
                        if (act) pvec[u] = radd(pvec[u], rdiv(r, from_u64<Real>(du)));
                        __syncwarp();
                    }
                }
            }
            __syncwarp();
            const Real ps = pvec[src];
            for (uint32_t pos = rb + lane; pos < re; pos += 32)
                p.preds[pos] = radd(p.preds[pos], rdiv(rsub(ps, pvec[__ldg(adj + pos)]), ds));
            for (uint32_t i = lane; i < qns; i += 32) vis[qn[i] >> 5] = 0;
            __syncwarp();
            { uint32_t* tmp = q; q = qn; qn = tmp; }
            qs = qns;
            ++ell;
            // ---- frontier statistics and the push/walk cost test (:483-502) ----
            unsigned long long pc = 0;
            Real mx = Real(0), mn = Real(1);
            for (uint32_t i = lane; i < qs; i += 32) {
                const uint32_t v = q[i];
                pc += __ldg(deg + v);
                const Real val = pvec[v];
                mx = std_max(mx, val);
                mn = std_min(mn, val);
            }
            pc = warp_sum_u64(pc);
            gmax = warp_max(mx);
            gmin = warp_min(mn);
            gmin = qs < n ? Real(0) : gmin;
            const double picost = double(pc);
            const double dse0 = __dmul_rn(double(ds), p.eps);
            const double dse2 = __dmul_rn(dse0, dse0);
            double rw = 0;
            for (uint32_t c = 0; c < dsi; c += 32) {
                const uint32_t pos = rb + c + lane;
                double nrd = 0;
                bool has = false;
                if (c + lane < dsi) {
                    const int rest = __ldg(p.taus + pos) - ell;
                    if (rest > 0) {
                        const double chi = __dmul_rn(__dmul_rn(2.0, double(rest)),
                                                     __dsub_rn(double(gmax), double(gmin)));
                        const double num = __dmul_rn(__dmul_rn(8.0, __dmul_rn(chi, chi)), p.logmd);
                        nrd = std_max(ceil(__ddiv_rn(num, dse2)), 1.0);
                        has = true;
                    }
                }
                unsigned hb = __ballot_sync(kFullMask, has);
                while (hb) {
                    const int l = __ffs(hb) - 1;
                    hb &= hb - 1;
                    rw = __dadd_rn(rw, __shfl_sync(kFullMask, nrd, l));
                }
            }
            if (picost >= __dmul_rn(25.0, rw)) break;
            if (globaltimer_ns() > deadline) {
                timed_out = true;
                break;
            }
        }
        if (timed_out) {
            if (lane == 0) atomicOr(p.work + 1, kErrDeadline);
            break;
        }
        st_rounds += ell;
        if (lane == 0 && p.ell_out) p.ell_out[src] = ell;

        // ---- edge bound (:414-442, :504-506) ----
        Real edge_max;
        if (p.gamma == 1) {
            edge_max = rmul(Real(2), gmax);
        } else {
            const int nnz = int(qs);
            const int rg = p.gamma < nnz ? p.gamma : nnz;
            uint32_t* set = qn;  // free after the last swap
            int sc = 0;
            Real gamma_max;
            if (p.gamma < nnz) {
                Real t;
                int need_eq;
                kth_largest<Real>(q, qs, pvec, rg, t, need_eq);
                int taken_eq = 0;
                for (uint32_t i0 = 0; i0 < qs && sc < rg; i0 += 32) {
                    const uint32_t i = i0 + lane;
                    uint32_t u = 0;
                    Real x = Real(-INFINITY);
                    if (i < qs) {
                        u = q[i];
                        x = pvec[u];
                    }
                    const bool gt = x > t, eq = x == t;
                    const unsigned be = __ballot_sync(kFullMask, eq);
                    const bool take_eq = eq && taken_eq + __popc(be & ((1u << lane) - 1u)) < need_eq;
                    const bool take = gt || take_eq;
                    const unsigned bt = __ballot_sync(kFullMask, take);
                    if (take) set[sc + __popc(bt & ((1u << lane) - 1u))] = u;
                    sc += __popc(bt);
                    taken_eq += __popc(__ballot_sync(kFullMask, take_eq));
                }
                gamma_max = std_min(Real(1), t);
            } else {
                for (uint32_t i = lane; i < qs; i += 32) set[i] = q[i];
                sc = int(qs);
                gamma_max = Real(0);
            }
            __syncwarp();
            edge_max = radd(gmax, gamma_max);
            for (int i = lane; i < sc; i += 32) vis_test_set(vis, set[i]);
            __syncwarp();
            Real best = edge_max;
            for (int s = 0; s < sc; ++s) {
                const uint32_t u = set[s];
                const Real pu = pvec[u];
                const uint32_t ub = __ldg(idx + u), ue = __ldg(idx + u + 1);
                for (uint32_t e = ub + lane; e < ue; e += 32) {
                    const uint32_t w = __ldg(adj + e);
                    if (vis[w >> 5] & (1u << (w & 31))) best = std_max(best, radd(pu, pvec[w]));
                }
            }
            edge_max = warp_max(best);
            __syncwarp();
            for (int i = lane; i < sc; i += 32) vis[set[i] >> 5] = 0;
            __syncwarp();
        }

        // ---- chi and walk counts per edge (:508-521) ----
        Real smax = Real(0), smin = Real(FLT_MAX);
        for (uint32_t pos = rb + lane; pos < re; pos += 32) {
            const Real x = pvec[__ldg(adj + pos)];
            smax = std_max(smax, x);
            smin = std_min(smin, x);
        }
        smax = warp_max(smax);
        smin = warp_min(smin);
        uint32_t nitems = 0;
        for (uint32_t c = 0; c < dsi; c += 32) {
            const bool has = c + lane < dsi && __ldg(p.taus + rb + c + lane) - ell > 0;
            unsigned hb = __ballot_sync(kFullMask, has);
            while (hb) {
                const int l = __ffs(hb) - 1;
                hb &= hb - 1;
                const uint32_t pos = rb + c + l;
                const uint32_t v = __ldg(adj + pos);
                const int L = __ldg(p.taus + pos) - ell;
                Real tmax = Real(0), tmin = Real(FLT_MAX);
                const uint32_t vb = __ldg(idx + v), ve = __ldg(idx + v + 1);
                for (uint32_t e = vb + lane; e < ve; e += 32) {
                    const Real x = pvec[__ldg(adj + e)];
                    tmax = std_max(tmax, x);
                    tmin = std_min(tmin, x);
                }
                tmax = warp_max(tmax);
                tmin = warp_min(tmin);
                // get_chi (:410): float terms rounded as in the reference, summed in double
                const double A = __dadd_rn(double(gmax), __ddiv_rn(double(radd(smax, tmax)), 2.0));
                const double B = __dadd_rn(A, double(rmul(Real(L - 1), edge_max)));
                const double C = __dsub_rn(__dsub_rn(B, double(smin)), double(tmin));
                const double E = __dsub_rn(C, double(rmul(Real(2 * (L - 1)), gmin)));
                const Real chi = from_f64<Real>(E);
                // nr (:519-521)
                const Real c8 = rmul(Real(8), rmul(chi, chi));
                const double num = __dmul_rn(double(c8), p.logmd);
                const Real dse = from_f64<Real>(__dmul_rn(double(ds), p.eps));
                const double den = double(rmul(dse, dse));
                const double nrd = std_max(ceil(__ddiv_rn(num, den)), 1.0);
                unsigned long long nr = (unsigned long long)nrd;
                nr += 8ull - (nr % 8ull);
                if (nr > kMaxWalks) {
                    if (lane == 0) atomicOr(p.work + 1, kErrWalkCount);
                    continue;
                }
                if (lane == 0) items[nitems] = WalkItem{pos, v, uint32_t(L), 0u, nr};
                ++nitems;
                st_we += 1;
                st_wc += nr;
                st_wh += nr * (unsigned long long)L;
            }
        }
        __syncwarp();

        // ---- 2-way bouquet walks (:241-391): four bouquets per warp, one per 8-lane group ----
        {
            const uint32_t j = lane & 7, grp = lane >> 3;
            uint32_t next = 0;
            bool has = false, start = false, primary = true;
            WalkItem it{};
            unsigned long long bi = 0;
            uint32_t len = 0, step = 0, cur = 0, cur2 = 0, sec = 0, sec2 = 0, state = 0;
            Real x = Real(0);
            while (true) {
                const unsigned need = __ballot_sync(kFullMask, !has && j == 0);
                if (!has) {
                    const uint32_t rank = __popc(need & ((1u << (grp * 8)) - 1u));
                    const uint32_t my = next + rank;
                    if (my < nitems) {
                        it = items[my];
                        has = true;
                        start = true;
                        bi = 0;
                        x = Real(0);
                        step = uint32_t(0xffffffffull / it.nr);
                    }
                }
                next += __popc(need);
                if (!__any_sync(kFullMask, has)) break;
                if (has && start) {
                    cur = src;
                    cur2 = it.v;
                    sec = (uint32_t(bi) + j + 1u) * step;
                    sec2 = sec;
                    state = sec;
                    primary = true;
                    len = 0;
                    start = false;
                }
                const unsigned z =
                    __ballot_sync(kFullMask, has && primary && (sec == 0u || sec2 == 0u));
                if (has && primary && ((z >> (grp * 8)) & 0xffu)) {
                    primary = false;
                    if (j == 0) ++st_fb;
                }
                bool item_done = false;
                if (has) {
                    const uint32_t b1 = __ldg(idx + cur), d1 = __ldg(idx + cur + 1) - b1;
                    const uint32_t b2 = __ldg(idx + cur2), d2 = __ldg(idx + cur2 + 1) - b2;
                    uint32_t k1, k2;
                    if (primary) {
                        k1 = __umulhi(sec ^ fmix32(cur), d1);
                        k2 = __umulhi(sec2 ^ fmix32(cur2), d2);
                        sec *= d1;
                        sec2 *= d2;
                    } else {
                        const uint32_t r1 = splitmix32(state);
                        const uint32_t r2 = splitmix32(state);
                        k1 = r1 % d1;
                        k2 = r2 % d2;
                    }
                    cur = __ldg(adj + b1 + k1);
                    cur2 = __ldg(adj + b2 + k2);
                    x = radd(x, rsub(pvec[cur], pvec[cur2]));
                    if (++len == it.len) {
                        bi += 8;
                        start = true;
                        item_done = bi >= it.nr;
                    }
                }
                if (__any_sync(kFullMask, item_done)) {
                    Real s = Real(0);
#pragma unroll
                    for (int b = 0; b < 8; ++b) s = radd(s, __shfl_sync(kFullMask, x, int(grp * 8 + b)));
                    if (item_done && j == 0)
                        p.preds[it.pos] = radd(p.preds[it.pos], rdiv(s, rmul(ds, from_u64<Real>(it.nr))));
                    if (item_done) has = false;
                }
            }
        }
        // ---- next source starts from an all-zero residual vector ----
        __syncwarp();
        for (uint32_t i = lane; i < qs; i += 32) pvec[q[i]] = Real(0);
        if (lane == 0) pvec[src] = Real(0);
        __syncwarp();
    }
    if (lane == 0) {
        atomicAdd(p.stats + kStPushRounds, st_rounds);
        atomicAdd(p.stats + kStPushVertices, st_pv);
        atomicAdd(p.stats + kStPushTraversals, st_tr);
        atomicAdd(p.stats + kStWalkEdges, st_we);
        atomicAdd(p.stats + kStWalkCount, st_wc);
        atomicAdd(p.stats + kStWalkHops, st_wh);
    }
    st_fb = warp_sum_u64(st_fb);
    if (lane == 0) atomicAdd(p.stats + kStFallback, st_fb);
}

// ---- stage 3: symmetrise -------------------------------------------------------------------------
template <class Real>
__global__ void symmetrize_kernel(const Real* __restrict__ preds, const uint32_t* __restrict__ sym_src,
                                  uint64_t m, float* __restrict__ out) {
    for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < m;
         q += uint64_t(gridDim.x) * blockDim.x) {
        Real s = preds[q];
        const uint32_t o = sym_src[q];
        if (o) s = radd(s, preds[o - 1]);
        out[q] = float(s);
    }
}

unsigned grid_cap(uint64_t work, int threads, int num_sms, int per_sm) {
    const uint64_t b = (work + threads - 1) / threads;
    return unsigned(std::max<uint64_t>(1, std::min<uint64_t>(b, uint64_t(num_sms) * per_sm)));
}

uint64_t deadline_from_env() {
    double s = 30.0;
    if (const char* e = std::getenv("TGTP_KERNEL_DEADLINE_S")) {
        const double v = std::atof(e);
        if (v > 0) s = v;
    }
    return uint64_t(s * 1e9);
}

template <class Real>
void run_form(tgtp_graph* g, const tgtp_config& cfg, float* out) {
    cudaStream_t s = g->stream;
    const uint64_t n = g->n, m = g->m;
    const uint32_t omega = uint32_t(cfg.omega);
    const Real* vec = std::is_same<Real, float>::value ? (const Real*)g->vec_f32.ptr
                                                        : (const Real*)g->vec_f64.ptr;
    const Real* etab = std::is_same<Real, float>::value ? (const Real*)g->etab_f.ptr
                                                         : (const Real*)g->etab.ptr;
    // host-side constants with the host libm (as the reference evaluates them)
    TauConst c;
    const double l1 = g->values[1], l2 = g->values[omega - 1];
    c.one_m_l1sq = 1.0 - (l1 * l1);
    c.b1 = std::log(double(1.0) / std::fabs(l1));
    c.one_m_l2sq = 1.0 - (l2 * l2);
    c.b2 = std::log(double(1.0) / std::fabs(l2));
    const double logmd = std::log(double(m) / cfg.delta);
    const Real eps_half = Real(cfg.epsilon / 2.0);

    g->taus.reserve(sizeof(int) * (m + 1));
    g->preds.reserve(sizeof(Real) * (m + 1));
    g->stats.reserve(sizeof(unsigned long long) * kStCount);
    g->work.reserve(sizeof(unsigned) * 4);
    auto* stats = g->stats.as<unsigned long long>();
    auto* work = g->work.as<unsigned>();
    TGTP_CUDA(cudaMemsetAsync(stats, 0, sizeof(unsigned long long) * kStCount, s));
    TGTP_CUDA(cudaMemsetAsync(work, 0, sizeof(unsigned) * 4, s));

    {
        ScopedKernel k(g->prof, s, "tau");
        tau_kernel<Real><<<grid_cap(g->num_forward, kTauThreads, g->num_sms, 16), kTauThreads, 0, s>>>(
            g->idx.as<uint32_t>(), g->adj.as<uint32_t>(), g->row_of.as<uint32_t>(),
            g->rev.as<uint32_t>(), g->forward.as<uint32_t>(), g->num_forward, vec, g->omega, omega,
            g->onep.as<double>(), g->onem.as<double>(), etab, g->etab.as<double>(), eps_half, m, c,
            g->taus.as<int>(), stats);
        TGTP_LAUNCH_CHECK("tau_kernel");
    }

    // source kernel: shared-memory residuals when four warps' vectors fit in a block
    const size_t pv_bytes = (size_t(n) * sizeof(Real) + 15) & ~size_t(15);
    const size_t vis_bytes = ((size_t((n + 31) / 32) * 4) + 15) & ~size_t(15);
    const size_t per_warp = pv_bytes + vis_bytes;
    const bool use_smem = per_warp * kSrcWarps <= size_t(200) * 1024;
    const size_t smem = use_smem ? per_warp * kSrcWarps : 0;
    auto kern = use_smem ? source_kernel<Real, true> : source_kernel<Real, false>;
    TGTP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int per_sm = 0;
    TGTP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSrcThreads, smem));
    if (per_sm < 1) fail(TGTP_ERR_UNSUPPORTED, "source kernel does not fit on an SM");
    uint64_t blocks = uint64_t(g->num_sms) * per_sm;
    blocks = std::min<uint64_t>(blocks, (n + kSrcWarps - 1) / kSrcWarps);
    const uint64_t warps = blocks * kSrcWarps;
    const size_t maxd = std::max<uint32_t>(g->max_degree, 1);
    size_t scratch = warps * (2 * size_t(n) * 4 + maxd * sizeof(WalkItem));
    if (!use_smem) scratch += warps * (size_t(n) * sizeof(Real) + size_t((n + 31) / 32) * 4);
    g->scratch.reserve(scratch + 256);
    unsigned char* base = g->scratch.as<unsigned char>();
    SourceParams<Real> p;
    p.idx = g->idx.as<uint32_t>();
    p.adj = g->adj.as<uint32_t>();
    p.deg = g->deg.as<uint32_t>();
    p.n = uint32_t(n);
    p.taus = g->taus.as<int>();
    p.preds = g->preds.as<Real>();
    p.work = work;
    p.qbuf = reinterpret_cast<uint32_t*>(base);
    base += warps * 2 * size_t(n) * 4;
    base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(base) + 15) & ~uintptr_t(15));
    p.items = reinterpret_cast<WalkItem*>(base);
    base += warps * maxd * sizeof(WalkItem);
    p.pvec_g = nullptr;
    p.vis_g = nullptr;
    if (!use_smem) {
        p.pvec_g = reinterpret_cast<Real*>(base);
        base += warps * size_t(n) * sizeof(Real);
        p.vis_g = reinterpret_cast<uint32_t*>(base);
    }
    p.smem_per_warp = per_warp;
    p.max_degree = uint32_t(maxd);
    p.eps = cfg.epsilon;
    p.logmd = logmd;
    p.gamma = cfg.gamma;
    p.ell_out = nullptr;
    p.stats = stats;
    p.budget_ns = deadline_from_env();
    {
        ScopedKernel k(g->prof, s, "source");
        kern<<<unsigned(blocks), kSrcThreads, smem, s>>>(p);
        TGTP_LAUNCH_CHECK("source_kernel");
    }
    {
        ScopedKernel k(g->prof, s, "symmetrize");
        symmetrize_kernel<Real><<<grid_cap(m, 256, g->num_sms, 8), 256, 0, s>>>(
            g->preds.as<Real>(), g->sym_src.as<uint32_t>(), m, out);
        TGTP_LAUNCH_CHECK("symmetrize_kernel");
    }
}

}  // namespace

void aesc_run(tgtp_graph* g, const tgtp_config& cfg, float* device_scores) {
    if (!(cfg.epsilon > 0 && cfg.epsilon < 1))
        fail(TGTP_ERR_INVALID_ARGUMENT, "require 0 < epsilon < 1, integer omega >= 2, integer gamma >= 1");
    if (cfg.gamma < 1)
        fail(TGTP_ERR_INVALID_ARGUMENT, "require 0 < epsilon < 1, integer omega >= 2, integer gamma >= 1");
    if (cfg.omega < 2 || uint64_t(cfg.omega) > g->n)
        fail(TGTP_ERR_INVALID_ARGUMENT, "omega must be between 2 and vertex count");
    if (g->omega == 0 || uint32_t(cfg.omega) > g->omega)
        fail(TGTP_ERR_INVALID_ARGUMENT, "eigenpairs for this omega were not uploaded");
    if (!(cfg.delta > 0)) fail(TGTP_ERR_INVALID_ARGUMENT, "delta must be positive");
    if (g->min_degree == 0)
        fail(TGTP_ERR_INVALID_ARGUMENT,
             "graph vertex IDs must be contiguous with no isolated vertices");
    if (g->has_multi_edges)
        fail(TGTP_ERR_UNSUPPORTED, "rows with repeated neighbours are not supported by tgtp_run");
    switch (cfg.precision) {
        case TGTP_PRECISION_FP32:
            if (!g->has_f32) fail(TGTP_ERR_INVALID_ARGUMENT, "FP32 form needs F32 eigenvectors");
            run_form<float>(g, cfg, device_scores);
            break;
        case TGTP_PRECISION_FP64:
            if (!g->has_f64) fail(TGTP_ERR_INVALID_ARGUMENT, "FP64 form needs F64 eigenvectors");
            run_form<double>(g, cfg, device_scores);
            break;
        default:
            fail(TGTP_ERR_UNSUPPORTED, "unknown precision form");
    }
    g->last_precision = cfg.precision;
    g->have_run = true;
}

}  // namespace tgtp

using namespace tgtp;

namespace {
void finish_run(tgtp_graph* g) {
    unsigned flags[2];
    TGTP_CUDA(cudaMemcpyAsync(flags, g->work.ptr, sizeof(flags), cudaMemcpyDeviceToHost, g->stream));
    TGTP_CUDA(cudaStreamSynchronize(g->stream));
    if (flags[1] & kErrDeadline)
        fail(TGTP_ERR_TIMEOUT, "device time budget exceeded (TGTP_KERNEL_DEADLINE_S)");
    if (flags[1] & kErrWalkCount)
        fail(TGTP_ERR_UNSUPPORTED, "a walk count exceeds the 32-bit walk grid");
}
}  // namespace

extern "C" {

tgtp_status tgtp_run_device(tgtp_graph* g, const tgtp_config* cfg, float* device_scores) {
    return guarded([&] {
        if (!g || !cfg || !device_scores) fail(TGTP_ERR_INVALID_ARGUMENT, "null argument");
        aesc_run(g, *cfg, device_scores);
    });
}

tgtp_status tgtp_run(tgtp_graph* g, const tgtp_config* cfg, float* host_scores) {
    return guarded([&] {
        if (!g || !cfg || !host_scores) fail(TGTP_ERR_INVALID_ARGUMENT, "null argument");
        g->out.reserve(sizeof(float) * (g->m + 1));
        aesc_run(g, *cfg, g->out.as<float>());
        finish_run(g);
        TGTP_CUDA(cudaMemcpyAsync(host_scores, g->out.ptr, sizeof(float) * g->m,
                                  cudaMemcpyDeviceToHost, g->stream));
        TGTP_CUDA(cudaStreamSynchronize(g->stream));
    });
}

tgtp_status tgtp_last_run_stats(tgtp_graph* g, tgtp_run_stats* out) {
    return guarded([&] {
        if (!g || !out) fail(TGTP_ERR_INVALID_ARGUMENT, "null argument");
        if (!g->have_run) fail(TGTP_ERR_INVALID_ARGUMENT, "no run on this graph yet");
        finish_run(g);
        unsigned long long st[kStCount];
        TGTP_CUDA(cudaMemcpyAsync(st, g->stats.ptr, sizeof(st), cudaMemcpyDeviceToHost, g->stream));
        TGTP_CUDA(cudaStreamSynchronize(g->stream));
        out->push_rounds = st[kStPushRounds];
        out->push_vertices = st[kStPushVertices];
        out->push_traversals = st[kStPushTraversals];
        out->walk_edges = st[kStWalkEdges];
        out->walk_count = st[kStWalkCount];
        out->walk_hops = st[kStWalkHops];
        out->fallback_bouquets = st[kStFallback];
        out->tau_iterations = st[kStTauIters];
        out->tau_ambiguous = st[kStTauAmbiguous];
    });
}

tgtp_status tgtp_last_taus(tgtp_graph* g, int32_t* host_taus) {
    return guarded([&] {
        if (!g || !host_taus) fail(TGTP_ERR_INVALID_ARGUMENT, "null argument");
        if (!g->have_run) fail(TGTP_ERR_INVALID_ARGUMENT, "no run on this graph yet");
        TGTP_CUDA(cudaMemcpyAsync(host_taus, g->taus.ptr, sizeof(int32_t) * g->m,
                                  cudaMemcpyDeviceToHost, g->stream));
        TGTP_CUDA(cudaStreamSynchronize(g->stream));
    });
}

}  // extern "C"
