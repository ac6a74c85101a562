// tgtp() on sm_100a: the TGT+ approximate edge spanning centrality of src/aesc.h:113-551.
//
// Stages (all on the graph's stream, consecutive kernels joined by programmatic dependent launch):
//   1. tau per undirected edge (u <= v): the omega-eigenvector walk-length bound (calculate_taus,
//      :164-216), written to both CSR slots; rows with a slot of tau > 1 are listed.
//        FP32 form           tau_kernel<float>: the reference's sequential sums, lane per edge.
//        FP64 / mixed forms  tau_sums_kernel (eight lanes per edge gather the rows) then
//                            tau_bound_kernel (lane per edge evaluates the bound).
//   2. the listed sources: push rounds until the push/walk cost test stops them (:456-503), the
//      top-gamma edge bound (:414-442), the per-edge chi and walk count (:392-412, :508-521) and
//      the 2-way bouquet walks (:241-391), accumulating each source's CSR row (:524-525).
//        source_kernel       persistent warps, one source at a time per warp;
//        push_block_kernel   mixed form on large graphs: the push of 32 sources per CTA as a
//                            pull product, then source_kernel for the rest (PrePush mode).
//   3. finish_kernel: score[q] = row[q] + row[reverse slot] (:532-550), with the rows of unlisted
//      sources (every tau <= 1: one push round, no walks) in closed form.
//
// The parity forms (FP32 = the reference's own arithmetic, FP64 = every real held in double)
// keep the reference's evaluation order wherever a rounding depends on it:
//   * the push of one source is sequential over its frontier, in discovery order; the lanes of the
//     warp share one frontier vertex's adjacency (distinct neighbours update distinct words; a run
//     of one repeated neighbour is applied by its first lane, one add per repeat, in order);
//   * float sums run in the reference's order (walk lanes per bouquet lane in bouquet order, the
//     eight lanes summed 0..7; the FP32 form's tau dot products per edge in index order, the FP64
//     form's in its fixed eight-way split);
//   * every operation is a correctly rounded intrinsic, never contracted into an FMA except the
//     FP64 form's tau terms, which are defined as fused multiply-adds.
// Max/min/integer reductions are order-free and run across lanes.
#include <cuda_bf16.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <map>
#include <memory>
#include <vector>
#include <mutex>
#include <tuple>
#include <type_traits>

#include <cub/device/device_radix_sort.cuh>

#include "common.cuh"
#include "internal.hpp"

namespace tgtp {
namespace {

constexpr int kTauThreads = 32;
constexpr int kSrcMaxThreads = 128;
constexpr int kPushAhead = 4;         // adjacency chunks loaded ahead in the push
constexpr int kB = 4;                 // 32-wide chunks per pipelined load step
constexpr int kTopK = 16;            // register top-k used for gamma <= 16
// per-warp shared scratch of the chi step: 64 u64 max/min images + 33 + 32 u32 slot offsets
constexpr size_t kAccBytes = 1280;
constexpr int kTauTableRows = 64;    // rows of the eigen_t_1 power table (api.cu)
constexpr uint64_t kMaxWalks = 0xffffffffull;  // nr beyond the 32-bit grid is not supported

enum : unsigned { kErrDeadline = 1u, kErrWalkCount = 2u };

enum StatIdx {
    kStPushRounds = 0, kStPushVertices, kStPushTraversals, kStWalkEdges, kStWalkCount,
    kStWalkHops, kStFallback, kStTauIters, kStTauAmbiguous, kStPhase0,
    kStCount = kStPhase0 + 8
};
// The run counters are striped over kStStripes copies (block index modulo kStStripes) so that the
// warps of a launch do not all meet on one address; the host adds the copies up.
constexpr int kStStripes = 32;
static_assert(kStCount <= kRunStatSlots, "aesc_read_stats writes kStCount counters");

// Forms with their own tuned source-kernel layout on a handle: FP32, FP64, MIXED over F32 rows,
// MIXED over BF16 rows.  A layout is (kLayoutSmem if the residual vectors live in shared memory) |
// warps per block; 0 = the default rule.
constexpr uint16_t kLayoutSmem = 0x100;
constexpr uint16_t kLayoutBlock = 0x200;  // mixed form: multi-source block push
// parity forms: bit 0x400 set = the windowed sequential push, 0x800 = one vertex at a time (neither
// set: the default rule, by average degree)
constexpr uint16_t kLayoutWindow = 0x400;
constexpr uint16_t kLayoutNoWindow = 0x800;
// block push: the frontier size below which a round is compacted, as m / list_div, in bits 12-13
// (0 = the default list_div of 4, 1 = 2, 2 = 16, 3 = never compacted)
constexpr int kLayoutListShift = 12;
inline uint32_t layout_list_div(uint16_t layout) {
    switch ((layout >> kLayoutListShift) & 3) {
        case 1: return 2;
        case 2: return 16;
        case 3: return 0;
        default: return 4;
    }
}
inline int form_key(const tgtp_config& cfg) {
    if (cfg.precision == TGTP_PRECISION_FP32) return 0;
    if (cfg.precision == TGTP_PRECISION_FP64) return 1;
    return cfg.vec_dtype == TGTP_VEC_BF16 ? 3 : 2;
}

// The run's work words ([0] next list entry, [1] error flags, [2] list length, [3] unused) sit
// behind the striped counters in the same buffer, and the per-row marks behind them.
inline unsigned* run_work(tgtp_graph* g) {
    return reinterpret_cast<unsigned*>(g->stats.as<unsigned char>() +
                                       sizeof(unsigned long long) * kStCount * kStStripes);
}

__device__ __forceinline__ void stat_add(unsigned long long* stats, int i, unsigned long long v) {
    if (v) atomicAdd(stats + size_t(blockIdx.x % kStStripes) * kStCount + i, v);
}

struct TauConst {
    double one_m_l1sq, b1;  // 1 - lambda_1^2, log(1/|lambda_1|)
    double one_m_l2sq, b2;  // the same for lambda_{omega-1}
};

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Programmatic dependent launch: a kernel lets the next one in the stream start its blocks early
// (launch_dependents) and the next one waits for it to finish, with its memory visible, before it
// touches its results (wait).  Without the launch attribute wait returns at once.
__device__ __forceinline__ void pdl_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

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

// Rows whose every tau is at most 1 stop after their first push round: with ell = 1 every slot has
// rest = tau - ell <= 0, so rwcost = 0 <= picost (src/aesc.h:483-502) and no slot walks
// (:508-526).  Their scores follow from the closed-form first round and they skip the source
// kernel.  The tau kernels mark each row that has a slot with tau > 1 (mark[r] == epoch) and append
// it, once per run, to the list the source kernel claims its sources from.
struct RowMarks {
    uint32_t* mark;
    uint32_t* list;
    unsigned* len;
    uint32_t epoch;
};

__device__ __forceinline__ void mark_row(const RowMarks& rm, uint32_t r) {
    if (*reinterpret_cast<volatile const uint32_t*>(rm.mark + r) == rm.epoch) return;
    if (atomicExch(rm.mark + r, rm.epoch) != rm.epoch) rm.list[atomicAdd(rm.len, 1u)] = r;
}

// ---- stage 1: tau per undirected edge ------------------------------------------------------------
// A warp takes 32 forward slots (one lane each) and sweeps the eigen index i in chunks of 32.  For
// each chunk the 32 edges' x_u and x_v pieces are copied into shared memory with asynchronous
// copies (every copy of the chunk in flight at once, coalesced 128/256-byte rows), double buffered
// so the next chunk streams in while the lanes consume the current one from odd-stride tiles
// (conflict-free).  Each lane keeps its edge's sums in index order, exactly as the reference does:
// the first sweep carries upsilon and the first delta term together (two independent chains), any
// further delta iteration takes one more sweep.
__device__ __forceinline__ void cp_async_elem(void* smem_dst, const void* gsrc, int bytes) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gsrc) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// x / y for a positive divisor known in advance, correctly rounded (round to nearest even), with
// Markstein's method (P. Markstein, IBM J. Res. Dev. 34(1), 1990): q0 = x * r with r = RN(1/y) and
// one correction q1 = q0 + r * (x - q0 y), remainders exact by FMA.  The result is then checked:
// with rho = x - q1 y exact, q1 = RN(x / y) when |rho| < y * (half the gap from q1 to its
// neighbour on x / y's side): half an ulp of q1, a quarter ulp below a power of two.  Whenever the
// check cannot prove it (x zero or negative, q1 out of the safe exponent range, a divisor the host
// marked with r = NaN), the quotient comes from the correctly rounded division instead.
__device__ __forceinline__ double div_fixed(double x, double y, double r) {
    const double q0 = __dmul_rn(x, r);
    const double q1 = __fma_rn(__fma_rn(-q0, y, x), r, q0);
    const double rho = __fma_rn(-q1, y, x);
    const unsigned hi = unsigned(__double2hiint(q1));
    const unsigned e = hi >> 20;  // sign bit clear for positive q1
    double half = __hiloint2double(int((e - 53u) << 20), 0);
    if (((hi & 0xfffffu) | unsigned(__double2loint(q1))) == 0u && rho < 0.0) half *= 0.5;
    const bool ok = (e - 65u) < (0x600u - 65u) && fabs(rho) < __dmul_rn(y, half);
    return ok ? q1 : __ddiv_rn(x, y);
}

template <class Real>
__global__ void __launch_bounds__(kTauThreads)
tau_kernel(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ adj,
           const uint32_t* __restrict__ row_of, const uint32_t* __restrict__ rev,
           const uint32_t* __restrict__ forward, uint64_t num_forward,
           const Real* __restrict__ vec, uint32_t stride, uint32_t omega,
           const double* __restrict__ onep_g, const double* __restrict__ onem_g,
           const Real* __restrict__ etab, const double* __restrict__ etabd, Real epsilon,
           uint64_t m, TauConst c, int* __restrict__ taus, RowMarks rm,
           unsigned long long* __restrict__ stats) {
    constexpr uint32_t CH = 128 / sizeof(Real);  // chunk: one 128-byte row piece
    constexpr uint32_t LD = CH + 1;              // odd tile stride: conflict-free own-row reads
    extern __shared__ __align__(16) unsigned char tsm[];
    pdl_launch_dependents();
    const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t wpb = blockDim.x >> 5;
    // per index: (1 + lambda_i, 1 - lambda_i) and (RN(1 / (1 - lambda_i)), eigen_t_1 row 0)
    double2* cA = reinterpret_cast<double2*>(tsm);
    double2* cB = cA + omega;
    Real* tiles = reinterpret_cast<Real*>(cB + omega) + size_t(wib) * 4 * 32 * LD;  // [2][U,V][32][LD]
    for (uint32_t i = threadIdx.x; i < omega; i += blockDim.x) {
        const double y = onem_g[i];
        const double r = (y > 1e-150 && y < 8.0) ? __drcp_rn(y) : __longlong_as_double(0x7ff8000000000000ull);
        cA[i] = make_double2(onep_g[i], y);
        cB[i] = make_double2(r, double(etab[i]));
    }
    __syncthreads();
    unsigned long long iters = 0, ambiguous = 0;
    const Real mreal = from_u64<Real>(m);
    const uint64_t nw = uint64_t(gridDim.x) * wpb;
    const uint32_t nchunks = (omega + CH - 1) / CH;
    // lanes stage CH consecutive indices of 32 / CH edges per step
    constexpr uint32_t EPS = 32 / CH;  // edges per staging step (1 for float, 2 for double)
    const uint32_t sub = lane / CH, col = lane % CH;
    for (uint64_t base = (uint64_t(blockIdx.x) * wpb + wib) * 32; base < num_forward; base += nw * 32) {
        const uint64_t e = base + lane;
        const bool act = e < num_forward;
        uint32_t pos = 0, u = 0, v = 0, du = 0, dv = 0;
        if (act) {
            pos = __ldg(forward + e);
            u = __ldg(row_of + pos);
            v = __ldg(adj + pos);
            du = __ldg(idx + u + 1) - __ldg(idx + u);
            dv = __ldg(idx + v + 1) - __ldg(idx + v);
        }
        const uint32_t cnt = uint32_t(min(uint64_t(32), num_forward - base));
        auto stage = [&](uint32_t chunk, uint32_t buf) {
            Real* U = tiles + size_t(buf) * 2 * 32 * LD;
            Real* V = U + 32 * LD;
            const uint32_t i = chunk * CH + col;
            for (uint32_t t0 = 0; t0 < cnt; t0 += EPS) {
                const uint32_t t = t0 + sub;
                const uint32_t ut = __shfl_sync(kFullMask, u, t & 31u);
                const uint32_t vt = __shfl_sync(kFullMask, v, t & 31u);
                if (t < cnt && i < omega) {
                    cp_async_elem(U + t * LD + col, vec + size_t(ut) * stride + i, int(sizeof(Real)));
                    cp_async_elem(V + t * LD + col, vec + size_t(vt) * stride + i, int(sizeof(Real)));
                }
            }
            cp_async_commit();
        };
        Real ups = 0, del = 0;
        int tau = 0, t = 1;
        bool done = !act;
        for (uint32_t k = 0; __any_sync(kFullMask, !done); ++k) {
            del = Real(0);
            stage(0, 0);
            for (uint32_t ch = 0; ch < nchunks; ++ch) {
                if (ch + 1 < nchunks) {
                    stage(ch + 1, (ch + 1) & 1);
                    cp_async_wait<1>();
                } else {
                    cp_async_wait<0>();
                }
                __syncwarp();
                if (!done) {
                    const Real* U = tiles + size_t(ch & 1) * 2 * 32 * LD + lane * LD;
                    const Real* V = U + 32 * LD;
                    const uint32_t i0 = ch * CH;
                    const uint32_t lo = i0 == 0 ? 1u : 0u;
                    const uint32_t hi = min(CH, omega - 1 - i0);  // indices i < omega - 1
                    // get_upsilon (:151-162) with get_delta (:137-150) at eigen_t_1 = lambda^2,
                    // or get_delta alone at lambda^(2(k+1))
                    auto term0 = [&](uint32_t j) {
                        const uint32_t i = i0 + j;
                        const Real d = rsub(U[j], V[j]);
                        const Real d2 = rmul(d, d);
                        const double2 a = cA[i], b = cB[i];
                        ups = from_f64<Real>(__dadd_rn(double(ups), __dmul_rn(double(d2), a.x)));
                        del = from_f64<Real>(__dadd_rn(
                            double(del), div_fixed(double(rmul(d2, Real(b.y))), a.y, b.x)));
                    };
                    auto termk = [&](uint32_t j) {
                        const uint32_t i = i0 + j;
                        const Real d = rsub(U[j], V[j]);
                        const Real et = etab_value<Real>(etab, etabd, stride, k, i);
                        const double2 a = cA[i], b = cB[i];
                        del = from_f64<Real>(__dadd_rn(
                            double(del), div_fixed(double(rmul(rmul(d, d), et)), a.y, b.x)));
                    };
                    if (k == 0) {
                        if (lo == 0 && hi == CH) {
#pragma unroll
                            for (uint32_t j = 0; j < CH; ++j) term0(j);
                        } else {
                            for (uint32_t j = lo; j < hi; ++j) term0(j);
                        }
                    } else {
                        for (uint32_t j = lo; j < hi; ++j) termk(j);
                    }
                }
                __syncwarp();
            }
            if (!done) {
                if (k == 0) {
                    ups = rdiv(ups, mreal);
                    tau = get_tau<Real>(du, dv, epsilon, c.one_m_l1sq, c.b1, Real(0), Real(0), ambiguous);
                }
                del = rdiv(del, mreal);
                ++iters;
                const int tp = get_tau<Real>(du, dv, epsilon, c.one_m_l2sq, c.b2, del, ups, ambiguous);
                if (t <= tp && tp < tau) {
                    tau = tp;
                    t += 2;
                } else {
                    done = true;
                    taus[pos] = tau;
                    taus[__ldg(rev + pos)] = tau;
                    if (tau > 1) {
                        mark_row(rm, u);
                        mark_row(rm, v);
                    }
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        iters += __shfl_xor_sync(kFullMask, iters, o);
        ambiguous += __shfl_xor_sync(kFullMask, ambiguous, o);
    }
    if (lane == 0) {
        stat_add(stats, kStTauIters, iters);
        stat_add(stats, kStTauAmbiguous, ambiguous);
    }
}

// ---- stage 1 helpers of the mixed form: compensated FP32 sums, FP64 bound, fixed-point residuals
// d_i^2 = (x_u[i] - x_v[i])^2 and the weighted terms d_i^2 (1 + lambda_i) and
// d_i^2 lambda_i^(2(k+1)) / (1 - lambda_i) are formed in FP32 from F32 or BF16 eigenvectors; the
// bound itself (get_tau: logs, ceil, odd rounding, the delta iteration) is evaluated in FP64.

__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    const float bp = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bp)), __fsub_rn(b, bp));
}

// Residual arithmetic of the mixed form's push: the residual a vertex u receives in a round is the
// exact integer sum of its frontier neighbours' residuals in 2^-62 fixed point, divided (rounding
// down) by deg(u), then rounded once to FP32.  The sum does not depend on the order of the
// additions, so the per-warp push and the multi-source block push give the same bits.  Residuals
// never exceed 1 and a round conserves their total, so no sum exceeds 2^62.
constexpr unsigned long long kFixOne = 1ull << 62;
__device__ __forceinline__ unsigned long long to_fixed(float r) {
    return __float2ull_rn(__fmul_rn(r, 0x1p62f));
}
__device__ __forceinline__ float from_fixed(unsigned long long s, uint32_t d) {
    return __fmul_rn(__ull2float_rn(s / d), 0x1p-62f);
}

__device__ __forceinline__ float vec_load(const float* p) { return __ldg(p); }
__device__ __forceinline__ float vec_load(const __nv_bfloat16* p) {
    return __bfloat162float(__ushort_as_bfloat16(__ldg(reinterpret_cast<const unsigned short*>(p))));
}

// get_tau (src/aesc.h:129-135) in FP64 for the mixed form (no bit-level parity asked): the degree
// terms from reciprocals, one division and the precomputed 1 / log(1/|lambda|).
__device__ __forceinline__ int get_tau_mixed(double inv1, double inv2, double epsilon,
                                             double one_m_lam2, double inv_b, double delta,
                                             double ups) {
    const double ed = epsilon - delta;
    const double eps_delta = ed > 0.0 ? ed : epsilon;
    const double x = (inv2 + inv1) - 2.0 * inv2 * inv1 - ups;
    const double a = log(std_max(x / (eps_delta * one_m_lam2), 1.0));
    const int tau = x86_f64_to_i32(std_max(ceil(a * inv_b - 1.0), 1.0));
    return tau % 2 == 0 ? tau + 1 : tau;
}

// Error-free combination of the eight partial sums of a lane group (TwoSum tree, the rounding
// errors carried and added back).
__device__ __forceinline__ double group_reduce(float a) {
    float ca = 0.f;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
        const float a2 = __shfl_xor_sync(kFullMask, a, o);
        const float ca2 = __shfl_xor_sync(kFullMask, ca, o);
        float t, e;
        two_sum(a, a2, t, e);
        a = t;
        ca = __fadd_rn(__fadd_rn(ca, ca2), e);
    }
    return double(a) + double(ca);
}

// ---- stage 1 (FP64 and mixed forms): tau with eight lanes per edge ---------------------------------
// A warp takes four forward slots at a time, one per group of eight lanes.  Lane s of a group owns
// the index pieces {C j + P s, ..., C j + P s + P - 1} of the slot's two eigen rows (P = 2 FP64,
// 4 F32, 8 BF16 elements: one 16-byte load per row and piece; C = 8 P) and accumulates the terms
// d_i^2 w_i over them with fused multiply-adds, in index order, where d_i = x_u[i] - x_v[i] and
// w_i = 1 + lambda_i (upsilon, src/aesc.h:151-162) or lambda_i^(2(k+1)) / (1 - lambda_i) (delta_k,
// :137-150).  The weights are exactly zero at the indices the reference leaves out (0 and
// omega - 1) and past omega, so those terms add nothing.  The eight partial sums are combined by a
// fixed tree: ((S0 + S1) + (S2 + S3)) + ((S4 + S5) + (S6 + S7)) in FP64 for the FP64 form, the
// compensated group_reduce into FP64 for the mixed form.  The bound and the delta iteration follow
// :164-216 (get_tau, t += 2 while t <= tau' < tau).
template <class Vec> struct Split;
template <> struct Split<double> {
    static constexpr uint32_t P = 2;
    using Part = double;
};
template <> struct Split<float> {
    static constexpr uint32_t P = 4;
    using Part = float;
};
template <> struct Split<__nv_bfloat16> {
    static constexpr uint32_t P = 8;
    using Part = float;
};

// P consecutive elements starting at i0 (a multiple of P below omega); one 16-byte load when the
// row stride keeps pieces aligned, else element loads masked at omega.
__device__ __forceinline__ void load_piece(const double* __restrict__ row, uint32_t i0,
                                           uint32_t omega, bool vec_ok, double (&x)[2]) {
    if (vec_ok) {
        const double2 t = __ldg(reinterpret_cast<const double2*>(row + i0));
        x[0] = t.x;
        x[1] = t.y;
    } else {
        x[0] = __ldg(row + i0);
        x[1] = i0 + 1 < omega ? __ldg(row + i0 + 1) : 0.0;
    }
}
__device__ __forceinline__ void load_piece(const float* __restrict__ row, uint32_t i0,
                                           uint32_t omega, bool vec_ok, float (&x)[4]) {
    if (vec_ok) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(row + i0));
        x[0] = t.x;
        x[1] = t.y;
        x[2] = t.z;
        x[3] = t.w;
    } else {
#pragma unroll
        for (uint32_t e = 0; e < 4; ++e) x[e] = i0 + e < omega ? __ldg(row + i0 + e) : 0.f;
    }
}
__device__ __forceinline__ void load_piece(const __nv_bfloat16* __restrict__ row, uint32_t i0,
                                           uint32_t omega, bool vec_ok, float (&x)[8]) {
    if (vec_ok) {
        const uint4 t = __ldg(reinterpret_cast<const uint4*>(row + i0));
        const uint32_t w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
        for (int h = 0; h < 4; ++h) {  // a bf16 is the upper half of its float
            x[2 * h] = __uint_as_float(w[h] << 16);
            x[2 * h + 1] = __uint_as_float(w[h] & 0xffff0000u);
        }
    } else {
#pragma unroll
        for (uint32_t e = 0; e < 8; ++e) x[e] = i0 + e < omega ? vec_load(row + i0 + e) : 0.f;
    }
}

// P consecutive elements from 16-byte aligned shared memory (the bulk-copied rows).
__device__ __forceinline__ void load_piece_shared(const double* p, double (&x)[2]) {
    const double2 t = *reinterpret_cast<const double2*>(p);
    x[0] = t.x;
    x[1] = t.y;
}
__device__ __forceinline__ void load_piece_shared(const float* p, float (&x)[4]) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    x[0] = t.x;
    x[1] = t.y;
    x[2] = t.z;
    x[3] = t.w;
}
__device__ __forceinline__ void load_piece_shared(const __nv_bfloat16* p, float (&x)[8]) {
    const uint4 t = *reinterpret_cast<const uint4*>(p);
    const uint32_t w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
    for (int h = 0; h < 4; ++h) {
        x[2 * h] = __uint_as_float(w[h] << 16);
        x[2 * h + 1] = __uint_as_float(w[h] & 0xffff0000u);
    }
}

__device__ __forceinline__ double split_fma(double a, double w, double s) {
    const double d2 = __dmul_rn(a, a);
    return __fma_rn(d2, w, s);
}
__device__ __forceinline__ float split_fma(float a, float w, float s) {
    const float d2 = __fmul_rn(a, a);
    return __fmaf_rn(d2, w, s);
}
__device__ __forceinline__ double split_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float split_sub(float a, float b) { return __fsub_rn(a, b); }

__device__ __forceinline__ double split_reduce(double s) {
    s = __dadd_rn(s, __shfl_xor_sync(kFullMask, s, 1));
    s = __dadd_rn(s, __shfl_xor_sync(kFullMask, s, 2));
    return __dadd_rn(s, __shfl_xor_sync(kFullMask, s, 4));
}
__device__ __forceinline__ double split_reduce(float s) { return group_reduce(s); }

// Weight of index i in delta_k: row k + 1 of the padded table while k < kTauTableRows, beyond it
// the FP64 power chain continued from the last row of the eigen_t_1 table (src/aesc.h:201-203).
template <class Part>
__device__ __forceinline__ Part split_weight(const Part* __restrict__ wtab, uint32_t wpad,
                                             uint32_t k, uint32_t i, uint32_t omega,
                                             const double* __restrict__ etabd, uint32_t stride,
                                             const double* __restrict__ onem) {
    if (k < uint32_t(kTauTableRows)) return __ldg(wtab + size_t(k + 1) * wpad + i);
    if (i < 1 || i + 1 >= omega) return Part(0);
    double e = __ldg(etabd + size_t(kTauTableRows - 1) * stride + i);
    const double sq = __ldg(etabd + i);
    for (uint32_t r = kTauTableRows - 1; r < k; ++r) e = __dmul_rn(e, sq);
    return Part(__ddiv_rn(e, __ldg(onem + i)));
}

// Pass of one 8-lane group over the rows of one edge: lane sl's partial sums of d_i^2 wa_i and
// d_i^2 wb_i (two weight rows at once) or of d_i^2 w(k, i) alone.
template <class Vec, int ROWS>
__device__ __forceinline__ void split_pass(const Vec* __restrict__ ur, const Vec* __restrict__ vr,
                                           uint32_t omega, bool vec_ok, uint32_t sl,
                                           const typename Split<Vec>::Part* wa,
                                           const typename Split<Vec>::Part* wb,
                                           typename Split<Vec>::Part& sa,
                                           typename Split<Vec>::Part& sb) {
    using Part = typename Split<Vec>::Part;
    constexpr uint32_t P = Split<Vec>::P, C = 8 * P;
#pragma unroll 4
    for (uint32_t i0 = sl * P; i0 < omega; i0 += C) {
        Part xu[P], xv[P];
        load_piece(ur, i0, omega, vec_ok, xu);
        load_piece(vr, i0, omega, vec_ok, xv);
#pragma unroll
        for (uint32_t j = 0; j < P; ++j) {
            const Part d = split_sub(xu[j], xv[j]);
            if (ROWS == 2) sa = split_fma(d, wa[i0 + j], sa);
            sb = split_fma(d, wb[i0 + j], sb);
        }
    }
}

// Stage 1a: the first sweep of every forward edge (upsilon and delta_0 sums), a pure gather.  A
// warp takes eight edges at a time, two per group; the edge records of the next step are fetched
// one step ahead.
template <class Vec>
__global__ void __launch_bounds__(256, 4)
tau_sums_kernel(const uint4* __restrict__ fedge, uint64_t num_forward, const Vec* __restrict__ vec,
                uint32_t stride, uint32_t omega, const typename Split<Vec>::Part* __restrict__ wtab,
                uint32_t wpad, double2* __restrict__ sums) {
    using Part = typename Split<Vec>::Part;
    extern __shared__ __align__(16) unsigned char ssm[];
    pdl_launch_dependents();
    Part* wu = reinterpret_cast<Part*>(ssm);  // upsilon weights, then delta_0 weights
    Part* wd = wu + wpad;
    for (uint32_t i = threadIdx.x; i < 2 * wpad; i += blockDim.x) wu[i] = __ldg(wtab + i);
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, grp = lane >> 3, sl = lane & 7;
    const uint64_t gw = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    const bool vec_ok = stride % Split<Vec>::P == 0;
    uint4 n0 = make_uint4(0, 0, 0, 0), n1 = n0;
    if (gw * 8 + grp < num_forward) n0 = __ldg(fedge + gw * 8 + grp);
    if (gw * 8 + 4 + grp < num_forward) n1 = __ldg(fedge + gw * 8 + 4 + grp);
    for (uint64_t base = gw * 8; base < num_forward; base += nw * 8) {
        const uint64_t e0 = base + grp, e1 = e0 + 4;
        const uint4 r0 = n0, r1 = n1;
        if (e0 + nw * 8 < num_forward) n0 = __ldg(fedge + e0 + nw * 8);
        if (e1 + nw * 8 < num_forward) n1 = __ldg(fedge + e1 + nw * 8);
        Part su0 = Part(0), sd0 = Part(0), su1 = Part(0), sd1 = Part(0);
        if (e0 < num_forward)
            split_pass<Vec, 2>(vec + size_t(r0.x) * stride, vec + size_t(r0.y) * stride, omega,
                               vec_ok, sl, wu, wd, su0, sd0);
        if (e1 < num_forward)
            split_pass<Vec, 2>(vec + size_t(r1.x) * stride, vec + size_t(r1.y) * stride, omega,
                               vec_ok, sl, wu, wd, su1, sd1);
        const double u0 = split_reduce(su0), d0 = split_reduce(sd0);
        const double u1 = split_reduce(su1), d1 = split_reduce(sd1);
        if (sl == 0 && e0 < num_forward) sums[e0] = make_double2(u0, d0);
        if (sl == 0 && e1 < num_forward) sums[e1] = make_double2(u1, d1);
    }
}

// ---- bulk-copy pipeline helpers (cp.async.bulk + mbarrier, CTA scope, no multicast) -------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// bytes (a multiple of 16) from 16-byte aligned global memory into 16-byte aligned shared memory,
// completing on the mbarrier
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}
// Bounded wait on an mbarrier phase: false (and the run's error flag set) if it never completes.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, unsigned* work) {
    for (uint32_t it = 0; it < (1u << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    atomicOr(work + 1, kErrDeadline);
    return false;
}

// Stage 1a over bulk copies: each warp runs its own NST-stage pipeline; a stage holds the two
// eigen rows (omega elements, a multiple of 16 bytes) of the warp's next four edges, brought into
// shared memory by one lane per edge with cp.async.bulk and completed on the stage's mbarrier.
// The eight lanes of group g then sum edge g's terms from shared memory exactly as
// tau_sums_kernel does from global memory (same pieces, same order), so the sums are identical.
template <class Vec> struct BulkShape;
template <> struct BulkShape<double> { static constexpr int WPB = 2; };
template <> struct BulkShape<float> { static constexpr int WPB = 4; };
template <> struct BulkShape<__nv_bfloat16> { static constexpr int WPB = 8; };
constexpr int kBulkStages = 4;

template <class Vec>
__global__ void __launch_bounds__(32 * BulkShape<Vec>::WPB)
tau_sums_bulk_kernel(const uint4* __restrict__ fedge, uint64_t num_forward,
                     const Vec* __restrict__ vec, uint32_t stride, uint32_t omega,
                     const typename Split<Vec>::Part* __restrict__ wtab, uint32_t wpad,
                     double2* __restrict__ sums, unsigned* __restrict__ work) {
    using Part = typename Split<Vec>::Part;
    constexpr uint32_t P = Split<Vec>::P, C = 8 * P;
    constexpr int NST = kBulkStages;
    extern __shared__ __align__(128) unsigned char bsm[];
    pdl_launch_dependents();
    const uint32_t rowb = omega * uint32_t(sizeof(Vec));
    const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5, grp = lane >> 3, sl = lane & 7;
    // layout: per warp NST stages x 4 edges x 2 rows, then the warp's NST mbarriers; the weights
    // after all warps
    const size_t per_warp = size_t(NST) * 8 * rowb + NST * 8;
    unsigned char* wbase = bsm + size_t(wib) * per_warp;
    const uint32_t bars = smem_u32(wbase + size_t(NST) * 8 * rowb);
    Part* wu = reinterpret_cast<Part*>(bsm + size_t(blockDim.x >> 5) * per_warp);
    Part* wd = wu + wpad;
    for (uint32_t i = threadIdx.x; i < 2 * wpad; i += blockDim.x) wu[i] = __ldg(wtab + i);
    if (lane == 0) {
        for (int st = 0; st < NST; ++st) mbar_init(bars + 8 * st, 1);
        mbar_fence_init();
    }
    __syncthreads();
    const uint64_t gw = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    auto step_base = [&](uint64_t t) { return (gw + t * nw) * 4; };
    // lane l < 4 holds the record of edge l of a step, fetched a step before the copies need it
    auto fetch = [&](uint64_t t) {
        const uint64_t e = step_base(t) + lane;
        return (lane < 4 && e < num_forward) ? __ldg(fedge + e) : make_uint4(0, 0, 0, 0);
    };
    // stage st <- the rows of step t's edges (records in r)
    auto issue = [&](uint64_t t, int st, uint4 r) {
        const uint64_t eb = step_base(t);
        if (eb >= num_forward) return;
        const uint32_t cnt = uint32_t(min(uint64_t(4), num_forward - eb));
        const uint32_t bar = bars + 8 * st;
        if (lane == 0) {
            fence_proxy_async();  // the stage's previous contents were read through the generic proxy
            mbar_expect_tx(bar, cnt * 2 * rowb);
        }
        __syncwarp();
        if (lane < cnt) {
            unsigned char* dst = wbase + (size_t(st) * 8 + lane * 2) * rowb;
            bulk_g2s(smem_u32(dst), vec + size_t(r.x) * stride, rowb, bar);
            bulk_g2s(smem_u32(dst + rowb), vec + size_t(r.y) * stride, rowb, bar);
        }
    };
    for (int st = 0; st < NST; ++st) issue(uint64_t(st), st, fetch(uint64_t(st)));
    uint4 ahead = fetch(uint64_t(NST));
    bool ok = true;
    uint64_t t = 0;
    for (; step_base(t) < num_forward; ++t) {
        const int st = int(t % NST);
        const uint4 next_rec = ahead;
        ahead = fetch(t + NST + 1);
        if (!mbar_wait_bounded(bars + 8 * st, uint32_t((t / NST) & 1), work)) {
            ok = false;
            break;
        }
        const uint64_t e = step_base(t) + grp;
        Part su = Part(0), sd = Part(0);
        if (e < num_forward) {
            const Vec* ur = reinterpret_cast<const Vec*>(wbase + (size_t(st) * 8 + grp * 2) * rowb);
            const Vec* vr = ur + omega;
#pragma unroll 4
            for (uint32_t i0 = sl * P; i0 < omega; i0 += C) {
                Part xu[P], xv[P];
                load_piece_shared(ur + i0, xu);
                load_piece_shared(vr + i0, xv);
#pragma unroll
                for (uint32_t j = 0; j < P; ++j) {
                    const Part d = split_sub(xu[j], xv[j]);
                    su = split_fma(d, wu[i0 + j], su);
                    sd = split_fma(d, wd[i0 + j], sd);
                }
            }
        }
        const double us = split_reduce(su), ds = split_reduce(sd);
        if (sl == 0 && e < num_forward) sums[e] = make_double2(us, ds);
        __syncwarp();  // every lane is done with the stage
        issue(t + NST, st, next_rec);
    }
    if (!ok) {  // drain what is still in flight before the shared memory goes away (bounded)
        for (uint64_t u = t + 1; u < t + NST && step_base(u) < num_forward; ++u)
            if (!mbar_wait_bounded(bars + 8 * int(u % NST), uint32_t((u / NST) & 1), work)) break;
    }
}

// The bound of one edge per lane (src/aesc.h:181-207): tau_0 from lambda_1, then tau' from
// delta_k while t <= tau' < tau (t += 2).  Edges that need a further delta sweep are served four
// at a time by the warp's 8-lane groups.  Writes tau to both slots and marks the two rows when
// tau > 1.  All 32 lanes of the warp call it together; act says whether the lane holds an edge.
template <class Vec>
struct BoundArgs {
    const uint32_t* deg;
    const Vec* vec;
    uint32_t stride, omega;
    const typename Split<Vec>::Part* wtab;
    uint32_t wpad;
    const double* etabd;
    const double* onem;
    double eps_half, mdbl;
    TauConst c;
    int* taus;
    RowMarks rm;
};

template <class Vec>
__device__ __forceinline__ void bound_lanes(const BoundArgs<Vec>& A, bool act, uint4 rec, double2 sm,
                                            unsigned long long& iters,
                                            unsigned long long& ambiguous) {
    using Part = typename Split<Vec>::Part;
    constexpr bool kF64 = std::is_same<Vec, double>::value;
    constexpr uint32_t P = Split<Vec>::P, C = 8 * P;
    const uint32_t lane = threadIdx.x & 31, grp = lane >> 3, sl = lane & 7;
    const bool vec_ok = A.stride % P == 0;
    const double inv_b1 = 1.0 / A.c.b1, inv_b2 = 1.0 / A.c.b2;
    uint32_t du = 1, dv = 1;
    if (act) {
        du = __ldg(A.deg + rec.x);
        dv = __ldg(A.deg + rec.y);
    }
    const double inv1 = 1.0 / double(du), inv2 = 1.0 / double(dv);
    auto bound = [&](double one_m_lam2, double b, double inv_b, double dl, double up) {
        if constexpr (kF64) {
            return get_tau<double>(du, dv, A.eps_half, one_m_lam2, b, dl, up, ambiguous);
        } else {
            return get_tau_mixed(inv1, inv2, A.eps_half, one_m_lam2, inv_b, dl, up);
        }
    };
    int tau = 0, t = 1;
    uint32_t k = 1;
    bool need = false;
    double ups = 0;
    if (act) {
        ups = kF64 ? __ddiv_rn(sm.x, A.mdbl) : sm.x / A.mdbl;
        const double del = kF64 ? __ddiv_rn(sm.y, A.mdbl) : sm.y / A.mdbl;
        tau = bound(A.c.one_m_l1sq, A.c.b1, inv_b1, 0.0, 0.0);
        ++iters;
        const int tp = bound(A.c.one_m_l2sq, A.c.b2, inv_b2, del, ups);
        if (t <= tp && tp < tau) {
            tau = tp;
            t += 2;
            need = true;
        }
    }
    // further delta sweeps (:191-204), four edges at a time
    unsigned nb;
    while ((nb = __ballot_sync(kFullMask, need)) != 0) {
        int sel[4];
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            sel[g] = nb ? __ffs(nb) - 1 : -1;
            if (nb) nb &= nb - 1;
        }
        const uint32_t src_lane = sel[grp] < 0 ? 0u : uint32_t(sel[grp]);
        const uint32_t gu = __shfl_sync(kFullMask, rec.x, src_lane);
        const uint32_t gv = __shfl_sync(kFullMask, rec.y, src_lane);
        const uint32_t gk = __shfl_sync(kFullMask, k, src_lane);
        Part s2 = Part(0);
        if (sel[grp] >= 0) {
            const Vec* ur = A.vec + size_t(gu) * A.stride;
            const Vec* vr = A.vec + size_t(gv) * A.stride;
            if (gk < uint32_t(kTauTableRows)) {
                split_pass<Vec, 1>(ur, vr, A.omega, vec_ok, sl, nullptr,
                                   A.wtab + size_t(gk + 1) * A.wpad, s2, s2);
            } else {
                for (uint32_t i0 = sl * P; i0 < A.omega; i0 += C) {
                    Part xu[P], xv[P];
                    load_piece(ur, i0, A.omega, vec_ok, xu);
                    load_piece(vr, i0, A.omega, vec_ok, xv);
#pragma unroll
                    for (uint32_t j = 0; j < P; ++j)
                        s2 = split_fma(split_sub(xu[j], xv[j]),
                                       split_weight<Part>(A.wtab, A.wpad, gk, i0 + j, A.omega,
                                                          A.etabd, A.stride, A.onem),
                                       s2);
                }
            }
        }
        const double dsum = split_reduce(s2);
        double mine = 0.0;
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            const double r = __shfl_sync(kFullMask, dsum, g * 8);
            if (sel[g] == int(lane)) mine = r;
        }
        bool served = false;
#pragma unroll
        for (int g = 0; g < 4; ++g) served |= sel[g] == int(lane);
        if (served) {
            const double del = kF64 ? __ddiv_rn(mine, A.mdbl) : mine / A.mdbl;
            ++iters;
            const int tp = bound(A.c.one_m_l2sq, A.c.b2, inv_b2, del, ups);
            if (t <= tp && tp < tau) {
                tau = tp;
                t += 2;
                ++k;
            } else {
                need = false;
            }
        }
    }
    if (act) {
        A.taus[rec.z] = tau;
        A.taus[rec.w] = tau;
        if (tau > 1) {
            mark_row(A.rm, rec.x);
            mark_row(A.rm, rec.y);
        }
    }
}

__device__ __forceinline__ void flush_tau_stats(unsigned long long iters, unsigned long long ambiguous,
                                                unsigned long long* stats) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        iters += __shfl_xor_sync(kFullMask, iters, o);
        ambiguous += __shfl_xor_sync(kFullMask, ambiguous, o);
    }
    if ((threadIdx.x & 31) == 0) {
        stat_add(stats, kStTauIters, iters);
        stat_add(stats, kStTauAmbiguous, ambiguous);
    }
}

// Stage 1b: the bound per edge, one lane per edge (a variant that evaluated the bounds inside the
// gather kernel, 32 edges per warp at a time, measured slower: the bound's FP64 chains then sit on
// the gather's critical path).
template <class Vec>
__global__ void __launch_bounds__(256)
tau_bound_kernel(const uint4* __restrict__ fedge, uint64_t num_forward,
                 const double2* __restrict__ sums, BoundArgs<Vec> A,
                 unsigned long long* __restrict__ stats) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t gw = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = (uint64_t(gridDim.x) * blockDim.x) >> 5;
    unsigned long long iters = 0, ambiguous = 0;
    pdl_launch_dependents();
    pdl_wait();  // the sums of tau_sums_kernel
    for (uint64_t base = gw * 32; base < num_forward; base += nw * 32) {
        const uint64_t e = base + lane;
        const bool act = e < num_forward;
        uint4 rec = make_uint4(0, 0, 0, 0);
        double2 sm = make_double2(0.0, 0.0);
        if (act) {
            rec = __ldg(fedge + e);
            sm = sums[e];
        }
        bound_lanes<Vec>(A, act, rec, sm, iters, ambiguous);
    }
    flush_tau_stats(iters, ambiguous, stats);
}

// ---- stage 2: per-source push, edge bound and walks -----------------------------------------------
struct WalkItem {
    uint32_t pos, v, len, pad;  // pad: in a walk queue, the item's list entry (its source)
    unsigned long long nr;
};

// Outcome of the push of one listed source in push_block_kernel.
struct PrePush {
    int ell;           // rounds pushed
    float gmax, gmin;  // residual max / min over the final frontier (gmin before the |q| < n rule)
    uint32_t support;  // size of the final frontier
};

template <class Real, class Acc>
struct SourceParams {
    const uint32_t* idx;
    const uint32_t* adj;
    const uint32_t* deg;
    uint32_t n;
    const int* taus;
    Acc* preds;           // pre-symmetric row scores (Real in the parity forms, double in MIXED)
    unsigned* work;       // [0] next list entry, [1] error flags, [2] list length
    const uint32_t* rows; // the sources to run (rows with a slot of tau > 1), in any order
    uint32_t* qbuf;       // 2 * n per warp
    WalkItem* items;      // max_degree per warp
    Real* pvec_g;         // n per warp (global tier)
    unsigned long long* fx_g;  // n per warp: fixed-point accumulators (Jacobi push, global tier)
    unsigned char* wclean;     // per warp: 1 = its HBM vectors are all zero (left so by its last run)
    unsigned char* vis_g; // vis_stride per warp (global tier)
    size_t vis_stride;
    size_t smem_per_warp;
    uint32_t max_degree;
    double eps;
    double logmd;         // log(m / delta), formed on the host
    int gamma;
    unsigned long long* stats;
    const uint2* adjd;    // (neighbour, neighbour degree) per slot
    uint64_t budget_ns;   // device time budget; past it every warp stops and flags a timeout
    unsigned* claim;      // the claim counter of this launch
    uint32_t list_base;   // this launch runs list entries [list_base, list_base + list_cap)
    uint32_t list_cap;
    // PrePush mode (mixed form, large graphs): the push ran in push_block_kernel; entry k's final
    // residual vector is column (k - list_base) % S of its CTA's block
    const PrePush* pre;
    const float* pre_cols;
    const uint32_t* pre_final;
    // The graph has rows that repeat a neighbour or hold their own vertex (the reference's loader
    // keeps duplicate edges and self-loops, src/graph.h:63-66, 75-78): the first round takes the
    // general path and the push serialises each run of a repeated neighbour (parity forms only).
    bool multi;
    // Vertex count the per-warp scratch is laid out for (the graph's n, or the largest n of a
    // batch whose graphs share the scratch of one persistent launch).
    uint32_t scratch_n;
    bool gs_window;  // parity forms: the windowed sequential push (else one vertex at a time)
    // Optional run trace (null when off): the walk count nr of every walking slot, and the rounds
    // pushed (ell) of every listed row.
    uint32_t* trace_nr;
    uint32_t* trace_ell;
    // PrePush mode: when set, a source's walking slots (with their nr) are appended to this queue
    // instead of being walked by the warp here: light items from the front (walk_count[0] counts
    // them; walk_queue_kernel walks them), heavy ones (many walks of few hops) from the back
    // (walk_count[2]; heavy_walk_kernel).  walk_cap entries.
    WalkItem* walk_queue;
    unsigned* walk_count;
    uint32_t walk_cap;
};

// The source kernel's parameters: one graph (N = 1), or up to N graphs whose listed rows one
// persistent launch works through as a single queue of (graph, row) items.  Every entry shares the
// first entry's per-warp scratch (qbuf, items, residual vectors, flags, claim counter).  The pack
// travels in the kernel's parameter space, so a warp reads its graph's fields from the constant
// bank with a warp-uniform index.
template <class Real, class Acc, int N>
struct SourcePack {
    static constexpr int kMax = N;
    uint32_t count;
    SourceParams<Real, Acc> g[N];
};
constexpr int kBatchPack = 64;  // graphs per persistent batch launch

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

// Runs over [0, count) in steps of 32 * kB: load(i0, regs) issues the loads of one step into
// registers, proc(i0, regs) consumes them.  The next step's loads are issued before the current
// step is processed, so a pass over a frontier or a row waits for memory once, not once per step.
template <class T, class Load, class Proc>
__device__ __forceinline__ void pipelined(uint32_t count, Load load, Proc proc) {
    if (count == 0) return;
    T a[kB], b[kB];
    load(0u, a);
    for (uint32_t i0 = 0; i0 < count; i0 += 32 * kB) {
        if (i0 + 32 * kB < count) load(i0 + 32 * kB, b);
        proc(i0, a);
#pragma unroll
        for (int k = 0; k < kB; ++k) a[k] = b[k];
    }
}

// preds[pos] += (pvec[src] - pvec[w]) / ds (:236): in the row's own real type in the parity forms,
// accumulated in FP64 in the mixed form.
template <class Real, class Acc>
__device__ __forceinline__ Acc row_update(Acc old, Real ps, Real pv, Real ds) {
    if constexpr (std::is_same<Real, Acc>::value) {
        return radd(old, rdiv(rsub(ps, pv), ds));
    } else {
        return __dadd_rn(old, __ddiv_rn(__dsub_rn(double(ps), double(pv)), double(ds)));
    }
}

// Order-preserving integer images of non-negative reals (residuals are never negative), so that
// shared-memory integer atomics give max / min.
__device__ __forceinline__ unsigned long long ord_bits(float x) { return __float_as_uint(x); }
__device__ __forceinline__ unsigned long long ord_bits(double x) {
    return (unsigned long long)__double_as_longlong(x);
}
template <class Real> __device__ __forceinline__ Real from_ord(unsigned long long b);
template <> __device__ __forceinline__ float from_ord<float>(unsigned long long b) {
    return __uint_as_float(unsigned(b));
}
template <> __device__ __forceinline__ double from_ord<double>(unsigned long long b) {
    return __longlong_as_double((long long)b);
}

// The real_gamma-th largest residual of the frontier (counting multiplicity) and how many of the
// chosen values equal it.  gamma <= kTopK: one pass keeping a sorted top-k per lane, then a
// warp merge.  Larger gamma: one pass per distinct value from the top.
template <class Real>
__device__ void kth_largest(const uint32_t* q, uint32_t qs, const Real* pvec, int rg, Real& t,
                            int& n_eq_taken) {
    const uint32_t lane = threadIdx.x & 31;
    auto load_q = [&](uint32_t i0, uint32_t* r) {
#pragma unroll
        for (int b = 0; b < kB; ++b) {
            const uint32_t i = i0 + 32 * b + lane;
            r[b] = i < qs ? q[i] : 0xffffffffu;
        }
    };
    if (rg <= kTopK) {
        Real L[kTopK];
#pragma unroll
        for (int j = 0; j < kTopK; ++j) L[j] = Real(-INFINITY);
        pipelined<uint32_t>(qs, load_q, [&](uint32_t, const uint32_t* r) {
#pragma unroll
            for (int b = 0; b < kB; ++b) {
                if (r[b] == 0xffffffffu) continue;
                const Real x = pvec[r[b]];
                if (x > L[kTopK - 1]) {
#pragma unroll
                    for (int j = kTopK - 1; j > 0; --j) {
                        const Real prev = L[j - 1];
                        L[j] = x > prev ? prev : (x > L[j] ? x : L[j]);
                    }
                    L[0] = x > L[0] ? x : L[0];
                }
            }
        });
        Real last = Real(-INFINITY);
        int run = 0;
        for (int r = 0; r < rg; ++r) {
            const Real mx = warp_max(L[0]);
            const unsigned who = __ballot_sync(kFullMask, L[0] == mx);
            if (lane == uint32_t(__ffs(who) - 1)) {
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
        pipelined<uint32_t>(qs, load_q, [&](uint32_t, const uint32_t* r) {
#pragma unroll
            for (int b = 0; b < kB; ++b) {
                if (r[b] == 0xffffffffu) continue;
                const Real x = pvec[r[b]];
                if (x < thr) {
                    if (x > best) {
                        best = x;
                        cnt = 1;
                    } else if (x == best) {
                        ++cnt;
                    }
                }
            }
        });
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

// kth_largest over the positive entries of a dense vector (the residual column the block push
// leaves, whose positive entries are exactly the final frontier, in vertex order): the same
// selection without the frontier list, as contiguous pipelined loads.
template <class Real>
__device__ void kth_largest_col(const Real* col, uint32_t n, int rg, Real& t, int& n_eq_taken,
                                uint32_t* cand = nullptr, uint32_t* ncand = nullptr) {
    const uint32_t lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    auto load_v = [&](uint32_t i0, Real* r) {
#pragma unroll
        for (int b = 0; b < kB; ++b) {
            const uint32_t i = i0 + 32 * b + lane;
            const Real x = i < n ? col[i] : Real(0);
            r[b] = x > Real(0) ? x : Real(-INFINITY);
        }
    };
    if (rg <= kTopK) {
        Real L[kTopK];
#pragma unroll
        for (int j = 0; j < kTopK; ++j) L[j] = Real(-INFINITY);
        // With cand: every positive entry that reaches its lane's top kTopK so far (x >= the
        // lane's current kTopK-th value) is listed, in index order.  An entry not listed had
        // kTopK >= rg larger ones before it, so it is below the rg-th largest value; every entry
        // at or above that value has fewer than rg larger ones and is listed.
        uint32_t nc = 0;
        pipelined<Real>(n, load_v, [&](uint32_t i0, const Real* r) {
#pragma unroll
            for (int b = 0; b < kB; ++b) {
                const Real x = r[b];
                if (cand) {
                    const bool rec = x > Real(-INFINITY) && x >= L[kTopK - 1];
                    const unsigned bal = __ballot_sync(kFullMask, rec);
                    if (rec) cand[nc + __popc(bal & below)] = i0 + 32 * b + lane;
                    nc += __popc(bal);
                }
                if (x > L[kTopK - 1]) {
#pragma unroll
                    for (int j = kTopK - 1; j > 0; --j) {
                        const Real prev = L[j - 1];
                        L[j] = x > prev ? prev : (x > L[j] ? x : L[j]);
                    }
                    L[0] = x > L[0] ? x : L[0];
                }
            }
        });
        Real last = Real(-INFINITY);
        int run = 0;
        for (int r = 0; r < rg; ++r) {
            const Real mx = warp_max(L[0]);
            const unsigned who = __ballot_sync(kFullMask, L[0] == mx);
            if (lane == uint32_t(__ffs(who) - 1)) {
#pragma unroll
                for (int j = 0; j < kTopK - 1; ++j) L[j] = L[j + 1];
                L[kTopK - 1] = Real(-INFINITY);
            }
            run = (r > 0 && mx == last) ? run + 1 : 1;
            last = mx;
        }
        t = last;
        n_eq_taken = run;
        if (ncand) *ncand = nc;
        return;
    }
    Real thr = Real(INFINITY);
    int remaining = rg;
    while (true) {
        Real best = Real(-INFINITY);
        unsigned cnt = 0;
        pipelined<Real>(n, load_v, [&](uint32_t, const Real* r) {
#pragma unroll
            for (int b = 0; b < kB; ++b) {
                const Real x = r[b];
                if (x < thr && x > Real(-INFINITY)) {
                    if (x > best) {
                        best = x;
                        cnt = 1;
                    } else if (x == best) {
                        ++cnt;
                    }
                }
            }
        });
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

// Segmented max / min over lanes whose segment ids are non-decreasing: after the shuffles, the
// last lane of each segment holds the segment's extremum.
template <class Real>
__device__ __forceinline__ void seg_maxmin(uint32_t seg, Real& mx, Real& mn) {
    const uint32_t lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Real ymx = __shfl_up_sync(kFullMask, mx, o);
        const Real ymn = __shfl_up_sync(kFullMask, mn, o);
        const uint32_t ys = __shfl_up_sync(kFullMask, seg, o);
        if (lane >= uint32_t(o) && ys == seg) {
            mx = std_max(mx, ymx);
            mn = std_min(mn, ymn);
        }
    }
}

// ---- stage 2a (mixed form, large graphs): multi-source Jacobi push as a pull product -----------
// In the mixed form a push round drains the whole frontier at once (Jacobi), so a round is exactly
// r <- D^-1 A r: with r supported on the frontier q, every vertex u receives the residuals of its
// frontier neighbours divided by deg(u), and the frontier's own residuals are pushed out.  For
// graphs whose residual vector does not fit in shared memory, each CTA takes S = 32 listed sources
// at a time and keeps their residual vectors as the columns of an n x S row-major block in HBM; a
// round is one pass over the CSR in which warp w pulls rows u = w, w + 32, ...: lane j adds the
// column-j entries of u's neighbours in CSR order (one coalesced 128-byte row read per neighbour)
// and divides by deg(u).  The same pass accumulates each column's frontier statistics (degree sum,
// max, min, size of the support), so the stop test of src/aesc.h:483-502 needs no further pass.
// Columns whose source has stopped are carried over unchanged, so when the last one stops every
// column holds its source's final residual vector; the edge bound, chi and walks of those sources
// then run in source_kernel (PrePush mode), which copies the column into its own residual vector.
constexpr int kBlockCols = 32;
// Walk items of the block push's sources with at least kHeavyNr walks of at most kHeavyLen hops
// go to heavy_walk_kernel, which walks 32 of their bouquets at once instead of one after another.
constexpr unsigned long long kHeavyNr = 512;
constexpr uint32_t kHeavyLen = 32;
// rows a warp of push_block_kernel claims at a time (their dependent loads are issued together).
// Measured on three graphs (n = 25,860 / 143,522 / 199,772): 1 row is 3-6 % faster than the plain
// loop (the row's own value and first adjacency chunk are requested before its neighbours are
// read), 2 and 4 rows 0-25 % slower (the kernel is at its 64-register cap).
constexpr int kRowBatch = 1;


struct PushBlockParams {
    const uint32_t* idx;
    const uint32_t* adj;
    const uint32_t* deg;
    const uint2* adjd;
    uint32_t n;
    uint64_t m;
    const int* taus;
    double* preds;
    unsigned* work;        // [1] error flags, [2] list length
    const uint32_t* rows;  // the list of sources
    uint32_t base;         // first list entry of this wave
    double eps, logmd;
    float* cols;           // per CTA: two n x S blocks
    uint32_t* final_buf;   // per CTA: the block that holds the final columns
    PrePush* pre;          // per list entry
    bool bits;             // the three row masks fit in shared memory (else they live in gbits)
    bool cur_smem;         // (when !bits) the current round's mask alone fits in shared memory
    uint32_t* gbits;       // per CTA: three n-bit row masks in global memory (L2), when not in smem
    uint32_t* lists;       // per CTA: four row lists of n entries (see push_block_kernel)
    uint32_t list_div;     // a round is compacted when its live rows' degree sum * list_div < m
    int rounds_mode;       // 0 = by that rule, 1 = every round compacted, 2 = every round full
    unsigned long long* stats;
    uint64_t budget_ns;
};

// Exclusive prefix sum over the block's threads (blockDim.x a multiple of 32, at most 1024); the
// block total goes to *total.  Uses `tmp` (32 words of shared memory).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* tmp, uint32_t* total) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFullMask, incl, o);
        if (lane >= uint32_t(o)) incl += y;
    }
    if (lane == 31) tmp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < nwarp ? tmp[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFullMask, wi, o);
            if (lane >= uint32_t(o)) wi += y;
        }
        if (lane < nwarp) tmp[lane] = wi - w;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    const uint32_t out = tmp[warp] + incl - v;
    __syncthreads();
    return out;
}

// The rows whose bit is set in `mask` (words of 32 rows), in increasing order, into `out`; the
// count goes to *count.  Each thread takes a contiguous run of words.
__device__ __forceinline__ void compact_mask(const uint32_t* mask, uint32_t words, uint32_t n,
                                             uint32_t* out, uint32_t* tmp, uint32_t* count) {
    const uint32_t per = (words + blockDim.x - 1) / blockDim.x;
    const uint32_t w0 = min(words, threadIdx.x * per), w1 = min(words, w0 + per);
    uint32_t c = 0;
    for (uint32_t w = w0; w < w1; ++w) c += __popc(mask[w]);
    uint32_t pos = block_exclusive_scan(c, tmp, count);
    for (uint32_t w = w0; w < w1; ++w) {
        uint32_t b = mask[w];
        while (b) {
            const uint32_t r = w * 32u + uint32_t(__ffs(b) - 1);
            b &= b - 1;
            if (r < n) out[pos++] = r;
        }
    }
}

__global__ void __launch_bounds__(1024, 1)
push_block_kernel(PushBlockParams p) {
    constexpr int S = kBlockCols;
    // Row masks, one bit per row: bcur / bnxt mark the rows with a nonzero running column in the
    // cur / nxt block (the pull skips the 128-byte reads of neighbour rows whose bit is clear);
    // tmask marks the rows a compacted round processes.  In shared memory while the three fit
    // (p.bits), else in this CTA's part of p.gbits (L2-resident).
    //
    // Row lists (n entries each, in p.lists): Lc = rows with any nonzero column in cur, Lp = the
    // same for the block nxt still holds from the round before, Ln = those of the round being
    // formed, P = the rows a compacted round processes.  A round is either a full pass over all n
    // rows (dense frontiers) or a compacted one over P = (neighbours of the running-live rows of
    // cur) U Lc U Lp, in increasing row order: a row outside the neighbourhood of the live rows
    // receives nothing, Lc carries the stopped columns and zeroes the running ones, and Lp covers
    // every row nxt still holds from two rounds before, so no stale row survives.  Both give the
    // same values; the choice per round is by the live rows' degree sum (the scatter work of the
    // compaction) against m / list_div.
    extern __shared__ uint32_t s_bits[];
    __shared__ uint32_t s_src[S], s_rb[S], s_ds[S], s_support[S], s_ell[S];
    __shared__ unsigned long long s_picost[S];
    __shared__ unsigned s_max[S], s_min[S];  // float bits of non-negative residuals
    __shared__ int s_active[S];
    __shared__ int s_any;
    __shared__ uint32_t s_tmp[32];
    __shared__ uint32_t s_lc, s_lp, s_ln, s_pn;  // list lengths
    __shared__ uint32_t s_next;                  // next row of the round (claimed by warps)
    __shared__ unsigned long long s_live_deg;   // degree sum of the running-live rows of cur
    pdl_launch_dependents();
    pdl_wait();  // the list, and the previous wave's readers of these blocks
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const uint32_t n = p.n;
    const unsigned len = p.work[2];
    const uint64_t first = uint64_t(p.base) + uint64_t(blockIdx.x) * S;
    if (first >= len) return;
    const uint32_t cnt = uint32_t(min(uint64_t(S), len - first));
    float* A = p.cols + size_t(blockIdx.x) * 2 * size_t(n) * S;
    float* B = A + size_t(n) * S;
    const uint64_t deadline = globaltimer_ns() + p.budget_ns;
    unsigned long long st_pv = 0, st_tr = 0, st_rounds = 0;

    // both blocks start at zero (a compacted round writes only the rows it processes)
    for (size_t i = threadIdx.x; i < size_t(n) * S / 2; i += blockDim.x)
        reinterpret_cast<float4*>(A)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t words = (n + 31) / 32;
    // Mask placement: all three in shared memory; or (cur_smem) bcur in shared memory -- it is
    // read for every neighbour chunk of the pull -- with bnxt and tmask in global memory, bnxt
    // copied into bcur at each round's end; or all three in global memory.
    uint32_t* const gb = p.gbits ? p.gbits + size_t(blockIdx.x) * 3 * words : nullptr;
    uint32_t* bcur = (p.bits || p.cur_smem) ? s_bits : gb;
    uint32_t* bnxt = p.bits ? s_bits + words : gb + words;
    uint32_t* tmask = p.bits ? s_bits + 2 * words : gb + 2 * words;
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) {
        bcur[i] = 0u;
        bnxt[i] = 0u;
        tmask[i] = 0u;
    }
    uint32_t* const lbase = p.lists + size_t(blockIdx.x) * 4 * size_t(n);
    uint32_t* Lc = lbase;
    uint32_t* Lp = lbase + n;
    uint32_t* Ln = lbase + 2 * size_t(n);
    uint32_t* const P = lbase + 3 * size_t(n);
    if (threadIdx.x < S) {
        const uint32_t j = threadIdx.x;
        s_active[j] = j < cnt;
        s_src[j] = j < cnt ? __ldg(p.rows + first + j) : 0;
        s_picost[j] = 0;
        s_max[j] = 0;
        s_min[j] = __float_as_uint(1.f);
        s_ell[j] = 1;
    }
    if (threadIdx.x == 0) {
        s_lp = 0;
        s_live_deg = 0;
    }
    __syncthreads();
    // round 1 in closed form: the frontier {src} pushes 1 / deg(u) to every neighbour u
    if (warp < cnt) {
        const uint32_t j = warp, src = s_src[j];
        const uint32_t rb = __ldg(p.idx + src), dsi = __ldg(p.idx + src + 1) - rb;
        const float ds = float(dsi);
        const double pinit = __ddiv_rn(1.0, double(ds));
        unsigned long long pc = 0;
        float mx = 0.f, mn = 1.f;
        for (uint32_t o = lane; o < dsi; o += 32) {
            const uint2 a = __ldg(p.adjd + rb + o);
            const float pu = from_fixed(kFixOne, a.y);
            A[size_t(a.x) * S + j] = pu;
            atomicOr(bcur + (a.x >> 5), 1u << (a.x & 31));
            pc += a.y;
            mx = fmaxf(mx, pu);
            mn = fminf(mn, pu);
            p.preds[rb + o] = row_update<float, double>(pinit, 0.f, pu, ds);
        }
        pc = warp_sum_u64(pc);
        mx = warp_max(mx);
        mn = warp_min(mn);
        if (lane == 0) {
            s_rb[j] = rb;
            s_ds[j] = dsi;
            s_picost[j] = pc;
            s_max[j] = __float_as_uint(mx);
            s_min[j] = __float_as_uint(mn);
            s_support[j] = dsi;
        }
        st_pv += lane == 0 ? 1 : 0;
        st_tr += lane == 0 ? dsi : 0;
    }
    __syncthreads();
    // Lc after round 1: the rows of bcur (every column runs, so a nonzero row is running-live)
    compact_mask(bcur, words, n, Lc, s_tmp, &s_lc);
    __syncthreads();
    {
        unsigned long long d = 0;
        for (uint32_t k = threadIdx.x; k < s_lc; k += blockDim.x) d += __ldg(p.deg + Lc[k]);
        d = warp_sum_u64(d);
        if (lane == 0 && d) atomicAdd(&s_live_deg, d);
    }
    __syncthreads();
    float* cur = A;
    float* nxt = B;
    uint32_t fin = 0;
    while (true) {
        // ---- stop test of every running source (one warp per source) ----
        if (threadIdx.x == 0) s_any = 0;
        __syncthreads();
        if (warp < cnt && s_active[warp]) {
            const uint32_t j = warp, rb = s_rb[j], dsi = s_ds[j];
            const int ell = int(s_ell[j]);
            const float gmax = __uint_as_float(s_max[j]);
            const float gmin = s_support[j] < n ? 0.f : __uint_as_float(s_min[j]);
            const double dse0 = __dmul_rn(double(float(dsi)), p.eps);
            const double dse2 = __dmul_rn(dse0, dse0);
            double rw = 0;
            for (uint32_t c = 0; c < dsi; c += 32) {
                const uint32_t o = c + lane;
                const int rest = o < dsi ? __ldg(p.taus + rb + o) - ell : 0;
                double nrd = 0;
                const bool has = rest > 0;
                if (has) {
                    const double chi = __dmul_rn(__dmul_rn(2.0, double(rest)),
                                                 __dsub_rn(double(gmax), double(gmin)));
                    const double num = __dmul_rn(__dmul_rn(8.0, __dmul_rn(chi, chi)), p.logmd);
                    nrd = std_max(ceil(__ddiv_rn(num, dse2)), 1.0);
                }
                unsigned hb = __ballot_sync(kFullMask, has);
                while (hb) {  // rwcost += nr in slot order
                    const int l = __ffs(hb) - 1;
                    hb &= hb - 1;
                    rw = __dadd_rn(rw, __shfl_sync(kFullMask, nrd, l));
                }
            }
            const bool stop = double(s_picost[j]) >= __dmul_rn(25.0, rw);
            const bool late = globaltimer_ns() > deadline;
            if (lane == 0) {
                if (stop || late) {
                    s_active[j] = 0;
                    PrePush r;
                    r.ell = ell;
                    r.gmax = gmax;
                    r.gmin = __uint_as_float(s_min[j]);
                    r.support = s_support[j];
                    p.pre[first + j] = r;
                    st_rounds += uint64_t(ell);
                    if (late && !stop) atomicOr(p.work + 1, kErrDeadline);
                } else {
                    s_any = 1;
                    st_pv += s_support[j];
                    st_tr += s_picost[j];
                }
            }
        }
        __syncthreads();
        if (!s_any) break;
        // ---- the rows this round processes: all n, or the compacted list P ----
        const bool compact = p.rounds_mode == 1 ||
                             (p.rounds_mode == 0 &&
                              double(s_live_deg) * double(p.list_div) < double(p.m));
        __syncthreads();  // every thread has read s_live_deg before it is reset below
        if (compact) {
            for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) tmask[i] = 0u;
            __syncthreads();
            for (uint32_t k = threadIdx.x; k < s_lp; k += blockDim.x)
                atomicOr(tmask + (Lp[k] >> 5), 1u << (Lp[k] & 31));
            for (uint32_t k = warp; k < s_lc; k += nwarp) {
                const uint32_t w = Lc[k];
                if (lane == 0) atomicOr(tmask + (w >> 5), 1u << (w & 31));
                if (!((bcur[w >> 5] >> (w & 31)) & 1u)) continue;  // only stopped columns here
                const uint32_t wb = __ldg(p.idx + w), we = __ldg(p.idx + w + 1);
                for (uint32_t o = wb + lane; o < we; o += 32) {
                    const uint32_t u = __ldg(p.adj + o);
                    atomicOr(tmask + (u >> 5), 1u << (u & 31));
                }
            }
            __syncthreads();
            compact_mask(tmask, words, n, P, s_tmp, &s_pn);
        }
        // ---- one Jacobi round for the running columns; stopped columns are carried over ----
        if (threadIdx.x < S) {
            s_picost[threadIdx.x] = 0;
            s_max[threadIdx.x] = 0;
            s_min[threadIdx.x] = __float_as_uint(1.f);
            s_support[threadIdx.x] = 0;
        }
        if (threadIdx.x == 0) {
            s_ln = 0;
            s_live_deg = 0;
            s_next = nwarp * kRowBatch;
        }
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) bnxt[i] = 0u;
        __syncthreads();
        const uint32_t nrows = compact ? s_pn : n;
        const bool run = lane < cnt && s_active[lane];
        unsigned long long pc = 0, live_deg = 0;
        uint32_t sup = 0;
        float mx = 0.f, mn = 1.f;
        // Rows are claimed kRowBatch at a time from a shared counter (rows warp * kRowBatch .. first),
        // so a warp that meets a hub row does not hold the others at the round's barrier.  The
        // batch's row ids, offsets, first adjacency chunks and own values are loaded together, so
        // their dependent loads are paid once per batch, not once per row.
        for (uint32_t kb = warp * kRowBatch; kb < nrows;) {
            uint32_t myu = 0, myb = 0, myd = 0;
            if (lane < kRowBatch && kb + lane < nrows) {
                myu = compact ? P[kb + lane] : kb + lane;
                myb = __ldg(p.idx + myu);
                myd = __ldg(p.idx + myu + 1) - myb;
            }
            uint32_t nb0[kRowBatch];
            float own[kRowBatch];
#pragma unroll
            for (int i = 0; i < kRowBatch; ++i) {
                const uint32_t ui = __shfl_sync(kFullMask, myu, i);
                const uint32_t bi = __shfl_sync(kFullMask, myb, i);
                const uint32_t di = __shfl_sync(kFullMask, myd, i);
                const bool has = kb + uint32_t(i) < nrows;
                nb0[i] = has && lane < di ? __ldg(p.adj + bi + lane) : 0u;
                own[i] = has ? cur[size_t(ui) * S + lane] : 0.f;
            }
            unsigned nk = 0;
            if (lane == 0) nk = atomicAdd(&s_next, uint32_t(kRowBatch));
#pragma unroll
            for (int i = 0; i < kRowBatch; ++i) {
            if (kb + uint32_t(i) >= nrows) break;
            const uint32_t u = __shfl_sync(kFullMask, myu, i);
            const uint32_t ub = __shfl_sync(kFullMask, myb, i);
            const uint32_t ud = __shfl_sync(kFullMask, myd, i);
            unsigned long long acc = 0;
            for (uint32_t c = 0; c < ud; c += 32) {
                const uint32_t nb =
                    c == 0 ? nb0[i] : (c + lane < ud ? __ldg(p.adj + ub + c + lane) : 0u);
                // neighbours whose running columns are all zero add nothing: they are dropped, and
                // the live ones compacted into lanes 0 .. popc(live) - 1 (the fixed-point sum does
                // not depend on the order)
                const bool in = c + lane < ud;
                const unsigned live =
                    __ballot_sync(kFullMask, in && ((bcur[nb >> 5] >> (nb & 31)) & 1u));
                const uint32_t nth =
                    lane < uint32_t(__popc(live)) ? __fns(live, 0, int(lane) + 1) : 0u;
                const uint32_t packed = __shfl_sync(kFullMask, nb, nth);
                const uint32_t kk = __popc(live);
                // eight independent 128-byte row loads in flight per step; the last step's loads
                // past kk are predicated off (a zero adds nothing), so a row's remainder costs one
                // load latency, not one per neighbour
                for (uint32_t t = 0; t < kk; t += 8) {
                    float x[8];
#pragma unroll
                    for (int h = 0; h < 8; ++h) {
                        const uint32_t v = __shfl_sync(kFullMask, packed, int((t + h) & 31u));
                        x[h] = t + h < kk ? cur[size_t(v) * S + lane] : 0.f;
                    }
#pragma unroll
                    for (int h = 0; h < 8; ++h) acc += to_fixed(x[h]);
                }
            }
            float r = own[i];
            if (run) {
                r = acc ? from_fixed(acc, ud) : 0.f;
                if (r > 0.f) {
                    pc += ud;
                    ++sup;
                    mx = fmaxf(mx, r);
                    mn = fminf(mn, r);
                }
            }
            const bool running_live = __any_sync(kFullMask, run && r > 0.f);
            const bool any_nz = __any_sync(kFullMask, r != 0.f);
            if (lane == 0) {
                if (running_live) {
                    atomicOr(bnxt + (u >> 5), 1u << (u & 31));
                    live_deg += ud;
                }
                if (any_nz) Ln[atomicAdd(&s_ln, 1u)] = u;
            }
            nxt[size_t(u) * S + lane] = r;
            }
            kb = __shfl_sync(kFullMask, nk, 0);
        }
        if (run) {
            atomicAdd(s_picost + lane, pc);
            atomicAdd(s_support + lane, sup);
            atomicMax(s_max + lane, __float_as_uint(mx));
            atomicMin(s_min + lane, __float_as_uint(mn));
        }
        if (lane == 0 && live_deg) atomicAdd(&s_live_deg, live_deg);
        __syncthreads();
        // ---- preds[row] += (r[src] - r[t]) / ds for every slot of each running source ----
        if (warp < cnt && s_active[warp]) {
            const uint32_t j = warp, src = s_src[j], rb = s_rb[j], dsi = s_ds[j];
            const float ds = float(dsi);
            const float ps = nxt[size_t(src) * S + j];
            for (uint32_t o = lane; o < dsi; o += 32) {
                const uint32_t w = __ldg(p.adj + rb + o);
                p.preds[rb + o] = row_update<float, double>(p.preds[rb + o], ps,
                                                            nxt[size_t(w) * S + j], ds);
            }
            if (lane == 0) ++s_ell[j];
        }
        if (threadIdx.x == 0) {
            s_lp = s_lc;
            s_lc = s_ln;
        }
        __syncthreads();
        float* t = cur;
        cur = nxt;
        nxt = t;
        if (!p.bits && p.cur_smem) {
            // bcur stays in shared memory: take the new round's mask into it
            for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) bcur[i] = bnxt[i];
            __syncthreads();
        } else {
            uint32_t* tb = bcur;
            bcur = bnxt;
            bnxt = tb;
        }
        uint32_t* tl = Lp;
        Lp = Lc;
        Lc = Ln;
        Ln = tl;
        fin ^= 1u;
    }
    // The final columns, transposed into the other buffer: column j becomes n contiguous floats
    // at spare + j * n, so the per-source stage reads its residual vector with unit stride.  Warp
    // w takes tiles of 32 rows; lane l loads row (tile + l) whole (eight 16-byte loads of one
    // 128-byte row) and the 32 stores of the tile (one per column) are each 128 contiguous bytes.
    {
        float* spare = fin ? A : B;
        for (uint32_t t0 = warp * 32u; t0 < n; t0 += nwarp * 32u) {
            const uint32_t u = t0 + lane;
            float v[S];
            if (u < n) {
                const float4* row = reinterpret_cast<const float4*>(cur + size_t(u) * S);
#pragma unroll
                for (int k = 0; k < S / 4; ++k) {
                    const float4 f = row[k];
                    v[4 * k] = f.x;
                    v[4 * k + 1] = f.y;
                    v[4 * k + 2] = f.z;
                    v[4 * k + 3] = f.w;
                }
#pragma unroll
                for (int c = 0; c < S; ++c) spare[size_t(c) * n + u] = v[c];
            }
        }
    }
    if (threadIdx.x == 0) p.final_buf[blockIdx.x] = fin;
    st_pv = warp_sum_u64(st_pv);
    st_tr = warp_sum_u64(st_tr);
    st_rounds = warp_sum_u64(st_rounds);
    if (lane == 0) {
        stat_add(p.stats, kStPushRounds, st_rounds);
        stat_add(p.stats, kStPushVertices, st_pv);
        stat_add(p.stats, kStPushTraversals, st_tr);
    }
}

// Sort key of each row for the multi-source push: the row's largest tau if it is listed, else 0.
// A source stops pushing once ell reaches that tau (rwcost = 0 then), so CTAs whose 32 sources
// share a tau bound push for about the same number of rounds.
__global__ void row_key_kernel(const uint32_t* __restrict__ idx, const int* __restrict__ taus,
                               const uint32_t* __restrict__ mark, uint32_t n,
                               uint32_t* __restrict__ key, uint32_t* __restrict__ ids) {
    pdl_wait();  // taus and marks of the tau kernels
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n;
         v += (gridDim.x * blockDim.x) >> 5) {
        int t = 0;
        if (mark[v]) {
            const uint32_t b = __ldg(idx + v), e = __ldg(idx + v + 1);
            for (uint32_t o = b + lane; o < e; o += 32) t = max(t, __ldg(taus + o));
#pragma unroll
            for (int o = 16; o; o >>= 1) t = max(t, __shfl_xor_sync(kFullMask, t, o));
        }
        if (lane == 0) {
            key[v] = uint32_t(t);
            ids[v] = v;
        }
    }
}

// The HBM-tier variants with FP32 residuals keep at least three 128-thread blocks per SM (at most
// 168 registers, the occupancy they had before the windowed push and the column edge bound were
// added): their phases are latency-bound on HBM and need the warps.  The FP64 variant compiled to
// about 240 registers (two blocks per SM) without spills before and is left so.
template <class Real, class Acc, bool SMEM, bool JACOBI, class Pack>
__global__ void __launch_bounds__(kSrcMaxThreads, (!SMEM && sizeof(Real) == 4) ? 3 : 1)
source_kernel(Pack pk) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t s_pre[Pack::kMax + 1];  // item prefix over the pack's row lists
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t wib = threadIdx.x >> 5;
    const uint32_t wpb = blockDim.x >> 5;
    const uint64_t gw = uint64_t(blockIdx.x) * wpb + wib;
    // the per-warp scratch (shared by every graph of the pack) comes from the first entry
    const SourceParams<Real, Acc>& p0 = pk.g[0];
    const uint32_t sn = p0.scratch_n;
    const unsigned lt = (1u << lane) - 1u;
    constexpr uint32_t NONE = 0xffffffffu;
    Real* pvec;
    unsigned char* vis;       // per vertex: 1 = discovered this round, 2 = in the top-gamma set
    unsigned long long* acc;  // 64 per warp: per-slot neighbourhood max (0..31) / min (32..63)
    unsigned long long* fx;   // Jacobi push: per-vertex fixed-point accumulators (all zero between rounds)
    if (SMEM) {
        unsigned char* base = smem + size_t(wib) * p0.smem_per_warp;
        pvec = reinterpret_cast<Real*>(base);
        const size_t pv = (size_t(sn) * sizeof(Real) + 15) & ~size_t(15);
        vis = base + pv;
        const size_t vb = (size_t(sn) + 15) & ~size_t(15);
        // the fixed-point accumulators live in shared memory when they fit beside the residual
        // vector, else in HBM (p0.fx_g)
        const bool fx_here = JACOBI && p0.fx_g == nullptr;
        fx = fx_here ? reinterpret_cast<unsigned long long*>(base + pv + vb)
                     : (JACOBI ? p0.fx_g + gw * size_t(sn) : nullptr);
        acc = reinterpret_cast<unsigned long long*>(base + pv + vb +
                                                    (fx_here ? sizeof(unsigned long long) * sn : 0));
    } else {
        pvec = p0.pvec_g + gw * size_t(sn);
        vis = p0.vis_g + gw * p0.vis_stride;
        fx = JACOBI ? p0.fx_g + gw * size_t(sn) : nullptr;
        acc = reinterpret_cast<unsigned long long*>(smem + size_t(wib) * kAccBytes);
    }
    // pvec and flags are zeroed once, before the warp's first source, unless the warp's last run
    // (same layout, HBM tier) left them zero: every source resets what it touched
    bool cleared = !SMEM && p0.wclean[gw] != 0;
    bool dirty = false;  // a source stopped midway (time-out): its vectors are not zero
    uint32_t* qa = p0.qbuf + gw * 2 * size_t(sn);
    uint32_t* qb = qa + sn;
    WalkItem* items = p0.items + gw * size_t(p0.max_degree);
    unsigned long long st_rounds = 0, st_pv = 0, st_tr = 0, st_we = 0, st_wc = 0, st_wh = 0,
                       st_fb = 0;
    const uint64_t deadline = globaltimer_ns() + p0.budget_ns;
    // SM cycles spent per phase of a source (claim/init, push, post-push, cost test, edge bound,
    // chi/nr, walks, reset), summed over the warp's sources
    long long ph[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long tmark = clock64();
    auto lap = [&](int i) {
        const long long now = clock64();
        ph[i] += now - tmark;
        tmark = now;
    };

    // Run counters go to the stats of the graph a source belongs to: flushed when a warp moves
    // to another graph of the pack, and at the end.
    auto flush_stats = [&](unsigned long long* stats) {
        if (lane == 0) {
            stat_add(stats, kStPushRounds, st_rounds);
            stat_add(stats, kStPushVertices, st_pv);
            stat_add(stats, kStPushTraversals, st_tr);
        }
        st_we = warp_sum_u64(st_we);
        st_wc = warp_sum_u64(st_wc);
        st_wh = warp_sum_u64(st_wh);
        st_fb = warp_sum_u64(st_fb);
        if (lane == 0) {
            stat_add(stats, kStWalkEdges, st_we);
            stat_add(stats, kStWalkCount, st_wc);
            stat_add(stats, kStWalkHops, st_wh);
            stat_add(stats, kStFallback, st_fb);
#pragma unroll
            for (int i = 0; i < 8; ++i) stat_add(stats, kStPhase0 + i, (unsigned long long)ph[i]);
        }
        st_rounds = st_pv = st_tr = st_we = st_wc = st_wh = st_fb = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) ph[i] = 0;
    };
    __syncwarp();

    pdl_launch_dependents();
    pdl_wait();  // taus, row lists and their lengths from the tau kernels
    // items: the listed rows of the pack's graphs one after another (a list's length is final:
    // the tau kernel that appends to it has ended)
    if (threadIdx.x == 0) {
        uint32_t acc_items = 0;
        s_pre[0] = 0;
        for (uint32_t i = 0; i < pk.count; ++i) {
            const SourceParams<Real, Acc>& gp = pk.g[i];
            const unsigned total = gp.work[2];
            acc_items += total > gp.list_base ? min(total - gp.list_base, gp.list_cap) : 0u;
            s_pre[i + 1] = acc_items;
        }
    }
    __syncthreads();
    const unsigned nrows = s_pre[pk.count];
    // item gw first, then items past the grid's warps claimed one at a time (warps past the
    // end leave without touching the counter)
    const uint64_t nwarps = uint64_t(gridDim.x) * wpb;
    bool first_claim = true;
    uint32_t last_gi = 0xffffffffu;
    while (true) {
        uint64_t k = gw;
        if (!first_claim) {
            unsigned c = 0;
            if (lane == 0) c = atomicAdd(p0.claim, 1u);
            k = nwarps + __shfl_sync(kFullMask, c, 0);
        }
        first_claim = false;
        if (k >= nrows) break;
        // the item's graph: the last list whose prefix is at most k (warp-uniform)
        uint32_t gi = 0;
        if (Pack::kMax > 1) {
            uint32_t lo = 0, hi = pk.count;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (s_pre[mid] <= k) lo = mid;
                else hi = mid;
            }
            gi = lo;
        }
        const SourceParams<Real, Acc>& p = pk.g[gi];
        if (gi != last_gi) {
            if (last_gi != 0xffffffffu) flush_stats(pk.g[last_gi].stats);
            last_gi = gi;
        }
        if (globaltimer_ns() > deadline) {
            if (lane == 0) atomicOr(p.work + 1, kErrDeadline);
            break;
        }
        const uint32_t n = p.n;
        const uint32_t* __restrict__ idx = p.idx;
        const uint32_t* __restrict__ adj = p.adj;
        const int* __restrict__ taus = p.taus;
        const uint32_t entry = p.list_base + uint32_t(k - s_pre[gi]);
        const uint32_t src = __ldg(p.rows + entry);
        if (!cleared) {
            for (uint32_t i = lane; i < sn; i += 32) {
                pvec[i] = Real(0);
                vis[i] = 0;
                if (JACOBI) fx[i] = 0ull;
            }
            cleared = true;
            __syncwarp();
        }
        uint32_t* q = qa;
        uint32_t* qn = qb;
        const uint32_t rb = __ldg(idx + src), re = __ldg(idx + src + 1);
        const uint32_t dsi = re - rb;
        const Real ds = from_u64<Real>(dsi);
        // preds = 1.0 / ds (:468-470); stored together with the first round's update below
        const Acc pinit = from_f64<Acc>(__ddiv_rn(1.0, double(ds)));
        uint32_t qs = 0;
        int ell = 0;
        Real gmin, gmax;
        bool timed_out = false;
        unsigned long long pcost = 0;
        Real mx = Real(0), mn = Real(1);
        // row loaders (neighbour, tau) for the pipelined passes over the source's row
        auto load_adj = [&](uint32_t c, uint32_t* r) {
#pragma unroll
            for (int b = 0; b < kB; ++b) {
                const uint32_t o = c + 32 * b + lane;
                r[b] = o < dsi ? __ldg(adj + rb + o) : NONE;
            }
        };
        auto load_tau = [&](uint32_t c, int* r) {
#pragma unroll
            for (int b = 0; b < kB; ++b) {
                const uint32_t o = c + 32 * b + lane;
                r[b] = o < dsi ? __ldg(taus + rb + o) : 0;
            }
        };
        lap(0);
        if (p.pre) {
            // The push ran in push_block_kernel, which left the source's final residual vector as
            // n contiguous floats (its column, transposed into the CTA's other block buffer).  The
            // HBM tier reads it in place; the shared-memory tier copies it.  The final frontier
            // (the support) is rebuilt in vertex order.
            const PrePush pr = p.pre[entry];
            const uint32_t slot = entry - p.list_base;
            const uint32_t cta = slot / kBlockCols, col = slot % kBlockCols;
            const float* cb = p.pre_cols +
                              (size_t(cta) * 2 + (1u - p.pre_final[cta])) * size_t(n) * kBlockCols +
                              size_t(col) * n;
            if constexpr (!SMEM && std::is_same<Real, float>::value) pvec = const_cast<Real*>(cb);
            uint32_t cq = 0;
            // HBM tier: the column is read in place and the edge bound selects from it directly
            // (its positive entries are the frontier, in vertex order), so no frontier list is
            // built; the shared-memory tier copies the column and lists the frontier.  The scan
            // keeps 2 x kB coalesced 128-byte loads in flight (pipelined).
            if (!SMEM) cq = pr.support;
            else pipelined<Real>(n,
                [&](uint32_t i0, Real* r) {
#pragma unroll
                    for (int b = 0; b < kB; ++b) {
                        const uint32_t i = i0 + 32 * b + lane;
                        r[b] = i < n ? Real(cb[i]) : Real(0);
                    }
                },
                [&](uint32_t i0, const Real* r) {
#pragma unroll
                    for (int b = 0; b < kB; ++b) {
                        const uint32_t i = i0 + 32 * b + lane;
                        if (SMEM && i < n) pvec[i] = r[b];
                        const bool nz = r[b] > Real(0);
                        const unsigned bal = __ballot_sync(kFullMask, nz);
                        if (nz) q[cq + __popc(bal & lt)] = i;
                        cq += __popc(bal);
                    }
                });
            __syncwarp();
            qs = cq;
            ell = pr.ell;
            gmax = Real(pr.gmax);
            gmin = qs < n ? Real(0) : Real(pr.gmin);
            lap(1);
        } else {
            // ---- round 1 in closed form (:457-503, first pass of the loop) ----
            // The frontier is {src} with residual 1 (pvec[src] = 1.0, then zeroed as it is drained):
            // every neighbour u is discovered in row order and receives 0 + 1/deg(u) = 1/deg(u), so
            // the round's new frontier, residuals, degree sum, max / min and row update
            // preds = 1/ds + (0 - 1/deg(u)) / ds follow from one pass over the row when the
            // neighbours are distinct.  Rows of a graph with repeated neighbours or self-loops
            // (p.multi, parity forms) take the general path below instead.
            if (!JACOBI && p.multi) {
                // (1) each run of one neighbour u (rows are sorted, so repeats are adjacent) is
                // handled by its first slot: k repeats add 1/deg(u) k times in order, as the
                // reference's sequential += does; that slot discovers u (first-occurrence order)
                // and adds deg(u) to picost.  pvec[src] starts at 0 (it was drained), so a
                // self-loop run adds to it like to any neighbour.
                uint32_t found = 0;
                for (uint32_t c = 0; c < dsi; c += 32) {
                    const uint32_t o = c + lane;
                    const bool in = o < dsi;
                    const uint2 a = in ? __ldg(p.adjd + rb + o) : make_uint2(NONE, 1u);
                    const bool lead = in && (o == 0 || __ldg(adj + rb + o - 1) != a.x);
                    Real pu = Real(0);
                    if (lead) {
                        const Real x = rdiv(Real(1), from_u64<Real>(a.y));
                        pu = x;
                        for (uint32_t k = o + 1; k < dsi && __ldg(adj + rb + k) == a.x; ++k)
                            pu = radd(pu, x);
                        pvec[a.x] = pu;
                        pcost += a.y;
                        mx = std_max(mx, pu);
                        mn = std_min(mn, pu);
                    }
                    const unsigned bl = __ballot_sync(kFullMask, lead);
                    if (lead) qn[found + __popc(bl & lt)] = a.x;
                    found += __popc(bl);
                }
                __syncwarp();
                // (2) preds[s -> t] = 1/ds + (pvec[s] - pvec[t]) / ds with the round's residuals
                const Real ps = pvec[src];
                for (uint32_t o = lane; o < dsi; o += 32)
                    p.preds[rb + o] = row_update<Real, Acc>(pinit, ps, pvec[__ldg(adj + rb + o)], ds);
                qs = found;
            } else {
            pipelined<uint2>(dsi,
                [&](uint32_t c, uint2* r) {
    #pragma unroll
                    for (int b = 0; b < kB; ++b) {
                        const uint32_t o = c + 32 * b + lane;
                        r[b] = o < dsi ? __ldg(p.adjd + rb + o) : make_uint2(NONE, 1u);
                    }
                },
                [&](uint32_t c, const uint2* r) {
    #pragma unroll
                    for (int b = 0; b < kB; ++b) {
                        if (r[b].x == NONE) continue;
                        const uint32_t o = c + 32 * b + lane;
                        const Real pu = JACOBI ? Real(from_fixed(kFixOne, r[b].y))
                                               : rdiv(Real(1), from_u64<Real>(r[b].y));
                        pvec[r[b].x] = pu;
                        qn[o] = r[b].x;
                        pcost += r[b].y;
                        mx = std_max(mx, pu);
                        mn = std_min(mn, pu);
                        p.preds[rb + o] = row_update<Real, Acc>(pinit, Real(0), pu, ds);
                    }
                });
            qs = dsi;
            }
            st_pv += 1;
            st_tr += dsi;
            ell = 1;
            { uint32_t* tmp = q; q = qn; qn = tmp; }
            __syncwarp();
            lap(1);
            while (true) {
                // ---- the push/walk cost test (:483-502) ----
                const double picost = double(warp_sum_u64(pcost));
                gmax = warp_max(mx);
                gmin = warp_min(mn);
                gmin = qs < n ? Real(0) : gmin;
                const double dse0 = __dmul_rn(double(ds), p.eps);
                const double dse2 = __dmul_rn(dse0, dse0);
                double rw = 0;
                pipelined<int>(dsi, load_tau, [&](uint32_t c, const int* tv) {
    #pragma unroll
                    for (int b = 0; b < kB; ++b) {
                        const uint32_t o = c + 32 * b + lane;
                        const int rest = tv[b] - ell;
                        double nrd = 0;
                        const bool has = o < dsi && rest > 0;
                        if (has) {
                            const double chi = __dmul_rn(__dmul_rn(2.0, double(rest)),
                                                         __dsub_rn(double(gmax), double(gmin)));
                            const double num = __dmul_rn(__dmul_rn(8.0, __dmul_rn(chi, chi)), p.logmd);
                            nrd = std_max(ceil(__ddiv_rn(num, dse2)), 1.0);
                        }
                        unsigned hb = __ballot_sync(kFullMask, has);
                        while (hb) {  // rwcost += nr in slot order
                            const int l = __ffs(hb) - 1;
                            hb &= hb - 1;
                            rw = __dadd_rn(rw, __shfl_sync(kFullMask, nrd, l));
                        }
                    }
                });
                lap(3);
                if (picost >= __dmul_rn(25.0, rw)) break;
                if (globaltimer_ns() > deadline) {
                    timed_out = true;
                    break;
                }
                uint32_t qns = 0;
                pcost = 0;
                st_pv += qs;
                if constexpr (!JACOBI) {
                if (p.gs_window) {
                // ---- diffuse (:218-239), windowed ----
                // The reference drains the frontier one vertex at a time: r = pvec[v], pvec[v] = 0,
                // then pvec[u] += r / deg(u) for u in N(v) in row order, discovering each u on its
                // first visit.  Here up to 32 consecutive frontier vertices form a window whose
                // residuals are taken at once and whose rows are concatenated and processed 32
                // entries per step, in order.  That gives the reference's values as long as no
                // entry of a window vertex j targets a later window vertex k (it would have changed
                // r_k before k was drained): such an entry cuts the window before k -- found before
                // anything of its step is applied, the cut vertices get their residuals back and
                // are drained by a later window.  Entries targeting the vertex itself or an earlier
                // window vertex are ordinary adds (those were drained first in the reference too).
                // Lanes of one step that hit the same neighbour form a group whose lowest lane adds
                // the group's contributions one by one in lane (= the reference's) order; the
                // lowest lane is also the first visit, so discovery order is the reference's.  vis
                // holds 1 + the window index in its upper six bits while a vertex is in a window.
                uint32_t* exs = reinterpret_cast<uint32_t*>(acc + 64 + 32);  // 33 entry offsets
                uint32_t* vbs = exs + 33;                                     // 32 row starts
                for (uint32_t i0 = 0; i0 < qs;) {
                    const uint32_t cnt = min(32u, qs - i0);
                    uint32_t myv = 0, vb = 0, vd = 0;
                    Real rv = Real(0);
                    if (lane < cnt) {
                        myv = q[i0 + lane];
                        vb = __ldg(idx + myv);
                        vd = __ldg(idx + myv + 1) - vb;
                        rv = pvec[myv];
                    }
                    __syncwarp();
                    if (lane < cnt) {
                        pvec[myv] = Real(0);
                        vis[myv] = (unsigned char)((vis[myv] & 3u) | ((lane + 1u) << 2));
                    }
                    uint32_t incl = vd;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t y = __shfl_up_sync(kFullMask, incl, o);
                        if (lane >= uint32_t(o)) incl += y;
                    }
                    const uint32_t total = __shfl_sync(kFullMask, incl, 31);
                    exs[lane] = incl - vd;
                    vbs[lane] = vb;
                    if (lane == 31) exs[32] = total;
                    __syncwarp();
                    uint32_t wend = cnt;  // the window: frontier vertices i0 .. i0 + wend - 1
                    uint32_t pm = 0;      // entry cursor of the loader (one step ahead)
                    auto load_step = [&](uint32_t e0, uint32_t& cur_m, uint32_t& sg, uint2& a) {
                        const uint32_t e = e0 + lane;
                        sg = 32u;
                        a = make_uint2(NONE, 1u);
                        if (e < total) {
                            while (exs[cur_m + 1] <= e) ++cur_m;
                            sg = cur_m;
                            a = __ldg(p.adjd + vbs[cur_m] + (e - exs[cur_m]));
                        }
                    };
                    uint32_t sg = 32u, nsg = 32u;
                    uint2 ea, nea;
                    load_step(0u, pm, sg, ea);
                    for (uint32_t e0 = 0; e0 < total; e0 += 32) {
                        if (e0 + 32 < total) load_step(e0 + 32, pm, nsg, nea);
                        if (__all_sync(kFullMask, sg >= wend)) break;  // past the (cut) window
                        const bool valid = sg < wend;
                        const uint32_t u = ea.x, du = ea.y;
                        const uint32_t vv = valid ? uint32_t(vis[u]) : 0u;
                        const uint32_t wk = vv >> 2;  // 1 + window index of u, 0 if none
                        const bool conflict = valid && wk > sg + 1u;
                        if (__any_sync(kFullMask, conflict)) {
                            uint32_t kmin = conflict ? wk - 1u : 32u;
#pragma unroll
                            for (int o = 16; o; o >>= 1) kmin = min(kmin, __shfl_xor_sync(kFullMask, kmin, o));
                            // window vertices kmin .. wend - 1 leave the window undrained
                            if (lane >= kmin && lane < wend) {
                                pvec[myv] = rv;
                                vis[myv] = (unsigned char)(vis[myv] & 3u);
                            }
                            wend = kmin;
                            __syncwarp();
                        }
                        const bool apply = sg < wend;
                        const uint32_t vis_u = apply ? uint32_t(vis[u]) : 0u;
                        const unsigned grp = __match_any_sync(kFullMask, apply ? u : (0xffffffe0u | lane));
                        const bool lead = apply && lane == uint32_t(__ffs(grp) - 1);
                        const Real r = __shfl_sync(kFullMask, rv, int(sg & 31u));
                        const Real c = apply ? rdiv(r, from_u64<Real>(du)) : Real(0);
                        bool fresh = false;
                        if (lead && (vis_u & 1u) == 0u) {
                            vis[u] = (unsigned char)(vis_u | 1u);
                            fresh = true;
                        }
                        const unsigned bal = __ballot_sync(kFullMask, fresh);
                        if (fresh) {
                            qn[qns + __popc(bal & lt)] = u;
                            pcost += du;
                        }
                        qns += __popc(bal);
                        const unsigned others = __ballot_sync(kFullMask, apply && !lead);
                        Real pv = Real(0);
                        if (lead) pv = radd(pvec[u], c);
                        for (unsigned mm = others; mm; mm &= mm - 1) {
                            const int t = __ffs(mm) - 1;
                            const Real ct = __shfl_sync(kFullMask, c, t);
                            if (lead && ((grp >> t) & 1u)) pv = radd(pv, ct);
                        }
                        if (lead) pvec[u] = pv;
                        __syncwarp();
                        sg = nsg;
                        ea = nea;
                        nsg = 32u;
                    }
                    if (lane < wend) vis[myv] = (unsigned char)(vis[myv] & 3u);
                    st_tr += __shfl_sync(kFullMask, incl, int(wend - 1));
                    __syncwarp();
                    i0 += wend;
                }
                } else {
                // ---- diffuse (:218-239) ----
                // The frontier is drained in order, one vertex at a time; the lanes share the
                // vertex's adjacency (distinct neighbours, so the lanes' flag and residual updates
                // touch distinct bytes and words).  Per batch of 32 frontier vertices the adjacency is
                // cut into 32-slot chunks walked by a cursor; a chunk's (neighbour, degree) pairs are
                // one coalesced 8-byte load per lane, issued kPushAhead chunks before use.  picost (the
                // new frontier's degree sum) is summed on discovery.  Every vertex has at least one
                // chunk: tgtp_run rejects isolated vertices.

                for (uint32_t i0 = 0; i0 < qs; i0 += 32) {
                    uint32_t myv = 0, myb = 0, myd = 0;
                    if (i0 + lane < qs) {
                        myv = q[i0 + lane];
                        myb = __ldg(idx + myv);
                        myd = __ldg(idx + myv + 1) - myb;
                    }
                    const uint32_t cnt = min(32u, qs - i0);
                    uint32_t pt = 0, pc = 0;  // prefetch cursor: batch vertex, chunk offset
                    uint2 cur[kPushAhead];
                    uint32_t ct[kPushAhead], cco[kPushAhead];
                    auto load_group = [&](uint2* dst, uint32_t* dt, uint32_t* dc) {
    #pragma unroll
                        for (int jj = 0; jj < kPushAhead; ++jj) {
                            dst[jj] = make_uint2(0u, 1u);
                            dt[jj] = cnt;
                            dc[jj] = 0;
                            if (pt < cnt) {
                                const uint32_t vb = __shfl_sync(kFullMask, myb, pt);
                                const uint32_t vd = __shfl_sync(kFullMask, myd, pt);
                                if (pc + lane < vd) dst[jj] = __ldg(p.adjd + vb + pc + lane);
                                dt[jj] = pt;
                                dc[jj] = pc;
                                pc += 32;
                                if (pc >= vd) {
                                    ++pt;
                                    pc = 0;
                                }
                            }
                        }
                    };
                    load_group(cur, ct, cco);
                    Real r = Real(0);
                    while (ct[0] < cnt) {
                        uint2 nxt[kPushAhead];
                        uint32_t nt[kPushAhead], nc[kPushAhead];
                        load_group(nxt, nt, nc);
    #pragma unroll
                        for (int jj = 0; jj < kPushAhead; ++jj) {
                            if (ct[jj] < cnt) {
                                const uint32_t t = ct[jj], c0 = cco[jj];
                                const uint32_t vd = __shfl_sync(kFullMask, myd, t);
                                if (c0 == 0) {
                                    const uint32_t v = __shfl_sync(kFullMask, myv, t);
                                    r = pvec[v];
                                    __syncwarp();
                                    if (lane == 0) pvec[v] = Real(0);
                                    __syncwarp();
                                    st_tr += vd;
                                }
                                const bool act = c0 + lane < vd;
                                const uint32_t cu = cur[jj].x, cd = cur[jj].y;
                                // a run of one repeated neighbour (adjacent lanes: rows are
                                // sorted) is applied by its first lane, one add per repeat in
                                // order; runs continued from the previous chunk were applied
                                // before this one, as the reference's sequential loop does
                                bool lead = act;
                                uint32_t reps = 1;
                                if (!JACOBI && p.multi) {
                                    const uint32_t pcu = __shfl_up_sync(kFullMask, cu, 1);
                                    const bool follow = act && lane > 0 && pcu == cu;
                                    const unsigned fb = __ballot_sync(kFullMask, follow);
                                    lead = act && !follow;
                                    const unsigned rest = lane == 31 ? 0u : (fb >> (lane + 1));
                                    reps = uint32_t(__ffs(int(~rest)));
                                }
                                bool fresh = false;
                                if (lead && vis[cu] == 0) {
                                    vis[cu] = 1;
                                    fresh = true;
                                }
                                const unsigned bal = __ballot_sync(kFullMask, fresh);
                                if (fresh) {
                                    qn[qns + __popc(bal & lt)] = cu;
                                    pcost += cd;
                                }
                                qns += __popc(bal);
                                if (lead) {
                                    const Real add = rdiv(r, from_u64<Real>(cd));
                                    Real pv = pvec[cu];
                                    for (uint32_t k = 0; k < reps; ++k) pv = radd(pv, add);
                                    pvec[cu] = pv;
                                }
                                __syncwarp();
                            }
                        }
    #pragma unroll
                        for (int jj = 0; jj < kPushAhead; ++jj) {
                            cur[jj] = nxt[jj];
                            ct[jj] = nt[jj];
                            cco[jj] = nc[jj];
                        }
                    }
                }
                }
                } else {
                    // ---- Jacobi push (mixed form) ----
                    // The frontier's residuals are taken together, in 2^-62 fixed point
                    // (r_i = to_fixed(pvec[q_i]), pvec[q_i] = 0, read as each group of 32 frontier
                    // vertices starts: the round's pushes go to the accumulators, never to pvec, so
                    // every r_i is the value the round started with), then pushed over the
                    // concatenated adjacency of 32 frontier vertices at a time: each lane walks
                    // entries lane, lane + 32, ... with a cursor over the vertices' start offsets,
                    // and every entry (v -> u) adds r_v to u's 64-bit accumulator with an integer
                    // atomic, so the sums do not depend on the order.  The touched vertices form the
                    // new frontier in discovery order; once the round is over their residuals become
                    // acc[u] / deg(u) (from_fixed), exactly as push_block_kernel computes them.
                    unsigned long long* rvs = acc + 64;
                    uint32_t* exs = reinterpret_cast<uint32_t*>(rvs + 32);
                    uint32_t* vbs = exs + 33;
                    for (uint32_t i0 = 0; i0 < qs; i0 += 32) {
                        uint32_t vb = 0, vd = 0;
                        unsigned long long rv = 0;
                        if (i0 + lane < qs) {
                            const uint32_t v = q[i0 + lane];
                            vb = __ldg(idx + v);
                            vd = __ldg(idx + v + 1) - vb;
                            rv = to_fixed(float(pvec[v]));
                            pvec[v] = Real(0);
                        }
                        uint32_t incl = vd;
#pragma unroll
                        for (int o = 1; o < 32; o <<= 1) {
                            const uint32_t y = __shfl_up_sync(kFullMask, incl, o);
                            if (lane >= uint32_t(o)) incl += y;
                        }
                        const uint32_t total = __shfl_sync(kFullMask, incl, 31);
                        exs[lane] = incl - vd;
                        vbs[lane] = vb;
                        rvs[lane] = rv;
                        if (lane == 31) exs[32] = total;
                        __syncwarp();
                        st_tr += total;
                        uint32_t cm = 0;
                        struct PEnt {
                            uint32_t seg, u, du;
                        };
                        pipelined<PEnt>(total,
                            [&](uint32_t e0, PEnt* r) {
#pragma unroll
                                for (int b = 0; b < kB; ++b) {
                                    const uint32_t e = e0 + 32 * b + lane;
                                    r[b].seg = 32u;
                                    r[b].u = NONE;
                                    r[b].du = 1u;
                                    if (e < total) {
                                        while (exs[cm + 1] <= e) ++cm;
                                        const uint2 a = __ldg(p.adjd + vbs[cm] + (e - exs[cm]));
                                        r[b].seg = cm;
                                        r[b].u = a.x;
                                        r[b].du = a.y;
                                    }
                                }
                            },
                            [&](uint32_t, const PEnt* r) {
#pragma unroll
                                for (int b = 0; b < kB; ++b) {
                                    const bool valid = r[b].seg < 32u;
                                    const uint32_t u = r[b].u;
                                    // entries of one frontier vertex are distinct neighbours; only a
                                    // step that spans several vertices can repeat one, and then the
                                    // first lane of a repeated neighbour adds the group's residuals
                                    // (integers: any order gives the same sum) and discovers it.
                                    // The accumulators are this warp's own, so with one writer per
                                    // neighbour a step needs no atomics.
                                    unsigned long long add = valid ? rvs[r[b].seg] : 0ull;
                                    const uint32_t seg0 = __shfl_sync(kFullMask, r[b].seg, 0);
                                    const bool one_seg = __all_sync(kFullMask, !valid || r[b].seg == seg0);
                                    const unsigned grp =
                                        one_seg ? (1u << lane) : __match_any_sync(kFullMask, u);
                                    const bool leader = valid && lane == uint32_t(__ffs(grp) - 1);
                                    if (!one_seg) {
                                        const unsigned others = __ballot_sync(kFullMask, valid && !leader);
                                        for (unsigned mm = others; mm; mm &= mm - 1) {
                                            const int t = __ffs(mm) - 1;
                                            const unsigned long long ct = __shfl_sync(kFullMask, add, t);
                                            if (leader && ((grp >> t) & 1u)) add += ct;
                                        }
                                    }
                                    if (leader) fx[u] += add;
                                    bool fresh = false;
                                    if (leader && vis[u] == 0) {
                                        vis[u] = 1;
                                        fresh = true;
                                    }
                                    const unsigned bal = __ballot_sync(kFullMask, fresh);
                                    if (fresh) {
                                        qn[qns + __popc(bal & lt)] = u;
                                        pcost += r[b].du;
                                    }
                                    qns += __popc(bal);
                                    __syncwarp();
                                }
                            });
                        __syncwarp();
                    }
                    // the touched vertices' new residuals; in the same pass their flags are
                    // cleared and their residual max / min taken (:484-491), which the GS push
                    // does after the row update below (neither touches what it reads)
                    mx = Real(0);
                    mn = Real(1);
                    pipelined<uint32_t>(qns,
                        [&](uint32_t i0, uint32_t* r) {
#pragma unroll
                            for (int b = 0; b < kB; ++b) {
                                const uint32_t i = i0 + 32 * b + lane;
                                r[b] = i < qns ? qn[i] : NONE;
                            }
                        },
                        [&](uint32_t, const uint32_t* r) {
#pragma unroll
                            for (int b = 0; b < kB; ++b) {
                                if (r[b] == NONE) continue;
                                const Real val = Real(from_fixed(fx[r[b]], __ldg(p.deg + r[b])));
                                pvec[r[b]] = val;
                                fx[r[b]] = 0ull;
                                vis[r[b]] = 0;
                                mx = std_max(mx, val);
                                mn = std_min(mn, val);
                            }
                        });
                }
                __syncwarp();
                lap(1);
                // preds[row] += (pvec[src] - pvec[adj]) / ds (:235-237); the first round adds to the
                // initial 1 / ds directly
                {
                    const Real ps = pvec[src];
                    struct SlotPred {
                        uint32_t w;
                        Acc old;
                    };
                    pipelined<SlotPred>(dsi,
                        [&](uint32_t c, SlotPred* r) {
    #pragma unroll
                            for (int b = 0; b < kB; ++b) {
                                const uint32_t o = c + 32 * b + lane;
                                r[b].w = NONE;
                                r[b].old = pinit;
                                if (o < dsi) {
                                    r[b].w = __ldg(adj + rb + o);
                                    if (ell > 0) r[b].old = p.preds[rb + o];
                                }
                            }
                        },
                        [&](uint32_t c, const SlotPred* r) {
    #pragma unroll
                            for (int b = 0; b < kB; ++b)
                                if (r[b].w != NONE)
                                    p.preds[rb + c + 32 * b + lane] =
                                        row_update<Real, Acc>(r[b].old, ps, pvec[r[b].w], ds);
                        });
                }
                // clear the new frontier's flags and take its residual max / min (:484-491; max and
                // min do not depend on order); the Jacobi push did this with its new residuals
                if constexpr (!JACOBI) {
                mx = Real(0);
                mn = Real(1);
                pipelined<uint32_t>(qns,
                    [&](uint32_t i0, uint32_t* r) {
    #pragma unroll
                        for (int b = 0; b < kB; ++b) {
                            const uint32_t i = i0 + 32 * b + lane;
                            r[b] = i < qns ? qn[i] : NONE;
                        }
                    },
                    [&](uint32_t, const uint32_t* r) {
    #pragma unroll
                        for (int b = 0; b < kB; ++b) {
                            if (r[b] == NONE) continue;
                            vis[r[b]] = 0;
                            const Real val = pvec[r[b]];
                            mx = std_max(mx, val);
                            mn = std_min(mn, val);
                        }
                    });
                }
                __syncwarp();
                { uint32_t* tmp = q; q = qn; qn = tmp; }
                qs = qns;
                ++ell;
                lap(2);
            }
        }
        if (timed_out) {
            if (lane == 0) atomicOr(p.work + 1, kErrDeadline);
            dirty = true;
            break;
        }
        if (!p.pre) st_rounds += ell;  // PrePush rounds are counted by push_block_kernel
        if (p.trace_ell && lane == 0) p.trace_ell[src] = uint32_t(ell);

        // slots that still need walks (rest = tau - ell > 0), compacted in slot order
        uint32_t nitems = 0;
        pipelined<int>(dsi, load_tau, [&](uint32_t c, const int* tv) {
#pragma unroll
            for (int b = 0; b < kB; ++b) {
                const uint32_t o = c + 32 * b + lane;
                const bool has = o < dsi && tv[b] - ell > 0;
                const unsigned hb = __ballot_sync(kFullMask, has);
                if (has)
                    items[nitems + __popc(hb & lt)] =
                        WalkItem{rb + o, __ldg(adj + rb + o), uint32_t(tv[b] - ell), 0u, 0ull};
                nitems += __popc(hb);
            }
        });
        __syncwarp();

        // ---- edge bound (:414-442, :504-506); it only feeds chi of walking slots ----
        Real edge_max = Real(0);
        if (nitems == 0) {
        } else if (p.gamma == 1) {
            edge_max = rmul(Real(2), gmax);
        } else {
            const int nnz = int(qs);
            const int rg = p.gamma < nnz ? p.gamma : nnz;
            uint32_t* set = qn;  // free after the last swap
            int sc = 0;
            Real gamma_max;
            const bool from_col = !SMEM && p.pre != nullptr;  // select from the column
            if (p.gamma < nnz && from_col) {
                Real t;
                int need_eq;
                // top-gamma threshold and, for gamma <= kTopK, the list of the only entries that
                // can reach it (in index order, into q, free in this mode): the set is then taken
                // from that list instead of a second pass over the column
                const bool use_cand = rg <= kTopK;
                uint32_t nc = 0;
                kth_largest_col<Real>(pvec, n, rg, t, need_eq, use_cand ? q : nullptr, &nc);
                int taken_eq = 0;
                __syncwarp();
                if (use_cand) {
                    pipelined<uint32_t>(nc,
                        [&](uint32_t i0, uint32_t* r) {
#pragma unroll
                            for (int b = 0; b < kB; ++b) {
                                const uint32_t i = i0 + 32 * b + lane;
                                r[b] = i < nc ? q[i] : NONE;
                            }
                        },
                        [&](uint32_t, const uint32_t* r) {
#pragma unroll
                            for (int b = 0; b < kB; ++b) {
                                const bool valid = r[b] != NONE;
                                const Real v = valid ? pvec[r[b]] : Real(0);
                                const Real x = v > Real(0) ? v : Real(-INFINITY);
                                const bool gt = valid && x > t, eq = valid && x == t;
                                const unsigned be = __ballot_sync(kFullMask, eq);
                                const bool take_eq = eq && taken_eq + __popc(be & lt) < need_eq;
                                const bool take = (gt || take_eq) && sc < rg;
                                const unsigned bt = __ballot_sync(kFullMask, take);
                                if (take) set[sc + __popc(bt & lt)] = r[b];
                                sc += __popc(bt);
                                taken_eq += __popc(__ballot_sync(kFullMask, take_eq));
                            }
                        });
                } else
                pipelined<Real>(n,
                    [&](uint32_t i0, Real* r) {
#pragma unroll
                        for (int b = 0; b < kB; ++b) {
                            const uint32_t i = i0 + 32 * b + lane;
                            r[b] = i < n ? pvec[i] : Real(0);
                        }
                    },
                    [&](uint32_t i0, const Real* r) {
#pragma unroll
                        for (int b = 0; b < kB; ++b) {
                            const uint32_t i = i0 + 32 * b + lane;
                            const Real x = r[b] > Real(0) ? r[b] : Real(-INFINITY);
                            const bool gt = x > t, eq = x == t;
                            const unsigned be = __ballot_sync(kFullMask, eq);
                            const bool take_eq = eq && taken_eq + __popc(be & lt) < need_eq;
                            const bool take = (gt || take_eq) && sc < rg;
                            const unsigned bt = __ballot_sync(kFullMask, take);
                            if (take) set[sc + __popc(bt & lt)] = i;
                            sc += __popc(bt);
                            taken_eq += __popc(__ballot_sync(kFullMask, take_eq));
                        }
                    });
                gamma_max = std_min(Real(1), t);
            } else if (from_col) {
                // every frontier vertex is in the set: the column's positive entries in order
                pipelined<Real>(n,
                    [&](uint32_t i0, Real* r) {
#pragma unroll
                        for (int b = 0; b < kB; ++b) {
                            const uint32_t i = i0 + 32 * b + lane;
                            r[b] = i < n ? pvec[i] : Real(0);
                        }
                    },
                    [&](uint32_t i0, const Real* r) {
#pragma unroll
                        for (int b = 0; b < kB; ++b) {
                            const uint32_t i = i0 + 32 * b + lane;
                            const bool nz = r[b] > Real(0);
                            const unsigned bal = __ballot_sync(kFullMask, nz);
                            if (nz) set[sc + __popc(bal & lt)] = i;
                            sc += __popc(bal);
                        }
                    });
                gamma_max = Real(0);
            } else if (p.gamma < nnz) {
                Real t;
                int need_eq;
                kth_largest<Real>(q, qs, pvec, rg, t, need_eq);
                int taken_eq = 0;
                pipelined<uint32_t>(qs,
                    [&](uint32_t i0, uint32_t* r) {
#pragma unroll
                        for (int b = 0; b < kB; ++b) {
                            const uint32_t i = i0 + 32 * b + lane;
                            r[b] = i < qs ? q[i] : NONE;
                        }
                    },
                    [&](uint32_t, const uint32_t* r) {
#pragma unroll
                        for (int b = 0; b < kB; ++b) {
                            const Real x = r[b] != NONE ? pvec[r[b]] : Real(-INFINITY);
                            const bool gt = x > t, eq = x == t;
                            const unsigned be = __ballot_sync(kFullMask, eq);
                            const bool take_eq = eq && taken_eq + __popc(be & lt) < need_eq;
                            const bool take = (gt || take_eq) && sc < rg;
                            const unsigned bt = __ballot_sync(kFullMask, take);
                            if (take) set[sc + __popc(bt & lt)] = r[b];
                            sc += __popc(bt);
                            taken_eq += __popc(__ballot_sync(kFullMask, take_eq));
                        }
                    });
                gamma_max = std_min(Real(1), t);
            } else {
                for (uint32_t i = lane; i < qs; i += 32) set[i] = q[i];
                sc = int(qs);
                gamma_max = Real(0);
            }
            __syncwarp();
            edge_max = radd(gmax, gamma_max);
            for (int i = lane; i < sc; i += 32) vis[set[i]] = 2;
            __syncwarp();
            // pairs (u, w) with both in the set and w adjacent to u: the members' adjacency lists
            // are flattened 32 members at a time so a warp scans them in parallel
            Real best = edge_max;
            for (int s0 = 0; s0 < sc; s0 += 32) {
                uint32_t ub = 0, ud = 0;
                Real pu = Real(0);
                if (s0 + int(lane) < sc) {
                    const uint32_t u = set[s0 + lane];
                    pu = pvec[u];
                    ub = __ldg(idx + u);
                    ud = __ldg(idx + u + 1) - ub;
                }
                uint32_t incl = ud;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(kFullMask, incl, o);
                    if (lane >= uint32_t(o)) incl += y;
                }
                const uint32_t total = __shfl_sync(kFullMask, incl, 31);
                const uint32_t excl = incl - ud;
                for (uint32_t e0 = 0; e0 < total; e0 += 32) {
                    const uint32_t e = e0 + lane;
                    uint32_t mm = 0;
#pragma unroll
                    for (uint32_t step = 16; step; step >>= 1) {
                        const uint32_t cand = mm + step;
                        const uint32_t ex = __shfl_sync(kFullMask, excl, cand & 31u);
                        if (cand < 32u && ex <= e) mm = cand;
                    }
                    const uint32_t mb = __shfl_sync(kFullMask, ub, mm);
                    const uint32_t mex = __shfl_sync(kFullMask, excl, mm);
                    const Real mpu = __shfl_sync(kFullMask, pu, mm);
                    if (e < total) {
                        const uint32_t w = __ldg(adj + mb + (e - mex));
                        if (vis[w] == 2) best = std_max(best, radd(mpu, pvec[w]));
                    }
                }
            }
            edge_max = warp_max(best);
            __syncwarp();
            for (int i = lane; i < sc; i += 32) vis[set[i]] = 0;
            __syncwarp();
        }
        lap(4);

        // ---- chi and walk counts per edge (:392-412, :508-521) ----
        // Neighbourhood max / min of the walking slots' targets, 32 slots at a time: their
        // adjacency lists are concatenated and each lane walks entries lane, lane + 32, ... with a
        // cursor over the slots' start offsets (in shared memory; entries of a slot are
        // consecutive, so the cursor rarely moves), keeps its running max / min in registers and
        // flushes them with one shared atomic when it leaves a slot.  Then each lane forms its
        // slot's chi and nr with the reference's roundings.
        if (nitems) {
            Real smax = Real(0), smin = Real(FLT_MAX);
            pipelined<uint32_t>(dsi, load_adj, [&](uint32_t, const uint32_t* w) {
#pragma unroll
                for (int b = 0; b < kB; ++b) {
                    if (w[b] == NONE) continue;
                    const Real x = pvec[w[b]];
                    smax = std_max(smax, x);
                    smin = std_min(smin, x);
                }
            });
            smax = warp_max(smax);
            smin = warp_min(smin);
            const Real dse = from_f64<Real>(__dmul_rn(double(ds), p.eps));
            const double den = double(rmul(dse, dse));
            uint32_t* exs = reinterpret_cast<uint32_t*>(acc + 64);  // 33 slot offsets
            uint32_t* vbs = exs + 33;                               // 32 row starts
            for (uint32_t s0 = 0; s0 < nitems; s0 += 32) {
                const uint32_t my = s0 + lane;
                uint32_t vb = 0, vd = 0, L = 0;
                if (my < nitems) {
                    const WalkItem it = items[my];
                    vb = __ldg(idx + it.v);
                    vd = __ldg(idx + it.v + 1) - vb;
                    L = it.len;
                }
                acc[lane] = ord_bits(Real(0));
                acc[32 + lane] = ord_bits(Real(FLT_MAX));
                uint32_t incl = vd;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(kFullMask, incl, o);
                    if (lane >= uint32_t(o)) incl += y;
                }
                const uint32_t total = __shfl_sync(kFullMask, incl, 31);
                exs[lane] = incl - vd;
                vbs[lane] = vb;
                if (lane == 31) exs[32] = total;
                __syncwarp();
                uint32_t cm = 0;                  // address cursor
                uint32_t cseg = 32;               // accumulation cursor (32: none yet)
                Real amx = Real(0), amn = Real(FLT_MAX);
                auto flush = [&]() {
                    if (cseg < 32u) {
                        atomicMax(acc + cseg, ord_bits(amx));
                        atomicMin(acc + 32 + cseg, ord_bits(amn));
                    }
                };
                struct Ent {
                    uint32_t seg, w;
                };
                pipelined<Ent>(total,
                    [&](uint32_t e0, Ent* r) {
#pragma unroll
                        for (int b = 0; b < kB; ++b) {
                            const uint32_t e = e0 + 32 * b + lane;
                            r[b].seg = 32u;
                            r[b].w = 0u;
                            if (e < total) {
                                while (exs[cm + 1] <= e) ++cm;
                                r[b].seg = cm;
                                r[b].w = __ldg(adj + vbs[cm] + (e - exs[cm]));
                            }
                        }
                    },
                    [&](uint32_t, const Ent* r) {
#pragma unroll
                        for (int b = 0; b < kB; ++b) {
                            if (r[b].seg == 32u) continue;
                            if (r[b].seg != cseg) {
                                flush();
                                cseg = r[b].seg;
                                amx = Real(0);
                                amn = Real(FLT_MAX);
                            }
                            const Real x = pvec[r[b].w];
                            amx = std_max(amx, x);
                            amn = std_min(amn, x);
                        }
                    });
                flush();
                if (my < nitems) {
                    const Real tmax = from_ord<Real>(acc[lane]);
                    const Real tmin = from_ord<Real>(acc[32 + lane]);
                    // get_chi (:410): float terms rounded as in the reference, summed in double
                    const int Li = int(L);
                    const double A = __dadd_rn(double(gmax), __ddiv_rn(double(radd(smax, tmax)), 2.0));
                    const double B = __dadd_rn(A, double(rmul(Real(Li - 1), edge_max)));
                    const double C = __dsub_rn(__dsub_rn(B, double(smin)), double(tmin));
                    const double E = __dsub_rn(C, double(rmul(Real(2 * (Li - 1)), gmin)));
                    const Real chi = from_f64<Real>(E);
                    // nr (:519-521)
                    const Real c8 = rmul(Real(8), rmul(chi, chi));
                    const double num = __dmul_rn(double(c8), p.logmd);
                    const double nrd = std_max(ceil(__ddiv_rn(num, den)), 1.0);
                    unsigned long long nr = (unsigned long long)nrd;
                    nr += 8ull - (nr % 8ull);
                    if (nr > kMaxWalks) {
                        atomicOr(p.work + 1, kErrWalkCount);
                        nr = 0;  // skipped by the walk loop
                    } else {
                        st_we += 1;
                        st_wc += nr;
                        st_wh += nr * (unsigned long long)L;
                    }
                    items[my].nr = nr;
                    if (p.trace_nr) p.trace_nr[items[my].pos] = uint32_t(nr);
                }
                __syncwarp();
            }
        }
        lap(5);

        // ---- 2-way bouquet walks (:241-391): four bouquets per warp, one per 8-lane group ----
        if (nitems && p.walk_queue) {
            // handed to walk_queue_kernel / heavy_walk_kernel (the same walks, lanes and adds;
            // more warps in flight)
            for (uint32_t c = 0; c < nitems; c += 32) {
                const uint32_t i = c + lane;
                const bool has = i < nitems;
                WalkItem w{};
                bool heavy = false;
                if (has) {
                    w = items[i];
                    w.pad = entry;
                    heavy = w.nr >= kHeavyNr && w.len <= kHeavyLen;
                }
                const unsigned bh = __ballot_sync(kFullMask, has && heavy);
                const unsigned bl = __ballot_sync(kFullMask, has && !heavy);
                unsigned lb = 0, hb = 0;
                if (lane == 0) {
                    if (bl) lb = atomicAdd(p.walk_count, unsigned(__popc(bl)));
                    if (bh) hb = atomicAdd(p.walk_count + 2, unsigned(__popc(bh)));
                }
                lb = __shfl_sync(kFullMask, lb, 0);
                hb = __shfl_sync(kFullMask, hb, 0);
                if (has) {
                    if (heavy) p.walk_queue[p.walk_cap - 1u - (hb + __popc(bh & lt))] = w;
                    else p.walk_queue[lb + __popc(bl & lt)] = w;
                }
            }
        } else if (nitems) {
            const uint32_t j = lane & 7, grp = lane >> 3;
            uint32_t next = 0;
            bool has = false, start = false, primary = true;
            WalkItem it{};
            unsigned long long bi = 0;
            uint32_t len = 0, step = 0, cur = 0, cur2 = 0, sec = 0, sec2 = 0, state = 0;
            Real x = Real(0);
            // Each hop's residual difference is added to x one hop later (after the next hop's
            // row offsets are requested), so the residual loads overlap the next hop instead of
            // stalling it; the adds stay in hop order, and the last one is made before the
            // item's lanes are summed.
            Real pa = Real(0), pb = Real(0);
            bool pend = false;
            while (true) {
                const unsigned need = __ballot_sync(kFullMask, !has && j == 0);
                if (!has) {
                    const uint32_t rank = __popc(need & ((1u << (grp * 8)) - 1u));
                    const uint32_t my = next + rank;
                    if (my < nitems) {
                        it = items[my];
                        if (it.nr) {
                            has = true;
                            start = true;
                            bi = 0;
                            x = Real(0);
                            step = uint32_t(0xffffffffull / it.nr);
                        }
                    }
                }
                next += __popc(need);
                if (!__any_sync(kFullMask, has) && next >= nitems) break;
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
                    if (pend) x = radd(x, rsub(pa, pb));
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
                    pa = pvec[cur];
                    pb = pvec[cur2];
                    pend = true;
                    if (++len == it.len) {
                        bi += 8;
                        start = true;
                        item_done = bi >= it.nr;
                    }
                }
                if (__any_sync(kFullMask, item_done)) {
                    if (item_done && pend) {
                        x = radd(x, rsub(pa, pb));
                        pend = false;
                    }
                    if constexpr (std::is_same<Real, Acc>::value) {
                        // the eight lanes summed 0..7, then preds += xij / (ds * nr) (:386-390, :525)
                        Real s = Real(0);
#pragma unroll
                        for (int b = 0; b < 8; ++b)
                            s = radd(s, __shfl_sync(kFullMask, x, int(grp * 8 + b)));
                        if (item_done && j == 0)
                            p.preds[it.pos] =
                                radd(p.preds[it.pos], rdiv(s, rmul(ds, from_u64<Real>(it.nr))));
                    } else {
                        double s = 0;
#pragma unroll
                        for (int b = 0; b < 8; ++b)
                            s += double(__shfl_sync(kFullMask, x, int(grp * 8 + b)));
                        if (item_done && j == 0)
                            p.preds[it.pos] += s / (double(ds) * double(it.nr));
                    }
                    if (item_done) has = false;
                }
            }
        }
        lap(6);
        // ---- next source starts from an all-zero residual vector ----
        __syncwarp();
        if (!SMEM && p.pre) {
            // the residual vector was the block push's column, read in place: the warp's own
            // vector is untouched (and the flags used by the edge bound are back to zero)
            pvec = p0.pvec_g + gw * size_t(sn);
            lap(7);
            continue;
        }
        pipelined<uint32_t>(qs,
            [&](uint32_t i0, uint32_t* r) {
#pragma unroll
                for (int b = 0; b < kB; ++b) {
                    const uint32_t i = i0 + 32 * b + lane;
                    r[b] = i < qs ? q[i] : NONE;
                }
            },
            [&](uint32_t, const uint32_t* r) {
#pragma unroll
                for (int b = 0; b < kB; ++b)
                    if (r[b] != NONE) pvec[r[b]] = Real(0);
            });
        if (lane == 0) pvec[src] = Real(0);
        __syncwarp();
        lap(7);
    }
    if (!SMEM && lane == 0) p0.wclean[gw] = (cleared && !dirty) ? 1 : 0;
    flush_stats(pk.g[last_gi == 0xffffffffu ? 0u : last_gi].stats);
}

// ---- walks of the block push's sources, as their own launch --------------------------------------
// In PrePush mode the source kernel (a large kernel: 3 four-warp blocks per SM) leaves each
// source's walking slots in a queue; this lean kernel walks them with many more warps in flight.
// Everything a lane computes is what the source kernel's walk loop computes for the same item:
// an 8-lane group takes one item, lane j walks the item's walks j, j + 8, ... in order over the
// source's residual column, each hop's residual difference added to x in hop order, then the
// group's eight x are summed in lane order into preds[slot] (src/aesc.h:241-391, 524-525).
struct WalkQueueParams {
    const uint32_t* idx;
    const uint32_t* adj;
    const uint32_t* rows;      // list entry -> source
    const float* pre_cols;     // the block push's column blocks
    const uint32_t* pre_final;
    uint32_t list_base;        // first list entry of this wave
    uint32_t n;
    double* preds;
    const WalkItem* items;
    const unsigned* count;     // items in the queue
    unsigned* claim;           // next item (zeroed before the launch)
    unsigned long long* stats;
};
constexpr int kWalkThreads = 256;

__global__ void __launch_bounds__(kWalkThreads, 5) walk_queue_kernel(const WalkQueueParams q) {
    pdl_launch_dependents();
    pdl_wait();  // the queue and the columns of this wave
    const uint32_t lane = threadIdx.x & 31, j = lane & 7, grp = lane >> 3;
    const uint32_t total = *q.count;
    const uint32_t* __restrict__ idx = q.idx;
    const uint32_t* __restrict__ adj = q.adj;
    unsigned long long st_fb = 0;
    bool has = false, start = false, primary = true, done = false;
    WalkItem it{};
    unsigned long long bi = 0;
    uint32_t len = 0, step = 0, cur = 0, cur2 = 0, sec = 0, sec2 = 0, state = 0, src = 0;
    float ds = 0.f;
    const float* pvec = nullptr;
    float x = 0.f, pa = 0.f, pb = 0.f;
    bool pend = false;
    while (true) {
        // a group without an item claims the next one (items with nr = 0 are skipped)
        if (!has && !done) {
            unsigned my = 0;
            if (j == 0) my = atomicAdd(q.claim, 1u);
            my = __shfl_sync(0xffu << (grp * 8), my, int(grp * 8));
            if (my >= total) {
                done = true;
            } else {
                it = q.items[my];
                if (it.nr) {
                    has = true;
                    start = true;
                    bi = 0;
                    x = 0.f;
                    step = uint32_t(0xffffffffull / it.nr);
                    src = __ldg(q.rows + it.pad);
                    ds = float(__ldg(idx + src + 1) - __ldg(idx + src));
                    const uint32_t slot = it.pad - q.list_base;
                    const uint32_t cta = slot / kBlockCols, col = slot % kBlockCols;
                    pvec = q.pre_cols +
                           (size_t(cta) * 2 + (1u - q.pre_final[cta])) * size_t(q.n) * kBlockCols +
                           size_t(col) * q.n;
                }
            }
        }
        if (!__any_sync(kFullMask, has || !done)) break;
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
        const unsigned z = __ballot_sync(kFullMask, has && primary && (sec == 0u || sec2 == 0u));
        if (has && primary && ((z >> (grp * 8)) & 0xffu)) {
            primary = false;
            if (j == 0) ++st_fb;
        }
        bool item_done = false;
        if (has) {
            const uint32_t b1 = __ldg(idx + cur), d1 = __ldg(idx + cur + 1) - b1;
            const uint32_t b2 = __ldg(idx + cur2), d2 = __ldg(idx + cur2 + 1) - b2;
            if (pend) x = radd(x, rsub(pa, pb));
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
            pa = pvec[cur];
            pb = pvec[cur2];
            pend = true;
            if (++len == it.len) {
                bi += 8;
                start = true;
                item_done = bi >= it.nr;
            }
        }
        if (__any_sync(kFullMask, item_done)) {
            if (item_done && pend) {
                x = radd(x, rsub(pa, pb));
                pend = false;
            }
            double sum = 0;
#pragma unroll
            for (int b = 0; b < 8; ++b) sum += double(__shfl_sync(kFullMask, x, int(grp * 8 + b)));
            if (item_done && j == 0) q.preds[it.pos] += sum / (double(ds) * double(it.nr));
            if (item_done) has = false;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) st_fb += __shfl_xor_sync(kFullMask, st_fb, o);
    if (lane == 0) stat_add(q.stats, kStFallback, st_fb);
}

// Heavy walk items (at least kHeavyNr walks of at most kHeavyLen hops; a few per wave, which would
// otherwise hold a whole wave for one 8-lane group walking them one bouquet after another; on large
// graphs low-degree sources reach 10^6 walks and more).  One 1,024-thread block per item walks 128
// bouquets at once: thread 8r + j walks walk bi + j of bouquet r (bi = the bouquet's first walk)
// and keeps each hop's residual difference in shared memory; then thread j (the item's lane j)
// adds its walks' differences to x in walk order and hop order -- the adds, values and order of
// walk_queue_kernel's lane j -- and the eight x are summed as there.
constexpr int kHeavyThreads = 1024;
constexpr size_t kHeavySmem = sizeof(float) * kHeavyThreads * (kHeavyLen + 1);

__global__ void __launch_bounds__(kHeavyThreads) heavy_walk_kernel(const WalkQueueParams q,
                                                                   uint32_t cap) {
    extern __shared__ float s_heavy[];
    float (*s_d)[kHeavyLen + 1] = reinterpret_cast<float (*)[kHeavyLen + 1]>(s_heavy);
    __shared__ unsigned s_item;
    pdl_launch_dependents();
    pdl_wait();
    const uint32_t tid = threadIdx.x, lane = tid & 31, j = tid & 7, grp = lane >> 3;
    const uint32_t r = tid >> 3;  // bouquet of the chunk
    const uint32_t total = *q.count;
    const uint32_t* __restrict__ idx = q.idx;
    const uint32_t* __restrict__ adj = q.adj;
    unsigned long long st_fb = 0;
    while (true) {
        if (tid == 0) s_item = atomicAdd(q.claim, 1u);
        __syncthreads();
        const unsigned my = s_item;
        __syncthreads();
        if (my >= total) break;
        const WalkItem it = q.items[cap - 1u - my];
        const uint32_t src = __ldg(q.rows + it.pad);
        const float ds = float(__ldg(idx + src + 1) - __ldg(idx + src));
        const uint32_t slot = it.pad - q.list_base;
        const uint32_t cta = slot / kBlockCols, col = slot % kBlockCols;
        const float* pvec = q.pre_cols +
                            (size_t(cta) * 2 + (1u - q.pre_final[cta])) * size_t(q.n) * kBlockCols +
                            size_t(col) * q.n;
        const uint32_t step = uint32_t(0xffffffffull / it.nr);
        const uint32_t L = it.len;
        float x = 0.f;  // threads 0..7
        for (unsigned long long c0 = 0; c0 < it.nr; c0 += kHeavyThreads) {
            const unsigned long long bi = c0 + 8ull * r;
            const bool active = bi < it.nr;
            uint32_t cur = src, cur2 = it.v;
            uint32_t sec = (uint32_t(bi) + j + 1u) * step, sec2 = sec, state = sec;
            bool primary = true;
            // each hop's residual pair is stored one hop later, after the next hop's row offsets
            // are requested, so the residual loads stay off the walk's chain of dependent loads
            float pa = 0.f, pb = 0.f;
            for (uint32_t h = 0; h < L; ++h) {
                const unsigned z =
                    __ballot_sync(kFullMask, active && primary && (sec == 0u || sec2 == 0u));
                if (active && primary && ((z >> (grp * 8)) & 0xffu)) {
                    primary = false;
                    if (j == 0) ++st_fb;
                }
                if (active) {
                    const uint32_t b1 = __ldg(idx + cur), d1 = __ldg(idx + cur + 1) - b1;
                    const uint32_t b2 = __ldg(idx + cur2), d2 = __ldg(idx + cur2 + 1) - b2;
                    if (h > 0) s_d[tid][h - 1] = rsub(pa, pb);
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
                    pa = pvec[cur];
                    pb = pvec[cur2];
                }
            }
            if (active && L > 0) s_d[tid][L - 1] = rsub(pa, pb);
            __syncthreads();
            if (tid < 8) {
                for (uint32_t b = 0; b < kHeavyThreads / 8 && c0 + 8ull * b < it.nr; ++b)
                    for (uint32_t h = 0; h < L; ++h) x = radd(x, s_d[8 * b + tid][h]);
            }
            __syncthreads();
        }
        if (tid < 32) {
            double sum = 0;
#pragma unroll
            for (int b = 0; b < 8; ++b) sum += double(__shfl_sync(kFullMask, x, b));
            if (tid == 0) q.preds[it.pos] += sum / (double(ds) * double(it.nr));
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) st_fb += __shfl_xor_sync(kFullMask, st_fb, o);
    if (lane == 0) stat_add(q.stats, kStFallback, st_fb);
}

// ---- stage 3: symmetrise (src/aesc.h:532-550) -----------------------------------------------------
// score[q] = p[q] + p[q'] with q' the slot that lands on q (sym_src; none in a row without its
// reverse).  p comes from the source kernel for listed rows, and in closed form for the others:
// after the first round of source s, pvec[s] = 0 and pvec[u] = 1 / deg(u) for each neighbour u, so
// p[s -> u] = 1 / ds + (0 - 1 / deg(u)) / ds in the form's arithmetic.  Those rows' work counters
// (one round, one frontier vertex, ds traversals) are added here.
template <class Real, class Acc>
__device__ __forceinline__ Acc closed_row_score(uint32_t ds, uint32_t du) {
    const Real d = from_u64<Real>(ds);
    const Acc pinit = from_f64<Acc>(__ddiv_rn(1.0, double(d)));
    // the mixed form (FP32 residuals, FP64 scores) forms 1 / deg(u) as its push does
    constexpr bool kMixed = std::is_same<Real, float>::value && std::is_same<Acc, double>::value;
    const Real pu = kMixed ? Real(from_fixed(kFixOne, du)) : rdiv(Real(1), from_u64<Real>(du));
    return row_update<Real, Acc>(pinit, Real(0), pu, d);
}

template <class Real, class Acc>
__global__ void __launch_bounds__(256)
finish_kernel(const Acc* __restrict__ preds, const uint32_t* __restrict__ sym_src,
              const uint32_t* __restrict__ row_of, const uint2* __restrict__ adjd,
              const uint32_t* __restrict__ deg, const uint32_t* __restrict__ mark, uint32_t epoch,
              uint64_t m, float* __restrict__ out, unsigned long long* __restrict__ stats) {
    unsigned long long rows = 0, trav = 0;
    pdl_wait();  // pre-symmetric scores of the source kernel
    for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < m;
         q += uint64_t(gridDim.x) * blockDim.x) {
        // first level: the slot's row, its (neighbour, degree) and the slot landing on it
        const uint32_t s = __ldg(row_of + q);
        const uint2 tv = __ldg(adjd + q);
        const uint32_t o = __ldg(sym_src + q);
        const bool first = q == 0 || __ldg(row_of + q - 1) != s;
        // second level, all at once: both rows' marks, both pre-symmetric scores, and the degree of
        // s (the reverse slot's neighbour degree; only graphs without repeated neighbours or
        // self-loops have rows in closed form, every row of the others is listed)
        const uint32_t r = o ? o - 1 : 0;
        const bool ls = __ldg(mark + s) == epoch;
        const bool lt = o && __ldg(mark + tv.x) == epoch;  // slot r lies in row tv.x
        const Acc pq = preds[q];
        const Acc pr = o ? preds[r] : Acc(0);
        const uint32_t ds = o ? __ldg(adjd + r).y : __ldg(deg + s);
        Acc a = ls ? pq : closed_row_score<Real, Acc>(ds, tv.y);
        if (!ls && first) {
            ++rows;
            trav += ds;
        }
        if (o) a = radd(a, lt ? pr : closed_row_score<Real, Acc>(tv.y, ds));
        out[q] = float(a);
    }
    rows = warp_sum_u64(rows);
    trav = warp_sum_u64(trav);
    if ((threadIdx.x & 31) == 0) {
        stat_add(stats, kStPushRounds, rows);
        stat_add(stats, kStPushVertices, rows);
        stat_add(stats, kStPushTraversals, trav);
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

// Buffer growth of a run.  A graph captured in a live batch must keep every buffer the batch's
// CUDA graph points at, so a run on it that would need a larger buffer is refused.
void grow(tgtp_graph* g, DeviceBuffer& b, size_t want) {
    if (g->batch_refs > 0 && (!b.ptr || b.bytes < want))
        fail(TGTP_ERR_INVALID_ARGUMENT,
             "this graph belongs to a live batch and the run needs larger buffers than the batch's; "
             "free the batch first");
    b.reserve(want);
}

// Weight tables of the split tau kernel for the configured omega, cached on the graph and formed
// on the device: row 0 = 1 + lambda_i, row k + 1 = lambda_i^(2(k+1)) / (1 - lambda_i) from the
// parity forms' eigen_t_1 table, zero at the indices the reference leaves out (0 and omega - 1)
// and in the padding of each row to a multiple of 64.  FP64 for the FP64 form, FP32 (rounded from
// the FP64 values) for the mixed form.
uint32_t split_pad(uint32_t omega) { return (omega + 63u) & ~63u; }

__global__ void split_tables_kernel(const double* __restrict__ onep, const double* __restrict__ onem,
                                    const double* __restrict__ etab, uint32_t stride,
                                    uint32_t omega, uint32_t wpad, uint32_t total,
                                    double* __restrict__ t64, float* __restrict__ t32) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= total) return;
    const uint32_t k = x / wpad, i = x % wpad;
    double v = 0.0;
    if (i >= 1 && i + 1 < omega)
        v = k == 0 ? onep[i] : __ddiv_rn(etab[size_t(k - 1) * stride + i], onem[i]);
    t64[x] = v;
    t32[x] = __double2float_rn(v);
}

void prepare_split_tables(tgtp_graph* g, uint32_t omega) {
    if (g->split_omega == omega && g->wtab32.ptr && g->wtab64.ptr) return;
    if (g->batch_refs > 0)
        fail(TGTP_ERR_INVALID_ARGUMENT,
             "this graph belongs to a live batch built for another omega; free the batch first");
    const uint32_t rows = 1 + kTauTableRows, wpad = split_pad(omega);
    g->wtab64.reserve(sizeof(double) * rows * wpad);
    g->wtab32.reserve(sizeof(float) * rows * wpad);
    const uint32_t total = rows * wpad;
    split_tables_kernel<<<(total + 255) / 256, 256, 0, g->stream>>>(
        g->onep.as<double>(), g->onem.as<double>(), g->etab.as<double>(), g->omega, omega, wpad,
        total, g->wtab64.as<double>(), g->wtab32.as<float>());
    TGTP_LAUNCH_CHECK("split_tables_kernel");
    g->split_omega = omega;
}

// Graphs with repeated neighbours or self-loops: every row is listed before the tau kernels run
// (so none is scored in closed form, which assumes distinct neighbours and pvec[s] = 0 after the
// first round), and the tau kernels, finding every row marked, append none.
__global__ void list_all_rows_kernel(RowMarks rm, uint32_t n) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        rm.mark[r] = rm.epoch;
        rm.list[r] = r;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *rm.len = n;
}

// Row marks of this run: they sit behind the work words in the counter buffer, so the run's one
// zeroing clears them too (a captured run replays correctly), and a marked row holds 1.
RowMarks begin_row_marks(tgtp_graph* g) {
    grow(g, g->row_list, sizeof(uint32_t) * (g->n + 1));
    RowMarks rm;
    rm.mark = run_work(g) + 4;
    rm.list = g->row_list.as<uint32_t>();
    rm.len = run_work(g) + 2;
    rm.epoch = 1;
    return rm;
}

// Kernel launch on the handle's stream; with pdl the launch may begin while the previous kernel
// finishes (the kernel waits for it with pdl_wait).  TGTP_PDL=0 turns the overlap off.
bool pdl_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("TGTP_PDL");
        return !(e && std::string(e) == "0");
    }();
    return on;
}

template <class... KArgs, class... Args>
void launch(void (*kern)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
            bool pdl, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = (pdl && pdl_enabled()) ? 1 : 0;
    TGTP_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
}

// Resident blocks per SM of a kernel at a block size and dynamic shared memory, cached; the kernel's
// dynamic shared-memory limit is raised to the largest size asked for so far.
int blocks_per_sm(const void* kern, int threads, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, size_t, int>, int> cache;
    static std::map<const void*, size_t> limit;
    int dev = 0;
    TGTP_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_tuple(kern, threads, smem, dev);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    if (smem > limit[kern]) {
        TGTP_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        limit[kern] = smem;
    }
    int per_sm = 0;
    TGTP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
    cache[key] = per_sm;
    return per_sm;
}

// Symmetrisation of one run (stage 3) on the graph's stream.
template <class Real, class Acc>
void launch_finish(tgtp_graph* g, float* out) {
    const RowMarks rm{run_work(g) + 4, g->row_list.as<uint32_t>(), run_work(g) + 2, 1u};
    ScopedKernel k(g->prof, g->stream, "finish");
    launch(finish_kernel<Real, Acc>, grid_cap(g->m, 256, g->num_sms, 8), 256, 0, g->stream, true,
           g->preds.as<Acc>(), g->sym_src.as<uint32_t>(), g->row_of.as<uint32_t>(),
           g->adjd.as<uint2>(), g->deg.as<uint32_t>(), rm.mark, rm.epoch, g->m, out,
           g->stats.as<unsigned long long>());
    TGTP_LAUNCH_CHECK("finish_kernel");
}

}  // namespace

// ---- batched runs: one persistent source kernel over the rows of many graphs --------------------
// While a batch is captured (batch.cu), each run_form of a graph whose per-source stage runs as
// per-warp pushes stops after its tau kernels and leaves that stage and the symmetrisation to the
// batch: the batch joins every graph's branch, launches one persistent source kernel per
// (arithmetic form, residual-vector tier) over the listed rows of all its graphs, then launches
// each graph's finish kernel on the graph's own stream again.  The graphs of a group share one
// per-warp scratch laid out for the group's largest graph.
struct BatchEntry {
    tgtp_graph* g;
    float* out;
    int key;    // form_key of the run
    bool smem;  // residual vectors in shared memory
    std::vector<unsigned char> params;  // the run's SourceParams<Real, Acc>
};
struct BatchGroup {
    int key;
    bool smem;
    std::vector<size_t> members;  // indices into BatchPlan::entries
    DeviceBuffer scratch, wclean, claims;
};
struct BatchPlan {
    std::vector<BatchEntry> entries;
    std::vector<std::unique_ptr<BatchGroup>> groups;
};
namespace {
thread_local BatchPlan* t_collect = nullptr;

template <class Real, class Acc>
bool defer_to_batch(tgtp_graph* g, const tgtp_config& cfg, float* out, bool smem,
                    const SourceParams<Real, Acc>& p) {
    if (!t_collect) return false;
    BatchEntry e;
    e.g = g;
    e.out = out;
    e.key = form_key(cfg);
    e.smem = smem;
    e.params.resize(sizeof(p));
    std::memcpy(e.params.data(), &p, sizeof(p));
    t_collect->entries.push_back(std::move(e));
    return true;
}

// One tgtp() run.  Real = residual / eigen projection type, Acc = score accumulator,
// Whether a warp's FP32 residual vector and flags (the mixed form's) exceed the 112 KB of the
// shared-memory tier, so that the per-warp push works on vectors in HBM.
bool mixed_beyond_smem(uint64_t n) {
    return ((n * 4 + 15) & ~uint64_t(15)) + ((n + 15) & ~uint64_t(15)) + kAccBytes > uint64_t(112) * 1024;
}
void poll_push_hint(tgtp_graph* g);
void post_push_hint(tgtp_graph* g, int key, double eps);

// JACOBI = mixed form (lane-parallel tau over Vec storage, frontier-parallel push).
template <class Real, class Acc, bool JACOBI, class Vec>
void run_form(tgtp_graph* g, const tgtp_config& cfg, float* out) {
    cudaStream_t s = g->stream;
    const uint64_t n = g->n, m = g->m;
    const uint32_t omega = uint32_t(cfg.omega);
    // host-side constants with the host libm (as the reference evaluates them)
    TauConst c;
    const double l1 = g->values[1], l2 = g->values[omega - 1];
    c.one_m_l1sq = 1.0 - (l1 * l1);
    c.b1 = std::log(double(1.0) / std::fabs(l1));
    c.one_m_l2sq = 1.0 - (l2 * l2);
    c.b2 = std::log(double(1.0) / std::fabs(l2));
    const double logmd = std::log(double(m) / cfg.delta);

    grow(g, g->taus, sizeof(int) * (m + 1));
    grow(g, g->preds, sizeof(Acc) * (m + 1));
    // one zeroing for the striped counters, the work words and the row marks behind them
    const size_t stat_bytes = sizeof(unsigned long long) * kStCount * kStStripes;
    // mixed form, residual vectors too large for shared memory: multi-source push in waves of
    // block_ctas x kBlockCols listed sources (each wave has its own claim counter)
    // The block push gives the same bits as the per-warp push (fixed-point residual sums), so the
    // choice is only about speed: the handle's tuned layout, else TGTP_MIXED_BLOCK, else what the
    // last completed mixed run on this graph at this epsilon measured (push_hint), else the block
    // push for
    // vectors beyond shared memory at eps <= 0.01 (deep pushes: the block push was the faster one
    // on every such graph measured) and the per-warp push otherwise.
    const int key = form_key(cfg);
    if (JACOBI) poll_push_hint(g);
    bool block_mode = false;
    if (g->src_layout[key]) block_mode = JACOBI && (g->src_layout[key] & kLayoutBlock) != 0;
    else if (const char* e = std::getenv("TGTP_MIXED_BLOCK")) block_mode = JACOBI && std::atoi(e) != 0;
    else if (g->push_hint[key] && g->push_hint_eps[key] == cfg.epsilon)
        block_mode = JACOBI && g->push_hint[key] == 2;
    else block_mode = JACOBI && mixed_beyond_smem(n) && cfg.epsilon <= 0.01;
    g->last_key = key;
    g->last_eps = cfg.epsilon;
    // CTAs of the block push: one per SM, within a budget for their residual blocks of 24 GB or
    // half the device memory free now (beside what the blocks already hold), whichever is larger
    // (TGTP_BLOCK_CTAS lowers the count, e.g. to exercise many waves on small graphs)
    uint32_t block_ctas = uint32_t(g->num_sms);
    if (block_mode) {
        const size_t per_cta = 2 * size_t(n) * kBlockCols * sizeof(float);
        size_t free_b = 0, total_b = 0;
        TGTP_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const size_t budget = std::max(size_t(24) << 30, (free_b + g->block_cols.bytes) / 2);
        block_ctas = uint32_t(std::max<size_t>(1, std::min<size_t>(block_ctas, budget / per_cta)));
        if (const char* e = std::getenv("TGTP_BLOCK_CTAS"))
            block_ctas = std::max(1u, std::min(block_ctas, uint32_t(std::atoi(e))));
    }
    const uint32_t waves =
        block_mode ? uint32_t((n + uint64_t(block_ctas) * kBlockCols - 1) / (uint64_t(block_ctas) * kBlockCols))
                   : 0u;
    const size_t zero_bytes = stat_bytes + sizeof(unsigned) * (4 + n + 1 + waves);
    grow(g, g->stats, zero_bytes);
    auto* stats = g->stats.as<unsigned long long>();
    auto* work = run_work(g);
    TGTP_CUDA(cudaMemsetAsync(stats, 0, zero_bytes, s));

    const RowMarks rm = begin_row_marks(g);
    const bool multi = !JACOBI && g->has_multi_edges;
    if (multi) {
        // the reference leaves tau = 0 in the slots no forward edge writes (the later repeats of
        // a neighbour u < v in row v, src/aesc.h:179-209), and every row goes to the source kernel
        TGTP_CUDA(cudaMemsetAsync(g->taus.ptr, 0, sizeof(int) * m, s));
        list_all_rows_kernel<<<grid_cap(n, 256, g->num_sms, 8), 256, 0, s>>>(rm, uint32_t(n));
        TGTP_LAUNCH_CHECK("list_all_rows_kernel");
    }
    if constexpr (JACOBI || std::is_same<Real, double>::value) {
        // FP64 and mixed forms: eight lanes per edge over F64 / F32 / BF16 rows
        prepare_split_tables(g, omega);
        using Part = typename Split<Vec>::Part;
        const Vec* vec = std::is_same<Vec, double>::value ? (const Vec*)g->vec_f64.ptr
                         : std::is_same<Vec, float>::value ? (const Vec*)g->vec_f32.ptr
                                                           : (const Vec*)g->vec_bf16.ptr;
        const Part* wtab = std::is_same<Part, double>::value ? (const Part*)g->wtab64.ptr
                                                             : (const Part*)g->wtab32.ptr;
        const uint32_t wpad = split_pad(omega);
        const size_t ssmem = 2 * sizeof(Part) * wpad;
        BoundArgs<Vec> ba;
        ba.deg = g->deg.as<uint32_t>();
        ba.vec = vec;
        ba.stride = g->omega;
        ba.omega = omega;
        ba.wtab = wtab;
        ba.wpad = wpad;
        ba.etabd = g->etab.as<double>();
        ba.onem = g->onem.as<double>();
        ba.eps_half = cfg.epsilon / 2.0;
        ba.mdbl = double(m);
        ba.c = c;
        ba.taus = g->taus.as<int>();
        ba.rm = rm;
        {
            const int per_sm =
                blocks_per_sm(reinterpret_cast<const void*>(tau_sums_kernel<Vec>), 256, ssmem);
            if (per_sm < 1) fail(TGTP_ERR_UNSUPPORTED, "omega too large for the tau kernel");
            grow(g, g->tau_sums, sizeof(double2) * (g->num_forward + 1));
            const uint64_t need = (g->num_forward + 63) / 64;  // 64 edges per block and step
            const unsigned blocks = unsigned(std::max<uint64_t>(
                1, std::min<uint64_t>(need, uint64_t(g->num_sms) * per_sm)));
            // TGTP_TAU_BULK=1: the bulk-copy pipeline instead of the gather (rows whose bytes are a
            // multiple of 16, with a row stride that keeps them aligned).  On the 4,039-vertex graph
            // it measured 0.056 ms per FP64 step against the gather's 0.046: the rows are
            // L2-resident, so the gather's 32 warps per SM hide the latency better than six
            // pipelined warps, and the bulk copies fetch each edge's u row again.
            const char* bulk_env = std::getenv("TGTP_TAU_BULK");
            const bool bulk = (bulk_env && std::atoi(bulk_env) == 1) &&
                              (size_t(omega) * sizeof(Vec)) % 16 == 0 &&
                              (size_t(g->omega) * sizeof(Vec)) % 16 == 0;
            constexpr int WPB = BulkShape<Vec>::WPB;
            const size_t bsmem = size_t(WPB) * (size_t(kBulkStages) * 8 * omega * sizeof(Vec) +
                                                kBulkStages * 8) + ssmem;
            const int bper_sm = bulk ? blocks_per_sm(
                reinterpret_cast<const void*>(tau_sums_bulk_kernel<Vec>), 32 * WPB, bsmem) : 0;
            if (bulk && bper_sm >= 1) {
                const uint64_t bneed = (g->num_forward + 4 * WPB - 1) / (4 * WPB);
                const unsigned bblocks = unsigned(std::max<uint64_t>(
                    1, std::min<uint64_t>(bneed, uint64_t(g->num_sms) * bper_sm)));
                ScopedKernel k(g->prof, s, "tau_sums");
                launch(tau_sums_bulk_kernel<Vec>, bblocks, unsigned(32 * WPB), bsmem, s, false,
                       g->fedge.as<uint4>(), g->num_forward, vec, g->omega, omega, wtab, wpad,
                       g->tau_sums.as<double2>(), work);
                TGTP_LAUNCH_CHECK("tau_sums_bulk_kernel");
            } else {
                ScopedKernel k(g->prof, s, "tau_sums");
                launch(tau_sums_kernel<Vec>, blocks, 256u, ssmem, s, false,
                    g->fedge.as<uint4>(), g->num_forward, vec, g->omega, omega, wtab, wpad,
                    g->tau_sums.as<double2>());
                TGTP_LAUNCH_CHECK("tau_sums_kernel");
            }
            ScopedKernel k(g->prof, s, "tau_bound");
            launch(tau_bound_kernel<Vec>, grid_cap(g->num_forward, 256, g->num_sms, 8), 256u,
                   size_t(0), s, true, g->fedge.as<uint4>(), g->num_forward,
                   static_cast<const double2*>(g->tau_sums.as<double2>()), ba, stats);
            TGTP_LAUNCH_CHECK("tau_bound_kernel");
        }
    } else {
        // FP32 form: the reference's arithmetic and summation order
        const Real* vec = (const Real*)g->vec_f32.ptr;
        const Real* etab = (const Real*)g->etab_f.ptr;
        const Real eps_half = Real(cfg.epsilon / 2.0);
        // per block: two double2 constants per index; per warp: two buffers of (x_u, x_v) chunks
        // of 32 edges x one 128-byte row piece, rows padded by one element
        const size_t tau_smem = 2 * sizeof(double2) * omega +
                                size_t(kTauThreads / 32) * 4 * 32 * (128 / sizeof(Real) + 1) * sizeof(Real);
        if (tau_smem > size_t(227) * 1024)
            fail(TGTP_ERR_UNSUPPORTED, "omega too large for the tau kernel tile");
        const int tau_per_sm =
            blocks_per_sm(reinterpret_cast<const void*>(tau_kernel<Real>), kTauThreads, tau_smem);
        if (tau_per_sm < 1) fail(TGTP_ERR_UNSUPPORTED, "omega too large for the tau kernel tile");
        const uint64_t groups = (g->num_forward + 31) / 32;
        const uint64_t tau_blocks = std::max<uint64_t>(1, std::min<uint64_t>(
            (groups + kTauThreads / 32 - 1) / (kTauThreads / 32), uint64_t(g->num_sms) * tau_per_sm));
        ScopedKernel k(g->prof, s, "tau");
        tau_kernel<Real><<<unsigned(tau_blocks), kTauThreads, tau_smem, s>>>(
            g->idx.as<uint32_t>(), g->adj.as<uint32_t>(), g->row_of.as<uint32_t>(),
            g->rev.as<uint32_t>(), g->forward.as<uint32_t>(), g->num_forward, vec, g->omega, omega,
            g->onep.as<double>(), g->onem.as<double>(), etab, g->etab.as<double>(), eps_half, m, c,
            g->taus.as<int>(), rm, stats);
        TGTP_LAUNCH_CHECK("tau_kernel");
    }

    // source kernel.  Shared-memory tier: each warp's residual vector and flags in shared memory.
    // Global tier (large n): vectors in HBM.  The layout (tier, warps per block) comes from the
    // handle's tuned choice for this form, else from the default rule (shared memory with one-warp
    // blocks while a warp's copy fits in 112 KB, else HBM with four warps per block);
    // TGTP_PVEC_TIER=smem|global overrides the tier of the default rule.
    const size_t pv_bytes = (size_t(n) * sizeof(Real) + 15) & ~size_t(15);
    const size_t vis_bytes = (size_t(n) + 15) & ~size_t(15);
    const size_t fx_bytes = JACOBI ? sizeof(unsigned long long) * size_t(n) : 0;
    // the mixed form's fixed-point accumulators join the shared-memory copy only while the three
    // arrays fit in 112 KB; beyond that they move to HBM and the residual vector stays in shared
    // memory up to the same size as in the other forms
    const bool fx_in_smem = JACOBI && pv_bytes + vis_bytes + fx_bytes + kAccBytes <= size_t(112) * 1024;
    const size_t per_warp = pv_bytes + vis_bytes + (fx_in_smem ? fx_bytes : 0) + kAccBytes;
    bool use_smem;
    int wpb;
    if (g->src_layout[key]) {
        use_smem = (g->src_layout[key] & kLayoutSmem) != 0;
        wpb = std::max(1, g->src_layout[key] & 0xff);
    } else {
        use_smem = per_warp <= size_t(112) * 1024;
        if (const char* t = std::getenv("TGTP_PVEC_TIER")) {
            if (std::string(t) == "global") use_smem = false;
            else if (std::string(t) == "smem" && per_warp <= size_t(227) * 1024) use_smem = true;
        }
        wpb = use_smem ? 1 : 4;
    }
    if (use_smem && per_warp * wpb > size_t(227) * 1024)
        fail(TGTP_ERR_UNSUPPORTED, "source layout does not fit in shared memory");
    const int threads = wpb * 32;
    const size_t smem = use_smem ? per_warp * wpb : size_t(wpb) * kAccBytes;
    using Pack1 = SourcePack<Real, Acc, 1>;
    auto kern = use_smem ? source_kernel<Real, Acc, true, JACOBI, Pack1>
                         : source_kernel<Real, Acc, false, JACOBI, Pack1>;
    const int per_sm = blocks_per_sm(reinterpret_cast<const void*>(kern), threads, smem);
    if (per_sm < 1) fail(TGTP_ERR_UNSUPPORTED, "source kernel does not fit on an SM");
    uint64_t blocks = uint64_t(g->num_sms) * per_sm;
    blocks = std::min<uint64_t>(blocks, (n + wpb - 1) / wpb);
    const uint64_t warps = blocks * wpb;
    const size_t maxd = std::max<uint32_t>(g->max_degree, 1);
    auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t q_bytes = align(warps * 2 * size_t(n) * 4);
    const size_t it_bytes = align(warps * maxd * sizeof(WalkItem));
    const size_t pvg_bytes = use_smem ? 0 : align(warps * size_t(n) * sizeof(Real));
    const size_t visg_bytes = use_smem ? 0 : align(warps * vis_bytes);
    const size_t fxg_bytes = (JACOBI && !(use_smem && fx_in_smem)) ? align(warps * fx_bytes) : 0;
    grow(g, g->scratch, q_bytes + it_bytes + pvg_bytes + visg_bytes + fxg_bytes + 256);
    unsigned char* base = g->scratch.as<unsigned char>();
    SourceParams<Real, Acc> p;
    p.idx = g->idx.as<uint32_t>();
    p.adj = g->adj.as<uint32_t>();
    p.deg = g->deg.as<uint32_t>();
    p.n = uint32_t(n);
    p.taus = g->taus.as<int>();
    p.preds = g->preds.as<Acc>();
    p.work = work;
    p.rows = rm.list;
    p.qbuf = reinterpret_cast<uint32_t*>(base);
    base += q_bytes;
    p.items = reinterpret_cast<WalkItem*>(base);
    base += it_bytes;
    p.pvec_g = use_smem ? nullptr : reinterpret_cast<Real*>(base);
    base += pvg_bytes;
    p.vis_g = use_smem ? nullptr : base;
    base += visg_bytes;
    p.fx_g = fxg_bytes ? reinterpret_cast<unsigned long long*>(base) : nullptr;
    // the per-warp "vectors are zero" marks hold only for the same carving of the same scratch
    {
        const uint64_t sig[5] = {uint64_t(key) | (uint64_t(use_smem) << 8) | (uint64_t(wpb) << 16),
                                 blocks, uint64_t(n),
                                 uint64_t(reinterpret_cast<uintptr_t>(g->scratch.ptr)),
                                 uint64_t(g->scratch.bytes)};
        grow(g, g->wclean, warps + 16);
        if (std::memcmp(sig, g->wclean_sig, sizeof(sig)) != 0) {
            TGTP_CUDA(cudaMemsetAsync(g->wclean.ptr, 0, warps + 16, s));
            std::memcpy(g->wclean_sig, sig, sizeof(sig));
        }
        p.wclean = g->wclean.as<unsigned char>();
    }
    p.vis_stride = vis_bytes;
    p.smem_per_warp = per_warp;
    p.max_degree = uint32_t(maxd);
    p.eps = cfg.epsilon;
    p.logmd = logmd;
    p.gamma = cfg.gamma;
    p.stats = stats;
    p.adjd = g->adjd.as<uint2>();
    p.budget_ns = deadline_from_env();
    p.trace_nr = p.trace_ell = nullptr;
    p.walk_queue = nullptr;
    p.walk_count = nullptr;
    p.walk_cap = 0;
    if (g->trace_on) {
        grow(g, g->trace, sizeof(uint32_t) * (m + n));
        TGTP_CUDA(cudaMemsetAsync(g->trace.ptr, 0, sizeof(uint32_t) * (m + n), s));
        p.trace_nr = g->trace.as<uint32_t>();
        p.trace_ell = p.trace_nr + m;
        g->trace_valid = true;
    }
    p.pre = nullptr;
    p.pre_cols = nullptr;
    p.pre_final = nullptr;
    p.multi = multi;
    p.scratch_n = uint32_t(n);
    {
        // The windowed push pays off when rows are short: several frontier vertices share a
        // 32-entry step.  When rows average 32 entries or more, each vertex fills its steps anyway
        // and adjacent frontier vertices cut windows often, so one vertex at a time is used
        // (4,039-vertex Chung-Lu graph, 44 entries per row: 0.73 against 0.86 ms at eps = 0.01;
        // sparse Chung-Lu, 9.3 per row: 4.1 against 1.4 s at eps = 0.005).  The tuned layout,
        // then TGTP_GS_WINDOW=0/1, override the rule.
        const uint16_t lay = g->src_layout[key];
        const char* e = std::getenv("TGTP_GS_WINDOW");
        if (lay & kLayoutWindow) p.gs_window = true;
        else if (lay & kLayoutNoWindow) p.gs_window = false;
        else if (e) p.gs_window = std::string(e) != "0";
        else p.gs_window = m < 32 * n;
    }
    Pack1 pk;
    pk.count = 1;
    if (!block_mode) {
        p.claim = work;
        p.list_base = 0;
        p.list_cap = uint32_t(n);
        if (defer_to_batch<Real, Acc>(g, cfg, out, use_smem, p)) return;
        pk.g[0] = p;
        ScopedKernel k(g->prof, s, "source");
        launch(kern, unsigned(blocks), unsigned(threads), smem, s, true, pk);
        TGTP_LAUNCH_CHECK("source_kernel");
    } else if constexpr (JACOBI) {  // the block push exists for the mixed form only
        grow(g, g->block_cols, 2 * size_t(n) * kBlockCols * sizeof(float) * block_ctas);
        grow(g, g->block_pre, sizeof(PrePush) * (n + 1));
        grow(g, g->block_final, sizeof(uint32_t) * (block_ctas + 1));
        PushBlockParams bp;
        bp.idx = p.idx;
        bp.adj = p.adj;
        bp.deg = p.deg;
        bp.adjd = p.adjd;
        bp.n = uint32_t(n);
        bp.taus = p.taus;
        bp.preds = p.preds;
        bp.work = work;
        bp.rows = rm.list;
        bp.eps = cfg.epsilon;
        bp.logmd = logmd;
        bp.cols = g->block_cols.as<float>();
        bp.final_buf = g->block_final.as<uint32_t>();
        bp.pre = g->block_pre.as<PrePush>();
        bp.stats = stats;
        bp.budget_ns = p.budget_ns;
        // three row masks in shared memory while they fit beside the kernel's static 1.5 KB, else
        // the current round's mask alone (n up to about 1.6 million), else none; the others in
        // global memory; four row lists of n entries per CTA.  TGTP_BLOCK_MASKS=global|cur picks
        // the placement of larger graphs on small ones.
        const size_t mask_bytes = sizeof(uint32_t) * ((size_t(n) + 31) / 32);
        const size_t bits_bytes = 3 * mask_bytes;
        bp.bits = bits_bytes <= size_t(200) * 1024;
        bp.cur_smem = !bp.bits && mask_bytes <= size_t(200) * 1024;
        if (const char* e = std::getenv("TGTP_BLOCK_MASKS")) {
            if (std::string(e) == "global") bp.bits = bp.cur_smem = false;
            else if (std::string(e) == "cur") {
                bp.bits = false;
                bp.cur_smem = true;
            }
        }
        const size_t bsm = bp.bits ? bits_bytes : (bp.cur_smem ? mask_bytes : 0);
        if (!bp.bits) grow(g, g->block_bits, bits_bytes * block_ctas + 16);
        bp.gbits = bp.bits ? nullptr : g->block_bits.as<uint32_t>();
        grow(g, g->block_lists, sizeof(uint32_t) * 4 * size_t(n) * block_ctas + 16);
        bp.lists = g->block_lists.as<uint32_t>();
        bp.m = m;
        // a round is compacted when its live rows' degree sum is below m / list_div (the tuned
        // layout's threshold, else TGTP_BLOCK_LIST_DIV, else 4); TGTP_BLOCK_ROUNDS=compact|full
        // fixes the choice (the values do not depend on it)
        bp.list_div = layout_list_div(g->src_layout[key]);
        if (const char* e = std::getenv("TGTP_BLOCK_LIST_DIV"))
            if (!g->src_layout[key]) bp.list_div = uint32_t(std::atoi(e));
        bp.rounds_mode = bp.list_div == 0 ? 2 : 0;
        if (const char* e = std::getenv("TGTP_BLOCK_ROUNDS")) {
            if (std::string(e) == "compact") bp.rounds_mode = 1;
            else if (std::string(e) == "full") bp.rounds_mode = 2;
        }
        if (bsm) (void)blocks_per_sm(reinterpret_cast<const void*>(push_block_kernel), 1024, bsm);
        p.pre = bp.pre;
        p.pre_cols = bp.cols;
        p.pre_final = bp.final_buf;
        // the listed rows ordered by their largest tau (unlisted rows sort last, key 0)
        grow(g, g->block_keys, sizeof(uint32_t) * 4 * (n + 1));
        uint32_t* key = g->block_keys.as<uint32_t>();
        uint32_t* ids = key + (n + 1);
        uint32_t* skey = ids + (n + 1);
        uint32_t* sorted = skey + (n + 1);
        size_t tbytes = 0;
        TGTP_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tbytes, key, skey, ids, sorted,
                                                            int(n), 0, 32, s));
        grow(g, g->block_tmp, tbytes + 16);
        {
            ScopedKernel k(g->prof, s, "row_key");
            launch(row_key_kernel, grid_cap(uint64_t(n) * 32, 256, g->num_sms, 8), 256u, size_t(0), s,
                   true, g->idx.as<uint32_t>(), g->taus.as<int>(), rm.mark, uint32_t(n), key, ids);
            TGTP_LAUNCH_CHECK("row_key_kernel");
        }
        TGTP_CUDA(cub::DeviceRadixSort::SortPairsDescending(g->block_tmp.ptr, tbytes, key, skey, ids,
                                                            sorted, int(n), 0, 32, s));
        bp.rows = sorted;
        p.rows = sorted;
        unsigned* claims = work + 4 + n + 1;
        // the walks of each wave's sources: a queue of (slot, its source's list entry) items that
        // walk_queue_kernel works through (a wave's sources hold at most m slots), and per wave a
        // queue length and a claim counter
        grow(g, g->walk_queue, sizeof(WalkItem) * (m + 1));
        grow(g, g->walk_ctl, sizeof(unsigned) * 4 * (waves + 1));
        unsigned* ctl = g->walk_ctl.as<unsigned>();
        TGTP_CUDA(cudaMemsetAsync(ctl, 0, sizeof(unsigned) * 4 * (waves + 1), s));
        p.walk_queue = g->walk_queue.as<WalkItem>();
        p.walk_cap = uint32_t(m + 1);
        WalkQueueParams wq;
        wq.idx = p.idx;
        wq.adj = p.adj;
        wq.rows = sorted;
        wq.pre_cols = bp.cols;
        wq.pre_final = bp.final_buf;
        wq.n = uint32_t(n);
        wq.preds = reinterpret_cast<double*>(p.preds);
        wq.items = p.walk_queue;
        wq.stats = stats;
        const int walk_per_sm =
            blocks_per_sm(reinterpret_cast<const void*>(walk_queue_kernel), kWalkThreads, 0);
        const unsigned walk_blocks = unsigned(g->num_sms) * unsigned(std::max(walk_per_sm, 1));
        const int heavy_per_sm = blocks_per_sm(reinterpret_cast<const void*>(heavy_walk_kernel),
                                               kHeavyThreads, kHeavySmem);
        const unsigned heavy_blocks = unsigned(g->num_sms) * unsigned(std::max(heavy_per_sm, 1));
        for (uint32_t w = 0; w < waves; ++w) {
            bp.base = w * block_ctas * kBlockCols;
            {
                ScopedKernel k(g->prof, s, "push_block");
                launch(push_block_kernel, block_ctas, 1024u, bsm, s, true, bp);
                TGTP_LAUNCH_CHECK("push_block_kernel");
            }
            p.claim = claims + w;
            p.list_base = bp.base;
            p.list_cap = block_ctas * kBlockCols;
            p.walk_count = ctl + 4 * w;
            pk.g[0] = p;
            {
                ScopedKernel k(g->prof, s, "source");
                launch(kern, unsigned(blocks), unsigned(threads), smem, s, true, pk);
                TGTP_LAUNCH_CHECK("source_kernel");
            }
            wq.list_base = bp.base;
            wq.count = ctl + 4 * w;
            wq.claim = ctl + 4 * w + 1;
            {
                ScopedKernel k(g->prof, s, "walk_queue");
                launch(walk_queue_kernel, walk_blocks, unsigned(kWalkThreads), size_t(0), s, true, wq);
                TGTP_LAUNCH_CHECK("walk_queue_kernel");
            }
            WalkQueueParams wh = wq;
            wh.count = ctl + 4 * w + 2;
            wh.claim = ctl + 4 * w + 3;
            ScopedKernel k(g->prof, s, "heavy_walk");
            launch(heavy_walk_kernel, heavy_blocks, unsigned(kHeavyThreads), kHeavySmem, s, true, wh,
                   uint32_t(m + 1));
            TGTP_LAUNCH_CHECK("heavy_walk_kernel");
        }
    }
    launch_finish<Real, Acc>(g, out);
}

// The persistent source kernel of one batch group: per-warp scratch for the group's largest
// graph, packs of up to kBatchPack graphs, each pack one launch on `s` with its own claim counter.
template <class Real, class Acc, bool SMEM, bool JACOBI>
void launch_group(BatchPlan& plan, BatchGroup& grp, cudaStream_t s, int num_sms) {
    using Pack = SourcePack<Real, Acc, kBatchPack>;
    static_assert(sizeof(Pack) < 32000, "pack must fit in the kernel parameter space");
    uint32_t sn = 1, maxd = 1;
    uint64_t rows = 0;
    for (size_t i : grp.members) {
        const tgtp_graph* g = plan.entries[i].g;
        sn = std::max<uint32_t>(sn, uint32_t(g->n));
        maxd = std::max<uint32_t>(maxd, g->max_degree);
        rows += g->n;
    }
    const size_t pv_bytes = (size_t(sn) * sizeof(Real) + 15) & ~size_t(15);
    const size_t vis_bytes = (size_t(sn) + 15) & ~size_t(15);
    const size_t fx_bytes = JACOBI ? sizeof(unsigned long long) * size_t(sn) : 0;
    const bool fx_in_smem = SMEM && JACOBI &&
                            pv_bytes + vis_bytes + fx_bytes + kAccBytes <= size_t(112) * 1024;
    const size_t per_warp = pv_bytes + vis_bytes + (fx_in_smem ? fx_bytes : 0) + kAccBytes;
    const int wpb = SMEM ? 1 : 4;
    const int threads = 32 * wpb;
    const size_t smem = SMEM ? per_warp * wpb : size_t(wpb) * kAccBytes;
    auto kern = source_kernel<Real, Acc, SMEM, JACOBI, Pack>;
    const int per_sm = blocks_per_sm(reinterpret_cast<const void*>(kern), threads, smem);
    if (per_sm < 1) fail(TGTP_ERR_UNSUPPORTED, "batch source kernel does not fit on an SM");
    uint64_t blocks = std::min<uint64_t>(uint64_t(num_sms) * per_sm, (rows + wpb - 1) / wpb);
    blocks = std::max<uint64_t>(blocks, 1);
    const uint64_t warps = blocks * wpb;
    auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t q_bytes = align(warps * 2 * size_t(sn) * 4);
    const size_t it_bytes = align(warps * maxd * sizeof(WalkItem));
    const size_t pvg_bytes = SMEM ? 0 : align(warps * size_t(sn) * sizeof(Real));
    const size_t visg_bytes = SMEM ? 0 : align(warps * vis_bytes);
    const size_t fxg_bytes = (JACOBI && !fx_in_smem) ? align(warps * fx_bytes) : 0;
    grp.scratch.reserve(q_bytes + it_bytes + pvg_bytes + visg_bytes + fxg_bytes + 256);
    grp.wclean.reserve(warps + 16);
    const size_t packs = (grp.members.size() + kBatchPack - 1) / kBatchPack;
    grp.claims.reserve(sizeof(unsigned) * (packs + 1));
    unsigned char* base = grp.scratch.as<unsigned char>();
    // each replay starts from "vectors not known to be zero" and fresh claim counters
    TGTP_CUDA(cudaMemsetAsync(grp.wclean.ptr, 0, warps + 16, s));
    TGTP_CUDA(cudaMemsetAsync(grp.claims.ptr, 0, sizeof(unsigned) * (packs + 1), s));
    for (size_t pk0 = 0; pk0 < grp.members.size(); pk0 += kBatchPack) {
        Pack pk;
        pk.count = uint32_t(std::min<size_t>(kBatchPack, grp.members.size() - pk0));
        for (uint32_t j = 0; j < pk.count; ++j) {
            SourceParams<Real, Acc> p;
            std::memcpy(&p, plan.entries[grp.members[pk0 + j]].params.data(), sizeof(p));
            unsigned char* b = base;
            p.qbuf = reinterpret_cast<uint32_t*>(b);
            b += q_bytes;
            p.items = reinterpret_cast<WalkItem*>(b);
            b += it_bytes;
            p.pvec_g = SMEM ? nullptr : reinterpret_cast<Real*>(b);
            b += pvg_bytes;
            p.vis_g = SMEM ? nullptr : b;
            b += visg_bytes;
            p.fx_g = fxg_bytes ? reinterpret_cast<unsigned long long*>(b) : nullptr;
            p.wclean = grp.wclean.as<unsigned char>();
            p.vis_stride = vis_bytes;
            p.smem_per_warp = per_warp;
            p.max_degree = maxd;
            p.scratch_n = sn;
            p.claim = grp.claims.as<unsigned>() + pk0 / kBatchPack;
            pk.g[j] = p;
        }
        launch(kern, unsigned(blocks), unsigned(threads), smem, s, false, pk);
        TGTP_LAUNCH_CHECK("source_kernel (batch)");
    }
}

}  // namespace

BatchPlan* batch_plan_new() { return new BatchPlan(); }
void batch_plan_free(BatchPlan* plan) { delete plan; }
void batch_plan_collect(BatchPlan* plan) {
    if (plan) plan->entries.clear();
    t_collect = plan;
}

size_t batch_plan_deferred(const BatchPlan* plan) { return plan->entries.size(); }

void batch_plan_launch(BatchPlan* plan, cudaStream_t s, int num_sms) {
    plan->groups.clear();
    for (size_t i = 0; i < plan->entries.size(); ++i) {
        const BatchEntry& e = plan->entries[i];
        BatchGroup* grp = nullptr;
        for (auto& g : plan->groups)
            if (g->key == e.key && g->smem == e.smem) grp = g.get();
        if (!grp) {
            plan->groups.push_back(std::make_unique<BatchGroup>());
            grp = plan->groups.back().get();
            grp->key = e.key;
            grp->smem = e.smem;
        }
        grp->members.push_back(i);
    }
    for (auto& grp : plan->groups) {
        switch (grp->key) {
            case 0:
                if (grp->smem) launch_group<float, float, true, false>(*plan, *grp, s, num_sms);
                else launch_group<float, float, false, false>(*plan, *grp, s, num_sms);
                break;
            case 1:
                if (grp->smem) launch_group<double, double, true, false>(*plan, *grp, s, num_sms);
                else launch_group<double, double, false, false>(*plan, *grp, s, num_sms);
                break;
            default:
                if (grp->smem) launch_group<float, double, true, true>(*plan, *grp, s, num_sms);
                else launch_group<float, double, false, true>(*plan, *grp, s, num_sms);
                break;
        }
    }
}

void batch_plan_finish(BatchPlan* plan) {
    for (const BatchEntry& e : plan->entries) {
        if (e.key == 0) launch_finish<float, float>(e.g, e.out);
        else if (e.key == 1) launch_finish<double, double>(e.g, e.out);
        else launch_finish<float, double>(e.g, e.out);
    }
}

std::vector<tgtp_graph*> batch_plan_graphs(const BatchPlan* plan) {
    std::vector<tgtp_graph*> v;
    for (const BatchEntry& e : plan->entries) v.push_back(e.g);
    return v;
}


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
    if (g->has_multi_edges && cfg.precision == TGTP_PRECISION_MIXED)
        fail(TGTP_ERR_UNSUPPORTED,
             "the mixed form does not take rows with repeated neighbours or self-loops; "
             "use the FP32 or FP64 form");
    switch (cfg.precision) {
        case TGTP_PRECISION_FP32:
            if (!g->has_f32) fail(TGTP_ERR_INVALID_ARGUMENT, "FP32 form needs F32 eigenvectors");
            run_form<float, float, false, float>(g, cfg, device_scores);
            break;
        case TGTP_PRECISION_FP64:
            if (!g->has_f64) fail(TGTP_ERR_INVALID_ARGUMENT, "FP64 form needs F64 eigenvectors");
            run_form<double, double, false, double>(g, cfg, device_scores);
            break;
        case TGTP_PRECISION_MIXED:
            if (cfg.vec_dtype == TGTP_VEC_BF16) {
                if (!g->has_bf16) fail(TGTP_ERR_INVALID_ARGUMENT, "MIXED/BF16 needs BF16 eigenvectors");
                run_form<float, double, true, __nv_bfloat16>(g, cfg, device_scores);
            } else if (cfg.vec_dtype == TGTP_VEC_F32) {
                if (!g->has_f32) fail(TGTP_ERR_INVALID_ARGUMENT, "MIXED/F32 needs F32 eigenvectors");
                run_form<float, double, true, float>(g, cfg, device_scores);
            } else {
                fail(TGTP_ERR_INVALID_ARGUMENT, "MIXED form stores eigenvectors as F32 or BF16");
            }
            post_push_hint(g, form_key(cfg), cfg.epsilon);
            break;
        default:
            fail(TGTP_ERR_UNSUPPORTED, "unknown precision form");
    }
    g->last_precision = cfg.precision;
    g->have_run = true;
}

void aesc_check_flags(tgtp_graph* g) {
    unsigned flags[2];
    TGTP_CUDA(cudaMemcpyAsync(flags, run_work(g), sizeof(flags), cudaMemcpyDeviceToHost, g->stream));
    TGTP_CUDA(cudaStreamSynchronize(g->stream));
    if (flags[1] & kErrDeadline)
        fail(TGTP_ERR_TIMEOUT, "device time budget exceeded (TGTP_KERNEL_DEADLINE_S)");
    if (flags[1] & kErrWalkCount)
        fail(TGTP_ERR_UNSUPPORTED, "a walk count exceeds the 32-bit walk grid");
}

namespace {

// Mixed form: a dense round of the block push reads every slot once per 32 sources, about 40
// times cheaper per slot than a per-warp push reads a frontier entry (scattered residual updates in
// HBM).  So the block push pays off when a round's frontier averages more than m / 40 traversals
// -- for graphs whose residual vectors do not fit in shared memory (smaller ones push per warp in
// shared memory).  Measured on the sparse Chung-Lu graph (n = 25,860) at eps 0.05 / 0.01 / 0.005,
// R-MAT (n = 143,522) at 0.05 / 0.01 and Chung-Lu (n = 199,772) at 0.05 / 0.01 / 0.005, the rule
// picks the faster push every time (or one within 3 %).
void learn_push_hint(tgtp_graph* g, int key, double eps, unsigned long long rounds,
                     unsigned long long traversals) {
    if (key < 2 || rounds == 0) return;
    const double per_round = double(traversals) / double(rounds);
    g->push_hint[key] = (mixed_beyond_smem(g->n) && per_round * 40.0 > double(g->m)) ? 2 : 1;
    g->push_hint_eps[key] = eps;
}

// The counters of a completed mixed run copied to pinned memory (see tgtp_graph::hint_host), if
// that copy has finished; never waits.
void poll_push_hint(tgtp_graph* g) {
    if (g->hint_key < 0 || !g->hint_event) return;
    const cudaError_t e = cudaEventQuery(g->hint_event);
    if (e == cudaErrorNotReady) {
        (void)cudaGetLastError();
        return;
    }
    TGTP_CUDA(e);
    unsigned long long rounds = 0, trav = 0;
    for (int c = 0; c < kStStripes; ++c) {
        rounds += g->hint_host[size_t(c) * kStCount + kStPushRounds];
        trav += g->hint_host[size_t(c) * kStCount + kStPushTraversals];
    }
    learn_push_hint(g, g->hint_key, g->hint_eps, rounds, trav);
    g->hint_key = -1;
}

// After a mixed run on the handle's stream (not while capturing) on a graph whose vectors exceed
// shared memory (smaller ones always push per warp): copy its counters to pinned memory and
// record the event poll_push_hint looks at.
void post_push_hint(tgtp_graph* g, int key, double eps) {
    if (!mixed_beyond_smem(g->n)) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    TGTP_CUDA(cudaStreamIsCapturing(g->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return;
    const size_t bytes = sizeof(unsigned long long) * kStCount * kStStripes;
    if (!g->hint_host) {
        void* h = nullptr;
        TGTP_CUDA(cudaHostAlloc(&h, bytes, cudaHostAllocDefault));
        g->hint_host = static_cast<unsigned long long*>(h);
    }
    if (!g->hint_event) TGTP_CUDA(cudaEventCreateWithFlags(&g->hint_event, cudaEventDisableTiming));
    TGTP_CUDA(cudaMemcpyAsync(g->hint_host, g->stats.ptr, bytes, cudaMemcpyDeviceToHost, g->stream));
    TGTP_CUDA(cudaEventRecord(g->hint_event, g->stream));
    g->hint_key = key;
    g->hint_eps = eps;
}

}  // namespace

void aesc_read_stats(tgtp_graph* g, unsigned long long* st) {
    // the striped counters and the work words behind them, in one copy
    unsigned long long stripes[kStCount * kStStripes + 2];
    TGTP_CUDA(cudaMemcpyAsync(stripes, g->stats.ptr, sizeof(stripes), cudaMemcpyDeviceToHost,
                              g->stream));
    TGTP_CUDA(cudaStreamSynchronize(g->stream));
    unsigned work[4];
    std::memcpy(work, stripes + kStCount * kStStripes, sizeof(work));
    if (work[1] & kErrDeadline)
        fail(TGTP_ERR_TIMEOUT, "device time budget exceeded (TGTP_KERNEL_DEADLINE_S)");
    if (work[1] & kErrWalkCount)
        fail(TGTP_ERR_UNSUPPORTED, "a walk count exceeds the 32-bit walk grid");
    for (int i = 0; i < kStCount; ++i) st[i] = 0;
    for (int c = 0; c < kStStripes; ++c)
        for (int i = 0; i < kStCount; ++i) st[i] += stripes[size_t(c) * kStCount + i];
    learn_push_hint(g, g->last_key, g->last_eps, st[kStPushRounds], st[kStPushTraversals]);
}

int aesc_tune(tgtp_graph* g, const tgtp_config& cfg, float* device_scores, int trials) {
    const int key = form_key(cfg);
    const size_t rs = cfg.precision == TGTP_PRECISION_FP64 ? 8 : 4;
    const bool mixed = cfg.precision == TGTP_PRECISION_MIXED;
    size_t per_warp = ((g->n * rs + 15) & ~size_t(15)) + ((g->n + 15) & ~size_t(15)) + kAccBytes;
    if (mixed && per_warp + 8 * g->n <= size_t(112) * 1024) per_warp += 8 * g->n;
    std::vector<uint16_t> cand;
    // the parity forms also try the windowed and the one-vertex-at-a-time push in each layout
    const std::vector<uint16_t> push_kinds =
        mixed ? std::vector<uint16_t>{0} : std::vector<uint16_t>{kLayoutWindow, kLayoutNoWindow};
    for (uint16_t pk : push_kinds) {
        for (int w : {1, 2})
            if (per_warp * w <= size_t(227) * 1024) cand.push_back(uint16_t(pk | kLayoutSmem | w));
        for (int w : {1, 2, 4}) cand.push_back(uint16_t(pk | w));
    }
    if (mixed) {  // the block push, with the per-source stage in the best layout that fits,
                  // at each compaction threshold
        const uint16_t post = per_warp <= size_t(112) * 1024 ? uint16_t(kLayoutSmem | 1) : uint16_t(4);
        for (int ld = 0; ld < 4; ++ld)
            cand.push_back(uint16_t(kLayoutBlock | post | (ld << kLayoutListShift)));
    }
    cudaEvent_t e0, e1;
    TGTP_CUDA(cudaEventCreate(&e0));
    TGTP_CUDA(cudaEventCreate(&e1));
    const bool prof = g->prof.enabled;
    g->prof.enabled = false;
    float best = 0;
    uint16_t pick = 0;
    try {
        for (uint16_t c : cand) {
            g->src_layout[key] = c;
            try {
                aesc_run(g, cfg, device_scores);  // warm-up (and scratch for this layout)
            } catch (const Error&) {
                continue;  // the layout does not fit this graph
            }
            float t = 0;
            for (int i = 0; i < std::max(trials, 1); ++i) {
                TGTP_CUDA(cudaEventRecord(e0, g->stream));
                aesc_run(g, cfg, device_scores);
                TGTP_CUDA(cudaEventRecord(e1, g->stream));
                TGTP_CUDA(cudaEventSynchronize(e1));
                float ms = 0;
                TGTP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                t = i == 0 ? ms : std::min(t, ms);
            }
            if (!pick || t < best) {
                best = t;
                pick = c;
            }
        }
    } catch (...) {
        g->src_layout[key] = 0;
        g->prof.enabled = prof;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    g->src_layout[key] = pick;
    g->prof.enabled = prof;
    TGTP_CUDA(cudaEventDestroy(e0));
    TGTP_CUDA(cudaEventDestroy(e1));
    if (!pick) fail(TGTP_ERR_UNSUPPORTED, "no source-kernel layout fits this graph");
    return pick;
}

}  // namespace tgtp

using namespace tgtp;

namespace {
void finish_run(tgtp_graph* g) { aesc_check_flags(g); }
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
        TGTP_CUDA(cudaMemcpyAsync(host_scores, g->out.ptr, sizeof(float) * g->m,
                                  cudaMemcpyDeviceToHost, g->stream));
        unsigned long long st[kStCount];
        aesc_read_stats(g, st);  // synchronises once for scores, counters and error flags
    });
}

tgtp_status tgtp_last_run_stats(tgtp_graph* g, tgtp_run_stats* out) {
    return guarded([&] {
        if (!g || !out) fail(TGTP_ERR_INVALID_ARGUMENT, "null argument");
        if (!g->have_run) fail(TGTP_ERR_INVALID_ARGUMENT, "no run on this graph yet");
        finish_run(g);
        unsigned long long st[kStCount] = {};
        aesc_read_stats(g, st);
        out->push_rounds = st[kStPushRounds];
        out->push_vertices = st[kStPushVertices];
        out->push_traversals = st[kStPushTraversals];
        out->walk_edges = st[kStWalkEdges];
        out->walk_count = st[kStWalkCount];
        out->walk_hops = st[kStWalkHops];
        out->fallback_bouquets = st[kStFallback];
        out->tau_iterations = st[kStTauIters];
        out->tau_ambiguous = st[kStTauAmbiguous];
        for (int i = 0; i < 8; ++i) out->phase_cycles[i] = st[kStPhase0 + i];
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
