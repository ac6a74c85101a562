// Internal declarations of libtgtp_gpu: error plumbing, device buffers, the graph handle and the
// per-kernel event profiler.  Nothing here crosses the C ABI (include/tgtp_gpu.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "tgtp_gpu.h"

namespace tgtp {

// Internal failures travel as exceptions and are turned into a status at the ABI boundary.
struct Error {
    tgtp_status code;
    std::string msg;
};

[[noreturn]] inline void fail(tgtp_status code, const std::string& msg) { throw Error{code, msg}; }

void set_last_error(const std::string& msg);

#define TGTP_CUDA(call)                                                                        \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            (void)cudaGetLastError();                                                          \
            ::tgtp::fail(e_ == cudaErrorMemoryAllocation ? TGTP_ERR_OUT_OF_MEMORY : TGTP_ERR_CUDA, \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                 \
        }                                                                                      \
    } while (0)

#define TGTP_LAUNCH_CHECK(name)                                                                \
    do {                                                                                       \
        cudaError_t e_ = cudaGetLastError();                                                   \
        if (e_ != cudaSuccess)                                                                 \
            ::tgtp::fail(TGTP_ERR_CUDA, std::string("launch of ") + (name) + ": " +            \
                                            cudaGetErrorString(e_));                           \
    } while (0)

template <class F>
tgtp_status guarded(F&& f) {
    try {
        f();
        return TGTP_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return TGTP_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return TGTP_ERR_INVALID_ARGUMENT;
    }
}

// Process-wide cache of device blocks.  Graphs are created and released often (one per input in a
// batch, one per call through the plain C entry points), and cudaMalloc / cudaFree of the ~100 MB
// of per-run scratch would dominate such calls.  Blocks are rounded to a size class and kept per
// device after release; a release first waits for the device to be idle, so no queued kernel can
// still be using the block when it is handed out again.  tgtp_release_cached_memory() returns the
// cached blocks to the driver.
void* cache_alloc(size_t bytes, size_t* granted);
void cache_free(void* p, size_t granted);
void cache_trim();
cudaStream_t stream_acquire();
void stream_release(cudaStream_t s);

// Grow-only device allocation owned by a graph handle.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { release(); }
    void release() {
        if (ptr) cache_free(ptr, bytes);
        ptr = nullptr;
        bytes = 0;
    }
    void reserve(size_t want) {
        if (want <= bytes && ptr) return;
        release();
        if (want == 0) want = 16;
        ptr = cache_alloc(want, &bytes);
    }
    template <class T>
    T* as() const { return static_cast<T*>(ptr); }
};

// CUDA-event timing of each kernel launch on the handle's stream (off unless asked for).
class Profiler {
public:
    bool enabled = false;
    void begin(cudaStream_t s, const char* name);
    void end(cudaStream_t s);
    void clear();
    // Synchronises the pending events and folds them into the totals.
    void collect();
    struct Entry {
        std::string name;
        uint64_t launches = 0;
        double total_ms = 0;
    };
    std::vector<Entry> totals;
    ~Profiler();

private:
    struct Pending {
        std::string name;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending_;
    std::vector<cudaEvent_t> pool_;
    cudaEvent_t take();
    const char* open_name_ = nullptr;
    cudaEvent_t open_ = nullptr;
};

struct ScopedKernel {
    Profiler& p;
    cudaStream_t s;
    ScopedKernel(Profiler& p_, cudaStream_t s_, const char* name) : p(p_), s(s_) {
        if (p.enabled) p.begin(s, name);
    }
    ~ScopedKernel() {
        if (p.enabled) p.end(s);
    }
};

}  // namespace tgtp

// The opaque handle of the C ABI.
struct tgtp_graph {
    int device = 0;
    int num_sms = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    uint64_t n = 0, m = 0;
    uint32_t max_degree = 0, min_degree = 0;
    bool has_multi_edges = false;  // a row holds the same neighbour twice (loader keeps them)
    uint64_t num_forward = 0;      // slots (u, v) with v >= u
    uint64_t num_active = 0;       // vertices with nonzero degree

    // CSR and derived per-slot maps (device)
    tgtp::DeviceBuffer idx, adj, deg;
    tgtp::DeviceBuffer row_of;   // slot -> its row u
    tgtp::DeviceBuffer rev;      // slot (u,v) -> lower_bound of u in row v
    tgtp::DeviceBuffer sym_src;  // slot q -> 1 + last slot p with rev[p] == q (0: none)
    tgtp::DeviceBuffer forward;  // slots with v >= u, in CSR order
    tgtp::DeviceBuffer fedge;    // per forward slot: (u, v, slot, reverse slot)
    tgtp::DeviceBuffer adjd;     // slot -> (neighbour, neighbour's degree)
    tgtp::DeviceBuffer prep_cnt, prep_lbp;  // graph_prepare's per-row forward counts and bounds

    // eigenpairs
    uint32_t omega = 0;
    std::vector<double> values;  // host copy (constants of the tau bound are formed on the host)
    tgtp::DeviceBuffer d_values, vec_f32, vec_f64, vec_bf16;
    // tau-bound constants: onep[i] = 1 + lambda_i, onem[i] = 1 - lambda_i and the powers
    // lambda_i^(2(k+1)) for k < kTauTableRows, formed by the reference's repeated multiplication
    tgtp::DeviceBuffer onep, onem, etab, etab_f;
    tgtp::DeviceBuffer wtab32, wtab64;  // weights of the split tau kernel for split_omega
    uint32_t split_omega = 0;
    tgtp::DeviceBuffer row_list;  // rows with a slot of tau > 1 (their marks follow the counters)
    uint16_t src_layout[4] = {0, 0, 0, 0};  // tuned source-kernel layout per form (0 = default)
    tgtp::DeviceBuffer wclean;  // per warp of the source kernel: HBM vectors left all zero
    uint64_t wclean_sig[5] = {0, 0, 0, 0, 0};  // the scratch carving those marks belong to
    int batch_refs = 0;  // live batches whose CUDA graph points at this handle's buffers
    int last_key = -1;   // form of the last run (see form_key in aesc.cu)
    double last_eps = 0;  // and its epsilon
    // mixed form, per vector storage: 2 when the last completed run's frontiers were large enough
    // for the multi-source block push to pay off, 1 when not, 0 unknown
    uint8_t push_hint[4] = {0, 0, 0, 0};
    double push_hint_eps[4] = {0, 0, 0, 0};  // the epsilon each hint was measured at
    // each mixed run also copies its two push counters into pinned host memory behind an event;
    // the next run reads them there once the event has completed, so the hint is learned without
    // the caller reading the counters and without a synchronisation (hint_key: form of the copy
    // in flight, -1 none)
    // run trace (tgtp_graph_set_trace): m walk counts per slot, then n rounds per row
    bool trace_on = false, trace_valid = false;
    tgtp::DeviceBuffer trace;
    unsigned long long* hint_host = nullptr;
    cudaEvent_t hint_event = nullptr;
    int hint_key = -1;
    double hint_eps = 0;
    bool has_f32 = false, has_f64 = false, has_bf16 = false;

    // run scratch
    tgtp::DeviceBuffer taus, preds, stats, counters, sums, scratch, out;
    tgtp::DeviceBuffer tau_sums;  // per forward edge: (upsilon, delta_0) sums of the split forms
    tgtp::DeviceBuffer block_cols, block_pre, block_final, block_keys, block_tmp;  // multi-source push
    tgtp::DeviceBuffer block_bits;   // the block push's row masks when they do not fit in smem
    tgtp::DeviceBuffer block_lists;  // the block push's row lists (four of n entries per CTA)
    tgtp::DeviceBuffer walk_queue, walk_ctl;  // the block push's walk items; per wave length, claim
    // walk copy of the graph renumbered by degree (built on the first saba_count)
    tgtp::DeviceBuffer saba_info, saba_adj, saba_cnt;
    bool saba_ready = false;
    // the same copy with each slot holding its target's row record (16 bytes per slot; built on
    // the first saba_count that walks the inlined copy)
    tgtp::DeviceBuffer saba_adj16;
    bool saba_inline_ready = false;
    // the walk layout saba_tune chose: walkers per lane (low byte: 1, 2 or 4, so 4, 8 or 16
    // bouquets per warp) and 0x100 for the inlined copy; 0 = not tuned
    uint16_t saba_choice = 0;
    int32_t last_precision = -1;
    bool have_run = false;

    tgtp::Profiler prof;

    ~tgtp_graph();
};

namespace tgtp {
void saba_run(tgtp_graph* g, uint32_t depth, uint32_t n_walks, uint32_t* device_counters);
// Times the walk layouts (walkers per lane 1 / 2 / 4, plain or inlined copy) for this graph and
// walk configuration, `trials` runs each after a warm-up, and keeps the fastest on the handle.
int saba_tune(tgtp_graph* g, uint32_t depth, uint32_t n_walks, int trials);
void saba_summarize(tgtp_graph* g, const uint32_t* device_counters, uint64_t* host_sums3);
// The reference's MT19937 walk baselines (scalar or 8-lane bouquet draw order) into
// device_counters (n uint32), asynchronous; the sums of saba_summarize then describe them.
void mt_walk_run(tgtp_graph* g, uint32_t depth, uint32_t n_walks, bool simd, uint32_t* device_counters);
void aesc_run(tgtp_graph* g, const tgtp_config& cfg, float* device_scores);
// Times the candidate source-kernel layouts of cfg's form on this graph (trials runs each, after
// one warm-up) and keeps the fastest on the handle.  Returns the chosen layout code.
int aesc_tune(tgtp_graph* g, const tgtp_config& cfg, float* device_scores, int trials);
// Error flags of the handle's last run as a failure (synchronises the handle's stream).
void aesc_check_flags(tgtp_graph* g);
// Run counters of the last run summed over their stripes (synchronises the handle's stream); also
// records from them which push of the mixed form suits this graph (push_hint).  st holds
// kRunStatSlots entries (the counters fill the first ones).
constexpr int kRunStatSlots = 32;
void aesc_read_stats(tgtp_graph* g, unsigned long long* st);
void graph_prepare(tgtp_graph* g);
// Batched runs (aesc.cu): while collection is on for this thread (batch_plan_collect(plan)),
// aesc_run leaves the per-source stage and the symmetrisation of per-warp-push runs to the plan;
// batch_plan_launch then runs one persistent source kernel per (form, tier) group over all the
// deferred graphs' rows on stream s, and batch_plan_finish each deferred graph's finish kernel on
// the graph's own stream.  batch_plan_collect(nullptr) ends collection.
struct BatchPlan;
BatchPlan* batch_plan_new();
void batch_plan_free(BatchPlan* plan);
void batch_plan_collect(BatchPlan* plan);
size_t batch_plan_deferred(const BatchPlan* plan);
void batch_plan_launch(BatchPlan* plan, cudaStream_t s, int num_sms);
void batch_plan_finish(BatchPlan* plan);
std::vector<tgtp_graph*> batch_plan_graphs(const BatchPlan* plan);
}  // namespace tgtp
