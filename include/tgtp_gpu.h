/*
 * tgtp_gpu.h — C ABI of the B200 (sm_100a) implementation of the tgtp hot path:
 * the TGT+ approximate edge spanning centrality tgtp() and the SABA walk counter.
 *
 * Every entry point takes plain pointers and sizes, returns a tgtp_status (0 = success) and never
 * throws.  Host buffers are owned by the caller; the library never keeps a host pointer after a
 * call returns.  A graph handle owns one CUDA stream (or borrows the caller's, see
 * tgtp_graph_set_stream); calls on one handle must not run concurrently from several threads.
 * On failure tgtp_last_error() returns a message for the calling thread.
 *
 * Reference interfaces replaced (paths within ggokturk/tgtp):
 *   fuser::graph_t::load_txt            src/graph.h:29-97      -> tgtp_load_graph_txt + tgtp_graph_upload
 *   EigenVecs<float>::load_txt          src/aesc.h:51-64       -> tgtp_load_eigens_txt + tgtp_eigens_upload
 *   AESCGraph(graph, eigens, omega)     src/aesc.h:85-92       -> tgtp_graph_upload + tgtp_eigens_upload
 *   AESCConfig{epsilon,delta,omega,gamma} src/aesc.h:98-102    -> tgtp_config
 *   float* AESC::tgtp()                 src/aesc.h:120-127     -> tgtp_run / tgtp_run_device
 *   saba_randomwalk + runner reduction  src/rw_experiment_saba.cpp:65-145,186-208 -> saba_count
 *   scalar_randomwalk + runner reduction src/rw_experiment.cpp:34-47,88-118      -> mt_walk_count(0)
 *   simd_randomwalk + runner reduction  src/rw_experiment_simd.cpp:44-83,128-156  -> mt_walk_count(1)
 *   AESCGraph::free / graph_t::free     src/aesc.h:93-96, src/graph.h:22-28 -> tgtp_graph_free
 *   exception -> "tgtp: msg", exit 1    src/main.cpp:46-49     -> tgtp_status + tgtp_last_error
 */
#ifndef TGTP_GPU_H
#define TGTP_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TGTP_ABI_VERSION 1

typedef enum {
    TGTP_OK = 0,
    TGTP_ERR_INVALID_ARGUMENT = 1, /* bad sizes, omega, epsilon, gamma, isolated vertex, ...     */
    TGTP_ERR_CUDA = 2,             /* a CUDA runtime call or kernel launch failed                */
    TGTP_ERR_OUT_OF_MEMORY = 3,    /* device or host allocation failed                           */
    TGTP_ERR_TIMEOUT = 4,          /* a bounded device-side wait gave up (error flag set)        */
    TGTP_ERR_IO = 5,               /* file could not be opened, parsed or written                */
    TGTP_ERR_UNSUPPORTED = 6,      /* configuration outside what this build supports             */
    TGTP_ERR_OVERFLOW = 7          /* a result exceeded its integer type (e.g. a uint32 counter) */
} tgtp_status;

/* Storage type of eigenvectors on the device. */
typedef enum {
    TGTP_VEC_F32 = 0,  /* the reference's own storage (EigenVecs<float>) */
    TGTP_VEC_F64 = 1,
    TGTP_VEC_BF16 = 2
} tgtp_vec_dtype;

/* Arithmetic form of tgtp_run. */
typedef enum {
    /* The reference's arithmetic: FP32 residuals/eigenvectors, FP64 logs, the reference's
     * evaluation order everywhere.  Bit-exact with the reference built at -O2. Needs F32 vectors. */
    TGTP_PRECISION_FP32 = 0,
    /* Every float of the reference held in double (needs F64 vectors). */
    TGTP_PRECISION_FP64 = 1,
    /* FP32 residuals, lane-parallel compensated FP32 eigen projections over F32 or BF16 vectors,
     * FP64 tau bounds, stop test and per-edge score accumulation; reductions in parallel order. */
    TGTP_PRECISION_MIXED = 2
} tgtp_precision;

typedef struct {
    double epsilon;    /* 0 < epsilon < 1                                        */
    double delta;      /* the reference's callers pass 1/n (src/main.cpp:36)      */
    int32_t omega;     /* number of eigenpairs used, 2 <= omega <= uploaded omega */
    int32_t gamma;     /* top-gamma residuals for the edge bound, >= 1            */
    int32_t precision; /* tgtp_precision                                          */
    int32_t vec_dtype; /* tgtp_vec_dtype read by TGTP_PRECISION_MIXED             */
} tgtp_config;

typedef struct tgtp_graph tgtp_graph;

/* Work counters of the last tgtp_run on a graph (same meaning as the oracle's counters). */
typedef struct {
    uint64_t push_rounds;       /* sum over sources of the final push round count ell   */
    uint64_t push_vertices;     /* frontier vertices drained                             */
    uint64_t push_traversals;   /* adjacency entries visited while pushing               */
    uint64_t walk_edges;        /* CSR slots that ran the 2-way walk                     */
    uint64_t walk_count;        /* sum of walk counts nr over those slots                */
    uint64_t walk_hops;         /* sum of nr * remaining length (pairs of hops)          */
    uint64_t fallback_bouquets; /* bouquets that switched to the SplitMix32 phase        */
    uint64_t tau_iterations;    /* delta-term evaluations of the tau bound               */
    uint64_t tau_ambiguous;     /* tau bounds whose ceil() argument lay within 1e-12 of an
                                   integer (where a last-place libm difference could matter)  */
    uint64_t phase_cycles[8];   /* SM cycles of the per-source kernel by phase, summed over
                                   warps: claim/init, push, post-push, cost test, edge bound,
                                   chi/walk counts, walks, reset                               */
} tgtp_run_stats;

typedef struct {
    uint64_t visit_count;       /* sum of all counters (exact)                            */
    uint64_t checksum;          /* sum of (v + 1) * counter[v] (exact)                    */
    uint64_t fallback_bouquets; /* bouquets that switched to the SplitMix32 phase         */
} saba_result;

/* Per-kernel device time accumulated while profiling is on (tgtp_graph_set_profiling). */
typedef struct {
    char name[48];
    uint64_t launches;
    double total_ms;
} tgtp_kernel_stat;

/* ---- errors / version ---------------------------------------------------------------------- */
const char* tgtp_last_error(void);
int tgtp_abi_version(void);

/* ---- host-side file loaders (reference file formats) ---------------------------------------- */
/* graph.txt -> CSR exactly as src/graph.h:29-97 builds it (mirrored edges, rows sorted, no dedup,
 * n = max id + 1, '#'/'%' comment lines).  *idx (n+1) and *adj (m) are allocated by the library;
 * release them with tgtp_host_free. */
tgtp_status tgtp_load_graph_txt(const char* path, uint32_t** idx, uint32_t** adj, uint64_t* n,
                                uint64_t* m);
/* sorted_eigens_<omega>.txt -> values[omega] (double) and vertex-major vectors[n*omega], parsed
 * straight to float (vec_f32) and/or double (vec_f64) as src/aesc.h:51-64 does; either vector
 * pointer may be NULL.  Caller-allocated buffers. */
tgtp_status tgtp_load_eigens_txt(const char* path, uint64_t n, uint32_t omega, double* values,
                                 float* vec_f32, double* vec_f64);
void tgtp_host_free(void* p);

/* ---- graphs ----------------------------------------------------------------------------------- */
/* Copies the CSR (host buffers, m = idx[n]) to the current CUDA device.  Rejects m >= 2^32,
 * non-monotone offsets and out-of-range neighbours. */
tgtp_status tgtp_graph_upload(const uint32_t* idx, const uint32_t* adj, uint64_t n, uint64_t m,
                              tgtp_graph** out);
tgtp_status tgtp_graph_free(tgtp_graph* g);
/* Use the caller's cudaStream_t (NULL: go back to the handle's own stream). */
tgtp_status tgtp_graph_set_stream(tgtp_graph* g, void* cuda_stream);
void* tgtp_graph_stream(tgtp_graph* g);
tgtp_status tgtp_graph_info(const tgtp_graph* g, uint64_t* n, uint64_t* m);

/* Uploads omega eigenpairs (values: double[omega]; vectors: vertex-major n*omega of `dtype`,
 * F32 or F64 host data).  The device storage may differ from the host type (F64 host data stored
 * as F32 or BF16, F32 host data as BF16): pass the host dtype in `dtype` and the device storage in
 * `store_dtype`.  Several storages may be
 * uploaded side by side; each call replaces the storage it names. */
tgtp_status tgtp_eigens_upload(tgtp_graph* g, const double* values, const void* vectors,
                               uint32_t omega, int32_t dtype, int32_t store_dtype);

/* ---- tgtp ----------------------------------------------------------------------------------- */
/* Scores of every CSR slot (m float32, symmetric), written to caller-owned host memory.
 * Synchronous.  AESCConfig validation as src/main.cpp:27-30 and src/aesc.h:87-89. */
tgtp_status tgtp_run(tgtp_graph* g, const tgtp_config* cfg, float* host_scores);
/* Same, into caller-owned device memory (m float32), asynchronous on the handle's stream.
 * Input validation and scratch allocation still happen on the host before the launch. */
tgtp_status tgtp_run_device(tgtp_graph* g, const tgtp_config* cfg, float* device_scores);
/* Work counters of the last completed run (synchronises the handle's stream). */
tgtp_status tgtp_last_run_stats(tgtp_graph* g, tgtp_run_stats* out);
/* Per-slot tau of the last run (m int32, host). */
tgtp_status tgtp_last_taus(tgtp_graph* g, int32_t* host_taus);

/* Times the candidate layouts of the source kernel (per-source residual vectors in shared memory
 * or in HBM, warps per block; for the mixed form also the multi-source block push at four
 * push-frontier thresholds) for cfg's precision form on this graph, `trials` runs each after a
 * warm-up, and keeps the fastest on the handle for later runs of that form.  Scores are identical
 * under every layout.  *layout (may be NULL) receives the choice: 0x100 bit = shared memory, low
 * byte = warps per block, 0x200 = block push, bits 12-13 = its compaction threshold (a round is
 * compacted to the rows next to the live ones when their degree sum is below m / 4, m / 2,
 * m / 16, or never); for the FP32 and FP64 forms 0x400 = the windowed sequential push, 0x800 =
 * one frontier vertex at a time.  The reference has no counterpart (its OpenMP loop has one
 * layout). */
tgtp_status tgtp_graph_tune(tgtp_graph* g, const tgtp_config* cfg, float* device_scores,
                            int32_t trials, int32_t* layout);

/* ---- batched tgtp ----------------------------------------------------------------------------- */
/* Many tgtp() runs (src/aesc.h:120-127 each: its own graph, epsilon, omega, gamma and precision
 * form) replayed as one CUDA graph.  Creation runs each configuration once (sizing its buffers;
 * with tune_trials > 0 also tgtp_graph_tune), then captures all runs as parallel branches, one per
 * graph; every graph may appear once.  Scores go to the caller-owned device buffers given here
 * (m float32 each) on every tgtp_batch_run.  While the batch lives, its graphs keep their buffers:
 * tgtp_eigens_upload, tgtp_graph_free and runs that would need larger buffers are refused. */
typedef struct tgtp_batch tgtp_batch;
tgtp_status tgtp_batch_create(tgtp_graph* const* graphs, const tgtp_config* configs,
                              float* const* device_scores, uint32_t count, int32_t tune_trials,
                              tgtp_batch** out);
/* One cudaGraphLaunch on cuda_stream (NULL: the batch's own stream); asynchronous. */
tgtp_status tgtp_batch_run(tgtp_batch* b, void* cuda_stream);
/* Waits for the last tgtp_batch_run and reports a device time-out or walk-count error of any run;
 * afterwards tgtp_last_run_stats of each graph describes its run in the batch. */
tgtp_status tgtp_batch_wait(tgtp_batch* b);
tgtp_status tgtp_batch_free(tgtp_batch* b);

/* ---- SABA walk counter ---------------------------------------------------------------------- */
/* n_walks walks of `depth` hops from every vertex with nonzero degree; counters[v] = visits of v
 * (start vertex excluded).  host_counters (n uint32) may be NULL.  Synchronous.
 * n_walks must be a multiple of 8 (src/rw_experiment_saba.cpp:160-163). */
tgtp_status saba_count(tgtp_graph* g, uint32_t depth, uint32_t n_walks, uint32_t* host_counters,
                       saba_result* out);
/* Counters into caller-owned device memory (n uint32), asynchronous on the handle's stream. */
tgtp_status saba_count_device(tgtp_graph* g, uint32_t depth, uint32_t n_walks,
                              uint32_t* device_counters);

/* Times the walk layouts for this graph and walk configuration and keeps the fastest on the handle
 * for later saba_count calls: 1, 2 or 4 walkers per lane (4, 8 or 16 eight-lane bouquets per warp)
 * over the degree-renumbered walk copy, plain (with none, 3,072 or 4,096 of the highest-degree row
 * records held in shared memory) or with the next row's record inlined in each slot.  `trials`
 * timed runs each after a warm-up.  *choice (may be NULL) receives the pick: low byte = walkers per
 * lane, 0x100 = inlined copy, bits 12-14 = c for 1,024 x c shared row records.
 * Counters are identical under every layout.  The reference has no counterpart (its OpenMP loop
 * has one layout). */
tgtp_status saba_tune(tgtp_graph* g, uint32_t depth, uint32_t n_walks, int32_t trials,
                      int32_t* choice);

/* ---- MT19937 walk baselines ------------------------------------------------------------------ */
/* The reference's comparison walks: from every vertex with a neighbour, n_walks walks of `depth`
 * hops with std::mt19937 reseeded to 42 + src and k = draw % degree per hop; simd = 0 takes the
 * scalar runner's draw order (walk-major, src/rw_experiment.cpp:34-47), simd = 1 the AVX2 runner's
 * (bouquets of 8 walks, the 8 draws of a hop in lane order, src/rw_experiment_simd.cpp:44-83;
 * n_walks a multiple of 8).  counters[v] = visits of v (start vertex excluded), exact uint32
 * (the reference's float counters stop at 2^24 per thread); host_counters (n uint32) may be NULL;
 * out->fallback_bouquets is 0.  Synchronous. */
tgtp_status mt_walk_count(tgtp_graph* g, uint32_t depth, uint32_t n_walks, int32_t simd,
                          uint32_t* host_counters, saba_result* out);

/* No counterpart in the reference: the walk counter for callers that cannot allocate device
 * memory, e.g. a process whose device memory is owned by another allocator or budget, or a
 * latency-critical loop where cudaMalloc/cudaFree would synchronise the device.  It allocates
 * nothing: the caller passes the CSR already on the device (n + 1 offsets, and device_adj holding
 * the idx[n] neighbours the offsets declare) and gets the walk runner's summary.  The per-vertex
 * counters and sums live in one fixed 16 MiB device array inside the library, present on every
 * GPU that loads it until the process exits, so n is limited to 4,194,304 vertices (larger n is
 * rejected with TGTP_ERR_INVALID_ARGUMENT).  Before any walk the CSR is checked on the device:
 * offsets starting at 0 and never decreasing, neighbour ids below n, and no edge into a vertex
 * without neighbours; a CSR that fails is refused with TGTP_ERR_INVALID_ARGUMENT and no walk runs.
 * Every call clears and reuses the same array: calls that overlap on the GPU (other streams,
 * other threads) race and give wrong results.  Runs on cuda_stream (NULL: the default stream) and
 * synchronises it (twice: after the check and at the end), so it cannot be called while that
 * stream is being captured into a CUDA graph. */
tgtp_status saba_count_static(const uint32_t* device_idx, const uint32_t* device_adj, uint64_t n,
                              uint32_t depth, uint32_t n_walks, void* cuda_stream,
                              saba_result* out);

/* ---- exact spanning centrality of sampled edges (the accuracy reference) -------------------- */
/* The quantity of src/exact_sc.cpp:24-49 (and scripts/paper_accuracy.py:13-54) for graphs too large
 * for its dense solve: R(u, v) = (e_u - e_v)^T L^+ (e_u - e_v) for each listed CSR slot (u, v), on the
 * simple graph of the CSR (a repeated neighbour counts once, self-loops are ignored; a self-loop slot
 * gives 0).  Jacobi-preconditioned conjugate gradients in FP64 on the device, 32 slots at a time;
 * every slot iterates until its residual norm is at most tol * ||e_u - e_v|| (TGTP_ERR_TIMEOUT when
 * max_iter iterations do not get there).  host_iterations (may be NULL) receives the iteration count
 * of each batch of 32 slots (ceil(count / 32) entries).  Synchronous; scratch is allocated per call
 * (5 blocks of n x 32 doubles). */
tgtp_status tgtp_exact_sc_slots(tgtp_graph* g, const uint32_t* host_slots, uint32_t count,
                                double tol, uint32_t max_iter, double* host_resistance,
                                uint32_t* host_iterations);

/* ---- memory ---------------------------------------------------------------------------------- */
/* Device blocks of released graphs are kept for reuse (creating a graph per input would otherwise
 * pay cudaMalloc/cudaFree for its scratch every time).  This returns every cached block to the
 * driver; blocks held by live graphs are unaffected. */
tgtp_status tgtp_release_cached_memory(void);

/* ---- profiling ------------------------------------------------------------------------------ */
/* When on, every kernel launch is bracketed by CUDA events on the handle's stream and its device
 * time is accumulated per kernel name.  Turning it on clears the table. */
tgtp_status tgtp_graph_set_profiling(tgtp_graph* g, int enable);
/* Copies up to `cap` entries; *count = entries available.  Synchronises the stream. */
tgtp_status tgtp_graph_kernel_stats(tgtp_graph* g, tgtp_kernel_stat* out, int32_t cap,
                                    int32_t* count);
/* Run trace, no counterpart in the reference (its per-source locals ell and nr,
 * src/aesc.h:473-521, are not kept).  When on, every later run on the handle records the rounds
 * pushed (ell) of each row that ran in the source kernel and the walk count nr of each walking
 * slot; rows scored in closed form read 0 rounds, slots without walks 0.  Costs one store per row
 * and per walking slot.  Not for runs captured into a batch. */
tgtp_status tgtp_graph_set_trace(tgtp_graph* g, int enable);
/* The trace of the handle's last run: host_walks m entries, host_rounds n entries (either may be
 * NULL).  Synchronises the stream; TGTP_ERR_INVALID_ARGUMENT when the trace is off or no run has
 * been made since it was turned on. */
tgtp_status tgtp_graph_read_trace(tgtp_graph* g, uint32_t* host_walks, uint32_t* host_rounds);

#ifdef __cplusplus
}
#endif
#endif /* TGTP_GPU_H */
