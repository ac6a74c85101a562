// Batched tgtp(): many (graph, configuration) runs replayed as one CUDA graph.
//
// A batch is built once: every run is executed once on its graph handle (which sizes all of the
// handle's buffers and weight tables, and optionally times the candidate source-kernel layouts and
// keeps the fastest), then all runs are captured from one origin stream that forks to each handle's
// stream.  Each graph's branch runs its tau kernels; the per-source stage of every run that pushes
// per warp is left to the batch (aesc.cu, BatchPlan): the branches join, one persistent source
// kernel per (arithmetic form, residual-vector tier) works through the listed rows of all those
// graphs as one queue of (graph, row) items, so the rows of small graphs fill the SMs that a large
// graph leaves idle, and the branches fork again for each graph's symmetrisation.  Runs whose push
// is the multi-source block push keep their whole run in their branch.  tgtp_batch_run is one
// cudaGraphLaunch.  While a batch is alive its graphs keep their buffers: runs on them that would
// need larger buffers, eigen uploads and frees are refused.  TGTP_BATCH_PERSISTENT=0 captures every
// run whole in its branch instead (no shared persistent kernel).
#include <algorithm>
#include <cstdlib>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "internal.hpp"

struct tgtp_batch {
    std::vector<tgtp_graph*> graphs;
    std::vector<tgtp_config> configs;
    std::vector<float*> outs;
    std::vector<cudaEvent_t> events;
    cudaStream_t origin = nullptr;
    cudaStream_t last = nullptr;  // stream of the last launch
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    tgtp::BatchPlan* plan = nullptr;  // the deferred per-source stages and their shared scratch

    ~tgtp_batch() {
        if (last) cudaStreamSynchronize(last);
        if (origin) cudaStreamSynchronize(origin);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (plan) tgtp::batch_plan_free(plan);
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        if (origin) tgtp::stream_release(origin);
        for (tgtp_graph* g : graphs) --g->batch_refs;
    }
};

using namespace tgtp;

namespace {

cudaEvent_t new_event(tgtp_batch* b) {
    cudaEvent_t e = nullptr;
    TGTP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->events.push_back(e);
    return e;
}

void capture(tgtp_batch* b) {
    std::vector<cudaStream_t> streams;
    for (tgtp_graph* g : b->graphs)
        if (std::find(streams.begin(), streams.end(), g->stream) == streams.end())
            streams.push_back(g->stream);
    std::vector<bool> prof;
    for (tgtp_graph* g : b->graphs) {
        prof.push_back(g->prof.enabled);
        g->prof.enabled = false;
    }
    TGTP_CUDA(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeRelaxed));
    try {
        cudaEvent_t fork = new_event(b);
        TGTP_CUDA(cudaEventRecord(fork, b->origin));
        for (cudaStream_t s : streams) TGTP_CUDA(cudaStreamWaitEvent(s, fork, 0));
        const char* pe = std::getenv("TGTP_BATCH_PERSISTENT");
        const bool persistent = !(pe && std::string(pe) == "0");
        if (persistent) {
            if (!b->plan) b->plan = batch_plan_new();
            batch_plan_collect(b->plan);
        }
        try {
            for (size_t i = 0; i < b->graphs.size(); ++i)
                aesc_run(b->graphs[i], b->configs[i], b->outs[i]);
        } catch (...) {
            batch_plan_collect(nullptr);
            throw;
        }
        batch_plan_collect(nullptr);
        auto join_all = [&]() {
            for (cudaStream_t s : streams) {
                cudaEvent_t join = new_event(b);
                TGTP_CUDA(cudaEventRecord(join, s));
                TGTP_CUDA(cudaStreamWaitEvent(b->origin, join, 0));
            }
        };
        join_all();
        if (persistent && batch_plan_deferred(b->plan) > 0) {
            // the persistent source kernels on the origin stream, then every deferred graph's
            // symmetrisation on its own stream again
            batch_plan_launch(b->plan, b->origin, b->graphs[0]->num_sms);
            cudaEvent_t fork2 = new_event(b);
            TGTP_CUDA(cudaEventRecord(fork2, b->origin));
            for (cudaStream_t s : streams) TGTP_CUDA(cudaStreamWaitEvent(s, fork2, 0));
            batch_plan_finish(b->plan);
            join_all();
        }
    } catch (...) {
        cudaGraph_t dead = nullptr;
        cudaStreamEndCapture(b->origin, &dead);
        if (dead) cudaGraphDestroy(dead);
        for (size_t i = 0; i < b->graphs.size(); ++i) b->graphs[i]->prof.enabled = prof[i];
        throw;
    }
    TGTP_CUDA(cudaStreamEndCapture(b->origin, &b->graph));
    for (size_t i = 0; i < b->graphs.size(); ++i) b->graphs[i]->prof.enabled = prof[i];
    TGTP_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
}

}  // namespace

extern "C" {

tgtp_status tgtp_graph_tune(tgtp_graph* g, const tgtp_config* cfg, float* device_scores,
                            int32_t trials, int32_t* layout) {
    return guarded([&] {
        if (!g || !cfg || !device_scores) fail(TGTP_ERR_INVALID_ARGUMENT, "null argument");
        const int pick = aesc_tune(g, *cfg, device_scores, trials);
        aesc_check_flags(g);
        if (layout) *layout = pick;
    });
}

tgtp_status tgtp_batch_create(tgtp_graph* const* graphs, const tgtp_config* configs,
                              float* const* device_scores, uint32_t count, int32_t tune_trials,
                              tgtp_batch** out) {
    return guarded([&] {
        if (!graphs || !configs || !device_scores || !out || count == 0)
            fail(TGTP_ERR_INVALID_ARGUMENT, "null argument or empty batch");
        *out = nullptr;
        std::set<tgtp_graph*> seen;
        for (uint32_t i = 0; i < count; ++i) {
            if (!graphs[i] || !device_scores[i]) fail(TGTP_ERR_INVALID_ARGUMENT, "null graph or output");
            if (!seen.insert(graphs[i]).second)
                fail(TGTP_ERR_INVALID_ARGUMENT, "a graph appears twice in one batch");
        }
        // one plain run each (sizes every buffer), the layout search if asked, then the capture
        for (uint32_t i = 0; i < count; ++i) {
            if (tune_trials > 0) aesc_tune(graphs[i], configs[i], device_scores[i], tune_trials);
            aesc_run(graphs[i], configs[i], device_scores[i]);
        }
        for (uint32_t i = 0; i < count; ++i) {
            aesc_check_flags(graphs[i]);
            unsigned long long st[kRunStatSlots];
            aesc_read_stats(graphs[i], st);  // measures which push suits a mixed run
            if (tune_trials <= 0) aesc_run(graphs[i], configs[i], device_scores[i]);
        }
        // The replays run on the CUDA graph's own streams, which do not wait for work still
        // queued on the handles' streams: let those plain runs finish before the first replay.
        for (uint32_t i = 0; i < count; ++i) aesc_check_flags(graphs[i]);
        auto b = std::make_unique<tgtp_batch>();
        b->origin = stream_acquire();
        for (uint32_t i = 0; i < count; ++i) {
            b->graphs.push_back(graphs[i]);
            b->configs.push_back(configs[i]);
            b->outs.push_back(device_scores[i]);
            ++graphs[i]->batch_refs;
        }
        capture(b.get());
        *out = b.release();
    });
}

tgtp_status tgtp_batch_run(tgtp_batch* b, void* cuda_stream) {
    return guarded([&] {
        if (!b) fail(TGTP_ERR_INVALID_ARGUMENT, "null batch");
        cudaStream_t s = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : b->origin;
        TGTP_CUDA(cudaGraphLaunch(b->exec, s));
        b->last = s;
        for (tgtp_graph* g : b->graphs) g->have_run = true;
    });
}

tgtp_status tgtp_batch_wait(tgtp_batch* b) {
    return guarded([&] {
        if (!b) fail(TGTP_ERR_INVALID_ARGUMENT, "null batch");
        if (b->last) TGTP_CUDA(cudaStreamSynchronize(b->last));
        for (tgtp_graph* g : b->graphs) aesc_check_flags(g);
    });
}

tgtp_status tgtp_batch_free(tgtp_batch* b) {
    return guarded([&] { delete b; });
}

}  // extern "C"
