// tgtp_aesc.hpp — header-only C++ mirror of the reference's AESC interface (src/aesc.h:83-127)
// over the C ABI of libtgtp_gpu (tgtp_gpu.h).  A C++ caller of the reference switches by including
// this header instead of "aesc.h" and linking -ltgtp_gpu:
//
//   AESCGraph graph(graph_path, eigen_path, omega);     // src/aesc.h:85-92
//   AESCConfig config{}; ... config.delta = 1.0 / graph.n;
//   AESC algo(graph, config);
//   std::unique_ptr<float[]> scores(algo.tgtp());       // caller owns new float[m], as before
//
// Errors are thrown as std::runtime_error / std::invalid_argument with the reference's messages.
// The arithmetic form is AESCConfig::precision (default: the reference's own FP32 arithmetic) or,
// for the CLIs, the TGTP_PRECISION environment variable (fp32 | fp64 | mixed).
#pragma once

#include <cstdint>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "tgtp_gpu.h"

namespace tgtp_b200 {

inline void check(tgtp_status s) {
    if (s == TGTP_OK) return;
    const std::string msg = tgtp_last_error();
    if (s == TGTP_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

inline int precision_from_env(int fallback = TGTP_PRECISION_FP32) {
    const char* p = std::getenv("TGTP_PRECISION");
    if (!p || !*p) return fallback;
    const std::string s(p);
    if (s == "fp32") return TGTP_PRECISION_FP32;
    if (s == "fp64") return TGTP_PRECISION_FP64;
    if (s == "mixed") return TGTP_PRECISION_MIXED;
    throw std::invalid_argument("TGTP_PRECISION must be fp32, fp64 or mixed");
}

// Device storage of the eigenvectors for the command-line runners: TGTP_VECTORS=f32 (default) |
// bf16.  BF16 storage is read by the mixed form only, so it is refused with any other form.
inline int vectors_from_env(int precision) {
    const char* p = std::getenv("TGTP_VECTORS");
    if (!p || !*p || std::string(p) == "f32") return TGTP_VEC_F32;
    if (std::string(p) != "bf16") throw std::invalid_argument("TGTP_VECTORS must be f32 or bf16");
    if (precision != TGTP_PRECISION_MIXED)
        throw std::invalid_argument("TGTP_VECTORS=bf16 needs TGTP_PRECISION=mixed");
    return TGTP_VEC_BF16;
}

// CSR as fuser::graph_t<uint32_t, uint32_t> builds it (src/graph.h:10-98), resident on the device.
struct Graph {
    std::vector<uint32_t> idx, adj;  // host copies, same layout as graph_t::idx / graph_t::adj
    size_t n = 0, m = 0;
    tgtp_graph* handle = nullptr;

    Graph() = default;
    Graph(const Graph&) = delete;
    Graph& operator=(const Graph&) = delete;
    ~Graph() { free(); }

    uint32_t degree(uint32_t v) const { return idx[v + 1] - idx[v]; }

    void load_txt(const std::string& path) {
        uint32_t *i = nullptr, *a = nullptr;
        uint64_t n64 = 0, m64 = 0;
        check(tgtp_load_graph_txt(path.c_str(), &i, &a, &n64, &m64));
        idx.assign(i, i + n64 + 1);
        adj.assign(a, a + m64);
        tgtp_host_free(i);
        tgtp_host_free(a);
        n = n64;
        m = m64;
        check(tgtp_graph_upload(idx.data(), adj.data(), n, m, &handle));
    }
    void free() {
        if (handle) tgtp_graph_free(handle);
        handle = nullptr;
    }
};

// src/aesc.h:83-97: CSR + omega eigenpairs, validated as the reference does.
struct AESCGraph : Graph {
    size_t omega = 0;
    // vec_store: device storage of FP32/mixed-form vectors (TGTP_VEC_F32, or TGTP_VEC_BF16 for
    // the mixed form); the FP64 form always stores FP64
    AESCGraph(const std::string& graph_path, const std::string& eigen_path, size_t omega_,
              int precision = TGTP_PRECISION_FP32, int vec_store = TGTP_VEC_F32)
        : omega(omega_) {
        load_txt(graph_path);
        if (omega < 2 || omega > n) throw std::runtime_error("omega must be between 2 and vertex count");
        for (size_t v = 0; v < n; ++v)
            if (degree(uint32_t(v)) == 0)
                throw std::runtime_error("graph vertex IDs must be contiguous with no isolated vertices");
        std::vector<double> values(omega);
        const bool f64 = precision == TGTP_PRECISION_FP64;
        std::vector<float> v32(f64 ? 0 : n * omega);
        std::vector<double> v64(f64 ? n * omega : 0);
        check(tgtp_load_eigens_txt(eigen_path.c_str(), n, uint32_t(omega), values.data(),
                                   f64 ? nullptr : v32.data(), f64 ? v64.data() : nullptr));
        if (f64)
            check(tgtp_eigens_upload(handle, values.data(), v64.data(), uint32_t(omega),
                                     TGTP_VEC_F64, TGTP_VEC_F64));
        else
            check(tgtp_eigens_upload(handle, values.data(), v32.data(), uint32_t(omega),
                                     TGTP_VEC_F32, vec_store));
    }
};

// src/aesc.h:98-102 plus the arithmetic form.
struct AESCConfig {
    double epsilon = 0, delta = 0;
    std::string strFolder, strGraph;
    int omega = 0, gamma = 0;
    int precision = TGTP_PRECISION_FP32;
    int vec_dtype = TGTP_VEC_F32;  // storage the mixed form reads (TGTP_VEC_F32 or TGTP_VEC_BF16)
};

// src/aesc.h:113-127
struct AESC {
    AESCGraph& g;
    AESCConfig& config;
    AESC(AESCGraph& g_, AESCConfig& config_) : g(g_), config(config_) {}
    // Returns new float[m] (CSR order, symmetric); the caller owns it, as with the reference.
    float* tgtp() {
        std::unique_ptr<float[]> out(new float[g.m]);
        tgtp_config c{};
        c.epsilon = config.epsilon;
        c.delta = config.delta;
        c.omega = config.omega;
        c.gamma = config.gamma;
        c.precision = config.precision;
        c.vec_dtype = config.vec_dtype;
        check(tgtp_run(g.handle, &c, out.get()));
        return out.release();
    }
};

}  // namespace tgtp_b200
