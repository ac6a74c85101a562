// Test infrastructure only (the checker, never the product): a driver around the reference's own
// MT19937 walk routines, compiled from the reference source files where they lie.  The reference
// runners (src/rw_experiment.cpp:49-152, src/rw_experiment_simd.cpp:85-191) print visit_count and
// checksum at 6 significant digits only; this driver calls the same static walk routine
// (scalar_randomwalk, src/rw_experiment.cpp:34-47, or with -DTGTP_MT_SIMD simd_randomwalk,
// src/rw_experiment_simd.cpp:44-83) on every source with a neighbour, reseeding std::mt19937 with
// 42 + src as the runners do (:110), single-threaded so the float counters stay exact, and dumps
// the whole per-vertex counter array.
//
// usage: ref_mt_harness <graph.txt> <depth> <n_walks> <counts_out.u32>
//   prints "n m visit_count checksum" (integers, exact) on stdout.
#define main tgtp_reference_mt_runner_main
#ifdef TGTP_MT_SIMD
#include "rw_experiment_simd.cpp"
#define TGTP_WALK simd_randomwalk
#else
#include "rw_experiment.cpp"
#define TGTP_WALK scalar_randomwalk
#endif
#undef main

#include <cstdio>

int main(int argc, char** argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s <graph.txt> <depth> <n_walks> <counts_out.u32>\n", argv[0]);
    return 1;
  }
  try {
    fuser::graph_t<uint32_t, uint32_t> g;
    g.load_txt(argv[1]);
    const size_t depth = std::strtoull(argv[2], nullptr, 10);
    const size_t n_walks = std::strtoull(argv[3], nullptr, 10);
#ifdef TGTP_MT_SIMD
    if (n_walks % 8 != 0) {
      std::fprintf(stderr, "n_walks must be a multiple of 8\n");
      return 1;
    }
#endif
    std::vector<float> counters(g.n, 0.0f);
    std::mt19937 rng(42u);
    for (size_t src = 0; src < g.n; ++src) {
      if (g.degree((uint32_t)src) == 0) continue;
      rng.seed(42u + (uint32_t)src);
      if (n_walks > 0) TGTP_WALK((uint32_t)src, depth, n_walks, counters.data(), g, rng);
    }
    std::vector<uint32_t> out(g.n);
    unsigned long long visits = 0, checksum = 0;
    for (size_t v = 0; v < g.n; ++v) {
      if (counters[v] >= 16777216.0f) {
        std::fprintf(stderr, "float counter of vertex %zu reached 2^24; not exact\n", v);
        return 2;
      }
      out[v] = (uint32_t)counters[v];
      visits += out[v];
      checksum += (unsigned long long)(v + 1) * out[v];
    }
    FILE* f = std::fopen(argv[4], "wb");
    if (!f || std::fwrite(out.data(), sizeof(uint32_t), out.size(), f) != out.size()) {
      std::fprintf(stderr, "cannot write %s\n", argv[4]);
      return 1;
    }
    std::fclose(f);
    std::printf("%zu %zu %llu %llu\n", g.n, g.m, visits, checksum);
    g.free();
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_mt_harness: %s\n", e.what());
    return 1;
  }
  return 0;
}
