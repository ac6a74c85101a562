// Test infrastructure only (the checker, never the product): a driver around
// the reference's own SABA walk routine, compiled from the reference source
// file where it lies.  The reference runner (src/rw_experiment_saba.cpp:147-247)
// prints visit_count/checksum at 6 significant digits only; this driver calls
// the same static saba_randomwalk (src/rw_experiment_saba.cpp:65-145) on every
// source, single-threaded so the reference's float counters (:192) stay exact,
// and dumps the whole per-vertex counter array.
//
// usage: ref_saba_harness <graph.txt> <depth> <n_walks> <counts_out.u32>
//   prints "n m visit_count checksum" (integers, exact) on stdout.
#define main tgtp_reference_saba_runner_main
#include "rw_experiment_saba.cpp"
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
    if (n_walks % 8 != 0 || n_walks > UINT32_MAX) {
      std::fprintf(stderr, "n_walks must be a multiple of 8\n");
      return 1;
    }
    std::vector<float> counters(g.n, 0.0f);
    for (size_t src = 0; src < g.n; ++src) {
      if (g.degree((uint32_t)src) == 0) continue;
      if (n_walks > 0) saba_randomwalk((uint32_t)src, depth, n_walks, counters.data(), g);
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
    std::fprintf(stderr, "ref_saba_harness: %s\n", e.what());
    return 1;
  }
  return 0;
}
