// Test infrastructure only (the checker): dumps what the reference's own loaders build, compiled
// from the reference headers where they lie.
//   ref_load_dump graph <graph.txt> <out_prefix>          -> <prefix>.idx.u32, <prefix>.adj.u32
//       (fuser::graph_t::load_txt, src/graph.h:29-97)
//   ref_load_dump eigens <graph.txt> <eigens.txt> <omega> <out_prefix>
//       -> <prefix>.values.f64, <prefix>.vectors.f32   (AESCGraph, src/aesc.h:85-92 and :51-64)
// On a loader exception it prints "ERROR <what>" and exits 3.
#include "aesc.h"

#include <cstdio>

static void dump(const std::string& path, const void* p, size_t bytes) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f || std::fwrite(p, 1, bytes, f) != bytes) throw std::runtime_error("cannot write " + path);
  std::fclose(f);
}

int main(int argc, char** argv) {
  try {
    const std::string mode = argc > 1 ? argv[1] : "";
    if (mode == "graph" && argc == 4) {
      fuser::graph_t<uint32_t, uint32_t> g;
      g.load_txt(argv[2]);
      dump(std::string(argv[3]) + ".idx.u32", g.idx, sizeof(uint32_t) * (g.n + 1));
      dump(std::string(argv[3]) + ".adj.u32", g.adj, sizeof(uint32_t) * g.m);
      std::printf("%zu %zu\n", g.n, g.m);
      g.free();
      return 0;
    }
    if (mode == "eigens" && argc == 6) {
      AESCGraph g(argv[2], argv[3], std::strtoull(argv[4], nullptr, 10));
      dump(std::string(argv[5]) + ".values.f64", g.eigens.values, sizeof(double) * g.eigens.omega);
      dump(std::string(argv[5]) + ".vectors.f32", g.eigens.vectors,
           sizeof(float) * g.eigens.omega * g.n);
      std::printf("%zu %zu\n", g.n, g.eigens.omega);
      g.free();
      return 0;
    }
  } catch (const std::exception& e) {
    std::printf("ERROR %s\n", e.what());
    return 3;
  }
  std::fprintf(stderr, "usage: ref_load_dump graph <graph.txt> <prefix> | eigens <graph.txt> <eigens.txt> <omega> <prefix>\n");
  return 1;
}
