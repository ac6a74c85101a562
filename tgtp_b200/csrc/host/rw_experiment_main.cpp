// Drop-in for the reference's MT19937 walk runners: `rw_experiment` (src/rw_experiment.cpp:49-152)
// and, built with -DTGTP_MT_SIMD, `rw_experiment_simd` (src/rw_experiment_simd.cpp:85-191).
//
//   rw_experiment[_simd] <datasets_folder> <dataset> <depth> <n_walks> [threads]
//
// Counts the visits of n_walks walks of `depth` hops from every vertex of
// <datasets_folder>/<dataset>/graph.txt on the GPU (std::mt19937 reseeded to 42 + src, the
// runner's draw order), writes results/rw/<variant>_<dataset>_d<D>_w<W>.txt ("key value" lines)
// and prints the same values as one TSV row.  t_load_s covers reading graph.txt and placing the
// CSR on the device; t_rw_s covers zeroing the counters, every walk and the visit_count / checksum
// reduction (the reference's timed scope).  The counters are exact integers; visit_count and
// checksum are printed as doubles, as the reference prints them.  `threads` is echoed for format
// compatibility.
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <string>

#include "cli.hpp"
#include "tgtp_aesc.hpp"

namespace {

#ifdef TGTP_MT_SIMD
constexpr const char* kVariant = "simd";
constexpr int32_t kSimd = 1;
#else
constexpr const char* kVariant = "regular";
constexpr int32_t kSimd = 0;
#endif

struct Walks {
    std::string folder, dataset;
    size_t depth = 0, n_walks = 0;
    int threads = 1;
};

double seconds_between(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
}

void count_walks(const Walks& w) {
    using clock = std::chrono::steady_clock;
    tgtp_b200::Graph g;
    const auto t_start = clock::now();
    g.load_txt((std::filesystem::path(w.folder) / w.dataset / "graph.txt").string());
    const auto t_loaded = clock::now();
    saba_result res{};
    tgtp_b200::check(mt_walk_count(g.handle, uint32_t(w.depth), uint32_t(w.n_walks), kSimd, nullptr, &res));
    const auto t_walked = clock::now();
    const size_t n = g.n, m = g.m;
    g.free();

    const double t_load = seconds_between(t_start, t_loaded);
    const double t_rw = seconds_between(t_loaded, t_walked);
    const double walks = double(n) * double(w.n_walks) * double(w.depth);
    tgtp_cli::Record rec;
    rec.add("variant", kVariant)
        .add("dataset", w.dataset)
        .add("depth", w.depth)
        .add("n_walks", w.n_walks)
        .add("threads", w.threads)
        .add("n_vertices", n)
        .add("n_edges", m)
        .add("t_load_s", t_load)
        .add("t_rw_s", t_rw)
        .add("total_s", seconds_between(t_start, t_walked))
        .add("total_walks", walks)
        .add("walks_per_sec", t_rw > 0 ? walks / t_rw : 0.0)
        .add("visit_count", double(res.visit_count))
        .add("checksum", double(res.checksum));

    const std::filesystem::path dir = "results/rw";
    std::filesystem::create_directories(dir);
    const std::string file = std::string(kVariant) + "_" + w.dataset + "_d" + std::to_string(w.depth) +
                             "_w" + std::to_string(w.n_walks) + ".txt";
    {
        std::ofstream out(dir / file);
        rec.write_lines(out);
    }
    rec.write_row(std::cout);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 5) {
        std::cerr << "Usage: " << argv[0] << " <datasets_folder> <dataset> <depth> <n_walks> [threads]\n";
        return 1;
    }
    Walks w;
    w.folder = argv[1];
    w.dataset = argv[2];
    w.depth = std::strtoull(argv[3], nullptr, 10);
    w.n_walks = std::strtoull(argv[4], nullptr, 10);
#ifdef TGTP_MT_SIMD
    if (w.n_walks % 8 != 0) {  // whole bouquets of 8 walks (src/rw_experiment_simd.cpp:97-100)
        std::cerr << "n_walks must be a multiple of 8\n";
        return 1;
    }
#endif
    if (w.n_walks > UINT32_MAX || w.depth > UINT32_MAX) {
        std::cerr << "depth and n_walks must fit in 32 bits\n";
        return 1;
    }
    w.threads = argc > 5 ? std::atoi(argv[5]) : 1;
    if (w.threads < 1) w.threads = 1;
    try {
        count_walks(w);
    } catch (const std::exception& e) {
        std::cerr << (kSimd ? "rw_experiment_simd: " : "rw_experiment: ") << e.what() << '\n';
        return 1;
    }
    return 0;
}
