// Drop-in for the reference's `rw_experiment_saba` (src/rw_experiment_saba.cpp:147-247): same argv,
// same results/rw/saba_<dataset>_d<D>_w<W>.txt keys and the same TSV row.  t_load_s covers reading
// graph.txt and placing the CSR on the device; t_rw_s covers zeroing the counters, every walk and
// the visit_count / checksum reduction (the reference's timed scope).  The counters are exact
// integers; visit_count and checksum are printed as doubles as the reference prints them.
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <string>

#include "tgtp_aesc.hpp"

namespace fs = std::filesystem;
static const char* const VARIANT = "saba";

int main(int argc, char** argv) {
    if (argc < 5) {
        std::cerr << "Usage: " << argv[0] << " <datasets_folder> <dataset> <depth> <n_walks> [threads]\n";
        return 1;
    }
    const std::string folder = argv[1];
    const std::string dataset = argv[2];
    const size_t depth = std::strtoull(argv[3], nullptr, 10);
    const size_t n_walks = std::strtoull(argv[4], nullptr, 10);
    if (n_walks % 8 != 0 || n_walks > UINT32_MAX) {
        std::cerr << "n_walks must be a multiple of 8 within the 32-bit grid domain\n";
        return 1;
    }
    int threads = (argc > 5) ? std::atoi(argv[5]) : 1;
    if (threads < 1) threads = 1;
    try {
        const fs::path graph_path = fs::path(folder) / dataset / "graph.txt";
        tgtp_b200::Graph g;
        auto t0 = std::chrono::high_resolution_clock::now();
        g.load_txt(graph_path.string());
        auto t1 = std::chrono::high_resolution_clock::now();
        const double t_load = std::chrono::duration<double>(t1 - t0).count();
        const size_t n = g.n, m = g.m;

        auto t2 = std::chrono::high_resolution_clock::now();
        saba_result res{};
        tgtp_b200::check(saba_count(g.handle, uint32_t(depth), uint32_t(n_walks), nullptr, &res));
        auto t3 = std::chrono::high_resolution_clock::now();
        const double t_rw = std::chrono::duration<double>(t3 - t2).count();
        const double total = std::chrono::duration<double>(t3 - t0).count();
        const double total_walks = (double)n * (double)n_walks * (double)depth;
        const double walks_per_sec = (t_rw > 0.0) ? (total_walks / t_rw) : 0.0;
        const double visit_count = double(res.visit_count);
        const double checksum = double(res.checksum);
        g.free();

        fs::create_directories("results/rw");
        const std::string resfile = "results/rw/" + std::string(VARIANT) + "_" + dataset + "_d" +
                                    std::to_string(depth) + "_w" + std::to_string(n_walks) + ".txt";
        {
            std::ofstream out(resfile);
            out << "variant " << VARIANT << "\n";
            out << "dataset " << dataset << "\n";
            out << "depth " << depth << "\n";
            out << "n_walks " << n_walks << "\n";
            out << "threads " << threads << "\n";
            out << "n_vertices " << n << "\n";
            out << "n_edges " << m << "\n";
            out << "t_load_s " << t_load << "\n";
            out << "t_rw_s " << t_rw << "\n";
            out << "total_s " << total << "\n";
            out << "total_walks " << total_walks << "\n";
            out << "walks_per_sec " << walks_per_sec << "\n";
            out << "visit_count " << visit_count << "\n";
            out << "checksum " << checksum << "\n";
        }
        std::cout << VARIANT << "\t" << dataset << "\t" << depth << "\t" << n_walks << "\t" << threads
                  << "\t" << n << "\t" << m << "\t" << t_load << "\t" << t_rw << "\t" << total << "\t"
                  << total_walks << "\t" << walks_per_sec << "\t" << visit_count << "\t" << checksum
                  << "\n";
    } catch (const std::exception& e) {
        std::cerr << "rw_experiment_saba: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
