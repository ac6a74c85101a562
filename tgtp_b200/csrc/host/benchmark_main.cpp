// Drop-in for the reference's `benchmark` executable (src/benchmark.cpp:9-53).
//
//   benchmark dataset [eps_csv=0.05,0.01,0.005] [threads_csv=1,2,4,8,16] [repeats=3]
//             [data_root=datasets] [omega=128] [gamma=10] [warmups=1]
//
// Prints the reference's TSV (sampler, dataset, epsilon, threads, repeat, seconds, checksum) with
// one row per timed tgtp() call, after `warmups` untimed calls per (epsilon, threads) pair.
// `seconds` covers tgtp() alone: the graph and eigenpairs are loaded and resident first, as the
// reference excludes loading.  The threads column is carried for format compatibility; the GPU
// run does not depend on it.  Errors: exit 1 with "benchmark: <message>".
#include <chrono>
#include <cmath>
#include <cstdint>
#include <filesystem>
#include <iomanip>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cli.hpp"
#include "tgtp_aesc.hpp"

namespace {

constexpr const char* kSampler = "seed32-grid-multiply-high";

struct Plan {
    std::string dataset, root = "datasets";
    std::vector<std::string> eps, threads;  // as typed: the TSV echoes the thread items verbatim
    uint32_t repeats = 3, warmups = 1;
    int omega = 128, gamma = 10;
};

// Argument i of argv, or `fallback` when the command line is shorter.
const char* arg(int argc, char** argv, int i, const char* fallback) {
    return argc > i ? argv[i] : fallback;
}

// The checks run in the reference's order, so the first bad argument is the one reported.
Plan read_plan(int argc, char** argv) {
    using namespace tgtp_cli;
    Plan plan;
    plan.dataset = argv[1];
    plan.eps = csv_items(arg(argc, argv, 2, "0.05,0.01,0.005"));
    plan.threads = csv_items(arg(argc, argv, 3, "1,2,4,8,16"));
    plan.repeats = bench_positive(arg(argc, argv, 4, "3"));
    const double warmups = bench_number(arg(argc, argv, 8, "1"));
    if (!integral_in(warmups, 0, INT32_MAX)) throw std::invalid_argument("invalid warmups");
    plan.warmups = uint32_t(warmups);
    plan.root = arg(argc, argv, 5, "datasets");
    plan.omega = int(bench_positive(arg(argc, argv, 6, "128")));
    plan.gamma = int(bench_positive(arg(argc, argv, 7, "10")));
    return plan;
}

// Sum of the scores in CSR order; a non-finite score is an error.
double checksum(const float* scores, size_t m) {
    double sum = 0;
    for (size_t q = 0; q < m; ++q) {
        if (!std::isfinite(scores[q])) throw std::runtime_error("nonfinite score");
        sum += scores[q];
    }
    return sum;
}

void measure(const Plan& plan) {
    using namespace tgtp_b200;
    AESCConfig config{};
    config.strFolder = plan.root;
    config.strGraph = plan.dataset;
    config.omega = plan.omega;
    config.gamma = plan.gamma;
    config.precision = precision_from_env();
    config.vec_dtype = vectors_from_env(config.precision);
    std::vector<double> eps;
    for (const auto& e : plan.eps) {
        eps.push_back(tgtp_cli::bench_number(e));
        if (!(eps.back() > 0 && eps.back() < 1))
            throw std::invalid_argument("epsilon must be between zero and one");
    }
    for (const auto& t : plan.threads) (void)tgtp_cli::bench_positive(t);

    const auto dir = std::filesystem::path(plan.root) / plan.dataset;
    const auto eigens = dir / ("sorted_eigens_" + std::to_string(plan.omega) + ".txt");
    AESCGraph graph((dir / "graph.txt").string(), eigens.string(), size_t(plan.omega), config.precision,
                    config.vec_dtype);
    config.delta = 1.0 / double(graph.n);

    std::cout << std::setprecision(10) << std::unitbuf;
    std::cout << "sampler\tdataset\tepsilon\tthreads\trepeat\tseconds\tchecksum\n";
    for (const double e : eps) {
        config.epsilon = e;
        for (const auto& t : plan.threads) {
            const uint64_t calls = uint64_t(plan.warmups) + plan.repeats;
            for (uint64_t call = 0; call < calls; ++call) {
                AESC run(graph, config);
                const auto t0 = std::chrono::steady_clock::now();
                const std::unique_ptr<float[]> scores(run.tgtp());
                const std::chrono::duration<double> took = std::chrono::steady_clock::now() - t0;
                const double sum = checksum(scores.get(), graph.m);
                if (call < plan.warmups) continue;
                std::cout << kSampler << '\t' << plan.dataset << '\t' << e << '\t' << t << '\t'
                          << call - plan.warmups << '\t' << took.count() << '\t' << sum << '\n';
            }
        }
    }
    graph.free();
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2 || argc > 9) {
        std::cerr << "Usage: benchmark dataset [eps_csv=0.05,0.01,0.005] [threads_csv=1,2,4,8,16]"
                     " [repeats=3] [data_root=datasets] [omega=128] [gamma=10] [warmups=1]\n";
        return 1;
    }
    try {
        measure(read_plan(argc, argv));
    } catch (const std::exception& e) {
        std::cerr << "benchmark: " << e.what() << '\n';
        return 1;
    }
    return 0;
}
