// Drop-in for the reference's `tgtp` executable (src/main.cpp:8-50).
//
//   tgtp <folder> <graph> <epsilon> <omega> <gamma> <outfile>
//
// Reads <folder>/<graph>/graph.txt and sorted_eigens_<omega>.txt, scores every CSR slot on the GPU
// and writes the m scores as raw native-endian float32 in CSR order.  Exit 0, or 1 with
// "tgtp: <message>" on stderr (argument errors as the reference words them, tgtp_cli).
// Arithmetic form: TGTP_PRECISION=fp32 (default, the reference's arithmetic) | fp64 | mixed; with
// mixed, TGTP_VECTORS=bf16 stores the eigenvectors as BF16 (default f32).
#include <climits>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>

#include "cli.hpp"
#include "tgtp_aesc.hpp"

namespace {

struct Job {
    std::string folder, graph, outfile;
    double epsilon = 0;
    int omega = 0, gamma = 0;
};

// argv[1..6]; the three numbers are read in order before any of them is range-checked.
Job read_job(char** argv) {
    const std::string complaint = "invalid numeric argument";
    Job job;
    job.folder = argv[1];
    job.graph = argv[2];
    job.outfile = argv[6];
    job.epsilon = tgtp_cli::whole_number(argv[3], complaint);
    const double omega = tgtp_cli::whole_number(argv[4], complaint);
    const double gamma = tgtp_cli::whole_number(argv[5], complaint);
    const bool ok = job.epsilon > 0 && job.epsilon < 1 && tgtp_cli::integral_in(omega, 2, INT_MAX) &&
                    tgtp_cli::integral_in(gamma, 1, INT_MAX);
    if (!ok)
        throw std::invalid_argument("require 0 < epsilon < 1, integer omega >= 2, integer gamma >= 1");
    job.omega = int(omega);
    job.gamma = int(gamma);
    return job;
}

void score(const Job& job) {
    using namespace tgtp_b200;
    AESCConfig config{};
    config.strFolder = job.folder;
    config.strGraph = job.graph;
    config.epsilon = job.epsilon;
    config.omega = job.omega;
    config.gamma = job.gamma;
    config.precision = precision_from_env();
    config.vec_dtype = vectors_from_env(config.precision);
    const auto dir = std::filesystem::path(job.folder) / job.graph;
    const auto eigens = dir / ("sorted_eigens_" + std::to_string(job.omega) + ".txt");
    AESCGraph graph((dir / "graph.txt").string(), eigens.string(), size_t(job.omega), config.precision,
                    config.vec_dtype);
    config.delta = 1.0 / double(graph.n);
    // the output file is opened once the inputs have loaded, so an input error leaves no file
    std::ofstream sink(job.outfile, std::ios::binary);
    if (!sink) throw std::runtime_error("cannot open output file");
    AESC run(graph, config);
    const std::unique_ptr<float[]> scores(run.tgtp());
    sink.write(reinterpret_cast<const char*>(scores.get()),
               std::streamsize(graph.m * sizeof(float)));
    sink.close();
    if (!sink) throw std::runtime_error("failed to write output file");
    graph.free();
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 7) {
        std::cerr << "Usage: " << argv[0] << " <folder> <graph> <epsilon> <omega> <gamma> <outfile>\n";
        return 1;
    }
    try {
        score(read_job(argv));
    } catch (const std::exception& e) {
        std::cerr << "tgtp: " << e.what() << '\n';
        return 1;
    }
    return 0;
}
