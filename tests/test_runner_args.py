"""The drop-in executables' argument handling on the CPU: every rejected command line exits 1 with
the reference runner's message (src/main.cpp:9-31, src/benchmark.cpp:10-28 with
src/benchmark_options.h, src/rw_experiment_saba.cpp:150-163, src/rw_experiment.cpp:52-57,
src/rw_experiment_simd.cpp:88-100), checked before any device work.
The expected messages are pinned here; where the reference binaries built under oracle/_ref are
present (the -O2 parity builds for tgtp and benchmark: the -Ofast build drops tgtp's isfinite
test), each case is also run through them and must give the same exit code and output."""
from __future__ import annotations

import os
import subprocess

import pytest

from conftest import ROOT

BIN = os.path.join(ROOT, "tgtp_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")
REQUIRE = "tgtp: require 0 < epsilon < 1, integer omega >= 2, integer gamma >= 1"
BENCH_USAGE = ("Usage: benchmark dataset [eps_csv=0.05,0.01,0.005] [threads_csv=1,2,4,8,16]"
               " [repeats=3] [data_root=datasets] [omega=128] [gamma=10] [warmups=1]")

TGTP_CASES = [
    (["x", "y", "1.5", "16", "10", "o"], REQUIRE),
    (["x", "y", "0", "16", "10", "o"], REQUIRE),
    (["x", "y", "abc", "16", "10", "o"], "tgtp: stod"),
    (["x", "y", "0.05x", "16", "10", "o"], "tgtp: invalid numeric argument"),
    (["x", "y", "inf", "16", "10", "o"], "tgtp: invalid numeric argument"),
    (["x", "y", "nan", "16", "10", "o"], "tgtp: invalid numeric argument"),
    (["x", "y", "1e999", "16", "10", "o"], "tgtp: stod"),
    (["x", "y", "0.05", "2.5", "10", "o"], REQUIRE),
    (["x", "y", "0.05", "1", "10", "o"], REQUIRE),
    (["x", "y", "0.05", "16", "0", "o"], REQUIRE),
    (["x", "y", "0.05", "16", "3e9", "o"], REQUIRE),
    (["x", "y", "0.05", "16", "10x", "o"], "tgtp: invalid numeric argument"),
    (["nofolder", "g", "0.05", "16", "10", "o"], "tgtp: cannot open graph: nofolder/g/graph.txt"),
]

BENCH_CASES = [
    (["a", "b", "c", "d", "e", "f", "g", "h", "i"], BENCH_USAGE),
    (["ds", ""], "benchmark: empty CSV list/item"),
    (["ds", "0.05,,0.01"], "benchmark: empty CSV item"),
    (["ds", "0.05,"], "benchmark: empty CSV list/item"),
    (["ds", ","], "benchmark: empty CSV item"),
    (["ds", ",0.05"], "benchmark: empty CSV item"),
    (["ds", "1.5"], "benchmark: epsilon must be between zero and one"),
    (["ds", "0.05,0"], "benchmark: epsilon must be between zero and one"),
    (["ds", "0.05x"], "benchmark: invalid number: 0.05x"),
    (["ds", "inf"], "benchmark: invalid number: inf"),
    (["ds", "0.05", "1,x"], "benchmark: stod"),
    (["ds", "0.05", "1,0"], "benchmark: invalid positive integer: 0"),
    (["ds", "0.05", "1", "0"], "benchmark: invalid positive integer: 0"),
    (["ds", "0.05", "1", "2.5"], "benchmark: invalid positive integer: 2.5"),
    (["ds", "0.05", "1", "2", "r", "16", "10", "-1"], "benchmark: invalid warmups"),
    (["ds", "0.05", "1", "2", "r", "16", "10", "0.5"], "benchmark: invalid warmups"),
    (["ds", "0.05", "1", "2", "r", "1.5"], "benchmark: invalid positive integer: 1.5"),
    (["ds", "0.05", "1", "2", "r", "16", "0"], "benchmark: invalid positive integer: 0"),
    (["ds", "0.05", "1", "2", "nofolder", "16", "10", "1"],
     "benchmark: cannot open graph: nofolder/ds/graph.txt"),
]

SABA_MULTIPLE = "n_walks must be a multiple of 8 within the 32-bit grid domain"
SABA_CASES = [
    (["f", "d", "5", "12"], SABA_MULTIPLE),
    (["f", "d", "5", "8589934592"], SABA_MULTIPLE),
    (["f", "d", "5", "4294967304", "4"], SABA_MULTIPLE),
]


MT_SIMD_CASES = [
    (["f", "d", "5", "12"], "n_walks must be a multiple of 8"),
    (["f", "d", "5", "4", "4"], "n_walks must be a multiple of 8"),
]


@pytest.fixture(scope="module")
def runners(tgtp_lib):
    from tgtp_b200 import build

    build.build(runners=True)
    return BIN


def _run(exe, args, cwd):
    r = subprocess.run([exe] + args, capture_output=True, text=True, cwd=cwd, timeout=60)
    return r.returncode, r.stdout, r.stderr.strip()


def _check(runners, tmp_path, name, ref_name, args, message):
    rc, out, err = _run(os.path.join(runners, name), args, tmp_path)
    assert (rc, out, err) == (1, "", message), args
    ref = os.path.join(REF, ref_name)
    if os.path.exists(ref):
        assert _run(ref, args, tmp_path) == (rc, out, err), args


@pytest.mark.parametrize("args,message", TGTP_CASES)
def test_tgtp_rejects_like_the_reference(runners, tmp_path, args, message):
    _check(runners, tmp_path, "tgtp", "tgtp_O2", args, message)


@pytest.mark.parametrize("args,message", BENCH_CASES)
def test_benchmark_rejects_like_the_reference(runners, tmp_path, args, message):
    _check(runners, tmp_path, "benchmark", "benchmark_O2", args, message)


@pytest.mark.parametrize("args,message", SABA_CASES)
def test_rw_experiment_saba_rejects_like_the_reference(runners, tmp_path, args, message):
    _check(runners, tmp_path, "rw_experiment_saba", "rw_experiment_saba", args, message)


@pytest.mark.parametrize("args,message", MT_SIMD_CASES)
def test_rw_experiment_simd_rejects_like_the_reference(runners, tmp_path, args, message):
    _check(runners, tmp_path, "rw_experiment_simd", "rw_experiment_simd", args, message)


@pytest.mark.parametrize("name,args", [("tgtp", []), ("tgtp", ["a"] * 7), ("benchmark", []),
                                       ("rw_experiment_saba", ["f", "d", "5"]),
                                       ("rw_experiment", ["f", "d", "5"]),
                                       ("rw_experiment_simd", [])])
def test_usage_lines(runners, tmp_path, name, args):
    exe = os.path.join(runners, name)
    rc, out, err = _run(exe, args, tmp_path)
    assert rc == 1 and out == ""
    if name == "tgtp":
        assert err == f"Usage: {exe} <folder> <graph> <epsilon> <omega> <gamma> <outfile>"
    elif name == "benchmark":
        assert err == BENCH_USAGE
    else:
        assert err == f"Usage: {exe} <datasets_folder> <dataset> <depth> <n_walks> [threads]"
    ref = os.path.join(REF, {"tgtp": "tgtp_O2", "benchmark": "benchmark_O2"}.get(name, name))
    if os.path.exists(ref):
        rrc, rout, rerr = _run(ref, args, tmp_path)
        assert (rrc, rout, rerr.replace(ref, exe)) == (rc, out, err)


@pytest.mark.parametrize("name", ["rw_experiment_saba", "rw_experiment", "rw_experiment_simd"])
def test_walk_runners_report_an_unreadable_graph(runners, tmp_path, name):
    # the reference lets this exception escape (the process aborts); here it is a message and exit 1
    rc, out, err = _run(os.path.join(runners, name), ["nofolder", "ds", "5", "16"], tmp_path)
    assert (rc, out, err) == (1, "", f"{name}: cannot open graph: nofolder/ds/graph.txt")


@pytest.mark.parametrize("name", ["rw_experiment", "rw_experiment_simd"])
def test_mt_walk_runners_refuse_counts_beyond_32_bits(runners, tmp_path, name):
    """The reference would start 2^33 walks per vertex; the GPU runners take 32-bit counts."""
    rc, out, err = _run(os.path.join(runners, name), ["f", "d", "5", "8589934592"], tmp_path)
    assert (rc, out, err) == (1, "", "depth and n_walks must fit in 32 bits")


@pytest.mark.parametrize("name,args", [("tgtp", ["x", "y", "0.05", "16", "10", "o"]),
                                       ("benchmark", ["ds", "0.05", "1", "1", "nofolder"])])
@pytest.mark.parametrize("env,message", [
    ({"TGTP_PRECISION": "fp16"}, "TGTP_PRECISION must be fp32, fp64 or mixed"),
    ({"TGTP_VECTORS": "bf16"}, "TGTP_VECTORS=bf16 needs TGTP_PRECISION=mixed"),
    ({"TGTP_VECTORS": "bf16", "TGTP_PRECISION": "fp64"}, "TGTP_VECTORS=bf16 needs TGTP_PRECISION=mixed"),
    ({"TGTP_VECTORS": "fp8", "TGTP_PRECISION": "mixed"}, "TGTP_VECTORS must be f32 or bf16"),
])
def test_runner_form_variables_are_checked_before_loading(runners, tmp_path, name, args, env,
                                                          message):
    """The arithmetic form (TGTP_PRECISION) and the mixed form's vector storage (TGTP_VECTORS)
    of the runners: a bad choice is reported before any input is read."""
    r = subprocess.run([os.path.join(runners, name)] + args, capture_output=True, text=True,
                       cwd=tmp_path, timeout=60, env=dict(os.environ, **env))
    assert (r.returncode, r.stdout, r.stderr.strip()) == (1, "", f"{name}: {message}")
