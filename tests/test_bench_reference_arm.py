"""bench.py's reference arm on the CPU: the reference's own `benchmark` binary timed on the host's
cores prints one JSON line with the bench contract's keys, and under a multi-rank launch only rank
0 does work."""
from __future__ import annotations

import json
import os
import subprocess
import sys

from conftest import ROOT


def _bench(*args, env=None):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        *args], capture_output=True, text=True, cwd=ROOT, timeout=600,
                       env=dict(os.environ, **(env or {})))
    assert r.returncode == 0, r.stderr[-2000:]
    return [line for line in r.stdout.splitlines() if line.startswith("{")]


def test_reference_arm_prints_the_contract_line():
    lines = _bench("--steps", "1", "--warmup", "3")
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:  # the reference binaries under oracle/_ref were not built here
        assert set(d) == {"impl", "unavailable"}
        return
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["unit"] == "edges/s" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert abs(d["ms_per_step"] * 1e-3 * d["value"] - 88234) < 1e-6 * 88234
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1
    assert cb["omp_num_threads"] == cb["cores"] and cb["cpu_model"]
    assert d["e2e"] == {"value": d["value"], "unit": "edges/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert "workload" in d["config"]
    # both arms print the same config dict (bench.bench_config), so they describe one workload
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert d["config"] == bench.bench_config(1)


def test_reference_arm_runs_on_rank_zero_only():
    assert _bench("--steps", "1", "--warmup", "3", env={"RANK": "1", "WORLD_SIZE": "2"}) == []


def test_cpu_baseline_line_reports_both_thread_counts():
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    # one sampling rule for the reference arm and cpu_baseline: the mean of the timed calls
    line = bench.cpu_baseline_line(1000, [0.5, 0.25, 0.25], 16, [2.0, 4.0], "sample")
    assert line["value"] == 1000 / (1.0 / 3.0) and line["cores"] == 16
    assert line["omp_num_threads"] == 16
    assert line["single_thread"]["value"] == 1000 / 3.0 and line["single_thread"]["cores"] == 1
    assert line["cpu_model"] and line["kind"] == "reference"
    assert "single_thread" not in bench.cpu_baseline_line(1000, [0.5], 16, None, "sample")


def test_saba_cpu_reference_counts_transitions_once(tmp_path):
    """The reference SABA runner's total_walks already counts every hop: the rate bench.py reports
    is n * W * D over the runner's own walk time, the fastest of the runs."""
    import importlib.util

    from tgtp_b200 import synth

    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    g = synth.rmat(12, 8, 0.57, 0.19, 0.19, 5)
    ref = bench.saba_cpu_reference(g, str(tmp_path), 5, 64, runs=2)
    if ref is None:  # the reference binaries under oracle/_ref were not built here
        return
    assert ref["transitions"] == g.n * 64 * 5
    assert ref["transitions_per_s"] == ref["transitions"] / ref["walk_seconds"]
