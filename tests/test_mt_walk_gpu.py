"""The MT19937 walk baselines on the GPU (mt_walk_count: src/rw_experiment.cpp:34-47 and
src/rw_experiment_simd.cpp:44-83, std::mt19937 reseeded to 42 + src) against the oracle's
restatement, which tests/test_oracle_golden.py pins to the reference's own walk routines: every
per-vertex counter equal, through the C ABI and through the drop-in runners."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _graph(name):
    from tgtp_b200 import synth

    return {"config1": lambda: synth.config1_graph(1),
            "rmat14": lambda: synth.rmat(14, 8, 0.57, 0.19, 0.19, 3),
            "rmat12": lambda: synth.rmat(12, 8, 0.57, 0.19, 0.19, 5)}[name]()


@pytest.mark.parametrize("simd", [False, True])
@pytest.mark.parametrize("graph,depth,walks", [("config1", 5, 2048), ("config1", 15, 16),
                                               ("rmat14", 10, 24), ("rmat12", 100, 8),
                                               ("rmat12", 700, 8), ("rmat12", 1, 8),
                                               ("rmat12", 5, 0), ("rmat12", 0, 8)])
def test_mt_walks_match_the_oracle(cuda_device, oracle_lib, simd, graph, depth, walks):
    """Walk lengths up to and beyond the 624-word generator block (100, 700): fewer walks then
    step side by side; zero walks or zero depth leave every counter at zero."""
    from tgtp_b200.aesc import AESCGraph, mt_walk_count

    g = _graph(graph)
    idx, adj = g.csr()
    dg = AESCGraph.from_csr(idx, adj)
    counts, visits, checksum = mt_walk_count(dg, depth, walks, simd=simd)
    dg.free()
    want = oracle_lib.mt_walks(idx, adj, depth, walks, simd=simd)
    assert np.array_equal(counts.astype(np.uint64), want)
    active = int((np.diff(idx.astype(np.int64)) > 0).sum())
    assert visits == active * walks * depth == int(want.sum())
    assert checksum == int((want * np.arange(1, g.n + 1, dtype=np.uint64)).sum())


@pytest.mark.parametrize("walks", [13, 32, 33])
def test_mt_scalar_walk_counts_need_not_be_whole_bouquets(cuda_device, oracle_lib, walks):
    from tgtp_b200.aesc import AESCGraph, mt_walk_count

    g = _graph("rmat12")
    idx, adj = g.csr()
    dg = AESCGraph.from_csr(idx, adj)
    counts, _, _ = mt_walk_count(dg, 7, walks)
    with pytest.raises(Exception):
        mt_walk_count(dg, 7, walks if walks % 8 else walks + 1, simd=True)
    dg.free()
    assert np.array_equal(counts.astype(np.uint64), oracle_lib.mt_walks(idx, adj, 7, walks))


@pytest.mark.parametrize("name,simd", [("rw_experiment", False), ("rw_experiment_simd", True)])
def test_mt_walk_runners_print_the_oracle_sums(cuda_device, oracle_lib, tmp_path, name, simd):
    """The drop-in runners on a dataset folder: the TSV row and the results file carry the
    reference's keys, and visit_count / checksum are the oracle's."""
    from conftest import ROOT
    from tgtp_b200 import build, synth

    build.build(runners=True)
    g = _graph("config1")
    os.makedirs(tmp_path / "ds" / "G")
    synth.write_graph_txt(g, str(tmp_path / "ds" / "G" / "graph.txt"))
    exe = os.path.join(ROOT, "tgtp_b200", "bin", name)
    r = subprocess.run([exe, "ds", "G", "5", "64", "4"], capture_output=True, text=True,
                       cwd=tmp_path, timeout=300)
    assert r.returncode == 0, r.stderr
    row = r.stdout.strip().split("\t")
    variant = "simd" if simd else "regular"
    assert row[:7] == [variant, "G", "5", "64", "4", str(g.n), str(int(g.csr()[0][-1]))]
    idx, adj = g.csr()
    want = oracle_lib.mt_walks(idx, adj, 5, 64, simd=simd)
    assert float(row[12]) == float(want.sum())
    assert float(row[13]) == pytest.approx(float((want * np.arange(1, g.n + 1, dtype=np.uint64)).sum()), rel=1e-5)
    lines = (tmp_path / "results" / "rw" / f"{variant}_G_d5_w64.txt").read_text().splitlines()
    assert [ln.split(" ")[0] for ln in lines] == [
        "variant", "dataset", "depth", "n_walks", "threads", "n_vertices", "n_edges", "t_load_s",
        "t_rw_s", "total_s", "total_walks", "walks_per_sec", "visit_count", "checksum"]


@pytest.mark.parametrize("case", range(8))
def test_mt_walks_match_the_committed_reference_counters(cuda_device, case):
    """The GPU walks against tests/golden/mt_walks.json (the reference's own walk routines, run by
    tests/golden/make_mt_walks.py): every counter, by SHA-256 of the array."""
    import json

    from conftest import GOLDEN
    from make_mt_walks import graph
    from make_saba_rmat18 import graph_fingerprint, sha256_u32

    from tgtp_b200.aesc import AESCGraph, mt_walk_count

    with open(os.path.join(GOLDEN, "mt_walks.json")) as f:
        c = json.load(f)["cases"][case]
    g = graph(c["graph"])
    idx, adj = g.csr()
    assert graph_fingerprint(idx, adj) == c["graph_fingerprint"]
    dg = AESCGraph.from_csr(idx, adj)
    counts, visits, checksum = mt_walk_count(dg, c["depth"], c["n_walks"], simd=c["simd"])
    dg.free()
    assert (visits, checksum, int(counts.max())) == (c["visit_count"], c["checksum"],
                                                    c["max_counter"])
    assert sha256_u32(counts) == c["counters_sha256"]
