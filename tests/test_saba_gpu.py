"""SABA walk counter on the GPU, through the C ABI: counters bit-exact with the reference's golden
vectors and with the oracle at larger sizes; visit_count = active vertices * W * D exactly."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _graph(path):
    from tgtp_b200.aesc import AESCGraph

    return AESCGraph(path)


def test_saba_matches_reference_golden(manifest, cuda_device):
    from tgtp_b200.aesc import saba_count

    for run in manifest["saba"]:
        g = _graph(os.path.join(GOLDEN, "saba", run["graph"]))
        counts, visits, checksum, _ = saba_count(g, run["depth"], run["n_walks"])
        want = np.load(os.path.join(GOLDEN, "saba", run["counts"]))
        assert np.array_equal(counts, want), run
        assert visits == run["visit_count"] and checksum == run["checksum"]
        g.free()


@pytest.mark.parametrize("depth,walks", [(5, 2048), (10, 64), (15, 16)])
def test_saba_config1_graph_matches_oracle(cuda_device, oracle_lib, depth, walks):
    from tgtp_b200 import synth
    from tgtp_b200.aesc import AESCGraph, saba_count

    g = synth.config1_graph(1)
    idx, adj = g.csr()
    dg = AESCGraph.from_csr(idx, adj)
    counts, visits, checksum, fb = saba_count(dg, depth, walks)
    want = oracle_lib.saba(idx, adj, depth, walks)
    assert np.array_equal(counts.astype(np.uint64), want)
    assert visits == g.n * walks * depth
    assert checksum == int((want * np.arange(1, g.n + 1, dtype=np.uint64)).sum())
    dg.free()


def test_saba_rmat_beyond_shared_counters_matches_oracle(cuda_device, oracle_lib):
    """n above the shared-memory counter range: hot ids in shared memory, the rest in L2."""
    from tgtp_b200 import synth
    from tgtp_b200.aesc import AESCGraph, saba_count

    g = synth.rmat(15, 8, 0.57, 0.19, 0.19, 9)
    idx, adj = g.csr()
    assert g.n > 12288
    dg = AESCGraph.from_csr(idx, adj)
    counts, visits, _, _ = saba_count(dg, 7, 32)
    want = oracle_lib.saba(idx, adj, 7, 32)
    assert np.array_equal(counts.astype(np.uint64), want)
    assert visits == g.n * 32 * 7
    dg.free()


def test_saba_fallback_phase_is_exercised(cuda_device, oracle_lib):
    """16-regular graph: secrets hit zero after 8 hops and the SplitMix32 phase takes over."""
    from tgtp_b200.aesc import AESCGraph, saba_count

    run = [r for r in [dict(graph="circ16.graph.txt", depth=10, n_walks=64)]][0]
    g = _graph(os.path.join(GOLDEN, "saba", run["graph"]))
    _, _, _, fb = saba_count(g, run["depth"], run["n_walks"], counters=False)
    assert fb == g.n * run["n_walks"] // 8
    g.free()


def test_saba_rejects_partial_bouquets(cuda_device):
    from tgtp_b200.aesc import TgtpError, saba_count

    g = _graph(os.path.join(GOLDEN, "saba", "cl300.graph.txt"))
    with pytest.raises(TgtpError) as e:
        saba_count(g, 5, 12)
    assert "multiple of 8" in str(e.value)
    g.free()


def test_saba_zero_walks_and_zero_depth(cuda_device):
    from tgtp_b200.aesc import saba_count

    g = _graph(os.path.join(GOLDEN, "saba", "cl300.graph.txt"))
    for d, w in ((0, 64), (5, 0)):
        counts, visits, checksum, _ = saba_count(g, d, w)
        assert visits == 0 and checksum == 0 and not counts.any()
    g.free()


def test_saba_rmat18_counters_match_oracle_at_full_graph_size(cuda_device, oracle_lib):
    """The R-MAT scale-18 walk graph (174,015 vertices, 7.6M slots) with 8 walks of depth 5 per
    vertex: every counter equal to the oracle's."""
    from tgtp_b200 import synth
    from tgtp_b200.aesc import AESCGraph, saba_count

    g = synth.config3_graph(1)
    idx, adj = g.csr()
    dg = AESCGraph.from_csr(idx, adj)
    counts, visits, _, _ = saba_count(dg, 5, 8)
    want = oracle_lib.saba(idx, adj, 5, 8)
    assert np.array_equal(counts.astype(np.uint64), want)
    assert visits == g.n * 8 * 5
    dg.free()


def _rmat18_fixture():
    import json

    with open(os.path.join(GOLDEN, "saba_rmat18.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def rmat18():
    """The R-MAT scale-18 walk graph, checked against the fingerprint the fixture was made on."""
    from tgtp_b200 import synth
    from tgtp_b200.aesc import AESCGraph

    from make_saba_rmat18 import graph_fingerprint

    g = synth.config3_graph(1)
    idx, adj = g.csr()
    assert graph_fingerprint(idx, adj) == _rmat18_fixture()["fingerprint"]
    dg = AESCGraph.from_csr(idx, adj)
    yield dict(g=g, idx=idx, adj=adj, dg=dg)
    dg.free()


@pytest.mark.parametrize("depth,walks", [(5, 2048), (10, 2048), (15, 2048), (5, 16384),
                                         (10, 16384), (15, 16384)])
def test_saba_rmat18_every_counter_matches_reference_and_oracle(cuda_device, rmat18, depth, walks):
    """Every depth x walks cell of the throughput workload on the R-MAT scale-18 graph (174,015
    vertices): the SHA-256 of all 174,015 counters, the visit count and the checksum equal those of
    tests/golden/saba_rmat18.json, which come from the reference's own walk routine where its float
    counters stay exact (D = 5 and 10 at W = 2,048) and from the oracle's integer restatement
    elsewhere (made by tests/golden/make_saba_rmat18.py)."""
    from make_saba_rmat18 import sha256_u32

    from tgtp_b200.aesc import saba_count

    cell = [c for c in _rmat18_fixture()["cells"]
            if (c["depth"], c["n_walks"]) == (depth, walks)][0]
    counts, visits, checksum, _ = saba_count(rmat18["dg"], depth, walks)
    assert visits == cell["visit_count"] == rmat18["g"].n * walks * depth
    assert checksum == cell["checksum"]
    assert int(counts.max()) == cell["max_counter"]
    assert sha256_u32(counts) == cell["counters_sha256"], cell["source"]


@pytest.mark.parametrize("depth,walks", [(5, 2048), (15, 16384)])
def test_saba_rmat18_static_entry_point_matches_the_fixture(cuda_device, rmat18, depth, walks):
    """The plain walk kernel behind saba_count_static (no degree renumbering) gives the fixture's
    visit count and checksum at the benchmark size and at the largest cell."""
    import ctypes as C

    import torch

    from tgtp_b200 import _lib

    cell = [c for c in _rmat18_fixture()["cells"]
            if (c["depth"], c["n_walks"]) == (depth, walks)][0]
    d_idx = torch.from_numpy(rmat18["idx"].astype(np.int32)).cuda()
    d_adj = torch.from_numpy(rmat18["adj"].astype(np.int32)).cuda()
    torch.cuda.synchronize()
    res = _lib.SabaResult()
    _lib.check(_lib.lib().saba_count_static(C.c_void_p(d_idx.data_ptr()),
                                            C.c_void_p(d_adj.data_ptr()), rmat18["g"].n, depth,
                                            walks, None, C.byref(res)))
    assert (int(res.visit_count), int(res.checksum)) == (cell["visit_count"], cell["checksum"])


def test_saba_tuned_layout_gives_the_same_counters(cuda_device, oracle_lib):
    """saba_tune times 1 / 2 / 4 walkers per lane over the plain walk copy (with 0 / 3,072 / 4,096
    row records in shared memory) and the inlined one and keeps the fastest; every layout, and so
    the chosen one, gives the oracle's counters."""
    from tgtp_b200 import synth
    from tgtp_b200.aesc import AESCGraph, saba_count, saba_tune

    g = synth.rmat(15, 8, 0.57, 0.19, 0.19, 9)
    idx, adj = g.csr()
    want = oracle_lib.saba(idx, adj, 7, 32)
    dg = AESCGraph.from_csr(idx, adj)
    choice = saba_tune(dg, 7, 32, trials=1)
    assert (choice & 0xff) in (1, 2, 4) and (choice & ~0x71ff) == 0
    assert (choice >> 12) in (0, 3, 4) and not ((choice & 0x100) and (choice >> 12))
    counts, visits, _, _ = saba_count(dg, 7, 32)
    assert np.array_equal(counts.astype(np.uint64), want)
    assert visits == g.n * 32 * 7
    dg.free()


@pytest.mark.parametrize("inline", ["0", "1"])
@pytest.mark.parametrize("wpl", ["1", "2", "4"])
def test_saba_every_walk_layout_matches_the_oracle(cuda_device, oracle_lib, monkeypatch, inline,
                                                   wpl):
    from tgtp_b200 import synth
    from tgtp_b200.aesc import AESCGraph, saba_count

    monkeypatch.setenv("TGTP_SABA_INLINE", inline)
    monkeypatch.setenv("TGTP_SABA_WPL", wpl)
    g = synth.rmat(14, 8, 0.57, 0.19, 0.19, 3)
    idx, adj = g.csr()
    dg = AESCGraph.from_csr(idx, adj)
    counts, visits, checksum, _ = saba_count(dg, 10, 64)
    want = oracle_lib.saba(idx, adj, 10, 64)
    assert np.array_equal(counts.astype(np.uint64), want)
    dg.free()


@pytest.mark.parametrize("hot,hot_rec", [("12288", "0"), ("12288", "1024"), ("12288", "4096"),
                                         ("8192", "4096"), ("1024", "8192"), ("12288", "8192")])
@pytest.mark.parametrize("wpl", ["1", "4"])
def test_saba_shared_row_records_give_the_oracle_counters(cuda_device, oracle_lib, monkeypatch,
                                                          hot, hot_rec, wpl):
    """The plain walk copy with the highest-degree row records in shared memory: hops landing on
    those numbers read the record there, the others from the copy in global memory (records are
    capped at the shared counters' count, as in ("1024", "8192"))."""
    from tgtp_b200 import synth
    from tgtp_b200.aesc import AESCGraph, saba_count

    monkeypatch.setenv("TGTP_SABA_INLINE", "0")
    monkeypatch.setenv("TGTP_SABA_HOT", hot)
    monkeypatch.setenv("TGTP_SABA_HOT_REC", hot_rec)
    monkeypatch.setenv("TGTP_SABA_WPL", wpl)
    g = synth.rmat(14, 8, 0.57, 0.19, 0.19, 3)
    idx, adj = g.csr()
    dg = AESCGraph.from_csr(idx, adj)
    counts, visits, _, fb = saba_count(dg, 10, 64)
    want = oracle_lib.saba(idx, adj, 10, 64)
    assert np.array_equal(counts.astype(np.uint64), want)
    assert visits == g.n * 64 * 10
    dg.free()
