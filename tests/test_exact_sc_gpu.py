"""Exact spanning centrality of sampled edges on the GPU (tgtp_exact_sc_slots: FP64 conjugate
gradients on the Laplacian, the quantity of src/exact_sc.cpp:24-49), through the C ABI:

* against the dense oracle (oracle/exact_sc.py, itself pinned to the reference's
  scripts/paper_accuracy.py) on the golden graphs and on the 4,039-vertex Chung-Lu graph;
* then as the accuracy reference on graphs too large for a dense solve: the mixed form keeps the
  FP64 form's fraction of edges within epsilon on >= 10^4 sampled edges of the R-MAT scale-18 graph
  and of the largest graph of the batched workload (above 10^5 vertices)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_tgtp_case

pytestmark = pytest.mark.gpu

SIMPLE_CASES = ["cl300", "sparse400", "grid", "cycle9", "complete12"]


def _forward_sample(idx, adj, count, seed):
    """`count` distinct undirected edges (their slot with u < v), seeded."""
    rows = np.repeat(np.arange(len(idx) - 1), np.diff(idx.astype(np.int64)))
    fwd = np.flatnonzero(adj.astype(np.int64) > rows)
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(fwd, size=min(count, len(fwd)), replace=False)).astype(np.uint32)


@pytest.mark.parametrize("name", SIMPLE_CASES)
def test_exact_sc_matches_the_dense_oracle_on_every_slot(manifest, cuda_device, name):
    from oracle import exact_sc
    from tgtp_b200.aesc import AESCGraph, exact_sc_slots

    c = golden_tgtp_case(manifest, name)
    want = exact_sc.exact_scores(c["idx"], c["adj"])
    g = AESCGraph.from_csr(c["idx"], c["adj"])
    got, iters = exact_sc_slots(g, np.arange(len(c["adj"]), dtype=np.uint32), tol=1e-12)
    g.free()
    assert np.max(np.abs(got - want)) < 1e-9, name
    assert iters.max() < 20000


def test_exact_sc_matches_the_dense_oracle_on_the_config1_graph(cuda_device):
    from oracle import exact_sc
    from tgtp_b200 import synth
    from tgtp_b200.aesc import AESCGraph, exact_sc_slots

    g = synth.config1_graph(1)
    idx, adj = g.csr()
    want = exact_sc.exact_scores(idx, adj)
    slots = _forward_sample(idx, adj, 2048, 3)
    dg = AESCGraph.from_csr(idx, adj)
    got, _ = exact_sc_slots(dg, slots, tol=1e-12)
    dg.free()
    assert np.max(np.abs(got - want[slots])) < 1e-9


def test_exact_sc_of_a_self_loop_slot_is_zero_and_repeats_count_once(cuda_device):
    """Multigraph slots score on the simple graph, as the dense oracle does."""
    from oracle import exact_sc
    from tgtp_b200.aesc import AESCGraph, exact_sc_slots

    # triangle 0-1-2 with 2-3, the edge 0-1 listed twice and a self-loop at 3
    idx = np.array([0, 3, 6, 9, 12], np.uint32)
    adj = np.array([1, 1, 2, 0, 0, 2, 0, 1, 3, 2, 3, 3], np.uint32)
    want = exact_sc.exact_scores(idx, adj)
    g = AESCGraph.from_csr(idx, adj)
    got, _ = exact_sc_slots(g, np.arange(len(adj), dtype=np.uint32), tol=1e-12)
    g.free()
    assert np.max(np.abs(got - want)) < 1e-10
    assert got[10] == 0.0 and got[11] == 0.0


def _within_eps_fractions(g, eps, slots, exact):
    """Fraction of the sampled slots within eps of the exact value, FP64 and mixed (BF16) forms."""
    from tgtp_b200 import eigenprep_gpu
    from tgtp_b200.aesc import (AESC, AESCConfig, AESCGraph, PRECISION_FP64, PRECISION_MIXED,
                                VEC_BF16, VEC_F64)

    idx, adj = g.csr()
    vals, vecs, _, _, _ = eigenprep_gpu.compute(g.n, g.u, g.v, 128, seed=1, tol=1e-4, max_iter=60)
    v64 = np.ascontiguousarray(vecs.T).ravel()
    dg = AESCGraph.from_csr(idx, adj)
    dg.upload_eigens(vals, v64, VEC_F64)
    dg.upload_eigens(vals, v64.astype(np.float32), VEC_BF16)
    out = {}
    for label, cfg in (("fp64", AESCConfig(eps, precision=PRECISION_FP64)),
                       ("mixed", AESCConfig(eps, precision=PRECISION_MIXED, vec_dtype=VEC_BF16))):
        s = AESC(dg, cfg).tgtp()
        err = np.abs(s[slots].astype(np.float64) - exact)
        out[label] = (float(np.mean(err <= eps)), float(err.max()))
    dg.free()
    return out


@pytest.mark.parametrize("which", ["rmat18", "batch_largest"])
def test_mixed_form_keeps_the_fp64_fraction_within_eps_on_large_graphs(cuda_device, which):
    """10^4 sampled edges, exact values from the GPU solver: the mixed form (BF16 vectors, FP32
    residuals) has at least the FP64 form's fraction of edges within epsilon, less half a percent."""
    import os

    from tgtp_b200 import synth
    from tgtp_b200.aesc import AESCGraph, exact_sc_slots

    os.environ.setdefault("TGTP_KERNEL_DEADLINE_S", "300")
    if which == "rmat18":
        g, eps = synth.config3_graph(1), 0.05
    else:
        g, eps = max(synth.config5_graphs(5, 64), key=lambda ge: ge[0].n)
        assert g.n > 100_000
    idx, adj = g.csr()
    slots = _forward_sample(idx, adj, 10_000, 11)
    dg = AESCGraph.from_csr(idx, adj)
    exact, _ = exact_sc_slots(dg, slots, tol=1e-9)
    dg.free()
    assert np.all((exact > 0) & (exact <= 1 + 1e-9))
    fr = _within_eps_fractions(g, eps, slots, exact)
    print(which, g.n, eps, fr)
    assert fr["mixed"][0] >= fr["fp64"][0] - 0.005, fr
