"""The MIXED form on the GPU: FP32 residuals and lane-parallel compensated FP32 eigen projections
(F32 or BF16 storage), FP64 tau bounds / stop test / score accumulation, frontier-parallel push.
It is not bit-exact with the reference by design; it must be deterministic, symmetric and as
accurate against exact spanning centrality (oracle/exact_sc.py) as the FP64 form."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_tgtp_case

pytestmark = pytest.mark.gpu


def _graph(c):
    from tgtp_b200.aesc import VEC_BF16, VEC_F32, VEC_F64, AESCGraph

    g = AESCGraph.from_csr(c["idx"], c["adj"])
    g.upload_eigens(c["values"], c["v32"], VEC_F32)
    g.upload_eigens(c["values"], c["v32"], VEC_BF16)
    g.upload_eigens(c["values"], c["v64"], VEC_F64)
    return g


def _rev(idx, adj):
    rows = np.repeat(np.arange(len(idx) - 1), np.diff(idx.astype(np.int64)))
    key = rows.astype(np.int64) * len(idx) + adj
    order = np.argsort(key)
    return order[np.searchsorted(key[order], adj.astype(np.int64) * len(idx) + rows)]


@pytest.mark.parametrize("block", ["0", "1"])
@pytest.mark.parametrize("name", ["cl300", "sparse400", "grid", "cycle9", "complete12"])
def test_mixed_deterministic_symmetric_and_as_accurate_as_fp64(manifest, cuda_device, name, block,
                                                              monkeypatch):
    """block = 1 forces the multi-source push (push_block_kernel + source_kernel in PrePush mode)
    that large graphs take; 0 the per-warp push."""
    monkeypatch.setenv("TGTP_MIXED_BLOCK", block)
    from oracle import exact_sc
    from tgtp_b200.aesc import (AESC, AESCConfig, PRECISION_FP64, PRECISION_MIXED, VEC_BF16,
                                VEC_F32)

    c = golden_tgtp_case(manifest, name)
    g = _graph(c)
    exact = exact_sc.exact_scores(c["idx"], c["adj"])
    rev = _rev(c["idx"], c["adj"])
    for run in c["runs"]:
        eps, gamma = run["epsilon"], run["gamma"]
        f64 = AESC(g, AESCConfig(eps, omega=c["omega"], gamma=gamma, precision=PRECISION_FP64)).tgtp()
        acc64 = exact_sc.accuracy(f64, exact, eps)
        for vd in (VEC_F32, VEC_BF16):
            a = AESC(g, AESCConfig(eps, omega=c["omega"], gamma=gamma, precision=PRECISION_MIXED,
                                   vec_dtype=vd))
            s1, s2 = a.tgtp(), a.tgtp()
            assert np.array_equal(s1.view(np.uint32), s2.view(np.uint32)), "not deterministic"
            assert np.all(np.isfinite(s1)) and np.array_equal(s1, s1[rev])
            accm = exact_sc.accuracy(s1, exact, eps)
            # as accurate as the FP64 form against the exact scores: (almost) as many slots within
            # epsilon, or no larger maximum and mean error (graphs where the bound's mixing
            # assumption fails, like odd cycles, put few slots of either form within epsilon)
            as_many = accm["fraction_within_epsilon"] >= acc64["fraction_within_epsilon"] - 0.01
            no_worse = (accm["max_absolute_error"] <= acc64["max_absolute_error"] * (1 + 1e-6) and
                        accm["mean_absolute_error"] <= acc64["mean_absolute_error"] * (1 + 1e-6))
            assert as_many or no_worse, (run, vd, accm, acc64)
            assert accm["max_absolute_error"] <= max(2 * acc64["max_absolute_error"], eps), (
                run, vd, accm, acc64)
    g.free()


def test_mixed_matches_fp64_when_no_walks_run(cuda_device, config1_inputs):
    """With one push round and no walks (epsilon 0.05 on the 4,039-vertex graph) the forms differ
    only by rounding: FP32 residuals and FP32 projections against FP64."""
    from tgtp_b200.aesc import (AESC, AESCConfig, AESCGraph, PRECISION_FP64, PRECISION_MIXED,
                                VEC_BF16, VEC_F32, VEC_F64)

    c = config1_inputs
    g = AESCGraph.from_csr(c["idx"], c["adj"])
    g.upload_eigens(c["values"], c["v32"], VEC_F32)
    g.upload_eigens(c["values"], c["v64"], VEC_F64)
    g.upload_eigens(c["values"], c["v32"], VEC_BF16)
    f64 = AESC(g, AESCConfig(0.05, precision=PRECISION_FP64)).tgtp()
    for vd in (VEC_F32, VEC_BF16):
        a = AESC(g, AESCConfig(0.05, precision=PRECISION_MIXED, vec_dtype=vd))
        mixed = a.tgtp()
        assert a.stats()["walk_edges"] == 0
        np.testing.assert_allclose(mixed, f64, rtol=1e-5, atol=0)
    g.free()


@pytest.mark.parametrize("rounds", ["auto", "compact", "full", "compact_global_masks",
                                    "compact_cur_masks"])
@pytest.mark.parametrize("ctas", ["0", "2"])
@pytest.mark.parametrize("name", ["cl300", "sparse400", "grid", "cycle9", "complete12"])
def test_mixed_block_push_gives_the_same_bits(manifest, cuda_device, name, ctas, rounds,
                                              monkeypatch):
    """The per-warp push and the multi-source block push sum residuals in fixed point, so the two
    give identical scores, taus and work counters.  ctas = 2 runs the block push with two CTAs,
    64 sources per wave, so the larger graphs take several waves.  The block push's rounds are
    chosen by their frontier size (auto), or all compacted to the rows next to the live ones, or
    all full passes; compact_global_masks keeps its row masks in global memory and
    compact_cur_masks only the current round's mask in shared memory, as on graphs whose masks do
    not all fit in shared memory."""
    if ctas != "0":
        monkeypatch.setenv("TGTP_BLOCK_CTAS", ctas)
    if rounds != "auto":
        monkeypatch.setenv("TGTP_BLOCK_ROUNDS", rounds.split("_")[0])
    if rounds == "compact_global_masks":
        monkeypatch.setenv("TGTP_BLOCK_MASKS", "global")
    if rounds == "compact_cur_masks":  # only the current round's mask in shared memory
        monkeypatch.setenv("TGTP_BLOCK_MASKS", "cur")
    from tgtp_b200.aesc import AESC, AESCConfig, PRECISION_MIXED, VEC_BF16, VEC_F32

    c = golden_tgtp_case(manifest, name)
    g = _graph(c)
    for run in c["runs"]:
        for vd in (VEC_F32, VEC_BF16):
            got = {}
            for block in ("0", "1"):
                monkeypatch.setenv("TGTP_MIXED_BLOCK", block)
                a = AESC(g, AESCConfig(run["epsilon"], omega=c["omega"], gamma=run["gamma"],
                                       precision=PRECISION_MIXED, vec_dtype=vd))
                s = a.tgtp()
                st = a.stats()
                got[block] = (s, a.taus(), {k: st[k] for k in ("push_rounds", "push_vertices",
                                                               "push_traversals", "walk_edges",
                                                               "walk_count", "walk_hops")})
            assert np.array_equal(got["0"][0].view(np.uint32), got["1"][0].view(np.uint32)), run
            assert np.array_equal(got["0"][1], got["1"][1])
            assert got["0"][2] == got["1"][2], (run, got["0"][2], got["1"][2])
    g.free()


@pytest.mark.parametrize("name", ["cl300", "sparse400", "grid", "cycle9", "complete12"])
def test_mixed_block_push_with_hbm_per_source_stage_gives_the_same_bits(manifest, cuda_device,
                                                                         name, monkeypatch):
    """After the block push, the per-source stage in the HBM tier reads each source's residual
    column in place and selects the top-gamma residuals straight from it (no frontier list), as
    on large graphs; its scores, taus and counters equal the per-warp push's."""
    from tgtp_b200.aesc import AESC, AESCConfig, PRECISION_MIXED, VEC_BF16

    monkeypatch.setenv("TGTP_PVEC_TIER", "global")
    monkeypatch.setenv("TGTP_BLOCK_CTAS", "2")
    c = golden_tgtp_case(manifest, name)
    g = _graph(c)
    for run in c["runs"]:
        got = {}
        for block in ("0", "1"):
            monkeypatch.setenv("TGTP_MIXED_BLOCK", block)
            a = AESC(g, AESCConfig(run["epsilon"], omega=c["omega"], gamma=run["gamma"],
                                   precision=PRECISION_MIXED, vec_dtype=VEC_BF16))
            s = a.tgtp()
            st = a.stats()
            got[block] = (s, {k: st[k] for k in ("push_rounds", "walk_edges", "walk_count",
                                                 "walk_hops")})
        assert np.array_equal(got["0"][0].view(np.uint32), got["1"][0].view(np.uint32)), run
        assert got["0"][1] == got["1"][1], run
    g.free()


def test_mixed_push_choice_is_learned_from_the_previous_run_without_a_counter_read(cuda_device,
                                                                                   monkeypatch):
    """Sparse Chung-Lu graph (28,000 ids, 120,000 edges, exponent 2.1): residual vectors beyond
    shared memory, eps = 0.05.  The first run has no measurement and pushes per warp; its push
    counters reach the handle through pinned memory, so the next run -- with no stats() call in
    between -- takes the block push (frontiers averaging more than m / 40 traversals a round), with
    the same bits."""
    import torch

    from tgtp_b200 import synth, workloads
    from tgtp_b200.aesc import AESC, AESCConfig, AESCGraph, PRECISION_MIXED, VEC_BF16

    monkeypatch.delenv("TGTP_MIXED_BLOCK", raising=False)
    monkeypatch.setenv("TGTP_KERNEL_DEADLINE_S", "120")
    g = synth.chung_lu(28000, 120000, 2.1, 1)
    idx, adj = g.csr()
    values, v32, _ = workloads._eigenpairs(g, 128)
    dg = AESCGraph.from_csr(idx, adj)
    dg.upload_eigens(values, v32, VEC_BF16)
    a = AESC(dg, AESCConfig(0.05, precision=PRECISION_MIXED, vec_dtype=VEC_BF16))
    outs, kernels = [], []
    for _ in range(3):
        out = torch.empty(int(idx[-1]), dtype=torch.float32, device="cuda")
        dg.set_profiling(True)
        a.tgtp_device(out.data_ptr())
        torch.cuda.synchronize()
        kernels.append(set(dg.kernel_stats()))
        dg.set_profiling(False)
        outs.append(out.cpu().numpy())
    assert "push_block" not in kernels[0] and "push_block" in kernels[1] and "push_block" in kernels[2]
    for o in outs[1:]:
        assert np.array_equal(o.view(np.uint32), outs[0].view(np.uint32))
    dg.free()


def test_mixed_and_fp64_differ_only_on_slots_next_to_a_pushed_row(cuda_device):
    """Where the two forms' scores part, per slot (batch graphs of the batched workload, own eps):
    a slot both of whose rows finish in closed form in both forms (no round past the first, no
    walk; the run trace reads 0 rounds) agrees to float rounding (1e-6 relative); every larger
    difference sits on a slot one of whose rows pushed.  The mixed form's Jacobi rounds and the
    FP64 form's Gauss-Seidel rounds leave different residuals, so such slots differ even when
    their tau, rounds and walk counts agree; both stay within eps of the exact value at the same
    rate (tests/test_exact_sc_gpu.py)."""
    from tgtp_b200 import eigenprep_gpu, synth
    from tgtp_b200.aesc import (AESC, AESCConfig, AESCGraph, PRECISION_FP64, PRECISION_MIXED,
                                VEC_BF16, VEC_F64)

    work = sorted(synth.config5_graphs(5, 64), key=lambda ge: ge[0].n)[:6]
    pushed_total = 0
    for g, eps in work:
        idx, adj = g.csr()
        vals, vecs, _, _, _ = eigenprep_gpu.compute(g.n, g.u, g.v, 128, seed=1, tol=1e-6,
                                                    max_iter=60)
        v64 = np.ascontiguousarray(vecs.T).ravel()
        dg = AESCGraph.from_csr(idx, adj)
        dg.upload_eigens(vals, v64, VEC_F64)
        dg.upload_eigens(vals, v64.astype(np.float32), VEC_BF16)
        dg.set_trace(True)
        out = {}
        for label, cfg in (("fp64", AESCConfig(eps, precision=PRECISION_FP64)),
                           ("mixed", AESCConfig(eps, precision=PRECISION_MIXED,
                                                vec_dtype=VEC_BF16))):
            s = AESC(dg, cfg).tgtp().astype(np.float64)
            out[label] = (s, dg.read_trace()[1])
        dg.free()
        rows = np.repeat(np.arange(g.n), np.diff(idx.astype(np.int64)))
        closed = (out["fp64"][1] == 0) & (out["mixed"][1] == 0)
        both_closed = closed[rows] & closed[adj]
        dev = np.abs(out["mixed"][0] - out["fp64"][0]) / np.abs(out["fp64"][0])
        assert np.all(dev[both_closed] <= 1e-6), (g.n, float(dev[both_closed].max()))
        assert np.all(~both_closed[dev > 1e-6])
        pushed_total += int((~both_closed).sum())
    assert pushed_total > 0


@pytest.mark.parametrize("vec", ["f32", "bf16"])
def test_block_push_walk_kernels_give_the_per_warp_walks_bits(cuda_device, monkeypatch, vec):
    """After the block push the walks run in walk_queue_kernel (light items) and
    heavy_walk_kernel (items of at least 512 walks of at most 32 hops, 32 bouquets at once): on
    the sparse Chung-Lu graph (28,000 ids, 120,000 edges, exponent 2.1) at eps = 0.005, with both
    kinds present (read from the run trace), the scores and walk counters equal the per-warp
    push's, whose walks run in the source kernel."""
    from tgtp_b200 import synth, workloads
    from tgtp_b200.aesc import (AESC, AESCConfig, AESCGraph, PRECISION_MIXED, VEC_BF16,
                                VEC_F32)

    monkeypatch.setenv("TGTP_KERNEL_DEADLINE_S", "120")
    sg = synth.chung_lu(28000, 120000, 2.1, 1)
    idx, adj = sg.csr()
    values, v32, _ = workloads._eigenpairs(sg, 128)
    c = {"idx": idx, "adj": adj, "n": sg.n}
    store = VEC_BF16 if vec == "bf16" else VEC_F32
    g = AESCGraph.from_csr(idx, adj)
    g.upload_eigens(values, v32, store)
    got = {}
    for block in ("0", "1"):
        monkeypatch.setenv("TGTP_MIXED_BLOCK", block)
        g.set_trace(True)
        a = AESC(g, AESCConfig(0.005, precision=PRECISION_MIXED, vec_dtype=store))
        s = a.tgtp()
        st = a.stats()
        nr, ell = g.read_trace()
        taus = a.taus()[: len(c["adj"])].astype(np.int64)
        g.set_trace(False)
        got[block] = (s, {k: st[k] for k in ("push_rounds", "walk_edges", "walk_count", "walk_hops",
                                             "fallback_bouquets")}, nr, ell, taus)
    g.free()
    assert np.array_equal(got["0"][0].view(np.uint32), got["1"][0].view(np.uint32))
    assert got["0"][1] == got["1"][1]
    nr, ell, taus = got["1"][2], got["1"][3], got["1"][4]
    rows = np.repeat(np.arange(c["n"]), np.diff(c["idx"].astype(np.int64)))
    walk_len = taus - ell[rows].astype(np.int64)
    heavy = (nr >= 512) & (walk_len <= 32)
    light = (nr > 0) & ~heavy
    assert heavy.sum() > 0 and light.sum() > 0, (int(heavy.sum()), int(light.sum()))
