"""Batched tgtp (one CUDA graph over many graphs and configurations) and the source-kernel layout
tuner, through the C ABI: every layout and the batched replay give the same scores, bit for bit,
as single runs of the same form."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import golden_tgtp_case, load_golden_scores

pytestmark = pytest.mark.gpu

CASES = ["cl300", "sparse400", "grid", "cycle9", "complete12"]


def _graph(c):
    from tgtp_b200.aesc import VEC_BF16, VEC_F32, VEC_F64, AESCGraph

    g = AESCGraph.from_csr(c["idx"], c["adj"])
    g.upload_eigens(c["values"], c["v32"], VEC_F32)
    g.upload_eigens(c["values"], c["v64"], VEC_F64)
    g.upload_eigens(c["values"], c["v32"], VEC_BF16)
    return g


def _configs(c):
    from tgtp_b200.aesc import (AESCConfig, PRECISION_FP32, PRECISION_FP64, PRECISION_MIXED,
                                VEC_BF16, VEC_F32)

    run = c["runs"][-1]
    return [AESCConfig(run["epsilon"], omega=c["omega"], gamma=run["gamma"],
                       precision=PRECISION_FP32),
            AESCConfig(run["epsilon"], omega=c["omega"], gamma=run["gamma"],
                       precision=PRECISION_FP64),
            AESCConfig(run["epsilon"], omega=c["omega"], gamma=run["gamma"],
                       precision=PRECISION_MIXED, vec_dtype=VEC_F32),
            AESCConfig(run["epsilon"], omega=c["omega"], gamma=run["gamma"],
                       precision=PRECISION_MIXED, vec_dtype=VEC_BF16)], run


@pytest.mark.parametrize("name", CASES)
def test_every_source_layout_gives_the_same_scores(manifest, cuda_device, name):
    import torch

    from tgtp_b200.aesc import AESC

    c = golden_tgtp_case(manifest, name)
    g = _graph(c)
    cfgs, run = _configs(c)
    for cfg in cfgs:
        a = AESC(g, cfg)
        want = a.tgtp()
        os.environ["TGTP_PVEC_TIER"] = "global"
        try:
            glob = a.tgtp()
        finally:
            del os.environ["TGTP_PVEC_TIER"]
        assert np.array_equal(glob.view(np.uint32), want.view(np.uint32)), cfg
        out = torch.empty(g.m, dtype=torch.float32, device="cuda")
        code = a.tune(out.data_ptr(), trials=1)
        assert code & 0xff in (1, 2, 4)
        tuned = a.tgtp()
        assert np.array_equal(tuned.view(np.uint32), want.view(np.uint32)), (cfg, hex(code))
    # the FP32 form under its tuned layout is still the reference's output
    assert np.array_equal(AESC(g, cfgs[0]).tgtp().view(np.uint32),
                          load_golden_scores(run).view(np.uint32))
    g.free()


def test_batch_replays_match_single_runs(manifest, cuda_device):
    import torch

    from tgtp_b200.aesc import AESC, Batch

    graphs, runs, want, stats = [], [], [], []
    for i, name in enumerate(CASES):
        c = golden_tgtp_case(manifest, name)
        g = _graph(c)
        cfg = _configs(c)[0][i % 4]
        a = AESC(g, cfg)
        want.append(a.tgtp())
        stats.append(a.stats())
        graphs.append(g)
        runs.append((a, torch.empty(g.m, dtype=torch.float32, device="cuda")))
    b = Batch([(a, o.data_ptr()) for a, o in runs], tune_trials=1)
    for rep in range(2):
        for _, o in runs:
            o.fill_(-1.0)
        torch.cuda.synchronize()  # the fills (torch's stream) end before the batch's stream
        b.run()
        b.wait()
        for (a, o), w, st in zip(runs, want, stats):
            got = o.cpu().numpy()
            assert np.array_equal(got.view(np.uint32), w.view(np.uint32)), (rep, a.config)
            got_st = a.stats()
            for k in ("push_rounds", "push_traversals", "walk_edges", "walk_hops", "tau_iterations"):
                assert got_st[k] == st[k], (k, a.config)
    b.free()
    for g in graphs:
        g.free()


def test_batched_graph_keeps_its_buffers(manifest, cuda_device):
    import torch

    from tgtp_b200.aesc import AESC, Batch, PRECISION_FP64, TgtpError, VEC_F32

    c = golden_tgtp_case(manifest, "cl300")
    g = _graph(c)
    cfgs, _ = _configs(c)
    a = AESC(g, cfgs[0])
    out = torch.empty(g.m, dtype=torch.float32, device="cuda")
    b = Batch([(a, out.data_ptr())])
    with pytest.raises(TgtpError):
        g.upload_eigens(c["values"], c["v32"], VEC_F32)
    with pytest.raises(TgtpError):
        g.free()
    # a run of the same configuration on the batched graph is fine
    a.tgtp()
    b.free()
    g.upload_eigens(c["values"], c["v32"], VEC_F32)
    assert AESC(g, cfgs[1]).tgtp().shape == (g.m,)
    g.free()


@pytest.mark.parametrize("tier", ["smem", "global"])
@pytest.mark.parametrize("form", ["fp32", "fp64", "mixed_bf16"])
def test_one_persistent_launch_over_all_graphs_matches_single_runs(manifest, cuda_device, tier,
                                                                   form, monkeypatch):
    """Every graph of the batch in one form: their listed rows form one queue that a single
    persistent source kernel works through (per residual-vector tier), and every graph's scores
    and work counters equal its single run, on two replays; with the shared kernel switched off
    (TGTP_BATCH_PERSISTENT=0, one branch per graph) the replays give the same bits too."""
    import torch

    from tgtp_b200.aesc import (AESC, AESCConfig, Batch, PRECISION_FP32, PRECISION_FP64,
                                PRECISION_MIXED, VEC_BF16)

    monkeypatch.setenv("TGTP_PVEC_TIER", tier)
    names = CASES + (["multi300"] if form != "mixed_bf16" else [])
    prec = {"fp32": PRECISION_FP32, "fp64": PRECISION_FP64, "mixed_bf16": PRECISION_MIXED}[form]
    graphs, runs, want, stats = [], [], [], []
    for name in names:
        c = golden_tgtp_case(manifest, name)
        g = _graph(c)
        run = c["runs"][-1]
        a = AESC(g, AESCConfig(run["epsilon"], omega=c["omega"], gamma=run["gamma"],
                               precision=prec, vec_dtype=VEC_BF16))
        want.append(a.tgtp())
        stats.append(a.stats())
        graphs.append(g)
        runs.append((a, torch.empty(g.m, dtype=torch.float32, device="cuda")))
    for persistent in ("1", "0"):
        monkeypatch.setenv("TGTP_BATCH_PERSISTENT", persistent)
        b = Batch([(a, o.data_ptr()) for a, o in runs])
        for rep in range(2):
            for _, o in runs:
                o.fill_(-1.0)
            torch.cuda.synchronize()  # the fills (torch's stream) end before the batch's stream
            b.run()
            b.wait()
            for (a, o), w, st in zip(runs, want, stats):
                got = o.cpu().numpy()
                assert np.array_equal(got.view(np.uint32), w.view(np.uint32)), (persistent, rep)
                got_st = a.stats()
                for k in ("push_rounds", "push_vertices", "push_traversals", "walk_edges",
                          "walk_count", "walk_hops", "fallback_bouquets"):
                    assert got_st[k] == st[k], (k, persistent, rep)
        b.free()
    for g in graphs:
        g.free()
