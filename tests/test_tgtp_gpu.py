"""tgtp() on the GPU, through the C ABI.

FP32 form: bit-exact with the reference (golden vectors) and with the oracle.
FP64 form: bit-exact with the oracle's FP64 restatement (same operations, same order) and within
           1e-6 relative (or 2 float32 ulps) of the reference on every slot.
Work counters (push rounds, traversals, walks, fallbacks) equal the oracle's."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_tgtp_case, load_golden_scores

pytestmark = pytest.mark.gpu

# multi300: the cl300 graph with repeated edges and self-loops, which the reference's loader keeps
CASES = ["cl300", "sparse400", "grid", "cycle9", "complete12", "multi300"]
STAT_KEYS = ["push_rounds", "push_vertices", "push_traversals", "walk_edges", "walk_count",
             "walk_hops", "fallback_bouquets", "tau_iterations"]


def _device_graph(c, fp64=False):
    from tgtp_b200.aesc import VEC_F32, VEC_F64, AESCGraph

    g = AESCGraph.from_csr(c["idx"], c["adj"])
    g.upload_eigens(c["values"], c["v32"], VEC_F32)
    if fp64:
        g.upload_eigens(c["values"], c["v64"], VEC_F64)
    return g


@pytest.mark.parametrize("name", CASES)
def test_fp32_bit_exact_with_reference(manifest, cuda_device, name):
    from tgtp_b200.aesc import AESC, AESCConfig

    c = golden_tgtp_case(manifest, name)
    g = _device_graph(c)
    for run in c["runs"]:
        a = AESC(g, AESCConfig(run["epsilon"], omega=c["omega"], gamma=run["gamma"]))
        got = a.tgtp()
        want = load_golden_scores(run)
        bad = np.flatnonzero(got.view(np.uint32) != want.view(np.uint32))
        assert bad.size == 0, (run, bad[:8], got[bad[:4]], want[bad[:4]])
        assert a.stats()["tau_ambiguous"] == 0
    g.free()


@pytest.mark.parametrize("name", CASES)
def test_fp32_taus_and_work_counters_match_oracle(manifest, cuda_device, oracle_lib, name):
    from tgtp_b200.aesc import AESC, AESCConfig

    c = golden_tgtp_case(manifest, name)
    g = _device_graph(c)
    for run in c["runs"]:
        a = AESC(g, AESCConfig(run["epsilon"], omega=c["omega"], gamma=run["gamma"]))
        a.tgtp()
        _, det = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v32"], run["epsilon"],
                                 gamma=run["gamma"], details=True)
        assert np.array_equal(a.taus(), det["taus"])
        st = a.stats()
        for k in STAT_KEYS:
            assert st[k] == det["stats"][k], (run, k, st[k], det["stats"][k])
    g.free()


@pytest.mark.parametrize("name", CASES)
def test_fp64_matches_oracle_and_reference(manifest, cuda_device, oracle_lib, name):
    from tgtp_b200.aesc import AESC, AESCConfig, PRECISION_FP64

    c = golden_tgtp_case(manifest, name)
    g = _device_graph(c, fp64=True)
    for run in c["runs"]:
        a = AESC(g, AESCConfig(run["epsilon"], omega=c["omega"], gamma=run["gamma"],
                               precision=PRECISION_FP64))
        got = a.tgtp()
        ora = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v64"], run["epsilon"],
                              gamma=run["gamma"], fp64=True)
        assert np.array_equal(got.view(np.uint32), ora.view(np.uint32)), run
        want = load_golden_scores(run)
        bad = _outside_reference_tolerance(got, want)
        assert bad.size == 0, (run, bad[:8])
    g.free()


def _outside_reference_tolerance(got, want):
    """Slots where the FP64 form is further than 1e-6 relative and 2 float32 ulps from the
    reference's float32 score."""
    want = np.asarray(want, np.float32)
    tol = np.maximum(1e-6 * np.abs(want.astype(np.float64)),
                     2 * np.spacing(np.abs(want)).astype(np.float64))
    return np.flatnonzero(np.abs(got.astype(np.float64) - want.astype(np.float64)) > tol)


@pytest.mark.parametrize("eps", [0.05, 0.01, 0.005])
def test_config1_fp32_bit_exact_with_oracle(cuda_device, oracle_lib, config1_inputs, eps):
    from tgtp_b200.aesc import AESC, AESCConfig, AESCGraph, VEC_F32

    c = config1_inputs
    g = AESCGraph.from_csr(c["idx"], c["adj"])
    g.upload_eigens(c["values"], c["v32"], VEC_F32)
    got = AESC(g, AESCConfig(eps)).tgtp()
    want = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v32"], eps)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    g.free()


def test_config1_fp64_bit_exact_with_oracle(cuda_device, oracle_lib, config1_inputs):
    from tgtp_b200.aesc import AESC, AESCConfig, AESCGraph, PRECISION_FP64, VEC_F64

    c = config1_inputs
    g = AESCGraph.from_csr(c["idx"], c["adj"])
    g.upload_eigens(c["values"], c["v64"], VEC_F64)
    got = AESC(g, AESCConfig(0.05, precision=PRECISION_FP64)).tgtp()
    want = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v64"], 0.05, fp64=True)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    g.free()


@pytest.mark.parametrize("eps", [0.05, 0.01, 0.005])
def test_config2_fp64_matches_oracle_bitwise_and_the_reference_on_every_slot(
        cuda_device, oracle_lib, config1_inputs, eps):
    """The FP64 form on the 4,039-vertex Chung-Lu graph with 128 eigenpairs, gamma 10: every slot
    bit-equal to the FP64 oracle and within 1e-6 relative (or 2 float32 ulps) of the reference's
    own tgtp (oracle/_ref/tgtp_O2, compiled from the reference sources, run on the same graph.txt
    and sorted_eigens_128.txt), with no slot outside.  At eps 0.01 and 0.005 sources push past
    their first round and slots walk, so the push, chi and walk code runs on this graph."""
    import os
    import subprocess
    import tempfile

    from tgtp_b200.aesc import AESC, AESCConfig, AESCGraph, PRECISION_FP64, VEC_F64

    exe = oracle_lib.ref_binary("tgtp_O2")
    if exe is None:
        pytest.fail("oracle/_ref/tgtp_O2 (the reference built from its sources) is missing")
    c = config1_inputs
    g = AESCGraph.from_csr(c["idx"], c["adj"])
    g.upload_eigens(c["values"], c["v64"], VEC_F64)
    a = AESC(g, AESCConfig(eps, precision=PRECISION_FP64))
    got = a.tgtp()
    st = a.stats()
    g.free()
    ora, det = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v64"], eps, fp64=True,
                               details=True)
    assert np.array_equal(got.view(np.uint32), ora.view(np.uint32))
    for k in STAT_KEYS:
        assert st[k] == det["stats"][k], k
    if eps < 0.05:
        assert st["push_rounds"] > c["n"] and st["walk_edges"] > 0
    out = os.path.join(tempfile.mkdtemp(prefix="tgtp_ref_"), "scores.bin")
    folder = c["folder"]
    r = subprocess.run([exe, os.path.dirname(folder), os.path.basename(folder), str(eps), "128",
                        "10", out], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    ref = np.fromfile(out, dtype=np.float32)
    assert ref.shape == got.shape
    bad = _outside_reference_tolerance(got, ref)
    assert bad.size == 0, (bad[:8], got[bad[:4]], ref[bad[:4]])


def test_multigraph_taus_leave_the_unwritten_repeats_at_zero(manifest, cuda_device, oracle_lib):
    """In a row that repeats a smaller neighbour, the reference writes tau only into the first of
    the repeats (lower_bound, src/aesc.h:207-209) and leaves the others 0; the GPU run does the
    same, and the mixed form refuses such a graph (TGTP_ERR_UNSUPPORTED) instead of guessing."""
    from tgtp_b200.aesc import (AESC, AESCConfig, PRECISION_MIXED, TgtpError, VEC_F32)

    c = golden_tgtp_case(manifest, "multi300")
    g = _device_graph(c)
    a = AESC(g, AESCConfig(0.01, omega=c["omega"]))
    a.tgtp()
    taus = a.taus()
    _, det = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v32"], 0.01, details=True)
    assert np.array_equal(taus, det["taus"])
    assert (taus == 0).sum() == 12  # the 12 repeated edges' later slots in the larger end's row
    with pytest.raises(TgtpError) as e:
        AESC(g, AESCConfig(0.01, omega=c["omega"], precision=PRECISION_MIXED,
                           vec_dtype=VEC_F32)).tgtp()
    assert e.value.status == 6
    g.free()


def test_invalid_arguments_are_rejected(manifest, cuda_device):
    from tgtp_b200.aesc import AESC, AESCConfig, AESCGraph, TgtpError, PRECISION_FP64

    c = golden_tgtp_case(manifest, "cl300")
    g = _device_graph(c)
    for cfg in (AESCConfig(0.0, omega=16), AESCConfig(1.0, omega=16),
                AESCConfig(0.05, omega=16, gamma=0), AESCConfig(0.05, omega=1),
                AESCConfig(0.05, omega=32), AESCConfig(0.05, omega=16, precision=PRECISION_FP64)):
        with pytest.raises(TgtpError) as e:
            AESC(g, cfg).tgtp()
        assert e.value.status == 1, cfg
    g.free()
    # isolated vertex: AESCGraph rejects it (src/aesc.h:88-89)
    idx = np.array([0, 1, 2, 2, 2], np.uint32)
    adj = np.array([1, 0], np.uint32)
    g = AESCGraph.from_csr(idx, adj)
    with pytest.raises(TgtpError):
        g.upload_eigens(np.array([1.0, 0.5]), np.zeros(8, np.float32))
        AESC(g, AESCConfig(0.05, omega=2)).tgtp()
    g.free()
    # an edge into a vertex without neighbours (a walk would have nowhere to go): refused at upload
    for idx, adj in ((np.array([0, 1, 1], np.uint32), np.array([1], np.uint32)),
                     (np.array([0, 2, 3, 3], np.uint32), np.array([1, 2, 0], np.uint32))):
        with pytest.raises(TgtpError) as e:
            AESCGraph.from_csr(idx, adj)
        assert e.value.status == 1 and "without neighbours" in str(e.value)


def test_fp64_bulk_copy_tau_gives_the_same_bits(manifest, cuda_device, oracle_lib, monkeypatch):
    """TGTP_TAU_BULK=1 moves the eigen rows into shared memory with cp.async.bulk before summing;
    the sums, and so the scores, are the same bits as the FP64 oracle's."""
    from tgtp_b200.aesc import AESC, AESCConfig, PRECISION_FP64

    monkeypatch.setenv("TGTP_TAU_BULK", "1")
    c = golden_tgtp_case(manifest, "cl300")
    g = _device_graph(c, fp64=True)
    for run in c["runs"]:
        got = AESC(g, AESCConfig(run["epsilon"], omega=c["omega"], gamma=run["gamma"],
                                 precision=PRECISION_FP64)).tgtp()
        ora = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v64"], run["epsilon"],
                              gamma=run["gamma"], fp64=True)
        assert np.array_equal(got.view(np.uint32), ora.view(np.uint32)), run
    g.free()


@pytest.mark.parametrize("tier", ["smem", "global"])
def test_device_time_budget_gives_a_timeout_status_and_leaves_the_graph_usable(
        config1_inputs, cuda_device, monkeypatch, tier):
    """Failure detection without a GPU fault: with a device time budget of 1 ns every warp of the
    source kernel gives up at its next check and the run returns TGTP_ERR_TIMEOUT; the next run on
    the same graph handle (residual vectors in shared memory, or in HBM where a warp that gave up
    left them dirty) gives the same bits and work counters as a run before the time-out."""
    from tgtp_b200.aesc import AESC, AESCConfig, AESCGraph, PRECISION_FP64, TgtpError, VEC_F64

    monkeypatch.setenv("TGTP_PVEC_TIER", tier)
    c = config1_inputs
    g = AESCGraph.from_csr(c["idx"], c["adj"])
    g.upload_eigens(c["values"], c["v64"], VEC_F64)
    cfg = AESCConfig(0.005, precision=PRECISION_FP64)
    a = AESC(g, cfg)
    want = a.tgtp()
    want_st = a.stats()
    assert want_st["push_rounds"] > 0  # listed rows: the source kernel pushes
    monkeypatch.setenv("TGTP_KERNEL_DEADLINE_S", "1e-9")
    with pytest.raises(TgtpError) as e:
        a.tgtp()
    assert e.value.status == 4  # TGTP_ERR_TIMEOUT
    monkeypatch.delenv("TGTP_KERNEL_DEADLINE_S")
    for _ in range(2):
        got = a.tgtp()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        st = a.stats()
        for k in STAT_KEYS:
            assert st[k] == want_st[k], k
    g.free()


@pytest.mark.parametrize("name", ["cl300", "sparse400", "multi300"])
def test_one_vertex_at_a_time_push_gives_the_same_bits(manifest, cuda_device, monkeypatch, name):
    """The parity forms' push drains a window of frontier vertices per step by default; with
    TGTP_GS_WINDOW=0 it drains one vertex at a time.  Both are the reference's sequential push:
    the FP32 form equals the golden vectors either way."""
    from tgtp_b200.aesc import AESC, AESCConfig

    monkeypatch.setenv("TGTP_GS_WINDOW", "0")
    c = golden_tgtp_case(manifest, name)
    g = _device_graph(c)
    for run in c["runs"]:
        got = AESC(g, AESCConfig(run["epsilon"], omega=c["omega"], gamma=run["gamma"])).tgtp()
        want = load_golden_scores(run)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), run
    g.free()


@pytest.mark.parametrize("window", ["0", "1"])
def test_config1_both_sequential_pushes_are_bit_exact(cuda_device, oracle_lib, config1_inputs,
                                                      monkeypatch, window):
    """On the 4,039-vertex graph (44 entries per row: the default drains one frontier vertex at a
    time) both the windowed and the one-vertex push give the oracle's FP32 and FP64 bits at
    eps = 0.005, where sources push for several rounds."""
    from tgtp_b200.aesc import AESC, AESCConfig, AESCGraph, PRECISION_FP64, VEC_F32, VEC_F64

    monkeypatch.setenv("TGTP_GS_WINDOW", window)
    c = config1_inputs
    g = AESCGraph.from_csr(c["idx"], c["adj"])
    g.upload_eigens(c["values"], c["v32"], VEC_F32)
    g.upload_eigens(c["values"], c["v64"], VEC_F64)
    got32 = AESC(g, AESCConfig(0.005)).tgtp()
    got64 = AESC(g, AESCConfig(0.005, precision=PRECISION_FP64)).tgtp()
    g.free()
    want32 = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v32"], 0.005)
    want64 = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v64"], 0.005, fp64=True)
    assert np.array_equal(got32.view(np.uint32), want32.view(np.uint32))
    assert np.array_equal(got64.view(np.uint32), want64.view(np.uint32))


@pytest.mark.parametrize("form", ["fp32", "fp64", "mixed"])
def test_run_trace_adds_up_to_the_run_counters(cuda_device, config1_inputs, form):
    """The run trace (rounds pushed per row, walk count per slot) against the run's own counters
    on the 4,039-vertex graph at eps = 0.005: the rounds of the rows that ran in the source kernel
    plus one round per closed-form row are push_rounds, the walk counts sum to walk_count, the
    walking slots are walk_edges; a row with walks pushed at least one round, and turning the
    trace off leaves the scores as they were."""
    from tgtp_b200.aesc import (AESC, AESCConfig, AESCGraph, PRECISION_FP32, PRECISION_FP64,
                                PRECISION_MIXED, VEC_F32, VEC_F64)

    c = config1_inputs
    g = AESCGraph.from_csr(c["idx"], c["adj"])
    g.upload_eigens(c["values"], c["v32"], VEC_F32)
    g.upload_eigens(c["values"], c["v64"], VEC_F64)
    prec = {"fp32": PRECISION_FP32, "fp64": PRECISION_FP64, "mixed": PRECISION_MIXED}[form]
    a = AESC(g, AESCConfig(0.005, precision=prec))
    plain = a.tgtp()
    g.set_trace(True)
    traced = a.tgtp()
    st = a.stats()
    nr, ell = g.read_trace()
    g.set_trace(False)
    assert np.array_equal(plain.view(np.uint32), traced.view(np.uint32))
    closed = int((ell == 0).sum())
    assert int(ell.sum()) + closed == st["push_rounds"]
    assert int(nr.astype(np.int64).sum()) == st["walk_count"]
    assert int((nr > 0).sum()) == st["walk_edges"] > 0
    rows = np.repeat(np.arange(c["n"]), np.diff(c["idx"].astype(np.int64)))
    assert np.all(ell[rows[nr > 0]] >= 1)
    assert np.all(nr[nr > 0] % 8 == 0)
    g.free()


def test_run_trace_is_refused_before_a_traced_run(cuda_device, config1_inputs):
    """read_trace without a traced run on the handle (trace off, or on but no run since) is an
    invalid-argument status, not stale data."""
    from tgtp_b200.aesc import AESC, AESCConfig, AESCGraph, TgtpError, VEC_F32

    c = config1_inputs
    g = AESCGraph.from_csr(c["idx"], c["adj"])
    g.upload_eigens(c["values"], c["v32"], VEC_F32)
    with pytest.raises(TgtpError) as e:
        g.read_trace()
    assert e.value.status == 1
    AESC(g, AESCConfig(0.05)).tgtp()
    g.set_trace(True)
    with pytest.raises(TgtpError):
        g.read_trace()
    AESC(g, AESCConfig(0.05)).tgtp()
    nr, ell = g.read_trace()
    assert nr.shape == (len(c["adj"]),) and ell.shape == (c["n"],)
    g.free()
