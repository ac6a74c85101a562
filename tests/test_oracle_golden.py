"""The oracle (oracle/tgtp_oracle.c) pinned against golden vectors produced by the reference's own
code (tests/golden/make_golden.py).  CPU only."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_tgtp_case, load_golden_scores

SIMPLE_CASES = ["cl300", "sparse400", "grid", "cycle9", "complete12"]
# multi300 repeats edges and holds self-loops: its scores are not symmetric slot by slot (only the
# last repeat's value lands on the reverse slot, src/aesc.h:538-545) and it has no exact fixture
TGTP_CASES = SIMPLE_CASES + ["multi300"]


def _csr_from_graph(path):
    from tgtp_b200.aesc import load_graph_txt

    return load_graph_txt(path)


def test_saba_oracle_matches_reference_counters(manifest, oracle_lib, tgtp_lib):
    for run in manifest["saba"]:
        idx, adj = _csr_from_graph(os.path.join(GOLDEN, "saba", run["graph"]))
        got = oracle_lib.saba(idx, adj, run["depth"], run["n_walks"], threads=2)
        want = np.load(os.path.join(GOLDEN, "saba", run["counts"])).astype(np.uint64)
        assert np.array_equal(got, want), run
        assert int(got.sum()) == run["visit_count"]
        assert int((got * np.arange(1, got.size + 1, dtype=np.uint64)).sum()) == run["checksum"]


@pytest.mark.parametrize("name", TGTP_CASES)
def test_tgtp_oracle_fp32_is_bit_exact_with_reference(manifest, oracle_lib, tgtp_lib, name):
    c = golden_tgtp_case(manifest, name)
    for run in c["runs"]:
        got = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v32"], run["epsilon"],
                              gamma=run["gamma"], threads=2)
        want = load_golden_scores(run)
        assert got.shape == want.shape
        bad = np.flatnonzero(got.view(np.uint32) != want.view(np.uint32))
        assert bad.size == 0, (run, bad[:10], got[bad[:5]], want[bad[:5]])


@pytest.mark.parametrize("name", TGTP_CASES)
def test_tgtp_oracle_fp64_close_to_reference(manifest, oracle_lib, tgtp_lib, name):
    """Plain FP64 form vs the reference: within 1e-6 relative, or 2 float32 ulps of the score,
    on all but a stated allowance of slots whose walk-length or walk-count decision flips."""
    c = golden_tgtp_case(manifest, name)
    for run in c["runs"]:
        got = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v64"], run["epsilon"],
                              gamma=run["gamma"], fp64=True, threads=2)
        want = load_golden_scores(run)
        tol = np.maximum(1e-6 * np.abs(want), 2 * np.spacing(np.abs(want)))
        bad = np.abs(got.astype(np.float64) - want) > tol
        assert bad.mean() <= 0.01, (run, int(bad.sum()))


@pytest.mark.parametrize("name", SIMPLE_CASES)
def test_reference_scores_are_symmetric_and_sane(manifest, tgtp_lib, name):
    c = golden_tgtp_case(manifest, name)
    idx, adj = c["idx"], c["adj"]
    rows = np.repeat(np.arange(len(idx) - 1), np.diff(idx.astype(np.int64)))
    key = rows.astype(np.int64) * len(idx) + adj
    rkey = adj.astype(np.int64) * len(idx) + rows
    order = np.argsort(key)
    rev = order[np.searchsorted(key[order], rkey)]
    for run in c["runs"]:
        s = load_golden_scores(run)
        assert np.array_equal(s, s[rev])
        assert np.all(np.isfinite(s))


def test_oracle_eigen_parse_matches_reference(manifest, oracle_lib):
    e = manifest["eigens"][0]
    folder = os.path.join(GOLDEN, "eigens")
    vals, v32, v64 = oracle_lib.parse_eigens(os.path.join(folder, e["eigens"]), e["n"], e["omega"])
    want = np.load(os.path.join(folder, e["parsed"]))
    assert np.array_equal(vals, want["values"])
    assert np.array_equal(v32.view(np.uint32), want["vectors"].view(np.uint32))
    # vertex 2 of eigenvector 0 is the float-midpoint token: parsed straight to float it rounds
    # up, through double it would round to even (down), so the fixture really pins strtof
    k = 2 * e["omega"] + 0
    assert v32[k] == np.nextafter(np.float32(1), np.float32(2))
    assert np.float32(v64[k]) == np.float32(1)


def test_oracle_saba_rejects_partial_bouquets(oracle_lib, tgtp_lib):
    idx, adj = _csr_from_graph(os.path.join(GOLDEN, "saba", "cl300.graph.txt"))
    with pytest.raises(ValueError):
        oracle_lib.saba(idx, adj, 3, 12)


def test_sampled_exact_matches_dense_exact():
    """The sampled-edge oracle (block PCG) against the dense solve on a graph both can handle."""
    from oracle import exact_sc
    from tgtp_b200 import synth

    g = synth.chung_lu(800, 4000, 2.3, 3)
    idx, adj = g.csr()
    exact = exact_sc.exact_scores(idx, adj)
    slots = np.random.default_rng(0).choice(len(adj), 200, replace=False)
    got = exact_sc.sampled_scores(idx, adj, slots)
    assert np.max(np.abs(got - exact[slots])) < 1e-9


def _csr(n, edges):
    rows = [[] for _ in range(n)]
    for u, v in edges:
        rows[u].append(v)
        rows[v].append(u)
    idx = np.zeros(n + 1, np.uint32)
    idx[1:] = np.cumsum([len(r) for r in rows])
    adj = np.array([x for r in rows for x in sorted(r)], np.uint32)
    return idx, adj


def test_exact_oracle_known_answers():
    """Closed forms of the effective resistance of an edge: (n-1)/n on the cycle C_n, 2/n on K_n,
    1 on every edge of a tree; Foster's theorem (the resistances of all edges sum to n - 1) on a
    random graph; the sampled-edge oracle gives the same values."""
    from oracle import exact_sc
    from tgtp_b200 import synth

    n = 9
    idx, adj = _csr(n, [(k, (k + 1) % n) for k in range(n)])
    assert np.allclose(exact_sc.exact_scores(idx, adj), (n - 1) / n, rtol=0, atol=1e-12)
    assert np.allclose(exact_sc.sampled_scores(idx, adj, np.arange(len(adj))), (n - 1) / n,
                       rtol=0, atol=1e-9)
    n = 12
    idx, adj = _csr(n, [(x, y) for x in range(n) for y in range(x + 1, n)])
    assert np.allclose(exact_sc.exact_scores(idx, adj), 2 / n, rtol=0, atol=1e-12)
    rng = np.random.default_rng(1)
    n = 50
    idx, adj = _csr(n, [(k, int(rng.integers(0, k))) for k in range(1, n)])
    assert np.allclose(exact_sc.exact_scores(idx, adj), 1.0, rtol=0, atol=1e-12)
    g = synth.chung_lu(300, 1500, 2.3, 5)
    idx, adj = g.csr()
    exact = exact_sc.exact_scores(idx, adj)
    assert abs(exact.sum() / 2 - (g.n - 1)) < 1e-9 * g.n


def test_reference_scores_on_complete_graph_are_within_eps_of_2_over_n(manifest):
    """The reference's own scores on K_12 against the closed form 2/n, at every golden epsilon."""
    c = golden_tgtp_case(manifest, "complete12")
    n = len(c["idx"]) - 1
    for run in c["runs"]:
        s = load_golden_scores(run).astype(np.float64)
        assert np.max(np.abs(s - 2 / n)) <= run["epsilon"], run


@pytest.fixture(scope="module")
def omega128_case(tmp_path_factory):
    """A Chung-Lu graph (1,200 vertices, 9,000 edges) with 128 eigenpairs in the reference's file
    layout, for the reference binary and the oracle."""
    from tgtp_b200 import eigenprep, synth
    from tgtp_b200.aesc import load_eigens_txt

    root = tmp_path_factory.mktemp("omega128")
    g = synth.chung_lu(1200, 9000, 2.4, 21)
    (root / "g").mkdir()
    synth.write_graph_txt(g, str(root / "g" / "graph.txt"))
    path = eigenprep.eigenprep_folder(str(root / "g"), 128)
    idx, adj = g.csr()
    values, v32, v64 = load_eigens_txt(path, g.n, 128)
    return dict(root=root, idx=idx, adj=adj, values=values, v32=v32, v64=v64)


@pytest.mark.parametrize("eps", [0.05, 0.01, 0.005])
def test_oracle_matches_the_reference_binary_at_omega_128(omega128_case, oracle_lib, tgtp_lib,
                                                          eps):
    """The golden fixtures use omega <= 16; at the path's omega = 128 the reference's own tgtp
    (oracle/_ref/tgtp_O2, run here) pins the oracle: FP32 bit-exact, FP64 within 1e-6 relative
    (or 2 float32 ulps) on every slot."""
    import subprocess

    from conftest import ROOT

    exe = os.path.join(ROOT, "oracle", "_ref", "tgtp_O2")
    if not os.path.exists(exe):
        pytest.skip("the reference binaries are not built (oracle/_ref)")
    c = omega128_case
    out = c["root"] / f"scores_{eps}.bin"
    r = subprocess.run([exe, str(c["root"]), "g", str(eps), "128", "10", str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    want = np.fromfile(out, dtype=np.float32)
    got, det = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v32"], eps, gamma=10,
                               details=True)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    if eps == 0.005:
        assert det["stats"]["walk_hops"] > 0  # the walk phase is part of what is pinned
    got64 = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], c["v64"], eps, gamma=10, fp64=True)
    tol = np.maximum(1e-6 * np.abs(want), 2 * np.spacing(np.abs(want)))
    assert np.all(np.abs(got64.astype(np.float64) - want) <= tol)
    # the paper's -Ofast build reassociates the omega sums: not bit-equal, within 1e-6 relative
    fast_exe = os.path.join(ROOT, "oracle", "_ref", "tgtp")
    if os.path.exists(fast_exe):
        fast_out = c["root"] / f"scores_fast_{eps}.bin"
        r = subprocess.run([fast_exe, str(c["root"]), "g", str(eps), "128", "10", str(fast_out)],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        fast = np.fromfile(fast_out, dtype=np.float32).astype(np.float64)
        assert np.all(np.abs(got.astype(np.float64) - fast) <= 1e-6 * np.abs(fast))


@pytest.mark.parametrize("graph,depth,walks", [("config1", 5, 2048), ("rmat14", 10, 64)])
def test_saba_oracle_matches_the_reference_walks_at_benchmark_size(tmp_path, oracle_lib, tgtp_lib,
                                                                  graph, depth, walks):
    """The SABA walk configuration of the benchmark (the 4,039-vertex graph, depth 5, 2,048 walks)
    and an R-MAT scale-14 graph: every counter of the oracle equal to the reference's own walk
    routine (oracle/_ref/saba_harness_O2, run here; its float counters stay below 2^24 here)."""
    import subprocess

    from conftest import ROOT
    from tgtp_b200 import synth

    exe = os.path.join(ROOT, "oracle", "_ref", "saba_harness_O2")
    if not os.path.exists(exe):
        pytest.skip("the reference binaries are not built (oracle/_ref)")
    g = synth.config1_graph(1) if graph == "config1" else synth.rmat(14, 8, 0.57, 0.19, 0.19, 3)
    synth.write_graph_txt(g, str(tmp_path / "graph.txt"))
    out = tmp_path / "counts.u32"
    r = subprocess.run([exe, str(tmp_path / "graph.txt"), str(depth), str(walks), str(out)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    want = np.fromfile(out, dtype=np.uint32).astype(np.uint64)
    idx, adj = g.csr()
    got = oracle_lib.saba(idx, adj, depth, walks)
    assert np.array_equal(got, want)
    n, m, visits, checksum = (int(x) for x in r.stdout.split())
    assert (n, m) == (g.n, len(adj)) and visits == int(got.sum())
    assert checksum == int((got * np.arange(1, n + 1, dtype=np.uint64)).sum())


@pytest.mark.parametrize("name", SIMPLE_CASES)
def test_exact_oracle_matches_the_reference_accuracy_script(manifest, name):
    """oracle/exact_sc.py against the exact scores of the reference's scripts/paper_accuracy.py
    (tests/golden/exact/, made by tests/golden/make_exact.py) on the golden graphs."""
    from oracle import exact_sc

    c = golden_tgtp_case(manifest, name)
    want = np.load(os.path.join(GOLDEN, "exact", f"{name}.npy"))
    got = exact_sc.exact_scores(c["idx"], c["adj"])
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) < 1e-12


def test_oracle_does_not_depend_on_its_thread_count(manifest, oracle_lib):
    """Like the reference (each source writes only its own row; walk seeds come from the grid),
    the oracle's scores and SABA counters are the same bits on 1 and 4 threads."""
    c = golden_tgtp_case(manifest, "cl300")
    for fp64 in (False, True):
        vec = c["v64"] if fp64 else c["v32"]
        a = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], vec, 0.005, fp64=fp64, threads=1)
        b = oracle_lib.tgtp(c["idx"], c["adj"], c["values"], vec, 0.005, fp64=fp64, threads=4)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(oracle_lib.saba(c["idx"], c["adj"], 5, 64, threads=1),
                          oracle_lib.saba(c["idx"], c["adj"], 5, 64, threads=4))


def test_saba_rmat18_fixture_is_reproduced_by_the_oracle(oracle_lib):
    """tests/golden/saba_rmat18.json (the R-MAT scale-18 walk counters the GPU tests compare with):
    the graph generator still gives the graph it was made on, every cell's visit count is n * W * D,
    and the oracle reproduces the benchmark cell (depth 5, 2,048 walks) hash for hash, the cell
    where the fixture holds the reference's own counters."""
    import json

    from make_saba_rmat18 import CELLS, graph_fingerprint, sha256_u32

    from tgtp_b200 import synth

    with open(os.path.join(GOLDEN, "saba_rmat18.json")) as f:
        fx = json.load(f)
    g = synth.config3_graph(1)
    idx, adj = g.csr()
    assert graph_fingerprint(idx, adj) == fx["fingerprint"]
    assert sorted((c["depth"], c["n_walks"]) for c in fx["cells"]) == sorted(CELLS)
    for c in fx["cells"]:
        assert c["visit_count"] == g.n * c["n_walks"] * c["depth"]
        assert c["max_counter"] < 2**32
    cell = [c for c in fx["cells"] if (c["depth"], c["n_walks"]) == (5, 2048)][0]
    assert cell["source"].startswith("reference")
    got = oracle_lib.saba(idx, adj, 5, 2048)
    assert sha256_u32(got) == cell["counters_sha256"]
    assert int((got * np.arange(1, g.n + 1, dtype=np.uint64)).sum()) == cell["checksum"]


def test_mt19937_restatement_known_answers(oracle_lib):
    """std::mt19937 restated in the oracle: the C++ standard's check value (the 10,000th draw of the
    default seed 5489 is 4123659995) and the first draws of the walk runners' seed 42."""
    assert oracle_lib.mt19937_nth(5489, 10000) == 4123659995
    assert oracle_lib.mt19937_nth(5489, 1) == 3499211612
    assert [oracle_lib.mt19937_nth(42, k) for k in (1, 2, 3)] == [1608637542, 3421126067, 4083286876]


@pytest.mark.parametrize("simd", [False, True])
@pytest.mark.parametrize("graph,depth,walks", [("config1", 5, 64), ("rmat14", 10, 24),
                                               ("rmat12", 100, 8), ("rmat12", 700, 8)])
def test_mt_walk_oracle_matches_the_reference_walks(tmp_path, oracle_lib, tgtp_lib, simd, graph,
                                                    depth, walks):
    """The MT19937 walk baselines: every counter of the oracle equal to the reference's own walk
    routine (scalar_randomwalk / simd_randomwalk, run by oracle/_ref/mt_harness_O2 and
    mt_simd_harness_O2 with std::mt19937 reseeded to 42 + src as the runners do)."""
    import subprocess

    from conftest import ROOT
    from tgtp_b200 import synth

    exe = os.path.join(ROOT, "oracle", "_ref", "mt_simd_harness_O2" if simd else "mt_harness_O2")
    if not os.path.exists(exe):
        pytest.skip("the reference binaries are not built (oracle/_ref)")
    g = {"config1": lambda: synth.config1_graph(1),
         "rmat14": lambda: synth.rmat(14, 8, 0.57, 0.19, 0.19, 3),
         "rmat12": lambda: synth.rmat(12, 8, 0.57, 0.19, 0.19, 5)}[graph]()
    synth.write_graph_txt(g, str(tmp_path / "graph.txt"))
    out = tmp_path / "counts.u32"
    r = subprocess.run([exe, str(tmp_path / "graph.txt"), str(depth), str(walks), str(out)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    want = np.fromfile(out, dtype=np.uint32).astype(np.uint64)
    idx, adj = g.csr()
    got = oracle_lib.mt_walks(idx, adj, depth, walks, simd=simd)
    assert np.array_equal(got, want)
    n, m, visits, checksum = (int(x) for x in r.stdout.split())
    assert (n, m) == (g.n, len(adj)) and visits == int(got.sum())
    assert checksum == int((got * np.arange(1, n + 1, dtype=np.uint64)).sum())


@pytest.mark.parametrize("simd", [False, True])
def test_mt_walk_oracle_does_not_depend_on_its_thread_count(oracle_lib, simd):
    """Every source reseeds its own generator, so the counters are the same however the sources are
    spread over threads (the reference's OpenMP loop relies on the same property)."""
    from tgtp_b200 import synth

    g = synth.rmat(12, 8, 0.57, 0.19, 0.19, 5)
    idx, adj = g.csr()
    one = oracle_lib.mt_walks(idx, adj, 7, 24, simd=simd, threads=1)
    four = oracle_lib.mt_walks(idx, adj, 7, 24, simd=simd, threads=4)
    assert np.array_equal(one, four)
    assert int(one.sum()) == int((np.diff(idx.astype(np.int64)) > 0).sum()) * 24 * 7


def _mt_fixture():
    import json

    with open(os.path.join(GOLDEN, "mt_walks.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("case", range(8))
def test_mt_walk_oracle_matches_the_committed_reference_counters(oracle_lib, case):
    """The oracle's MT19937 walks against tests/golden/mt_walks.json (the reference's own walk
    routines, run by tests/golden/make_mt_walks.py): every counter, by SHA-256 of the array, so the
    pin holds where the reference binaries are not built."""
    from make_mt_walks import graph
    from make_saba_rmat18 import graph_fingerprint, sha256_u32

    c = _mt_fixture()["cases"][case]
    g = graph(c["graph"])
    idx, adj = g.csr()
    assert graph_fingerprint(idx, adj) == c["graph_fingerprint"]
    got = oracle_lib.mt_walks(idx, adj, c["depth"], c["n_walks"], simd=c["simd"])
    assert int(got.sum()) == c["visit_count"]
    assert int((got * np.arange(1, g.n + 1, dtype=np.uint64)).sum()) == c["checksum"]
    assert sha256_u32(got.astype(np.uint32)) == c["counters_sha256"]
