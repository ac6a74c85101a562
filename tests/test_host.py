"""Host side of the library on the CPU: the C ABI loads and exports every entry point the header
declares; the graph and eigen readers reproduce the reference's loaders (golden dumps from
src/graph.h and src/aesc.h); the synthetic generators are deterministic simple graphs."""
from __future__ import annotations

import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "tgtp_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tgtp_\w+|saba_\w+|mt_walk_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(tgtp_lib):
    from tgtp_b200 import _lib

    names = _declared_functions()
    assert len(names) >= 19
    for name in names:
        assert hasattr(tgtp_lib, name), name
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)
    assert tgtp_lib.tgtp_abi_version() == 1


@pytest.mark.parametrize("case", ["comments", "selfloop_dup", "isolated_gap", "unsorted",
                                  "bad_negative", "bad_single", "bad_text", "empty"])
def test_graph_loader_matches_reference_loader(manifest, tgtp_lib, case):
    from tgtp_b200.aesc import TgtpError, load_graph_txt

    entry = [e for e in manifest["loader"] if e["case"] == case][0]
    path = os.path.join(GOLDEN, "loader", entry["file"])
    if entry["ok"]:
        idx, adj = load_graph_txt(path)
        want = np.load(os.path.join(GOLDEN, "loader", entry["csr"]))
        assert np.array_equal(idx, want["idx"]) and np.array_equal(adj, want["adj"])
    else:
        with pytest.raises(TgtpError) as e:
            load_graph_txt(path)
        assert e.value.message == entry["error"].replace("{path}", path)


def test_graph_loader_missing_file(tgtp_lib):
    from tgtp_b200.aesc import TgtpError, load_graph_txt

    with pytest.raises(TgtpError) as e:
        load_graph_txt("/nonexistent/graph.txt")
    assert e.value.status == 5 and "cannot open graph" in e.value.message


def test_eigen_loader_matches_reference_loader(manifest, tgtp_lib):
    from tgtp_b200.aesc import load_eigens_txt

    e = manifest["eigens"][0]
    folder = os.path.join(GOLDEN, "eigens")
    vals, v32, v64 = load_eigens_txt(os.path.join(folder, e["eigens"]), e["n"], e["omega"])
    want = np.load(os.path.join(folder, e["parsed"]))
    assert np.array_equal(vals, want["values"])
    assert np.array_equal(v32.view(np.uint32), want["vectors"].view(np.uint32))


def test_eigen_loader_rejects_short_and_nonfinite(tmp_path, tgtp_lib):
    from tgtp_b200.aesc import TgtpError, load_eigens_txt

    p = tmp_path / "e.txt"
    p.write_text("1 0.5 0.5\n")
    with pytest.raises(TgtpError):
        load_eigens_txt(str(p), 2, 2)
    p.write_text("1 0.5 nan\n0.5 1 1\n")
    with pytest.raises(TgtpError):
        load_eigens_txt(str(p), 2, 2)


def _eigen_text(n, omega, seed):
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(omega):
        x = rng.standard_normal(n) * 10.0 ** rng.integers(-30, 3, n)
        rows.append(" ".join(["%.17g" % (1 - i / omega)] + ["%.17g" % v for v in x.tolist()]))
    return rows


def test_eigen_loader_parallel_chunks_agree_with_sequential_reading(tmp_path, tgtp_lib, oracle_lib):
    """A 19 MB eigen file is read in many chunks on several threads: the same bits as the oracle's
    sequential parser, the first bad number in file order decides the error (eigenvalue or
    eigenvector), a file that ends early is rejected, and text after the numbers that are needed
    is never examined."""
    from tgtp_b200.aesc import TgtpError, load_eigens_txt

    n, omega = 50000, 16
    rows = _eigen_text(n, omega, 5)
    path = tmp_path / "sorted_eigens_16.txt"
    path.write_text("\n".join(rows) + "\n")
    assert path.stat().st_size > 16 << 20
    got = load_eigens_txt(str(path), n, omega)
    want = oracle_lib.parse_eigens(str(path), n, omega)
    for x, y in zip(got, want):
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8))
    # glued numbers ("a-b") are two numbers, read the same way
    glued = list(rows)
    toks = glued[7].split(" ")
    glued[7] = " ".join(toks[:100] + [toks[100] + "-0.25"] + toks[102:])
    path.write_text("\n".join(glued) + "\n")
    got = load_eigens_txt(str(path), n, omega)
    want = oracle_lib.parse_eigens(str(path), n, omega)
    for x, y in zip(got, want):
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8))

    def rejected(text, message):
        path.write_text(text)
        with pytest.raises(TgtpError) as e:
            load_eigens_txt(str(path), n, omega)
        assert e.value.message == f"{message} in {path}"

    def with_token(rs, r, j, tok):
        rs = list(rs)
        t = rs[r].split(" ")
        t[j] = tok
        rs[r] = " ".join(t)
        return rs

    rejected("\n".join(with_token(rows, 14, 40000, "abc")) + "\n", "invalid eigenvector")
    rejected("\n".join(with_token(rows, 3, 17, "1e999")) + "\n", "invalid eigenvector")
    both = with_token(with_token(rows, 12, 0, "x"), 14, 5, "y")
    rejected("\n".join(both) + "\n", "invalid eigenvalue")
    early = with_token(with_token(rows, 14, 5, "y"), 12, 30000, "x")
    rejected("\n".join(early) + "\n", "invalid eigenvector")
    rejected("\n".join(rows[:10]) + "\n", "invalid eigenvalue")
    rejected("\n".join(rows[:15]) + "\n" + " ".join(rows[15].split(" ")[:20000]),
             "invalid eigenvector")
    path.write_text("\n".join(rows) + "\nnot numbers after the last pair 1e999 nan\n")
    got = load_eigens_txt(str(path), n, omega)
    want = oracle_lib.parse_eigens(str(path), n, omega)
    for x, y in zip(got, want):
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8))


def test_eigen_loader_agrees_with_oracle_parser_on_golden_files(manifest, tgtp_lib, oracle_lib):
    from tgtp_b200.aesc import load_eigens_txt

    for case in {r["case"]: r for r in manifest["tgtp"]}.values():
        path = os.path.join(GOLDEN, "tgtp", case["case"], f"sorted_eigens_{case['omega']}.txt")
        a = load_eigens_txt(path, case["n"], case["omega"])
        b = oracle_lib.parse_eigens(path, case["n"], case["omega"])
        for x, y in zip(a, b):
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8))


def test_synthetic_generators_are_seeded_simple_connected():
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components

    from tgtp_b200 import synth

    for make in (lambda s: synth.chung_lu(500, 3000, 2.3, s),
                 lambda s: synth.rmat(9, 8, 0.57, 0.19, 0.19, s),
                 lambda s: synth.grid_chords(12, 15, 6.0, s)):
        g1, g2, g3 = make(1), make(1), make(2)
        assert np.array_equal(g1.u, g2.u) and np.array_equal(g1.v, g2.v)
        assert not (np.array_equal(g1.u, g3.u) and np.array_equal(g1.v, g3.v))
        assert np.all(g1.u < g1.v)
        key = g1.u * g1.n + g1.v
        assert np.unique(key).size == key.size
        a = coo_matrix((np.ones(g1.num_edges), (g1.u, g1.v)), shape=(g1.n, g1.n))
        assert connected_components(a, directed=False)[0] == 1
        idx, adj = g1.csr()
        assert idx[-1] == 2 * g1.num_edges and np.all(np.diff(idx.astype(np.int64)) > 0)


def test_config1_graph_shape():
    from tgtp_b200 import synth

    g = synth.config1_graph(1)
    assert g.n == 4039 and g.num_edges == 88234


def test_eigenprep_pairs_are_eigenpairs_of_the_random_walk_matrix(tmp_path):
    """x = D^-1/2 v * sqrt(2m) for A_hat v = lambda v  <=>  D^-1 A x = lambda x."""
    from tgtp_b200 import eigenprep, synth

    g = synth.chung_lu(200, 1200, 2.5, 3)
    synth.write_graph_txt(g, str(tmp_path / "graph.txt"))
    path = eigenprep.eigenprep_folder(str(tmp_path), 12)
    rows = np.loadtxt(path)
    vals, vecs = rows[:, 0], rows[:, 1:]
    idx, adj = g.csr()
    deg = np.diff(idx.astype(np.int64))
    assert np.all(np.diff(np.abs(vals)) <= 1e-12)
    assert abs(vals[0] - 1) < 1e-8
    for lam, x in zip(vals, vecs):
        ax = np.add.reduceat(x[adj], idx[:-1]) / deg
        assert np.max(np.abs(ax - lam * x)) < 1e-5 * np.max(np.abs(x))
    assert (tmp_path / "stat.txt").read_text().startswith("n=200\nm=")


def test_gpu_eigen_prep_solver_matches_the_scipy_restatement_on_cpu():
    """The Chebyshev-filtered subspace iteration of eigenprep_gpu, run with torch on the CPU: the
    same eigenvalues as the scipy (Lanczos) restatement, sorted by |lambda| descending, each vector
    an eigenvector of D^-1 A with sum_i deg_i x_i^2 = 2m, equal to scipy's up to sign (the
    eigenvalues of this graph are separated by at least 2.9e-3)."""
    from tgtp_b200 import eigenprep, eigenprep_gpu, synth

    g = synth.chung_lu(600, 3000, 2.3, 9)
    v1, x1, _ = eigenprep.compute(g.n, g.u, g.v, 16, seed=0)
    v2, x2, m, _, worst = eigenprep_gpu.compute(g.n, g.u, g.v, 16, seed=1, tol=1e-10,
                                                device="cpu")
    assert worst < 1e-10
    assert np.max(np.abs(v1 - v2)) < 1e-10
    assert np.all(np.diff(np.abs(v2)) <= 1e-12)
    idx, adj = g.csr()
    deg = np.diff(idx.astype(np.int64)).astype(np.float64)
    for lam, x, y in zip(v2, x2, x1):
        ax = np.add.reduceat(x[adj], idx[:-1]) / deg
        assert np.max(np.abs(ax - lam * x)) < 1e-8 * np.max(np.abs(x))
        assert abs(np.dot(deg, x * x) - 2 * m) < 1e-8 * m
        cos = np.dot(deg, x * y) / np.sqrt(np.dot(deg, x * x) * np.dot(deg, y * y))
        assert abs(abs(cos) - 1) < 1e-8


def test_input_cache_reuses_parsed_inputs_and_follows_the_text(tmp_path, monkeypatch, manifest, tgtp_lib):
    """TGTP_INPUT_CACHE=1: the loaders write '<file>.tgtpcache' beside the text, later loads read
    it and give the same arrays, and a change of the text file invalidates it."""
    import shutil

    from conftest import golden_tgtp_case
    from tgtp_b200.aesc import load_eigens_txt, load_graph_txt

    c = golden_tgtp_case(manifest, "cl300")
    gpath = tmp_path / "graph.txt"
    epath = tmp_path / f"sorted_eigens_{c['omega']}.txt"
    shutil.copy(os.path.join(c["folder"], "graph.txt"), gpath)
    shutil.copy(os.path.join(c["folder"], f"sorted_eigens_{c['omega']}.txt"), epath)
    plain_g = load_graph_txt(str(gpath))
    plain_e = load_eigens_txt(str(epath), c["n"], c["omega"])
    assert not (tmp_path / "graph.txt.tgtpcache").exists()
    monkeypatch.setenv("TGTP_INPUT_CACHE", "1")
    for _ in range(2):  # the first call writes the caches, the second reads them
        g = load_graph_txt(str(gpath))
        e = load_eigens_txt(str(epath), c["n"], c["omega"])
        assert all(np.array_equal(a, b) for a, b in zip(g, plain_g))
        assert all(np.array_equal(a, b) for a, b in zip(e, plain_e))
        assert (tmp_path / "graph.txt.tgtpcache").exists()
        assert (tmp_path / f"sorted_eigens_{c['omega']}.txt.tgtpcache").exists()
    # an edited text file is parsed again (its size and time no longer match the cache)
    with open(gpath, "a") as f:
        f.write(f"0 {c['n'] - 1}\n")
    g2 = load_graph_txt(str(gpath))
    assert int(g2[0][-1]) == int(plain_g[0][-1]) + 2  # the loader mirrors and keeps every line


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """Without the built library there is no fallback: the first call raises."""
    from tgtp_b200 import _lib

    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "libtgtp_gpu.so"))
    with pytest.raises(RuntimeError, match="is missing"):
        _lib.lib()
