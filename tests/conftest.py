"""Shared fixtures.  `-m gpu` tests need a CUDA device and call the library through its C ABI;
everything else runs on the CPU (oracle vs golden vectors, host-side loaders, symbol table, the
multi-process host logic)."""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)  # the fixture generators' helpers (hashes, fingerprints)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the sm_100a library")


@pytest.fixture(scope="session")
def manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    oracle.build(reference=False)
    return oracle


@pytest.fixture(scope="session")
def tgtp_lib():
    """libtgtp_gpu.so, built in-tree if it is missing or stale (host code only is exercised on CPU)."""
    from tgtp_b200 import build

    build.build(runners=False)
    from tgtp_b200 import _lib

    return _lib.lib()


@pytest.fixture(scope="session")
def cuda_device(tgtp_lib):
    """A CUDA device for the gpu tests; the GPU tests fail (not skip) without one."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("gpu test run without a CUDA device")
    torch.cuda.init()
    return 0


def golden_tgtp_case(manifest, name):
    folder = os.path.join(GOLDEN, "tgtp", name)
    from tgtp_b200 import synth  # noqa: F401  (package import check)
    import oracle

    runs = [r for r in manifest["tgtp"] if r["case"] == name]
    n, omega = runs[0]["n"], runs[0]["omega"]
    from tgtp_b200.aesc import load_graph_txt

    idx, adj = load_graph_txt(os.path.join(folder, "graph.txt"))
    values, v32, v64 = oracle.parse_eigens(os.path.join(folder, f"sorted_eigens_{omega}.txt"), n,
                                           omega)
    return dict(folder=folder, idx=idx, adj=adj, values=values, v32=v32, v64=v64, runs=runs,
                n=n, omega=omega)


def load_golden_scores(run):
    return np.load(os.path.join(GOLDEN, "tgtp", run["scores"]))


@pytest.fixture(scope="session")
def config1_inputs():
    """Chung-Lu n=4,039 with 128 eigenpairs written and parsed back like the reference's files."""
    from tgtp_b200 import eigenprep, synth
    from tgtp_b200.aesc import load_eigens_txt

    g = synth.config1_graph(1)
    d = tempfile.mkdtemp(prefix="tgtp_cfg1_")
    synth.write_graph_txt(g, os.path.join(d, "graph.txt"))
    path = eigenprep.eigenprep_folder(d, 128)
    idx, adj = g.csr()
    values, v32, v64 = load_eigens_txt(path, g.n, 128)
    return dict(idx=idx, adj=adj, values=values, v32=v32, v64=v64, n=g.n, folder=d)
