"""The drop-in executables (tgtp_b200/bin/*) on the GPU: same argv, output files and TSV rows as the
reference's tgtp / benchmark / rw_experiment_saba, with the reference's golden results."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu
BIN = os.path.join(ROOT, "tgtp_b200", "bin")


@pytest.fixture(scope="module")
def runners(tgtp_lib):
    from tgtp_b200 import build

    build.build(runners=True)
    return BIN


def test_tgtp_cli_writes_reference_scores(manifest, cuda_device, runners, tmp_path):
    for run in [r for r in manifest["tgtp"] if r["case"] in ("cl300", "sparse400")]:
        out = tmp_path / "s.bin"
        r = subprocess.run([os.path.join(runners, "tgtp"), os.path.join(GOLDEN, "tgtp"),
                            run["case"], str(run["epsilon"]), str(run["omega"]), str(run["gamma"]),
                            str(out)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        got = np.fromfile(out, dtype=np.float32)
        want = np.load(os.path.join(GOLDEN, "tgtp", run["scores"]))
        assert got.tobytes() == want.tobytes(), run


def test_tgtp_cli_fp64_form_and_errors(manifest, cuda_device, runners, tmp_path):
    run = [r for r in manifest["tgtp"] if r["case"] == "cl300"][0]
    out = tmp_path / "s.bin"
    env = dict(os.environ, TGTP_PRECISION="fp64")
    r = subprocess.run([os.path.join(runners, "tgtp"), os.path.join(GOLDEN, "tgtp"), "cl300",
                        str(run["epsilon"]), "16", "10", str(out)], capture_output=True, text=True,
                       env=env)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, dtype=np.float32)
    want = np.load(os.path.join(GOLDEN, "tgtp", run["scores"]))
    assert np.max(np.abs(got - want) / np.abs(want)) < 1e-5
    r = subprocess.run([os.path.join(runners, "tgtp"), os.path.join(GOLDEN, "tgtp"), "cl300",
                        "0.05", "400", "10", str(out)], capture_output=True, text=True)
    assert r.returncode == 1 and "omega must be between 2 and vertex count" in r.stderr


def test_benchmark_cli_tsv(manifest, cuda_device, runners):
    r = subprocess.run([os.path.join(runners, "benchmark"), "cl300", "0.05,0.01", "1,8", "2",
                        os.path.join(GOLDEN, "tgtp"), "16", "10", "1"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[0] == "sampler\tdataset\tepsilon\tthreads\trepeat\tseconds\tchecksum"
    rows = [line.split("\t") for line in lines[1:]]
    assert len(rows) == 2 * 2 * 2
    for row in rows:
        assert row[0] == "seed32-grid-multiply-high" and row[1] == "cl300"
        eps = float(row[2])
        want = np.load(os.path.join(GOLDEN, "tgtp", "cl300", f"scores_eps{row[2]}_g10.npy"))
        assert abs(float(row[6]) - float(np.sum(want.astype(np.float64)))) <= 1e-6 * abs(float(row[6]))
        assert eps in (0.05, 0.01) and float(row[5]) > 0


def test_rw_experiment_saba_cli(manifest, cuda_device, runners, tmp_path):
    import shutil

    run = [r for r in manifest["saba"] if r["graph"] == "cl300.graph.txt" and r["depth"] == 5][0]
    ds = tmp_path / "data" / "cl300"
    ds.mkdir(parents=True)
    shutil.copy(os.path.join(GOLDEN, "saba", run["graph"]), ds / "graph.txt")
    r = subprocess.run([os.path.join(runners, "rw_experiment_saba"), str(tmp_path / "data"),
                        "cl300", "5", str(run["n_walks"]), "16"], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    f = r.stdout.strip().split("\t")
    assert f[0] == "saba" and f[1] == "cl300" and f[2] == "5" and f[3] == str(run["n_walks"])
    assert float(f[12]) == pytest.approx(run["visit_count"], rel=1e-6)
    assert float(f[13]) == pytest.approx(run["checksum"], rel=1e-6)
    res = (tmp_path / "results" / "rw" / f"saba_cl300_d5_w{run['n_walks']}.txt").read_text()
    keys = [line.split(" ")[0] for line in res.strip().splitlines()]
    assert keys == ["variant", "dataset", "depth", "n_walks", "threads", "n_vertices", "n_edges",
                    "t_load_s", "t_rw_s", "total_s", "total_walks", "walks_per_sec", "visit_count",
                    "checksum"]
    r = subprocess.run([os.path.join(runners, "rw_experiment_saba"), str(tmp_path / "data"),
                        "cl300", "5", "12"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 1 and "multiple of 8" in r.stderr
