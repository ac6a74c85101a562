"""Generate the golden vectors under tests/golden/ from the reference itself.

The reference ships no fixtures, so these are produced by running the reference's own code, compiled
from its sources (oracle/Makefile -> oracle/_ref/):
  * saba/     per-vertex SABA counters from the reference's saba_randomwalk
              (oracle/ref_saba_harness.cpp around src/rw_experiment_saba.cpp:65-145);
  * tgtp/     float32 CSR scores written by the reference `tgtp` CLI (src/main.cpp) at -O2;
  * loader/   the CSR that src/graph.h:29-97 builds for edge-case edge lists, or its error;
  * eigens/   the values/vectors that src/aesc.h:51-64 parses, including a token where parsing
              straight to float differs from parsing to double and rounding.
Graphs and eigenpairs are seeded synthetic inputs (tgtp_b200.synth, tgtp_b200.eigenprep).

Run where the reference checkout is present (TGTP_REFERENCE, default /root/reference) and the
oracle/_ref binaries are built from it:
    python tests/golden/make_golden.py                    # every case
    python tests/golden/make_golden.py --cases multi300   # only the named multigraph tgtp cases
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tgtp_b200 import eigenprep, synth  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")


def circulant(n: int, offsets) -> synth.EdgeList:
    u, v = [], []
    for i in range(n):
        for o in offsets:
            u.append(i)
            v.append((i + o) % n)
    a, b = np.minimum(u, v), np.maximum(u, v)
    key = np.unique(np.asarray(a) * n + np.asarray(b))
    return synth.EdgeList(n, key // n, key % n, f"circulant{n}")


def complete(n: int) -> synth.EdgeList:
    u, v = np.triu_indices(n, 1)
    return synth.EdgeList(n, u.astype(np.int64), v.astype(np.int64), f"complete{n}")


def cycle(n: int) -> synth.EdgeList:
    u = np.arange(n)
    v = (u + 1) % n
    a, b = np.minimum(u, v), np.maximum(u, v)
    return synth.EdgeList(n, a.astype(np.int64), b.astype(np.int64), f"cycle{n}")


SABA_CASES = {
    "cl300": (lambda: synth.chung_lu(300, 2000, 2.5, 11), [(5, 2048), (3, 24), (15, 16)]),
    "circ16": (lambda: circulant(200, range(1, 9)), [(10, 64), (12, 8)]),
    "rmat10": (lambda: synth.rmat(10, 8, 0.57, 0.19, 0.19, 3), [(5, 2048), (15, 16)]),
}
# the loader keeps self-loops and duplicates and leaves isolated ids; SABA skips isolated sources
SABA_RAW = {
    "multi": ("# comment\n0 1\n1 2\n2 0\n2 3\n3 5\n5 6\n6 3\n1 1\n2 3\n", [(4, 16), (9, 64)]),
}

TGTP_CASES = {
    # name: (graph, omega, [(eps, gamma)])
    "cl300": (lambda: synth.chung_lu(300, 2000, 2.5, 11), 16,
              [(0.05, 10), (0.01, 10), (0.005, 10), (0.01, 1), (0.01, 40)]),
    "sparse400": (lambda: synth.chung_lu(400, 700, 2.1, 5), 16,
                  [(0.05, 10), (0.01, 10), (0.005, 10), (0.005, 3)]),
    "grid": (lambda: synth.grid_chords(10, 12, 5.0, 2), 8, [(0.05, 10), (0.01, 10), (0.01, 2)]),
    "cycle9": (lambda: cycle(9), 4, [(0.05, 10), (0.01, 3)]),
    "complete12": (lambda: complete(12), 6, [(0.05, 10), (0.005, 10)]),
}



def multigraph_text() -> str:
    """The cl300 graph with 12 of its edges listed again and 5 self-loops: the loader keeps both
    (src/graph.h:63-66, 75-78), so rows repeat neighbours and hold their own vertex."""
    g = synth.chung_lu(300, 2000, 2.5, 11)
    rng = np.random.default_rng(17)
    lines = [f"{a} {b}" for a, b in zip(g.u.tolist(), g.v.tolist())]
    for e in rng.choice(len(lines), 12, replace=False):
        lines.append(lines[e])
    for v in rng.choice(g.n, 5, replace=False):
        lines.append(f"{v} {v}")
    return "\n".join(lines) + "\n"


# multigraph cases: (text of graph.txt, eigenpairs of this simple graph, omega, runs); the
# eigenpairs are inputs only, so they come from the simple graph the text extends
TGTP_RAW = {
    "multi300": (multigraph_text, lambda: synth.chung_lu(300, 2000, 2.5, 11), 16,
                 [(0.05, 10), (0.01, 10), (0.005, 10), (0.01, 1)]),
}

LOADER_CASES = {
    "comments": "# header\n% other\n0 1\n\n   \n  # indented comment\n1 2 extra tokens\n2 0\r\n",
    "selfloop_dup": "0 1\n1 1\n0 1\n1 2\n2 0\n",
    "isolated_gap": "0 1\n1 3\n3 0\n",
    "unsorted": "4 0\n3 1\n2 0\n1 0\n4 2\n3 2\n",
    "bad_negative": "0 1\n-1 2\n",
    "bad_single": "0 1\n7\n",
    "bad_text": "0 1\nx y\n",
    "empty": "# nothing\n\n",
}


def run(cmd, **kw):
    return subprocess.run(cmd, check=True, capture_output=True, text=True, **kw)


def tgtp_runs(name, folder, omega, n, runs, manifest):
    """The reference's tgtp (-O2) on folder/graph.txt for each (eps, gamma); scores saved as .npy."""
    for eps, gamma in runs:
        out = os.path.join(folder, f"scores_eps{eps}_g{gamma}.f32")
        run([os.path.join(REF, "tgtp_O2"), os.path.join(HERE, "tgtp"), name, str(eps),
             str(omega), str(gamma), out], env=dict(os.environ, OMP_NUM_THREADS="2"))
        s = np.fromfile(out, dtype=np.float32)
        os.remove(out)
        np.save(out.replace(".f32", ".npy"), s)
        manifest["tgtp"].append(dict(case=name, omega=omega, epsilon=eps, gamma=gamma,
                                     n=int(n), m=int(s.size),
                                     scores=os.path.join(name, os.path.basename(
                                         out.replace(".f32", ".npy")))))


def raw_tgtp_case(name, manifest):
    text, simple, omega, runs = TGTP_RAW[name]
    folder = os.path.join(HERE, "tgtp", name)
    shutil.rmtree(folder, ignore_errors=True)
    os.makedirs(folder)
    with open(os.path.join(folder, "graph.txt"), "w") as f:
        f.write(text())
    g = simple()
    vals, vecs, m = eigenprep.compute(g.n, g.u, g.v, omega, seed=0)
    eigenprep.write_files(folder, g.n, m, vals, vecs)
    tgtp_runs(name, folder, omega, g.n, runs, manifest)


def main():
    for need in ("tgtp_O2", "saba_harness_O2", "ref_load_dump"):
        if not os.access(os.path.join(REF, need), os.X_OK):
            sys.exit(f"missing {REF}/{need}: run `make -C oracle ref` first")
    if len(sys.argv) > 2 and sys.argv[1] == "--cases":
        # (re)make only the named multigraph tgtp cases, keeping the rest of the manifest
        with open(os.path.join(HERE, "manifest.json")) as f:
            manifest = json.load(f)
        for name in sys.argv[2].split(","):
            manifest["tgtp"] = [r for r in manifest["tgtp"] if r["case"] != name]
            raw_tgtp_case(name, manifest)
        with open(os.path.join(HERE, "manifest.json"), "w") as f:
            json.dump(manifest, f, indent=1)
        return
    for sub in ("saba", "tgtp", "loader", "eigens"):
        shutil.rmtree(os.path.join(HERE, sub), ignore_errors=True)
        os.makedirs(os.path.join(HERE, sub))
    manifest = {"saba": [], "tgtp": [], "loader": [], "eigens": []}

    # ---- SABA ----
    def saba_case(name, text, runs):
        gpath = os.path.join(HERE, "saba", f"{name}.graph.txt")
        with open(gpath, "w") as f:
            f.write(text)
        for d, w in runs:
            out = os.path.join(HERE, "saba", f"{name}_d{d}_w{w}.u32")
            r = run([os.path.join(REF, "saba_harness_O2"), gpath, str(d), str(w), out])
            n, m, visits, checksum = map(int, r.stdout.split())
            counts = np.fromfile(out, dtype=np.uint32)
            os.remove(out)
            np.save(out.replace(".u32", ".npy"), counts)
            manifest["saba"].append(dict(graph=os.path.basename(gpath), depth=d, n_walks=w, n=n,
                                         m=m, visit_count=visits, checksum=checksum,
                                         counts=os.path.basename(out.replace(".u32", ".npy"))))

    for name, (make, runs) in SABA_CASES.items():
        g = make()
        saba_case(name, "".join(f"{a} {b}\n" for a, b in zip(g.u.tolist(), g.v.tolist())), runs)
    for name, (text, runs) in SABA_RAW.items():
        saba_case(name, text, runs)

    # ---- tgtp ----
    for name, (make, omega, runs) in TGTP_CASES.items():
        g = make()
        folder = os.path.join(HERE, "tgtp", name)
        synth.write_graph_txt(g, os.path.join(folder, "graph.txt"))
        n, u, v = eigenprep.read_edges(os.path.join(folder, "graph.txt"))
        vals, vecs, m = eigenprep.compute(n, u, v, omega, seed=0)
        eigenprep.write_files(folder, n, m, vals, vecs)
        tgtp_runs(name, folder, omega, n, runs, manifest)
    for name in TGTP_RAW:
        raw_tgtp_case(name, manifest)

    # ---- loader ----
    for name, text in LOADER_CASES.items():
        path = os.path.join(HERE, "loader", f"{name}.txt")
        with open(path, "w", newline="") as f:
            f.write(text)
        prefix = os.path.join(HERE, "loader", name)
        r = subprocess.run([os.path.join(REF, "ref_load_dump"), "graph", path, prefix],
                           capture_output=True, text=True)
        if r.returncode == 0:
            idx = np.fromfile(prefix + ".idx.u32", dtype=np.uint32)
            adj = np.fromfile(prefix + ".adj.u32", dtype=np.uint32)
            os.remove(prefix + ".idx.u32")
            os.remove(prefix + ".adj.u32")
            np.savez(prefix + ".npz", idx=idx, adj=adj)
            manifest["loader"].append(dict(case=name, file=f"{name}.txt", ok=True,
                                           csr=f"{name}.npz"))
        else:
            manifest["loader"].append(dict(case=name, file=f"{name}.txt", ok=False,
                                           error=r.stdout.strip().replace("ERROR ", "", 1)
                                           .replace(path, "{path}")))

    # ---- eigen parsing ----
    folder = os.path.join(HERE, "eigens")
    with open(os.path.join(folder, "graph.txt"), "w") as f:
        f.write("0 1\n1 2\n2 0\n2 3\n")
    # 1 + 2^-24 is the midpoint of two floats; one more decimal digit above it makes strtof round
    # up while strtod gives the midpoint exactly, which then rounds to even (down).
    rows = ["1 0.5 -0.25 1.0000000596046447753906251 3",
            "-0.5 1e-3 2.5e+2 -7.125 0.1",
            "0.25 3.4028234663852886e38 -1.1754943508222875e-38 1.401298464324817e-45 0"]
    with open(os.path.join(folder, "sorted_eigens_3.txt"), "w") as f:
        f.write("\n".join(rows) + "\n")
    prefix = os.path.join(folder, "parsed")
    run([os.path.join(REF, "ref_load_dump"), "eigens", os.path.join(folder, "graph.txt"),
         os.path.join(folder, "sorted_eigens_3.txt"), "3", prefix])
    vals = np.fromfile(prefix + ".values.f64", dtype=np.float64)
    vecs = np.fromfile(prefix + ".vectors.f32", dtype=np.float32)
    os.remove(prefix + ".values.f64")
    os.remove(prefix + ".vectors.f32")
    np.savez(prefix + ".npz", values=vals, vectors=vecs)
    manifest["eigens"].append(dict(graph="graph.txt", eigens="sorted_eigens_3.txt", n=4, omega=3,
                                   parsed="parsed.npz"))

    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)
    print(json.dumps({k: len(v) for k, v in manifest.items()}))


if __name__ == "__main__":
    main()
