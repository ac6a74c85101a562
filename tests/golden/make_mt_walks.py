"""Generates tests/golden/mt_walks.json: the counters of the reference's MT19937 walk routines
(scalar_randomwalk, src/rw_experiment.cpp:34-47, and simd_randomwalk, src/rw_experiment_simd.cpp:
44-83, with std::mt19937 reseeded to 42 + src as the runners do at :110) on seeded graphs, as run by
the reference compiled here (oracle/_ref/mt_harness_O2 and mt_simd_harness_O2, single-threaded, so
the float counters stay exact).

Each case records the graph's fingerprint, the exact visit count and checksum, the largest counter
and the SHA-256 of the whole uint32 counter array (little-endian, vertex order), so the oracle and
the GPU can be compared with the reference on every counter where the reference binaries are not
present.

    python tests/golden/make_mt_walks.py      # a few seconds
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from make_saba_rmat18 import graph_fingerprint, sha256_u32  # noqa: E402

# (graph, depth, walks): walk lengths below, at and above the generator's 624-word block
CASES = [("config1", 5, 64), ("rmat14", 10, 24), ("rmat12", 100, 8), ("rmat12", 700, 8)]


def graph(name):
    from tgtp_b200 import synth

    return {"config1": lambda: synth.config1_graph(1),
            "rmat14": lambda: synth.rmat(14, 8, 0.57, 0.19, 0.19, 3),
            "rmat12": lambda: synth.rmat(12, 8, 0.57, 0.19, 0.19, 5)}[name]()


def main() -> int:
    from tgtp_b200 import synth

    ref = os.path.join(ROOT, "oracle", "_ref")
    out = {"generator": "tests/golden/make_mt_walks.py", "cases": []}
    with tempfile.TemporaryDirectory() as tmp:
        for name, depth, walks in CASES:
            g = graph(name)
            idx, adj = g.csr()
            path = os.path.join(tmp, "graph.txt")
            synth.write_graph_txt(g, path)
            for simd in (False, True):
                exe = os.path.join(ref, "mt_simd_harness_O2" if simd else "mt_harness_O2")
                dump = os.path.join(tmp, "counts.u32")
                r = subprocess.run([exe, path, str(depth), str(walks), dump], capture_output=True,
                                   text=True, check=True)
                counts = np.fromfile(dump, dtype=np.uint32)
                n, m, visits, checksum = (int(x) for x in r.stdout.split())
                assert (n, m) == (len(idx) - 1, len(adj))
                out["cases"].append({
                    "graph": name, "depth": depth, "n_walks": walks, "simd": simd,
                    "graph_fingerprint": graph_fingerprint(idx, adj),
                    "visit_count": visits, "checksum": checksum,
                    "max_counter": int(counts.max()), "counters_sha256": sha256_u32(counts),
                    "source": os.path.basename(exe)})
    with open(os.path.join(HERE, "mt_walks.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
