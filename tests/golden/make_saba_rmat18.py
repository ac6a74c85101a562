"""Generates tests/golden/saba_rmat18.json: the SABA walk counters of the R-MAT scale-18 walk graph
(seeded, largest component kept: 174,015 vertices, 7,610,832 slots) at every depth x walks cell of
the throughput workload, D in {5, 10, 15} x W in {2048, 16384}.

Each cell records the exact visit count, checksum, largest counter and the SHA-256 of the whole
uint32 counter array (little-endian, vertex order), so a GPU test that hashes its counters compares
every one of the 174,015 counters.  Where the reference's own walk routine stays exact (its float
counters below 2^24: the two W = 2048 cells of depth 5 and 10) the counters come from the
reference compiled here (oracle/_ref/saba_harness_O2, single-threaded, src/rw_experiment_saba.cpp:
65-145) and the oracle must agree with them; in the other cells the reference's float counters
saturate, and the counters come from the oracle's integer restatement (oracle/tgtp_oracle.c),
which those two cells and the smaller golden cases pin to the reference.

    python tests/golden/make_saba_rmat18.py      # about 4 minutes on 8 cores
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CELLS = [(5, 2048), (10, 2048), (15, 2048), (5, 16384), (10, 16384), (15, 16384)]
REFERENCE_CELLS = {(5, 2048), (10, 2048)}


def sha256_u32(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


def graph_fingerprint(idx, adj) -> dict:
    return {"n": int(len(idx) - 1), "m": int(len(adj)), "idx_sha256": sha256_u32(idx),
            "adj_sha256": sha256_u32(adj)}


def main() -> None:
    import oracle
    from tgtp_b200 import synth

    oracle.build(reference=True)
    g = synth.config3_graph(1)
    idx, adj = g.csr()
    out = {"graph": "synth.config3_graph(1): R-MAT scale 18, edge factor 16, a=0.57, b=c=0.19, "
                    "seed 1, largest component",
           "fingerprint": graph_fingerprint(idx, adj), "cells": []}
    harness = oracle.ref_binary("saba_harness_O2")
    tmp = tempfile.mkdtemp(prefix="saba_rmat18_")
    gpath = os.path.join(tmp, "graph.txt")
    synth.write_graph_txt(g, gpath)
    weights = np.arange(1, g.n + 1, dtype=np.uint64)
    for depth, walks in CELLS:
        counts = oracle.saba(idx, adj, depth, walks)
        assert counts.max() < 2**32
        source = "oracle (integer restatement)"
        if (depth, walks) in REFERENCE_CELLS:
            if harness is None:
                raise SystemExit("the reference harness oracle/_ref/saba_harness_O2 is missing")
            cpath = os.path.join(tmp, "counts.u32")
            r = subprocess.run([harness, gpath, str(depth), str(walks), cpath], capture_output=True,
                               text=True, check=True)
            ref = np.fromfile(cpath, dtype=np.uint32).astype(np.uint64)
            if not np.array_equal(ref, counts):
                raise SystemExit(f"oracle differs from the reference at D={depth} W={walks}")
            assert int(r.stdout.split()[2]) == int(ref.sum())
            source = "reference saba_harness_O2 (oracle equal)"
        cell = {"depth": depth, "n_walks": walks, "visit_count": int(counts.sum()),
                "checksum": int((counts * weights).sum()), "max_counter": int(counts.max()),
                "counters_sha256": sha256_u32(counts), "source": source}
        print(cell, flush=True)
        out["cells"].append(cell)
    with open(os.path.join(HERE, "saba_rmat18.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
