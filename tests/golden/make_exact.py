"""Generate tests/golden/exact/: the exact spanning centrality of the golden tgtp graphs, computed
by the reference's own accuracy script (scripts/paper_accuracy.py, exact_scores), imported from the
reference sources in this container.  One float64 array per graph, in CSR slot order.

Run where the reference checkout is present (TGTP_REFERENCE, default /root/reference):
    python tests/golden/make_exact.py
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SCRIPT = os.path.join(os.environ.get("TGTP_REFERENCE", "/root/reference"), "scripts",
                      "paper_accuracy.py")
CASES = ["cl300", "sparse400", "grid", "cycle9", "complete12"]


def main() -> int:
    sys.dont_write_bytecode = True  # nothing is written beside the reference's sources
    spec = importlib.util.spec_from_file_location("reference_paper_accuracy", SCRIPT)
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    out_dir = os.path.join(HERE, "exact")
    os.makedirs(out_dir, exist_ok=True)
    index = {}
    for case in CASES:
        graph = os.path.join(HERE, "tgtp", case, "graph.txt")
        exact, validation = ref.exact_scores(graph)
        np.save(os.path.join(out_dir, f"{case}.npy"), np.asarray(exact, dtype=np.float64))
        index[case] = {"slots": int(len(exact)), "foster_error": validation["foster_error"],
                       "max_solve_residual": validation["max_solve_residual"]}
    with open(os.path.join(out_dir, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)
        f.write("\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
