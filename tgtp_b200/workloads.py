"""Seeded workloads from the command line, for profiling and quick checks on a GPU.

    python -m tgtp_b200.workloads aesc --graph config1 --eps 0.005 --precision mixed [--repeat 2]
    python -m tgtp_b200.workloads aesc --graph config4 --eps 0.005 --precision mixed \
        --vectors bf16 --deadline 600
    python -m tgtp_b200.workloads saba --graph config3 --depth 5 --walks 2048 [--repeat 2]

Graphs: config1 (Chung-Lu n=4,039, 88,234 edges, exponent 2.5), config3 (R-MAT scale 18, edge
factor 16, a=0.57), config4 (Chung-Lu n=10^6, 10^7 edges, exponent 2.3, seed 4), sparse5k
(Chung-Lu n=5,000, 12,000 edges, exponent 2.1), sparse25k (Chung-Lu 28,000 ids, 120,000 edges,
exponent 2.1, seed 1: largest component n=25,860, E=119,972), cl200k (Chung-Lu n=200,000, 2*10^6
edges, exponent 2.3: a fifth of config4's scale), rmat16 (R-MAT scale 16, edge factor 16),
batch_rmat (graph 28 of the batched workload: R-MAT, n=143,522, 1,732,704 edges, its eps 0.005).  AESC inputs get 128 eigenpairs: from the scipy
eigen prep (written and parsed back as sorted_eigens_128.txt) up to 20,000 vertices, from the GPU
eigen prep (tolerance 1e-4) above.  --deadline sets the device time budget of one kernel
(TGTP_KERNEL_DEADLINE_S; default 30 s).  Prints one line per run: seconds and work counters.
"""
from __future__ import annotations

import argparse
import os
import tempfile
import time


def _graph(name: str):
    from . import synth

    if name == "config1":
        return synth.config1_graph(1)
    if name == "config3":
        return synth.config3_graph(1)
    if name == "sparse5k":
        return synth.chung_lu(5000, 12000, 2.1, 7)
    if name == "sparse25k":
        return synth.chung_lu(28000, 120000, 2.1, 1)
    if name == "cl200k":
        return synth.chung_lu(200_000, 2_000_000, 2.3, 4)
    if name == "rmat16":
        return synth.rmat(16, 16, 0.57, 0.19, 0.19, 2)
    if name == "batch_rmat":
        return synth.config5_graphs(5, 64)[28][0]
    if name == "config4":
        return synth.chung_lu(1_000_000, 10_000_000, 2.3, 4)
    raise SystemExit(f"unknown graph {name}")


def _eigenpairs(g, omega: int):
    """(values, F32 vectors, F64 vectors), vertex-major as the loaders return them."""
    import numpy as np

    from . import aesc as A

    if g.n <= 20_000:
        from . import eigenprep, synth

        d = tempfile.mkdtemp(prefix="tgtp_workload_")
        synth.write_graph_txt(g, os.path.join(d, "graph.txt"))
        return A.load_eigens_txt(eigenprep.eigenprep_folder(d, omega), g.n, omega)
    from . import eigenprep_gpu

    values, vecs, _, _, _ = eigenprep_gpu.compute(g.n, g.u, g.v, omega, seed=1, tol=1e-4,
                                                  max_iter=60)
    v64 = np.ascontiguousarray(vecs.T).ravel()
    return values, v64.astype(np.float32), v64


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("kind", choices=["aesc", "saba"])
    ap.add_argument("--graph", default="config1")
    ap.add_argument("--eps", type=float, default=0.05)
    ap.add_argument("--precision", choices=["fp32", "fp64", "mixed"], default="fp64")
    ap.add_argument("--vectors", choices=["f32", "bf16"], default="f32")
    ap.add_argument("--depth", type=int, default=5)
    ap.add_argument("--walks", type=int, default=2048)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--deadline", type=float, default=None,
                    help="device time budget of one kernel, seconds (TGTP_KERNEL_DEADLINE_S)")
    args = ap.parse_args(argv)
    if args.deadline is not None:
        os.environ["TGTP_KERNEL_DEADLINE_S"] = repr(args.deadline)

    from . import aesc as A

    g = _graph(args.graph)
    idx, adj = g.csr()
    dg = A.AESCGraph.from_csr(idx, adj)
    if args.kind == "saba":
        for _ in range(args.repeat):
            t = time.perf_counter()
            _, vc, cs, fb = A.saba_count(dg, args.depth, args.walks, counters=False)
            print(f"saba {args.graph} d{args.depth} w{args.walks}: {time.perf_counter() - t:.4f} s "
                  f"visit_count {vc} checksum {cs} fallback_bouquets {fb}", flush=True)
        dg.free()
        return 0
    values, v32, v64 = _eigenpairs(g, 128)
    prec = {"fp32": A.PRECISION_FP32, "fp64": A.PRECISION_FP64, "mixed": A.PRECISION_MIXED}
    if args.precision == "fp64":
        dg.upload_eigens(values, v64, A.VEC_F64)
    elif args.vectors == "bf16":
        dg.upload_eigens(values, v32, A.VEC_BF16)
    else:
        dg.upload_eigens(values, v32, A.VEC_F32)
    cfg = A.AESCConfig(args.eps, precision=prec[args.precision],
                       vec_dtype=A.VEC_BF16 if args.vectors == "bf16" else A.VEC_F32)
    a = A.AESC(dg, cfg)
    for _ in range(args.repeat):
        t = time.perf_counter()
        a.tgtp()
        st = a.stats()
        print(f"aesc {args.graph} eps {args.eps} {args.precision}: {time.perf_counter() - t:.4f} s "
              f"rounds {st['push_rounds']} traversals {st['push_traversals']} "
              f"walk_hops {st['walk_hops']}", flush=True)
    dg.free()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
