"""Benchmark of the tgtp hot path on B200.

Headline workload (one GPU): tgtp() on a seeded Chung-Lu graph, n = 4,039, 88,234 undirected edges,
degree exponent 2.5, omega = 128 eigenpairs (scipy restatement of the reference's eigen prep),
gamma = 10, epsilon = 0.05, in the plain FP64 form.  A step is one tgtp() call over that graph;
metric: undirected edges scored per second (the reference's benchmark.cpp timing scope).  The same
line carries the other forms and the SABA walk counter (transitions per second) as extra keys.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value`  = device time (CUDA events on the launching stream) of K steps, inputs resident in HBM,
           L2 flushed (256 MiB write) before every step, outside the events.
`e2e`    = the same metric through the public API with pinned host buffers: graph + eigen upload,
           tgtp_run, score download and graph release inside every step.
`roofline` = the dominant kernel's algorithmic bytes per launch / its event-timed launch time.
N > 1: one process per GPU (torchrun), every rank scores its own graph (seed + rank): weak scaling,
no collective on the data path; the slowest rank's time counts.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from tgtp_b200 import replicas  # noqa: E402

METRIC = "walk transitions/s; AESC edges/s at ε, mixed vs FP64 on 1 B200; % HBM peak"
N_VERT, N_EDGES, EXPONENT, OMEGA, GAMMA, EPS = 4039, 88234, 2.5, 128, 10, 0.05
WORKLOAD = ("tgtp AESC, plain FP64 form: Chung-Lu n=4039 E=88234 exp 2.5 (LCC), omega=128, "
            "gamma=10, eps=0.05")
L2_FLUSH_BYTES = 256 << 20
# push-bound companion workload: sparse Chung-Lu (28,000 ids, 120,000 target edges, exponent 2.1;
# largest component n = 25,860, E = 119,972), where sources push for several rounds and walk
SPARSE = dict(n0=28000, edges=120000, exponent=2.1, seed=1)
PUSH_EPS = (0.01, 0.005)


def bench_config(world: int) -> dict:
    """The `config` both arms print (the same dict, so the two lines describe one workload)."""
    return {"workload": WORKLOAD, "graph_seed": "1 + rank",
            "l2": "GPU arm: flushed (256 MiB write) before every timed step; CPU arm: n/a",
            "parallelism": f"replicas x{world}"}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_inputs(seed: int, folder: str):
    """graph.txt + sorted_eigens_128.txt for the headline graph (cached by seed)."""
    from tgtp_b200 import eigenprep, synth

    g = synth.chung_lu(N_VERT, N_EDGES, EXPONENT, seed)
    os.makedirs(folder, exist_ok=True)
    gpath = os.path.join(folder, "graph.txt")
    epath = os.path.join(folder, f"sorted_eigens_{OMEGA}.txt")
    if not os.path.exists(epath):
        synth.write_graph_txt(g, gpath)
        eigenprep.eigenprep_folder(folder, OMEGA)
    return g, gpath, epath


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self._wait_for(1)  # a sample taken before the timed region starts
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def _wait_for(self, count, limit_s=5.0):
        t0 = time.time()
        while len(self.lines) < count and time.time() - t0 < limit_s:
            time.sleep(0.01)

    def __exit__(self, *exc):
        if self.proc:
            # the timed region can be shorter than the sampling period: keep sampling until one
            # more sample has come in, so the region is bracketed by samples
            self._wait_for(len(self.lines) + 1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_model() -> str:
    """The host CPU's model name (first processor of /proc/cpuinfo), or the platform's answer."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


def cpu_baseline_line(edges: int, secs_all, threads: int, secs_one, sample: str) -> dict:
    """cpu_baseline of the JSON line: the reference on all host cores (the value), the same on one
    core beside it, the core count, OMP_NUM_THREADS and the CPU model."""
    out = {"value": edges / statistics.mean(secs_all), "unit": "edges/s", "cores": threads,
           "kind": "reference", "omp_num_threads": threads, "cpu_model": cpu_model(),
           "sample": sample}
    if secs_one:
        out["single_thread"] = {"value": edges / statistics.mean(secs_one), "unit": "edges/s",
                                "cores": 1, "sample": "mean of 3 tgtp() calls (after 1 warm-up), "
                                                      "OMP_NUM_THREADS=1"}
    return out


def cpu_reference_run(folder_root: str, dataset: str, threads: int, repeats: int, warmups: int,
                      eps: float = EPS):
    """Seconds of each timed tgtp() call of the reference's own benchmark binary (compiled from its
    sources into oracle/_ref), or None when it was not built."""
    import oracle

    exe = oracle.ref_binary("benchmark")
    if exe is None:
        return None
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    r = subprocess.run([exe, dataset, str(eps), str(threads), str(repeats), folder_root,
                        str(OMEGA), str(GAMMA), str(warmups)], capture_output=True, text=True,
                       env=env, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError("reference benchmark failed: " + r.stderr[-400:])
    secs = [float(line.split("\t")[5]) for line in r.stdout.splitlines()[1:] if line.strip()]
    return secs


def saba_cpu_reference(g, root: str, depth: int, walks: int, runs: int = 3,
                       binary: str = "rw_experiment_saba"):
    """The reference's walk runner `binary` (rw_experiment_saba, or the MT19937 rw_experiment /
    rw_experiment_simd; built from its sources into oracle/_ref) on `g`, on all host cores: the mean
    of `runs` runs, as transitions per second of its own walk timer, or None when the binary is
    missing or fails."""
    import oracle
    from tgtp_b200 import synth

    exe = oracle.ref_binary(binary)
    if exe is None:
        return None
    folder = os.path.join(root, "saba_data")
    os.makedirs(os.path.join(folder, "g"), exist_ok=True)
    synth.write_graph_txt(g, os.path.join(folder, "g", "graph.txt"))
    threads = os.cpu_count() or 1
    walk_s = []
    for _ in range(runs):
        r = subprocess.run([exe, folder, "g", str(depth), str(walks), str(threads)],
                           capture_output=True, text=True, cwd=root, timeout=900,
                           env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
        if r.returncode != 0:
            return None
        # TSV fields (src/rw_experiment_saba.cpp:241-244): 8 = t_rw_s, 10 = total_walks, which
        # already counts every hop (n * n_walks * depth): transitions
        f = r.stdout.strip().splitlines()[-1].split("\t")
        walk_s.append((float(f[8]), float(f[10])))
    t_rw = statistics.mean(t for t, _ in walk_s)
    total = walk_s[0][1]
    return {"transitions_per_s": total / t_rw, "transitions": total, "cores": threads,
            "omp_num_threads": threads, "walk_seconds": t_rw,
            "sample": f"mean of {runs} runs of the reference {binary} (-Ofast, OpenMP) "
                      "on the same graph"}


def saba_rmat18(hbm: float, peak_kind: str, root: str, with_cpu: bool):
    """SABA walk counter at scale: seeded R-MAT scale 18, edge factor 16 (a=0.57, b=c=0.19), largest
    component; depth 5, 2048 walks per vertex, and beside it every depth x walks cell of the
    walk experiment (D 5 / 10 / 15 x W 2,048 / 16,384).  Kernel time from the library's CUDA events
    (3 runs after 1 warm-up); transitions = active vertices x walks x depth; 20 algorithmic bytes
    per transition (idx pair 8, adj 4, counter read + write 8).  The reference's
    rw_experiment_saba, built from its sources, timed once on the host cores beside it (D 5,
    W 2,048)."""
    from tgtp_b200 import synth
    from tgtp_b200.aesc import AESCGraph, saba_count

    g = synth.config3_graph(1)
    idx, adj = g.csr()
    dg = AESCGraph.from_csr(idx, adj)

    def cell(depth, walks):
        saba_count(dg, depth, walks, counters=False)
        dg.set_profiling(True)
        for _ in range(3):
            _, vc, cs, fb = saba_count(dg, depth, walks, counters=False)
        ks = dg.kernel_stats()
        dg.set_profiling(False)
        ms = ks["saba_walk"][1] / ks["saba_walk"][0]
        trans = g.n * walks * depth
        return ms, ks, trans, vc, cs, fb

    ms, ks, trans, vc, cs, fb = cell(5, 2048)
    out = {"workload": f"SABA d5 w2048 on R-MAT scale 18 (LCC n={g.n}, E={g.num_edges})",
           "transitions_per_s": trans / (ms * 1e-3), "kernel_ms": ms,
           "kernel_ms_all": {k: v[1] / v[0] for k, v in ks.items()},
           "hbm_frac_of_" + peak_kind: trans * 20 / (ms * 1e-3) / 1e9 / hbm,
           "visit_count": vc, "checksum": cs, "fallback_bouquets": fb}
    cells = []
    for depth in (5, 10, 15):
        for walks in (2048, 16384):
            ms_c, _, tr_c, vc_c, cs_c, _ = cell(depth, walks)
            cells.append({"depth": depth, "walks": walks, "kernel_ms": ms_c,
                          "transitions_per_s": tr_c / (ms_c * 1e-3),
                          "hbm_frac_of_" + peak_kind: tr_c * 20 / (ms_c * 1e-3) / 1e9 / hbm,
                          "visit_count": vc_c, "checksum": cs_c})
    out["cells"] = cells
    # the MT19937 comparison walks (src/rw_experiment.cpp, src/rw_experiment_simd.cpp), D 5, W 2,048
    from tgtp_b200.aesc import mt_walk_count

    mt = {}
    for simd in (False, True):
        mt_walk_count(dg, 5, 2048, simd=simd, counters=False)
        dg.set_profiling(True)
        for _ in range(3):
            _, vc_m, cs_m = mt_walk_count(dg, 5, 2048, simd=simd, counters=False)
        ks_m = dg.kernel_stats()
        dg.set_profiling(False)
        ms_m = ks_m["mt_walk"][1] / ks_m["mt_walk"][0]
        tr_m = g.n * 2048 * 5
        cell_m = {"kernel_ms": ms_m, "transitions_per_s": tr_m / (ms_m * 1e-3),
                  "hbm_frac_of_" + peak_kind: tr_m * 20 / (ms_m * 1e-3) / 1e9 / hbm,
                  "visit_count": vc_m, "checksum": cs_m}
        if with_cpu:
            ref_m = saba_cpu_reference(g, root, 5, 2048, runs=1,
                                       binary="rw_experiment_simd" if simd else "rw_experiment")
            if ref_m is not None:
                cell_m["cpu_reference"] = ref_m
        mt["simd" if simd else "regular"] = cell_m
    out["mt19937_walks"] = mt
    dg.free()
    if with_cpu:
        ref = saba_cpu_reference(g, root, 5, 2048)
        if ref is not None:
            out["cpu_reference"] = ref
    return out


def source_bytes(st: dict, taus, idx) -> tuple[int, int]:
    """Algorithmic bytes of the per-source stage (source_kernel and, in the mixed form's block
    mode, push_block) of one run: 20 B per push traversal (adjacency 4, the vertex's offset pair 8,
    residual read-modify-write 8) + 12 B per frontier vertex + 32 B per two-walker hop, without the
    rows that finish in closed form (every tau <= 1: finish_kernel scores them, and the run counters
    include their one round).  Returns (bytes, closed-form traversals)."""
    import numpy as np

    deg = np.diff(idx.astype(np.int64))
    row_max = np.maximum.reduceat(taus, idx[:-1].astype(np.int64)) if len(taus) else taus
    closed = row_max <= 1
    closed_trav = int(deg[closed].sum())
    closed_rows = int(closed.sum())
    trav = st["push_traversals"] - closed_trav
    pv = st["push_vertices"] - closed_rows
    return 20 * trav + 12 * pv + 32 * st["walk_hops"], closed_trav


def push_bound_section(dg, idx, E, folder_root, dataset, eps_list, stream, out, flush, hbm,
                       peak_kind, steps, with_cpu, flush_l2=True):
    """tgtp() where the work is: epsilon values at which sources push past their first round and
    slots walk.  Per epsilon and form: edges/s and ms per step (CUDA events on the launching stream,
    `steps` timed runs after 2 warm-up, L2 flushed before each), the work counters, the per-source
    stage's share and its algorithmic bytes / event-timed time against the HBM peak; beside them the
    reference's benchmark binary on the same graph and eigen files (mean of 2 calls after 1 warm-up
    on all host cores)."""
    import torch

    from tgtp_b200.aesc import (AESC, AESCConfig, PRECISION_FP64, PRECISION_MIXED, VEC_BF16,
                                VEC_F32)

    forms = (("fp64", PRECISION_FP64, VEC_F32), ("mixed_f32_vectors", PRECISION_MIXED, VEC_F32),
             ("mixed_bf16_vectors", PRECISION_MIXED, VEC_BF16))
    res = {}
    for eps in eps_list:
        cell = {}
        for label, prec, vec in forms:
            a = AESC(dg, AESCConfig(eps, omega=OMEGA, gamma=GAMMA, precision=prec, vec_dtype=vec))
            for _ in range(2):
                a.tgtp_device(out.data_ptr())
            torch.cuda.synchronize()
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(steps)]
            for e0, e1 in ev:
                if flush_l2:
                    flush.zero_()
                e0.record(stream)
                a.tgtp_device(out.data_ptr())
                e1.record(stream)
            torch.cuda.synchronize()
            ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)
            st = a.stats()
            taus = a.taus()
            dg.set_profiling(True)
            a.tgtp_device(out.data_ptr())
            ks = dg.kernel_stats()
            dg.set_profiling(False)
            src_ms = sum(v[1] for k, v in ks.items() if k in ("source", "push_block", "row_key"))
            tot_ms = sum(v[1] for v in ks.values())
            sbytes, closed_trav = source_bytes(st, taus, idx)
            achieved = sbytes / (src_ms * 1e-3) / 1e9 if src_ms > 0 else None
            cell[label] = {
                "edges_per_s": E / (ms * 1e-3), "ms_per_step": ms,
                "counters": {k: st[k] for k in ("push_rounds", "push_vertices", "push_traversals",
                                                "walk_edges", "walk_count", "walk_hops")},
                "kernel_ms": {k: v[1] / v[0] for k, v in ks.items()},
                "per_source_stage": {"kernels": "source (+ push_block, row_key)",
                                     "share": src_ms / tot_ms if tot_ms else None,
                                     "algorithmic_bytes": sbytes,
                                     "closed_form_traversals_excluded": closed_trav,
                                     "achieved_gbs": achieved,
                                     "frac_of_" + peak_kind + "_hbm":
                                         achieved / hbm if achieved else None},
            }
            if label == "fp64":
                fp64_out = out.double().clone()
            else:
                dev = (out.double() - fp64_out).abs() / fp64_out.abs()
                cell[label]["rel_dev_vs_fp64"] = {"median": float(dev.median()),
                                                  "p99": float(torch.quantile(dev.float(), 0.99)),
                                                  "max": float(dev.max())}
                cell[label]["speedup_vs_fp64"] = cell["fp64"]["ms_per_step"] / ms
        if with_cpu:
            threads = os.cpu_count() or 1
            secs = cpu_reference_run(folder_root, dataset, threads, 2, 1, eps)
            if secs:
                cell["cpu_reference"] = {"edges_per_s": E / statistics.mean(secs),
                                         "seconds": statistics.mean(secs), "cores": threads,
                                         "omp_num_threads": threads,
                                         "sample": "mean of 2 tgtp() calls after 1 warm-up, "
                                                   "reference benchmark binary"}
        res[f"eps_{eps}"] = cell
    return res


def sparse_inputs(root: str):
    """The sparse Chung-Lu companion graph with its 128 eigenpairs (scipy restatement of the eigen
    prep), written and parsed back like the reference's files."""
    from tgtp_b200 import eigenprep, synth
    from tgtp_b200.aesc import load_eigens_txt

    g = synth.chung_lu(SPARSE["n0"], SPARSE["edges"], SPARSE["exponent"], SPARSE["seed"])
    folder = os.path.join(root, "sparse")
    os.makedirs(folder, exist_ok=True)
    synth.write_graph_txt(g, os.path.join(folder, "graph.txt"))
    epath = eigenprep.eigenprep_folder(folder, OMEGA)
    values, v32, v64 = load_eigens_txt(epath, g.n, OMEGA)
    return g, values, v32, v64


def batch_measure(work, steps: int, accuracy_slots: int = 0) -> dict:
    """The batched form against one-by-one runs on `work` = [(EdgeList, eps)]: eigenpairs from the
    GPU eigen prep; every graph in the plain FP64 form one after another (each run timed by CUDA
    events on one stream), the mixed form (BF16 vectors) the same way, then the mixed form as one
    batch (one CUDA graph whose per-source stage is one persistent launch over all graphs' rows),
    `steps` timed replays after one untimed.  With accuracy_slots > 0, the fraction of that many
    sampled edges per graph within the graph's epsilon of the exact spanning centrality (the
    library's GPU conjugate-gradient solver), for both forms."""
    import numpy as np
    import torch

    from tgtp_b200 import eigenprep_gpu
    from tgtp_b200.aesc import (AESC, AESCConfig, AESCGraph, Batch, PRECISION_FP64,
                                PRECISION_MIXED, VEC_BF16, VEC_F32, VEC_F64, exact_sc_slots)

    t0 = time.perf_counter()
    graphs = []
    for g, eps in work:
        vals, vecs, _, _, _ = eigenprep_gpu.compute(g.n, g.u, g.v, OMEGA, seed=1, tol=1e-6,
                                                    max_iter=60)
        idx, adj = g.csr()
        dg = AESCGraph.from_csr(idx, adj)
        v64 = np.ascontiguousarray(vecs.T).ravel()
        dg.upload_eigens(vals, v64, VEC_F64)
        dg.upload_eigens(vals, v64.astype(np.float32), VEC_F32)
        dg.upload_eigens(vals, v64.astype(np.float32), VEC_BF16)
        graphs.append((g, eps, dg))
    prep_s = time.perf_counter() - t0
    E = sum(g.num_edges for g, _, _ in graphs)
    outs = [torch.empty(dg.m, dtype=torch.float32, device="cuda") for _, _, dg in graphs]
    stream = torch.cuda.Stream()

    def one_by_one(cfgs):
        """Each run on one shared stream, timed by events on it, one after another."""
        runs = [AESC(dg, c) for (_, _, dg), c in zip(graphs, cfgs)]
        for _, _, dg in graphs:
            dg.set_stream(stream.cuda_stream)
        secs = []
        for a, o in zip(runs, outs):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            a.tgtp_device(o.data_ptr())
            e1.record(stream)
            e1.synchronize()
            a.stats()  # raises on a device time-out or walk-count error
            secs.append(e0.elapsed_time(e1) * 1e-3)
        for _, _, dg in graphs:
            dg.set_stream(None)  # back to each graph's own stream (parallel batch branches)
        return runs, secs

    fp64_cfgs = [AESCConfig(eps, omega=OMEGA, gamma=GAMMA, precision=PRECISION_FP64)
                 for _, eps, _ in graphs]
    mixed_cfgs = [AESCConfig(eps, omega=OMEGA, gamma=GAMMA, precision=PRECISION_MIXED,
                             vec_dtype=VEC_BF16) for _, eps, _ in graphs]
    _, fp64_secs = one_by_one(fp64_cfgs)
    fp64 = [o.cpu().numpy().copy() for o in outs]
    runs, mixed_secs = one_by_one(mixed_cfgs)
    b = Batch([(a, o.data_ptr()) for a, o in zip(runs, outs)])
    b.run(stream.cuda_stream)
    b.wait()
    times = []
    for _ in range(max(1, steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.run(stream.cuda_stream)
        e1.record(stream)
        b.wait()
        times.append(e0.elapsed_time(e1) * 1e-3)
    batch_s = float(np.median(times))
    mixed = [o.cpu().numpy().copy() for o in outs]
    dev = np.concatenate([np.abs(m.astype(np.float64) - f) / np.abs(f)
                          for m, f in zip(mixed, fp64)])
    b.free()
    out = {"graphs": len(graphs), "undirected_edges": E, "vertices": sum(g.n for g, _, _ in graphs),
           "batched_mixed_seconds": batch_s, "batched_mixed_edges_per_s": E / batch_s,
           "fp64_one_by_one": {"edges_per_s": E / sum(fp64_secs), "seconds": sum(fp64_secs),
                               "slowest": sorted(((round(s, 3), g.name, eps) for s, (g, eps, _)
                                                  in zip(fp64_secs, graphs)), reverse=True)[:3]},
           "mixed_one_by_one": {"edges_per_s": E / sum(mixed_secs), "seconds": sum(mixed_secs)},
           "speedup_batched_mixed_vs_fp64_one_by_one": sum(fp64_secs) / batch_s,
           "mixed_vs_fp64_rel_dev": {"median": float(np.median(dev)),
                                     "p99": float(np.percentile(dev, 99)),
                                     "max": float(dev.max())},
           "input_prep_s": prep_s}
    if accuracy_slots:
        rng = np.random.default_rng(7)
        per_graph, tot = [], {"fp64": 0, "mixed": 0, "slots": 0}
        for (g, eps, dg), f, m in zip(graphs, fp64, mixed):
            idx, adj = g.csr()
            rows = np.repeat(np.arange(g.n), np.diff(idx.astype(np.int64)))
            fwd = np.flatnonzero(adj.astype(np.int64) > rows)
            slots = np.sort(rng.choice(fwd, size=min(accuracy_slots, len(fwd)),
                                       replace=False)).astype(np.uint32)
            exact, _ = exact_sc_slots(dg, slots, tol=1e-9)
            wf = int(np.sum(np.abs(f[slots] - exact) <= eps))
            wm = int(np.sum(np.abs(m[slots] - exact) <= eps))
            per_graph.append({"graph": g.name, "n": g.n, "eps": eps, "slots": len(slots),
                              "fp64_within_eps": wf / len(slots),
                              "mixed_within_eps": wm / len(slots)})
            tot["fp64"] += wf
            tot["mixed"] += wm
            tot["slots"] += len(slots)
        out["accuracy_vs_exact_sc"] = {
            "sampled_edges": tot["slots"], "fp64_within_eps": tot["fp64"] / tot["slots"],
            "mixed_within_eps": tot["mixed"] / tot["slots"], "per_graph": per_graph,
            "exact": "tgtp_exact_sc_slots (FP64 conjugate gradients, tol 1e-9)"}
    for _, _, dg in graphs:
        dg.free()
    return out


def run_batch_workload(args):
    """64 seeded graphs of uneven size (n log-uniform in [1,000, 200,000]; Chung-Lu exponent
    2.1-2.8, R-MAT a=0.57, 2-D grid with chords; average degree 8-40), each with its own epsilon
    from {0.05, 0.01, 0.005}, omega=128, gamma=10.  value = sum of undirected edges / device time
    of one replay of the batched mixed form (BF16 vectors), against the same graphs run one after
    another in the plain FP64 form (see batch_measure).  The inputs are far larger than L2
    (per-source residual blocks of GBs), so no flush is needed between steps."""
    import torch

    from tgtp_b200 import synth

    rank, world, local = replicas.rank_info()
    torch.cuda.set_device(local)
    os.environ.setdefault("TGTP_KERNEL_DEADLINE_S", "300")
    work = synth.config5_graphs(replicas.workload_seed(5, rank), 64)
    steps = max(1, min(args.steps, 3))
    r = batch_measure(work, steps)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    batch_s, fp64_total = replicas.slowest([r["batched_mixed_seconds"],
                                            r["fp64_one_by_one"]["seconds"]], device="cuda")
    if rank == 0:
        E = r["undirected_edges"]
        line = {
            "metric": METRIC, "value": replicas.job_rate(E, batch_s, world), "unit": "edges/s",
            "n_gpus": world,
            "steps": steps, "warmup": 1, "ms_per_step": batch_s * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (mixed form, bf16 vectors)",
            "data": "synthetic (64 seeded graphs + GPU eigen prep)",
            "config": {"workload": "batched AESC: 64 graphs, n log-uniform in [1e3, 2e5], "
                                   "Chung-Lu / R-MAT / grid+chords, avg degree 8-40, own eps "
                                   "from {0.05, 0.01, 0.005}, omega=128, gamma=10",
                       "undirected_edges": E, "vertices": r["vertices"],
                       "l2": "inputs larger than L2", "parallelism": f"replicas x{world}"},
            **{k: v for k, v in r.items() if k not in ("undirected_edges", "vertices")},
            "speedup_batched_mixed_vs_fp64_one_by_one": fp64_total / batch_s,
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    root = tempfile.mkdtemp(prefix="tgtp_bench_ref_")
    g, _, _ = make_inputs(1, os.path.join(root, "cl4039"))
    threads = os.cpu_count() or 1
    secs = cpu_reference_run(root, "cl4039", threads, args.steps, args.warmup)
    if secs is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference binaries were not built (oracle/_ref missing)"}))
        return 0
    mean = statistics.mean(secs)
    value = g.num_edges / mean
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "edges/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mean * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Chung-Lu + scipy eigenpairs)",
        "config": bench_config(args.gpus),
        "cpu_baseline": {"value": value, "unit": "edges/s", "cores": threads, "kind": "reference",
                         "omp_num_threads": threads, "cpu_model": cpu_model(),
                         "sample": f"{args.steps} timed tgtp() calls after {args.warmup} warm-up, "
                                   "reference benchmark binary (-Ofast -march=x86-64-v3, OpenMP)"},
        "e2e": {"value": value, "unit": "edges/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-rmat", action="store_true", help="skip the R-MAT scale-18 walk line")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the 16-graph batched-form measurement")
    ap.add_argument("--no-push", action="store_true",
                    help="skip the push-bound tgtp measurements (eps 0.01 / 0.005, sparse graph)")
    ap.add_argument("--workload", choices=["aesc", "batch"], default="aesc",
                    help="batch: the 64-graph batched workload instead of the headline")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "batch":
        return run_batch_workload(args)

    import numpy as np
    import torch

    rank, world, local = replicas.rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from tgtp_b200.aesc import (AESC, AESCConfig, AESCGraph, PRECISION_FP32, PRECISION_FP64,
                                PRECISION_MIXED, VEC_BF16, VEC_F32, VEC_F64, load_eigens_txt,
                                saba_count)

    seed = replicas.workload_seed(1, rank)
    root = tempfile.mkdtemp(prefix=f"tgtp_bench_r{rank}_")
    g, gpath, epath = make_inputs(seed, os.path.join(root, "cl4039"))
    idx, adj = g.csr()
    n, m, E = g.n, int(idx[-1]), g.num_edges
    values, v32, v64 = load_eigens_txt(epath, n, OMEGA)

    # A dedicated stream: events, the L2 flush and the library's kernels all run on it.  (The
    # legacy default stream has handle 0, which tgtp_graph_set_stream reads as "own stream".)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0
    dg = AESCGraph.from_csr(idx, adj)
    dg.set_stream(stream.cuda_stream)
    dg.upload_eigens(values, v64, VEC_F64)
    dg.upload_eigens(values, v32, VEC_F32)
    dg.upload_eigens(values, v32, VEC_BF16)
    out = torch.empty(m, dtype=torch.float32, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def timed(form: int, steps: int, warmup: int, profile: bool, vec: int = VEC_F32):
        a = AESC(dg, AESCConfig(EPS, omega=OMEGA, gamma=GAMMA, precision=form, vec_dtype=vec))
        for _ in range(warmup):
            a.tgtp_device(out.data_ptr())
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        barrier()
        torch.cuda.synchronize()
        dg.set_profiling(profile)
        t0 = time.perf_counter()
        for i in range(steps):
            flush.zero_()
            starts[i].record(stream)
            a.tgtp_device(out.data_ptr())
            ends[i].record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        barrier()
        kstats = dg.kernel_stats() if profile else {}
        dg.set_profiling(False)
        ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
        return ms, wall, kstats, a.stats()

    # ---- headline: FP64 form, inputs resident ----
    with ClockSampler(local) as clocks:
        ms64, wall64, _, st64 = timed(PRECISION_FP64, args.steps, args.warmup, False)
    # per-kernel CUDA events (they sit between the kernels, so they are taken on a separate pass)
    side_steps = max(args.steps // 4, 10)
    _, _, k64, _ = timed(PRECISION_FP64, side_steps, args.warmup, True)
    out64 = out.clone()
    ms32, _, _, _ = timed(PRECISION_FP32, side_steps, args.warmup, False)
    _, _, k32, _ = timed(PRECISION_FP32, side_steps, args.warmup, True)
    mixed = {}
    for label, vec in (("mixed_f32_vectors", VEC_F32), ("mixed_bf16_vectors", VEC_BF16)):
        msx, _, _, _ = timed(PRECISION_MIXED, side_steps, args.warmup, False, vec)
        dev = (out.double() - out64.double()).abs() / out64.double().abs()
        _, _, kx, _ = timed(PRECISION_MIXED, side_steps, args.warmup, True, vec)
        mixed[label] = {"ms_per_step": msx / side_steps,
                        "kernel_ms": {k: v[1] / v[0] for k, v in kx.items()},
                        "max_rel_dev_vs_fp64": float(dev.max())}

    (ms_step,) = replicas.slowest([ms64 / args.steps], device="cuda")
    value = replicas.job_rate(E, ms_step * 1e-3, world)

    # ---- e2e: public API with pinned host buffers ----
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()  # noqa: E731
    h_idx, h_adj, h_vals, h_vec = pin(idx), pin(adj), pin(values), pin(v64)
    h_out = torch.empty(m, dtype=torch.float32).pin_memory()
    h2d = h_idx.numel() * 4 + h_adj.numel() * 4 + h_vals.numel() * 8 + h_vec.numel() * 8
    d2h = m * 4

    def e2e_step():
        eg = AESCGraph.from_csr(h_idx.numpy(), h_adj.numpy())
        eg.upload_eigens(h_vals.numpy(), h_vec.numpy(), VEC_F64)
        from tgtp_b200 import _lib
        import ctypes as C

        cfg = AESCConfig(EPS, omega=OMEGA, gamma=GAMMA, precision=PRECISION_FP64).to_c(n)
        _lib.check(_lib.lib().tgtp_run(eg.handle, C.byref(cfg), C.c_void_p(h_out.data_ptr())))
        eg.free()

    for _ in range(3):
        e2e_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / args.e2e_steps
    (e2e_slowest,) = replicas.slowest([e2e_s], device="cuda")
    e2e_value = replicas.job_rate(E, e2e_slowest, world)
    # parity guard on the e2e output (same scores as the resident run)
    ok_e2e = bool(np.array_equal(h_out.numpy(), out64.cpu().numpy()))

    line = None
    if rank == 0:
        hbm, peak_kind = peaks()
        # algorithmic bytes per launch of each kernel of the FP64 form:
        #   tau_sums: both omega-element FP64 eigen rows of every undirected edge, its 16-byte record
        #             and the 16-byte (upsilon, delta_0) sums written;
        #   tau_bound: record, sums, two degrees and two tau words per edge, plus both rows again for
        #             every further delta sweep (tau_iterations - E of them);
        #   source: 20 B per push traversal + 12 B per frontier vertex + 32 B per 2-walker hop;
        #   finish: 24 B per slot
        E_fwd = E
        per_launch = {
            "tau_sums": E_fwd * (2 * OMEGA * 8 + 32),
            "tau_bound": E_fwd * 48 + 2 * OMEGA * 8 * max(st64["tau_iterations"] - E_fwd, 0),
            "source": 20 * st64["push_traversals"] + 12 * st64["push_vertices"]
                      + 32 * st64["walk_hops"],
            "finish": 24 * m,
        }
        top = max(k64, key=lambda k: k64[k][1])
        launches, tot = k64[top]
        avg_ms = tot / launches
        achieved = per_launch[top] / (avg_ms * 1e-3) / 1e9
        share = {k: round(v[1] / sum(x[1] for x in k64.values()), 4) for k, v in k64.items()}
        traffic = None
        tf = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tf):
            try:
                traffic = json.load(open(tf)).get(f"fp64_{top}")
            except Exception:
                traffic = None

        # ---- SABA walk counter on the same graph (the reference's rw_experiment_saba) ----
        for _ in range(3):
            saba_count(dg, 5, 2048, counters=False)
        dg.set_profiling(True)
        for _ in range(10):
            saba_count(dg, 5, 2048, counters=False)
        ks = dg.kernel_stats()
        dg.set_profiling(False)
        saba_ms = ks["saba_walk"][1] / ks["saba_walk"][0]
        trans = n * 2048 * 5
        saba = {"workload": "SABA d5 w2048 on the same graph", "transitions_per_s":
                trans / (saba_ms * 1e-3), "kernel_ms": saba_ms,
                "hbm_frac_of_" + peak_kind: trans * 20 / (saba_ms * 1e-3) / 1e9 / hbm}
        if not args.no_rmat:
            saba["rmat18"] = saba_rmat18(hbm, peak_kind, root, not args.no_cpu_baseline)

        # ---- the batched form on the 16 smallest graphs of the batched workload ----
        batch16 = None
        if not args.no_batch:
            from tgtp_b200 import synth

            work = sorted(synth.config5_graphs(5, 64), key=lambda ge: ge[0].n)[:16]
            batch16 = {"workload": "the 16 smallest of the 64 batched-workload graphs (seed 5), "
                                   "own eps each, omega=128, gamma=10",
                       **batch_measure(work, 3, accuracy_slots=256)}

        # ---- tgtp where the push and the walks run ----
        push = {}
        if not args.no_push:
            push["chunglu4039"] = push_bound_section(
                dg, idx, E, root, "cl4039", PUSH_EPS, stream, out, flush, hbm, peak_kind, 10,
                not args.no_cpu_baseline)
            sg, svals, sv32, sv64 = sparse_inputs(root)
            sidx, sadj = sg.csr()
            sdg = AESCGraph.from_csr(sidx, sadj)
            sdg.set_stream(stream.cuda_stream)
            sdg.upload_eigens(svals, sv64, VEC_F64)
            sdg.upload_eigens(svals, sv32, VEC_F32)
            sdg.upload_eigens(svals, sv32, VEC_BF16)
            sout = torch.empty(int(sidx[-1]), dtype=torch.float32, device="cuda")
            push["sparse_chunglu"] = {
                "graph": f"Chung-Lu {SPARSE['n0']} ids, {SPARSE['edges']} target edges, exponent "
                         f"{SPARSE['exponent']}, seed {SPARSE['seed']}, largest component: "
                         f"n={sg.n}, E={sg.num_edges}; omega=128, gamma=10",
                **push_bound_section(sdg, sidx, sg.num_edges, root, "sparse", (0.005,), stream,
                                     sout, flush, hbm, peak_kind, 3, not args.no_cpu_baseline)}
            sdg.free()

        cpu = None
        if not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            secs = cpu_reference_run(root, "cl4039", threads, 5, 1)
            if secs:
                one = cpu_reference_run(root, "cl4039", 1, 3, 1)
                cpu = cpu_baseline_line(E, secs, threads, one,
                                        "mean of 5 tgtp() calls (after 1 warm-up) of the reference "
                                        "benchmark binary on the same graph and eigen files")
        line = {
            "metric": METRIC, "value": value, "unit": "edges/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Chung-Lu graph + scipy eigenpairs)",
            "config": bench_config(world),
            "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                         "traffic": traffic, "algorithmic_bytes_per_launch": per_launch[top]},
            "kernel_share": share,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "edges/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "matches_resident_run": ok_e2e},
            # the library's kernels per step (from the event pass) times the timed steps
            "gpu_launches": int(round(sum(v[0] for v in k64.values()) / side_steps)) * args.steps,
            # cross-check: the library's own per-kernel events, summed per step (<= ms_per_step)
            "kernel_ms_sum_per_step": sum(v[1] for v in k64.values()) / side_steps,
            "clocks": clocks.summary(),
            "forms": {"fp64": {"edges_per_s": value / world, "ms_per_step": ms_step},
                      "fp32_reference_arithmetic": {"edges_per_s": E / (ms32 / side_steps * 1e-3),
                                                    "kernel_ms": {k: v[1] / v[0] for k, v in k32.items()}},
                      **{k: dict(v, edges_per_s=E / (v["ms_per_step"] * 1e-3),
                                 speedup_vs_fp64=ms_step / v["ms_per_step"])
                         for k, v in mixed.items()}},
            "saba": saba,
            "push_bound": push,
            "batch16": batch16,
            "wall_s_timed_region": wall64,
        }
        print(json.dumps(line))
    dg.free()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
