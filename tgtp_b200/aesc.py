"""Python mirror of the reference's tgtp interface, on the sm_100a library.

Names and argument meanings follow the reference so that its callers read the same:

    AESCGraph(graph_path, eigen_path, omega)      src/aesc.h:83-97
    AESCConfig(epsilon, delta, omega, gamma)      src/aesc.h:98-102
    AESC(graph, config).tgtp() -> float32[m]      src/aesc.h:113-127
    saba_count(graph, depth, n_walks)             src/rw_experiment_saba.cpp:65-145, 186-208

Errors raise `TgtpError` (the reference throws std::runtime_error / std::invalid_argument; its CLI
maps them to "tgtp: <msg>" and exit 1).  All compute runs in libtgtp_gpu.so on the current CUDA
device; nothing here computes scores on the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (PRECISION_FP32, PRECISION_FP64, PRECISION_MIXED, VEC_BF16, VEC_F32, VEC_F64,
                   TgtpError, check, lib, ptr)

__all__ = ["AESCGraph", "AESCConfig", "AESC", "Batch", "saba_count", "load_graph_txt", "load_eigens_txt",
           "TgtpError", "PRECISION_FP32", "PRECISION_FP64", "PRECISION_MIXED", "VEC_F32", "VEC_F64",
           "VEC_BF16"]


def load_graph_txt(path: str):
    """graph.txt -> (idx uint32[n+1], adj uint32[m]) exactly as src/graph.h:29-97 builds them."""
    L = lib()
    ip, ap = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
    n, m = C.c_uint64(), C.c_uint64()
    check(L.tgtp_load_graph_txt(path.encode(), C.byref(ip), C.byref(ap), C.byref(n), C.byref(m)))
    try:
        idx = np.ctypeslib.as_array(ip, shape=(n.value + 1,)).copy()
        adj = np.ctypeslib.as_array(ap, shape=(max(m.value, 1),))[: m.value].copy()
    finally:
        L.tgtp_host_free(C.cast(ip, C.c_void_p))
        L.tgtp_host_free(C.cast(ap, C.c_void_p))
    return idx, adj


def load_eigens_txt(path: str, n: int, omega: int, f32: bool = True, f64: bool = True):
    """sorted_eigens_<omega>.txt -> (values f64[omega], vectors f32[n*omega] | None,
    vectors f64[n*omega] | None), vertex-major, parsed as src/aesc.h:51-64 does."""
    values = np.zeros(omega, np.float64)
    v32 = np.zeros(n * omega, np.float32) if f32 else None
    v64 = np.zeros(n * omega, np.float64) if f64 else None
    check(lib().tgtp_load_eigens_txt(path.encode(), n, omega, ptr(values),
                                     ptr(v32) if v32 is not None else None,
                                     ptr(v64) if v64 is not None else None))
    return values, v32, v64


@dataclass
class AESCConfig:
    """src/aesc.h:98-102 plus the arithmetic form of this implementation."""

    epsilon: float
    delta: float = 0.0          # 0 -> 1/n, what the reference's callers set (src/main.cpp:36)
    omega: int = 128
    gamma: int = 10
    precision: int = PRECISION_FP32
    vec_dtype: int = VEC_F32

    def to_c(self, n: int) -> _lib.Config:
        d = self.delta if self.delta > 0 else 1.0 / n
        return _lib.Config(self.epsilon, d, self.omega, self.gamma, self.precision, self.vec_dtype)


class AESCGraph:
    """Device-resident CSR (+ eigenpairs).  src/aesc.h:83-97."""

    def __init__(self, graph_path: str | None = None, eigen_path: str | None = None,
                 omega: int | None = None, *, store=(VEC_F32, VEC_F64)):
        self._h = None
        if graph_path is None:
            return
        idx, adj = load_graph_txt(graph_path)
        self._upload(idx, adj)
        if eigen_path is not None:
            if omega is None or omega < 2 or omega > self.n:
                raise TgtpError(1, "omega must be between 2 and vertex count")
            deg = np.diff(self.idx.astype(np.int64))
            if np.any(deg == 0):
                raise TgtpError(1, "graph vertex IDs must be contiguous with no isolated vertices")
            vals, v32, v64 = load_eigens_txt(eigen_path, self.n, omega,
                                             f32=VEC_F32 in store or VEC_BF16 in store,
                                             f64=VEC_F64 in store)
            for st in store:
                if st == VEC_F64:
                    self.upload_eigens(vals, v64, VEC_F64)
                else:
                    self.upload_eigens(vals, v32, st)

    @classmethod
    def from_csr(cls, idx, adj, values=None, vectors=None, store=None) -> "AESCGraph":
        g = cls()
        g._upload(np.ascontiguousarray(idx, np.uint32), np.ascontiguousarray(adj, np.uint32))
        if values is not None:
            g.upload_eigens(values, vectors, store)
        return g

    def _upload(self, idx, adj):
        h = C.c_void_p()
        n = len(idx) - 1
        m = int(idx[-1])
        check(lib().tgtp_graph_upload(ptr(idx), ptr(adj) if m else None, n, m, C.byref(h)))
        self._h = h
        self.idx, self.adj, self.n, self.m = idx, adj, n, m

    def upload_eigens(self, values, vectors, store=None):
        values = np.ascontiguousarray(values, np.float64)
        vectors = np.asarray(vectors)
        host = VEC_F64 if vectors.dtype == np.float64 else VEC_F32
        vectors = np.ascontiguousarray(vectors, np.float64 if host == VEC_F64 else np.float32)
        store = host if store is None else store
        check(lib().tgtp_eigens_upload(self._h, ptr(values), ptr(vectors), len(values), host,
                                       store))
        self.omega = len(values)

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr: int | None):
        check(lib().tgtp_graph_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def set_profiling(self, on: bool):
        check(lib().tgtp_graph_set_profiling(self._h, 1 if on else 0))

    def kernel_stats(self):
        arr = (_lib.KernelStat * 32)()
        cnt = C.c_int32()
        check(lib().tgtp_graph_kernel_stats(self._h, arr, 32, C.byref(cnt)))
        return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].total_ms))
                for i in range(min(cnt.value, 32))}

    def set_trace(self, on: bool):
        """Record, in every later run, the rounds pushed per row and the walk count per slot."""
        check(lib().tgtp_graph_set_trace(self._h, 1 if on else 0))

    def read_trace(self):
        """(walk count per slot (m), rounds pushed per row (n)) of the last traced run; rows scored
        in closed form and slots without walks read 0."""
        nr = np.zeros(self.m, dtype=np.uint32)
        ell = np.zeros(self.n, dtype=np.uint32)
        check(lib().tgtp_graph_read_trace(self._h, nr.ctypes.data, ell.ctypes.data))
        return nr, ell

    def free(self):
        if self._h is not None:
            check(lib().tgtp_graph_free(self._h))
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class AESC:
    """src/aesc.h:113-127: tgtp() returns the m float32 scores in CSR order (symmetric)."""

    def __init__(self, g: AESCGraph, config: AESCConfig):
        self.g = g
        self.config = config

    def tgtp(self) -> np.ndarray:
        out = np.empty(self.g.m, np.float32)
        cfg = self.config.to_c(self.g.n)
        check(lib().tgtp_run(self.g.handle, C.byref(cfg), ptr(out)))
        return out

    def tgtp_device(self, device_ptr: int) -> None:
        """Scores into caller-owned device memory, asynchronous on the graph's stream."""
        cfg = self.config.to_c(self.g.n)
        check(lib().tgtp_run_device(self.g.handle, C.byref(cfg), C.c_void_p(device_ptr)))

    def stats(self) -> dict:
        st = _lib.RunStats()
        check(lib().tgtp_last_run_stats(self.g.handle, C.byref(st)))
        return st.as_dict()

    def taus(self) -> np.ndarray:
        out = np.empty(self.g.m, np.int32)
        check(lib().tgtp_last_taus(self.g.handle, ptr(out)))
        return out

    def tune(self, device_ptr: int, trials: int = 3) -> int:
        """Times the source-kernel layouts for this form on this graph and keeps the fastest
        (tgtp_graph_tune); returns the layout code (0x100 = shared memory | warps per block)."""
        cfg = self.config.to_c(self.g.n)
        code = C.c_int32(0)
        check(lib().tgtp_graph_tune(self.g.handle, C.byref(cfg), C.c_void_p(device_ptr), trials,
                                    C.byref(code)))
        return int(code.value)


class Batch:
    """Many tgtp() runs replayed as one CUDA graph (tgtp_batch_*).  `runs` is a list of
    (AESC, device output pointer); every graph may appear once."""

    def __init__(self, runs, tune_trials: int = 0):
        self.runs = list(runs)
        k = len(self.runs)
        graphs = (C.c_void_p * k)(*[a.g.handle for a, _ in self.runs])
        cfgs = (_lib.Config * k)(*[a.config.to_c(a.g.n) for a, _ in self.runs])
        outs = (C.c_void_p * k)(*[C.c_void_p(p) for _, p in self.runs])
        h = C.c_void_p()
        check(lib().tgtp_batch_create(graphs, cfgs, outs, k, tune_trials, C.byref(h)))
        self._h = h

    def run(self, stream_ptr: int | None = None) -> None:
        check(lib().tgtp_batch_run(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def wait(self) -> None:
        check(lib().tgtp_batch_wait(self._h))

    def free(self) -> None:
        if self._h is not None:
            check(lib().tgtp_batch_free(self._h))
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def saba_count(g: AESCGraph, depth: int, n_walks: int, counters: bool = True):
    """(counters uint32[n] | None, visit_count, checksum, fallback_bouquets)."""
    out = np.empty(g.n, np.uint32) if counters else None
    res = _lib.SabaResult()
    check(lib().saba_count(g.handle, depth, n_walks, ptr(out) if out is not None else None,
                           C.byref(res)))
    return out, int(res.visit_count), int(res.checksum), int(res.fallback_bouquets)


def mt_walk_count(g: AESCGraph, depth: int, n_walks: int, simd: bool = False,
                  counters: bool = True):
    """The reference's MT19937 walk baselines (scalar or, with simd, 8-lane bouquet draw order):
    (counters uint32[n] | None, visit_count, checksum)."""
    out = np.empty(g.n, np.uint32) if counters else None
    res = _lib.SabaResult()
    check(lib().mt_walk_count(g.handle, depth, n_walks, 1 if simd else 0,
                              ptr(out) if out is not None else None, C.byref(res)))
    return out, int(res.visit_count), int(res.checksum)


def saba_tune(g: AESCGraph, depth: int, n_walks: int, trials: int = 3) -> int:
    """Times the walk layouts for this graph and configuration and keeps the fastest on the
    handle; returns the choice (low byte: walkers per lane, 0x100: inlined walk copy, bits 12-14:
    c for 1024 x c row records in shared memory)."""
    choice = C.c_int32(0)
    check(lib().saba_tune(g.handle, depth, n_walks, trials, C.byref(choice)))
    return int(choice.value)


def exact_sc_slots(g: AESCGraph, slots, tol: float = 1e-10, max_iter: int = 20000):
    """Exact spanning centrality (effective resistance) of the given CSR slots on the device:
    (resistances float64[len(slots)], iterations per batch of 32 slots)."""
    slots = np.ascontiguousarray(slots, dtype=np.uint32)
    out = np.empty(len(slots), np.float64)
    iters = np.zeros(max(1, (len(slots) + 31) // 32), np.uint32)
    check(lib().tgtp_exact_sc_slots(g.handle, ptr(slots), len(slots), tol, max_iter, ptr(out),
                                    ptr(iters)))
    return out, iters
