"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle (oracle/tgtp_oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this package, and only
as the checker.  The product (tgtp_b200/ and the C-ABI library) never loads it.

`build()` compiles the restatement (and, where the reference sources are present, the reference
binaries under oracle/_ref/) with oracle/Makefile.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
# The reference checkout (ggokturk/tgtp); TGTP_REFERENCE overrides the default location.
REFERENCE = os.environ.get("TGTP_REFERENCE", "/root/reference")
REFERENCE_SRC = os.path.join(REFERENCE, "src")

_lib = None


class Stats(C.Structure):
    _fields_ = [(name, C.c_uint64) for name in (
        "push_rounds", "push_vertices", "push_traversals", "walk_edges", "walk_count",
        "walk_hops", "fallback_bouquets", "tau_iterations")]

    def as_dict(self):
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


def build(reference: bool = True) -> None:
    """Compile liboracle.so and, when the reference sources exist here, oracle/_ref/*."""
    subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)
    if reference and os.path.isdir(REFERENCE_SRC):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "-j4", "REF=" + REFERENCE], check=True)


def ref_binary(name: str) -> str | None:
    p = os.path.join(REF_DIR, name)
    return p if os.access(p, os.X_OK) else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(reference=False)
        L = C.CDLL(LIB_PATH)
        u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
        u64p = np.ctypeslib.ndpointer(np.uint64, flags="C")
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
        vp = C.c_void_p
        L.oracle_saba.argtypes = [u32p, u32p, C.c_uint64, C.c_uint32, C.c_uint32, u64p, C.c_int]
        L.oracle_taus_f32.argtypes = [u32p, u32p, C.c_uint64, f64p, f32p, C.c_int, C.c_double,
                                      i32p, vp, C.c_int]
        L.oracle_taus_f64.argtypes = [u32p, u32p, C.c_uint64, f64p, f64p, C.c_int, C.c_double,
                                      i32p, vp, C.c_int]
        for fn, vec in ((L.oracle_tgtp_f32, f32p), (L.oracle_tgtp_f64, f64p)):
            fn.argtypes = [u32p, u32p, C.c_uint64, f64p, vec, C.c_int, C.c_double, C.c_double,
                           C.c_int, f32p, vp, vp, vp, vp, vp, C.c_int]
        L.oracle_parse_eigens.argtypes = [C.c_char_p, C.c_uint64, C.c_int, f64p, vp, vp]
        L.oracle_walk2_f32.argtypes = [u32p, u32p, C.c_uint32, C.c_uint32, C.c_uint64,
                                       C.c_uint32, f32p]
        L.oracle_walk2_f32.restype = C.c_float
        L.oracle_mt19937_nth.argtypes = [C.c_uint32, C.c_uint64]
        L.oracle_mt19937_nth.restype = C.c_uint32
        L.oracle_mt_walks.argtypes = [u32p, u32p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_int, u64p,
                                      C.c_int]
        for fn in (L.oracle_saba, L.oracle_taus_f32, L.oracle_taus_f64, L.oracle_tgtp_f32,
                   L.oracle_tgtp_f64, L.oracle_parse_eigens, L.oracle_mt_walks):
            fn.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def saba(idx, adj, depth, n_walks, threads=0):
    """Per-vertex visit counters (uint64) of the SABA walk from every vertex."""
    n = len(idx) - 1
    out = np.zeros(n, dtype=np.uint64)
    rc = lib().oracle_saba(idx, adj, n, depth, n_walks, out, threads)
    if rc:
        raise ValueError("n_walks must be a multiple of 8")
    return out


def mt19937_nth(seed, k):
    """The k-th draw (1-based) of std::mt19937 seeded with `seed`."""
    return int(lib().oracle_mt19937_nth(seed, k))


def mt_walks(idx, adj, depth, n_walks, simd=False, threads=0):
    """Per-vertex visit counters (uint64) of the reference's MT19937 walk baseline (scalar or
    8-lane bouquet draw order) from every vertex with a neighbour."""
    n = len(idx) - 1
    out = np.zeros(n, dtype=np.uint64)
    rc = lib().oracle_mt_walks(idx, adj, n, depth, n_walks, 1 if simd else 0, out, threads)
    if rc:
        raise ValueError("n_walks must be a multiple of 8")
    return out


def taus(idx, adj, values, vectors, eps_half, fp64=False, threads=0):
    n = len(idx) - 1
    out = np.zeros(int(idx[-1]), dtype=np.int32)
    st = Stats()
    fn = lib().oracle_taus_f64 if fp64 else lib().oracle_taus_f32
    vec = np.ascontiguousarray(vectors, dtype=np.float64 if fp64 else np.float32)
    fn(idx, adj, n, values, vec, len(values), eps_half, out, C.byref(st), threads)
    return out, st.as_dict()


def tgtp(idx, adj, values, vectors, eps, gamma=10, fp64=False, threads=0, details=False,
         delta=None):
    """Full tgtp(); returns float32 scores (and per-slot details when asked)."""
    n = len(idx) - 1
    m = int(idx[-1])
    scores = np.zeros(m, dtype=np.float32)
    st = Stats()
    tau = np.zeros(m, dtype=np.int32) if details else None
    ell = np.zeros(n, dtype=np.int32) if details else None
    pre = np.zeros(m, dtype=np.float64 if fp64 else np.float32) if details else None
    nr = np.zeros(m, dtype=np.uint64) if details else None
    vec = np.ascontiguousarray(vectors, dtype=np.float64 if fp64 else np.float32)
    fn = lib().oracle_tgtp_f64 if fp64 else lib().oracle_tgtp_f32
    d = 1.0 / n if delta is None else delta
    rc = fn(idx, adj, n, np.ascontiguousarray(values, np.float64), vec, len(values), eps, d,
            gamma, scores, _ptr(tau), _ptr(ell), _ptr(pre), _ptr(nr), C.byref(st), threads)
    if rc:
        raise RuntimeError("oracle tgtp failed")
    if details:
        return scores, dict(taus=tau, ell=ell, presym=pre, nr=nr, stats=st.as_dict())
    return scores


def parse_eigens(path, n, omega):
    """(values f64[omega], vec_f32[n*omega], vec_f64[n*omega]) with the reference's parsing."""
    values = np.zeros(omega, dtype=np.float64)
    v32 = np.zeros(n * omega, dtype=np.float32)
    v64 = np.zeros(n * omega, dtype=np.float64)
    rc = lib().oracle_parse_eigens(path.encode(), n, omega, values, _ptr(v32), _ptr(v64))
    if rc:
        raise RuntimeError(f"invalid eigen file {path} ({rc})")
    return values, v32, v64


def walk2(idx, adj, src, v, num_walk, len_walk, pvec):
    return float(lib().oracle_walk2_f32(idx, adj, src, v, num_walk, len_walk,
                                        np.ascontiguousarray(pvec, np.float32)))
