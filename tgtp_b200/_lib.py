"""ctypes binding of libtgtp_gpu.so (include/tgtp_gpu.h).

The shared library is built in-tree by tgtp_b200.build.  Loading it is mandatory: there is no CPU
fallback anywhere in this package, and every entry point raises if the library is missing or a
call fails.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libtgtp_gpu.so")

STATUS = {0: "OK", 1: "INVALID_ARGUMENT", 2: "CUDA", 3: "OUT_OF_MEMORY", 4: "TIMEOUT", 5: "IO",
          6: "UNSUPPORTED", 7: "OVERFLOW"}

VEC_F32, VEC_F64, VEC_BF16 = 0, 1, 2
PRECISION_FP32, PRECISION_FP64, PRECISION_MIXED = 0, 1, 2


class TgtpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.message = message


class Config(C.Structure):
    _fields_ = [("epsilon", C.c_double), ("delta", C.c_double), ("omega", C.c_int32),
                ("gamma", C.c_int32), ("precision", C.c_int32), ("vec_dtype", C.c_int32)]


class RunStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in (
        "push_rounds", "push_vertices", "push_traversals", "walk_edges", "walk_count",
        "walk_hops", "fallback_bouquets", "tau_iterations", "tau_ambiguous")] + [
        ("phase_cycles", C.c_uint64 * 8)]

    PHASES = ("init", "push", "post_push", "cost_test", "edge_bound", "chi_nr", "walks", "reset")

    def as_dict(self):
        d = {k: int(getattr(self, k)) for k, _ in self._fields_ if k != "phase_cycles"}
        d["phase_cycles"] = dict(zip(self.PHASES, (int(x) for x in self.phase_cycles)))
        return d


class SabaResult(C.Structure):
    _fields_ = [("visit_count", C.c_uint64), ("checksum", C.c_uint64),
                ("fallback_bouquets", C.c_uint64)]


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("launches", C.c_uint64), ("total_ms", C.c_double)]


# every symbol include/tgtp_gpu.h declares, with its ctypes signature
_vp, _u32p, _u64 = C.c_void_p, C.POINTER(C.c_uint32), C.c_uint64
SIGNATURES = {
    "tgtp_last_error": (C.c_char_p, []),
    "tgtp_abi_version": (C.c_int, []),
    "tgtp_load_graph_txt": (C.c_int, [C.c_char_p, C.POINTER(_u32p), C.POINTER(_u32p),
                                      C.POINTER(_u64), C.POINTER(_u64)]),
    "tgtp_load_eigens_txt": (C.c_int, [C.c_char_p, _u64, C.c_uint32, _vp, _vp, _vp]),
    "tgtp_host_free": (None, [_vp]),
    "tgtp_graph_upload": (C.c_int, [_vp, _vp, _u64, _u64, C.POINTER(_vp)]),
    "tgtp_graph_free": (C.c_int, [_vp]),
    "tgtp_graph_set_stream": (C.c_int, [_vp, _vp]),
    "tgtp_graph_stream": (_vp, [_vp]),
    "tgtp_graph_info": (C.c_int, [_vp, C.POINTER(_u64), C.POINTER(_u64)]),
    "tgtp_eigens_upload": (C.c_int, [_vp, _vp, _vp, C.c_uint32, C.c_int32, C.c_int32]),
    "tgtp_run": (C.c_int, [_vp, C.POINTER(Config), _vp]),
    "tgtp_run_device": (C.c_int, [_vp, C.POINTER(Config), _vp]),
    "tgtp_last_run_stats": (C.c_int, [_vp, C.POINTER(RunStats)]),
    "tgtp_last_taus": (C.c_int, [_vp, _vp]),
    "saba_count": (C.c_int, [_vp, C.c_uint32, C.c_uint32, _vp, C.POINTER(SabaResult)]),
    "saba_count_device": (C.c_int, [_vp, C.c_uint32, C.c_uint32, _vp]),
    "saba_tune": (C.c_int, [_vp, C.c_uint32, C.c_uint32, C.c_int32, C.POINTER(C.c_int32)]),
    "tgtp_exact_sc_slots": (C.c_int, [_vp, _vp, C.c_uint32, C.c_double, C.c_uint32, _vp, _vp]),
    "saba_count_static": (C.c_int, [_vp, _vp, _u64, C.c_uint32, C.c_uint32, _vp,
                                    C.POINTER(SabaResult)]),
    "tgtp_graph_tune": (C.c_int, [_vp, C.POINTER(Config), _vp, C.c_int32, C.POINTER(C.c_int32)]),
    "tgtp_batch_create": (C.c_int, [C.POINTER(_vp), C.POINTER(Config), C.POINTER(_vp), C.c_uint32,
                                    C.c_int32, C.POINTER(_vp)]),
    "tgtp_batch_run": (C.c_int, [_vp, _vp]),
    "tgtp_batch_wait": (C.c_int, [_vp]),
    "tgtp_batch_free": (C.c_int, [_vp]),
    "tgtp_release_cached_memory": (C.c_int, []),
    "tgtp_graph_set_profiling": (C.c_int, [_vp, C.c_int]),
    "tgtp_graph_kernel_stats": (C.c_int, [_vp, C.POINTER(KernelStat), C.c_int32,
                                          C.POINTER(C.c_int32)]),
    "tgtp_graph_set_trace": (C.c_int, [_vp, C.c_int]),
    "mt_walk_count": (C.c_int, [_vp, C.c_uint32, C.c_uint32, C.c_int32, _vp, C.POINTER(SabaResult)]),
    "tgtp_graph_read_trace": (C.c_int, [_vp, _vp, _vp]),
}

_lib = None


def lib():
    """The loaded library; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m tgtp_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != 0:
        msg = lib().tgtp_last_error()
        raise TgtpError(status, msg.decode() if msg else "")


def ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)
