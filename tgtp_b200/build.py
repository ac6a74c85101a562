"""In-tree build of libtgtp_gpu.so (sm_100a) and the drop-in host runners.

    python -m tgtp_b200.build            # library + runners, only what is out of date
    python -m tgtp_b200.build --force    # rebuild everything
    python -m tgtp_b200.build --verbose  # also print ptxas register / spill / shared-memory lines

Outputs (git-ignored, they travel with the tree):
    tgtp_b200/libtgtp_gpu.so
    tgtp_b200/bin/{tgtp,benchmark,rw_experiment_saba,rw_experiment,rw_experiment_simd}
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libtgtp_gpu.so")
BIN = os.path.join(PKG, "bin")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-I" + INCLUDE, "-I" + CSRC, "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-I" + INCLUDE, "-I" + CSRC,
             "-I" + os.path.join(CUDA_HOME, "include")]

CU_SOURCES = ["api.cu", "saba.cu", "aesc.cu", "batch.cu", "exact_sc.cu", "mt_walk.cu"]
CPP_SOURCES = ["host_io.cpp"]
# executable -> (source under csrc/host, extra flags)
RUNNERS = {"tgtp": ("tgtp_main.cpp", []), "benchmark": ("benchmark_main.cpp", []),
           "rw_experiment_saba": ("rw_experiment_saba_main.cpp", []),
           "rw_experiment": ("rw_experiment_main.cpp", []),
           "rw_experiment_simd": ("rw_experiment_main.cpp", ["-DTGTP_MT_SIMD"])}


def _headers():
    return glob.glob(os.path.join(CSRC, "*.hpp")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h")) + glob.glob(os.path.join(INCLUDE, "*.hpp")) + \
        glob.glob(os.path.join(CSRC, "host", "*.hpp"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    out = (res.stdout + res.stderr).strip()
    if verbose and out:
        print(out, flush=True)
    return out


def build(force: bool = False, verbose: bool = False, runners: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + headers):
            extra = ["-Xptxas", "-v"] if verbose else []
            _run([NVCC] + NVCC_FLAGS + extra + ["-c", s, "-o", o], verbose)
        objs.append(o)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + headers):
            _run(["g++"] + CXX_FLAGS + ["-c", s, "-o", o], verbose)
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt",
                                                             "-lpthread", "-ldl"], verbose)
    if runners:
        os.makedirs(BIN, exist_ok=True)
        for name, (src, flags) in RUNNERS.items():
            s = os.path.join(CSRC, "host", src)
            if not os.path.exists(s):
                continue
            exe = os.path.join(BIN, name)
            if force or _stale(exe, [s, LIB] + headers):
                _run(["g++"] + CXX_FLAGS + flags + ["-o", exe, s, "-L" + PKG, "-ltgtp_gpu",
                                                    "-Wl,-rpath,$ORIGIN/.."], verbose)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
