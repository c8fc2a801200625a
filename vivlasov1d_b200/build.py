"""Build libvv.so (the CUDA kernels and the C ABI) in-tree for sm_100a.

    python -m vivlasov1d_b200.build [--verbose]

The library is written next to this file so that it travels with the source
tree; nothing is installed into site-packages or a JIT cache.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libvv.so")

SOURCES = ["vv_api.cu", "vv_noalloc.cu"]
HEADERS = ["vv_common.cuh", "vv_bracket.cuh", "vv_pc.cuh", "vv_pcj.cuh", "vv_pcv.cuh", "vv_coll.cuh", "vv_vec.cuh", "vv_batch.cuh", "vv_adjoint.cuh", "vv_pred.cuh"]

NVCC_FLAGS = [
    "-O3", "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC,-O3",
    "--expt-relaxed-constexpr",
]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force=False, verbose=False):
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(INCLUDE, "vv.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + ["-I", INCLUDE, "-I", CSRC, "-shared", "-o", LIB + ".tmp"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("nvcc failed building libvv.so")
    if verbose:
        sys.stderr.write(proc.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build_library(force=True, verbose="--verbose" in sys.argv)
    print(LIB)
