"""Builds the in-tree shared library tensors_b200/libtensors_b200.so.

nvcc compiles the CUDA kernels for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) together with the host-side symbolic
analysis and the C-ABI.  The system g++ is the host compiler so the library
links the process's libstdc++ dynamically.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtensors_b200.so")
BUILD_DIR = os.path.join(HERE, "_build")

SOURCES = ["trace.cpp", "symbolic.cpp", "plan.cpp", "plan_check.cpp", "schedule.cpp", "batch.cpp", "serve.cpp", "matrix_market.cpp", "ordering.cpp", "kernels.cu", "gemm_tc.cu", "handle.cu"]
HEADERS = ["trace.hpp", "common.hpp", "parallel.hpp", "symbolic.hpp", "plan.hpp", "plan_check.hpp", "schedule.hpp", "kernels.cuh"]

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "tensors_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source into libtensors_b200.so (skipped when up to date)."""
    if not force and not _stale():
        return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    common = [
        "-std=c++17", "-O3", "-lineinfo", *GENCODE,
        "-Xcompiler", "-fPIC", "-ccbin", _host_cxx(),
        "-I", os.path.join(HERE, "..", "include"),
    ]
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(BUILD_DIR, src + ".o")
        cmd = [nvcc, *common, "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(" ".join(cmd) + "\n" + (out or ""))
        failed |= p.returncode != 0
    if failed:
        raise RuntimeError("nvcc compilation failed")
    tmp = LIB + ".tmp"
    link = [nvcc, *GENCODE, "-shared", "-ccbin", _host_cxx(), "-o", tmp, *objs, "-lcudart_static", "-lpthread", "-ldl", "-lrt"]
    subprocess.run(link, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
