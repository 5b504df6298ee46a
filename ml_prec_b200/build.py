"""Builds the CUDA library ml_prec_b200/lib/libmlp_b200.so for sm_100a, the
C++ host interface lib/libml_prec_host.so above it (host/ml_prec.h, the
reference's types and calls) and the command-line driver lib/ml_prec_b200.

Each .cu file under csrc/ is compiled with nvcc; setup.cu (the hierarchy
construction) is compiled with -fmad=false so that its floating-point
expressions round exactly like the reference's CPU build. Run as
``python -m ml_prec_b200.build`` or through ``__graft_entry__.build()``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib")
LIB = os.path.join(OUT, "libmlp_b200.so")
HOST = os.path.join(HERE, "host")
HOST_LIB = os.path.join(OUT, "libml_prec_host.so")
HOST_EXE = os.path.join(OUT, "ml_prec_b200")
INCLUDE = os.path.join(HERE, "..", "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "--expt-relaxed-constexpr", "-DNDEBUG"]
NO_FMA = {"setup.cu"}
SOURCES = ["util.cu", "setup.cu", "small.cu", "persist.cu", "solve.cu", "adjoint.cu", "capi.cu"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    objdir = os.path.join(OUT, "obj")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "mlp_b200.h"))
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nvcc()] + ARCH + COMMON + (["-fmad=false"] if src in NO_FMA else []) + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    build_host(verbose, force)
    return LIB


def build_host(verbose: bool = False, force: bool = False):
    """g++ build of the C++ host interface and driver, linked to the CUDA library."""
    hdrs = [os.path.join(HOST, "ml_prec.h"), os.path.join(INCLUDE, "mlp_b200.h")]
    flags = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-I" + HOST, "-I" + INCLUDE]
    rpath = "-Wl,-rpath,$ORIGIN"
    steps = [
        (HOST_LIB, [os.path.join(HOST, "ml_prec.cc")] + hdrs + [LIB],
         ["g++"] + flags + ["-shared", os.path.join(HOST, "ml_prec.cc"), "-o", HOST_LIB, "-L" + OUT, "-lmlp_b200",
                            rpath]),
        (HOST_EXE, [os.path.join(HOST, "main.cc"), HOST_LIB] + hdrs,
         ["g++"] + flags + [os.path.join(HOST, "main.cc"), "-o", HOST_EXE, "-L" + OUT, "-lml_prec_host",
                            "-lmlp_b200", rpath]),
    ]
    for target, deps, cmd in steps:
        if force or _stale(target, deps):
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
