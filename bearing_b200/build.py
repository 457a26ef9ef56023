"""Builds the package's native libraries in-tree.

  bearing_b200/libbearing_gpu.so    nvcc, sm_100a only, FP64 with contraction off (-fmad=false)
  bearing_b200/libbearing_host.so   g++, -ffp-contract=off
  oracle/_build/liboracle.so        g++, -ffp-contract=off: the tests' CPU checker (built
                                    here because it is compiled code; nothing in the package
                                    loads it)

Every FP64 operation must round exactly as the reference's JavaScript does, so nothing is built
with fast-math, and multiply-adds are never fused.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", shutil.which("g++") or "g++")

GPU_SOURCES = [os.path.join(PKG, "csrc", "bearing_gpu.cu")]
GPU_DEPS = [os.path.join(PKG, "csrc", f) for f in ("layout.cuh", "stage.cuh", "adjoint.cuh", "tape.hpp", "colour.cuh", "contact.cuh")] + [
    os.path.join(PKG, "host", "collide_impl.hpp"), os.path.join(PKG, "host", "collide.hpp"),
    os.path.join(ROOT, "include", "bearing_gpu.h")]
HOST_SOURCES = [os.path.join(PKG, "host", "world.cpp"), os.path.join(PKG, "host", "collide.cpp")]
HOST_DEPS = [os.path.join(PKG, "host", "collide.hpp"), os.path.join(PKG, "host", "collide_impl.hpp"),
             os.path.join(PKG, "csrc", "tape.hpp"), os.path.join(ROOT, "include", "bearing_world.h"),
             os.path.join(ROOT, "include", "bearing_gpu.h")]
ORACLE_SOURCES = [os.path.join(ROOT, "oracle", "solve_stage.cpp")]

GPU_LIB = os.path.join(PKG, "libbearing_gpu.so")
HOST_LIB = os.path.join(PKG, "libbearing_host.so")
ORACLE_LIB = os.path.join(ROOT, "oracle", "_build", "liboracle.so")

# -split-compile=0 spreads the device code's optimisation over every host core (the one translation
# unit holds the stage, batch, adjoint and contact kernels); the arithmetic is the same IEEE FP64
# either way (no contraction, no reassociation), and the parity tests hold it to the oracle's bits.
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-lineinfo", "-fmad=false",
              "-split-compile=0", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math", "-shared"]
CXX_FLAGS = ["-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-Wall", "-Wextra"]


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build_gpu(force=False, verbose=False):
    if force or _stale(GPU_LIB, GPU_SOURCES + GPU_DEPS):
        extra = ["-Xptxas", "-v"] if verbose else []
        r = _run([NVCC] + NVCC_FLAGS + extra + ["-o", GPU_LIB] + GPU_SOURCES)
        if verbose:
            sys.stderr.write(r.stderr)
    return GPU_LIB


def build_host(force=False):
    if force or _stale(HOST_LIB, HOST_SOURCES + HOST_DEPS):
        _run([CXX] + CXX_FLAGS + ["-o", HOST_LIB] + HOST_SOURCES)
    return HOST_LIB


def build_oracle(force=False):
    os.makedirs(os.path.dirname(ORACLE_LIB), exist_ok=True)
    deps = [os.path.join(ROOT, "include", f) for f in ("bearing_gpu.h", "bearing_world.h")] + [
        os.path.join(ROOT, "oracle", "dual.hpp"), os.path.join(PKG, "host", "collide_impl.hpp")]
    if force or _stale(ORACLE_LIB, ORACLE_SOURCES + deps):
        _run([CXX] + CXX_FLAGS + ["-o", ORACLE_LIB] + ORACLE_SOURCES + ["-lpthread"])
    return ORACLE_LIB


def build(force=False, verbose=False):
    build_host(force)
    build_oracle(force)
    build_gpu(force, verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built", GPU_LIB, HOST_LIB, ORACLE_LIB)
