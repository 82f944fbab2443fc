"""Builds the engine's shared library in-tree with nvcc for sm_100a.

The library (gtpower_b200/lib/libgtpb200.so) exports the C ABI of
include/gtpb200.h; it has no dependency on torch or Python.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libgtpb200.so")
SYNTH_LIB = os.path.join(LIBDIR, "libgtpb200_synth.so")
SYNTHDEV_LIB = os.path.join(LIBDIR, "libgtpb200_synthdev.so")

ENGINE_SOURCES = ["abi.cu", "power_kernel.cu", "pack.cpp", "writers.cpp", "vcd_gpu.cu", "umma_gemm.cu", "proxy.cu"]
SYNTH_SOURCES = ["synth.cpp"]
SYNTHDEV_SOURCES = ["synth_dev.cu"]

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def cutlass_include() -> str:
    """CuTe/CUTLASS header tree (descriptor unions for tcgen05 operands).
    Taken from an installed package that vendors it; not linked, headers only."""
    import importlib.util
    cands = [os.environ.get("CUTLASS_INCLUDE", "")]
    for pkg, sub in (("flashinfer", ("data", "cutlass", "include")),
                     ("tilelang", ("3rdparty", "cutlass", "include"))):
        spec = importlib.util.find_spec(pkg)
        if spec is not None and spec.submodule_search_locations:
            cands.append(os.path.join(spec.submodule_search_locations[0], *sub))
    for c in cands:
        if c and os.path.exists(os.path.join(c, "cute", "arch", "mma_sm100_desc.hpp")):
            return c
    raise RuntimeError("CuTe headers (cute/arch/mma_sm100_desc.hpp) not found; set CUTLASS_INCLUDE")


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    deps = sources + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    incdir = os.path.join(os.path.dirname(HERE), "include")
    deps += [os.path.join(incdir, f) for f in os.listdir(incdir) if f.endswith(".h")]
    return any(os.path.getmtime(s) > t for s in deps if os.path.exists(s))


def build_engine(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, f) for f in ENGINE_SOURCES]
    if not force and not _newer(LIB, srcs):
        return LIB
    cmd = [nvcc(), *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "-shared", "-I", cutlass_include(),
           "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
           "-o", LIB, *srcs, "-lpthread"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return LIB


def build_synth(force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, f) for f in SYNTH_SOURCES]
    if not force and not _newer(SYNTH_LIB, srcs):
        return SYNTH_LIB
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-pthread",
           "-o", SYNTH_LIB, *srcs]
    subprocess.run(cmd, check=True)
    return SYNTH_LIB


def build_synthdev(force: bool = False) -> str:
    """The synthetic-trace generator on the GPU (sm_100a)."""
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, f) for f in SYNTHDEV_SOURCES]
    if not force and not _newer(SYNTHDEV_LIB, srcs):
        return SYNTHDEV_LIB
    cmd = [nvcc(), *ARCH_FLAGS, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-o", SYNTHDEV_LIB, *srcs]
    subprocess.run(cmd, check=True)
    return SYNTHDEV_LIB


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_engine(force=force, verbose=verbose)
    build_synth(force=force)
    build_synthdev(force=force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
