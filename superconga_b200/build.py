"""Builds libscb200.so (the C-ABI engine) in-tree for sm_100a.

nvcc compiles the CUDA engine and g++ the host setup; both are linked into
``superconga_b200/libscb200.so``.  The build is incremental on source mtimes.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
ROOT = os.path.dirname(PKG)
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libscb200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps():
    return _sources() + glob.glob(os.path.join(CSRC, "*.hpp")) + glob.glob(os.path.join(CSRC, "*.cuh")) + [
        os.path.join(ROOT, "include", "scb200.h"), os.path.abspath(__file__)] + glob.glob(
        os.path.join(CSRC, "driver", "*"))


def up_to_date() -> bool:
    if not os.path.exists(LIB) or not all(os.path.exists(d) for d in DRIVERS.values()):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    for src in _sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if src.endswith(".cu"):
            cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp",
                   "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
        else:
            cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-fopenmp", "-I", os.path.join(ROOT, "include"),
                   "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-Xcompiler", "-fopenmp", "-o", tmp, *objs, "-lcudart", "-lgomp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    build_driver(verbose)
    return LIB


DRIVERS = {name: os.path.join(PKG, "bin", name) for name in ("simulation_b200", "postprocess_b200")}
DRIVER = DRIVERS["simulation_b200"]


def build_driver(verbose: bool = False) -> None:
    """The drop-in simulation and postprocess executables, linked against libscb200.so."""
    for name, exe in DRIVERS.items():
        os.makedirs(os.path.dirname(exe), exist_ok=True)
        cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
               os.path.join(CSRC, "driver", name + ".cpp"), "-o", exe,
               "-L", PKG, "-lscb200", "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
