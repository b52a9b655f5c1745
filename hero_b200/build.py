"""Builds the in-tree native artefacts.

    python -m hero_b200.build          # libhero_b200.so (sm_100a) + the hero_b200 drop-in CLI

nvcc cross-compiles for sm_100a without a GPU.  The outputs are written next
to the sources (hero_b200/libhero_b200.so, hero_b200/bin/hero_b200) so they
travel with the tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
LIB = os.path.join(HERE, "libhero_b200.so")
PEAK_LIB = os.path.join(HERE, "libhero_peak.so")
CLI = os.path.join(HERE, "bin", "hero_b200")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-O3"]
CU_SOURCES = ["hero_kernels.cu", "hero_api.cu", "hero_noalloc.cu", "hero_server.cu"]
PEAK_SOURCES = ["int_peak.cu"]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=not verbose, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout or ''}{r.stderr or ''}")


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps(folder, exts):
    if not os.path.isdir(folder):
        return []
    return [os.path.join(folder, f) for f in os.listdir(folder) if f.endswith(exts)]


def build_library(verbose: bool = False, force: bool = False) -> str:
    deps = ([os.path.join(CSRC, s) for s in CU_SOURCES] + _deps(CSRC, (".cuh", ".h")) +
            [os.path.join(ROOT, "include", "hero_gpu.h")])
    if not force and not _stale(LIB, deps):
        return LIB
    tmp = LIB + ".tmp"
    _run([NVCC] + ARCH + NVFLAGS + ["-shared", "-o", tmp] +
         [os.path.join(CSRC, s) for s in CU_SOURCES], verbose)
    os.replace(tmp, LIB)
    return LIB


def build_peak(verbose: bool = False, force: bool = False) -> str:
    deps = [os.path.join(CSRC, s) for s in PEAK_SOURCES]
    if not force and not _stale(PEAK_LIB, deps):
        return PEAK_LIB
    _run([NVCC] + ARCH + NVFLAGS + ["-shared", "-o", PEAK_LIB] + deps, verbose)
    return PEAK_LIB


def build_cli(verbose: bool = False, force: bool = False) -> str | None:
    srcs = sorted(_deps(HOST, (".cpp",)))
    if not srcs:
        return None
    deps = srcs + _deps(HOST, (".h",)) + [LIB]
    if not force and not _stale(CLI, deps):
        return CLI
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    cxx = shutil.which("g++") or "g++"
    _run([cxx, "-std=c++17", "-O3", "-pthread", "-I", os.path.join(ROOT, "include"), "-o", CLI]
         + srcs + ["-L", HERE, "-lhero_b200", "-Wl,-rpath,$ORIGIN/.."], verbose)
    return CLI


def build(verbose: bool = False, force: bool = False):
    build_library(verbose, force)
    build_peak(verbose, force)
    build_cli(verbose, force)


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
