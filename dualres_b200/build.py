"""Build the sm_100a shared library dualres_b200/_lib/libdualres_b200.so.

nvcc cross-compiles for sm_100a without a GPU.  The library is built in-tree
so that it travels with the repository snapshot; nothing is installed.

    python -m dualres_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libdualres_b200.so")
# the bounds-checked build (DRB_BOUNDS_CHECK): every data-dependent index tested before its access; loaded instead of
# LIB when DRB_LIBRARY=checked
LIB_CHECKED = os.path.join(LIBDIR, "libdualres_b200_checked.so")
SOURCES = ["api.cu", "host_setup.cpp", "estimate.cpp"]
DEPS = ["api.cu", "kernels.cu", "common.cuh", "fft.cuh", "tma.cuh", "mce.cuh", "kriging.cuh", "umma.cuh",
        "tc_products.cuh", "drb.h", "host_setup.cpp", "host_setup.h", "estimate.cpp", "estimate.h"]
CLI = os.path.join(LIBDIR, "dualgpmf")
CLI_SOURCES = ["dualgpmf.cpp", "nifti.cpp"]
CLI_DEPS = CLI_SOURCES + ["nifti.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(lib=LIB):
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    inc = os.path.join(HERE, "..", "include", "dualres_b200.h")
    deps = [os.path.join(CSRC, d) for d in DEPS] + [inc]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def _cli_stale():
    if not os.path.exists(CLI):
        return True
    t = os.path.getmtime(CLI)
    inc = os.path.join(HERE, "..", "include", "dualres_b200.h")
    deps = [os.path.join(CSRC, d) for d in CLI_DEPS] + [inc, LIB]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build_cli(force=False, verbose=False):
    """The dualgpmf command line, linked against the library (found next to it at run time)."""
    if not force and not _cli_stale():
        return CLI
    gxx = shutil.which("g++") or "g++"
    cmd = [gxx, "-std=c++17", "-O2", "-fopenmp", "-o", CLI + ".tmp",
           *[os.path.join(CSRC, s) for s in CLI_SOURCES], "-L" + LIBDIR, "-ldualres_b200", "-lz",
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=not verbose, text=True)
    if res.returncode != 0:
        sys.stderr.write((res.stdout or "") + (res.stderr or ""))
        raise RuntimeError("g++ failed (dualgpmf)")
    os.replace(CLI + ".tmp", CLI)
    return CLI


def _compile(lib, extra, verbose):
    os.makedirs(LIBDIR, exist_ok=True)
    gxx = shutil.which("g++") or "g++"
    cmd = [nvcc_path(), "-shared", "-std=c++17", "-O3", "-lineinfo", *ARCH, *extra,
           "-ccbin", gxx, "-Xcompiler", "-fPIC,-fopenmp,-O3",
           "--expt-relaxed-constexpr", "-Xptxas", "-O3",
           "-o", lib + ".tmp", *[os.path.join(CSRC, s) for s in SOURCES], "-lgomp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=not verbose, text=True)
    if res.returncode != 0:
        sys.stderr.write((res.stdout or "") + (res.stderr or ""))
        raise RuntimeError("nvcc failed")
    os.replace(lib + ".tmp", lib)


def build(force=False, verbose=False, checked=False):
    """The library (and the dualgpmf command line); with checked=True also the bounds-checked library."""
    if force or _stale():
        _compile(LIB, [], verbose)
        build_cli(True, verbose)
    else:
        build_cli(force, verbose)
    if checked and (force or _stale(LIB_CHECKED)):
        _compile(LIB_CHECKED, ["-DDRB_BOUNDS_CHECK"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, checked="--checked" in sys.argv)
    print(LIB)
