"""Build recipe of the engine's shared library (sm_100a) and of the CPU oracle.

    python -m futhark-benchmarks_b200.build      (or: python futhark-benchmarks_b200/build.py)

produces, in tree (so the library travels with the repository):

    futhark-benchmarks_b200/liblvc.so   the C-ABI library (include/LocVolCalib.h, tridiag.h)
    futhark-benchmarks_b200/libtke.so   the ocean model's tke step (include/tke.h)
    oracle/liblvc_oracle.so             the CPU oracle (tests and CPU baseline only)

nvcc cross-compiles for sm_100a without a GPU.  CUDA runtime is linked
statically, so the library depends only on the NVIDIA driver.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "liblvc.so")
TKE_LIB = os.path.join(PKG, "libtke.so")
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liblvc_oracle.so")

SOURCES = ["lvc_runtime.cu"]
HEADERS = ["lvc_kernels.cuh", "lvc_layout.h", "lvc_probe.cuh", "lvc_line.cuh", "lvc_pair.cuh", "lvc_tridiag.cuh"]
TKE_SOURCES = ["tke_runtime.cu"]
TKE_HEADERS: list = []
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-shared", "-cudart", "static",
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(force: bool = False, verbose: bool = False, extra=()) -> str:
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(REPO, "include", "LocVolCalib.h"))
    deps.append(os.path.join(REPO, "include", "tridiag.h"))
    deps.append(os.path.abspath(__file__))
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", os.path.join(REPO, "include"), "-I", CSRC,
           "-o", LIB + ".tmp", *[os.path.join(CSRC, f) for f in SOURCES]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_tke(force: bool = False, verbose: bool = False, extra=()) -> str:
    """libtke.so: a library of its own, since misc/ocean-sim/tke.fut's entry
    point is named futhark_entry_main like LocVolCalib's."""
    deps = [os.path.join(CSRC, f) for f in TKE_SOURCES + TKE_HEADERS]
    deps += [os.path.join(REPO, "include", "tke.h"), os.path.abspath(__file__)]
    if not force and not _stale(TKE_LIB, deps):
        return TKE_LIB
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", os.path.join(REPO, "include"), "-I", CSRC,
           "-o", TKE_LIB + ".tmp", *[os.path.join(CSRC, f) for f in TKE_SOURCES]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(TKE_LIB + ".tmp", TKE_LIB)
    return TKE_LIB


def build_oracle(force: bool = False) -> str:
    src = os.path.join(ORACLE_DIR, "lvc_oracle.cpp")
    if force or _stale(ORACLE_LIB, [src, os.path.join(ORACLE_DIR, "Makefile")]):
        subprocess.run(["make", "-C", ORACLE_DIR, "-B" if force else "--no-print-directory"],
                       check=True)
    return ORACLE_LIB


def main(argv=None) -> None:
    argv = sys.argv[1:] if argv is None else argv
    force = "--force" in argv
    verbose = "-v" in argv
    build_lib(force=force, verbose=verbose)
    build_tke(force=force, verbose=verbose)
    build_oracle(force=force)
    print(LIB)
    print(TKE_LIB)
    print(ORACLE_LIB)


if __name__ == "__main__":
    main()
