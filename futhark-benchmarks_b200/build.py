"""Build recipe of the engine's shared library (sm_100a) and of the CPU oracle.

    python -m futhark-benchmarks_b200.build      (or: python futhark-benchmarks_b200/build.py)

produces, in tree (so the library travels with the repository):

    futhark-benchmarks_b200/liblvc.so   the C-ABI library (include/LocVolCalib.h, tridiag.h)
    futhark-benchmarks_b200/libtke.so   the ocean model's tke step (include/tke.h)
    futhark-benchmarks_b200/libop.so    finpar OptionPricing (include/op.h)
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
OP_LIB = os.path.join(PKG, "libop.so")
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liblvc_oracle.so")

SOURCES = ["lvc_runtime.cu"]
HEADERS = ["lvc_kernels.cuh", "lvc_layout.h", "lvc_probe.cuh", "lvc_line.cuh", "lvc_pair.cuh", "lvc_tridiag.cuh"]
TKE_SOURCES = ["tke_runtime.cu"]
TKE_HEADERS = ["fut_api.cuh"]
OP_SOURCES = ["op_runtime.cu"]
OP_HEADERS = ["fut_api.cuh"]
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


def _build_program_lib(lib: str, sources, headers, public_header: str, force: bool, verbose: bool, extra) -> str:
    deps = [os.path.join(CSRC, f) for f in list(sources) + list(headers)]
    deps += [os.path.join(REPO, "include", public_header), os.path.abspath(__file__)]
    if not force and not _stale(lib, deps):
        return lib
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", os.path.join(REPO, "include"), "-I", CSRC,
           "-o", lib + ".tmp", *[os.path.join(CSRC, f) for f in sources]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(lib + ".tmp", lib)
    return lib


def build_tke(force: bool = False, verbose: bool = False, extra=()) -> str:
    """libtke.so: a library of its own, since misc/ocean-sim/tke.fut's entry
    point is named futhark_entry_main like LocVolCalib's."""
    return _build_program_lib(TKE_LIB, TKE_SOURCES, TKE_HEADERS, "tke.h", force, verbose, extra)


def build_op(force: bool = False, verbose: bool = False, extra=()) -> str:
    """libop.so: finpar/OptionPricing.fut's generated API.  --fmad=false
    rounds every f32 multiply and add on its own, as the reference does."""
    return _build_program_lib(OP_LIB, OP_SOURCES, OP_HEADERS, "op.h", force, verbose, ("--fmad=false", *extra))


def build_oracle(force: bool = False) -> str:
    srcs = [os.path.join(ORACLE_DIR, f) for f in ("lvc_oracle.cpp", "op_oracle.cpp", "Makefile")]
    if force or _stale(ORACLE_LIB, srcs):
        subprocess.run(["make", "-C", ORACLE_DIR, "-B" if force else "--no-print-directory"],
                       check=True)
    return ORACLE_LIB


def main(argv=None) -> None:
    argv = sys.argv[1:] if argv is None else argv
    force = "--force" in argv
    verbose = "-v" in argv
    build_lib(force=force, verbose=verbose)
    build_tke(force=force, verbose=verbose)
    build_op(force=force, verbose=verbose)
    build_oracle(force=force)
    print(LIB)
    print(TKE_LIB)
    print(OP_LIB)
    print(ORACLE_LIB)


if __name__ == "__main__":
    main()
