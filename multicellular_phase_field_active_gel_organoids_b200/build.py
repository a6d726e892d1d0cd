"""Build libpfag.so (the CUDA kernels and the C ABI) for sm_100a, in-tree,
and the drop-in libraries dropin/libpfag_dropin_fp{32,64}.so over it.

nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3 ... -shared, linked
against cuFFT (the plain comparison path) and the CUDA runtime.  The drop-in
libraries (the reference's step functions with their C++ signatures, in float
and in double) are host C++ compiled by g++ and linked against libpfag.so with
an $ORIGIN-relative run path.  Everything lands next to this file so it travels
with the source tree.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpfag.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
# The plain path mirrors the reference's FP64 operation order; without
# contraction into fused multiply-adds its rounding matches a host build of the
# reference, which keeps the far-field branch decisions (|grad phi| > 0 on the
# 2^-54 staircase of the initial profile) identical.
# The fused FP32 path keeps FP64 only for sums; its divisions and square roots
# are the hardware approximations (a few ulp), not the IEEE-rounded sequences.
PER_FILE = {"pfag_plain.cu": ["-fmad=false"], "pfag_fused_f64.cu": ["-fmad=false"],
            "pfag_fused_f32.cu": ["-prec-div=false", "-prec-sqrt=false"]}
OBJ_DIR = os.path.join(HERE, "_build")
DROPIN_SRC = os.path.join(HERE, "dropin", "pfag_dropin.cpp")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def dropin_lib(precision: int) -> str:
    return os.path.join(HERE, "dropin", f"libpfag_dropin_fp{precision}.so")


def build_dropin(force: bool = False) -> list[str]:
    """g++ the drop-in shim in float (fp32) and double (fp64)."""
    out = []
    inc = os.path.join(HERE, "..", "include")
    for prec in (32, 64):
        lib = dropin_lib(prec)
        out.append(lib)
        if not force and os.path.exists(lib) and os.path.getmtime(lib) >= max(
                os.path.getmtime(DROPIN_SRC), os.path.getmtime(LIB)):
            continue
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", "-Wno-unused-parameter",
               *(["-DPFAG_DROPIN_DOUBLE"] if prec == 64 else []),
               "-I", inc, "-I", os.path.join(CUDA_HOME, "include"), DROPIN_SRC, "-o", lib,
               "-L", HERE, "-lpfag", "-Wl,-rpath,$ORIGIN/..",
               "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("g++ failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return out


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps() -> list[str]:
    return sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [
        os.path.join(HERE, "..", "include", "pfag.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)

    def compile_one(src):
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, *PER_FILE.get(os.path.basename(src), []), "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose:
            sys.stderr.write(r.stderr)
        return obj

    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, sources()))
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcufft", "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print("\n".join(build_dropin(force="--force" in sys.argv)))
