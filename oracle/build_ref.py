"""Build recipe for the oracle binaries (test infrastructure only).

Compiles, with g++/gcc on the host,
  * the reference's own step sources, read in place from the reference checkout
    (functions/{useful,rho,cell_phase,initialisation}_functions.cpp,
    functions/declare_tables.cpp, functions/declare_fft_tables.cpp and, for the
    executable, main_code/run_with_active_gels.cpp), together with this
    directory's ref_params.cpp, ref_harness.cpp and cufft_shim.c, into
      oracle/_ref/libref_fp32.so, oracle/_ref/ref_main_fp32   (shipped precision)
      oracle/_ref/libref_fp64.so, oracle/_ref/ref_main_fp64   (FP64 oracle)
    The FP64 build compiles a copy of those sources, written to a temporary
    directory outside the repository, in which every `float` token is replaced by
    `double`; nothing else is changed.  This is the reference's own FP64 run.
  * this directory's C restatement pfag_oracle.c (the oracle "port") into
      oracle/lib/liboracle_fp32.so, oracle/lib/liboracle_fp64.so
  * the reference's own main and host files linked against the package's
    drop-in libraries (its step functions over the B200 library):
      oracle/_ref/dropin_main_fp32, oracle/_ref/dropin_main_fp64
    the harness of the drop-in test, not a checker.
  * the reference's initial-condition program
    (initialisation_code/prepare_initial_files.cpp) with its step files:
      oracle/_ref/ref_prepare_fp32, oracle/_ref/ref_prepare_fp64

The reference build needs the reference checkout (default /root/reference,
override with PFAG_REFERENCE_DIR); where it is absent the prebuilt files in
oracle/_ref/ are used as they are.  Flags: -O3 without -march so the binaries
run on any x86-64 host, -ffp-contract=off so that no fused multiply-add changes
rounding between builds.
"""
from __future__ import annotations

import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
LIB_OUT = os.path.join(HERE, "lib")
REF_FUNCS = [
    "useful_functions.cpp", "rho_functions.cpp", "cell_phase_functions.cpp",
    "initialisation_functions.cpp", "declare_tables.cpp", "declare_fft_tables.cpp",
]
REF_HEADERS = [
    "constants.h", "declare_tables.h", "declare_fft_tables.h", "useful_functions.h",
    "rho_functions.h", "cell_phase_functions.h", "initialisation_functions.h",
]
CXXFLAGS = ["-std=c++14", "-O3", "-fPIC", "-ffp-contract=off", "-Drestrict=__restrict",
            "-Wno-unknown-pragmas", "-w"]
CFLAGS = ["-std=c11", "-O3", "-fPIC", "-ffp-contract=off", "-w"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def reference_dir() -> str | None:
    d = os.environ.get("PFAG_REFERENCE_DIR", "/root/reference")
    return d if os.path.isdir(os.path.join(d, "functions")) else None


def _build_reference(ref: str, double: bool) -> None:
    tag = "fp64" if double else "fp32"
    with tempfile.TemporaryDirectory(prefix=f"pfag_ref_{tag}_") as tmp:
        src_funcs = os.path.join(ref, "functions")
        src_main = os.path.join(ref, "main_code", "run_with_active_gels.cpp")
        if double:
            # float -> double token rewrite of a build-directory copy
            for name in REF_FUNCS + REF_HEADERS:
                text = open(os.path.join(src_funcs, name)).read()
                open(os.path.join(tmp, name), "w").write(re.sub(r"\bfloat\b", "double", text))
            text = open(src_main).read()
            open(os.path.join(tmp, "run_with_active_gels.cpp"), "w").write(
                re.sub(r"\bfloat\b", "double", text))
            inc = tmp
            funcs = [os.path.join(tmp, n) for n in REF_FUNCS]
            main = os.path.join(tmp, "run_with_active_gels.cpp")
        else:
            inc = src_funcs
            funcs = [os.path.join(src_funcs, n) for n in REF_FUNCS]
            main = src_main
        defs = ["-DPFAG_REF_DOUBLE"] if double else []
        incs = ["-I", os.path.join(HERE, "shim_include"), "-I", inc]
        objs = []
        for src in funcs + [os.path.join(HERE, "ref_params.cpp"), os.path.join(HERE, "ref_harness.cpp")]:
            obj = os.path.join(tmp, os.path.basename(src) + ".o")
            _run(["g++", *CXXFLAGS, *defs, *incs, "-c", src, "-o", obj])
            objs.append(obj)
        shim = os.path.join(tmp, "cufft_shim.o")
        _run(["gcc", *CFLAGS, *defs, "-I", os.path.join(HERE, "shim_include"), "-c",
              os.path.join(HERE, "cufft_shim.c"), "-o", shim])
        objs.append(shim)
        _run(["g++", "-shared", "-o", os.path.join(REF_OUT, f"libref_{tag}.so"), *objs, "-lm"])
        mobj = os.path.join(tmp, "main.o")
        _run(["g++", *CXXFLAGS, *defs, *incs, "-c", main, "-o", mobj])
        _run(["g++", "-o", os.path.join(REF_OUT, f"ref_main_{tag}"), mobj,
              *[o for o in objs if not o.endswith("ref_harness.cpp.o")], "-lm"])


# Host files of the reference that stay in a drop-in build: everything but the
# three step-function files that libpfag_dropin replaces.
DROPIN_KEPT = ["initialisation_functions.cpp", "declare_tables.cpp", "declare_fft_tables.cpp"]
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
PKG = os.path.join(HERE, "..", "multicellular_phase_field_active_gel_organoids_b200")


def _build_dropin_main(ref: str, double: bool) -> None:
    """The reference's own main (main_code/run_with_active_gels.cpp) and its
    host files, compiled as they are (float -> double rewritten for fp64) and
    linked against the package's libpfag_dropin_fp{32,64}.so in place of
    useful_functions.cpp, rho_functions.cpp and cell_phase_functions.cpp.
    Parameters come from ref_params.cpp (PFAG_REF_PARAMS), real cuFFT headers
    and library (main creates its two plans itself), an empty openacc.h."""
    tag = "fp64" if double else "fp32"
    with tempfile.TemporaryDirectory(prefix=f"pfag_dropin_{tag}_") as tmp:
        src_funcs = os.path.join(ref, "functions")
        src_main = os.path.join(ref, "main_code", "run_with_active_gels.cpp")
        if double:
            for name in DROPIN_KEPT + REF_HEADERS:
                text = open(os.path.join(src_funcs, name)).read()
                open(os.path.join(tmp, name), "w").write(re.sub(r"\bfloat\b", "double", text))
            text = open(src_main).read()
            open(os.path.join(tmp, "run_with_active_gels.cpp"), "w").write(re.sub(r"\bfloat\b", "double", text))
            inc = tmp
            srcs = [os.path.join(tmp, n) for n in DROPIN_KEPT] + [os.path.join(tmp, "run_with_active_gels.cpp")]
        else:
            inc = src_funcs
            srcs = [os.path.join(src_funcs, n) for n in DROPIN_KEPT] + [src_main]
        acc = os.path.join(tmp, "acc")
        os.makedirs(acc)
        open(os.path.join(acc, "openacc.h"), "w").write("/* empty: OpenACC pragmas are inert under g++ */\n")
        defs = ["-DPFAG_REF_DOUBLE"] if double else []
        incs = ["-I", acc, "-I", inc, "-I", os.path.join(CUDA_HOME, "include")]
        objs = []
        for src in srcs + [os.path.join(HERE, "ref_params.cpp")]:
            obj = os.path.join(tmp, os.path.basename(src) + ".o")
            _run(["g++", *CXXFLAGS, *defs, *incs, "-c", src, "-o", obj])
            objs.append(obj)
        dropin = os.path.abspath(os.path.join(PKG, "dropin"))
        _run(["g++", "-o", os.path.join(REF_OUT, f"dropin_main_{tag}"), *objs,
              "-L", dropin, f"-lpfag_dropin_{tag}", "-L", os.path.abspath(PKG), "-lpfag",
              "-L", os.path.join(CUDA_HOME, "lib64"), "-lcufft", "-lcudart",
              "-Wl,-rpath,$ORIGIN/../../multicellular_phase_field_active_gel_organoids_b200/dropin",
              "-Wl,-rpath,$ORIGIN/../../multicellular_phase_field_active_gel_organoids_b200",
              "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64"), "-lm"])


def _build_prepare(ref: str, double: bool) -> None:
    """The reference's initial-condition program
    (initialisation_code/prepare_initial_files.cpp) with its step files, built
    like the reference's main against the CPU cuFFT shim: the oracle of the
    device generator (pfag_generate_initial)."""
    tag = "fp64" if double else "fp32"
    with tempfile.TemporaryDirectory(prefix=f"pfag_prep_{tag}_") as tmp:
        src_funcs = os.path.join(ref, "functions")
        src_main = os.path.join(ref, "initialisation_code", "prepare_initial_files.cpp")
        if double:
            for name in REF_FUNCS + REF_HEADERS:
                text = open(os.path.join(src_funcs, name)).read()
                open(os.path.join(tmp, name), "w").write(re.sub(r"\bfloat\b", "double", text))
            text = open(src_main).read()
            open(os.path.join(tmp, "prepare_initial_files.cpp"), "w").write(re.sub(r"\bfloat\b", "double", text))
            inc = tmp
            srcs = [os.path.join(tmp, n) for n in REF_FUNCS] + [os.path.join(tmp, "prepare_initial_files.cpp")]
        else:
            inc = src_funcs
            srcs = [os.path.join(src_funcs, n) for n in REF_FUNCS] + [src_main]
        defs = ["-DPFAG_REF_DOUBLE"] if double else []
        incs = ["-I", os.path.join(HERE, "shim_include"), "-I", inc]
        objs = []
        for src in srcs + [os.path.join(HERE, "ref_params.cpp")]:
            obj = os.path.join(tmp, os.path.basename(src) + ".o")
            _run(["g++", *CXXFLAGS, *defs, *incs, "-c", src, "-o", obj])
            objs.append(obj)
        shim = os.path.join(tmp, "cufft_shim.o")
        _run(["gcc", *CFLAGS, *defs, "-I", os.path.join(HERE, "shim_include"), "-c",
              os.path.join(HERE, "cufft_shim.c"), "-o", shim])
        _run(["g++", "-o", os.path.join(REF_OUT, f"ref_prepare_{tag}"), *objs, shim, "-lm"])


def build_prepare(force: bool = False) -> bool:
    """Build oracle/_ref/ref_prepare_fp{32,64}; False when the checkout is absent."""
    ref = reference_dir()
    if ref is None:
        return False
    os.makedirs(REF_OUT, exist_ok=True)
    for double in (False, True):
        tag = "fp64" if double else "fp32"
        if force or not os.path.exists(os.path.join(REF_OUT, f"ref_prepare_{tag}")):
            _build_prepare(ref, double)
    return True


def build_dropin_main(force: bool = False) -> bool:
    """Build oracle/_ref/dropin_main_fp{32,64}; needs the reference checkout and
    the package's drop-in libraries.  False when the checkout is absent."""
    ref = reference_dir()
    if ref is None:
        return False
    os.makedirs(REF_OUT, exist_ok=True)
    for double in (False, True):
        tag = "fp64" if double else "fp32"
        out = os.path.join(REF_OUT, f"dropin_main_{tag}")
        lib = os.path.join(PKG, "dropin", f"libpfag_dropin_{tag}.so")
        if not os.path.exists(lib):
            raise RuntimeError(f"{lib} is missing: build the package first")
        if force or not os.path.exists(out):
            _build_dropin_main(ref, double)
    return True


def build_reference(force: bool = False) -> bool:
    """Build oracle/_ref from the reference checkout; False when it is absent."""
    ref = reference_dir()
    if ref is None:
        return False
    os.makedirs(REF_OUT, exist_ok=True)
    for double in (False, True):
        tag = "fp64" if double else "fp32"
        if force or not os.path.exists(os.path.join(REF_OUT, f"libref_{tag}.so")):
            _build_reference(ref, double)
    return True


def build_port(force: bool = False) -> None:
    """Build the C restatement (always possible: it is this repository's code)."""
    os.makedirs(LIB_OUT, exist_ok=True)
    src = os.path.join(HERE, "pfag_oracle.c")
    shim = os.path.join(HERE, "cufft_shim.c")
    for double in (False, True):
        tag = "fp64" if double else "fp32"
        out = os.path.join(LIB_OUT, f"liboracle_{tag}.so")
        if not force and os.path.exists(out) and os.path.getmtime(out) >= max(
                os.path.getmtime(src), os.path.getmtime(shim)):
            continue
        defs = ["-DPFAG_REF_DOUBLE"] if double else []
        _run(["gcc", *CFLAGS, "-shared", *defs, "-I", os.path.join(HERE, "shim_include"),
              src, shim, "-o", out, "-lm"])


def main() -> int:
    force = "--force" in sys.argv
    build_port(force)
    ok = build_reference(force)
    if ok:
        build_prepare(force)
        build_dropin_main(force)
    print("oracle port built;", "reference built" if ok else "reference checkout absent (prebuilt files kept)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
