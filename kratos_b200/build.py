"""Build the sm_100a engine (kratos_b200/libkrb200.so) with nvcc, and
problem-generator executables on the C++ host layer (kratos_b200/host).

    python -m kratos_b200.build                      # the engine
    python -m kratos_b200.build --pgen usr.cpp -o kratos.x   # a pgen executable

A pgen written for the original Kratos (prob::run enrolling dynamics::hydro_t /
mhd_t subclasses, mesh.init / mesh.evolve) compiles unchanged against the host
headers and runs on the B200 engine.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "libkrb200.so")
SOURCES = [os.path.join(PKG, "csrc", f) for f in ("kr_core.cu", "kr_learn.cu")]
DEPS = SOURCES + [os.path.join(PKG, "csrc", f) for f in ("kr_math.cuh", "kr_fast.cuh", "kr_mlp.cuh", "problems.h",
                                                         "smr_tree.h", "kr_batch.cuh", "kr_smr_mhd.cuh")] + [
    os.path.join(ROOT, "include", "kratos_b200.h")]

HOST = os.path.join(PKG, "host")
HOST_SOURCES = [os.path.join(HOST, "src", f) for f in ("host.cpp", "main.cpp")]
CXX_FLAGS = ["-std=c++17", "-O2", "-ffp-contract=off"]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo",
              "-std=c++17", "-Xcompiler", "-fPIC", "-shared"]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


# Parity variant: the same sources without fused multiply-add (every product
# rounded before the add, as the reference's CPU build computes), so FP64 steps
# can be compared with the reference where rounding decides a solver branch.
# Test infrastructure; the product is LIB.
LIB_NOFMA = os.path.join(PKG, "libkrb200_nofma.so")


def up_to_date(lib=LIB):
    if not os.path.exists(lib):
        return False
    t = os.path.getmtime(lib)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def build(force=False, verbose=False):
    for lib, extra in ((LIB, []), (LIB_NOFMA, ["--fmad=false"])):
        if not force and up_to_date(lib):
            continue
        cmd = [nvcc()] + NVCC_FLAGS + extra + ["-I", os.path.join(ROOT, "include"), "-o", lib] + SOURCES
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


def build_host(pgen_sources, out, verbose=False):
    """Compile a problem generator with the host layer into the executable
    `out`, linked against libkrb200.so (found through its rpath)."""
    build(verbose=verbose)
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx] + CXX_FLAGS + ["-I", os.path.join(HOST, "include"), "-I", os.path.join(ROOT, "include"),
                               "-o", out] + HOST_SOURCES + list(pgen_sources) + [
        "-L", PKG, "-lkrb200", "-Wl,-rpath," + PKG]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return out


if __name__ == "__main__":
    if "--pgen" in sys.argv:
        a = sys.argv
        srcs = [a[i + 1] for i in range(len(a) - 1) if a[i] == "--pgen"]
        build_host(srcs, a[a.index("-o") + 1] if "-o" in a else "kratos.x", verbose=True)
    else:
        build(force="--force" in sys.argv, verbose=True)
