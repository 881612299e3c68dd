"""Build the CUDA engine into bfps_b200/_lib/libbfps_b200.so (sm_100a).

    python -m bfps_b200.build            # or bfps_b200.build.build()

Compiles bfps_b200/csrc/bfps_b200.cu with nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a); the shared library stays in the
source tree so that it ships with the repository snapshot.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libbfps_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
         "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cuh", ".h", ".inl"))] + [os.path.join(INCLUDE, "bfps_b200.h")]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force=False, verbose=False, extra=()):
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + FLAGS + list(extra) + [
        "-I", INCLUDE, "-I", CSRC, os.path.join(CSRC, "bfps_b200.cu"), "-o", tmp]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    verbose = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else []
    print(build(force=True, verbose=verbose, extra=extra))
