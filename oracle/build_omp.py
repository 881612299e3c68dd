"""Build the C++/OpenMP oracle (oracle/nsve_omp.cpp) into oracle/_lib/.

TEST INFRASTRUCTURE AND CPU BASELINE ONLY.  g++ compiles the one source file
(no external libraries) into ``oracle/_lib/libnsve_omp.so``; the library is
git-ignored and travels with the repository snapshot like the engine's own
shared library.  ``-ffp-contract=off`` keeps every product and sum a
separate rounding, as in the numpy restatement it is pinned against.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "nsve_omp.cpp")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libnsve_omp.so")


def build(force=False, verbose=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
           "-shared", "-fPIC", "-o", tmp, SRC]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="-f" in sys.argv, verbose=True))
