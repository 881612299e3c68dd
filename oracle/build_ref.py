"""Build the reference's own interpolation-kernel sources into oracle/_ref/.

TEST INFRASTRUCTURE ONLY. bfps' weight polynomials live in plain C++ files
that include nothing but <cmath> and their own headers
(bfps/cpp/Lagrange_polys.cpp, bfps/cpp/spline_n1.cpp .. spline_n10.cpp), so
they compile on their own.  This recipe runs g++ directly on those files
where they lie in the reference checkout and writes one shared library,
``oracle/_ref/libbfps_interp_ref.so``, which the CPU tests load to pin the
exact-rational restatement in ``oracle/interp.py`` (and through it the
coefficient header used by the CUDA gather kernel).

No reference source is copied; where the checkout is absent the build is
skipped and a previously built library is used if present.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libbfps_interp_ref.so")
REF_ROOT = os.environ.get("BFPS_REFERENCE", "/root/reference")
REF_CPP = os.path.join(REF_ROOT, "bfps", "cpp")


def build(verbose=False):
    if not os.path.isdir(REF_CPP):
        return os.path.exists(LIB)
    srcs = [os.path.join(REF_CPP, "Lagrange_polys.cpp")] + [
        os.path.join(REF_CPP, "spline_n%d.cpp" % n) for n in range(1, 11)]
    srcs.append(os.path.join(HERE, "ref_interp_shim.cpp"))
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) > os.path.getmtime(s) for s in srcs):
        return True
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["g++", "-O2", "-shared", "-fPIC", "-I", REF_CPP, "-o", LIB] + srcs
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return True


def load():
    """ctypes handle to the reference library, or None if not built."""
    import ctypes
    if not os.path.exists(LIB):
        return None
    return ctypes.CDLL(LIB)


if __name__ == "__main__":
    ok = build(verbose=True)
    print("built" if ok else "reference sources absent; nothing built")
    sys.exit(0)
