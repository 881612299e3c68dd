"""The drop-in headers (include/bfps: field, kspace, vorticity_equation,
particles/particles_system_builder) compile as bfps code is written and,
driven in the order NSVE / NSVEparticles call them (tests/cpp/
bfps_dropin.cpp), give the FP64 oracle's fields, tracer positions and
statistics to 1e-10, with the kspace tables of the reference
(kspace.cpp:34-167)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "bfps_dropin.cpp")
LIBDIR = os.path.join(ROOT, "bfps_b200", "_lib")


def _build(out):
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "include", "bfps"), SRC, "-o", out, "-L", LIBDIR,
           "-lbfps_b200", "-Wl,-rpath," + LIBDIR]
    subprocess.check_call(cmd)


def test_dropin_headers_compile_and_link(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    if not os.path.exists(os.path.join(LIBDIR, "libbfps_b200.so")):
        pytest.skip("library not built")
    _build(str(tmp_path / "bfps_dropin"))


@pytest.mark.gpu
def test_dropin_nsveparticles_matches_oracle(tmp_path):
    from bfps_b200 import ic
    from oracle import nsve as O
    from oracle import particles as P
    from oracle.nsveparticles import nsveparticles_step
    from gpu_util import rel_err
    n, nt, steps, dt, nbins = 32, 400, 3, 0.01, 64
    w0 = ic.vorticity_ic(n, seed=31)
    pos = ic.tracer_ic(nt, seed=32)
    exe = str(tmp_path / "bfps_dropin")
    _build(exe)
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(fin, "wb") as f:
        f.write(np.ascontiguousarray(w0).tobytes())
        f.write(np.ascontiguousarray(pos).tobytes())
    subprocess.check_call([exe, str(n), str(nt), str(steps), repr(dt), fin, fout])
    raw = open(fout, "rb").read()
    it, sidx, nshells, nh = np.frombuffer(raw[:16], np.int32)
    off = 16
    take = lambda dt_, cnt: np.frombuffer(raw, dt_, count=cnt, offset=off)
    w = take(np.complex128, w0.size).reshape(w0.shape); off += w.nbytes
    state = take(np.float64, 3 * nt).reshape(nt, 3); off += state.nbytes
    spec = take(np.float64, nshells * 9).reshape(nshells, 3, 3); off += spec.nbytes
    mom = take(np.float64, 40).reshape(10, 4); off += mom.nbytes
    hist = take(np.int64, nh).reshape(nbins, 4); off += hist.nbytes
    kM, dk, f10 = take(np.float64, 3); off += 24
    kshell = take(np.float64, nshells)
    assert it == steps and sidx == steps + 1

    ref = O.VorticityEquation(n)
    ref.nu, ref.forcing_type, ref.famplitude, ref.fk0, ref.fk1 = 0.05, "linear", 0.5, 1.5, 3.0
    ref.cvorticity = ref.read_checkpoint_semantics(w0)
    rps = P.ParticlesSystem(pos, np.zeros((3, nt, 3)), 3, 2, P.Geometry(n, n, n))
    for s in range(steps):
        if s == steps - 1:
            u = ref.compute_velocity(ref.cvorticity)
            sref, mref, href = O.compute_stats(ref, u, 1.0 / np.sqrt(3.0), nbins)
        nsveparticles_step(ref, rps, dt)
    assert rel_err(w, ref.cvorticity) < 1e-10
    assert rel_err(state, rps.pos) < 1e-10
    assert rel_err(spec, sref) < 1e-12
    assert rel_err(mom, mref) < 1e-10
    assert np.array_equal(hist, href)
    kk = ref.kk
    assert kM == kk.kM and dk == kk.dk and nshells == kk.nshells
    assert abs(f10 - kk.filter_table[10]) <= 1e-13 * abs(kk.filter_table[10])
    assert rel_err(kshell, kk.kshell) < 1e-13
