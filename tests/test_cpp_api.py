"""The C++ mirror (include/bfps_b200.hpp) of vorticity_equation,
particles_system and NSVEparticles::step: it compiles against the C-ABI, and
a C++ program driving it the way NSVEparticles does gives bit for bit the
results of the same calls through the Python mirror (also when the steps go
through a one-member C++ ensemble), and the oracle's to 1e-10 in FP64."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "nsve_cpp.cpp")
LIBDIR = os.path.join(ROOT, "bfps_b200", "_lib")


def _build(out):
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           SRC, "-o", out, "-L", LIBDIR, "-lbfps_b200", "-Wl,-rpath," + LIBDIR]
    subprocess.check_call(cmd)


def test_cpp_mirror_compiles_and_links(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    if not os.path.exists(os.path.join(LIBDIR, "libbfps_b200.so")):
        pytest.skip("library not built")
    _build(str(tmp_path / "nsve_cpp"))


@pytest.mark.gpu
@pytest.mark.parametrize("precision,mode", [("double", "alone"), ("single", "alone"),
                                            ("single", "ensemble")])
def test_cpp_driver_matches_python_mirror_and_oracle(tmp_path, precision, mode):
    from bfps_b200 import ic
    from bfps_b200.solver import vorticity_equation, particles_system, NSVEparticles_step
    from oracle import nsve as O
    from oracle import particles as P
    from oracle.nsveparticles import nsveparticles_step
    from gpu_util import rel_err
    n, nt, steps, dt = 32, 300, 4, 0.01
    rb = 8 if precision == "double" else 4
    cdt = np.complex128 if rb == 8 else np.complex64
    w0 = ic.vorticity_ic(n, seed=12, dtype=cdt)
    pos = ic.tracer_ic(nt, seed=13)
    exe = str(tmp_path / "nsve_cpp")
    _build(exe)
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(fin, "wb") as f:
        f.write(np.ascontiguousarray(w0).tobytes())
        f.write(np.ascontiguousarray(pos).tobytes())
    subprocess.check_call([exe, str(rb), str(n), str(nt), str(steps), repr(dt), fin, fout] +
                          (["ensemble"] if mode == "ensemble" else []))
    raw = open(fout, "rb").read()
    it, sidx = np.frombuffer(raw[:8], np.int32)
    off = 8
    w = np.frombuffer(raw, cdt, count=w0.size, offset=off).reshape(w0.shape)
    off += w.nbytes
    state = np.frombuffer(raw, np.float64, count=3 * nt, offset=off).reshape(nt, 3)
    off += state.nbytes
    rhs = np.frombuffer(raw, np.float64, count=9 * nt, offset=off).reshape(3, nt, 3)
    off += rhs.nbytes
    acc = np.frombuffer(raw, np.float64, count=3 * nt, offset=off).reshape(nt, 3)
    assert it == steps and sidx == 1 + steps

    # the same calls through the Python mirror
    ve = vorticity_equation(n, precision=precision)
    ve.nu, ve.forcing_type, ve.famplitude, ve.fk0, ve.fk1 = 0.05, "linear", 0.5, 1.5, 3.0
    ve.io_checkpoint_read(w0)
    ps = particles_system(ve, pos, 2, 1, 3)
    NSVEparticles_step(ve, ps, dt, steps)
    p_state, p_rhs, _ = ps.state()
    assert np.array_equal(w, ve.get_cvorticity())
    assert np.array_equal(state, p_state) and np.array_equal(rhs, p_rhs)
    assert np.array_equal(acc, ps.sample_acceleration())
    ps.close()
    ve.close()

    if precision == "double":
        ref = O.VorticityEquation(n)
        ref.nu, ref.forcing_type, ref.famplitude, ref.fk0, ref.fk1 = 0.05, "linear", 0.5, 1.5, 3.0
        ref.cvorticity = ref.read_checkpoint_semantics(w0)
        rps = P.ParticlesSystem(pos, np.zeros((3, nt, 3)), 2, 1, P.Geometry(n, n, n))
        for _ in range(steps):
            nsveparticles_step(ref, rps, dt)
        assert rel_err(w, ref.cvorticity) < 1e-10
        assert rel_err(state, rps.pos) < 1e-10
        ar = ref.ift(ref.compute_lagrangian_acceleration())
        assert rel_err(acc, P.sample(ar, rps.pos, 2, 1, P.Geometry(n, n, n))) < 1e-10
