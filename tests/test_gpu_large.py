"""Parity at the grid sizes the benchmark runs (256^3 and 512^3).

The smaller parity tests (32^3 - 128^3) do not reach the code paths the
benchmark sizes instantiate: the 8/4-column kx tiles of the column passes
and their Nyquist-only last tile (257 = 32*8 + 1 columns at 512^3), the
dynamic tile tickets of the two-CTA IZ pass, the 512-point shared-memory
transforms, and the periodic tracer cell re-sort, which only runs on grids of
256^3 and above.  Here the engine is compared at those sizes with

* pocketfft (scipy.fft, all host cores) for field::dft / field::ift;
* the C++/OpenMP oracle (oracle/nsve_omp.cpp, pinned on the numpy oracle by
  tests/test_oracle_omp.py, which is pinned on the reference's golden
  fixture) for the NSVEparticles step, FP64 at 1e-10 over six steps at
  256^3 (re-sort included) and FP32 against FP64 at 512^3 with the C3
  configuration.
"""
import os

import numpy as np
import pytest

from oracle import nsve as O
from oracle import fast as F
from bfps_b200 import ic
from gpu_util import rel_err

pytestmark = pytest.mark.gpu

WORKERS = os.cpu_count() or 1


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("n,precision", [(256, "single"), (256, "double"), (512, "single")])
def test_dft_ift_bench_sizes(n, precision):
    import torch
    from bfps_b200.solver import vorticity_equation
    from bfps_b200 import _lib
    ve = vorticity_equation(n, precision=precision)
    rng = np.random.default_rng(n + (7 if precision == "double" else 0))
    r = rng.standard_normal((n, n, n, 3)).astype(ve.rdtype)
    din = _dev(O.real_to_padded(r))
    c_ref = O.dft(r.astype(np.float64), workers=WORKERS)
    ctype = torch.complex64 if precision == "single" else torch.complex128
    dout = torch.zeros(ve.cshape, dtype=ctype, device="cuda")
    _lib.check(_lib.lib().bfg_dft(ve.handle, din.data_ptr(), dout.data_ptr()), ve.handle)
    tol = 1e-13 if precision == "double" else 3e-6
    assert rel_err(dout.cpu().numpy(), c_ref) < tol
    del dout, din
    # inverse of the Hermitian spectrum gives back n^3 r; padding stays zero
    cin = _dev(c_ref.astype(ve.cdtype))
    back = torch.zeros(ve.rshape, dtype=torch.float32 if precision == "single" else torch.float64,
                       device="cuda")
    _lib.check(_lib.lib().bfg_ift(ve.handle, cin.data_ptr(), back.data_ptr()), ve.handle)
    rb = back.cpu().numpy()
    assert np.all(rb[:, :, n:, :] == 0)
    assert rel_err(rb[:, :, :n], r.astype(np.float64) * float(n) ** 3) < tol
    ve.close()


def test_fp64_256_nsveparticles_six_steps_with_resort():
    """256^3 FP64, tracers on the C3 kernel (n = 3, m = 2) with AB3, six
    NSVEparticles steps: the cell re-sort (every 4 loops from 256^3 up) runs
    before the fifth loop.  Fields, positions and rhs histories within 1e-10
    of the FP64 oracle after every step (particles_system.hpp:210-217,
    vorticity_equation.cpp:358-439)."""
    from bfps_b200.solver import vorticity_equation, particles_system, NSVEparticles_step
    n, ntr, dt = 256, 20000, 0.002
    ve = vorticity_equation(n, precision="double")
    ref = F.VorticityEquation(n)
    for obj in (ve, ref):
        obj.nu, obj.forcing_type, obj.famplitude, obj.fk0, obj.fk1 = 0.005, "linear", 0.5, 1.5, 3.0
    w0 = ic.vorticity_ic(n, seed=0)
    ve.set_cvorticity(w0)
    ref.cvorticity = w0
    del w0
    pos = ic.tracer_ic(ntr, seed=1)
    ps = particles_system(ve, pos, 3, 2, 3)
    rps = F.ParticlesSystem(ref, pos, np.zeros((3, ntr, 3)), 3, 2)
    for s in range(6):
        NSVEparticles_step(ve, ps, dt)
        F.nsveparticles_step(ref, rps, dt)
        err = rel_err(ve.get_cvorticity(), ref.cvorticity)
        got, rhs, _ = ps.state()
        want, wrhs, wsi = rps.state()
        perr = rel_err(got, want)
        rerr = rel_err(rhs, wrhs)
        assert err < 1e-10, (s, err)
        assert perr < 1e-10 and rerr < 1e-10, (s, perr, rerr)
    assert ve.iteration == 6 and ps.step_idx == wsi == 7
    ps.close()
    ve.close()


def test_fp32_512_c3_step_against_fp64_oracle():
    """The C3 configuration (512^3, nu = 0.002, dt = 0.001, k0 = 4, linear
    forcing on 1.5 <= |k| <= 3, smooth dealiasing, 4e6 tracers with n = 3,
    m = 2 and AB3), one NSVEparticles step in FP32 against the FP64 oracle
    from the same FP32-rounded initial field and tracers.  Bounds: the field
    within 2e-5 of max|w| (the FP32-vs-FP64 bound of the 32^3 test), the
    sampled velocity within 1e-5 of max|u|, positions within 1e-9 of the
    box."""
    from bfps_b200.solver import vorticity_equation, particles_system, NSVEparticles_step
    n, ntr, dt = 512, 4000000, 0.001
    w0 = ic.vorticity_ic(n, seed=0, k0=4.0).astype(np.complex64)
    pos = ic.tracer_ic(ntr, seed=1)
    ve = vorticity_equation(n, precision="single")
    for obj in (ve,):
        obj.nu, obj.forcing_type, obj.famplitude, obj.fk0, obj.fk1 = 0.002, "linear", 0.5, 1.5, 3.0
    ve.set_cvorticity(w0)
    ps = particles_system(ve, pos, 3, 2, 3)
    NSVEparticles_step(ve, ps, dt)
    w_gpu = ve.get_cvorticity()
    got, rhs, _ = ps.state()
    ps.close()
    ve.close()
    ref = F.VorticityEquation(n)
    ref.nu, ref.forcing_type, ref.famplitude, ref.fk0, ref.fk1 = 0.002, "linear", 0.5, 1.5, 3.0
    ref.cvorticity = w0.astype(np.complex128)
    del w0
    rps = F.ParticlesSystem(ref, pos, np.zeros((3, ntr, 3)), 3, 2)
    F.nsveparticles_step(ref, rps, dt)
    want, wrhs, _ = rps.state()
    rps.close()
    w_ref = ref.cvorticity
    ref.close()
    assert rel_err(w_gpu, w_ref) < 2e-5
    # rhs[1] holds u(x(t)) after the history shift
    assert rel_err(rhs[1], wrhs[1]) < 1e-5
    assert np.abs(got - want).max() / (2 * np.pi) < 1e-9


@pytest.mark.parametrize("n", [64, 128, 256])
def test_fp32_step_64_to_256_against_fp64_oracle(n):
    """One NSVEparticles step in FP32 at 64^3, 128^3 and 256^3, where the x
    pass is the warp-group kernel (eight, four and two rows per warp), against the FP64
    oracle from the same FP32-rounded field and tracers: the field within
    2e-5 of max|w|, the sampled velocity (read from the real velocity the x
    pass writes in stage 1) within 1e-5 of max|u|, positions within 1e-9 of
    the box (vorticity_equation.cpp:358-439, NSVEparticles.cpp:33-41)."""
    from bfps_b200.solver import vorticity_equation, particles_system, NSVEparticles_step
    ntr, dt = 20000, 0.002
    w0 = ic.vorticity_ic(n, seed=3, k0=4.0).astype(np.complex64)
    pos = ic.tracer_ic(ntr, seed=4)
    ve = vorticity_equation(n, precision="single")
    ve.nu, ve.forcing_type, ve.famplitude, ve.fk0, ve.fk1 = 0.005, "linear", 0.5, 1.5, 3.0
    ve.set_cvorticity(w0)
    ps = particles_system(ve, pos, 3, 2, 3)
    NSVEparticles_step(ve, ps, dt)
    w_gpu = ve.get_cvorticity()
    got, rhs, _ = ps.state()
    ps.close()
    ve.close()
    ref = F.VorticityEquation(n)
    ref.nu, ref.forcing_type, ref.famplitude, ref.fk0, ref.fk1 = 0.005, "linear", 0.5, 1.5, 3.0
    ref.cvorticity = w0.astype(np.complex128)
    rps = F.ParticlesSystem(ref, pos, np.zeros((3, ntr, 3)), 3, 2)
    F.nsveparticles_step(ref, rps, dt)
    want, wrhs, _ = rps.state()
    rps.close()
    w_ref = ref.cvorticity
    ref.close()
    assert rel_err(w_gpu, w_ref) < 2e-5
    assert rel_err(rhs[1], wrhs[1]) < 1e-5
    assert np.abs(got - want).max() / (2 * np.pi) < 1e-9


@pytest.mark.parametrize("n", [64, 128])
def test_fp32_ensemble_equals_alone(n):
    """Two FP32 members of one size in one ensemble (one x-pass launch over
    both, row blocks numbered across members) give bit for bit what each
    gives stepped alone."""
    from bfps_b200.solver import vorticity_equation, particles_system, NSVEparticles_step, ensemble

    def make(seed):
        ve = vorticity_equation(n, precision="single")
        ve.nu, ve.forcing_type, ve.famplitude, ve.fk0, ve.fk1 = 0.01 * seed, "linear", 0.5, 1.5, 3.0
        ve.set_cvorticity(ic.vorticity_ic(n, seed=seed, k0=4.0).astype(np.complex64))
        ps = particles_system(ve, ic.tracer_ic(5000, seed=seed), 2, 1, 3)
        return ve, ps

    mem = [make(1), make(2)]
    alone = [make(1), make(2)]
    ens = ensemble()
    try:
        for ve, ps in mem:
            ens.add(ve, 0.002, ps)
        ens.step(3)
        for ve, ps in alone:
            NSVEparticles_step(ve, ps, 0.002, 3)
        for (a, pa), (b, pb) in zip(mem, alone):
            assert np.array_equal(a.get_cvorticity(), b.get_cvorticity())
            sa, sb = pa.state(), pb.state()
            assert np.array_equal(sa[0], sb[0]) and np.array_equal(sa[1], sb[1])
    finally:
        ens.close()
        for ve, ps in mem + alone:
            ps.close()
            ve.close()
