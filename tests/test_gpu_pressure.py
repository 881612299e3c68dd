"""Pressure and Lagrangian acceleration on the GPU against the oracle
(vorticity_equation.cpp:441-578) and against the Taylor-Green exact solution;
the acceleration sampled at the tracers as NSVEparticles::do_stats does
(NSVEparticles.cpp:84-91)."""
import numpy as np
import pytest

from oracle import nsve as O
from oracle import particles as P
from bfps_b200 import _lib, ic
from gpu_util import rel_err

pytestmark = pytest.mark.gpu


def _pair(n, dealias, precision="double"):
    from bfps_b200.solver import vorticity_equation
    ve = vorticity_equation(n, precision=precision, dealias_type=dealias)
    ref = O.VorticityEquation(n, dealias_type=dealias,
                              rdtype=np.float32 if precision == "single" else np.float64)
    for obj in (ve, ref):
        obj.nu = 0.03
        obj.forcing_type = "linear"
        obj.famplitude, obj.fk0, obj.fk1 = 0.5, 1.5, 3.0
    w0 = ic.vorticity_ic(n, seed=7, dealias_type=dealias,
                         dtype=np.complex64 if precision == "single" else np.complex128)
    ve.set_cvorticity(w0)
    ref.cvorticity = w0.copy()
    return ve, ref


@pytest.mark.parametrize("dealias", [_lib.SMOOTH, _lib.TWO_THIRDS])
def test_pressure_and_acceleration_match_oracle(dealias):
    n = 32
    ve, ref = _pair(n, dealias)
    p = ve.compute_pressure()
    want_p = ref.compute_pressure(ref.ift(ref.compute_velocity(ref.cvorticity)))
    assert rel_err(p, want_p) < 1e-10
    a = ve.compute_Lagrangian_acceleration()
    want_a = ref.compute_lagrangian_acceleration()
    assert rel_err(a, want_a) < 1e-10
    ve.close()


def test_acceleration_sampled_at_tracers():
    from bfps_b200.solver import particles_system
    n = 32
    ve, ref = _pair(n, _lib.SMOOTH)
    pos = ic.tracer_ic(500, seed=8)
    ps = particles_system(ve, pos, 3, 2, nsteps=2)
    got = ps.sample_acceleration()
    ar = ref.ift(ref.compute_lagrangian_acceleration())
    want = P.sample(ar, pos, 3, 2, P.Geometry(n, n, n))
    assert rel_err(got, want) < 1e-10
    # the velocity field the tracers advect with is left as it was
    ve.velocity_rspace()
    ur = ref.ift(ref.compute_velocity(ref.cvorticity))
    assert rel_err(ps.sample_velocity(), P.sample(ur, pos, 3, 2, P.Geometry(n, n, n))) < 1e-10
    ps.close()
    ve.close()


def test_acceleration_fp32_against_fp64_oracle():
    n = 32
    ve, _ = _pair(n, _lib.SMOOTH, precision="single")
    _, ref = _pair(n, _lib.SMOOTH)
    a = ve.compute_Lagrangian_acceleration()
    assert rel_err(a, ref.compute_lagrangian_acceleration()) < 2e-5
    ve.close()


def test_taylor_green_acceleration_is_minus_grad_p():
    # steady Euler flow u = (sin x cos y, -cos x sin y, 0): p = (cos 2x + cos 2y)/4
    from bfps_b200.solver import vorticity_equation
    n = 32
    ve = vorticity_equation(n, precision="double")
    ve.nu = 0.0
    ref = O.VorticityEquation(n)
    x = 2 * np.pi * np.arange(n) / n
    z, y, xx = np.meshgrid(x, x, x, indexing="ij")
    u = np.zeros((n, n, n, 3))
    u[..., 0] = np.sin(xx) * np.cos(y)
    u[..., 1] = -np.cos(xx) * np.sin(y)
    ve.set_cvorticity(ref.compute_vorticity(ref.dft(u) / n ** 3))
    p = ref.ift(ve.compute_pressure()[..., None])[..., 0]
    assert np.abs(p - (np.cos(2 * xx) + np.cos(2 * y)) / 4).max() < 1e-12
    a = ref.ift(ve.compute_Lagrangian_acceleration())
    assert np.abs(a[..., 0] - np.sin(2 * xx) / 2).max() < 1e-12
    assert np.abs(a[..., 1] - np.sin(2 * y) / 2).max() < 1e-12
    assert np.abs(a[..., 2]).max() < 1e-12
    ve.close()
