"""IF-RK3 vorticity step on the GPU against the FP64 oracle.

Gate: FP64 fields agree with the oracle to 1e-10 relative over the first 8
steps.
"""
import numpy as np
import pytest

from oracle import nsve as O
from bfps_b200 import ic
from gpu_util import rel_err

pytestmark = pytest.mark.gpu


def _pair(n, dealias, forcing, precision="double", seed=0):
    from bfps_b200.solver import vorticity_equation
    ve = vorticity_equation(n, precision=precision, dealias_type=dealias)
    ref = O.VorticityEquation(n, dealias_type=dealias)
    for obj in (ve, ref):
        obj.nu = 0.1
        obj.forcing_type = forcing
        obj.famplitude = 0.5
        obj.fk0 = 1.5
        obj.fk1 = 3.0
        obj.fmode = 2
    w0 = ic.vorticity_ic(n, seed=seed, dealias_type=dealias)
    ve.set_cvorticity(w0)
    ref.cvorticity = w0.astype(np.complex128).copy()
    return ve, ref


@pytest.mark.parametrize("dealias", [O.SMOOTH, O.TWO_THIRDS])
def test_fp64_step_matches_oracle_8_steps(dealias):
    ve, ref = _pair(32, dealias, "linear")
    for s in range(8):
        ve.step(0.01)
        ref.step(0.01)
        err = rel_err(ve.get_cvorticity(), ref.cvorticity)
        assert err < 1e-10, (s, err)
    assert ve.iteration == 8
    ve.close()


@pytest.mark.parametrize("forcing", ["none", "Kolmogorov"])
def test_fp64_forcing_variants(forcing):
    ve, ref = _pair(32, O.SMOOTH, forcing)
    for s in range(2):
        ve.step(0.01)
        ref.step(0.01)
    assert rel_err(ve.get_cvorticity(), ref.cvorticity) < 1e-10
    ve.close()


def test_fp64_n64():
    ve, ref = _pair(64, O.SMOOTH, "linear", seed=3)
    for s in range(2):
        ve.step(0.005)
        ref.step(0.005)
    assert rel_err(ve.get_cvorticity(), ref.cvorticity) < 1e-10
    ve.close()


def test_fp32_step_tracks_fp64_oracle():
    ve, ref = _pair(32, O.SMOOTH, "linear", precision="single")
    for s in range(4):
        ve.step(0.01)
        ref.step(0.01)
    assert rel_err(ve.get_cvorticity(), ref.cvorticity) < 2e-5
    ve.close()


def test_compute_velocity_and_rspace():
    ve, ref = _pair(32, O.SMOOTH, "linear")
    ve.compute_velocity()
    u_ref = ref.compute_velocity(ref.cvorticity)
    assert rel_err(ve.get_cvelocity(), u_ref) < 1e-13
    ve.velocity_rspace()
    r = ve.get_rvelocity()
    r_ref = ref.ift(u_ref)
    assert rel_err(r[:, :, :32], r_ref) < 1e-12
    ve.close()


def test_checkpoint_read_semantics():
    ve, ref = _pair(32, O.SMOOTH, "linear")
    rng = np.random.default_rng(7)
    a = (rng.standard_normal(ve.cshape) + 1j * rng.standard_normal(ve.cshape))
    ve.io_checkpoint_read(a)
    assert rel_err(ve.get_cvorticity(), ref.read_checkpoint_semantics(a)) < 1e-15
    ve.close()


def test_beltrami_decays_exactly():
    # ABC-type Beltrami field: u x w = 0, so with forcing off the IF-RK3 step
    # is w(t) = w(0) exp(-nu k^2 t) (oracle-independent check)
    from bfps_b200.solver import vorticity_equation
    n = 32
    ve = vorticity_equation(n, precision="double")
    ve.nu = 0.05
    ve.forcing_type = "none"
    x = np.arange(n) * 2 * np.pi / n
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    k = 2.0
    u = np.stack([np.sin(k * Z) + np.cos(k * Y), np.sin(k * X) + np.cos(k * Z),
                  np.sin(k * Y) + np.cos(k * X)], axis=-1)
    w_real = k * u  # curl u = k u for this field
    w = O.dft(w_real) / n ** 3
    ve.set_cvorticity(w)
    dt, nsteps = 0.02, 10
    ve.step(dt, nsteps)
    expect = w * np.exp(-ve.nu * k * k * dt * nsteps)
    assert rel_err(ve.get_cvorticity(), expect) < 1e-12
    ve.close()


def test_fp64_anisotropic_box_with_tracers():
    """dkx != dky != dkz (box lengths 2 pi, 4 pi, pi): k-space tables,
    dealiasing radius, forcing band and the tracers' box and cell size all
    follow the per-axis dk (kspace.cpp:34-167, particles_system_builder.hpp:
    176-179)."""
    from bfps_b200.solver import vorticity_equation, particles_system, NSVEparticles_step
    from oracle import particles as P
    from oracle.nsveparticles import nsveparticles_step
    n, dk = 32, (1.0, 0.5, 2.0)
    ve = vorticity_equation(n, n, n, *dk, precision="double")
    ref = O.VorticityEquation(n, n, n, *dk)
    for obj in (ve, ref):
        obj.nu, obj.forcing_type, obj.famplitude, obj.fk0, obj.fk1 = 0.05, "linear", 0.5, 1.5, 3.0
    w0 = ic.vorticity_ic(n, seed=9)
    ve.set_cvorticity(w0)
    ref.cvorticity = w0.copy()
    rng = np.random.default_rng(9)
    pos = rng.random((400, 3)) * np.array([2 * np.pi / d for d in dk]) * 1.5 - 1.0
    ps = particles_system(ve, pos, 2, 1, 3)
    rps = P.ParticlesSystem(pos, np.zeros((3, 400, 3)), 2, 1, P.Geometry(n, n, n, *dk))
    for _ in range(3):
        NSVEparticles_step(ve, ps, 0.005)
        nsveparticles_step(ref, rps, 0.005)
    assert rel_err(ve.get_cvorticity(), ref.cvorticity) < 1e-10
    got, rhs, _ = ps.state()
    assert rel_err(got, rps.pos) < 1e-10
    ps.close()
    ve.close()


def test_fp64_kolmogorov_with_tracers():
    """Kolmogorov forcing (mode fmode = 2) with tracers on the C3
    interpolation kernel (n = 3, m = 2), AB3, three NSVEparticles steps."""
    from bfps_b200.solver import particles_system, NSVEparticles_step
    from oracle import particles as P
    from oracle.nsveparticles import nsveparticles_step
    ve, ref = _pair(32, O.SMOOTH, "Kolmogorov", seed=4)
    pos = ic.tracer_ic(700, seed=44)
    ps = particles_system(ve, pos, 3, 2, 3)
    rps = P.ParticlesSystem(pos, np.zeros((3, 700, 3)), 3, 2, P.Geometry(32, 32, 32))
    for _ in range(3):
        NSVEparticles_step(ve, ps, 0.01)
        nsveparticles_step(ref, rps, 0.01)
    assert rel_err(ve.get_cvorticity(), ref.cvorticity) < 1e-10
    got, rhs, _ = ps.state()
    assert rel_err(got, rps.pos) < 1e-10
    assert rel_err(rhs[1], rps.rhs[1]) < 1e-10
    ps.close()
    ve.close()


def test_fp64_smooth_filter_shared_keys():
    """dky = 1.3: distinct k^2 share a filter key round(k^2 / dk^2), and the
    reference keeps the value written last in CLOOP order
    (kspace.cpp:119-150, applied by kspace.cpp:479); the engine's table and
    the oracle's keyed table give the same step.  With kM set by the y axis
    the kz = N/2 line lies inside kM, where compute_velocity's symmetrize
    (field.cpp:903-978) takes the kx = 0 velocity of rows ky > N/2 from
    their mirror rows."""
    from bfps_b200.solver import vorticity_equation
    n, dk = 32, (1.0, 1.3, 1.0)
    ve = vorticity_equation(n, n, n, *dk, precision="double")
    ref = O.VorticityEquation(n, n, n, *dk)
    for obj in (ve, ref):
        obj.nu, obj.forcing_type, obj.famplitude, obj.fk0, obj.fk1 = 0.05, "linear", 0.5, 1.5, 3.0
    w0 = ref.read_checkpoint_semantics(ic.vorticity_ic(n, seed=17))
    ve.set_cvorticity(w0)
    ref.cvorticity = w0.copy()
    direct = np.exp(-36.0 * np.power(ref.kk.K2 / ref.kk.kM2, 18.0))
    assert np.abs(ref.kk.filter - direct).max() > 1e-6  # keys do collide here
    for _ in range(2):
        ve.step(0.01)
        ref.step(0.01)
    assert rel_err(ve.get_cvorticity(), ref.cvorticity) < 1e-10
    ve.close()
