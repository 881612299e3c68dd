"""Tracer gather + Adams-Bashforth on the GPU against the oracle."""
import numpy as np
import pytest

from oracle import nsve as O
from oracle import particles as P
from oracle.nsveparticles import nsveparticles_step
from bfps_b200 import ic
from gpu_util import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nm", [(1, 0), (1, 1), (2, 0), (2, 2), (3, 2), (4, 1), (5, 2)])
def test_sample_matches_oracle(nm):
    from bfps_b200.solver import vorticity_equation, particles_system
    n = 32
    nb, mm = nm
    ve = vorticity_equation(n, precision="double")
    w0 = ic.vorticity_ic(n, seed=1)
    ve.set_cvorticity(w0)
    ve.velocity_rspace()
    ref = O.VorticityEquation(n)
    ur = ref.ift(ref.compute_velocity(w0))
    pos = ic.tracer_ic(777, seed=4)
    pos[:5] = [[0, 0, 0], [2 * np.pi - 1e-12, 0.1, 6.2], [-0.3, 7.0, 13.1], [3.0, 3.0, 3.0], [1e-9, 2.0, -1e-9]]
    ps = particles_system(ve, pos, nb, mm, nsteps=2)
    got = ps.sample_velocity()
    want = P.sample(ur, pos, nb, mm, P.Geometry(n, n, n))
    assert rel_err(got, want) < 1e-12
    ps.close()
    ve.close()


@pytest.mark.parametrize("nm,nsteps", [((2, 0), 2), ((2, 2), 4), ((3, 2), 3), ((1, 1), 6)])
def test_nsveparticles_steps_match_oracle(nm, nsteps):
    from bfps_b200.solver import vorticity_equation, particles_system, NSVEparticles_step
    n = 32
    ve = vorticity_equation(n, precision="double")
    ref = O.VorticityEquation(n)
    for obj in (ve, ref):
        obj.nu = 0.1
        obj.forcing_type = "linear"
        obj.famplitude = 0.5
        obj.fk0 = 1.5
        obj.fk1 = 3.0
    w0 = ic.vorticity_ic(n, seed=0)
    ve.set_cvorticity(w0)
    ref.cvorticity = w0.copy()
    pos = ic.tracer_ic(1024, seed=0)
    ps = particles_system(ve, pos, nm[0], nm[1], nsteps)
    rps = P.ParticlesSystem(pos, np.zeros((nsteps, 1024, 3)), nm[0], nm[1], P.Geometry(n, n, n))
    for s in range(8):
        NSVEparticles_step(ve, ps, 0.01)
        nsveparticles_step(ref, rps, 0.01)
    p, r, idx = ps.state()
    assert np.array_equal(idx, np.arange(1024))
    assert rel_err(p, rps.pos) < 1e-10
    assert rel_err(r, rps.rhs) < 1e-10
    assert np.all(r[0] == 0)
    assert ps.step_idx == 9
    assert rel_err(ve.get_cvorticity(), ref.cvorticity) < 1e-10
    ps.close()
    ve.close()


def test_arbitrary_global_indices_come_back_sorted():
    # tracers given out of index order (as after an MPI redistribute) are
    # written back in global index order (particles_output_hdf5.hpp)
    from bfps_b200.solver import vorticity_equation, particles_system
    n = 32
    ve = vorticity_equation(n, precision="double")
    w0 = ic.vorticity_ic(n, seed=2)
    ve.set_cvorticity(w0)
    ve.velocity_rspace()
    ref = O.VorticityEquation(n)
    ur = ref.ift(ref.compute_velocity(w0))
    rng = np.random.default_rng(3)
    pos = ic.tracer_ic(500, seed=9)
    perm = rng.permutation(500)
    gidx = 1000 + perm * 7  # any distinct global indices
    ps = particles_system(ve, pos, 2, 1, nsteps=3, idx=gidx)
    got = ps.sample_velocity()
    want = P.sample(ur, pos, 2, 1, P.Geometry(n, n, n))
    order = np.argsort(gidx)
    assert rel_err(got, want[order]) < 1e-12
    for _ in range(5):
        ps.completeLoop(0.01)
    p, r, idx = ps.state()
    assert np.array_equal(idx, np.sort(gidx))
    rps = P.ParticlesSystem(pos, np.zeros((3, 500, 3)), 2, 1, P.Geometry(n, n, n))
    for _ in range(5):
        rps.complete_loop(ur, 0.01)
    assert rel_err(p, rps.pos[order]) < 1e-12
    assert rel_err(r, rps.rhs[:, order]) < 1e-12
    ps.close()
    ve.close()


@pytest.mark.parametrize("n,nm", [(32, (1, 1)), (32, (3, 2)), (64, (2, 0)), (64, (5, 2))])
def test_fp32_field_sample_error_bound(n, nm):
    # Precision form: with an FP32 field the x sums of each stencil row run in
    # FP32 (weights rounded to FP32), the rest in FP64.  Against the FP64
    # oracle sampling of the same FP32 field the error stays below 2e-6 of
    # max|u| (FP32 rounding of 2n+2 weights and partial sums).
    from bfps_b200.solver import vorticity_equation, particles_system
    nb, mm = nm
    ve = vorticity_equation(n, precision="single")
    ve.set_cvorticity(ic.vorticity_ic(n, seed=5, dtype=np.complex64))
    ve.velocity_rspace()
    field = ve.get_rvelocity()[:, :, :n, :].astype(np.float64)
    pos = ic.tracer_ic(3000, seed=6)
    pos[:4] = [[0, 0, 0], [2 * np.pi - 1e-9, 0.2, 6.0], [-0.3, 7.0, 13.1], [6.27, 3.0, 0.01]]
    ps = particles_system(ve, pos, nb, mm, nsteps=2)
    got = ps.sample_velocity()
    want = P.sample(field, pos, nb, mm, P.Geometry(n, n, n))
    err = np.abs(got - want).max() / np.abs(field).max()
    assert err < 2e-6, err
    ps.close()
    ve.close()


def test_zero_tracers():
    """An empty tracer system: the step is the fluid step alone, the state
    arrays are empty, sampling returns nothing."""
    from bfps_b200.solver import vorticity_equation, particles_system, NSVEparticles_step
    n = 32
    w0 = ic.vorticity_ic(n, seed=21)
    out = []
    for with_ps in (True, False):
        ve = vorticity_equation(n, precision="double")
        ve.nu, ve.forcing_type = 0.05, "linear"
        ve.set_cvorticity(w0)
        ps = particles_system(ve, np.zeros((0, 3)), 2, 1, 3) if with_ps else None
        NSVEparticles_step(ve, ps, 0.01, 3)
        out.append(ve.get_cvorticity())
        if ps is not None:
            pos, rhs, idx = ps.state()
            assert pos.shape == (0, 3) and rhs.shape == (3, 0, 3) and idx.shape == (0,)
            assert ps.sample_velocity().shape == (0, 3)
            assert ps.step_idx == 4
            ps.close()
        ve.close()
    assert np.array_equal(out[0], out[1])


def test_cell_sort_over_many_bucket_blocks():
    """64^3: 4096 (z, y) buckets, scanned in four 1024-bucket blocks; the
    sorted tracers come back in index order unchanged and step as the
    oracle's."""
    from bfps_b200.solver import vorticity_equation, particles_system, NSVEparticles_step
    n = 64
    ve = vorticity_equation(n, precision="double")
    ref = O.VorticityEquation(n)
    for obj in (ve, ref):
        obj.nu, obj.forcing_type, obj.famplitude, obj.fk0, obj.fk1 = 0.02, "linear", 0.5, 1.5, 3.0
    w0 = ic.vorticity_ic(n, seed=31)
    ve.set_cvorticity(w0)
    ref.cvorticity = w0.copy()
    pos = ic.tracer_ic(5000, seed=32)
    ps = particles_system(ve, pos, 2, 1, 3)
    p0, r0, i0 = ps.state()
    assert np.array_equal(p0, pos) and np.array_equal(i0, np.arange(5000)) and not r0.any()
    rps = P.ParticlesSystem(pos, np.zeros((3, 5000, 3)), 2, 1, P.Geometry(n, n, n))
    for _ in range(2):
        NSVEparticles_step(ve, ps, 0.004)
        nsveparticles_step(ref, rps, 0.004)
    got, _, _ = ps.state()
    assert rel_err(got, rps.pos) < 1e-10
    ps.close()
    ve.close()
