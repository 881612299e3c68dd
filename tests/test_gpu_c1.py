"""The plain FP64 drop-in configuration (32^3 FP64, nu = 0.1, dt = 0.01,
linear forcing on 1.5 <= |k| <= 3, 2/3 dealiasing, 1024 tracers with the
6-point Lagrange kernel and AB2, 16 NSVEparticles steps) against the oracle:
energy spectra and tracer positions to 1e-10 relative over steps 1-8, then
the spectrum averaged over steps 9-16."""
import numpy as np
import pytest

from oracle import nsve as O
from oracle import particles as P
from oracle.nsveparticles import nsveparticles_step
from bfps_b200 import _lib, ic
from gpu_util import rel_err

pytestmark = pytest.mark.gpu


def test_c1_configuration_matches_oracle():
    from bfps_b200.solver import vorticity_equation, particles_system, NSVEparticles_step
    n, nu, dt, ntr = 32, 0.1, 0.01, 1024
    ve = vorticity_equation(n, precision="double", dealias_type=_lib.TWO_THIRDS)
    ref = O.VorticityEquation(n, dealias_type=O.TWO_THIRDS)
    for obj in (ve, ref):
        obj.nu = nu
        obj.forcing_type = "linear"
        obj.famplitude, obj.fk0, obj.fk1 = 0.5, 1.5, 3.0
    w0 = ic.vorticity_ic(n, seed=0, k0=3.0, dealias_type=_lib.TWO_THIRDS)
    ve.set_cvorticity(w0)
    ref.cvorticity = w0.copy()
    pos = ic.tracer_ic(ntr, seed=0)
    ps = particles_system(ve, pos, 2, 0, 2)
    rps = P.ParticlesSystem(pos, np.zeros((2, ntr, 3)), 2, 0, P.Geometry(n, n, n))
    avg_got, avg_want = 0.0, 0.0
    for step in range(1, 17):
        NSVEparticles_step(ve, ps, dt)
        nsveparticles_step(ref, rps, dt)
        got = ve.do_stats(1.0, 1.0, 8)["velocity"][0]
        want = O.nsve_do_stats(ref, 1.0, 1.0, 8)["velocity"][0]
        if step <= 8:
            assert rel_err(got, want) < 1e-10, step
            assert rel_err(ps.state()[0], rps.pos) < 1e-10, step
        else:
            avg_got = avg_got + got / 8
            avg_want = avg_want + want / 8
    assert rel_err(avg_got, avg_want) < 1e-9
    assert rel_err(ps.state()[0], rps.pos) < 1e-9
    assert ve.iteration == 16
    ps.close()
    ve.close()
