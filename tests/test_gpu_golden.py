"""The reference's own regression, replayed on the GPU.

bfps/test/test_bfps_NSVEparticles.py: N=32, single precision, 2 jobs of 32
steps, 10^4 tracers with beta_n1_m1 and AB4, compared to the fixture at
iterations 32 and 64 with max|diff| < 1e-5.  The restart between the jobs
re-reads the field with io_checkpoint semantics.
"""
import numpy as np
import pytest

from oracle.nsveparticles import golden_parameters

pytestmark = pytest.mark.gpu


def test_golden_replay_fp32(golden, golden_ic_positions):
    from bfps_b200.solver import vorticity_equation, particles_system, NSVEparticles_step
    p = golden_parameters()
    ve = vorticity_equation(p["n"], precision="single")
    ve.nu, ve.famplitude, ve.fk0, ve.fk1 = p["nu"], p["famplitude"], p["fk0"], p["fk1"]
    ve.forcing_type = p["forcing_type"]
    ve.io_checkpoint_read(golden["vorticity_0"])
    ps = particles_system(ve, golden_ic_positions, p["neighbours"], p["smoothness"], p["nsteps_ab"])
    nkeep = golden["state_32"].shape[0]
    for job in range(p["njobs"]):
        if job > 0:
            ve.io_checkpoint_read(ve.get_cvorticity())
        NSVEparticles_step(ve, ps, p["dt"], p["niter_todo"])
        it = ve.iteration
        v = ve.get_cvorticity()
        pos, rhs, _ = ps.state()
        assert np.abs(v - golden["vorticity_%d" % it]).max() < 1e-5
        assert np.abs(pos[:nkeep] - golden["state_%d" % it]).max() < 1e-5
        assert np.abs(rhs[:, :nkeep] - golden["rhs_%d" % it]).max() < 1e-5
    assert ve.iteration == 64
    ps.close()
    ve.close()
