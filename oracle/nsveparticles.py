"""Oracle: NSVEparticles time loop (TEST INFRASTRUCTURE ONLY).

NSVEparticles::step (bfps/cpp/full_code/NSVEparticles.cpp:33-41):
velocity at time t -> tracers advance with it -> fluid IF-RK3 step.
A restart re-reads the field with io_checkpoint semantics
(vorticity_equation.hpp:107-128) and resumes the tracers at
step_idx = iteration + 1 (NSVEparticles.cpp:23).
"""
import numpy as np

from .nsve import VorticityEquation, SMOOTH
from .particles import ParticlesSystem, Geometry


def nsveparticles_step(ve, ps, dt):
    u = ve.compute_velocity(ve.cvorticity)
    ur = ve.ift(u)
    if ps is not None:
        ps.complete_loop(ur, dt)
    ve.step(dt)


def golden_parameters():
    """Parameters implied by bfps/test/test_bfps_NSVEparticles.py and the
    DNS defaults (bfps/DNS.py:139-166, 513-550, 660-661): N=32, kMeta=2,
    dtfactor=0.5, linear forcing in [2, 4] with amplitude 0.5, beta_n1_m1,
    4 AB steps, 32 steps per job."""
    n = 32
    return dict(n=n, nu=(2.0 * 2 / n) ** (4. / 3), dt=0.5 / n, famplitude=0.5,
                fk0=2.0, fk1=4.0, forcing_type="linear", neighbours=1,
                smoothness=1, nsteps_ab=4, niter_todo=32, njobs=2)


def run_golden(v0, pos0, rdtype=np.float64, record=None):
    """Replay the reference regression from the fixture's iteration-0 field.

    Returns {iteration: (cvorticity, positions, rhs)} at 32 and 64.
    """
    p = golden_parameters()
    n = p["n"]
    ve = VorticityEquation(n, dealias_type=SMOOTH, rdtype=rdtype)
    ve.nu, ve.famplitude, ve.fk0, ve.fk1 = p["nu"], p["famplitude"], p["fk0"], p["fk1"]
    ve.forcing_type = p["forcing_type"]
    ve.cvorticity = ve.read_checkpoint_semantics(v0)
    geom = Geometry(n, n, n)
    rhs = np.zeros((p["nsteps_ab"],) + pos0.shape)
    ps = ParticlesSystem(pos0, rhs, p["neighbours"], p["smoothness"], geom, step_idx=1)
    out = {}
    for job in range(p["njobs"]):
        if job > 0:
            # restart: checkpoint stored in the run precision, re-read
            ve.cvorticity = ve.read_checkpoint_semantics(ve.cvorticity)
            ps.step_idx = ve.iteration + 1
        for _ in range(p["niter_todo"]):
            nsveparticles_step(ve, ps, p["dt"])
            if record is not None:
                record(ve, ps)
        out[ve.iteration] = (ve.cvorticity.copy(), ps.pos.copy(), ps.rhs.copy())
    return out
