"""Autotuner of the column passes (bfg_autotune / bfg_ens_autotune /
bfg_tune_get / bfg_tune_set): both schedules give the oracle's step, the
tuner records its measurements and choices per members-per-launch, appends
them to the cache file, and an ensemble tuned and switched to the other
schedule still equals its members stepped alone under that schedule."""
import os

import numpy as np
import pytest

from oracle import nsve as O
from oracle import particles as P
from oracle.nsveparticles import nsveparticles_step
from bfps_b200 import ic
from gpu_util import rel_err

pytestmark = pytest.mark.gpu
PASSES = ("IZ", "IY", "FY", "FZ")


@pytest.mark.parametrize("schedule", [0, 1])
def test_both_schedules_match_the_oracle(schedule):
    from bfps_b200.solver import vorticity_equation, particles_system, NSVEparticles_step
    n, nt = 32, 300
    ve = vorticity_equation(n, precision="double")
    try:
        for p in PASSES:
            ve.set_schedule(p, schedule)
        assert all(v[0] == schedule for v in ve.schedules().values())
        ref = O.VorticityEquation(n)
        for obj in (ve, ref):
            obj.nu, obj.forcing_type, obj.famplitude, obj.fk0, obj.fk1 = 0.05, "linear", 0.5, 1.5, 3.0
        w0 = ic.vorticity_ic(n, seed=41)
        ve.set_cvorticity(w0)
        ref.cvorticity = w0.copy()
        pos = ic.tracer_ic(nt, seed=42)
        ps = particles_system(ve, pos, 3, 2, 3)
        rps = P.ParticlesSystem(pos, np.zeros((3, nt, 3)), 3, 2, P.Geometry(n, n, n))
        for _ in range(3):
            NSVEparticles_step(ve, ps, 0.01)
            nsveparticles_step(ref, rps, 0.01)
        assert rel_err(ve.get_cvorticity(), ref.cvorticity) < 1e-10
        assert rel_err(ps.state()[0], rps.pos) < 1e-10
        ps.close()
    finally:
        for p in PASSES:
            ve.set_schedule(p, 0)
        ve.close()


def test_autotune_records_and_caches(tmp_path, monkeypatch):
    from bfps_b200.solver import vorticity_equation
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("BFPS_B200_TUNE_CACHE", str(cache))
    ve = vorticity_equation(64, precision="single")
    try:
        ve.set_cvorticity(ic.vorticity_ic(64, seed=43, dtype=np.complex64))
        got = ve.autotune(reps=2)
        for p in PASSES:
            sched, ms0, ms1 = got[p]
            assert ms0 > 0 and ms1 > 0
            assert sched == (1 if ms1 < ms0 * (1.0 - 0.02) else 0)
        lines = cache.read_text().split("\n")
        rows = [l.split() for l in lines if l.strip()]
        assert len(rows) == 4
        for r in rows:
            assert int(r[1]) == 64 and int(r[2]) == 4 and int(r[3]) in (0, 1, 3, 4)
            assert int(r[4]) == 1 and int(r[5]) in (0, 1)
            assert float(r[6]) > 0 and float(r[7]) > 0
        # a launch over several members is a different key, still untuned
        assert all(v == (0, 0.0, 0.0) for v in ve.schedules(members=3).values())
        # the state is untouched by the tuning launches
        w = ve.get_cvorticity()
        assert np.array_equal(w, ic.vorticity_ic(64, seed=43, dtype=np.complex64))
    finally:
        for p in PASSES:
            ve.set_schedule(p, 0)
        ve.close()


ENS = [  # (n, nu, seed, tracers, dt)
    (32, 0.02, 51, 200, 0.005),
    (16, 0.05, 52, 0, 0.01),
    (32, 0.04, 53, 0, 0.008),
    (32, 0.03, 54, 0, 0.006),
    (16, 0.03, 55, 100, 0.01),
]


def _member(spec):
    from bfps_b200.solver import vorticity_equation, particles_system
    n, nu, seed, nt, dt = spec
    ve = vorticity_equation(n, precision="double")
    ve.nu, ve.forcing_type, ve.famplitude, ve.fk0, ve.fk1 = nu, "linear", 0.5, 1.5, 3.0
    ve.set_cvorticity(ic.vorticity_ic(n, seed=seed))
    ps = particles_system(ve, ic.tracer_ic(nt, seed=seed), 2, 1, 3) if nt else None
    return ve, ps


@pytest.mark.parametrize("graphs", [True, False])
def test_ensemble_autotune_then_other_schedule_equals_alone(graphs):
    from bfps_b200.solver import ensemble, NSVEparticles_step
    counts = {16: 2, 32: 3}
    ens = ensemble()
    ens.use_graphs(graphs)
    mem = [_member(s) for s in ENS]
    alone = [_member(s) for s in ENS]
    try:
        for (ve, ps), s in zip(mem, ENS):
            ens.add(ve, s[4], ps)
        ens.step(1)
        tuned = ens.autotune(reps=2)
        assert set(tuned) == set(counts)
        for n, t in tuned.items():
            for p in PASSES:
                sched, ms0, ms1 = t[p]
                # two size groups: schedule 1 must win by 10 %
                assert ms0 > 0 and ms1 > 0 and sched == (1 if ms1 < ms0 * (1.0 - 0.10) else 0)
        # the group launches (3 x 32^3, 2 x 16^3) switched to schedule 1; the
        # graphs are re-captured at the next step
        for n, k in counts.items():
            ve = next(v for v, _ in mem if v.nx == n)
            for p in PASSES:
                ve.set_schedule(p, 1, members=k)
        ens.step(3)
        for (ve, ps), s in zip(alone, ENS):
            NSVEparticles_step(ve, ps, s[4], 1)
            for p in PASSES:
                ve.set_schedule(p, 1)
            NSVEparticles_step(ve, ps, s[4], 3)
            for p in PASSES:
                ve.set_schedule(p, 0)
        for (ve, ps), (ve1, ps1), s in zip(mem, alone, ENS):
            assert np.array_equal(ve.get_cvorticity(), ve1.get_cvorticity()), s
            if ps is not None:
                a, b = ps.state(), ps1.state()
                assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), s
    finally:
        ens.close()
        for n, k in counts.items():
            ve = next(v for v, _ in mem if v.nx == n)
            for p in PASSES:
                ve.set_schedule(p, 0, members=k)
                ve.set_schedule(p, 0)
        for ve, ps in mem + alone:
            if ps is not None:
                ps.close()
            ve.close()
