"""Batched form: an ensemble of mixed-size instances gives, member by member,
exactly the state each member reaches when stepped alone (same kernels, same
per-tile arithmetic), and one member matches the FP64 oracle."""
import numpy as np
import pytest

from oracle import nsve as O
from oracle import particles as P
from oracle.nsveparticles import nsveparticles_step
from bfps_b200 import ic
from gpu_util import rel_err

pytestmark = pytest.mark.gpu

SPECS = [  # (n, nu, seed, tracers, (neighbours, smoothness), AB steps, dt)
    (16, 0.05, 1, 0, None, None, 0.01),
    (32, 0.02, 2, 300, (2, 0), 4, 0.005),
    (16, 0.03, 3, 100, (1, 1), 2, 0.01),
    (64, 0.01, 4, 0, None, None, 0.004),
    (32, 0.04, 5, 0, None, None, 0.008),
]


def _make(spec, precision):
    from bfps_b200.solver import vorticity_equation, particles_system
    n, nu, seed, nt, nm, nab, dt = spec
    ve = vorticity_equation(n, precision=precision)
    ve.nu = nu
    ve.forcing_type = "linear"
    ve.famplitude, ve.fk0, ve.fk1 = 0.5, 1.5, 3.0
    ve.set_cvorticity(ic.vorticity_ic(n, seed=seed, dtype=ve.cdtype))
    ps = particles_system(ve, ic.tracer_ic(nt, seed=seed), nm[0], nm[1], nab) if nt else None
    return ve, ps


@pytest.mark.parametrize("graphs", [True, False])
def test_ensemble_equals_alone(graphs):
    from bfps_b200.solver import ensemble, NSVEparticles_step
    nsteps = 6
    ens = ensemble()
    ens.use_graphs(graphs)
    mixed = [_make(s, "double") for s in SPECS]
    for (ve, ps), s in zip(mixed, SPECS):
        ens.add(ve, s[6], ps)
    ens.step(nsteps)
    for (ve, ps), s in zip(mixed, SPECS):
        ve1, ps1 = _make(s, "double")
        NSVEparticles_step(ve1, ps1, s[6], nsteps)
        assert np.array_equal(ve.get_cvorticity(), ve1.get_cvorticity()), s
        assert ve.iteration == nsteps
        if ps is not None:
            a, b = ps.state(), ps1.state()
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), s
    ens.close()


def test_ensemble_launch_count_same_with_graphs():
    """The launch counter counts the nodes of replayed graphs: the same
    kernels are counted with and without graphs, the same number each step."""
    from bfps_b200.solver import ensemble
    counts = []
    for graphs in (True, False):
        ens = ensemble()
        ens.use_graphs(graphs)
        mixed = [_make(s, "single") for s in SPECS]
        for (ve, ps), s in zip(mixed, SPECS):
            ens.add(ve, s[6], ps)
        ens.step(1)
        one = ens.kernel_launches()
        ens.step(3)
        assert ens.kernel_launches() == 4 * one
        counts.append(one)
        ens.close()
        for ve, ps in mixed:
            if ps is not None:
                ps.close()
            ve.close()
    # three sizes x (5 passes x 3 stages + symmetrize) at least, plus tracers
    assert counts[0] == counts[1] and counts[0] >= 3 * 16


def test_ensemble_wait_polls_with_timeout():
    """bfg_ens_wait: a bounded poll of the last step call, then done."""
    from bfps_b200.solver import ensemble
    ens = ensemble()
    mixed = [_make(s, "single") for s in SPECS]
    for (ve, ps), s in zip(mixed, SPECS):
        ens.add(ve, s[6], ps)
    ens.step(200)
    first = ens.wait(0.0)          # one query, no wait
    assert first in (True, False)
    assert ens.wait(None) is True
    assert ens.wait(0.0) is True
    assert ens.last_ms() > 0
    ens.close()
    for ve, ps in mixed:
        if ps is not None:
            ps.close()
        ve.close()


def test_ensemble_member_matches_oracle():
    from bfps_b200.solver import ensemble
    s = SPECS[1]
    n, nu, seed, nt, nm, nab, dt = s
    ens = ensemble()
    members = [_make(x, "double") for x in SPECS[:3]]
    for (ve, ps), x in zip(members, SPECS[:3]):
        ens.add(ve, x[6], ps)
    ens.step(4)
    ref = O.VorticityEquation(n)
    ref.nu, ref.forcing_type, ref.famplitude, ref.fk0, ref.fk1 = nu, "linear", 0.5, 1.5, 3.0
    ref.cvorticity = ic.vorticity_ic(n, seed=seed)
    rps = P.ParticlesSystem(ic.tracer_ic(nt, seed=seed), np.zeros((nab, nt, 3)), nm[0], nm[1],
                            P.Geometry(n, n, n))
    for _ in range(4):
        nsveparticles_step(ref, rps, dt)
    ve, ps = members[1]
    assert rel_err(ve.get_cvorticity(), ref.cvorticity) < 1e-10
    assert rel_err(ps.state()[0], rps.pos) < 1e-10
    ens.close()


def test_ensemble_membership_changes():
    from bfps_b200.solver import ensemble, NSVEparticles_step
    ens = ensemble()
    a = _make(SPECS[0], "single")
    b = _make(SPECS[3], "single")
    ens.add(a[0], SPECS[0][6], a[1])
    ens.step(2)
    ens.add(b[0], SPECS[3][6], b[1])
    ens.step(2)
    ens.remove(a[0])
    ens.step(1)
    assert a[0].iteration == 4 and b[0].iteration == 3
    b1 = _make(SPECS[3], "single")
    NSVEparticles_step(b1[0], b1[1], SPECS[3][6], 3)
    assert np.array_equal(b[0].get_cvorticity(), b1[0].get_cvorticity())
    ens.close()


def test_serving_results_equal_alone():
    # continuous batching: requests arriving while others run give the same
    # result as the same request solved alone
    from bfps_b200 import serve
    from bfps_b200.solver import NSVEparticles_step, vorticity_equation, particles_system
    reqs = [serve.Request(rid=i, n=n, nu=nu, steps=st, ntracers=nt, arrival=arr, seed=i,
                          precision="double", neighbours=2, smoothness=2, nsteps_ab=4)
            for i, (n, nu, st, nt, arr) in enumerate([(16, 0.02, 7, 50, 0.0), (32, 0.01, 4, 0, 0.0),
                                                      (16, 0.05, 5, 0, 0.05), (32, 0.02, 6, 80, 0.1)])]
    for r in reqs:
        serve.prepare(r)
    srv = serve.Server(hbm_budget=1e9)
    done = srv.run(reqs)
    srv.close()
    assert sorted(r.rid for r in done) == [0, 1, 2, 3]
    for r in done:
        fs = vorticity_equation(r.n, precision="double")
        fs.nu, fs.forcing_type = r.nu, "linear"
        fs.famplitude, fs.fk0, fs.fk1 = r.famplitude, r.fk0, r.fk1
        fs.set_cvorticity(r.w0)
        ps = particles_system(fs, r.pos, 2, 2, 4) if r.ntracers else None
        NSVEparticles_step(fs, ps, r.dt, r.steps)
        assert r.result["iteration"] == r.steps
        assert r.result["vorticity_checksum"] == float(np.abs(fs.get_cvorticity()).sum())
        # statistics too, bit for bit (fixed-order spectrum reduction)
        spec_alone = 0.5 * np.einsum("kii->k", fs.do_stats()["velocity"][0])
        assert np.array_equal(r.result["energy_spectrum"], spec_alone)
        if ps is not None:
            assert np.array_equal(r.result["tracers"], ps.state()[0])
        assert r.finished >= r.admitted >= r.arrival


def test_context_reset_equals_new():
    """bfg_ctx_reset: a context that has run a solve, reset and given a new
    problem, steps bit for bit like a new context (the serving pool reuses
    contexts this way)."""
    from bfps_b200.solver import NSVEparticles_step
    spec = SPECS[1]  # 32^3 with tracers
    used, ps_used = _make(SPECS[4], "single")
    NSVEparticles_step(used, ps_used, SPECS[4][6], 3)
    ps_used.close() if ps_used is not None else None
    used.reset()
    assert used.iteration == 0
    n, nu, seed, nt, nm, nab, dt = spec
    used.nu = nu
    used.set_cvorticity(ic.vorticity_ic(n, seed=seed, dtype=used.cdtype))
    from bfps_b200.solver import particles_system
    ps = particles_system(used, ic.tracer_ic(nt, seed=seed), nm[0], nm[1], nab)
    NSVEparticles_step(used, ps, dt, 4)
    fresh, ps_fresh = _make(spec, "single")
    NSVEparticles_step(fresh, ps_fresh, dt, 4)
    assert np.array_equal(used.get_cvorticity(), fresh.get_cvorticity())
    assert np.array_equal(ps.state()[0], ps_fresh.state()[0])
    for obj in (ps, ps_fresh, used, fresh):
        obj.close()
