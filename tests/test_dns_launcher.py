"""The launcher (bfps_b200.dns, the counterpart of bfps.DNS) on the CPU:
launch arguments and derived parameters, the files written before the run
(parameters, statistics datasets, initial conditions), the reference's
initial-field generator and the checkpoint-file counter."""
import os

import numpy as np
import pytest

from bfps_b200 import dns, h5
from oracle.nsveparticles import golden_parameters

# bfps/test/test_bfps_NSVEparticles.py:16-34
REF_ARGS = ["NSVEparticles", "-n", "32", "--src-simname", "B32p1e4", "--src-iteration", "0",
            "--simname", "dns_nsveparticles", "--np", "4", "--ntpp", "1", "--niter_todo", "32",
            "--niter_out", "32", "--niter_stat", "1", "--checkpoints_per_file", "3",
            "--nparticles", "10000", "--particle-rand-seed", "2", "--njobs", "2"]


class NoRun(dns.DNS):
    def run(self, **kw):
        self.ran = kw


def _source(tmp_path, golden):
    src = tmp_path / "src"
    src.mkdir()
    with h5.File(str(src / "B32p1e4_checkpoint_0.h5"), "w") as f:
        f["vorticity/complex/0"] = golden["vorticity_0"]
    return str(src)


def test_reference_arguments_give_the_regression_parameters(tmp_path):
    c = NoRun()
    opt = c.prepare_launch(REF_ARGS + ["--src-wd", str(tmp_path), "--wd", str(tmp_path)])
    g = golden_parameters()
    p = c.parameters
    assert c.dns_type == "NSVEparticles" and c.fluid_precision == "single"
    assert (p["nx"], p["ny"], p["nz"]) == (32, 32, 32)
    assert p["nu"] == pytest.approx(g["nu"], rel=1e-15) and p["dt"] == g["dt"]
    assert (p["famplitude"], p["fk0"], p["fk1"], p["forcing_type"]) == (g["famplitude"], g["fk0"], g["fk1"], g["forcing_type"])
    assert (p["tracers0_neighbours"], p["tracers0_smoothness"], p["tracers0_integration_steps"]) == (g["neighbours"], g["smoothness"], g["nsteps_ab"])
    assert (p["niter_todo"], p["niter_out"], p["niter_stat"], p["niter_part"]) == (32, 32, 1, 1)
    assert (p["checkpoints_per_file"], p["nparticles"], p["dealias_type"]) == (3, 10000, 1)
    assert (p["dkx"], p["dky"], p["dkz"]) == (1.0, 1.0, 1.0)
    assert opt.njobs == 2 and opt.nb_processes == 4


def test_default_checkpoints_per_file_and_niter_out(tmp_path):
    c = NoRun()
    c.prepare_launch(["NSVE", "-n", "64", "--niter_todo", "12", "--niter_out", "4"])
    # checkpoint files of about 1 GB when not given
    assert c.parameters["checkpoints_per_file"] == int(1e9 / (3 * 66 * 64 * 64 * 4))
    assert (c.parameters["niter_todo"], c.parameters["niter_out"]) == (12, 4)
    # the niter_out fallback of prepare_launch looks at the defaults, before
    # the arguments are merged (DNS.py:664-665), so a command-line niter_out
    # that does not divide niter_todo reaches write_par's check
    c = NoRun()
    c.prepare_launch(["NSVE", "-n", "32", "--niter_todo", "12", "--niter_out", "5",
                      "--wd", str(tmp_path)])
    assert c.parameters["niter_out"] == 5
    with pytest.raises(AssertionError):
        c.write_par()
    c = NoRun()
    c.prepare_launch(["NSVE", "-n", "288"])
    assert c.parameters["famplitude"] == 0.45


def test_files_before_the_run(tmp_path, golden):
    src = _source(tmp_path, golden)
    wd = str(tmp_path / "run")
    c = NoRun()
    c.launch(REF_ARGS + ["--src-wd", src, "--wd", wd])
    assert c.ran["njobs"] == 2
    with h5.File(c.get_data_file_name()) as f:
        assert f["iteration"][()] == 0 and f["checkpoint"][()] == 0
        assert f["parameters/forcing_type"][()] == b"linear"
        assert f["parameters/nparticles"][()] == 10000
        assert f["bfps_info/exec_name"][()] == b"NSVEparticles-single-vb200"
        ns = f["kspace/nshell"].shape[0]
        assert ns == int(15 / 1.0) + 2 and f["kspace/kM"][()] == 15.0
        sp = f["statistics/spectra/velocity_velocity"]
        assert sp.shape == (1, ns, 3, 3) and sp.maxshape == (None, ns, 3, 3)
        assert sp.chunks == (2 ** 20 // (8 * 9 * ns), ns, 3, 3)
        assert f["statistics/moments/vorticity"].shape == (1, 10, 4)
        hist = f["statistics/histograms/velocity"]
        assert hist.shape == (1, 256, 4) and hist.dtype == np.int64
    with h5.File(c.get_checkpoint_0_fname()) as f:
        assert np.array_equal(f["vorticity/complex/0"][()], golden["vorticity_0"])
        np.random.seed(2)
        assert np.array_equal(f["tracers0/state/0"][()], np.random.random((10000, 3)) * 2 * np.pi)
        assert f["tracers0/rhs/0"].shape == (4, 10000, 3) and not f["tracers0/rhs/0"][()].any()
    with h5.File(c.get_particle_file_name()) as f:
        assert f["tracers0"].keys() == ["acceleration", "velocity"]
    with pytest.raises(FileExistsError):
        c.write_par()


def test_generated_initial_field():
    """generate_vector_field (DNS.py:734-806): Hermitian on kx = 0, modes
    beyond N/3 of the half grid zero, padded into the full grid."""
    c = NoRun()
    c.prepare_launch(["NSVE", "-n", "32"])
    a = c.generate_vector_field(spectra_slope=2.0, amplitude=0.05)
    assert a.shape == (32, 32, 17, 3) and a.dtype == np.complex64
    plane = a[:, :, 0]
    herm = np.conj(plane[(-np.arange(32)) % 32][:, (-np.arange(32)) % 32])
    assert np.abs(plane - herm).max() == 0
    assert a[0, 0, 0].tolist() == [0, 0, 0]
    assert not a[8:25].any() and not a[:, 8:25].any() and not a[:, :, 9:].any()
    b = c.generate_vector_field(spectra_slope=2.0, amplitude=0.05)
    assert np.array_equal(a, b)   # seeded (rseed 7547)


def test_checkpoint_counter(tmp_path):
    """update_checkpoint: a file takes checkpoints_per_file fields, then the
    next one opens (vorticity_equation.cpp:49-108)."""
    c = NoRun(work_dir=str(tmp_path), simname="s")
    job = dns._Job.__new__(dns._Job)
    job.dns, job.checkpoint, job.p = c, 0, {"checkpoints_per_file": 2}
    for it in (0, 8, 16, 24, 32):
        job.iteration = it
        job._update_checkpoint()
        with h5.File(job._fname(), "a") as f:
            f["vorticity/complex/%d" % it] = np.zeros(2)
    assert job.checkpoint == 2
    with h5.File(c.get_checkpoint_fname(1)) as f:
        assert f["vorticity/complex"].keys() == ["16", "24"]
    job.iteration = 32
    job._update_checkpoint()   # the field exists already: same file
    assert job.checkpoint == 2


class _FakeField:
    """Stand-in for solver.vorticity_equation: no physics, the iteration
    advances and the field is scaled, so the file flow can be checked on
    the CPU."""

    def __init__(self, nx, ny, nz, dkx, dky, dkz, precision, dealias_type, device):
        self.n, self.iteration, self.w = nx, 0, None
        self.cdtype = np.complex64 if precision == "single" else np.complex128

    def io_checkpoint_read(self, a):
        assert isinstance(self.forcing_type, str) and isinstance(self.nu, float)
        self.w = np.array(a, dtype=self.cdtype)

    def kspace(self):
        ns = int(self.n // 2 - 1) + 2
        return dict(kM=float(self.n // 2 - 1), dk=1.0, nshells=ns, kshell=np.arange(ns, dtype=float),
                    nshell=np.arange(ns, dtype=np.int64))

    def get_cvorticity(self):
        return self.w.copy()

    def count_nonfinite(self, field="vorticity"):
        return int((~np.isfinite(self.w.real)).sum() + (~np.isfinite(self.w.imag)).sum())

    def step(self, dt, n=1):
        self.iteration += n
        self.w *= 1.0

    def velocity_rspace(self):
        pass

    def do_stats(self, mv, mw, nbins):
        ns = self.kspace()["nshells"]
        t = float(self.iteration)
        return {k: (np.full((ns, 3, 3), t), np.full((10, 4), t), np.full((nbins, 4), self.iteration, np.int64))
                for k in ("velocity", "vorticity")}

    def close(self):
        pass


class _FakeTracers:
    def __init__(self, fs, pos, nb, mm, nsteps, rhs=None, step_idx=1):
        self.fs, self.pos, self.rhs, self.step_idx = fs, pos.copy(), rhs.copy(), step_idx

    def sample_velocity(self):
        return np.full(self.pos.shape, float(self.step_idx))

    def sample_acceleration(self):
        return -self.sample_velocity()

    def state(self):
        return self.pos.copy(), self.rhs.copy(), np.arange(len(self.pos))

    def close(self):
        pass


def _fake_step(fs, ps, dt, n=1):
    ps.pos += dt
    ps.step_idx += n
    fs.step(dt, n)


def test_job_flow_with_a_stand_in_engine(tmp_path, golden, monkeypatch):
    """main_loop / do_stats / write_checkpoint over two jobs, the engine
    replaced by a stand-in: iterations, statistics rows, checkpoint files,
    sampled datasets and the restart between jobs."""
    from bfps_b200 import solver
    monkeypatch.setattr(solver, "vorticity_equation", _FakeField)
    monkeypatch.setattr(solver, "particles_system", _FakeTracers)
    monkeypatch.setattr(solver, "NSVEparticles_step", _fake_step)
    src = _source(tmp_path, golden)
    c = dns.DNS()
    args = [a for a in REF_ARGS]
    args[args.index("--checkpoints_per_file") + 1] = "2"
    args[args.index("--niter_todo") + 1] = "8"
    args[args.index("--niter_out") + 1] = "4"
    args[args.index("--nparticles") + 1] = "50"
    c.launch(args + ["--niter_stat", "2", "--src-wd", src, "--wd", str(tmp_path / "run")])
    with h5.File(c.get_data_file_name()) as f:
        assert f["iteration"][()] == 16 and f["checkpoint"][()] == 2
        mom = f["statistics/moments/velocity"][()]
        assert mom.shape == (1 + 2 * 4, 10, 4)
        assert np.array_equal(mom[:, 0, 0], 2.0 * np.arange(9))   # row t holds iteration 2 t
        assert np.array_equal(f["statistics/histograms/vorticity"][()][:, 0, 0], 2 * np.arange(9))
        assert f["kspace/nshell"][()].tolist() == list(range(17))
    # checkpoints every 4 iterations, 2 per file: 0, 4 | 8, 12 | 16
    for cp, its in ((0, ["0", "4"]), (1, ["12", "8"]), (2, ["16"])):
        with h5.File(c.get_checkpoint_fname(cp)) as f:
            assert f["vorticity/complex"].keys() == its
            for it in its:
                if it != "0":
                    pos = f["tracers0/state/" + it][()]
                    assert f["tracers0/rhs/" + it].shape == (4, 50, 3)
                    np.random.seed(2)
                    p0 = np.random.random((50, 3)) * 2 * np.pi
                    assert np.allclose(pos - p0, int(it) * c.parameters["dt"])
    with h5.File(c.get_particle_file_name()) as f:
        # sampled at every step's statistics, named by step_idx; the restart
        # finds step 9 written already
        assert sorted(int(k) for k in f["tracers0/velocity"].keys()) == list(range(1, 18))
        assert f["tracers0/velocity/5"][()].shape == (1, 50, 3)
        assert np.all(f["tracers0/acceleration/5"][()] == -5.0)


def _stand_in(monkeypatch):
    from bfps_b200 import solver
    monkeypatch.setattr(solver, "vorticity_equation", _FakeField)
    monkeypatch.setattr(solver, "particles_system", _FakeTracers)
    monkeypatch.setattr(solver, "NSVEparticles_step", _fake_step)


def test_stop_file_ends_main_loop(tmp_path, monkeypatch):
    """code_base::check_stopping_condition (code_base.cpp:15-35): a file
    stop_<simname> in the working directory, checked after every iteration
    (direct_numerical_simulation.cpp:108-110), ends the job after the
    current iteration with the final statistics and checkpoint; every
    further job of the launch stops after one iteration too."""
    _stand_in(monkeypatch)
    wd = tmp_path / "run"
    wd.mkdir()
    (wd / "stop_st").write_text("")
    c = dns.DNS()
    c.launch(["NSVE", "-n", "16", "--simname", "st", "--niter_todo", "8", "--niter_out", "4",
              "--niter_stat", "1", "--njobs", "2", "--wd", str(wd)])
    with h5.File(c.get_data_file_name()) as f:
        assert f["iteration"][()] == 2
    with h5.File(c.get_checkpoint_0_fname()) as f:
        assert f["vorticity/complex"].keys() == ["0", "1", "2"]


def test_nonfinite_state_stops_the_run(tmp_path, golden, monkeypatch):
    """A NaN in the state (here in the initial field) stops the run with
    FloatingPointError before it reaches a statistics row or a checkpoint;
    the host-side stand-in for the floating-point trapping the reference
    enables (main_code.hpp:48-52)."""
    _stand_in(monkeypatch)
    src = tmp_path / "src"
    src.mkdir()
    w = np.array(golden["vorticity_0"])
    w[1, 2, 3, 0] = np.nan
    with h5.File(str(src / "B32p1e4_checkpoint_0.h5"), "w") as f:
        f["vorticity/complex/0"] = w
    c = dns.DNS()
    with pytest.raises(FloatingPointError):
        c.launch(["NSVE", "-n", "32", "--src-simname", "B32p1e4", "--src-iteration", "0",
                  "--simname", "nan", "--niter_todo", "4", "--niter_out", "4", "--niter_stat", "1",
                  "--src-wd", str(src), "--wd", str(tmp_path / "run")])
    with h5.File(c.get_data_file_name()) as f:
        assert f["iteration"][()] == 0
        assert np.all(f["statistics/moments/velocity"][()] == 0)


def test_command_line_and_postprocessing(tmp_path, golden, monkeypatch):
    """`python -m bfps_b200 DNS ...` (bfps/__main__.py) and
    DNS.compute_statistics on the run's statistics (DNS.py:196-336)."""
    from bfps_b200 import solver
    from bfps_b200.__main__ import main
    monkeypatch.setattr(solver, "vorticity_equation", _FakeField)
    monkeypatch.setattr(solver, "particles_system", _FakeTracers)
    monkeypatch.setattr(solver, "NSVEparticles_step", _fake_step)
    wd = str(tmp_path / "cli")
    main(["DNS", "NSVE", "-n", "32", "--simname", "cli", "--niter_todo", "4", "--niter_out", "4",
          "--niter_stat", "2", "--wd", wd])
    c = dns.DNS(work_dir=wd, simname="cli")
    with np.errstate(all="ignore"):   # the stand-in's enstrophy is 0 at t = 0
        c.compute_statistics()
    st = c.statistics
    assert np.allclose(st["t"], c.parameters["dt"] * 2 * np.arange(3))
    assert np.allclose(st["energy(t, k)"], 1.5 * 2 * np.arange(3)[:, None])
    assert np.allclose(st["energy(t)"], 1.5 * 2 * np.arange(3) * 17)
    assert np.allclose(st["renergy(t)"], np.arange(3))
    assert st["energy"] == pytest.approx(np.mean(1.5 * 2 * np.arange(3) * 17))
    with h5.File(str(tmp_path / "cli" / "cli_postprocess.h5")) as f:
        assert f["ii1"][()] == 2 and f["vel_max(t)"].shape == (3,)
    with pytest.raises(SystemExit):
        main(["PP"])


def test_generated_field_equals_the_reference_generator():
    """The launcher's initial field equals the reference's own
    generate_data_3D + padd_with_zeros run (tests/golden/make_ic_golden.py),
    bit for bit."""
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", "ic_vector_field_n16.npz"))["field"]
    c = NoRun()
    c.prepare_launch(["NSVE", "-n", "16"])
    got = c.generate_vector_field(spectra_slope=2.0, amplitude=0.05)
    assert got.dtype == ref.dtype and got.shape == ref.shape == (16, 16, 9, 3)
    assert np.array_equal(got, ref)
