"""The reference's own regression through the launcher.

bfps/test/test_bfps_NSVEparticles.py launches NSVEparticles from the
fixture's iteration-0 field with its arguments (2 jobs of 32 steps, 10^4
tracers, checkpoints every 32 steps, statistics every step) and compares
vorticity/complex, tracers0/state and tracers0/rhs of the run's
checkpoint file with the fixture at iterations 0, 32 and 64 (max|diff| <
1e-5).  Here the same launch goes through bfps_b200.dns: the parameter
file, checkpoints, statistics and tracer samples are written and read with
bfps_b200.h5, and the run is this package's engine."""
import numpy as np
import pytest

from bfps_b200 import h5

pytestmark = pytest.mark.gpu

REF_ARGS = ["NSVEparticles", "-n", "32", "--src-simname", "B32p1e4", "--src-iteration", "0",
            "--simname", "dns_nsveparticles", "--np", "4", "--ntpp", "1", "--niter_todo", "32",
            "--niter_out", "32", "--niter_stat", "1", "--checkpoints_per_file", "3",
            "--nparticles", "10000", "--particle-rand-seed", "2", "--njobs", "2"]


def test_reference_regression_through_launcher(tmp_path, golden):
    from bfps_b200.dns import DNS
    src = tmp_path / "src"
    src.mkdir()
    with h5.File(str(src / "B32p1e4_checkpoint_0.h5"), "w") as f:
        f["vorticity/complex/0"] = golden["vorticity_0"]
    c = DNS()
    c.launch(REF_ARGS + ["--src-wd", str(src), "--wd", str(tmp_path / "run")])
    nk = golden["state_32"].shape[0]
    with h5.File(c.get_checkpoint_0_fname()) as f:
        assert f["vorticity/complex"].keys() == ["0", "32", "64"]
        for it in (0, 32, 64):
            assert np.abs(f["vorticity/complex/%d" % it][()] - golden["vorticity_%d" % it]).max() < 1e-5
        for it in (32, 64):
            assert np.abs(f["tracers0/state/%d" % it][()][:nk] - golden["state_%d" % it]).max() < 1e-5
            assert np.abs(f["tracers0/rhs/%d" % it][()][:, :nk] - golden["rhs_%d" % it]).max() < 1e-5
    with h5.File(c.get_data_file_name()) as f:
        assert f["iteration"][()] == 64 and f["checkpoint"][()] == 0
        mom = f["statistics/moments/velocity"][()]
        spec = f["statistics/spectra/velocity_velocity"][()]
        hist = f["statistics/histograms/vorticity"][()]
        assert mom.shape == (65, 10, 4) and spec.shape[0] == 65 and hist.shape == (65, 256, 4)
        assert np.all(np.isfinite(mom)) and np.all(mom[:, 2, 3] > 0)   # <|u|^2> every step
        # energy from the spectrum and from the real-space moments agree
        # (Parseval; the spectrum stops at kM)
        e_k = 0.5 * (spec[:, :, 0, 0] + spec[:, :, 1, 1] + spec[:, :, 2, 2]).sum(axis=1)
        assert np.allclose(e_k, 0.5 * mom[:, 2, 3], rtol=0.05)
        counts = hist.sum(axis=1)[:, :3]
        assert np.all(counts > 0) and np.all(counts <= 32 ** 3)
        assert f["kspace/nshell"][()].sum() > 0
    with h5.File(c.get_particle_file_name()) as f:
        steps = sorted(int(k) for k in f["tracers0/velocity"].keys())
        assert steps == list(range(1, 66)) or len(steps) == 65
        v = f["tracers0/velocity/%d" % steps[0]][()]
        a = f["tracers0/acceleration/%d" % steps[0]][()]
        assert v.shape == (1, 10000, 3) and a.shape == (1, 10000, 3)
        assert np.all(np.isfinite(v)) and np.all(np.isfinite(a)) and np.abs(v).max() > 0


def test_launcher_fp64_nsve_matches_oracle(tmp_path):
    """NSVE in double precision from the generated initial field
    (generate_vector_field): the run's checkpoint matches the FP64 oracle
    stepped from the same file to 1e-10."""
    from bfps_b200.dns import DNS
    from oracle import nsve as O
    c = DNS()
    c.launch(["NSVE", "-n", "32", "--precision", "double", "--simname", "d", "--niter_todo", "4",
              "--niter_out", "4", "--niter_stat", "2", "--wd", str(tmp_path)])
    p = c.parameters
    with h5.File(c.get_checkpoint_0_fname()) as f:
        w0 = f["vorticity/complex/0"][()]
        w4 = f["vorticity/complex/4"][()]
    assert w0.dtype == np.complex128
    ref = O.VorticityEquation(32)
    ref.nu, ref.forcing_type, ref.famplitude, ref.fk0, ref.fk1 = p["nu"], "linear", p["famplitude"], p["fk0"], p["fk1"]
    ref.cvorticity = ref.read_checkpoint_semantics(w0)
    for _ in range(4):
        ref.step(p["dt"])
    err = np.abs(w4 - ref.cvorticity).max() / np.abs(ref.cvorticity).max()
    assert err < 1e-10, err
    with h5.File(c.get_data_file_name()) as f:
        assert f["statistics/moments/vorticity"].shape == (3, 10, 4)
        assert f["iteration"][()] == 4


def test_launcher_stop_file_ends_the_loop(tmp_path):
    """A file stop_<simname> in the working directory ends main_loop after
    the current iteration (code_base.cpp:15-35, checked every iteration by
    direct_numerical_simulation.cpp:108-110); the final statistics and
    checkpoint follow."""
    from bfps_b200.dns import DNS
    wd = tmp_path / "run"
    wd.mkdir()
    (wd / "stop_s").write_text("")
    c = DNS()
    c.launch(["NSVE", "-n", "16", "--simname", "s", "--niter_todo", "8", "--niter_out", "4",
              "--niter_stat", "1", "--wd", str(wd)])
    with h5.File(c.get_data_file_name()) as f:
        assert f["iteration"][()] == 1
    with h5.File(c.get_checkpoint_0_fname()) as f:
        assert f["vorticity/complex"].keys() == ["0", "1"]


def test_count_nonfinite_on_the_device():
    from bfps_b200.solver import vorticity_equation
    from bfps_b200 import ic
    ve = vorticity_equation(16, precision="single")
    w = ic.vorticity_ic(16, seed=3, dtype=np.complex64)
    ve.set_cvorticity(w)
    assert ve.count_nonfinite() == 0
    w[1, 2, 3, 0] = np.nan
    w[2, 1, 0, 2] = complex(0.0, np.inf)
    ve.set_cvorticity(w)
    assert ve.count_nonfinite() == 2
    ve.close()


def test_launcher_stops_on_nonfinite_state(tmp_path, golden):
    """A NaN in the initial field (injected on the host) makes the run stop
    with FloatingPointError before any statistics or checkpoint hold it."""
    from bfps_b200.dns import DNS
    src = tmp_path / "src"
    src.mkdir()
    w = np.array(golden["vorticity_0"])
    w[1, 2, 3, 0] = np.nan
    with h5.File(str(src / "B32p1e4_checkpoint_0.h5"), "w") as f:
        f["vorticity/complex/0"] = w
    c = DNS()
    with pytest.raises(FloatingPointError):
        c.launch(["NSVE", "-n", "32", "--src-simname", "B32p1e4", "--src-iteration", "0",
                  "--simname", "nan", "--niter_todo", "4", "--niter_out", "4", "--niter_stat", "1",
                  "--src-wd", str(src), "--wd", str(tmp_path / "run")])
    with h5.File(c.get_data_file_name()) as f:
        assert f["iteration"][()] == 0
