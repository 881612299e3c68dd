"""Launcher for the NSVE / NSVEparticles runs: the counterpart of bfps.DNS.

The reference's bfps.DNS (bfps/DNS.py) parses the launch arguments, writes
the parameter and statistics file `<simname>.h5`, the initial condition in
`<simname>_checkpoint_0.h5` and the tracer file `<simname>_particles.h5`,
then generates, compiles and runs (mpirun) a C++ executable whose
main_code drives NSVE / NSVEparticles through
direct_numerical_simulation::main_loop.  This module keeps the launch
arguments, parameter names and defaults, file names and dataset layouts,
and runs the jobs in-process through this package's engine on one GPU
(`--np` / `--ntpp` are accepted and recorded; the path does not shard).

  DNS().launch(['NSVEparticles', '-n', '32', '--simname', 'x', ...])

Reference anchors:
  parameters and defaults          bfps/DNS.py:139-166, bfps/_base.py:38-50
  arguments                        bfps/DNS.py:452-623, bfps/_base.py:316-328
  prepare_launch                   bfps/DNS.py:624-703
  write_par (statistics datasets)  bfps/DNS.py:372-452, bfps/_base.py:158-174
  initial conditions               bfps/DNS.py:711-844 (tracers, vector field),
                                   bfps/tools.py:96-144, 169-203
  launch_jobs                      bfps/DNS.py:845-929
  job: initialize / main_loop      bfps/cpp/full_code/NSVE.cpp:7-64,
                                   NSVEparticles.cpp:7-32,
                                   direct_numerical_simulation.cpp:9-118
  do_stats                         NSVE.cpp:101-135, NSVEparticles.cpp:66-98
  checkpoints                      vorticity_equation.cpp:49-108 (update_checkpoint),
                                   vorticity_equation.hpp:98-128, field.cpp:167-356,
                                   particles_output_hdf5.hpp:54-312
  sampled fields                   particles/particles_sampling.hpp:14-49
"""
import argparse
import os

import numpy as np

from . import h5

VERSION = "b200"
DNS_TYPES = ("NSVE", "NSVE_no_output", "NSVEparticles_no_output", "NSVEparticles")
PARTICLE_TYPES = ("NSVEparticles", "NSVEparticles_no_output")


# ------------------------------------------------------- initial fields --
# generate_data_3D and padd_with_zeros live in ic_bfps.py, a module derived
# from bfps/tools.py (GPL-3.0-or-later, see its header).
from .ic_bfps import generate_data_3D, padd_with_zeros  # noqa: E402


class DNS:
    """bfps.DNS for the NSVE family (bfps/DNS.py:42-929)."""

    def __init__(self, work_dir="./", simname="test"):
        self.work_dir = os.path.realpath(work_dir)
        self.simname = simname
        self.parameters = {"nx": 32, "ny": 32, "nz": 32}
        self.generate_default_parameters()
        self.set_precision("single")
        self.dns_type = None
        self.name = None
        self.job_info = {}
        self.statistics = {}

    # ---------------------------------------------------------- parameters
    def generate_default_parameters(self):
        p = self.parameters
        p["dealias_type"] = int(1)
        p["dkx"] = float(1.0)
        p["dky"] = float(1.0)
        p["dkz"] = float(1.0)
        p["niter_todo"] = int(8)
        p["niter_stat"] = int(1)
        p["niter_out"] = int(8)
        p["checkpoints_per_file"] = int(1)
        p["dt"] = float(0.01)
        p["nu"] = float(0.1)
        p["fmode"] = int(1)
        p["famplitude"] = float(0.5)
        p["fk0"] = float(2.0)
        p["fk1"] = float(4.0)
        p["forcing_type"] = "linear"
        p["histogram_bins"] = int(256)
        p["max_velocity_estimate"] = float(1)
        p["max_vorticity_estimate"] = float(1)
        self.NSVEp_extra_parameters = {
            "niter_part": int(1),
            "nparticles": int(10),
            "tracers0_integration_steps": int(4),
            "tracers0_neighbours": int(1),
            "tracers0_smoothness": int(1),
        }

    def set_precision(self, fluid_dtype):
        if fluid_dtype in ("single", np.float32):
            self.fluid_precision, self.rtype, self.ctype = "single", np.dtype(np.float32), np.dtype(np.complex64)
        elif fluid_dtype in ("double", np.float64):
            self.fluid_precision, self.rtype, self.ctype = "double", np.dtype(np.float64), np.dtype(np.complex128)
        else:
            raise ValueError("precision must be single or double")
        self.fluid_dtype = self.rtype

    def get_kspace(self):
        """kspace tables as bfps.DNS.get_kspace (DNS.py:167-195)."""
        p = self.parameters
        div = 2 if p["dealias_type"] == 1 else 3
        kM = max(p["dkx"] * (p["nx"] // div - 1), p["dky"] * (p["ny"] // div - 1),
                 p["dkz"] * (p["nz"] // div - 1))
        dk = min(p["dkx"], p["dky"], p["dkz"])
        nshells = int(kM / dk) + 2
        ks = {"kM": kM, "dk": dk, "nshell": np.zeros(nshells, np.int64),
              "kshell": np.zeros(nshells, np.float64),
              "kx": np.arange(0, p["nx"] // 2 + 1).astype(np.float64) * p["dkx"]}
        ky = np.arange(-p["ny"] // 2 + 1, p["ny"] // 2 + 1).astype(np.float64) * p["dky"]
        ks["ky"] = np.roll(ky, p["ny"] // 2 + 1)
        kz = np.arange(-p["nz"] // 2 + 1, p["nz"] // 2 + 1).astype(np.float64) * p["dkz"]
        ks["kz"] = np.roll(kz, p["nz"] // 2 + 1)
        return ks

    # ---------------------------------------------------------- file names
    def get_data_file_name(self):
        return os.path.join(self.work_dir, self.simname + ".h5")

    def get_particle_file_name(self):
        return os.path.join(self.work_dir, self.simname + "_particles.h5")

    def get_checkpoint_fname(self, checkpoint):
        return os.path.join(self.work_dir, self.simname + "_checkpoint_%d.h5" % checkpoint)

    def get_checkpoint_0_fname(self):
        return self.get_checkpoint_fname(0)

    def get_data_file(self):
        return h5.File(self.get_data_file_name(), "r")

    def get_particle_file(self):
        return h5.File(self.get_particle_file_name(), "r")

    # ---------------------------------------------------------- postprocessing
    def read_parameters(self):
        """Parameters of an existing run (bfps/_base.py:220-228)."""
        with self.get_data_file() as f:
            for k in f["parameters"].keys():
                if k in self.parameters:
                    v = f["parameters/" + k][()]
                    v = v.item() if hasattr(v, "item") else v
                    v = v.decode() if isinstance(v, bytes) else v
                    t = type(self.parameters[k])
                    self.parameters[k] = t(v) if t in (int, float, str) else v

    def compute_statistics(self, iter0=0, iter1=None):
        """Energy and enstrophy spectra, maximum velocity and energy per
        statistics step, then the time averages (bfps/DNS.py:196-272); the
        per-time quantities are kept in `<simname>_postprocess.h5`."""
        if len(self.statistics) > 0:
            return
        self.read_parameters()
        ns = self.parameters["niter_stat"]
        with self.get_data_file() as f:
            if "moments" not in f["statistics"].keys():
                return
            mom = f["statistics/moments/velocity"][()]
            iter0 = min(mom.shape[0] * ns - 1, iter0)
            last = int(f["iteration"][()])
            iter1 = last if iter1 is None else min(last, iter1)
            ii0, ii1 = iter0 // ns, iter1 // ns
            self.statistics["kshell"] = f["kspace/kshell"][()]
            self.statistics["kM"] = float(f["kspace/kM"][()])
            self.statistics["dk"] = float(f["kspace/dk"][()])
            uu = f["statistics/spectra/velocity_velocity"][()][ii0:ii1 + 1]
            ww = f["statistics/spectra/vorticity_vorticity"][()][ii0:ii1 + 1]
        pp = {"iter0": iter0, "iter1": iter1, "ii0": ii0, "ii1": ii1,
              "t": self.parameters["dt"] * ns * np.arange(ii0, ii1 + 1).astype(np.float64),
              "energy(t, k)": (uu[:, :, 0, 0] + uu[:, :, 1, 1] + uu[:, :, 2, 2]) / 2,
              "enstrophy(t, k)": (ww[:, :, 0, 0] + ww[:, :, 1, 1] + ww[:, :, 2, 2]) / 2,
              "vel_max(t)": mom[ii0:ii1 + 1, 9, 3],
              "renergy(t)": mom[ii0:ii1 + 1, 2, 3] / 2}
        name = os.path.join(self.work_dir, self.simname + "_postprocess.h5")
        with h5.File(name, "w") as f:
            for k, v in pp.items():
                f[k] = v
        for k in ("t", "energy(t, k)", "enstrophy(t, k)", "vel_max(t)", "renergy(t)"):
            self.statistics[k] = pp[k]
        self.compute_time_averages()

    def compute_time_averages(self):
        """Integral and Kolmogorov scales, Reynolds numbers (DNS.py:273-336)."""
        st, nu = self.statistics, self.parameters["nu"]
        for key in ("energy", "enstrophy"):
            st[key + "(t)"] = st["dk"] * np.sum(st[key + "(t, k)"], axis=1)
        st["Uint(t)"] = np.sqrt(2 * st["energy(t)"] / 3)
        with np.errstate(divide="ignore", invalid="ignore"):
            st["Lint(t)"] = ((st["dk"] * np.pi / (2 * st["Uint(t)"] ** 2)) *
                             np.nansum(st["energy(t, k)"] / st["kshell"][None, :], axis=1))
        for key in ("energy", "enstrophy", "vel_max", "Uint", "Lint"):
            if key + "(t)" in st:
                st[key] = np.average(st[key + "(t)"], axis=0)
        for sfx in ("", "(t)"):
            st["diss" + sfx] = nu * st["enstrophy" + sfx] * 2
            st["etaK" + sfx] = (nu ** 3 / st["diss" + sfx]) ** .25
            st["tauK" + sfx] = (nu / st["diss" + sfx]) ** .5
            st["Re" + sfx] = st["Uint" + sfx] * st["Lint" + sfx] / nu
            st["lambda" + sfx] = (15 * nu * st["Uint" + sfx] ** 2 / st["diss" + sfx]) ** .5
            st["Rlambda" + sfx] = st["Uint" + sfx] * st["lambda" + sfx] / nu
            st["kMeta" + sfx] = st["kM"] * st["etaK" + sfx]
            if self.parameters["dealias_type"] == 1:
                st["kMeta" + sfx] *= 0.8
        st["Tint"] = st["Lint"] / st["Uint"]
        st["Taylor_microscale"] = st["lambda"]

    # ---------------------------------------------------------- arguments
    @staticmethod
    def _job_arguments(parser):
        parser.add_argument("--ncpu", type=int, dest="ncpu", default=-1)
        parser.add_argument("--np", "--nprocesses", metavar="NPROCESSES", type=int,
                            dest="nb_processes", default=4,
                            help="number of MPI processes of the reference's launch (recorded; "
                                 "the run uses one GPU)")
        parser.add_argument("--ntpp", "--nthreads-per-process", type=int,
                            dest="nb_threads_per_process", metavar="NTHREADS_PER_PROCESS", default=1)
        parser.add_argument("--no-submit", action="store_true", dest="no_submit")
        parser.add_argument("--environment", type=str, dest="environment", default=None)
        parser.add_argument("--minutes", type=int, dest="minutes", default=5)
        parser.add_argument("--njobs", type=int, dest="njobs", default=1)

    @staticmethod
    def _simulation_arguments(parser):
        parser.add_argument("--simname", type=str, dest="simname", default="test")
        parser.add_argument("-n", "--grid-size", type=int, dest="n", default=32, metavar="N")
        for c in "xyz":
            parser.add_argument("--L%s" % c, "--box-length-%s" % c, type=float, dest="L%s" % c,
                                default=2.0, metavar="length%s" % c)
        parser.add_argument("--wd", type=str, dest="work_dir", default="./")
        parser.add_argument("--precision", choices=["single", "double"], type=str, default="single")
        parser.add_argument("--src-wd", type=str, dest="src_work_dir", default="")
        parser.add_argument("--src-simname", type=str, dest="src_simname", default="")
        parser.add_argument("--src-iteration", type=int, dest="src_iteration", default=0)
        parser.add_argument("--kMeta", type=float, dest="kMeta", default=2.0)
        parser.add_argument("--dtfactor", type=float, dest="dtfactor", default=0.5,
                            help="dt is computed as DTFACTOR / N")

    @staticmethod
    def _particle_arguments(parser):
        parser.add_argument("--particle-rand-seed", type=int, dest="particle_rand_seed", default=None)
        parser.add_argument("--pclouds", type=int, dest="pclouds", default=1)
        parser.add_argument("--pcloud-type", choices=["random-cube", "regular-cube"],
                            dest="pcloud_type", default="random-cube")
        parser.add_argument("--particle-cloud-size", type=float, dest="particle_cloud_size",
                            default=2 * np.pi)

    @staticmethod
    def _parameter_arguments(parser, parameters):
        for k in sorted(parameters):
            parser.add_argument("--%s" % k, type=type(parameters[k]), dest=k, default=None)

    def add_parser_arguments(self, parser):
        sub = parser.add_subparsers(dest="DNS_class", help="type of simulation to run")
        sub.required = True
        for t in DNS_TYPES:
            sp = sub.add_parser(t)
            self._simulation_arguments(sp)
            self._job_arguments(sp)
            if t in PARTICLE_TYPES:
                self._particle_arguments(sp)
            self._parameter_arguments(sp, self.parameters)
            if t in PARTICLE_TYPES:
                self._parameter_arguments(sp, self.NSVEp_extra_parameters)

    def pars_from_namespace(self, opt):
        """bfps/_base.py:229-247: n fills nx/ny/nz, set arguments override."""
        cmd = vars(opt)
        if "n" in cmd:
            for k in ("nx", "ny", "nz"):
                if cmd.get(k) is None:
                    cmd[k] = opt.n
        for k in self.parameters:
            if cmd.get(k) is not None:
                self.parameters[k] = cmd[k]
        self.simname = opt.simname
        self.work_dir = os.path.realpath(opt.work_dir)

    def prepare_launch(self, args=()):
        parser = argparse.ArgumentParser("bfps_b200 DNS")
        self.add_parser_arguments(parser)
        opt = parser.parse_args(list(args))
        if opt.ncpu != -1:
            opt.nb_processes, opt.nb_threads_per_process = opt.ncpu, 1
        self.set_precision(opt.precision)
        self.dns_type = opt.DNS_class
        self.name = self.dns_type + "-" + self.fluid_precision + "-v" + VERSION
        if self.dns_type in PARTICLE_TYPES:
            for k, v in self.NSVEp_extra_parameters.items():
                self.parameters[k] = v
        self.parameters["nu"] = (opt.kMeta * 2 / opt.n) ** (4. / 3)
        self.parameters["dt"] = opt.dtfactor / opt.n
        if opt.n == 288:
            self.parameters["famplitude"] = 0.45
        elif opt.n == 576:
            self.parameters["famplitude"] = 0.47
        if self.parameters["niter_todo"] % self.parameters["niter_out"] != 0:
            self.parameters["niter_out"] = self.parameters["niter_todo"]
        if len(opt.src_work_dir) == 0:
            opt.src_work_dir = os.path.realpath(opt.work_dir)
        if opt.dkx is None:
            opt.dkx = 2. / opt.Lx
        if opt.dky is None:
            opt.dky = 2. / opt.Ly
        # bfps/DNS.py:680-681 tests dkx again here, so dkz keeps its default
        # unless given on the command line
        if opt.dkx is None:
            opt.dkz = 2. / opt.Lz
        for c in ("nx", "ny", "nz"):
            if getattr(opt, c) is None:
                setattr(opt, c, opt.n)
        if opt.checkpoints_per_file is None:
            field_size = 3 * (opt.nx + 2) * opt.ny * opt.nz * self.fluid_dtype.itemsize
            size = field_size
            if self.dns_type in PARTICLE_TYPES:
                rhs = self.parameters["tracers0_integration_steps"]
                if opt.tracers0_integration_steps is not None:
                    rhs = opt.tracers0_integration_steps
                npart = opt.nparticles if opt.nparticles is not None else self.NSVEp_extra_parameters["nparticles"]
                size += (1 + rhs) * 3 * npart * 8
            if size < 1e9:
                opt.checkpoints_per_file = int(1e9 / size)
        self.pars_from_namespace(opt)
        return opt

    def launch(self, args=(), **kwargs):
        opt = self.prepare_launch(args=args)
        self.launch_jobs(opt=opt, **kwargs)

    # ---------------------------------------------------------- files
    def write_par(self, iter0=0):
        p = self.parameters
        assert p["niter_todo"] % p["niter_stat"] == 0
        assert p["niter_todo"] % p["niter_out"] == 0
        assert p["niter_out"] % p["niter_stat"] == 0
        if self.dns_type in PARTICLE_TYPES:
            assert p["niter_todo"] % p["niter_part"] == 0
            assert p["niter_out"] % p["niter_part"] == 0
        os.makedirs(self.work_dir, exist_ok=True)
        if os.path.exists(self.get_data_file_name()):
            raise FileExistsError(self.get_data_file_name())
        with h5.File(self.get_data_file_name(), "w") as f:
            for k, v in p.items():
                f["parameters/" + k] = np.bytes_(v.encode("ascii")) if isinstance(v, str) else v
            f["iteration"] = np.int64(iter0)
            f["bfps_info/solver_class"] = np.bytes_(type(self).__name__.encode())
            f["bfps_info/exec_name"] = np.bytes_(self.name.encode())
            f["bfps_info/version"] = np.bytes_(VERSION.encode())
            for k, v in self.job_info.items():
                f["bfps_info/" + k] = np.bytes_(str(v).encode())
            ks = self.get_kspace()
            for k, v in ks.items():
                f["kspace/" + k] = v
            nshells = ks["nshell"].shape[0]
            nbins = p["histogram_bins"]
            for k in ("velocity", "vorticity"):
                tc = max(2 ** 20 // (8 * 3 * 3 * nshells), 1)
                f.create_dataset("statistics/spectra/%s_%s" % (k, k), (1, nshells, 3, 3),
                                 chunks=(tc, nshells, 3, 3), maxshape=(None, nshells, 3, 3),
                                 dtype=np.float64)
                tc = max(2 ** 20 // (8 * 4 * 10), 1)
                f.create_dataset("statistics/moments/" + k, (1, 10, 4), chunks=(tc, 10, 4),
                                 maxshape=(None, 10, 4), dtype=np.float64)
                tc = max(2 ** 20 // (8 * 4 * nbins), 1)
                f.create_dataset("statistics/histograms/" + k, (1, nbins, 4), chunks=(tc, nbins, 4),
                                 maxshape=(None, nbins, 4), dtype=np.int64)
            f["checkpoint"] = np.int64(0)
        if self.dns_type not in PARTICLE_TYPES:
            return
        n = p["nparticles"]
        with h5.File(self.get_checkpoint_0_fname(), "a") as f:
            f.create_group("tracers0/rhs")
            f.create_group("tracers0/state")
            f.create_dataset("tracers0/rhs/0", (p["tracers0_integration_steps"], n, 3), np.float64)
            f.create_dataset("tracers0/state/0", (n, 3), np.float64)

    def generate_tracer_state(self, rseed=None, species=0):
        """Uniform positions in [0, 2 pi)^3 from numpy's legacy generator,
        drawn in batches of 10^6 (DNS.py:711-733; the batches continue one
        stream, so the result equals a single draw)."""
        if rseed is not None:
            np.random.seed(rseed)
        n = self.parameters["nparticles"]
        pos = np.empty((n, 3))
        batch = int(1e6)
        for c in range(0, n, batch):
            m = min(batch, n - c)
            pos[c:c + m] = np.random.random((m, 3)) * 2 * np.pi
        with h5.File(self.get_checkpoint_0_fname(), "a") as f:
            f["tracers%d/state/0" % species].write(pos)

    def generate_vector_field(self, rseed=7547, spectra_slope=1., amplitude=1.):
        """DNS.py:734-806 with tools.generate_data_3D: three random
        components, padded to the grid."""
        np.random.seed(rseed)
        p = self.parameters
        comps = [generate_data_3D(p["nz"] // 2, p["ny"] // 2, p["nx"] // 2, p=spectra_slope,
                                  amplitude=amplitude).astype(self.ctype) for _ in range(3)]
        k0 = np.zeros(comps[0].shape + (3,), comps[0].dtype)
        for i in range(3):
            k0[..., i] = comps[i]
        return padd_with_zeros(k0, p["nz"], p["ny"], p["nx"])

    def copy_complex_field(self, src_file_name, src_dset_name, dst_file, dst_dset_name):
        """DNS.py:807-844: same shape copies the field (converted to the run
        precision), another shape copies the common low modes."""
        p = self.parameters
        dst_shape = (p["nz"], p["ny"], (p["nx"] + 2) // 2, 3)
        with h5.File(src_file_name, "r") as src:
            a = src[src_dset_name][()]
        if a.shape == dst_shape:
            dst_file[dst_dset_name] = a.astype(self.ctype)
            return
        b = np.zeros(dst_shape, self.ctype)
        m = tuple(min(d, s) for d, s in zip(dst_shape[:3], a.shape[:3]))
        b[:m[0], :m[1], :m[2]] = a[:m[0], :m[1], :m[2]]
        dst_file[dst_dset_name] = b

    def launch_jobs(self, opt=None, particle_initial_condition=None):
        self.job_info = {"nb_processes": opt.nb_processes,
                         "nb_threads_per_process": opt.nb_threads_per_process}
        if not os.path.exists(self.get_data_file_name()):
            if not os.path.exists(self.get_checkpoint_0_fname()):
                os.makedirs(self.work_dir, exist_ok=True)
                with h5.File(self.get_checkpoint_0_fname(), "w") as f:
                    if len(opt.src_simname) > 0:
                        cp = 0
                        while True:
                            src = os.path.join(os.path.realpath(opt.src_work_dir),
                                               opt.src_simname + "_checkpoint_%d.h5" % cp)
                            with h5.File(src, "r") as f0:
                                if str(opt.src_iteration) in f0["vorticity/complex"].keys():
                                    break
                            cp += 1
                        self.copy_complex_field(src, "vorticity/complex/%d" % opt.src_iteration,
                                                f, "vorticity/complex/0")
                    else:
                        f["vorticity/complex/0"] = self.generate_vector_field(
                            spectra_slope=2.0, amplitude=0.05)
            self.write_par()
            if self.dns_type in PARTICLE_TYPES and self.parameters["nparticles"] > 0:
                self.generate_tracer_state(species=0, rseed=opt.particle_rand_seed)
                if not os.path.exists(self.get_particle_file_name()):
                    with h5.File(self.get_particle_file_name(), "w") as pf:
                        pf.create_group("tracers0/velocity")
                        pf.create_group("tracers0/acceleration")
        self.run(nb_processes=opt.nb_processes, nb_threads_per_process=opt.nb_threads_per_process,
                 njobs=opt.njobs)

    def run(self, nb_processes=1, nb_threads_per_process=1, njobs=1, device=0, **_):
        """The jobs of a launch, one after the other, each a fresh
        initialize / main_loop / finalize of the executable's main_code."""
        for _ in range(njobs):
            job = _Job(self, device)
            try:
                job.initialize()
                job.main_loop()
            finally:
                job.finalize()


class _Job:
    """One run of the generated executable: NSVE / NSVEparticles over
    direct_numerical_simulation (main_code.hpp), on this package's engine."""

    def __init__(self, dns, device):
        self.dns = dns
        self.device = device
        self.fs = None
        self.ps = None
        self.particles = dns.dns_type in PARTICLE_TYPES
        self.output = not dns.dns_type.endswith("_no_output")

    # direct_numerical_simulation::read_iteration, read_parameters
    def _read(self):
        d = self.dns
        with h5.File(d.get_data_file_name(), "r") as f:
            self.iteration = int(f["iteration"][()])
            self.checkpoint = int(f["checkpoint"][()])
            par = {}
            for k in f["parameters"].keys():
                v = f["parameters/" + k][()]
                v = v.item() if hasattr(v, "item") else v
                par[k] = v.decode() if isinstance(v, bytes) else v
        self.p = par

    def initialize(self):
        from .solver import particles_system, vorticity_equation
        d = self.dns
        self._read()
        p = self.p
        # grow the statistics datasets by this job's statistics steps
        with h5.File(d.get_data_file_name(), "a") as f:
            for name in self._stat_datasets(f):
                ds = f[name]
                ds.resize(ds.shape[0] + p["niter_todo"] // p["niter_stat"])
        self.fs = vorticity_equation(p["nx"], p["ny"], p["nz"], p["dkx"], p["dky"], p["dkz"],
                                     precision=d.fluid_precision, dealias_type=p["dealias_type"],
                                     device=self.device)
        fs = self.fs
        fs.nu, fs.fmode, fs.famplitude = p["nu"], p["fmode"], p["famplitude"]
        fs.fk0, fs.fk1, fs.forcing_type = p["fk0"], p["fk1"], p["forcing_type"]
        fs.iteration = self.iteration
        with h5.File(self._fname(), "r") as f:
            fs.io_checkpoint_read(f["vorticity/complex/%d" % self.iteration][()])
        if self.iteration == 0:
            # kspace::store (kspace.cpp:178-236)
            ks = fs.kspace()
            with h5.File(d.get_data_file_name(), "a") as f:
                f["kspace/kshell"].write(ks["kshell"])
                f["kspace/nshell"].write(ks["nshell"])
                f["kspace/kM"].write(np.float64(ks["kM"]))
                f["kspace/dk"].write(np.float64(ks["dk"]))
        if self.particles:
            with h5.File(self._fname(), "r") as f:
                pos = f["tracers0/state/%d" % self.iteration][()]
                rhs = f["tracers0/rhs/%d" % self.iteration][()]
            if rhs.shape[0] != p["tracers0_integration_steps"] or pos.shape[0] != p["nparticles"]:
                raise ValueError("tracer input does not match the parameters")
            self.ps = particles_system(fs, pos, p["tracers0_neighbours"], p["tracers0_smoothness"],
                                       p["tracers0_integration_steps"], rhs=rhs,
                                       step_idx=self.iteration + 1)

    @staticmethod
    def _stat_datasets(f):
        out = []
        for grp in ("spectra", "moments", "histograms"):
            for k in f["statistics/" + grp].keys():
                out.append("statistics/%s/%s" % (grp, k))
        return out

    def _fname(self):
        return self.dns.get_checkpoint_fname(self.checkpoint)

    # direct_numerical_simulation::main_loop
    # (direct_numerical_simulation.cpp:89-118): stats, step, checkpoint every
    # niter_out, then the stopping condition, every iteration
    def main_loop(self):
        p = self.p
        it = self.iteration
        max_iter = it + p["niter_todo"] - (it % p["niter_todo"])
        self.stopped = False
        while self.iteration < max_iter:
            self.do_stats()
            self.step()
            if self.iteration % p["niter_out"] == 0:
                self.write_checkpoint()
            if self.check_stopping_condition():
                self.stopped = True
                break
        self.do_stats()
        if self.iteration % p["niter_out"] != 0:
            self.write_checkpoint()

    # code_base::check_stopping_condition (code_base.cpp:15-35): a file
    # named stop_<simname> in the run's working directory ends the loop
    def check_stopping_condition(self):
        return os.path.exists(os.path.join(self.dns.work_dir, "stop_" + self.dns.simname))

    # The reference traps floating-point exceptions in its host arithmetic
    # (main_code.hpp:48-52); the arithmetic here runs on the device, so the
    # state is scanned on the device before statistics and checkpoints are
    # written, and a non-finite value stops the run with an error instead of
    # a corrupted file.
    def check_finite(self):
        bad = self.fs.count_nonfinite("vorticity")
        if bad:
            raise FloatingPointError("iteration %d: %d non-finite values in the vorticity field"
                                     % (self.iteration, bad))

    def step(self):
        from .solver import NSVEparticles_step
        if self.particles:
            NSVEparticles_step(self.fs, self.ps, self.p["dt"], 1)
        else:
            self.fs.step(self.p["dt"], 1)
        self.iteration = self.fs.iteration

    # NSVE::do_stats + NSVEparticles::do_stats
    def do_stats(self):
        p = self.p
        if self.iteration % p["niter_stat"] == 0:
            self.check_finite()
            st = self.fs.do_stats(p["max_velocity_estimate"], p["max_vorticity_estimate"],
                                  p["histogram_bins"])
            t = self.iteration // p["niter_stat"]
            with h5.File(self.dns.get_data_file_name(), "a") as f:
                for k in ("vorticity", "velocity"):
                    spec, mom, hist = st[k]
                    f["statistics/spectra/%s_%s" % (k, k)].write_rows(t, spec[None])
                    f["statistics/moments/" + k].write_rows(t, mom[None])
                    f["statistics/histograms/" + k].write_rows(t, hist[None])
        if not self.particles or self.iteration % p["niter_part"] != 0:
            return
        step_idx = self.ps.step_idx
        with h5.File(self.dns.get_particle_file_name(), "a") as pf:
            for field in ("velocity", "acceleration"):
                name = "tracers0/%s/%d" % (field, step_idx)
                if name in pf:   # DatasetExistsCol: stop if it exists
                    continue
                if field == "velocity":
                    self.fs.velocity_rspace()
                    vals = self.ps.sample_velocity()
                else:
                    vals = self.ps.sample_acceleration()
                pf[name] = vals[None]

    # vorticity_equation::update_checkpoint (vorticity_equation.cpp:49-108)
    def _update_checkpoint(self):
        fname = self._fname()
        if os.path.exists(fname):
            with h5.File(fname, "r") as f:
                stored = f["vorticity/complex"].keys() if "vorticity/complex" in f else []
            if len(stored) >= self.p["checkpoints_per_file"] and str(self.iteration) not in stored:
                self.checkpoint += 1
        else:
            with h5.File(fname, "w") as f:
                f.create_group("vorticity/complex")

    def write_checkpoint(self):
        if not self.output:
            return
        self.check_finite()
        self._update_checkpoint()
        fname = self._fname()
        with h5.File(fname, "a") as f:
            name = "vorticity/complex/%d" % self.iteration
            v = self.fs.get_cvorticity()
            if name in f:
                f[name].write(v)
            else:
                f[name] = v
            if self.particles:
                pos, rhs, _ = self.ps.state()
                f.require_group("tracers0/state")
                f.require_group("tracers0/rhs")
                f["tracers0/state/%d" % self.iteration] = pos
                f["tracers0/rhs/%d" % self.iteration] = rhs
        # direct_numerical_simulation::write_iteration
        with h5.File(self.dns.get_data_file_name(), "a") as f:
            f["iteration"].write(np.int64(self.iteration))
            f["checkpoint"].write(np.int64(self.checkpoint))

    def finalize(self):
        if self.ps is not None:
            self.ps.close()
            self.ps = None
        if self.fs is not None:
            self.fs.close()
            self.fs = None


def main(argv=None):
    import sys
    DNS().launch(sys.argv[1:] if argv is None else argv)


if __name__ == "__main__":
    main()
