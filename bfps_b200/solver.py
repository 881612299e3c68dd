"""Host-side mirror of bfps' building blocks over the C-ABI.

``vorticity_equation`` mirrors ``vorticity_equation<rnumber, FFTW>``
(bfps/cpp/vorticity_equation.hpp:46-134): public physical members, step(),
compute_velocity(), the io_checkpoint read semantics, and the iteration
counter.  ``particles_system`` mirrors ``abstract_particles_system``
(bfps/cpp/particles/abstract_particles_system.hpp:12-55) with
completeLoop(), and ``NSVEparticles_step`` is NSVEparticles::step
(bfps/cpp/full_code/NSVEparticles.cpp:33-41).  Fields cross the boundary in
the reference's host layouts (bfps/cpp/field.cpp:85-101).

All compute runs in the CUDA library; every method raises on failure.
"""
import atexit
import ctypes
import weakref

import numpy as np

from . import _lib
from ._lib import check, lib, ptr

# Objects still open when the interpreter exits are closed here, before the
# modules are torn down, ensembles first, then tracer sets, then their
# contexts (a tracer set's destruction synchronises its context's streams).
_live = {"ensemble": weakref.WeakSet(), "particles": weakref.WeakSet(),
         "context": weakref.WeakSet()}


@atexit.register
def _close_all():
    for kind in ("ensemble", "particles", "context"):
        for obj in list(_live[kind]):
            try:
                obj.close()
            except Exception:
                pass


class vorticity_equation:
    def __init__(self, nx, ny=None, nz=None, dkx=1.0, dky=1.0, dkz=1.0,
                 precision="double", dealias_type=_lib.SMOOTH, device=0):
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        self.nx, self.ny, self.nz = nx, ny, nz
        self.real_bytes = {"single": 4, "double": 8}[precision]
        self.rdtype = np.float32 if self.real_bytes == 4 else np.float64
        self.cdtype = np.complex64 if self.real_bytes == 4 else np.complex128
        h = ctypes.c_void_p()
        rc = lib().bfg_ctx_create(ctypes.byref(h), nx, ny, nz, dkx, dky, dkz,
                                  self.real_bytes, dealias_type, device)
        if rc != 0:
            raise _lib.BfgError(rc, "bfg_ctx_create(%d, %d, %d, precision=%s)" %
                                (nx, ny, nz, precision))
        self._h = h
        _live["context"].add(self)
        # defaults of the reference constructor (vorticity_equation.cpp:150-155)
        self._nu = 0.1
        self._forcing_type = "none"
        self._famplitude = 1.0
        self._fk0 = 2.0
        self._fk1 = 4.0
        self._fmode = 1
        self._push_physics()

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            lib().bfg_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- physical members ---------------------------------------------------
    def _push_physics(self):
        check(lib().bfg_set_physics(self._h, self._nu, _lib.FORCING[self._forcing_type],
                                    self._famplitude, self._fk0, self._fk1, self._fmode), self._h)

    def _prop(name):
        def get(self):
            return getattr(self, "_" + name)

        def set_(self, v):
            setattr(self, "_" + name, v)
            self._push_physics()
        return property(get, set_)

    nu = _prop("nu")
    forcing_type = _prop("forcing_type")
    famplitude = _prop("famplitude")
    fk0 = _prop("fk0")
    fk1 = _prop("fk1")
    fmode = _prop("fmode")
    del _prop

    @property
    def iteration(self):
        it = ctypes.c_int()
        check(lib().bfg_get_iteration(self._h, ctypes.byref(it)), self._h)
        return it.value

    @iteration.setter
    def iteration(self, v):
        check(lib().bfg_set_iteration(self._h, int(v)), self._h)

    # -- kspace --------------------------------------------------------------
    def kspace(self):
        kM, dk, ns = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        check(lib().bfg_kspace_info(self._h, ctypes.byref(kM), ctypes.byref(dk),
                                    ctypes.byref(ns), None, None), self._h)
        kshell = np.zeros(ns.value)
        nshell = np.zeros(ns.value, np.int64)
        check(lib().bfg_kspace_info(self._h, None, None, None, ptr(kshell),
                                    ptr(nshell, ctypes.c_int64)), self._h)
        return dict(kM=kM.value, dk=dk.value, nshells=ns.value, kshell=kshell, nshell=nshell)

    # -- fields ----------------------------------------------------------------
    @property
    def cshape(self):
        return (self.ny, self.nz, self.nx // 2 + 1, 3)

    @property
    def rshape(self):
        return (self.nz, self.ny, self.nx + 2, 3)

    def set_cvorticity(self, a):
        a = np.ascontiguousarray(a, dtype=self.cdtype)
        assert a.shape == self.cshape, a.shape
        check(lib().bfg_field_upload(self._h, _lib.FIELD_VORTICITY, a.ctypes.data), self._h)

    def get_cvorticity(self):
        out = np.empty(self.cshape, self.cdtype)
        check(lib().bfg_field_download(self._h, _lib.FIELD_VORTICITY, out.ctypes.data), self._h)
        return out

    def get_cvelocity(self):
        out = np.empty(self.cshape, self.cdtype)
        check(lib().bfg_field_download(self._h, _lib.FIELD_VELOCITY, out.ctypes.data), self._h)
        return out

    def get_rvelocity(self):
        out = np.empty(self.rshape, self.rdtype)
        check(lib().bfg_field_download(self._h, _lib.FIELD_RVELOCITY, out.ctypes.data), self._h)
        return out

    def set_rvelocity(self, r):
        r = np.ascontiguousarray(r, dtype=self.rdtype)
        assert r.shape == self.rshape
        check(lib().bfg_field_upload(self._h, _lib.FIELD_RVELOCITY, r.ctypes.data), self._h)

    def io_checkpoint_read(self, a):
        """Upload a checkpoint field and apply io_checkpoint(read) semantics
        (vorticity_equation.hpp:107-128): symmetrize, low_pass(kM), force_divfree."""
        self.set_cvorticity(a)
        check(lib().bfg_read_checkpoint_fixup(self._h), self._h)

    # -- solver ------------------------------------------------------------------
    def step(self, dt, nsteps=1):
        check(lib().bfg_step(self._h, float(dt), int(nsteps)), self._h)

    def compute_velocity(self):
        check(lib().bfg_compute_velocity(self._h), self._h)

    def velocity_rspace(self):
        check(lib().bfg_velocity_rspace(self._h), self._h)

    def compute_pressure(self):
        """vorticity_equation::compute_pressure (vorticity_equation.cpp:441-514)
        of the current state's velocity, (ny, nz, nx/2+1) complex."""
        out = np.empty(self.cshape[:3], self.cdtype)
        check(lib().bfg_compute_pressure(self._h, out.ctypes.data), self._h)
        return out

    def compute_Lagrangian_acceleration(self):
        """vorticity_equation::compute_Lagrangian_acceleration
        (vorticity_equation.cpp:516-578) of the current state, Fourier space."""
        out = np.empty(self.cshape, self.cdtype)
        check(lib().bfg_lagrangian_acceleration(self._h, out.ctypes.data), self._h)
        return out

    def count_nonfinite(self, field="vorticity"):
        """Number of NaN / Inf values in a field on the device
        (bfg_check_finite)."""
        fid = {"vorticity": _lib.FIELD_VORTICITY, "velocity": _lib.FIELD_VELOCITY,
               "rvelocity": _lib.FIELD_RVELOCITY}[field]
        n = ctypes.c_int64()
        check(lib().bfg_check_finite(self._h, fid, ctypes.byref(n)), self._h)
        return n.value

    def reset(self):
        """bfg_ctx_reset: the state of a new context of this grid (fields
        zero, iteration 0) on the same device memory."""
        check(lib().bfg_ctx_reset(self._h), self._h)

    def autotune(self, reps=3):
        """bfg_autotune: time both schedules of the IZ, IY, FY and FZ passes
        on this context and keep the faster for this device, grid size and
        precision, one member per launch.  Returns {pass: (schedule, ms0,
        ms1)}.  The context's velocity fields are used as work space
        (recompute them afterwards)."""
        check(lib().bfg_autotune(self._h, int(reps)), self._h)
        return self.schedules()

    def schedules(self, members=1):
        """{pass: (schedule, ms0, ms1)} for launches over `members` contexts
        of this grid size and precision (ensemble groups of that size)."""
        out = {}
        for kind, name in ((0, "IZ"), (1, "IY"), (3, "FY"), (4, "FZ")):
            sc, m0, m1 = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
            check(lib().bfg_tune_get(self._h, kind, int(members), ctypes.byref(sc),
                                     ctypes.byref(m0), ctypes.byref(m1)), self._h)
            out[name] = (sc.value, m0.value, m1.value)
        return out

    def set_schedule(self, name, schedule, members=1):
        kind = {"IZ": 0, "IY": 1, "FY": 3, "FZ": 4}[name]
        check(lib().bfg_tune_set(self._h, kind, int(members), int(schedule)), self._h)

    def last_step_ms(self):
        ms = ctypes.c_double()
        check(lib().bfg_last_step_ms(self._h, ctypes.byref(ms)), self._h)
        return ms.value

    def kernel_launches(self):
        n = ctypes.c_int64()
        check(lib().bfg_kernel_launches(self._h, ctypes.byref(n)), self._h)
        return n.value

    def do_stats(self, max_velocity_estimate=1.0, max_vorticity_estimate=1.0, nbins=256):
        """NSVE::do_stats (NSVE.cpp:101-135) results as numpy arrays."""
        ns = self.kspace()["nshells"]
        sv, sw = np.zeros((ns, 3, 3)), np.zeros((ns, 3, 3))
        mv, mw = np.zeros((10, 4)), np.zeros((10, 4))
        hv, hw = np.zeros((nbins, 4), np.int64), np.zeros((nbins, 4), np.int64)
        check(lib().bfg_stats(self._h, max_velocity_estimate, max_vorticity_estimate, nbins,
                              ptr(sv), ptr(sw), ptr(mv), ptr(mw), ptr(hv, ctypes.c_int64),
                              ptr(hw, ctypes.c_int64)), self._h)
        return {"velocity": (sv, mv, hv), "vorticity": (sw, mw, hw)}


class particles_system:
    """Tracers on the device (particles_system_builder + particles_system)."""

    def __init__(self, fs, pos, neighbours, smoothness, nsteps, rhs=None, idx=None, step_idx=1):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        n = pos.shape[0]
        if rhs is not None:
            rhs = np.ascontiguousarray(rhs, dtype=np.float64)
            assert rhs.shape == (nsteps, n, 3)
        if idx is not None:
            idx = np.ascontiguousarray(idx, dtype=np.int64)
        h = ctypes.c_void_p()
        check(lib().bfg_particles_create(fs.handle, ctypes.byref(h), n, neighbours, smoothness,
                                         nsteps, ptr(pos), ptr(rhs), ptr(idx, ctypes.c_int64),
                                         step_idx), fs.handle)
        self._h = h
        _live["particles"].add(self)
        self.fs = fs
        self.n = n
        self.nsteps = nsteps

    def close(self):
        if getattr(self, "_h", None):
            lib().bfg_particles_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def completeLoop(self, dt):
        check(lib().bfg_particles_complete_loop(self._h, float(dt)), self.fs.handle)

    def sample_velocity(self):
        out = np.empty((self.n, 3))
        check(lib().bfg_particles_sample_velocity(self._h, ptr(out)), self.fs.handle)
        return out

    def sample_acceleration(self):
        """Lagrangian acceleration of the current state at the tracers
        (NSVEparticles::do_stats, NSVEparticles.cpp:84-91), (n, 3)."""
        out = np.empty((self.n, 3))
        check(lib().bfg_particles_sample_acceleration(self._h, ptr(out)), self.fs.handle)
        return out

    def state(self):
        pos = np.empty((self.n, 3))
        rhs = np.empty((self.nsteps, self.n, 3))
        idx = np.empty(self.n, np.int64)
        check(lib().bfg_particles_download(self._h, ptr(pos), ptr(rhs),
                                           ptr(idx, ctypes.c_int64)), self.fs.handle)
        return pos, rhs, idx

    @property
    def step_idx(self):
        s = ctypes.c_int()
        check(lib().bfg_particles_info(self._h, None, None, ctypes.byref(s)), self.fs.handle)
        return s.value


def NSVEparticles_step(fs, ps, dt, nsteps=1):
    """NSVEparticles::step (NSVEparticles.cpp:33-41), nsteps times."""
    check(lib().bfg_nsveparticles_step(fs.handle, ps.handle if ps is not None else None,
                                       float(dt), int(nsteps)), fs.handle)


class ensemble:
    """Batched form: many contexts advanced together (bfg_ens_*).

    Members of equal grid size share one launch per pass and RK stage; the
    result of every member is the same as stepping it alone.
    """

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        check(lib().bfg_ens_create(ctypes.byref(h), device))
        self._h = h
        _live["ensemble"].add(self)
        self.members = []

    def _check(self, rc):
        if rc != 0:
            raise _lib.BfgError(rc, lib().bfg_ens_last_error(self._h).decode())

    def add(self, fs, dt, tracers=None):
        self._check(lib().bfg_ens_add(self._h, fs.handle,
                                      tracers.handle if tracers is not None else None, float(dt)))
        self.members.append((fs, tracers, dt))

    def remove(self, fs):
        self._check(lib().bfg_ens_remove(self._h, fs.handle))
        self.members = [m for m in self.members if m[0] is not fs]

    def step(self, nsteps=1):
        self._check(lib().bfg_ens_step(self._h, int(nsteps)))

    def last_ms(self):
        ms = ctypes.c_double()
        self._check(lib().bfg_ens_last_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def use_graphs(self, enable):
        self._check(lib().bfg_ens_use_graphs(self._h, int(bool(enable))))

    def autotune(self, reps=3):
        """bfg_ens_autotune: both column-pass schedules timed on every size
        group as step() launches it.  Returns {N: {pass: (schedule, ms0,
        ms1)}}.  The members' velocity fields are used as work space."""
        self._check(lib().bfg_ens_autotune(self._h, int(reps)))
        groups = {}
        for fs, _, _ in self.members:
            groups.setdefault(fs.nx, []).append(fs)
        return {n: fss[0].schedules(members=len(fss)) for n, fss in groups.items()}

    def wait(self, timeout_s=None):
        """True once the last step() call's work has finished; False if it
        is still running after timeout_s seconds (None: wait until done)."""
        done = ctypes.c_int()
        t = 1e300 if timeout_s is None else max(0.0, timeout_s * 1e3)
        self._check(lib().bfg_ens_wait(self._h, t, ctypes.byref(done)))
        return bool(done.value)

    def kernel_launches(self):
        """Kernels launched by step() so far (graph nodes included)."""
        n = ctypes.c_int64()
        self._check(lib().bfg_ens_kernel_launches(self._h, ctypes.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "_h", None):
            lib().bfg_ens_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
