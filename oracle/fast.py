"""Oracle: ctypes front end of the C++/OpenMP restatement (oracle/nsve_omp.cpp).

TEST INFRASTRUCTURE AND CPU BASELINE ONLY.  Used by tests/ as the checker
at grid sizes the numpy restatement (oracle/nsve.py, oracle/particles.py) is
too slow for, and by bench.py's CPU legs as the timed CPU path.  The
product never imports it.

The classes mirror the numpy restatement's interface (``cvorticity``,
``nu``, ``forcing_type``, ``famplitude``, ``fk0``, ``fk1``, ``fmode``,
``step``; ``ParticlesSystem.complete_loop``), and
tests/test_oracle_omp.py checks them against it, so the pin of the numpy
restatement on the reference's golden fixture carries over.
"""
import ctypes
import os

import numpy as np

from . import build_omp
from .interp import beta_coefficients
from .nsve import SMOOTH

_FORCING = {"none": 0, "linear": 1, "Kolmogorov": 2}
_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build_omp.LIB
        if not os.path.exists(path):
            build_omp.build()
        L = ctypes.CDLL(path)
        vp, d, i, i64 = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int64
        P = ctypes.POINTER
        L.orc_create.restype = vp
        L.orc_create.argtypes = [i, i, i, d, d, d, i]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_physics.argtypes = [vp, d, i, d, d, d, i]
        L.orc_kinfo.argtypes = [vp, P(d), P(d), P(i), P(i)]
        L.orc_filter.argtypes = [vp, vp]
        L.orc_set_state.argtypes = [vp, vp]
        L.orc_get_state.argtypes = [vp, vp]
        L.orc_iteration.argtypes = [vp]
        L.orc_iteration.restype = i
        L.orc_step.argtypes = [vp, d]
        L.orc_velocity.argtypes = [vp, vp, vp]
        L.orc_ift.argtypes = [vp, vp, vp]
        L.orc_dft.argtypes = [vp, vp, vp]
        L.orc_particles_create.restype = vp
        L.orc_particles_create.argtypes = [vp, i64, i, i, i, vp, vp, i, vp, i]
        L.orc_particles_destroy.argtypes = [vp]
        L.orc_particles_complete_loop.argtypes = [vp, vp, d]
        L.orc_particles_get.argtypes = [vp, vp, vp, P(i)]
        L.orc_nsveparticles_step.argtypes = [vp, vp, d]
        L.orc_threads.restype = i
        L.orc_set_threads.argtypes = [i]
        _lib = L
    return _lib


def threads():
    return lib().orc_threads()


def set_threads(n):
    lib().orc_set_threads(int(n))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class VorticityEquation:
    """FP64 ``vorticity_equation`` state on the host, stepped by the C++ oracle."""

    def __init__(self, nx, ny=None, nz=None, dkx=1.0, dky=1.0, dkz=1.0, dealias_type=SMOOTH):
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        self.nx, self.ny, self.nz = nx, ny, nz
        self.shape = (ny, nz, nx // 2 + 1, 3)
        self.h = lib().orc_create(nx, ny, nz, dkx, dky, dkz, dealias_type)
        self.nu = 0.1
        self.fmode = 1
        self.famplitude = 1.0
        self.fk0 = 2.0
        self.fk1 = 4.0
        self.forcing_type = "none"

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _physics(self):
        lib().orc_set_physics(self.h, float(self.nu), _FORCING[self.forcing_type],
                              float(self.famplitude), float(self.fk0), float(self.fk1),
                              int(self.fmode))

    @property
    def cvorticity(self):
        out = np.empty(self.shape, np.complex128)
        lib().orc_get_state(self.h, _ptr(out))
        return out

    @cvorticity.setter
    def cvorticity(self, a):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        assert a.shape == self.shape
        lib().orc_set_state(self.h, _ptr(a))

    @property
    def iteration(self):
        return lib().orc_iteration(self.h)

    def kinfo(self):
        kM, dk = ctypes.c_double(), ctypes.c_double()
        ns, nf = ctypes.c_int(), ctypes.c_int()
        lib().orc_kinfo(self.h, ctypes.byref(kM), ctypes.byref(dk), ctypes.byref(ns),
                        ctypes.byref(nf))
        filt = np.empty(nf.value)
        if nf.value:
            lib().orc_filter(self.h, _ptr(filt))
        return kM.value, dk.value, ns.value, filt

    def step(self, dt):
        self._physics()
        lib().orc_step(self.h, float(dt))

    def velocity(self):
        """(u^ symmetrised, its unnormalised C2R (nz, ny, nx, 3))."""
        self._physics()
        u = np.empty(self.shape, np.complex128)
        r = np.empty((self.nz, self.ny, self.nx, 3))
        lib().orc_velocity(self.h, _ptr(u), _ptr(r))
        return u, r

    def ift(self, c):
        c = np.ascontiguousarray(c, dtype=np.complex128)
        r = np.empty((self.nz, self.ny, self.nx, 3))
        lib().orc_ift(self.h, _ptr(c), _ptr(r))
        return r

    def dft(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        c = np.empty(self.shape, np.complex128)
        lib().orc_dft(self.h, _ptr(r), _ptr(c))
        return c


def _coef_table(n, m):
    polys = beta_coefficients(n, m)
    nc = max(len(p) for p in polys)
    tab = np.zeros((len(polys), nc))
    for i, p in enumerate(polys):
        tab[i, :len(p)] = [float(v) for v in p]
    return tab


class ParticlesSystem:
    """Single-rank ``particles_system`` (global index order) on the C++ oracle."""

    def __init__(self, ve, pos, rhs, neighbours, smoothness, step_idx=1):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        self.n = pos.shape[0]
        self.nsteps = rhs.shape[0]
        self.ve = ve
        tab = _coef_table(neighbours, smoothness)
        self.h = lib().orc_particles_create(ve.h, self.n, neighbours, smoothness, self.nsteps,
                                            _ptr(pos), _ptr(rhs), int(step_idx), _ptr(tab),
                                            tab.shape[1])

    def close(self):
        if self.h:
            lib().orc_particles_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def complete_loop(self, field_r, dt):
        f = np.ascontiguousarray(field_r, dtype=np.float64)
        lib().orc_particles_complete_loop(self.h, _ptr(f), float(dt))

    def state(self):
        pos = np.empty((self.n, 3))
        rhs = np.empty((self.nsteps, self.n, 3))
        si = ctypes.c_int()
        lib().orc_particles_get(self.h, _ptr(pos), _ptr(rhs), ctypes.byref(si))
        return pos, rhs, si.value


def nsveparticles_step(ve, ps, dt):
    """NSVEparticles::step (NSVEparticles.cpp:33-41): velocity(t) -> tracers
    -> fluid IF-RK3 step."""
    ve._physics()
    lib().orc_nsveparticles_step(ve.h, ps.h if ps is not None else None, float(dt))
