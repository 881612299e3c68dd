"""ctypes binding of include/bfps_b200.h.

The CUDA library is the only implementation of the solver: there is no CPU
fallback, and loading fails loudly if the library has not been built.
"""
import ctypes
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libbfps_b200.so")
HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "bfps_b200.h")

BFG_OK = 0
BFG_EINVAL = -1
BFG_ECUDA = -2
BFG_ENOMEM = -3
BFG_EUNSUP = -4
BFG_ESTATE = -5
TWO_THIRDS = 0
SMOOTH = 1
FORCING = {"none": 0, "linear": 1, "Kolmogorov": 2}
FIELD_VORTICITY = 0
FIELD_VELOCITY = 1
FIELD_RVELOCITY = 2
KINDS = ["IZ", "IY", "X", "FY", "FZ", "kspace", "tracers", "stats"]

_c = ctypes
_vp = _c.c_void_p
_i = _c.c_int
_d = _c.c_double
_i64 = _c.c_int64
_pd = _c.POINTER(_c.c_double)
_pi64 = _c.POINTER(_c.c_int64)

# name -> (restype, argtypes)
SIGNATURES = {
    "bfg_version": (_c.c_char_p, []),
    "bfg_ctx_create": (_i, [_c.POINTER(_vp), _i, _i, _i, _d, _d, _d, _i, _i, _i]),
    "bfg_ctx_destroy": (None, [_vp]),
    "bfg_last_error": (_c.c_char_p, [_vp]),
    "bfg_set_physics": (_i, [_vp, _d, _i, _d, _d, _d, _i]),
    "bfg_kspace_info": (_i, [_vp, _pd, _pd, _c.POINTER(_i), _pd, _pi64]),
    "bfg_field_upload": (_i, [_vp, _i, _vp]),
    "bfg_field_download": (_i, [_vp, _i, _vp]),
    "bfg_read_checkpoint_fixup": (_i, [_vp]),
    "bfg_step": (_i, [_vp, _d, _i]),
    "bfg_compute_velocity": (_i, [_vp]),
    "bfg_compute_pressure": (_i, [_vp, _vp]),
    "bfg_lagrangian_acceleration": (_i, [_vp, _vp]),
    "bfg_velocity_rspace": (_i, [_vp]),
    "bfg_ift": (_i, [_vp, _vp, _vp]),
    "bfg_dft": (_i, [_vp, _vp, _vp]),
    "bfg_get_iteration": (_i, [_vp, _c.POINTER(_i)]),
    "bfg_set_iteration": (_i, [_vp, _i]),
    "bfg_stats": (_i, [_vp, _d, _d, _i, _pd, _pd, _pd, _pd, _pi64, _pi64]),
    "bfg_particles_create": (_i, [_vp, _c.POINTER(_vp), _i64, _i, _i, _i, _pd, _pd, _pi64, _i]),
    "bfg_particles_destroy": (None, [_vp]),
    "bfg_particles_complete_loop": (_i, [_vp, _d]),
    "bfg_nsveparticles_step": (_i, [_vp, _vp, _d, _i]),
    "bfg_particles_sample_velocity": (_i, [_vp, _pd]),
    "bfg_particles_sample_acceleration": (_i, [_vp, _pd]),
    "bfg_particles_download": (_i, [_vp, _pd, _pd, _pi64]),
    "bfg_particles_upload": (_i, [_vp, _pd, _pd, _i]),
    "bfg_profile": (_i, [_vp, _i]),
    "bfg_profile_read": (_i, [_vp, _i, _pd, _c.POINTER(_i64)]),
    "bfg_particles_info": (_i, [_vp, _c.POINTER(_i64), _c.POINTER(_i), _c.POINTER(_i)]),
    "bfg_last_step_ms": (_i, [_vp, _pd]),
    "bfg_kernel_launches": (_i, [_vp, _c.POINTER(_i64)]),
    "bfg_rspace_stats_noalloc": (_i, [_vp, _i, _i, _i, _i, _d, _i, _vp, _vp, _vp]),
    "bfg_check_finite": (_i, [_vp, _i, _c.POINTER(_i64)]),
    "bfg_field_ift": (_i, [_vp, _i]),
    "bfg_autotune": (_i, [_vp, _i]),
    "bfg_ens_autotune": (_i, [_vp, _i]),
    "bfg_selftest_wait": (_i, [_vp]),
    "bfg_ctx_reset": (_i, [_vp]),
    "bfg_tune_get": (_i, [_vp, _i, _i, _c.POINTER(_i), _pd, _pd]),
    "bfg_tune_set": (_i, [_vp, _i, _i, _i]),
    "bfg_field_stats": (_i, [_vp, _vp, _d, _i, _pd, _pd, _pi64]),
    "bfg_ens_create": (_i, [_c.POINTER(_vp), _i]),
    "bfg_ens_destroy": (None, [_vp]),
    "bfg_ens_last_error": (_c.c_char_p, [_vp]),
    "bfg_ens_add": (_i, [_vp, _vp, _vp, _d]),
    "bfg_ens_remove": (_i, [_vp, _vp]),
    "bfg_ens_count": (_i, [_vp, _c.POINTER(_i)]),
    "bfg_ens_step": (_i, [_vp, _i]),
    "bfg_ens_last_ms": (_i, [_vp, _pd]),
    "bfg_ens_use_graphs": (_i, [_vp, _i]),
    "bfg_ens_kernel_launches": (_i, [_vp, _c.POINTER(_i64)]),
    "bfg_ens_wait": (_i, [_vp, _c.c_double, _c.POINTER(_c.c_int)]),
}

_LIB = None


class BfgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("bfps_b200 error %d: %s" % (code, msg))
        self.code = code


def lib():
    """Load the CUDA engine (raises if it is missing)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("bfps_b200 CUDA library not built (%s); run "
                               "python -m bfps_b200.build" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(rc, ctx=None):
    if rc != 0:
        msg = ""
        if ctx:
            m = lib().bfg_last_error(ctx)
            msg = m.decode() if m else ""
        raise BfgError(rc, msg or "error code %d" % rc)
    return rc


def ptr(a, ctype=ctypes.c_double):
    """ctypes pointer to a contiguous numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))
