"""Seeded synthetic initial conditions in the reference checkpoint layout.

Velocity: complex Gaussian modes on the half spectrum (numpy PCG64,
``default_rng(seed)``), projected divergence-free, scaled so that the shell
energy follows E(k) ~ k^4 exp(-2 (k/k0)^2), truncated to 0 < k^2 <= kM^2,
made Hermitian on the kx = 0 plane with the reference's symmetrize rule
(bfps/cpp/field.cpp:903-978) and normalised to energy
0.5 = sum_k w |u_k|^2 / 2, w = 1 on kx = 0 and 2 elsewhere (the NXMODES
weights of bfps/cpp/kspace.hpp:162-192).  The returned field is the
vorticity w = i k x u (vorticity_equation::compute_vorticity,
vorticity_equation.cpp:171-204), shape (ny, nz, nx/2+1, 3) -- the layout of
``vorticity/complex/<iteration>`` in a bfps checkpoint.

Tracers: uniform in [0, 2 pi / dk)^3 from ``default_rng(seed + 1)``, shape
(n, 3), with a zero rhs history.
"""
import math

import numpy as np

TWO_THIRDS = 0
SMOOTH = 1


def _kM(n, dealias_type, dk=1.0):
    # kspace.cpp:75-100 on a cubic grid
    if dealias_type == TWO_THIRDS:
        return dk * max((2 * (n // 2)) // 3 - 1, n // 3 - 1)
    return dk * (n // 2 - 1)


def _wavenumbers(n, dk=1.0):
    kx = np.arange(n // 2 + 1) * dk
    kk = np.array([i if i <= n // 2 else i - n for i in range(n)], dtype=np.float64) * dk
    KX = kx[None, None, :]
    KY = kk[:, None, None]
    KZ = kk[None, :, None]
    return KX, KY, KZ


def _symmetrize(a):
    n = a.shape[0]
    a[0, 0, 0, :] = a[0, 0, 0, :].real
    for ii in range(1, n // 2):
        a[0, n - ii, 0, :] = np.conj(a[0, ii, 0, :])
    for yy in range(1, n // 2):
        buf = a[yy, :, 0, :].copy()
        for ii in range(1, n):
            a[n - yy, ii, 0, :] = np.conj(buf[n - ii])
        a[n - yy, 0, 0, :] = np.conj(buf[0])
    return a


def vorticity_ic(n, seed=0, k0=3.0, energy=0.5, dealias_type=SMOOTH, dk=1.0,
                 dtype=np.complex128, return_velocity=False):
    rng = np.random.default_rng(seed)
    shape = (n, n, n // 2 + 1, 3)
    u = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    KX, KY, KZ = _wavenumbers(n, dk)
    K2 = (KX * KX + KY * KY) + KZ * KZ
    kM = _kM(n, dealias_type, dk)
    keep = (K2 > 0) & (K2 <= kM * kM)
    safe = np.where(K2 > 0, K2, 1.0)
    div = (KX * u[..., 0] + KY * u[..., 1] + KZ * u[..., 2]) / safe
    u[..., 0] -= div * KX
    u[..., 1] -= div * KY
    u[..., 2] -= div * KZ
    u[~keep] = 0
    w = np.where(KX == 0, 1.0, 2.0) * np.ones_like(K2)
    kn = np.sqrt(K2)
    shell = (kn / dk).astype(np.int64)
    e_mode = 0.5 * w * np.sum(np.abs(u) ** 2, axis=-1)
    e_shell = np.bincount(shell[keep], weights=e_mode[keep], minlength=shell.max() + 1)
    target = kn ** 4 * np.exp(-2.0 * (kn / k0) ** 2) * dk
    scale = np.zeros_like(K2)
    es = e_shell[shell]
    ok = keep & (es > 0)
    scale[ok] = np.sqrt(target[ok] / es[ok])
    u *= scale[..., None]
    _symmetrize(u)
    e = 0.5 * np.sum(w[..., None] * np.abs(u) ** 2)
    u *= math.sqrt(energy / e)
    # omega = i k x u for k^2 <= kM^2 (compute_vorticity), then symmetrize
    om = np.empty_like(u)
    om[..., 0] = 1j * (KY * u[..., 2] - KZ * u[..., 1])
    om[..., 1] = 1j * (KZ * u[..., 0] - KX * u[..., 2])
    om[..., 2] = 1j * (KX * u[..., 1] - KY * u[..., 0])
    om[~(K2 <= kM * kM)] = 0
    _symmetrize(om)
    if return_velocity:
        return om.astype(dtype), u.astype(dtype)
    return om.astype(dtype)


def tracer_ic(npart, seed=0, dk=1.0):
    rng = np.random.default_rng(seed + 1)
    return rng.random((npart, 3)) * (2 * np.pi / dk)


def cfl_dt(u_real_max, n, cfl=0.5, dk=1.0):
    """dt = cfl * dx / max|u| (fixed per instance; AB needs a constant dt)."""
    return cfl * (2 * np.pi / dk / n) / u_real_max
