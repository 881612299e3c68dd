"""The oracle's compute_pressure / compute_Lagrangian_acceleration pinned by
an exact solution: for the Taylor-Green flow u = (sin x cos y, -cos x sin y, 0)
the pressure of -lap p = d_i d_j (u_i u_j) is (cos 2x + cos 2y) / 4, and the
Lagrangian acceleration of this steady Euler flow (nu = 0, no forcing) is
-grad p."""
import numpy as np

from oracle import nsve as O


def _taylor_green(n):
    x = 2 * np.pi * np.arange(n) / n
    z, y, xx = np.meshgrid(x, x, x, indexing="ij")  # real layout [z][y][x]
    u = np.zeros((n, n, n, 3))
    u[..., 0] = np.sin(xx) * np.cos(y)
    u[..., 1] = -np.cos(xx) * np.sin(y)
    return u, xx, y


def test_pressure_of_taylor_green():
    n = 16
    ve = O.VorticityEquation(n)
    u, xx, y = _taylor_green(n)
    p = ve.ift(ve.compute_pressure(u)[..., None])[..., 0]
    want = (np.cos(2 * xx) + np.cos(2 * y)) / 4
    assert np.abs(p - want).max() < 1e-13


def test_acceleration_of_taylor_green_is_minus_grad_p():
    n = 16
    ve = O.VorticityEquation(n)
    ve.nu = 0.0
    u, xx, y = _taylor_green(n)
    uh = ve.dft(u) / n ** 3                    # u = ift(u^), unnormalised inverse
    ve.cvorticity = ve.compute_vorticity(uh)
    a = ve.ift(ve.compute_lagrangian_acceleration())
    # p = (cos 2x + cos 2y)/4  ->  -grad p = (sin 2x / 2, sin 2y / 2, 0)
    assert np.abs(a[..., 0] - np.sin(2 * xx) / 2).max() < 1e-12
    assert np.abs(a[..., 1] - np.sin(2 * y) / 2).max() < 1e-12
    assert np.abs(a[..., 2]).max() < 1e-12
