"""1024^3 FP32, the largest grid the C-ABI accepts (about 78 GB per
instance), through size-independent properties: the oracle cannot run a
1024^3 step in test time, so these check

* field::dft / field::ift: ift(dft(r)) = N^3 r for a random real field
  (device buffers, compared on the device);
* the whole IF-RK3 step on an ABC Beltrami field (u x w = 0): with forcing
  off, w(t) = w(0) exp(-nu k^2 t) exactly, so two steps at the C3 viscosity
  and time step must scale every mode by that factor and create no other
  mode (vorticity_equation.cpp:358-439);
* one full step with the nonlinear term and linear forcing on a field
  band-limited to |k_i| <= 4, against one step of the FP64 oracle at 128^3
  from the same modes: every product the step forms has modes below 64, so
  128^3 resolves it without aliasing, and the smooth filter at the modes
  that carry weight differs from 1 by less than 1e-8 on either grid.

Both skip where the GPU has less free memory than they need."""
import numpy as np
import pytest

from oracle import nsve as O

pytestmark = pytest.mark.gpu
N = 1024


def _free_gb():
    import torch
    free, _ = torch.cuda.mem_get_info()
    return free / 1e9


def test_dft_ift_round_trip_1024():
    import torch
    from bfps_b200 import _lib
    from bfps_b200.solver import vorticity_equation
    if _free_gb() < 125:
        pytest.skip("needs about 120 GB of free device memory")
    ve = vorticity_equation(N, precision="single")
    try:
        g = torch.Generator(device="cuda").manual_seed(1024)
        r = torch.zeros(ve.rshape, dtype=torch.float32, device="cuda")
        r[:, :, :N, :] = torch.randn((N, N, N, 3), generator=g, device="cuda")
        c = torch.zeros(ve.cshape, dtype=torch.complex64, device="cuda")
        _lib.check(_lib.lib().bfg_dft(ve.handle, r.data_ptr(), c.data_ptr()), ve.handle)
        # the mean of each component is the kx = ky = kz = 0 mode
        mean = r[:, :, :N, :].double().sum(dim=(0, 1, 2))
        assert torch.allclose(c[0, 0, 0].real.double(), mean, rtol=1e-4, atol=1e-2 * N ** 1.5)
        back = torch.zeros_like(r)
        _lib.check(_lib.lib().bfg_ift(ve.handle, c.data_ptr(), back.data_ptr()), ve.handle)
        del c
        assert torch.count_nonzero(back[:, :, N:, :]).item() == 0
        back = back[:, :, :N, :]
        back.div_(float(N) ** 3)
        back.sub_(r[:, :, :N, :])
        err = back.abs().max().item() / r.abs().max().item()
        assert err < 1e-5, err
    finally:
        ve.close()
        torch.cuda.empty_cache()


def test_beltrami_two_steps_1024():
    from bfps_b200.solver import vorticity_equation
    if _free_gb() < 85:
        pytest.skip("needs about 80 GB of free device memory")
    k = 2.0
    # exact Fourier coefficients of the ABC field's vorticity: the normalised
    # DFT of its samples on any grid finer than 2k + 1 points
    n0 = 16
    x = np.arange(n0) * 2 * np.pi / n0
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    u = np.stack([np.sin(k * Z) + np.cos(k * Y), np.sin(k * X) + np.cos(k * Z),
                  np.sin(k * Y) + np.cos(k * X)], axis=-1)
    w16 = O.dft(k * u) / n0 ** 3          # (ky, kz, kx, 3), curl u = k u
    idx = np.argwhere(np.abs(w16).max(axis=-1) > 1e-12)

    def wrap(i):
        return i if i <= n0 // 2 else i - n0

    ve = vorticity_equation(N, precision="single")
    try:
        ve.nu, ve.forcing_type = 0.002, "none"
        w = np.zeros(ve.cshape, np.complex64)
        modes = [(wrap(a) % N, wrap(b) % N, c) for a, b, c in idx]
        for (a, b, c), (a0, b0, c0) in zip(modes, idx):
            w[a, b, c] = w16[a0, b0, c0]
        ve.set_cvorticity(w)
        dt, nsteps = 0.001, 2
        ve.step(dt, nsteps)
        got = ve.get_cvorticity()
        f = np.exp(-ve.nu * k * k * dt * nsteps)
        scale = np.abs(w16).max()
        for (a, b, c), (a0, b0, c0) in zip(modes, idx):
            d = np.abs(got[a, b, c] - w16[a0, b0, c0] * f).max()
            assert d < 1e-5 * scale, ((a, b, c), d)
            got[a, b, c] = 0
        # no other mode appears
        assert np.abs(got).max() < 1e-5 * scale
    finally:
        ve.close()


def test_step_1024_matches_fp64_oracle_on_band_limited_field():
    from oracle import fast as F
    from bfps_b200.solver import vorticity_equation
    if _free_gb() < 85:
        pytest.skip("needs about 80 GB of free device memory")
    # w^ = i k x A^ of a random real field A on a 9^3 grid: modes |k_i| <= 4,
    # Hermitian, divergence-free
    n0 = 9
    A = np.random.default_rng(1024).standard_normal((n0, n0, n0, 3))
    a = O.dft(A) / n0 ** 3                 # (ky, kz, kx, 3)
    ky = np.fft.fftfreq(n0, 1.0 / n0)[:, None, None]
    kz = np.fft.fftfreq(n0, 1.0 / n0)[None, :, None]
    kx = np.arange(n0 // 2 + 1)[None, None, :]
    w9 = np.stack([1j * (ky * a[..., 2] - kz * a[..., 1]),
                   1j * (kz * a[..., 0] - kx * a[..., 2]),
                   1j * (kx * a[..., 1] - ky * a[..., 0])], axis=-1)
    # |w| <= 3.7 in real space: |u| dt / dx stays below 0.35 at 1024^3
    w9 *= 0.1 / np.abs(w9).max()

    def embed(n, dtype):
        w = np.zeros((n, n, n // 2 + 1, 3), dtype)
        for i in range(n0):
            for j in range(n0):
                w[int(ky[i, 0, 0]) % n, int(kz[0, j, 0]) % n, :n0 // 2 + 1] = w9[i, j]
        return w

    physics = dict(nu=0.01, forcing_type="linear", famplitude=0.5, fk0=1.5, fk1=3.0)
    dt = 1e-3
    ref = F.VorticityEquation(128)
    for k, v in physics.items():
        setattr(ref, k, v)
    w0 = embed(128, np.complex128)
    ref.cvorticity = w0
    ref.step(dt)
    want = ref.cvorticity
    ref.close()

    ve = vorticity_equation(N, precision="single")
    try:
        for k, v in physics.items():
            setattr(ve, k, v)
        ve.set_cvorticity(embed(N, np.complex64))
        ve.step(dt, 1)
        got = ve.get_cvorticity()
    finally:
        ve.close()
    scale = np.abs(want).max()
    # the modes |k_i| <= 32 of both grids, where the step can put weight
    sel = np.r_[0:33, -32:0]
    g = got[sel][:, sel][:, :, :33]
    r = want[sel][:, sel][:, :, :33]
    assert np.abs(g - r).max() < 1e-5 * scale, np.abs(g - r).max() / scale
    # the change over the step (viscosity, forcing and the nonlinear term,
    # about 6e-4 of the field) to 5e-3 of its own size
    d0 = w0[sel][:, sel][:, :, :33]
    inc = np.abs(r - d0).max()
    assert np.abs((g - d0) - (r - d0)).max() < 5e-3 * inc
    got[sel[:, None], sel[None, :], :33] = 0
    assert np.abs(got).max() < 1e-5 * scale
