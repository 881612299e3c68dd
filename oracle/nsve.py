"""Oracle: CPU restatement of bfps' vorticity-equation DNS step.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the ``cpu_baseline`` leg of bench.py, as the checker.  The product
(the CUDA library behind include/bfps_b200.h) never calls it.

Parity is pinned against the reference's golden end-to-end fixture
(bfps/test/B32p1e4_checkpoint_0.h5 with bfps/test/test_bfps_NSVEparticles.py)
through tests/test_oracle_golden.py.

Everything follows the reference line by line; citations are
``file:line`` inside the bfps checkout:

* layouts (bfps/cpp/field.cpp:85-101): real data is ``[z][y][x][c]``
  (the in-place buffer pads x to nx+2), complex data is the FFTW-MPI
  transposed-out layout ``[ky][kz][kx][c]`` with kx in 0..nx/2.
* transforms (field.cpp:144-162): unnormalised C2R / R2C.
* wavenumber tables, kM, shells and the smooth filter (kspace.cpp:34-167).
* dealias / low_pass / force_divfree / cospectrum (kspace.cpp:235-253,
  461-598).
* compute_velocity, add_forcing, omega_nonlin, IF-RK3 step
  (vorticity_equation.cpp:206-439); compute_pressure and
  compute_Lagrangian_acceleration (vorticity_equation.cpp:441-578).
* symmetrize (field.cpp:903-978), impose_zero_mode (field.hpp:226-233).
* real-space moments and histograms (field.cpp:661-889) and
  compute_stats (field.cpp:984-1040).

Arithmetic is float64 throughout, with an optional float32 storage mode
(``rdtype=np.float32``) that rounds every stored field to float32 the way a
``--precision single`` build stores them (the FFTs themselves stay float64).
"""
import math
import numpy as np

TWO_THIRDS = 0
SMOOTH = 1

try:  # multi-threaded pocketfft when available (only used as a speed-up)
    import scipy.fft as _sfft

    def _rfftn(a, axes, workers):
        return _sfft.rfftn(a, axes=axes, workers=workers)

    def _irfftn(a, s, axes, workers):
        return _sfft.irfftn(a, s=s, axes=axes, norm="forward", workers=workers)
except Exception:  # pragma: no cover - numpy fallback for the checker
    def _rfftn(a, axes, workers):
        return np.fft.rfftn(a, axes=axes)

    def _irfftn(a, s, axes, workers):
        return np.fft.irfftn(a, s=s, axes=axes, norm="forward")


class KSpace:
    """Wavenumber tables of bfps' ``kspace<FFTW, dt>`` (kspace.cpp:34-167)."""

    def __init__(self, nx, ny, nz, dkx=1.0, dky=1.0, dkz=1.0, dealias_type=SMOOTH):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dkx, self.dky, self.dkz = float(dkx), float(dky), float(dkz)
        self.dealias_type = dealias_type
        # clayout sizes are (ny, nz, nx/2+1) (field.cpp:98-100)
        s0, s1, s2 = ny, nz, nx // 2 + 1
        self.kx = np.arange(s2, dtype=np.float64) * self.dkx
        # kspace.cpp:60-74: ky wraps at sizes[1]/2, kz at sizes[0]/2
        self.ky = np.array([self.dky * i if i <= s1 // 2 else self.dky * (i - s1)
                            for i in range(s0)], dtype=np.float64)
        self.kz = np.array([self.dkz * i if i <= s0 // 2 else self.dkz * (i - s0)
                            for i in range(s1)], dtype=np.float64)
        if dealias_type == TWO_THIRDS:  # kspace.cpp:78-82
            kMx = self.dkx * (int(2 * (s2 - 1) // 3) - 1)
            kMy = self.dky * (s0 // 3 - 1)
            kMz = self.dkz * (s1 // 3 - 1)
        else:  # SMOOTH, kspace.cpp:83-87
            kMx = self.dkx * (s2 - 2)
            kMy = self.dky * (s0 // 2 - 1)
            kMz = self.dkz * (s1 // 2 - 1)
        self.kM = max(kMx, kMy, kMz)
        self.kM2 = self.kM * self.kM
        self.dk = min(self.dkx, self.dky, self.dkz)
        self.dk2 = self.dk * self.dk
        self.nshells = int(self.kM / self.dk) + 2
        KX = self.kx[None, None, :]
        KY = self.ky[:, None, None]
        KZ = self.kz[None, :, None]
        self.KX = np.broadcast_to(KX, (s0, s1, s2))
        self.KY = np.broadcast_to(KY, (s0, s1, s2))
        self.KZ = np.broadcast_to(KZ, (s0, s1, s2))
        # CLOOP_K2 order of summation: kx*kx + ky*ky + kz*kz (kspace.hpp:146-148)
        self.K2 = (KX * KX + KY * KY) + KZ * KZ
        self.nxmodes = np.where(np.arange(s2) == 0, 1, 2)[None, None, :] * np.ones((s0, s1, 1))
        # shells (kspace.cpp:109-150): strict k2 < kM2
        k2 = self.K2
        inside = k2 < self.kM2
        knorm = np.sqrt(k2)
        idx = (knorm / self.dk).astype(np.int64)
        self.nshell = np.bincount(idx[inside], weights=self.nxmodes[inside],
                                  minlength=self.nshells)[:self.nshells].astype(np.int64)
        ks = np.bincount(idx[inside], weights=(self.nxmodes * knorm)[inside],
                         minlength=self.nshells)[:self.nshells]
        self.kshell = np.where(self.nshell != 0, ks / np.maximum(self.nshell, 1), 0.0)
        if dealias_type == SMOOTH:
            # the reference keeps one filter value per key round(k2/dk2)
            # (kspace.cpp:119-150); where several k2 share a key (incommensurate
            # dk per axis) the entry written last in CLOOP order (y, z, x;
            # kspace.hpp:117-192) wins, as with one OpenMP thread.  Every mode
            # is then multiplied by the entry of its own key (kspace.cpp:479).
            keys = np.rint(k2 / self.dk2).astype(np.int64)  # round half to even
            # round() of the reference rounds halves away from zero
            half = np.abs(k2 / self.dk2 - np.floor(k2 / self.dk2) - 0.5) == 0
            keys = np.where(half, np.floor(k2 / self.dk2).astype(np.int64) + 1, keys)
            vals = np.exp(-36.0 * np.power(k2 / self.kM2, 18.0))
            flat_k = keys.reshape(-1)   # C order = CLOOP order (y, z, x)
            flat_v = vals.reshape(-1)
            table = np.zeros(int(flat_k.max()) + 1)
            # last occurrence of each key in CLOOP order
            rev = flat_k[::-1]
            uk, first_in_rev = np.unique(rev, return_index=True)
            table[uk] = flat_v[::-1][first_in_rev]
            self.filter_table = table
            self.filter = table[keys]
        else:
            self.filter = None
            self.filter_table = None

    # -- pointwise k-space operations ------------------------------------
    def dealias(self, a):
        """kspace.cpp:461-485 (in place)."""
        if self.dealias_type == TWO_THIRDS:
            self.low_pass(a, self.kM)
        else:
            a *= self.filter[..., None]
        return a

    def low_pass(self, a, kmax):
        """kspace.cpp:235-253: zero every mode with k2 >= kmax^2."""
        a[self.K2 >= kmax * kmax] = 0
        return a

    def force_divfree(self, a):
        """kspace.cpp:487-519 (in place), then zero the k=0 mode."""
        k2 = self.K2
        nz_ = k2 > 0
        safe = np.where(nz_, k2, 1.0)
        tval = (self.KX * a[..., 0] + self.KY * a[..., 1] + self.KZ * a[..., 2]) / safe
        tval = np.where(nz_, tval, 0)
        tval = tval.astype(a.dtype)  # stored as rnumber complex in the reference
        a[..., 0] -= tval * self.KX
        a[..., 1] -= tval * self.KY
        a[..., 2] -= tval * self.KZ
        a[0, 0, 0, :] = 0
        return a

    def cospectrum(self, a, b):
        """kspace.cpp:521-598: (nshells, 3, 3) float64 co-spectrum."""
        k2 = self.K2
        m = k2 <= self.kM2
        idx = (np.sqrt(k2[m]) / self.dk).astype(np.int64)
        w = self.nxmodes[m]
        aa = a[m].astype(np.complex128)
        bb = b[m].astype(np.complex128)
        out = np.zeros((self.nshells, 3, 3))
        for i in range(3):
            for j in range(3):
                v = w * (aa[:, i].real * bb[:, j].real + aa[:, i].imag * bb[:, j].imag)
                out[:, i, j] = np.bincount(idx, weights=v, minlength=self.nshells)[:self.nshells]
        return out


def symmetrize(a):
    """field.cpp:903-978 on a (ny, nz, nx/2+1, ncomp) complex array (in place)."""
    ny, nz = a.shape[0], a.shape[1]
    a[0, 0, 0, :] = a[0, 0, 0, :].real
    for ii in range(1, nz // 2):
        a[0, nz - ii, 0, :] = np.conj(a[0, ii, 0, :])
    for yy in range(1, ny // 2):
        buf = a[yy, :, 0, :].copy()
        for ii in range(1, nz):
            a[ny - yy, ii, 0, :] = np.conj(buf[nz - ii])
        a[ny - yy, 0, 0, :] = np.conj(buf[0])
    return a


def impose_zero_mode(a):
    """field.hpp:226-233."""
    a[0, 0, 0, :] = 0
    return a


def ift(c, nx, ny, nz, workers=1):
    """Unnormalised C2R of transposed-layout data -> real (nz, ny, nx, ncomp)."""
    ct = np.ascontiguousarray(np.swapaxes(c, 0, 1))  # -> [kz][ky][kx][c]
    return _irfftn(ct, s=(nz, ny, nx), axes=(0, 1, 2), workers=workers)


def dft(r, workers=1):
    """Unnormalised R2C of real (nz, ny, nx, ncomp) -> transposed [ky][kz][kx][c]."""
    c = _rfftn(r, axes=(0, 1, 2), workers=workers)
    return np.ascontiguousarray(np.swapaxes(c, 0, 1))


def real_to_padded(r):
    """(nz, ny, nx, c) -> reference in-place layout (nz, ny, nx+2, c)."""
    nz, ny, nx, nc = r.shape
    out = np.zeros((nz, ny, nx + 2, nc), dtype=r.dtype)
    out[:, :, :nx] = r
    return out


class VorticityEquation:
    """Restatement of ``vorticity_equation<rnumber, FFTW>`` (SMOOTH by default).

    ``cvorticity`` is the state in the transposed complex layout
    ``(ny, nz, nx/2+1, 3)``.
    """

    def __init__(self, nx, ny=None, nz=None, dkx=1.0, dky=1.0, dkz=1.0,
                 dealias_type=SMOOTH, rdtype=np.float64, workers=1):
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        self.nx, self.ny, self.nz = nx, ny, nz
        self.kk = KSpace(nx, ny, nz, dkx, dky, dkz, dealias_type)
        self.rdtype = np.dtype(rdtype)
        self.cdtype = np.complex64 if self.rdtype == np.float32 else np.complex128
        shape = (ny, nz, nx // 2 + 1, 3)
        self.cvorticity = np.zeros(shape, self.cdtype)
        self.v1 = np.zeros(shape, self.cdtype)
        self.v2 = np.zeros(shape, self.cdtype)
        self.npoints = nx * ny * nz
        self.workers = workers
        self.iteration = 0
        # defaults of the reference constructor (vorticity_equation.cpp:150-155)
        self.nu = 0.1
        self.fmode = 1
        self.famplitude = 1.0
        self.fk0 = 2.0
        self.fk1 = 4.0
        self.forcing_type = "none"
        knorm = np.sqrt(self.kk.K2)
        self._knorm = knorm

    # -- helpers -------------------------------------------------------------
    def _store(self, a):
        return a.astype(self.cdtype)

    def compute_velocity(self, vort):
        """vorticity_equation.cpp:206-239 (returns a new symmetrised array)."""
        kk = self.kk
        k2 = kk.K2
        m = (k2 <= kk.kM2) & (k2 > 0)
        w = vort.astype(np.complex128)
        safe = np.where(m, k2, 1.0)
        ky, kz, kx = kk.KY, kk.KZ, kk.KX
        u = np.empty(w.shape, np.complex128)
        u[..., 0] = (-(ky * w[..., 2].imag - kz * w[..., 1].imag) / safe
                     + 1j * (ky * w[..., 2].real - kz * w[..., 1].real) / safe)
        u[..., 1] = (-(kz * w[..., 0].imag - kx * w[..., 2].imag) / safe
                     + 1j * (kz * w[..., 0].real - kx * w[..., 2].real) / safe)
        u[..., 2] = (-(kx * w[..., 1].imag - ky * w[..., 0].imag) / safe
                     + 1j * (kx * w[..., 1].real - ky * w[..., 0].real) / safe)
        u[~m] = 0
        u = self._store(u)
        return symmetrize(u)

    def compute_vorticity(self, vel):
        """vorticity_equation.cpp:171-204: omega = i k x u for k2 <= kM2."""
        kk = self.kk
        m = kk.K2 <= kk.kM2
        u = vel.astype(np.complex128)
        ky, kz, kx = kk.KY, kk.KZ, kk.KX
        w = np.empty(u.shape, np.complex128)
        w[..., 0] = -(ky * u[..., 2].imag - kz * u[..., 1].imag) + 1j * (ky * u[..., 2].real - kz * u[..., 1].real)
        w[..., 1] = -(kz * u[..., 0].imag - kx * u[..., 2].imag) + 1j * (kz * u[..., 0].real - kx * u[..., 2].real)
        w[..., 2] = -(kx * u[..., 1].imag - ky * u[..., 0].imag) + 1j * (kx * u[..., 1].real - ky * u[..., 0].real)
        w[~m] = 0
        return symmetrize(self._store(w))

    def ift(self, c):
        r = ift(c.astype(np.complex128), self.nx, self.ny, self.nz, self.workers)
        return r.astype(self.rdtype)

    def dft(self, r):
        return dft(r.astype(np.float64), self.workers)

    def add_forcing(self, dst, vort, factor=1.0):
        """vorticity_equation.cpp:241-288 (dst is complex128 work array)."""
        if self.forcing_type == "none":
            return dst
        if self.forcing_type == "Kolmogorov":
            # cindex of (ky = fmode, kz = 0, kx = 0) and (ky = ny - fmode, ...)
            dst[self.fmode, 0, 0, 2] -= self.famplitude * factor / 2
            dst[self.ny - self.fmode, 0, 0, 2] -= self.famplitude * factor / 2
            return dst
        if self.forcing_type == "linear":
            band = (self.fk0 <= self._knorm) & (self.fk1 >= self._knorm)
            dst[band] += self.famplitude * vort[band].astype(np.complex128) * factor
            return dst
        raise ValueError("unknown forcing_type %r" % self.forcing_type)

    def omega_nonlin(self, src_field):
        """vorticity_equation.cpp:290-356; returns the complex nonlinear term."""
        kk = self.kk
        u = self.compute_velocity(src_field)
        ur = self.ift(u)
        wr = self.ift(src_field)
        ur64 = ur.astype(np.float64)
        wr64 = wr.astype(np.float64)
        cr = np.empty_like(ur64)
        for cc in range(3):
            c1, c2 = (cc + 1) % 3, (cc + 2) % 3
            cr[..., cc] = ur64[..., c1] * wr64[..., c2] - ur64[..., c2] * wr64[..., c1]
        cr = (cr / self.npoints).astype(self.rdtype)
        U = self._store(self.dft(cr))
        U = U.astype(np.complex128)
        kk.dealias(U)
        U = self._store(U).astype(np.complex128)
        ky, kz, kx = kk.KY, kk.KZ, kk.KX
        t = np.empty_like(U)
        t[..., 0] = -(ky * U[..., 2].imag - kz * U[..., 1].imag) + 1j * (ky * U[..., 2].real - kz * U[..., 1].real)
        t[..., 1] = -(kz * U[..., 0].imag - kx * U[..., 2].imag) + 1j * (kz * U[..., 0].real - kx * U[..., 2].real)
        t[..., 2] = -(kx * U[..., 1].imag - ky * U[..., 0].imag) + 1j * (kx * U[..., 1].real - ky * U[..., 0].real)
        t = self._store(t).astype(np.complex128)
        self.add_forcing(t, src_field, 1.0)
        t = self._store(t)
        kk.force_divfree(t)
        return t

    def step(self, dt):
        """vorticity_equation.cpp:358-439."""
        kk = self.kk
        k2 = kk.K2
        m = k2 <= kk.kM2
        mm = m[..., None]
        nu = self.nu
        v0 = self.cvorticity
        self.v1[...] = 0
        N = self.omega_nonlin(v0).astype(np.complex128)
        f0 = np.exp(-nu * k2 * dt)[..., None]
        v1 = (v0.astype(np.complex128) + dt * N) * f0
        self.v1 = self._store(np.where(mm, v1, 0))
        N = self.omega_nonlin(self.v1).astype(np.complex128)
        f0 = np.exp(-nu * k2 * dt / 2)[..., None]
        f1 = np.exp(nu * k2 * dt / 2)[..., None]
        v2 = (3 * v0.astype(np.complex128) * f0 + (self.v1.astype(np.complex128) + dt * N) * f1) * 0.25
        self.v2 = self._store(np.where(mm, v2, self.v2))
        N = self.omega_nonlin(self.v2).astype(np.complex128)
        f0 = np.exp(-nu * k2 * dt * 0.5)[..., None]
        v3 = (v0.astype(np.complex128) * f0 + 2 * (self.v2.astype(np.complex128) + dt * N)) * f0 / 3
        self.cvorticity = self._store(np.where(mm, v3, v0))
        kk.force_divfree(self.cvorticity)
        symmetrize(self.cvorticity)
        self.iteration += 1

    def compute_pressure(self, ur):
        """vorticity_equation.cpp:441-514: pressure (one complex component,
        ``(ny, nz, nx/2+1)``) from the real-space velocity ``ur``
        ((nz, ny, nx, 3), unnormalised inverse transform of u^).  The
        dealiased transforms of u_c u_c (diagonal) and u_c u_(c+1)
        (off-diagonal) are contracted with k_i k_j; p = 0 outside
        0 < k2 <= kM2; finally p /= npoints k2."""
        kk = self.kk
        u = ur.astype(np.float64)
        k2 = kk.K2
        m = (k2 <= kk.kM2) & (k2 > 0)
        kx, ky, kz = kk.KX, kk.KY, kk.KZ
        rd = self.rdtype
        # diagonal terms 11 22 33 (:451-480)
        d = np.empty_like(u)
        for cc in range(3):
            d[..., cc] = u[..., cc] * u[..., cc]
        G = self._store(self.dft(d.astype(rd))).astype(np.complex128)
        kk.dealias(G)
        G = self._store(G).astype(np.complex128)
        p = -(kx * kx * G[..., 0] + ky * ky * G[..., 1] + kz * kz * G[..., 2])
        p = np.where(m, p, 0)
        p = p.astype(self.cdtype).astype(np.complex128)
        # off-diagonal terms 12 23 31 (:481-513)
        for cc in range(3):
            d[..., cc] = u[..., cc] * u[..., (cc + 1) % 3]
        G = self._store(self.dft(d.astype(rd))).astype(np.complex128)
        kk.dealias(G)
        G = self._store(G).astype(np.complex128)
        q = p - 2 * (kx * ky * G[..., 0] + ky * kz * G[..., 1] + kz * kx * G[..., 2])
        q = q.astype(self.cdtype).astype(np.complex128)
        safe = np.where(m, k2, 1.0)
        q = q / (self.npoints * safe)
        return np.where(m, q, p).astype(self.cdtype)

    def compute_lagrangian_acceleration(self):
        """vorticity_equation.cpp:516-578: acceleration in Fourier space,
        a = -nu k2 u^ (+ famplitude u^ on the linear forcing band) - i k p^
        for k2 <= kM2, else 0; u^ from the current vorticity."""
        kk = self.kk
        u = self.compute_velocity(self.cvorticity)
        p = self.compute_pressure(self.ift(u)).astype(np.complex128)
        u = self.compute_velocity(self.cvorticity).astype(np.complex128)
        k2 = kk.K2
        m = k2 <= kk.kM2
        a = -self.nu * k2[..., None] * u
        a = a.astype(self.cdtype).astype(np.complex128)
        if self.forcing_type == "linear":
            band = m & (self.fk0 <= self._knorm) & (self.fk1 >= self._knorm)
            a[band] += self.famplitude * u[band]
            a = a.astype(self.cdtype).astype(np.complex128)
        for c, kc in enumerate((kk.KX, kk.KY, kk.KZ)):
            a[..., c] = (a[..., c].real + kc * p.imag) + 1j * (a[..., c].imag - kc * p.real)
        a[~m] = 0
        return a.astype(self.cdtype)

    def read_checkpoint_semantics(self, c):
        """What io_checkpoint(read) does to a field read from a file:
        field::io -> symmetrize (field.cpp:340), then low_pass(kM) and
        force_divfree (vorticity_equation.hpp:107-128)."""
        a = np.array(c, dtype=self.cdtype, copy=True)
        symmetrize(a)
        self.kk.low_pass(a, self.kk.kM)
        self.kk.force_divfree(a)
        return a


# -- statistics ----------------------------------------------------------
NMOMENTS = 10


def rspace_stats(r, max_estimate, nbins):
    """field.cpp:661-889 for a 3-component real field (nz, ny, nx, 3).

    ``max_estimate`` has 4 entries (3 components + magnitude).  Returns
    ``moments`` (10, 4) and ``hist`` (nbins, 4) int64.
    """
    v = r.reshape(-1, 3).astype(np.float64)
    npoints = v.shape[0]
    mag = np.sqrt((v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]) + v[:, 2] * v[:, 2])
    vals = np.concatenate([v, mag[:, None]], axis=1)
    me = np.asarray(max_estimate, dtype=np.float64)
    binsize = 2 * me / nbins
    moments = np.zeros((NMOMENTS, 4))
    # initial values: 0 for all, except the magnitude minimum (field.cpp:733-736)
    moments[0, :3] = np.minimum(0.0, vals[:, :3].min(axis=0))
    moments[0, 3] = min(me[3], mag.min())
    moments[9, :3] = np.maximum(0.0, vals[:, :3].max(axis=0))
    moments[9, 3] = max(0.0, mag.max())
    p = np.ones_like(vals)
    for n in range(1, NMOMENTS - 1):
        p = vals * p
        moments[n] = p.sum(axis=0) / npoints
    hist = np.zeros((nbins, 4), dtype=np.int64)
    for i in range(3):
        b = np.floor((vals[:, i] + me[i]) / binsize[i]).astype(np.int64)
        ok = (b >= 0) & (b < nbins)
        hist[:, i] = np.bincount(b[ok], minlength=nbins)[:nbins]
    b = np.floor(mag * 2 / binsize[3]).astype(np.int64)
    ok = (b >= 0) & (b < nbins)
    hist[:, 3] = np.bincount(b[ok], minlength=nbins)[:nbins]
    return moments, hist


def compute_stats(ve, c, max_estimate, nbins):
    """field::compute_stats (field.cpp:984-1040) for a complex 3-vector field
    in the state layout: co-spectrum, then ift and real-space stats.
    ``max_estimate`` is the scalar passed by NSVE::do_stats; the magnitude
    entry is scaled by sqrt(3) (field.cpp:1001-1004)."""
    spec = ve.kk.cospectrum(c, c)
    r = ve.ift(c)
    me = [max_estimate] * 3 + [max_estimate * math.sqrt(3)]
    moments, hist = rspace_stats(r, me, nbins)
    return spec, moments, hist


def nsve_do_stats(ve, max_velocity_estimate, max_vorticity_estimate, nbins):
    """NSVE::do_stats (bfps/cpp/full_code/NSVE.cpp:101-135)."""
    w = compute_stats(ve, ve.cvorticity, max_vorticity_estimate / math.sqrt(3), nbins)
    u = ve.compute_velocity(ve.cvorticity)
    v = compute_stats(ve, u, max_velocity_estimate / math.sqrt(3), nbins)
    return {"vorticity": w, "velocity": v}
