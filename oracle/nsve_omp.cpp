// Oracle (C++17 + OpenMP): CPU restatement of bfps' vorticity-equation IF-RK3
// step and Lagrangian tracer step, FP64 throughout.
//
// TEST INFRASTRUCTURE AND CPU BASELINE ONLY.  Loaded by tests/ (as the
// checker at the grid sizes the numpy restatement in oracle/nsve.py is too
// slow for), by __graft_entry__.smoke() and by the cpu_baseline / reference
// legs of bench.py (as the timed CPU path).  The product (the CUDA library
// behind include/bfps_b200.h) never loads it.
//
// It restates, function by function, what oracle/nsve.py and
// oracle/particles.py restate (each of those is pinned against the
// reference's golden fixture, bfps/test/B32p1e4_checkpoint_0.h5), and
// tests/test_oracle_omp.py pins this file against them.  Citations are
// file:line inside the bfps checkout:
//   layouts           bfps/cpp/field.cpp:85-101 (real [z][y][x][c], complex
//                     transposed [ky][kz][kx][c])
//   ift / dft         field.cpp:144-162 (unnormalised C2R / R2C)
//   kspace tables     kspace.cpp:34-167 (wrap rules, kM, smooth filter keyed
//                     by round(k2/dk2), last write in CLOOP order wins,
//                     kspace.cpp:135)
//   dealias           kspace.cpp:461-485; low_pass :235-253
//   force_divfree     kspace.cpp:487-519
//   compute_velocity  vorticity_equation.cpp:206-239
//   add_forcing       vorticity_equation.cpp:241-288
//   omega_nonlin      vorticity_equation.cpp:290-356
//   step (IF-RK3)     vorticity_equation.cpp:358-439
//   symmetrize        field.cpp:903-978
//   tracers           particles_system.hpp:210-217 (completeLoop),
//                     particles_field_computer.hpp:55-183 (gather),
//                     particles_adams_bashforth.hpp:18-133 (AB1..6)
//
// FFTs are this file's own: radix-2 iterative complex transforms on
// contiguous pencil copies, twiddles from long double sin/cos rounded once.
// Expression order follows oracle/nsve.py so that the two restatements
// agree to the rounding of their FFTs (compiled with -ffp-contract=off).
#include <omp.h>

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

typedef std::complex<double> cd;

// ------------------------------------------------------------- 1D FFT --
struct Fft1 {
    int n = 1, logn = 0;
    std::vector<cd> tw;     // exp(-2 pi i m / n), m < n/2
    std::vector<int> rev;   // bit reversal
    void init(int n_) {
        n = n_;
        logn = 0;
        while ((1 << logn) < n) ++logn;
        tw.resize(n / 2 > 0 ? n / 2 : 1);
        const long double pi = 3.141592653589793238462643383279502884L;
        for (int m = 0; m < n / 2; ++m) {
            const long double a = -2.0L * pi * (long double)m / (long double)n;
            tw[m] = cd((double)cosl(a), (double)sinl(a));
        }
        rev.resize(n);
        for (int i = 0; i < n; ++i) {
            int r = 0;
            for (int b = 0; b < logn; ++b)
                if (i & (1 << b)) r |= 1 << (logn - 1 - b);
            rev[i] = r;
        }
    }
    // in place, sign -1 (forward) or +1 (inverse, unnormalised)
    void run(cd* a, bool inverse) const {
        for (int i = 0; i < n; ++i)
            if (rev[i] > i) std::swap(a[i], a[rev[i]]);
        for (int len = 2; len <= n; len <<= 1) {
            const int half = len >> 1, step = n / len;
            for (int s = 0; s < n; s += len) {
                for (int j = 0; j < half; ++j) {
                    // explicit products: std::complex's operator* carries the
                    // C99 Annex G infinity handling (a library call per product)
                    const double wr = tw[j * step].real();
                    const double wi = inverse ? -tw[j * step].imag() : tw[j * step].imag();
                    const cd u = a[s + j];
                    const cd b = a[s + j + half];
                    const cd v(b.real() * wr - b.imag() * wi, b.real() * wi + b.imag() * wr);
                    a[s + j] = cd(u.real() + v.real(), u.imag() + v.imag());
                    a[s + j + half] = cd(u.real() - v.real(), u.imag() - v.imag());
                }
            }
        }
    }
};

// block of kx columns handled together by the strided passes
constexpr int KXB = 4;

struct Ctx {
    int nx, ny, nz, nxv;
    double dkx, dky, dkz;
    int dealias;  // 0 two-thirds, 1 smooth
    double kM, kM2, dk, dk2;
    int nshells;
    std::vector<double> kx, ky, kz;
    std::vector<double> filter;  // keyed by round(k2 / dk2)
    Fft1 fx, fy, fz;
    // physics
    double nu = 0.1;
    int forcing = 0;  // 0 none, 1 linear, 2 Kolmogorov
    double famp = 1.0, fk0 = 2.0, fk1 = 4.0;
    int fmode = 1;
    int iteration = 0;
    // state and work arrays
    std::vector<cd> w0, v1, v2;  // (ny, nz, nxv, 3)
    std::vector<cd> cw;          // work (nz, ny, nxv, 3)
    std::vector<cd> ua, tb;      // complex scratch, state layout
    std::vector<double> ur, wr;  // real (nz, ny, nx, 3)

    size_t csize() const { return (size_t)ny * nz * nxv * 3; }
    size_t rsize() const { return (size_t)nz * ny * nx * 3; }
    size_t ci(int iy, int iz, int ix) const { return (((size_t)iy * nz + iz) * nxv + ix) * 3; }
    double k2_at(int iy, int iz, int ix) const {
        // CLOOP_K2 order (kspace.hpp:146-148)
        return kx[ix] * kx[ix] + ky[iy] * ky[iy] + kz[iz] * kz[iz];
    }
};

// kspace<FFTW, dt> constructor (kspace.cpp:34-167)
void kspace_init(Ctx* c) {
    const int s0 = c->ny, s1 = c->nz, s2 = c->nxv;
    c->kx.resize(s2);
    c->ky.resize(s0);
    c->kz.resize(s1);
    for (int i = 0; i < s2; ++i) c->kx[i] = (double)i * c->dkx;
    for (int i = 0; i < s0; ++i) c->ky[i] = (i <= s1 / 2) ? c->dky * i : c->dky * (i - s1);
    for (int i = 0; i < s1; ++i) c->kz[i] = (i <= s0 / 2) ? c->dkz * i : c->dkz * (i - s0);
    double kMx, kMy, kMz;
    if (c->dealias == 0) {
        kMx = c->dkx * ((2 * (s2 - 1)) / 3 - 1);
        kMy = c->dky * (s0 / 3 - 1);
        kMz = c->dkz * (s1 / 3 - 1);
    } else {
        kMx = c->dkx * (s2 - 2);
        kMy = c->dky * (s0 / 2 - 1);
        kMz = c->dkz * (s1 / 2 - 1);
    }
    c->kM = kMx;
    if (c->kM < kMy) c->kM = kMy;
    if (c->kM < kMz) c->kM = kMz;
    c->kM2 = c->kM * c->kM;
    c->dk = c->dkx;
    if (c->dk > c->dky) c->dk = c->dky;
    if (c->dk > c->dkz) c->dk = c->dkz;
    c->dk2 = c->dk * c->dk;
    c->nshells = int(c->kM / c->dk) + 2;
    c->filter.clear();
    if (c->dealias == 1) {
        // last write in CLOOP order (y, z, x) wins, as with one OpenMP thread
        for (int iy = 0; iy < s0; ++iy)
            for (int iz = 0; iz < s1; ++iz)
                for (int ix = 0; ix < s2; ++ix) {
                    const double k2 = c->k2_at(iy, iz, ix);
                    const int key = int(std::round(k2 / c->dk2));
                    if (key >= (int)c->filter.size()) c->filter.resize(key + 1, 0.0);
                    c->filter[key] = std::exp(-36.0 * std::pow(k2 / c->kM2, 18.));
                }
    }
}

// ---------------------------------------------------------- 3D FFTs --
// unnormalised C2R of a 3-component state-layout array into real (nz,ny,nx,3)
void ift3(Ctx* c, const cd* in, double* out) {
    const int nx = c->nx, ny = c->ny, nz = c->nz, nxv = c->nxv;
    cd* W = c->cw.data();
    const int nxb = (nxv + KXB - 1) / KXB;
    // kz -> z: W[z][y=ky][kx][c]
#pragma omp parallel
    {
        std::vector<cd> p((size_t)nz * KXB * 3);
#pragma omp for schedule(static)
        for (long t = 0; t < (long)ny * nxb; ++t) {
            const int iy = (int)(t / nxb), kb = (int)(t % nxb) * KXB;
            const int nk = std::min(KXB, nxv - kb);
            for (int q = 0; q < nk * 3; ++q) {
                cd* pp = p.data() + (size_t)q * nz;
                for (int iz = 0; iz < nz; ++iz) pp[iz] = in[c->ci(iy, iz, kb) + q];
                c->fz.run(pp, true);
                for (int z = 0; z < nz; ++z)
                    W[(((size_t)z * ny + iy) * nxv + kb) * 3 + q] = pp[z];
            }
        }
    }
    // ky -> y in place
#pragma omp parallel
    {
        std::vector<cd> p((size_t)ny);
#pragma omp for schedule(static)
        for (long t = 0; t < (long)nz * nxb; ++t) {
            const int z = (int)(t / nxb), kb = (int)(t % nxb) * KXB;
            const int nk = std::min(KXB, nxv - kb);
            for (int q = 0; q < nk * 3; ++q) {
                for (int y = 0; y < ny; ++y) p[y] = W[(((size_t)z * ny + y) * nxv + kb) * 3 + q];
                c->fy.run(p.data(), true);
                for (int y = 0; y < ny; ++y) W[(((size_t)z * ny + y) * nxv + kb) * 3 + q] = p[y];
            }
        }
    }
    // kx -> x: Hermitian extension, full-length inverse, real part (the
    // imaginary parts of X[0] and X[nx/2] are ignored, as FFTW's c2r does)
#pragma omp parallel
    {
        std::vector<cd> p((size_t)nx);
#pragma omp for schedule(static)
        for (long r = 0; r < (long)nz * ny; ++r) {
            const cd* row = W + (size_t)r * nxv * 3;
            for (int q = 0; q < 3; ++q) {
                p[0] = cd(row[q].real(), 0.0);
                for (int k = 1; k < nx / 2; ++k) {
                    p[k] = row[k * 3 + q];
                    p[nx - k] = std::conj(row[k * 3 + q]);
                }
                p[nx / 2] = cd(row[(nx / 2) * 3 + q].real(), 0.0);
                c->fx.run(p.data(), true);
                double* o = out + (size_t)r * nx * 3 + q;
                for (int x = 0; x < nx; ++x) o[x * 3] = p[x].real();
            }
        }
    }
}

// unnormalised R2C of real (nz,ny,nx,3) into a state-layout array
void dft3(Ctx* c, const double* in, cd* out) {
    const int nx = c->nx, ny = c->ny, nz = c->nz, nxv = c->nxv;
    cd* W = c->cw.data();
    const int nxb = (nxv + KXB - 1) / KXB;
#pragma omp parallel
    {
        std::vector<cd> p((size_t)nx);
#pragma omp for schedule(static)
        for (long r = 0; r < (long)nz * ny; ++r) {
            cd* row = W + (size_t)r * nxv * 3;
            for (int q = 0; q < 3; ++q) {
                const double* s = in + (size_t)r * nx * 3 + q;
                for (int x = 0; x < nx; ++x) p[x] = cd(s[x * 3], 0.0);
                c->fx.run(p.data(), false);
                for (int k = 0; k < nxv; ++k) row[k * 3 + q] = p[k];
            }
        }
    }
#pragma omp parallel
    {
        std::vector<cd> p((size_t)ny);
#pragma omp for schedule(static)
        for (long t = 0; t < (long)nz * nxb; ++t) {
            const int z = (int)(t / nxb), kb = (int)(t % nxb) * KXB;
            const int nk = std::min(KXB, nxv - kb);
            for (int q = 0; q < nk * 3; ++q) {
                for (int y = 0; y < ny; ++y) p[y] = W[(((size_t)z * ny + y) * nxv + kb) * 3 + q];
                c->fy.run(p.data(), false);
                for (int y = 0; y < ny; ++y) W[(((size_t)z * ny + y) * nxv + kb) * 3 + q] = p[y];
            }
        }
    }
#pragma omp parallel
    {
        std::vector<cd> p((size_t)nz);
#pragma omp for schedule(static)
        for (long t = 0; t < (long)ny * nxb; ++t) {
            const int iy = (int)(t / nxb), kb = (int)(t % nxb) * KXB;
            const int nk = std::min(KXB, nxv - kb);
            for (int q = 0; q < nk * 3; ++q) {
                for (int z = 0; z < nz; ++z) p[z] = W[(((size_t)z * ny + iy) * nxv + kb) * 3 + q];
                c->fz.run(p.data(), false);
                for (int iz = 0; iz < nz; ++iz) out[c->ci(iy, iz, kb) + q] = p[iz];
            }
        }
    }
}

// --------------------------------------------------- k-space operations --
// field::symmetrize (field.cpp:903-978), as oracle/nsve.py:symmetrize
void symmetrize(Ctx* c, cd* a) {
    const int ny = c->ny, nz = c->nz;
    for (int q = 0; q < 3; ++q) a[c->ci(0, 0, 0) + q] = cd(a[c->ci(0, 0, 0) + q].real(), 0.0);
    for (int ii = 1; ii < nz / 2; ++ii)
        for (int q = 0; q < 3; ++q) a[c->ci(0, nz - ii, 0) + q] = std::conj(a[c->ci(0, ii, 0) + q]);
    std::vector<cd> buf((size_t)nz * 3);
    for (int yy = 1; yy < ny / 2; ++yy) {
        for (int iz = 0; iz < nz; ++iz)
            for (int q = 0; q < 3; ++q) buf[iz * 3 + q] = a[c->ci(yy, iz, 0) + q];
        for (int ii = 1; ii < nz; ++ii)
            for (int q = 0; q < 3; ++q) a[c->ci(ny - yy, ii, 0) + q] = std::conj(buf[(nz - ii) * 3 + q]);
        for (int q = 0; q < 3; ++q) a[c->ci(ny - yy, 0, 0) + q] = std::conj(buf[q]);
    }
}

template <class F>
void cloop(Ctx* c, F f) {
#pragma omp parallel for schedule(static)
    for (long r = 0; r < (long)c->ny * c->nz; ++r) {
        const int iy = (int)(r / c->nz), iz = (int)(r % c->nz);
        for (int ix = 0; ix < c->nxv; ++ix) f(iy, iz, ix, c->k2_at(iy, iz, ix), c->ci(iy, iz, ix));
    }
}

// compute_velocity (vorticity_equation.cpp:206-239) into u, symmetrised
void compute_velocity(Ctx* c, const cd* w, cd* u) {
    cloop(c, [&](int iy, int iz, int ix, double k2, size_t p) {
        if (k2 <= c->kM2 && k2 > 0) {
            const double kx = c->kx[ix], ky = c->ky[iy], kz = c->kz[iz];
            const cd w0 = w[p], w1 = w[p + 1], w2 = w[p + 2];
            u[p] = cd(-(ky * w2.imag() - kz * w1.imag()) / k2, (ky * w2.real() - kz * w1.real()) / k2);
            u[p + 1] = cd(-(kz * w0.imag() - kx * w2.imag()) / k2, (kz * w0.real() - kx * w2.real()) / k2);
            u[p + 2] = cd(-(kx * w1.imag() - ky * w0.imag()) / k2, (kx * w1.real() - ky * w0.real()) / k2);
        } else {
            u[p] = u[p + 1] = u[p + 2] = cd(0.0, 0.0);
        }
    });
    symmetrize(c, u);
}

// kspace::force_divfree (kspace.cpp:487-519), then the zero mode
void force_divfree(Ctx* c, cd* a) {
    cloop(c, [&](int iy, int iz, int ix, double k2, size_t p) {
        const double kx = c->kx[ix], ky = c->ky[iy], kz = c->kz[iz];
        cd t(0.0, 0.0);
        if (k2 > 0) {
            const cd s = cd(kx * a[p].real(), kx * a[p].imag()) + cd(ky * a[p + 1].real(), ky * a[p + 1].imag());
            const cd s2 = s + cd(kz * a[p + 2].real(), kz * a[p + 2].imag());
            t = cd(s2.real() / k2, s2.imag() / k2);
        }
        a[p] = cd(a[p].real() - t.real() * kx, a[p].imag() - t.imag() * kx);
        a[p + 1] = cd(a[p + 1].real() - t.real() * ky, a[p + 1].imag() - t.imag() * ky);
        a[p + 2] = cd(a[p + 2].real() - t.real() * kz, a[p + 2].imag() - t.imag() * kz);
    });
    for (int q = 0; q < 3; ++q) a[q] = cd(0.0, 0.0);
}

// vorticity_equation::omega_nonlin (vorticity_equation.cpp:290-356) of src
// into out (state layout)
void omega_nonlin(Ctx* c, const cd* src, cd* out) {
    compute_velocity(c, src, c->ua.data());
    ift3(c, c->ua.data(), c->ur.data());
    ift3(c, src, c->wr.data());
    const double inv = (double)((size_t)c->nx * c->ny * c->nz);
    const size_t npts = (size_t)c->nx * c->ny * c->nz;
    double* ur = c->ur.data();
    const double* wr = c->wr.data();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)npts; ++i) {
        const double u0 = ur[3 * i], u1 = ur[3 * i + 1], u2 = ur[3 * i + 2];
        const double w0 = wr[3 * i], w1 = wr[3 * i + 1], w2 = wr[3 * i + 2];
        ur[3 * i] = (u1 * w2 - u2 * w1) / inv;
        ur[3 * i + 1] = (u2 * w0 - u0 * w2) / inv;
        ur[3 * i + 2] = (u0 * w1 - u1 * w0) / inv;
    }
    dft3(c, ur, out);
    cloop(c, [&](int iy, int iz, int ix, double k2, size_t p) {
        cd U[3] = {out[p], out[p + 1], out[p + 2]};
        // dealias (kspace.cpp:461-485)
        if (c->dealias == 1) {
            const double f = c->filter[int(std::round(k2 / c->dk2))];
            for (int q = 0; q < 3; ++q) U[q] = cd(U[q].real() * f, U[q].imag() * f);
        } else if (k2 >= c->kM2) {
            for (int q = 0; q < 3; ++q) U[q] = cd(0.0, 0.0);
        }
        const double kx = c->kx[ix], ky = c->ky[iy], kz = c->kz[iz];
        cd t[3];
        t[0] = cd(-(ky * U[2].imag() - kz * U[1].imag()), ky * U[2].real() - kz * U[1].real());
        t[1] = cd(-(kz * U[0].imag() - kx * U[2].imag()), kz * U[0].real() - kx * U[2].real());
        t[2] = cd(-(kx * U[1].imag() - ky * U[0].imag()), kx * U[1].real() - ky * U[0].real());
        // add_forcing, linear band (vorticity_equation.cpp:241-288)
        if (c->forcing == 1) {
            const double kn = std::sqrt(k2);
            if (c->fk0 <= kn && c->fk1 >= kn) {
                for (int q = 0; q < 3; ++q) {
                    const cd s = src[p + q];
                    t[q] += cd(c->famp * s.real() * 1.0, c->famp * s.imag() * 1.0);
                }
            }
        }
        for (int q = 0; q < 3; ++q) out[p + q] = t[q];
    });
    if (c->forcing == 2) {
        out[c->ci(c->fmode, 0, 0) + 2] -= c->famp * 1.0 / 2;
        out[c->ci(c->ny - c->fmode, 0, 0) + 2] -= c->famp * 1.0 / 2;
    }
    force_divfree(c, out);
}

// vorticity_equation::step (vorticity_equation.cpp:358-439)
void step(Ctx* c, double dt) {
    const double nu = c->nu;
    cd* v0 = c->w0.data();
    cd* v1 = c->v1.data();
    cd* v2 = c->v2.data();
    cd* N = c->tb.data();
    std::fill(c->v1.begin(), c->v1.end(), cd(0.0, 0.0));
    omega_nonlin(c, v0, N);
    cloop(c, [&](int, int, int, double k2, size_t p) {
        if (k2 <= c->kM2) {
            const double f0 = std::exp(-nu * k2 * dt);
            for (int q = 0; q < 3; ++q) {
                const cd a = v0[p + q] + cd(dt * N[p + q].real(), dt * N[p + q].imag());
                v1[p + q] = cd(a.real() * f0, a.imag() * f0);
            }
        } else {
            for (int q = 0; q < 3; ++q) v1[p + q] = cd(0.0, 0.0);
        }
    });
    omega_nonlin(c, v1, N);
    cloop(c, [&](int, int, int, double k2, size_t p) {
        if (k2 <= c->kM2) {
            const double f0 = std::exp(-nu * k2 * dt / 2);
            const double f1 = std::exp(nu * k2 * dt / 2);
            for (int q = 0; q < 3; ++q) {
                const cd a = cd(3 * v0[p + q].real(), 3 * v0[p + q].imag());
                const cd af = cd(a.real() * f0, a.imag() * f0);
                const cd b = v1[p + q] + cd(dt * N[p + q].real(), dt * N[p + q].imag());
                const cd bf = cd(b.real() * f1, b.imag() * f1);
                const cd s = af + bf;
                v2[p + q] = cd(s.real() * 0.25, s.imag() * 0.25);
            }
        }
    });
    omega_nonlin(c, v2, N);
    cloop(c, [&](int, int, int, double k2, size_t p) {
        if (k2 <= c->kM2) {
            const double f0 = std::exp(-nu * k2 * dt * 0.5);
            for (int q = 0; q < 3; ++q) {
                const cd a = cd(v0[p + q].real() * f0, v0[p + q].imag() * f0);
                const cd b = v2[p + q] + cd(dt * N[p + q].real(), dt * N[p + q].imag());
                const cd s = a + cd(2 * b.real(), 2 * b.imag());
                v0[p + q] = cd(s.real() * f0 / 3, s.imag() * f0 / 3);
            }
        }
    });
    force_divfree(c, v0);
    symmetrize(c, v0);
    c->iteration += 1;
}

// --------------------------------------------------------------- tracers --
struct Part {
    Ctx* ctx;
    int64_t n;
    int nb, mm, nsteps, step_idx;
    std::vector<double> pos;  // (n, 3)
    std::vector<double> rhs;  // (nsteps, n, 3)
    std::vector<double> coef; // (2nb+2) polynomials of ncoef coefficients
    int ncoef;
    double box[3], h[3];
};

inline double horner(const double* c, int nc, double x) {
    double acc = 0.0;
    for (int k = nc - 1; k >= 0; --k) acc = acc * x + c[k];
    return acc;
}

// particles_adams_bashforth.hpp:41-131, the expression forms of
// oracle/particles.py:ab_update
inline double ab(double p, const double* r, int order, double dt) {
    switch (order) {
        case 1: return p + dt * r[0];
        case 2: return p + dt * (3. * r[0] - r[1]) / 2.;
        case 3: return p + dt * (23. * r[0] - 16. * r[1] + 5. * r[2]) / 12.;
        case 4: return p + dt * (55. * r[0] - 59. * r[1] + 37. * r[2] - 9. * r[3]) / 24.;
        case 5:
            return p + dt * (1901. * r[0] - 2774. * r[1] + 2616. * r[2] - 1274. * r[3] + 251. * r[4]) /
                           720.;
        case 6:
            return p + dt *
                           (4277. * r[0] - 7923. * r[1] + 9982. * r[2] - 7298. * r[3] + 2877. * r[4] -
                            475. * r[5]) /
                           1440.;
    }
    return p;
}

// particles_system::completeLoop on the real field ur (nz, ny, nx, 3)
void complete_loop(Part* P, const double* ur, double dt) {
    Ctx* c = P->ctx;
    const int nb = P->nb, np = 2 * nb + 2, nc = P->ncoef;
    const int g[3] = {c->nx, c->ny, c->nz};
    const int order = std::min(P->step_idx, P->nsteps);
    const int64_t n = P->n;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double b[3][12];
        int64_t lay[3];
        for (int d = 0; d < 3; ++d) {
            const double x = P->pos[3 * i + d];
            const double L = P->box[d], h = P->h[d];
            // get_norm_pos_in_cell (particles_field_computer.hpp:55-63)
            const double nbx = std::floor(x / L);
            const double pib = x - nbx * L;
            const double cell = std::floor(pib / h);
            const double fr = (pib - cell * h) / h;
            for (int k = 0; k < np; ++k) b[d][k] = horner(&P->coef[(size_t)k * nc], nc, fr);
            // pbc_field_layer (particles_field_computer.hpp:176-183)
            const int64_t lvl = (int64_t)std::floor(x / h);
            lay[d] = ((lvl % g[d]) + g[d]) % g[d];
        }
        double acc[3] = {0.0, 0.0, 0.0};
        for (int iz = 0; iz < np; ++iz) {
            const int64_t z = (((lay[2] - nb + iz) % g[2]) + g[2]) % g[2];
            for (int ix = 0; ix < np; ++ix) {
                const int64_t x = (((lay[0] - nb + ix) % g[0]) + g[0]) % g[0];
                for (int iy = 0; iy < np; ++iy) {
                    const int64_t y = (((lay[1] - nb + iy) % g[1]) + g[1]) % g[1];
                    const double cf = (b[2][iz] * b[1][iy]) * b[0][ix];
                    const double* f = ur + (((size_t)z * g[1] + y) * g[0] + x) * 3;
                    for (int q = 0; q < 3; ++q) acc[q] = acc[q] + f[q] * cf;
                }
            }
        }
        // compute(): rhs[0] += u(x); move(): Adams-Bashforth of this order
        double r[6];
        for (int q = 0; q < 3; ++q) {
            P->rhs[3 * i + q] = P->rhs[3 * i + q] + acc[q];
            for (int s = 0; s < P->nsteps; ++s) r[s] = P->rhs[((size_t)s * n + i) * 3 + q];
            P->pos[3 * i + q] = ab(P->pos[3 * i + q], r, order, dt);
        }
    }
    P->step_idx += 1;
    // shift_rhs_vectors: rotate the history by one, new rhs[0] = 0
    if (P->nsteps > 0) {
        const size_t blk = (size_t)n * 3;
        for (int s = P->nsteps - 1; s >= 1; --s)
            std::memcpy(&P->rhs[(size_t)s * blk], &P->rhs[(size_t)(s - 1) * blk], blk * sizeof(double));
        std::fill(P->rhs.begin(), P->rhs.begin() + blk, 0.0);
    }
}

}  // namespace

extern "C" {

int orc_threads(void) { return omp_get_max_threads(); }
void orc_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
}

void* orc_create(int nx, int ny, int nz, double dkx, double dky, double dkz, int dealias) {
    Ctx* c = new Ctx();
    c->nx = nx;
    c->ny = ny;
    c->nz = nz;
    c->nxv = nx / 2 + 1;
    c->dkx = dkx;
    c->dky = dky;
    c->dkz = dkz;
    c->dealias = dealias;
    kspace_init(c);
    c->fx.init(nx);
    c->fy.init(ny);
    c->fz.init(nz);
    c->w0.assign(c->csize(), cd(0.0, 0.0));
    c->v1.assign(c->csize(), cd(0.0, 0.0));
    c->v2.assign(c->csize(), cd(0.0, 0.0));
    c->ua.assign(c->csize(), cd(0.0, 0.0));
    c->tb.assign(c->csize(), cd(0.0, 0.0));
    c->cw.assign((size_t)nz * ny * c->nxv * 3, cd(0.0, 0.0));
    c->ur.assign(c->rsize(), 0.0);
    c->wr.assign(c->rsize(), 0.0);
    return c;
}

void orc_destroy(void* h) { delete (Ctx*)h; }

void orc_set_physics(void* h, double nu, int forcing, double famp, double fk0, double fk1, int fmode) {
    Ctx* c = (Ctx*)h;
    c->nu = nu;
    c->forcing = forcing;
    c->famp = famp;
    c->fk0 = fk0;
    c->fk1 = fk1;
    c->fmode = fmode;
}

void orc_kinfo(void* h, double* kM, double* dk, int* nshells, int* nfilter) {
    Ctx* c = (Ctx*)h;
    *kM = c->kM;
    *dk = c->dk;
    *nshells = c->nshells;
    *nfilter = (int)c->filter.size();
}
void orc_filter(void* h, double* out) {
    Ctx* c = (Ctx*)h;
    std::memcpy(out, c->filter.data(), c->filter.size() * sizeof(double));
}

// state as interleaved complex128, shape (ny, nz, nx/2+1, 3)
void orc_set_state(void* h, const double* w) {
    Ctx* c = (Ctx*)h;
    std::memcpy(c->w0.data(), w, c->csize() * sizeof(cd));
}
void orc_get_state(void* h, double* w) {
    Ctx* c = (Ctx*)h;
    std::memcpy(w, c->w0.data(), c->csize() * sizeof(cd));
}
int orc_iteration(void* h) { return ((Ctx*)h)->iteration; }

void orc_step(void* h, double dt) { step((Ctx*)h, dt); }

// u^ = compute_velocity(state) into out (state layout, complex128) if out
// is not null; its unnormalised C2R into the context's real velocity, and a
// copy into rout (nz, ny, nx, 3) if rout is not null
void orc_velocity(void* h, double* out, double* rout) {
    Ctx* c = (Ctx*)h;
    compute_velocity(c, c->w0.data(), c->ua.data());
    if (out) std::memcpy(out, c->ua.data(), c->csize() * sizeof(cd));
    ift3(c, c->ua.data(), c->ur.data());
    if (rout) std::memcpy(rout, c->ur.data(), c->rsize() * sizeof(double));
}

// plain transforms (for pinning against pocketfft)
void orc_ift(void* h, const double* cin, double* rout) {
    Ctx* c = (Ctx*)h;
    ift3(c, reinterpret_cast<const cd*>(cin), rout);
}
void orc_dft(void* h, const double* rin, double* cout) {
    Ctx* c = (Ctx*)h;
    dft3(c, rin, reinterpret_cast<cd*>(cout));
}

void* orc_particles_create(void* h, int64_t n, int neighbours, int smoothness, int nsteps,
                           const double* pos, const double* rhs, int step_idx, const double* coef,
                           int ncoef) {
    Ctx* c = (Ctx*)h;
    Part* P = new Part();
    P->ctx = c;
    P->n = n;
    P->nb = neighbours;
    P->mm = smoothness;
    P->nsteps = nsteps;
    P->step_idx = step_idx;
    P->pos.assign(pos, pos + (size_t)n * 3);
    P->rhs.assign(rhs, rhs + (size_t)nsteps * n * 3);
    P->ncoef = ncoef;
    P->coef.assign(coef, coef + (size_t)(2 * neighbours + 2) * ncoef);
    const double dk[3] = {c->dkx, c->dky, c->dkz};
    const int g[3] = {c->nx, c->ny, c->nz};
    for (int d = 0; d < 3; ++d) {
        // 4 acos(0) / dk (particles_system_builder.hpp:176-179), spacing box / N
        P->box[d] = 4 * std::acos(0.0) / dk[d];
        P->h[d] = P->box[d] / (double)g[d];
    }
    return P;
}
void orc_particles_destroy(void* p) { delete (Part*)p; }

// completeLoop on the context's current real velocity (orc_velocity), or on
// a caller-given real field (nz, ny, nx, 3) if ur is not null
void orc_particles_complete_loop(void* p, const double* ur, double dt) {
    Part* P = (Part*)p;
    complete_loop(P, ur ? ur : P->ctx->ur.data(), dt);
}
void orc_particles_get(void* p, double* pos, double* rhs, int* step_idx) {
    Part* P = (Part*)p;
    if (pos) std::memcpy(pos, P->pos.data(), P->pos.size() * sizeof(double));
    if (rhs) std::memcpy(rhs, P->rhs.data(), P->rhs.size() * sizeof(double));
    if (step_idx) *step_idx = P->step_idx;
}

// NSVEparticles::step (NSVEparticles.cpp:33-41): velocity(t) -> tracers ->
// fluid step; p may be null
void orc_nsveparticles_step(void* h, void* p, double dt) {
    Ctx* c = (Ctx*)h;
    compute_velocity(c, c->w0.data(), c->ua.data());
    ift3(c, c->ua.data(), c->ur.data());
    if (p) complete_loop((Part*)p, c->ur.data(), dt);
    step(c, dt);
}

}  // extern "C"
