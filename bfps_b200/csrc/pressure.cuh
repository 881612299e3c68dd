// Pressure and Lagrangian acceleration of the vorticity equation (sm_100a).
//
// Reference: vorticity_equation::compute_pressure (vorticity_equation.cpp:
// 441-514) and compute_Lagrangian_acceleration (:516-578), sampled at the
// tracers by NSVEparticles::do_stats (NSVEparticles.cpp:70-98).
//
// The transforms are the engine's passes; the kernels here are the
// pointwise steps between them:
//   products_kernel       u_c u_c or u_c u_(c+1) in real space
//   pressure_kernel       dealias the transformed products and contract them
//                         with k_i k_j into p^ (two calls: diagonal terms,
//                         then off-diagonal terms and the division by
//                         npoints k^2)
//   acceleration_kernel   -nu k^2 u^ (+ forcing) - i k p^
//   gather_rows_kernel    state-layout rows to the reference host layout
// Each keeps the reference's order of operations and its roundings to the
// storage precision (the reference stores every intermediate in rnumber).
#pragma once
#include "passes.cuh"

namespace bfg {

// out[p][c] = u[p][c] u[p][c] (off = 0) or u[p][c] u[p][(c+1) % 3] (off = 1)
// (vorticity_equation.cpp:452-462, 482-492); u and out are [z][y][x][3]
template <typename T>
__global__ void products_kernel(const T* __restrict__ u, T* __restrict__ out, size_t npts,
                                int off) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npts) return;
    const T a = u[p * 3], b = u[p * 3 + 1], c = u[p * 3 + 2];
    if (off == 0) {
        out[p * 3] = a * a;
        out[p * 3 + 1] = b * b;
        out[p * 3 + 2] = c * c;
    } else {
        out[p * 3] = a * b;
        out[p * 3 + 1] = b * c;
        out[p * 3 + 2] = c * a;
    }
}

// kspace::dealias of one transformed product mode (kspace.cpp:461-485)
template <typename T>
__device__ __forceinline__ void dealias_mode(const KParams& kp, const T* __restrict__ filt,
                                             double k2, cpx<T>* g) {
    if (kp.dealias == 1) {
        int key = (int)rint(k2 * kp.inv_dk2);
        key = key < kp.nfilt ? key : kp.nfilt - 1;
        const T f = filt[key];
#pragma unroll
        for (int c = 0; c < 3; ++c) g[c] = scale(g[c], f);
    } else if (k2 >= kp.kM2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) g[c] = zero_c<T>();
    }
}

// p^ from the transformed products G (state layout, 3 components): off = 0
// writes p = -(kx^2 G0 + ky^2 G1 + kz^2 G2) for 0 < k2 <= kM2 (else 0);
// off = 1 updates p -= 2 (kx ky G0 + ky kz G1 + kz kx G2), p /= npoints k2.
// p^ is component 0 of the 3-component buffer P.
template <typename T, int N>
__global__ void pressure_kernel(const KParams kp, const T* __restrict__ filt,
                                const cpx<T>* __restrict__ G, cpx<T>* P, int off) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t npts = (size_t)N * N * kp.nxv;
    if (e >= npts) return;
    const int ix = (int)(e % kp.nxv);
    const size_t r = e / kp.nxv;
    const int kz_i = (int)(r % N), ky_i = (int)(r / N);
    const double kx = ix * kp.dkx, ky = kwrap<N>(ky_i, kp.dky), kz = kwrap<N>(kz_i, kp.dkz);
    const double k2 = (kx * kx + ky * ky) + kz * kz;
    const size_t pt = r * kp.nxp + ix;
    cpx<T> g[3] = {G[pt * 3], G[pt * 3 + 1], G[pt * 3 + 2]};
    dealias_mode<T>(kp, filt, k2, g);
    const bool m = k2 <= kp.kM2 && k2 > 0.0;
    if (off == 0) {
        cpx<T> p = zero_c<T>();
        if (m) {
            p.x = (T)(-(kx * kx * (double)g[0].x + ky * ky * (double)g[1].x +
                        kz * kz * (double)g[2].x));
            p.y = (T)(-(kx * kx * (double)g[0].y + ky * ky * (double)g[1].y +
                        kz * kz * (double)g[2].y));
        }
        P[pt * 3] = p;
    } else if (m) {
        cpx<T> p = P[pt * 3];
        p.x = (T)((double)p.x - 2 * (kx * ky * (double)g[0].x + ky * kz * (double)g[1].x +
                                     kz * kx * (double)g[2].x));
        p.y = (T)((double)p.y - 2 * (kx * ky * (double)g[0].y + ky * kz * (double)g[1].y +
                                     kz * kx * (double)g[2].y));
        const double d = (double)N * (double)N * (double)N * k2;
        p.x = (T)((double)p.x / d);
        p.y = (T)((double)p.y / d);
        P[pt * 3] = p;
    }
}

// a^ = -nu k2 u^ (+ famplitude u^ on the linear forcing band) - i k p^ for
// k2 <= kM2, else 0 (vorticity_equation.cpp:533-576); u^ state layout,
// p^ component 0 of P
template <typename T, int N>
__global__ void acceleration_kernel(const KParams kp, double nu, const cpx<T>* __restrict__ U,
                                    const cpx<T>* __restrict__ P, cpx<T>* __restrict__ A) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t npts = (size_t)N * N * kp.nxv;
    if (e >= npts) return;
    const int ix = (int)(e % kp.nxv);
    const size_t r = e / kp.nxv;
    const int kz_i = (int)(r % N), ky_i = (int)(r / N);
    const double kx = ix * kp.dkx, ky = kwrap<N>(ky_i, kp.dky), kz = kwrap<N>(kz_i, kp.dkz);
    const double k2 = (kx * kx + ky * ky) + kz * kz;
    const size_t pt = r * kp.nxp + ix;
    cpx<T> a[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) a[c] = zero_c<T>();
    if (k2 <= kp.kM2) {
        cpx<T> u[3] = {U[pt * 3], U[pt * 3 + 1], U[pt * 3 + 2]};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            a[c].x = (T)(-nu * k2 * (double)u[c].x);
            a[c].y = (T)(-nu * k2 * (double)u[c].y);
        }
        if (kp.forcing == 1) {
            const double kn = sqrt(k2);
            if (kp.fk0 <= kn && kp.fk1 >= kn) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    a[c].x = (T)((double)a[c].x + kp.famp * (double)u[c].x);
                    a[c].y = (T)((double)a[c].y + kp.famp * (double)u[c].y);
                }
            }
        }
        const cpx<T> p = P[pt * 3];
        const double kk[3] = {kx, ky, kz};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            a[c].x = (T)((double)a[c].x + kk[c] * (double)p.y);
            a[c].y = (T)((double)a[c].y - kk[c] * (double)p.x);
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) A[pt * 3 + c] = a[c];
}

// rows of a state-layout buffer (nxp points of csrc complex components) to
// the reference host layout (nxv points of cout components)
template <typename T>
__global__ void gather_rows_kernel(const cpx<T>* __restrict__ src, int nxp, int nxv, int csrc,
                                   int cout, cpx<T>* __restrict__ dst, size_t rows) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t n = rows * nxv * cout;
    if (e >= n) return;
    const int c = (int)(e % cout);
    const size_t q = e / cout;
    const int ix = (int)(q % nxv);
    const size_t r = q / nxv;
    dst[e] = src[(r * nxp + ix) * csrc + c];
}

}  // namespace bfg
