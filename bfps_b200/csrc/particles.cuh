// Tracer step on sm_100a: tensor-product gather of the real velocity field at
// each tracer, fused with the Adams-Bashforth position update.
//
// Reference (single-rank semantics):
//   particles_field_computer::get_norm_pos_in_cell / pbc_field_layer /
//   apply_computation (bfps/cpp/particles/particles_field_computer.hpp:55-183)
//   particles_adams_bashforth::move_particles (particles_adams_bashforth.hpp:18-133)
//   particles_system::completeLoop (particles_system.hpp:210-217)
// The weights, positions and accumulation are double; the field is read in
// its storage precision and promoted, as in the reference.  The sum runs
// z-outer, x-middle, y-inner like apply_computation.
//
// The rhs history is a ring of nsteps slots: logical rhs[j] is slot
// (head + j) % nsteps.  The host rotates `head` after each loop
// (shift_rhs_vectors); logical rhs[0] is then known to be zero, so the
// kernel overwrites it instead of accumulating (accum = false).
#pragma once
#include <stdint.h>
#include "interp_coeffs.h"

namespace bfg {

struct PParams {
    int64_t n;
    int N;            // grid points per axis
    double box[3];    // 2 pi / dk per axis
    double hstep[3];  // box / N
    int nsteps;
    int head;
    int order;        // AB order of this move
    int accum;        // rhs[0] += u(x) instead of =
    int move;         // 0: sample only (into out), 1: full loop
    double dt;
};

template <int NB, int MM>
__device__ __forceinline__ void beta_weights(double x, double* w) {
    using C = interp_coeffs<NB, MM>;
#pragma unroll
    for (int i = 0; i < C::npts; ++i) {
        double acc = C::c(i, C::ncoef - 1);
#pragma unroll
        for (int k = C::ncoef - 2; k >= 0; --k) acc = acc * x + C::c(i, k);
        w[i] = acc;
    }
}

// get_norm_pos_in_cell and pbc_field_layer for one axis
__device__ __forceinline__ void cell_of(double pos, double box, double h, int N, int* cell,
                                        double* frac) {
    const double nb = floor(pos / box);
    const double pib = pos - nb * box;
    const double ci = floor(pib / h);
    *frac = (pib - ci * h) / h;
    const int lvl = (int)floor(pos / h);
    *cell = ((lvl % N) + N) % N;
}

template <typename T, int NB, int MM>
__global__ void __launch_bounds__(128)
tracer_kernel(const PParams pp, const T* __restrict__ ru, double* __restrict__ pos,
              double* __restrict__ hist, double* __restrict__ sample_out) {
    constexpr int NP = 2 * NB + 2;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pp.n) return;
    const int N = pp.N;
    double p[3];
    int g[3];
    double wx[NP], wy[NP], wz[NP];
#pragma unroll
    for (int d = 0; d < 3; ++d) p[d] = pos[i * 3 + d];
    double fr[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) cell_of(p[d], pp.box[d], pp.hstep[d], N, &g[d], &fr[d]);
    beta_weights<NB, MM>(fr[0], wx);
    beta_weights<NB, MM>(fr[1], wy);
    beta_weights<NB, MM>(fr[2], wz);

    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
    const size_t rowN = (size_t)N;
#pragma unroll 1
    for (int iz = 0; iz < NP; ++iz) {
        int z = g[2] - NB + iz;
        z = (z + N) % N;
#pragma unroll
        for (int ix = 0; ix < NP; ++ix) {
            int xx = g[0] - NB + ix;
            xx = (xx + N) % N;
            const double bzx = wz[iz];
#pragma unroll
            for (int iy = 0; iy < NP; ++iy) {
                int y = g[1] - NB + iy;
                y = (y + N) % N;
                const double coef = (bzx * wy[iy]) * wx[ix];
                const T* f = ru + (((size_t)z * rowN + y) * rowN + xx) * 3;
                acc0 += (double)f[0] * coef;
                acc1 += (double)f[1] * coef;
                acc2 += (double)f[2] * coef;
            }
        }
    }
    if (!pp.move) {
        sample_out[i * 3 + 0] = acc0;
        sample_out[i * 3 + 1] = acc1;
        sample_out[i * 3 + 2] = acc2;
        return;
    }
    const int ns = pp.nsteps;
    const size_t slot = (size_t)pp.n * 3;
    double r0[3] = {acc0, acc1, acc2};
    double* h0 = hist + (size_t)pp.head * slot + i * 3;
    if (pp.accum) {
#pragma unroll
        for (int d = 0; d < 3; ++d) r0[d] += h0[d];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) h0[d] = r0[d];
    double r[6][3];
#pragma unroll
    for (int d = 0; d < 3; ++d) r[0][d] = r0[d];
    for (int j = 1; j < pp.order; ++j) {
        const double* hj = hist + (size_t)((pp.head + j) % ns) * slot + i * 3;
#pragma unroll
        for (int d = 0; d < 3; ++d) r[j][d] = hj[d];
    }
    const double dt = pp.dt;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double x = p[d];
        switch (pp.order) {
            case 1: x += dt * r[0][d]; break;
            case 2: x += dt * (3. * r[0][d] - r[1][d]) / 2.; break;
            case 3: x += dt * (23. * r[0][d] - 16. * r[1][d] + 5. * r[2][d]) / 12.; break;
            case 4:
                x += dt * (55. * r[0][d] - 59. * r[1][d] + 37. * r[2][d] - 9. * r[3][d]) / 24.;
                break;
            case 5:
                x += dt * (1901. * r[0][d] - 2774. * r[1][d] + 2616. * r[2][d] -
                           1274. * r[3][d] + 251. * r[4][d]) / 720.;
                break;
            case 6:
                x += dt * (4277. * r[0][d] - 7923. * r[1][d] + 9982. * r[2][d] -
                           7298. * r[3][d] + 2877. * r[4][d] - 475. * r[5][d]) / 1440.;
                break;
            default: break;
        }
        pos[i * 3 + d] = x;
    }
}

}  // namespace bfg
