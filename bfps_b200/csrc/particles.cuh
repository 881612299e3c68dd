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
// as (b_z b_y) b_x f over z, then y, with x innermost along the contiguous
// row (apply_computation runs z, x, y; the sums agree to rounding).
//
// The rhs history is a ring of nsteps slots: logical rhs[j] is slot
// (head + j) % nsteps.  The host rotates `head` after each loop
// (shift_rhs_vectors); logical rhs[0] is then known to be zero, so the
// kernel overwrites it instead of accumulating (accum = false).
#pragma once
#include <stdint.h>
#include <type_traits>
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

// periodic index of a stencil point: c in [-N, 2N) (stencils are narrower
// than the grid), so one conditional add or subtract replaces the modulo
__device__ __forceinline__ int wrap_once(int c, int N) {
    return c < 0 ? c + N : (c >= N ? c - N : c);
}

// x-segment of one stencil row: 2n+2 points x 3 components, contiguous in
// [z][y][x][c] unless the stencil wraps across the periodic x boundary.
// Loads 16-byte vectors from the aligned-down start and accumulates
// sum_ix w[ix] * f(ix, c) in double.
template <typename T, int NB>
__device__ __forceinline__ void row_accumulate(const T* __restrict__ row, int x0, int N,
                                               const double* wxc, double& a0, double& a1,
                                               double& a2) {
    constexpr int NP = 2 * NB + 2;
    constexpr int VEC = 16 / (int)sizeof(T);  // elements per 16-byte vector
    constexpr int NV = (3 * NP + VEC - 1) / VEC + 1;  // vectors covering any alignment
    if (x0 >= 0 && x0 + NP <= N) {
        const int e0 = x0 * 3;
        const int base = e0 & ~(VEC - 1);
        const int off = e0 - base;
        T buf[NV * VEC];
        const int maxv = (N * 3 - base) / VEC;  // vectors left in this row
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            if (v < maxv) {
                if constexpr (sizeof(T) == 4) {
                    const float4 q = *reinterpret_cast<const float4*>(row + base + v * VEC);
                    buf[v * 4 + 0] = q.x; buf[v * 4 + 1] = q.y;
                    buf[v * 4 + 2] = q.z; buf[v * 4 + 3] = q.w;
                } else {
                    const double2 q = *reinterpret_cast<const double2*>(row + base + v * VEC);
                    buf[v * 2 + 0] = q.x; buf[v * 2 + 1] = q.y;
                }
            } else {
#pragma unroll
                for (int u = 0; u < VEC; ++u) buf[v * VEC + u] = (T)0;
            }
        }
#pragma unroll
        for (int ix = 0; ix < NP; ++ix) {
            T f[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int j = ix * 3 + c;
                // buf[j + off], off in [0, VEC)
                T v = buf[j];
#pragma unroll
                for (int o = 1; o < VEC; ++o) v = (off == o) ? buf[j + o] : v;
                f[c] = v;
            }
            a0 += (double)f[0] * wxc[ix];
            a1 += (double)f[1] * wxc[ix];
            a2 += (double)f[2] * wxc[ix];
        }
    } else {
#pragma unroll
        for (int ix = 0; ix < NP; ++ix) {
            const int xx = wrap_once(x0 + ix, N);
            a0 += (double)row[xx * 3 + 0] * wxc[ix];
            a1 += (double)row[xx * 3 + 1] * wxc[ix];
            a2 += (double)row[xx * 3 + 2] * wxc[ix];
        }
    }
}

// 32-byte vector load (one L1 sector per lane), sm_100; p 32-byte aligned
__device__ __forceinline__ void ld_v8(const float* p, float* v) {
    asm volatile("ld.global.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]),
                   "=f"(v[6]), "=f"(v[7])
                 : "l"(p));
}

constexpr int TRACER_THREADS = 128;

// Lanes that share one tracer: two for FP32 fields, one for FP64 fields.  A
// stencil row is read as up to four (six for n = 5) 32-byte sectors from its
// aligned-down start.  With one lane per tracer the gather is bound by L1
// wavefronts (about one per sector, as each lane's sector lies in another
// line); with the sectors of a row spread over two lanes of one load, a
// wavefront serves both, and the per-row address and FP64 work only doubles.
// Measured on B200 (4e6 tracers, n = 3, m = 2, 512^3): 3.26 ms with one lane,
// 2.70 ms with two, 4.47 ms with four (issue bound).
template <typename T>
__host__ __device__ constexpr int tracer_lanes() {
    return sizeof(T) == 4 ? 2 : 1;
}
// n = 3 stencils (8 rows per plane): the y loop of the FP32 gather is
// unrolled, so the y weights stay in registers instead of local memory, and
// the kernel is given the registers of five blocks per SM instead of six.
// Measured on B200 (4e6 tracers, n = 3, m = 2): 2.57 against 2.70 ms at
// 512^3; for n = 2 (ensembles) it was slower, for n = 4, 5 it spills.
template <int NB>
__host__ __device__ constexpr int tracer_row_unroll() {
    return NB == 3 ? 2 * NB + 2 : 1;
}
template <int NB>
__host__ __device__ constexpr int tracer_min_blocks() {
    return NB == 3 ? 5 : 6;
}
template <typename T>
__host__ __device__ constexpr int tracers_per_block() {
    return TRACER_THREADS / tracer_lanes<T>();
}

// sum of v over the L lanes of a tracer group, pairwise ((l0 + l1) + (l2 +
// l3) for four) on every lane (xor partners add the same two values, so all
// lanes agree)
template <int L>
__device__ __forceinline__ double group_sum(double v, unsigned gmask) {
#pragma unroll
    for (int m = 1; m < L; m *= 2) v += __shfl_xor_sync(gmask, v, m, L);
    return v;
}

// FP32 field (precision form), lane j (0..L-1) of the tracer's group, which
// reads vectors j, j + L, ... of each row: the x sums of the stencil rows run
// in FP32 with the x weights rounded to FP32, over the words a lane reads; the
// y/z weights, the accumulation of those sums over the rows, the sum over the
// lanes and everything after stay FP64.  Word i of the row segment read from the
// aligned-down start belongs to point (i - off) / 3, component
// (i - off) mod 3, so each lane's x weights are shifted once per tracer and its
// sums are kept per word phase i mod 3, mapped to components at the end.
#ifndef BFG_TRACER_ROWSUM_F64
#define BFG_TRACER_ROWSUM_F64 0
#endif
template <int NB, int L>
__device__ __forceinline__ void row_gather_f32(const float* __restrict__ ru, int N, const int* g,
                                               int x0, const double* wx, const double* wy,
                                               const double* wz, int j, unsigned gmask,
                                               double& a0, double& a1, double& a2) {
    using SumT = typename std::conditional<BFG_TRACER_ROWSUM_F64 != 0, double, float>::type;
    constexpr int NP = 2 * NB + 2;
    constexpr int VW = 8;                                // floats per vector
    constexpr int NVMAX = (3 * NP + 2 * (VW - 1)) / VW;  // vectors covering any alignment
    constexpr int VPL = (NVMAX + L - 1) / L;             // vectors per lane
    const size_t rowN = (size_t)N;
    SumT wxf[NP];
#pragma unroll
    for (int ix = 0; ix < NP; ++ix) wxf[ix] = (SumT)wx[ix];
    if (x0 >= 0 && x0 + NP <= N) {
        const int e0 = x0 * 3;
        const int base = e0 & ~(VW - 1);
        const int off = e0 - base;
        // vectors holding stencil words, none past the end of the row
        const int nv = min((off + 3 * NP + VW - 1) / VW, (N * 3 - base) / VW);
        SumT wl[VPL][VW];
#pragma unroll
        for (int t = 0; t < VPL; ++t)
#pragma unroll
            for (int u = 0; u < VW; ++u) {
                const int k = VW * (j + L * t) + u - off;  // 3 * point + component
                SumT w = 0;
#pragma unroll
                for (int pt = 0; pt < NP; ++pt) w = (k >= 3 * pt && k < 3 * pt + 3) ? wxf[pt] : w;
                wl[t][u] = w;
            }
        // word u of vector v = j + L t has phase (8 v + u) mod 3, that is
        // (2 j + 2 L t + u) mod 3: the sums are kept per lane-relative phase
        // (2 L t + u) mod 3 and rotated by 2 j at the end
        double ph[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
        for (int iz = 0; iz < NP; ++iz) {
            const int z = wrap_once(g[2] - NB + iz, N);
            const double bz = wz[iz];
#pragma unroll(tracer_row_unroll<NB>())
            for (int iy = 0; iy < NP; ++iy) {
                const int y = wrap_once(g[1] - NB + iy, N);
                const float* row = ru + ((size_t)z * rowN + y) * rowN * 3 + base;
                const double bzy = bz * wy[iy];
                SumT sp[3] = {0, 0, 0};
#pragma unroll
                for (int t = 0; t < VPL; ++t) {
                    if (j + L * t < nv) {
                        float q[VW];
                        ld_v8(row + VW * (j + L * t), q);
#pragma unroll
                        for (int u = 0; u < VW; ++u)
                            sp[(2 * L * t + u) % 3] = fma((SumT)q[u], wl[t][u], sp[(2 * L * t + u) % 3]);
                    }
                }
#pragma unroll
                for (int c = 0; c < 3; ++c) ph[c] = fma(bzy, (double)sp[c], ph[c]);
            }
        }
        // lane-relative phase (k - 2 j) mod 3 holds phase k
        const int r = (2 * j) % 3;
        double G[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
            G[k] = group_sum<L>(r == 0 ? ph[k] : (r == 1 ? ph[(k + 2) % 3] : ph[(k + 1) % 3]), gmask);
        // component c sits in phase (c + off) mod 3
        const int k0 = off % 3;
        a0 = k0 == 0 ? G[0] : (k0 == 1 ? G[1] : G[2]);
        a1 = k0 == 0 ? G[1] : (k0 == 1 ? G[2] : G[0]);
        a2 = k0 == 0 ? G[2] : (k0 == 1 ? G[0] : G[1]);
    } else {
        // stencil across the periodic x boundary: lane j takes the points
        // ix = j, j + L, ... with scalar loads
        constexpr int PPL = (NP + L - 1) / L;  // points per lane
        SumT wj[PPL];
        int xj[PPL];
#pragma unroll
        for (int m = 0; m < PPL; ++m) {
            const int ix = j + L * m;
            SumT w = 0;
#pragma unroll
            for (int pt = 0; pt < NP; ++pt) w = ix == pt ? wxf[pt] : w;
            wj[m] = w;
            xj[m] = ix < NP ? wrap_once(x0 + ix, N) : -1;
        }
        double A[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
        for (int iz = 0; iz < NP; ++iz) {
            const int z = wrap_once(g[2] - NB + iz, N);
            const double bz = wz[iz];
#pragma unroll(tracer_row_unroll<NB>())
            for (int iy = 0; iy < NP; ++iy) {
                const int y = wrap_once(g[1] - NB + iy, N);
                const float* row = ru + ((size_t)z * rowN + y) * rowN * 3;
                SumT s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
                for (int m = 0; m < PPL; ++m) {
                    if (xj[m] >= 0) {
                        s0 = fma((SumT)row[xj[m] * 3 + 0], wj[m], s0);
                        s1 = fma((SumT)row[xj[m] * 3 + 1], wj[m], s1);
                        s2 = fma((SumT)row[xj[m] * 3 + 2], wj[m], s2);
                    }
                }
                const double bzy = bz * wy[iy];
                A[0] = fma(bzy, (double)s0, A[0]);
                A[1] = fma(bzy, (double)s1, A[1]);
                A[2] = fma(bzy, (double)s2, A[2]);
            }
        }
        a0 = group_sum<L>(A[0], gmask);
        a1 = group_sum<L>(A[1], gmask);
        a2 = group_sum<L>(A[2], gmask);
    }
}

// tracer i of one system, lane j of its group (tracer_lanes<T>() lanes; gmask
// the group's lanes): gather u(x_i), then (move) the Adams-Bashforth step.
// With four lanes, lane d < 3 finishes component d.
template <typename T, int NB, int MM>
__device__ __forceinline__ void tracer_one(const PParams& pp, const T* __restrict__ ru,
                                           double* __restrict__ pos, double* __restrict__ hist,
                                           double* __restrict__ sample_out, int64_t i, int j,
                                           unsigned gmask) {
    constexpr int NP = 2 * NB + 2;
    constexpr int L = tracer_lanes<T>();
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

    double acc[3] = {0.0, 0.0, 0.0};
    const size_t rowN = (size_t)N;
    const int x0 = g[0] - NB;
    if constexpr (sizeof(T) == 4) {
        row_gather_f32<NB, L>(reinterpret_cast<const float*>(ru), N, g, x0, wx, wy, wz, j, gmask,
                           acc[0], acc[1], acc[2]);
    } else {
#pragma unroll 1
        for (int iz = 0; iz < NP; ++iz) {
            const int z = wrap_once(g[2] - NB + iz, N);
#pragma unroll 1
            for (int iy = 0; iy < NP; ++iy) {
                const int y = wrap_once(g[1] - NB + iy, N);
                // coefficient (bz * by) * bx of apply_computation
                const double bzy = wz[iz] * wy[iy];
                double wxc[NP];
#pragma unroll
                for (int ix = 0; ix < NP; ++ix) wxc[ix] = bzy * wx[ix];
                row_accumulate<T, NB>(ru + ((size_t)z * rowN + y) * rowN * 3, x0, N, wxc, acc[0],
                                      acc[1], acc[2]);
            }
        }
    }
    if (!pp.move) {
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (d % L == j) sample_out[i * 3 + d] = acc[d];
        return;
    }
    const int ns = pp.nsteps;
    const size_t slot = (size_t)pp.n * 3;
    const double dt = pp.dt;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d % L != j) continue;
        double* h0 = hist + (size_t)pp.head * slot + i * 3 + d;
        double r[6];
        r[0] = acc[d];
        if (pp.accum) r[0] += *h0;
        *h0 = r[0];
#pragma unroll
        for (int k = 1; k < 6; ++k) {
            r[k] = 0.0;
            if (k < pp.order) {
                int sl = pp.head + k;
                sl = sl >= ns ? sl - ns : sl;
                r[k] = hist[(size_t)sl * slot + i * 3 + d];
            }
        }
        double x = p[d];
        switch (pp.order) {
            case 1: x += dt * r[0]; break;
            case 2: x += dt * (3. * r[0] - r[1]) / 2.; break;
            case 3: x += dt * (23. * r[0] - 16. * r[1] + 5. * r[2]) / 12.; break;
            case 4:
                x += dt * (55. * r[0] - 59. * r[1] + 37. * r[2] - 9. * r[3]) / 24.;
                break;
            case 5:
                x += dt * (1901. * r[0] - 2774. * r[1] + 2616. * r[2] - 1274. * r[3] +
                           251. * r[4]) / 720.;
                break;
            case 6:
                x += dt * (4277. * r[0] - 7923. * r[1] + 9982. * r[2] - 7298. * r[3] +
                           2877. * r[4] - 475. * r[5]) / 1440.;
                break;
            default: break;
        }
        pos[i * 3 + d] = x;
    }
}

// lanes of the calling thread's tracer group, as a shuffle mask
template <int L>
__device__ __forceinline__ unsigned tracer_group_mask() {
    const int lane = threadIdx.x & 31;
    return L == 1 ? (1u << lane) : (((1u << L) - 1u) << (lane & ~(L - 1)));
}

template <typename T, int NB, int MM>
__global__ void __launch_bounds__(TRACER_THREADS, tracer_min_blocks<NB>())
tracer_kernel(const PParams pp, const T* __restrict__ ru, double* __restrict__ pos,
              double* __restrict__ hist, double* __restrict__ sample_out) {
    constexpr int L = tracer_lanes<T>();
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t i = t / L;
    if (i >= pp.n) return;  // whole groups leave together
    tracer_one<T, NB, MM>(pp, ru, pos, hist, sample_out, i, (int)(t % L), tracer_group_mask<L>());
}

// the tracer systems of many ensemble members in one launch
struct TracerSet {
    PParams pp;     // head, order and accum advance on the device after each loop
    int step_idx;
    const void* ru;
    double* pos;
    double* hist;
};

// inc_step_idx + shift_rhs_vectors of every set (particles_system.hpp:191-208)
__global__ void tracer_sets_advance(TracerSet* __restrict__ sets, int nsets) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nsets) return;
    TracerSet& s = sets[k];
    s.step_idx += 1;
    s.pp.head = (s.pp.head - 1 + s.pp.nsteps) % s.pp.nsteps;
    s.pp.order = min(s.step_idx, s.pp.nsteps);
    s.pp.accum = 0;
}

// Each set owns whole blocks: block b belongs to the set k with
// bstart[k] <= b < bstart[k+1]; the set is found once per block and its
// descriptor copied to shared memory.
template <typename T, int NB, int MM>
__global__ void __launch_bounds__(TRACER_THREADS, tracer_min_blocks<NB>())
tracer_batch_kernel(const TracerSet* __restrict__ sets, const int64_t* __restrict__ bstart,
                    int nsets) {
    __shared__ TracerSet s;
    __shared__ int s_k;
    if (threadIdx.x == 0) {
        const int64_t b = blockIdx.x;
        int lo = 0, hi = nsets - 1;
        while (lo < hi) {  // last k with bstart[k] <= b
            const int mid = (lo + hi + 1) / 2;
            if (bstart[mid] <= b) lo = mid;
            else hi = mid - 1;
        }
        s_k = lo;
    }
    __syncthreads();
    {
        static_assert(sizeof(TracerSet) % 4 == 0, "descriptor copy");
        const int* src = reinterpret_cast<const int*>(&sets[s_k]);
        int* dst = reinterpret_cast<int*>(&s);
        for (int w = threadIdx.x; w < (int)(sizeof(TracerSet) / 4); w += blockDim.x) dst[w] = src[w];
    }
    __syncthreads();
    constexpr int L = tracer_lanes<T>();
    const int64_t i = ((int64_t)blockIdx.x - bstart[s_k]) * (blockDim.x / L) + threadIdx.x / L;
    if (i >= s.pp.n) return;  // whole groups leave together
    tracer_one<T, NB, MM>(s.pp, (const T*)s.ru, s.pos, s.hist, nullptr, i, (int)(threadIdx.x % L),
                          tracer_group_mask<L>());
}

// ---------------------------------------------------------------------------
// Cell ordering of the tracers (counting sort on the (z, y) cell row).
// The single-rank reference reorders its arrays by z-layer in every
// redistribute (particles_distr_mpi.hpp:798-831); here the order only serves
// memory locality of the gather (every result is per tracer), so the arrays
// are re-sorted every few steps.  Order inside a bucket is not fixed.
__global__ void tracer_keys(const PParams pp, const double* __restrict__ pos,
                            unsigned* __restrict__ key, unsigned* __restrict__ rank,
                            unsigned* __restrict__ count) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pp.n) return;
    const int N = pp.N;
    int gz, gy;
    double fr;
    cell_of(pos[i * 3 + 2], pp.box[2], pp.hstep[2], N, &gz, &fr);
    cell_of(pos[i * 3 + 1], pp.box[1], pp.hstep[1], N, &gy, &fr);
    const unsigned k = (unsigned)gz * (unsigned)N + (unsigned)gy;
    key[i] = k;
    rank[i] = atomicAdd(&count[k], 1u);
}

// Exclusive scan of the nb bucket counts in three launches: the sum of each
// 1024-bucket block, an exclusive scan of those sums (one CTA: nb <= 2^20,
// i.e. N <= 1024), then each block's own scan plus its block offset.
// Integer sums, so the offsets do not depend on the order of the additions.
// 1024 threads per CTA; returns v's exclusive prefix within the CTA and the
// CTA's total in *total.
__device__ __forceinline__ unsigned cta_scan_1024(unsigned v, unsigned* ws, unsigned* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned w = ws[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        ws[lane] = w;  // inclusive over the warps
    }
    __syncthreads();
    *total = ws[31];
    return (warp == 0 ? 0u : ws[warp - 1]) + x - v;
}
__global__ void __launch_bounds__(1024) bucket_block_sums(const unsigned* __restrict__ count,
                                                          unsigned* __restrict__ bsum, int nb) {
    __shared__ unsigned ws[32];
    const int i = blockIdx.x * 1024 + threadIdx.x;
    unsigned total;
    cta_scan_1024(i < nb ? count[i] : 0u, ws, &total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}
__global__ void __launch_bounds__(1024) bucket_scan_sums(unsigned* __restrict__ bsum, int nblk) {
    __shared__ unsigned ws[32];
    const int t = threadIdx.x;
    const unsigned v = t < nblk ? bsum[t] : 0u;
    unsigned total;
    const unsigned ex = cta_scan_1024(v, ws, &total);  // every read precedes the barriers
    if (t < nblk) bsum[t] = ex;
}
__global__ void __launch_bounds__(1024) bucket_scan_blocks(const unsigned* __restrict__ count,
                                                           const unsigned* __restrict__ bsum,
                                                           unsigned* __restrict__ offset, int nb) {
    __shared__ unsigned ws[32];
    const int i = blockIdx.x * 1024 + threadIdx.x;
    unsigned total;
    const unsigned ex = cta_scan_1024(i < nb ? count[i] : 0u, ws, &total);
    if (i < nb) offset[i] = bsum[blockIdx.x] + ex;
}

// The tracers in cell order.  tracer_perm records the source of every
// destination (src[offset[key] + rank] = i, one 4-byte store per tracer);
// tracer_gather then copies positions, rhs history and indexes with the
// writes in order and the reads at random (random partial-sector writes,
// as a direct scatter makes them, cost a read-modify-write each).
__global__ void tracer_perm(const PParams pp, const unsigned* __restrict__ key,
                            const unsigned* __restrict__ rank, const unsigned* __restrict__ offset,
                            unsigned* __restrict__ src) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pp.n) return;
    src[offset[key[i]] + rank[i]] = (unsigned)i;
}

__global__ void tracer_gather(const PParams pp, const unsigned* __restrict__ src,
                              const double* __restrict__ pos, const double* __restrict__ hist,
                              const int64_t* __restrict__ idx, double* __restrict__ pos2,
                              double* __restrict__ hist2, int64_t* __restrict__ idx2) {
    const int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= pp.n) return;
    const int64_t i = src[d];
    const size_t slot = (size_t)pp.n * 3;
#pragma unroll
    for (int c = 0; c < 3; ++c) pos2[d * 3 + c] = pos[i * 3 + c];
    for (int s = 0; s < pp.nsteps; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c) hist2[s * slot + d * 3 + c] = hist[s * slot + i * 3 + c];
    idx2[d] = idx[i];
}

}  // namespace bfg
