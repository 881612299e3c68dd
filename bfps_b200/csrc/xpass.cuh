// Warp-per-row nonlinear x pass (the X pass of every RK stage), FP32, N = 512.
//
// Same result as row_nonlin (passes.cuh) -- per (z, y) row: C2R of the
// velocity and vorticity rows (half-length complex transforms with the
// C2R pre-processing), u x w / N^3 on the grid, R2C of the product -- but
// organised around the warp instead of the CTA:
//
//   * each warp owns whole rows: one TMA bulk copy per input row brings the
//     interleaved u and w rows (6240 bytes each) into the warp's own shared
//     memory, completing on one of the warp's two mbarriers; the next row's
//     u row is requested as soon as this row's u transforms are done, its w
//     row as soon as this row's output has left, so both arrive while the
//     warp still computes;
//   * a 256-point transform lives in registers, eight values per lane:
//     one radix-8 butterfly over registers, then two exchanges through the
//     warp's own shared buffer (radix-8 over 8-lane groups, radix-4 over
//     4-lane groups), so no step of a row waits for another warp
//     (__syncwarp only, no block barrier);
//   * the product is formed in registers on the transformed values of all
//     six transforms (every transform leaves the grid points in the same
//     lane / register order);
//   * the output row (and, in stage 1, the real velocity row u(t) for the
//     tracers) leaves by TMA bulk stores.
//
// Lane layout of a 256-point transform (k frequency, n grid pair index,
// z[n] = (x[2n], x[2n+1])): the spectrum side holds Z[l + 32 q] in lane l,
// register q; the grid side holds z[n1 + 8 m1 + 64 m2] in lane 4 n1 + j,
// register (m1 == j ? 0 : 4) + m2, m1 in {j, j + 4}.  With n = n1 + 8 n2,
// k = l + 32 q: W_256^{nk} = W_256^{n1 l} W_8^{n1 q} W_32^{n2 l}, and the
// 32-point factor splits again with n2 = m1 + 8 m2, l = l1 + 4 l2.
//
// Shared-memory pitches keep every exchange free of bank conflicts for
// 8-byte accesses (half-warp wavefronts): [n1][l] rows of 36, [n1][l1][m1]
// blocks of 68 / 17.
#pragma once
#include "bulk.cuh"
#include "passes.cuh"

namespace bfg {

namespace xw {

constexpr int NWARP = 12;              // warps per CTA, one CTA per SM
constexpr int XP1 = 36;                // exchange [n1][l] row pitch
constexpr int XP2 = 68, XQ2 = 17;      // exchange [n1][l1][m1] pitches
constexpr int XBUF = 8 * XP2;          // 544 >= 8 * XP1, >= 256
constexpr int T1P = 36;                // twiddle table [n1][l] row pitch
constexpr int T2P = 9;                 // twiddle table [l1][m1] row pitch: the inverse
                                       // reads it with l1 over the lanes, which a
                                       // pitch of 8 puts on two banks for four rows

template <int N>
struct Smem {
    static constexpr int RL = (N / 2 + 4) * 3;  // padded interleaved row (complex)
    cpx<float> su[RL];                          // u row in, real u row out
    cpx<float> sw[RL];                          // w row in, output row out
    cpx<float> x[XBUF];                         // exchanges
};

// 256-point inverse transform (sign +): Z[l + 32 q] in v[q] -> grid order
__device__ __forceinline__ void inv256(cpx<float> (&v)[8], cpx<float>* xb,
                                       const cpx<float>* __restrict__ t1,
                                       const cpx<float>* __restrict__ t2, int lane) {
    dft<float, true, 8>(v);  // over q -> n1
#pragma unroll
    for (int n1 = 1; n1 < 8; ++n1) v[n1] = cmulc(v[n1], t1[n1 * T1P + lane]);  // W_256^{-n1 l}
    __syncwarp();
#pragma unroll
    for (int n1 = 0; n1 < 8; ++n1) xb[n1 * XP1 + lane] = v[n1];
    __syncwarp();
    const int n1 = lane >> 2, l1 = lane & 3;
#pragma unroll
    for (int l2 = 0; l2 < 8; ++l2) v[l2] = xb[n1 * XP1 + l1 + 4 * l2];
    dft<float, true, 8>(v);  // over l2 -> m1
#pragma unroll
    for (int m1 = 1; m1 < 8; ++m1) v[m1] = cmulc(v[m1], t2[l1 * T2P + m1]);  // W_32^{-l1 m1}
    __syncwarp();
#pragma unroll
    for (int m1 = 0; m1 < 8; ++m1) xb[n1 * XP2 + l1 * XQ2 + m1] = v[m1];
    __syncwarp();
    const int j = lane & 3;
    cpx<float> a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        a[i] = xb[n1 * XP2 + i * XQ2 + j];
        b[i] = xb[n1 * XP2 + i * XQ2 + j + 4];
    }
    dft<float, true, 4>(a);  // over l1 -> m2
    dft<float, true, 4>(b);
#pragma unroll
    for (int m2 = 0; m2 < 4; ++m2) {
        v[m2] = a[m2];
        v[4 + m2] = b[m2];
    }
}

// 256-point forward transform (sign -): grid order in -> Z[l + 32 q] in v[q]
__device__ __forceinline__ void fwd256(cpx<float> (&v)[8], cpx<float>* xb,
                                       const cpx<float>* __restrict__ t1,
                                       const cpx<float>* __restrict__ t2, int lane) {
    const int n1 = lane >> 2, j = lane & 3;
    cpx<float> a[4], b[4];
#pragma unroll
    for (int m2 = 0; m2 < 4; ++m2) {
        a[m2] = v[m2];
        b[m2] = v[4 + m2];
    }
    dft<float, false, 4>(a);  // over m2 -> l1
    dft<float, false, 4>(b);
#pragma unroll
    for (int l1 = 1; l1 < 4; ++l1) {
        a[l1] = cmul(a[l1], t2[l1 * T2P + j]);      // W_32^{m1 l1}, m1 = j
        b[l1] = cmul(b[l1], t2[l1 * T2P + j + 4]);  // m1 = j + 4
    }
    __syncwarp();
#pragma unroll
    for (int l1 = 0; l1 < 4; ++l1) {
        xb[n1 * XP2 + l1 * XQ2 + j] = a[l1];
        xb[n1 * XP2 + l1 * XQ2 + j + 4] = b[l1];
    }
    __syncwarp();
    const int l1 = lane & 3;
#pragma unroll
    for (int m1 = 0; m1 < 8; ++m1) v[m1] = xb[n1 * XP2 + l1 * XQ2 + m1];
    dft<float, false, 8>(v);  // over m1 -> l2
#pragma unroll
    for (int l2 = 0; l2 < 8; ++l2) v[l2] = cmul(v[l2], t1[n1 * T1P + l1 + 4 * l2]);  // W_256^{n1 l}
    __syncwarp();
#pragma unroll
    for (int l2 = 0; l2 < 8; ++l2) xb[n1 * XP1 + l1 + 4 * l2] = v[l2];
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = xb[i * XP1 + lane];
    dft<float, false, 8>(v);  // over n1 -> q
}

}  // namespace xw

// Launch: one CTA of NWARP warps per SM (persistent), 208 KB of shared
// memory; warp w of CTA b takes rows b * NWARP + w, then strides by the
// number of warps in the grid.  Rows run over all members of the launch.
template <int N>
__host__ __device__ constexpr size_t xw_smem_bytes() {
    return (size_t)xw::NWARP * sizeof(xw::Smem<N>) +
           (size_t)(N + 8 * xw::T1P + 4 * xw::T2P) * sizeof(cpx<float>) + xw::NWARP * 16;
}

template <int N, bool WRITE_RU>
__global__ void __launch_bounds__(xw::NWARP * 32, 1)
row_nonlin_warp(const Member<float>* __restrict__ mem, const Roles rl,
                const cpx<float>* __restrict__ tw_g, int rows_per, int nrows) {
    static_assert(N == 512, "warp x pass: 256-point half-length transforms");
    using namespace xw;
    using C = cpx<float>;
    constexpr int M = N / 2;
    constexpr int RL = Smem<N>::RL;
    constexpr unsigned ROW_BYTES = RL * sizeof(C);         // 6240
    constexpr unsigned RU_BYTES = N * 3 * sizeof(float);   // 6144
    static_assert(ROW_BYTES % 16 == 0 && RU_BYTES % 16 == 0, "bulk copy sizes");
    static_assert(sizeof(Smem<N>) % 16 == 0, "warp regions stay 16-byte aligned");

    extern __shared__ __align__(128) unsigned char xw_smem_raw[];
    Smem<N>* ws = reinterpret_cast<Smem<N>*>(xw_smem_raw);
    C* tw = reinterpret_cast<C*>(ws + NWARP);  // exp(-2 pi i m / N), m < N
    C* t1 = tw + N;                            // [n1][l] = W_256^{n1 l}, pitch 36
    C* t2 = t1 + 8 * T1P;                      // [l1][m1] = W_32^{l1 m1}, pitch T2P
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(t2 + 4 * T2P);

    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int i = tid; i < N; i += blockDim.x) tw[i] = tw_g[i];
    for (int i = tid; i < 8 * 32; i += blockDim.x) {
        const int n1 = i >> 5, l = i & 31;
        t1[n1 * T1P + l] = tw_g[(2 * n1 * l) % N];
    }
    if (tid < 32) t2[(tid >> 3) * T2P + (tid & 7)] = tw_g[16 * ((tid >> 3) * (tid & 7))];
    if (tid < 2 * NWARP) mbar_init(&bars[tid], 1);
    fence_mbar_init();
    __syncthreads();

    Smem<N>& S = ws[wid];
    // bars[2 w]: the u row in su, bars[2 w + 1]: the w row in sw
    unsigned long long* bar_u = &bars[2 * wid];
    unsigned long long* bar_w = &bars[2 * wid + 1];
    unsigned par_u = 0, par_w = 0;
    const float inv_np = 1.0f / ((float)N * (float)N * (float)N);
    const int gw = blockIdx.x * NWARP + wid, nw = gridDim.x * NWARP;
    auto row_src = [&](int row, int b) -> const C* {
        const int m = row / rows_per;
        const size_t r = (size_t)(row - m * rows_per);
        return mbuf(mem[m], b ? rl.in1 : rl.in0) + r * RL;
    };
    // loads are issued by lane 0 after every lane's earlier reads of the
    // destination (fence: ordered before the async proxy's writes) and after
    // the bulk stores that read it (wait_group.read)
    auto issue = [&](int row, int b) {
        bulk_wait_read();
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) {
            unsigned long long* bb = b ? bar_w : bar_u;
            mbar_expect_tx(bb, ROW_BYTES);
            bulk_load(b ? S.sw : S.su, row_src(row, b), ROW_BYTES, bb);
        }
    };
    if (gw < nrows) {
        issue(gw, 0);
        issue(gw, 1);
    }
    bool ok = true;
    // grid position of register i of the grid side: n = n1 + 8 m1 + 64 m2
    const int n1 = lane >> 2, j = lane & 3;

    for (int row = gw; row < nrows && ok; row += nw) {
        const int m = row / rows_per;
        const size_t r = (size_t)(row - m * rows_per);
        const int next = row + nw;
        C U[3][8], Wv[3][8];
        // u: C2R pre-processing and inverse transforms (su -> U)
        ok = mbar_wait_bounded(bar_u, par_u);
        par_u ^= 1u;
        if (!ok) break;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            if (f == 3) {
                if constexpr (WRITE_RU) {
                    // u(t) in real space, [x][c] interleaved, through su.
                    // Lanes j and j + 2 hold grid pairs 16 apart (96 words,
                    // one bank): lanes j >= 2 store their odd x first, so
                    // that each store's 32 words fall on distinct banks
                    float* rr = reinterpret_cast<float*>(S.su);
                    const int hi = j >= 2 ? 1 : 0;
                    __syncwarp();
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int n = n1 + 8 * (i < 4 ? j : j + 4) + 64 * (i & 3);
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            rr[(2 * n + hi) * 3 + c] = hi ? U[c][i].y : U[c][i].x;
                            rr[(2 * n + 1 - hi) * 3 + c] = hi ? U[c][i].x : U[c][i].y;
                        }
                    }
                    fence_proxy_async();  // this lane's writes, visible to the bulk copy
                    __syncwarp();
                    if (lane == 0) {
                        bulk_store(mreal(mem[m], rl.rout) + r * (N * 3), rr, RU_BYTES);
                        bulk_commit();
                    }
                }
                // w: wait for its row
                ok = mbar_wait_bounded(bar_w, par_w);
                par_w ^= 1u;
                if (!ok) break;
            }
            const C* st = f < 3 ? S.su : S.sw;
            const int c = f % 3;
            C v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = lane + 32 * q;
                const C a = st[3 * k + c];
                if (k == 0) {
                    const float x0 = a.x, xm = st[3 * M + c].x;
                    v[q] = mk<float>(x0 + xm, x0 - xm);
                } else {
                    v[q] = c2r_lo(a, st[3 * (M - k) + c], tw[k]);
                }
            }
            xw::inv256(v, S.x, t1, t2, lane);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (f < 3) U[c][i] = v[i];
                else Wv[c][i] = v[i];
            }
        }
        if (!ok) break;
        // su is free: the next row's u streams in during the rest of this row
        if (next < nrows) issue(next, 0);
        // u x w / N^3 at every grid point (two per complex word)
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            C p[3];
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                const int c1 = (cc + 1) % 3, c2 = (cc + 2) % 3;
                const float tx = U[c1][i].x * Wv[c2][i].x - U[c2][i].x * Wv[c1][i].x;
                const float ty = U[c1][i].y * Wv[c2][i].y - U[c2][i].y * Wv[c1][i].y;
                p[cc] = mk<float>(tx * inv_np, ty * inv_np);
            }
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) U[cc][i] = p[cc];
        }
        // forward transforms and R2C post-processing into sw (free since the
        // w transforms)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            C v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = U[c][i];
            xw::fwd256(v, S.x, t1, t2, lane);
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 8; ++q) S.x[lane + 32 * q] = v[q];  // natural order
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = lane + 32 * q;
                if (k == 0) {
                    const C z0 = v[0];
                    S.sw[c] = mk<float>(z0.x + z0.y, 0.f);
                    S.sw[3 * M + c] = mk<float>(z0.x - z0.y, 0.f);
                } else {
                    S.sw[3 * k + c] = r2c_lo(v[q], S.x[M - k], tw[k]);
                }
            }
        }
        // padding points of the output row carry zeros
        if (lane < RL - 3 * (M + 1)) S.sw[3 * (M + 1) + lane] = zero_c<float>();
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) {
            bulk_store(mbuf(mem[m], rl.out0) + r * RL, S.sw, ROW_BYTES);
            bulk_commit();
        }
        // the next row's w once the store has read sw
        if (next < nrows) issue(next, 1);
    }
    bulk_wait_all();
}


// ---------------------------------------------------------------------------
// The same x pass for N = 64, 128 and 256 (FP32): G = N / 16 lanes per row
// and 32 / G rows per warp (8 rows at 64^3, 4 at 128^3, 2 at 256^3), so that
// every lane still keeps eight values of each transform.  A row's M = N / 2 = 8 G point
// transform is a radix-8 butterfly over the lane's registers (Z[l + G q],
// q = 0..7), a twiddle W_M^(n1 l), and a G-point transform over the row's
// lanes through the warp's exchange buffer:
//   G = 4:  one exchange [n1][l] (pitch 9), lane l then takes n1 = l and
//           l + 4: two radix-4 over l;
//   G = 8:  one exchange [n1][l] (pitch 9), radix 8 over l;
//   G = 16: l = l1 + 2 l2: exchange [n1][l] (pitch 18), radix 8 over l2,
//           twiddle W_16^(l1 m1), exchange [n1][l1][m1] (pitches 18, 9),
//           radix 2 over l1.
// The pitches put the 16 lanes of every half-warp on distinct banks for the
// 8-byte accesses of each exchange (rows of a 128^3 warp are 72 apart, 8
// modulo 16, and of a 64^3 warp 68, 4 modulo 16, so the rows sharing a
// half-warp also fall apart).  The forward
// transform retraces the inverse's steps, so both keep the grid points in
// the same lane and register order:
//   G = 4:  lane l, register 4 e + i: n = l + 4 e + 8 i;
//   G = 8:  lane l of a row, register i: grid pair n = l + 8 i;
//   G = 16: lane 2 n1 + j, register i + 4 m2 (i < 4): n = n1 + 8 (j + 2 i) + 64 m2.
// The warp's rows are consecutive in HBM: one TMA bulk copy brings its u
// rows, one its w rows, one store takes the output rows (and in stage 1 one
// the real-velocity rows).
namespace xwg {

constexpr int NWARP = 12;  // warps per CTA, one CTA per SM

template <int N>
struct Cfg {
    static constexpr int M = N / 2;
    static constexpr int G = M / 8;                // lanes per row
    static constexpr int Q = 32 / G;               // rows per warp
    static constexpr int RL = (N / 2 + 4) * 3;     // padded interleaved row (complex)
    static constexpr int XB = G == 4 ? 68 : (G == 8 ? 72 : 144);  // exchange block per row
    static constexpr int P1 = G == 16 ? 18 : 9;                   // [n1][l] pitch
    // twiddle table [n1][l] pitch: the forward transform of G = 16 reads it
    // with lane 2 n1 + l1 at column l1 + 2 l2, which a pitch of 16 would put
    // on one bank for all eight n1
    static constexpr int TP = G == 16 ? 18 : G;
};

template <int N>
struct Smem {
    cpx<float> su[Cfg<N>::Q * Cfg<N>::RL];  // u rows in, real u rows out
    cpx<float> sw[Cfg<N>::Q * Cfg<N>::RL];  // w rows in, output rows out
    cpx<float> x[Cfg<N>::Q * Cfg<N>::XB];   // exchanges, one block per row
};

// inverse (sign +): Z[l + G q] in v[q] -> grid order (layout above)
template <int N>
__device__ __forceinline__ void inv_g(cpx<float> (&v)[8], cpx<float>* xb,
                                      const cpx<float>* __restrict__ t1, int l) {
    constexpr int G = Cfg<N>::G, P1 = Cfg<N>::P1;
    dft<float, true, 8>(v);  // over q -> n1
#pragma unroll
    for (int n1 = 1; n1 < 8; ++n1) v[n1] = cmulc(v[n1], t1[n1 * Cfg<N>::TP + l]);  // W_M^{-n1 l}
    __syncwarp();
#pragma unroll
    for (int n1 = 0; n1 < 8; ++n1) xb[n1 * P1 + l] = v[n1];
    __syncwarp();
    if constexpr (G == 4) {
        cpx<float> a[4], b[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            a[k] = xb[l * P1 + k];        // n1 = l
            b[k] = xb[(l + 4) * P1 + k];  // n1 = l + 4
        }
        dft<float, true, 4>(a);  // over l -> n2
        dft<float, true, 4>(b);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            v[i] = a[i];
            v[4 + i] = b[i];
        }
    } else if constexpr (G == 8) {
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = xb[l * P1 + k];  // lane l now takes n1 = l
        dft<float, true, 8>(v);                            // over l -> n2
    } else {
        const int n1 = l >> 1, l1 = l & 1;
#pragma unroll
        for (int l2 = 0; l2 < 8; ++l2) v[l2] = xb[n1 * P1 + l1 + 2 * l2];
        dft<float, true, 8>(v);  // over l2 -> m1
        if (l1) {
#pragma unroll
            for (int m1 = 1; m1 < 8; ++m1) v[m1] = mul_wr<float, true, 16>(v[m1], m1);  // W_16^{-m1}
        }
        __syncwarp();
#pragma unroll
        for (int m1 = 0; m1 < 8; ++m1) xb[n1 * P1 + 9 * l1 + m1] = v[m1];
        __syncwarp();
        const int j = l & 1;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const cpx<float> a = xb[n1 * P1 + j + 2 * i];
            const cpx<float> b = xb[n1 * P1 + 9 + j + 2 * i];
            v[i] = a + b;  // m2 = 0
            v[i + 4] = a - b;  // m2 = 1
        }
    }
}

// forward (sign -): grid order in -> Z[l + G q] in v[q]
template <int N>
__device__ __forceinline__ void fwd_g(cpx<float> (&v)[8], cpx<float>* xb,
                                      const cpx<float>* __restrict__ t1, int l) {
    constexpr int G = Cfg<N>::G, P1 = Cfg<N>::P1;
    if constexpr (G == 4) {
        cpx<float> a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            a[i] = v[i];      // n1 = l
            b[i] = v[4 + i];  // n1 = l + 4
        }
        dft<float, false, 4>(a);  // over n2 -> k
        dft<float, false, 4>(b);
#pragma unroll
        for (int k = 1; k < 4; ++k) {
            a[k] = cmul(a[k], t1[l * Cfg<N>::TP + k]);        // W_M^{n1 k}
            b[k] = cmul(b[k], t1[(l + 4) * Cfg<N>::TP + k]);
        }
        __syncwarp();
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            xb[l * P1 + k] = a[k];
            xb[(l + 4) * P1 + k] = b[k];
        }
    } else if constexpr (G == 8) {
        dft<float, false, 8>(v);  // over n2 -> k (lane = n1)
#pragma unroll
        for (int k = 1; k < 8; ++k) v[k] = cmul(v[k], t1[k * Cfg<N>::TP + l]);  // W_M^{n1 k}, n1 = l
        __syncwarp();
#pragma unroll
        for (int k = 0; k < 8; ++k) xb[l * P1 + k] = v[k];
    } else {
        const int n1 = l >> 1, j = l & 1;
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const cpx<float> a = v[i], b = v[i + 4];
            xb[n1 * P1 + j + 2 * i] = a + b;                                           // l1 = 0
            xb[n1 * P1 + 9 + j + 2 * i] = mul_wr<float, false, 16>(a - b, j + 2 * i);  // l1 = 1
        }
        __syncwarp();
        const int l1 = l & 1;
#pragma unroll
        for (int m1 = 0; m1 < 8; ++m1) v[m1] = xb[n1 * P1 + 9 * l1 + m1];
        dft<float, false, 8>(v);  // over m1 -> l2
#pragma unroll
        for (int l2 = 0; l2 < 8; ++l2) v[l2] = cmul(v[l2], t1[n1 * Cfg<N>::TP + l1 + 2 * l2]);  // W_M^{n1 k}
        __syncwarp();
#pragma unroll
        for (int l2 = 0; l2 < 8; ++l2) xb[n1 * P1 + l1 + 2 * l2] = v[l2];
    }
    __syncwarp();
#pragma unroll
    for (int n1 = 0; n1 < 8; ++n1) v[n1] = xb[n1 * P1 + l];  // lane l takes spectrum column l
    dft<float, false, 8>(v);  // over n1 -> q
}

// grid pair index of register i of lane l (layout above)
template <int N>
__device__ __forceinline__ int grid_pair(int l, int i) {
    if constexpr (Cfg<N>::G == 4) return l + 4 * (i >> 2) + 8 * (i & 3);
    else if constexpr (Cfg<N>::G == 8) return l + 8 * i;
    else return (l >> 1) + 8 * ((l & 1) + 2 * (i & 3)) + 64 * (i >> 2);
}

}  // namespace xwg

template <int N>
__host__ __device__ constexpr size_t xwg_smem_bytes() {
    return (size_t)xwg::NWARP * sizeof(xwg::Smem<N>) +
           (size_t)(N + 8 * xwg::Cfg<N>::TP) * sizeof(cpx<float>) + xwg::NWARP * 16;
}

template <int N, bool WRITE_RU>
__global__ void __launch_bounds__(xwg::NWARP * 32, 1)
row_nonlin_wg(const Member<float>* __restrict__ mem, const Roles rl,
              const cpx<float>* __restrict__ tw_g, int rows_per, int nrows) {
    static_assert(N == 64 || N == 128 || N == 256, "warp-group x pass: 32- to 128-point half-length transforms");
    using namespace xwg;
    using C = cpx<float>;
    using CF = Cfg<N>;
    constexpr int M = CF::M, G = CF::G, Q = CF::Q, RL = CF::RL, XB = CF::XB;
    constexpr unsigned BLOCK_BYTES = Q * RL * sizeof(C);             // Q rows
    constexpr unsigned RU_BYTES = Q * N * 3 * sizeof(float);         // Q real rows
    static_assert(BLOCK_BYTES % 16 == 0 && RU_BYTES % 16 == 0, "bulk copy sizes");
    static_assert(sizeof(Smem<N>) % 16 == 0, "warp regions stay 16-byte aligned");
    static_assert(RU_BYTES <= BLOCK_BYTES, "real rows staged in su");

    extern __shared__ __align__(128) unsigned char xwg_smem_raw[];
    Smem<N>* ws = reinterpret_cast<Smem<N>*>(xwg_smem_raw);
    C* tw = reinterpret_cast<C*>(ws + NWARP);  // exp(-2 pi i m / N), m < N
    C* t1 = tw + N;                            // [n1][l] = W_M^{n1 l}, pitch TP
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(t1 + 8 * CF::TP);

    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int i = tid; i < N; i += blockDim.x) tw[i] = tw_g[i];
    for (int i = tid; i < 8 * G; i += blockDim.x) {
        const int n1 = i / G, l = i % G;
        t1[n1 * CF::TP + l] = tw_g[(2 * n1 * l) % N];
    }
    if (tid < 2 * NWARP) mbar_init(&bars[tid], 1);
    fence_mbar_init();
    __syncthreads();

    Smem<N>& S = ws[wid];
    unsigned long long* bar_u = &bars[2 * wid];
    unsigned long long* bar_w = &bars[2 * wid + 1];
    unsigned par_u = 0, par_w = 0;
    const float inv_np = 1.0f / ((float)N * (float)N * (float)N);
    const int nblk = nrows / Q;  // Q divides N^2: blocks never straddle members
    const int gw = blockIdx.x * NWARP + wid, nw = gridDim.x * NWARP;
    // this lane's row in the block and its lane in the row; G = 8 puts rows
    // 0, 2 (and 1, 3) in one half-warp: 2 RL apart (8 modulo 16), so the
    // strided row accesses of the two rows (3 k + c) fall on distinct banks
    const int grp = lane / G;
    const int rr_ = G == 8 ? (grp & 1) * 2 + (grp >> 1) : grp;
    const int l = lane % G;
    C* xb = S.x + grp * XB;      // exchange block of this lane group
    auto block_src = [&](int blk, int b) -> const C* {
        const int row0 = blk * Q;
        const int m = row0 / rows_per;
        const size_t r = (size_t)(row0 - m * rows_per);
        return mbuf(mem[m], b ? rl.in1 : rl.in0) + r * RL;
    };
    auto issue = [&](int blk, int b) {
        bulk_wait_read();
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) {
            unsigned long long* bb = b ? bar_w : bar_u;
            mbar_expect_tx(bb, BLOCK_BYTES);
            bulk_load(b ? S.sw : S.su, block_src(blk, b), BLOCK_BYTES, bb);
        }
    };
    if (gw < nblk) {
        issue(gw, 0);
        issue(gw, 1);
    }
    bool ok = true;

    for (int blk = gw; blk < nblk && ok; blk += nw) {
        const int row0 = blk * Q;
        const int m = row0 / rows_per;
        const size_t r0 = (size_t)(row0 - m * rows_per);
        const int next = blk + nw;
        C U[3][8], Wv[3][8];
        ok = mbar_wait_bounded(bar_u, par_u);
        par_u ^= 1u;
        if (!ok) break;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            if (f == 3) {
                if constexpr (WRITE_RU) {
                    // u(t) in real space, [x][c] interleaved, rows of N * 3
                    // floats one after the other, through su
                    float* rr = reinterpret_cast<float*>(S.su) + rr_ * (N * 3);
                    __syncwarp();
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int n = grid_pair<N>(l, i);
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            rr[(2 * n) * 3 + c] = U[c][i].x;
                            rr[(2 * n + 1) * 3 + c] = U[c][i].y;
                        }
                    }
                    fence_proxy_async();
                    __syncwarp();
                    if (lane == 0) {
                        bulk_store(mreal(mem[m], rl.rout) + r0 * (N * 3), S.su, RU_BYTES);
                        bulk_commit();
                    }
                }
                ok = mbar_wait_bounded(bar_w, par_w);
                par_w ^= 1u;
                if (!ok) break;
            }
            const C* st = (f < 3 ? S.su : S.sw) + rr_ * RL;
            const int c = f % 3;
            C v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = l + G * q;
                const C a = st[3 * k + c];
                if (k == 0) {
                    const float x0 = a.x, xm = st[3 * M + c].x;
                    v[q] = mk<float>(x0 + xm, x0 - xm);
                } else {
                    v[q] = c2r_lo(a, st[3 * (M - k) + c], tw[k]);
                }
            }
            inv_g<N>(v, xb, t1, l);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (f < 3) U[c][i] = v[i];
                else Wv[c][i] = v[i];
            }
        }
        if (!ok) break;
        // su is free: the next block's u streams in during the rest of this one
        if (next < nblk) issue(next, 0);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            C p[3];
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) {
                const int c1 = (cc + 1) % 3, c2 = (cc + 2) % 3;
                const float tx = U[c1][i].x * Wv[c2][i].x - U[c2][i].x * Wv[c1][i].x;
                const float ty = U[c1][i].y * Wv[c2][i].y - U[c2][i].y * Wv[c1][i].y;
                p[cc] = mk<float>(tx * inv_np, ty * inv_np);
            }
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) U[cc][i] = p[cc];
        }
        C* so = S.sw + rr_ * RL;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            C v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = U[c][i];
            fwd_g<N>(v, xb, t1, l);
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 8; ++q) xb[l + G * q] = v[q];  // natural order
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = l + G * q;
                if (k == 0) {
                    const C z0 = v[0];
                    so[c] = mk<float>(z0.x + z0.y, 0.f);
                    so[3 * M + c] = mk<float>(z0.x - z0.y, 0.f);
                } else {
                    so[3 * k + c] = r2c_lo(v[q], xb[M - k], tw[k]);
                }
            }
        }
        // padding points of the output rows carry zeros
        for (int e = l; e < RL - 3 * (M + 1); e += G) so[3 * (M + 1) + e] = zero_c<float>();
        fence_proxy_async();
        __syncwarp();
        if (lane == 0) {
            bulk_store(mbuf(mem[m], rl.out0) + r0 * RL, S.sw, BLOCK_BYTES);
            bulk_commit();
        }
        if (next < nblk) issue(next, 1);
    }
    bulk_wait_all();
}

}  // namespace bfg
