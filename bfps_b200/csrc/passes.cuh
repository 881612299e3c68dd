// Fused HBM passes of the IF-RK3 vorticity step (sm_100a).
//
// Device layouts (units of "points" = 3 complex numbers, one per component):
//   state  S: [ky][kz][kx]  point (ky*N + kz)*NXP + kx   (reference layout,
//                                                       rows padded to NXP)
//   work   W: [z][y][kx]    point (z*N + y)*NXP + kx     (after z / y passes)
//   real   R: [z][y][x][c]  scalar ((z*N + y)*N + x)*3 + c (unpadded)
// kx runs over NXV = N/2+1 valid columns; NXP = N/2+4 keeps every row
// 32-byte aligned.
//
// One RK stage is five launches:
//   IZ  (col pass, a=ky, FFT over kz)  S -> W : u^ = i k x w^ / k^2 (+ w^)
//   IY  (col pass, a=z,  FFT over ky)  W -> W
//   X   (row pass, one (z,y) row)      W -> W : C2R of u, w; u x w / N^3;
//                                               R2C of the product
//   FY  (col pass, a=z,  FFT over y)   W -> W
//   FZ  (col pass, a=ky, FFT over z)   W -> S : dealias, i k x, forcing,
//                                               force_divfree, RK update
// Reference: vorticity_equation.cpp:206-239 (compute_velocity), :290-356
// (omega_nonlin), :358-439 (step); kspace.cpp:461-519 (dealias,
// force_divfree).
#pragma once
#include "fft.cuh"

namespace bfg {

struct KParams {
    int nxv;           // N/2 + 1
    int nxp;           // padded row length (points)
    double dkx, dky, dkz;
    double kM2;
    int dealias;       // 0 two-thirds, 1 smooth
    double inv_dk2;    // 1 / dk^2 (smooth filter key)
    int nfilt;         // filter table length
    int forcing;       // 0 none, 1 linear, 2 Kolmogorov
    double famp, fk0, fk1;
    int fmode;
    double dt;
};

// One DNS instance as the kernels see it: parameters, its five complex
// buffers (0 w0 = state, 1 v1, 2 v2, 3 wa, 4 wb), real velocity and tables.
// A launch covers an array of members of the same N.
template <typename T>
struct Member {
    KParams kp;
    cpx<T>* buf[5];
    T* ru;
    const T* filt;
    const T* fac;
};
enum BufIdx { B_W0 = 0, B_V1 = 1, B_V2 = 2, B_WA = 3, B_WB = 4, B_RU = 5, B_NONE = -1 };
// which buffers play which part in one launch (B_* indices; rout / rin may
// also name a complex buffer used as real scratch)
struct Roles {
    int in0, in1, out0, out1, v0, vp, fsrc, rout, rin;
};
__host__ __device__ inline Roles roles(int in0, int in1, int out0, int out1, int v0 = B_NONE,
                                       int vp = B_NONE, int fsrc = B_NONE, int rout = B_NONE,
                                       int rin = B_NONE) {
    Roles r;
    r.in0 = in0; r.in1 = in1; r.out0 = out0; r.out1 = out1;
    r.v0 = v0; r.vp = vp; r.fsrc = fsrc; r.rout = rout; r.rin = rin;
    return r;
}
template <typename T>
__device__ __forceinline__ cpx<T>* mbuf(const Member<T>& m, int i) {
    return i >= 0 && i < 5 ? m.buf[i] : nullptr;
}
template <typename T>
__device__ __forceinline__ T* mreal(const Member<T>& m, int i) {
    return i == B_RU ? m.ru : (i >= 0 && i < 5 ? reinterpret_cast<T*>(m.buf[i]) : nullptr);
}

enum ColMode {
    CM_IZ_VEL = 0,    // S -> (u^, w^) in W
    CM_IZ_PLAIN = 1,  // S -> W (inverse over kz)
    CM_Y_INV2 = 2,    // W, W in place (inverse over ky)
    CM_Y_INV1 = 3,
    CM_Y_FWD1 = 4,    // W in place (forward over y)
    CM_FZ_RK1 = 5,    // W -> S with the stage-1 update
    CM_FZ_RK2 = 6,
    CM_FZ_RK3 = 7,
    CM_FZ_PLAIN = 8,  // W -> S (forward over z)
    CM_IZ_U = 9,      // S -> u^ in W (inverse over kz of compute_velocity)
};

__host__ __device__ constexpr int col_nb(int mode) {
    return (mode == CM_IZ_VEL || mode == CM_Y_INV2) ? 2 : 1;
}
__host__ __device__ constexpr int col_nbin(int mode) { return mode == CM_Y_INV2 ? 2 : 1; }
__host__ __device__ constexpr bool col_inverse(int mode) {
    return mode <= CM_Y_INV1 || mode == CM_IZ_U;
}
__host__ __device__ constexpr int pow2floor(int v) {
    return v < 2 ? 1 : 2 * pow2floor(v / 2);
}
constexpr int SMEM_BUDGET = 220 * 1024;  // dynamic shared memory per SM we plan for
__host__ __device__ constexpr bool col_fz(int mode) { return mode >= 5 && mode <= 7; }
// Schedules of a column pass.  Each pass is compiled in two schedules and
// the one used is chosen per (device, grid size, precision, pass) by the
// autotuner (bfg_autotune), schedule 0 where nothing was tuned:
//   0: two 256-thread CTAs per SM with one tile buffer each (one CTA's
//      barrier waits, loads and epilogue are covered by the other CTA's
//      work), 32-point butterflies in FP32 (two stages at 512^3 instead of
//      three);
//   1: one 512-thread CTA per SM with two tile buffers (the next tile loads
//      while this one is transformed), radix cap 8.
// Measured at 512^3 FP32, schedule 0 against 1: IZ 1.33 / 1.49, IY 1.60 /
// 1.79, FY 0.75 / 0.88, FZ 1.86 / 2.07 ms.  FP64 keeps a radix cap of 8 in
// both (twice the registers per value).
template <typename T, int MODE, int S>
__host__ __device__ constexpr int col_mr() {
    return col_max_radix<T, S == 0>();
}

// tile row pitch (complex) for a tile of TKX kx columns: keeps every row
// 16-byte aligned and breaks the worst bank patterns
template <typename T, int NB>
__host__ __device__ constexpr int col_pitch_for(int tkx) {
    return NB * 3 * tkx + (sizeof(T) == 4 ? 2 : 1);
}
// number of RK operand arrays the FZ epilogue reads (v0, and v_prev for
// stages 2-3).  They are read from global memory after an L2 prefetch at
// the start of the tile, not staged in shared memory: staging them took the
// shared memory of a tile twice as wide (4 instead of 8 kx columns at 512^3
// FP32), and the wider tile measured 19 % faster (2.42 -> 1.97 ms).
__host__ __device__ constexpr int col_nrk(int mode) {
    return mode == CM_FZ_RK1 ? 1 : ((mode == CM_FZ_RK2 || mode == CM_FZ_RK3) ? 2 : 0);
}
// Launch shape of a column pass (its schedule, above): schedule 0 runs two
// CTAs per SM where such a tile still has rows of at least 96 bytes, else
// one CTA with two buffers.
// shared memory: nbuf tile buffers + twiddles
template <typename T, int N, int MODE>
__host__ __device__ constexpr size_t col_bytes_nb(int tkx, int nbuf) {
    return (size_t)(nbuf * N * col_pitch_for<T, col_nb(MODE)>(tkx) + N) * sizeof(cpx<T>);
}
// kx columns per tile: the widest power of two (<= 16) within the budget
template <typename T, int N, int MODE>
__host__ __device__ constexpr int col_tkx_fit(int tkx, int nbuf, size_t budget) {
    return (tkx <= 1 || col_bytes_nb<T, N, MODE>(tkx, nbuf) <= budget)
               ? tkx
               : col_tkx_fit<T, N, MODE>(tkx / 2, nbuf, budget);
}
// one tile over all N/2+1 kx columns where it fits (small grids): otherwise
// the Nyquist column kx = N/2 gets a tile of its own, which costs a full tile
template <typename T, int N, int MODE>
__host__ __device__ constexpr int col_tkx_sel(int nbuf, size_t budget) {
    return col_bytes_nb<T, N, MODE>(N / 2 + 1, nbuf) <= budget
               ? N / 2 + 1
               : col_tkx_fit<T, N, MODE>(16, nbuf, budget);
}
template <typename T, int N, int MODE, int S>
__host__ __device__ constexpr bool col_two() {
    return S == 0 && col_tkx_sel<T, N, MODE>(1, SMEM_BUDGET / 2) * 3 * (int)sizeof(cpx<T>) >= 96;
}
template <typename T, int N, int MODE, int S>
__host__ __device__ constexpr int col_threads() { return col_two<T, N, MODE, S>() ? 256 : 512; }
template <typename T, int N, int MODE, int S>
__host__ __device__ constexpr int col_ctas() { return col_two<T, N, MODE, S>() ? 2 : 1; }
// From 1024-point columns up, schedule 1 keeps one buffer: two buffers of
// such columns leave tiles of one or two kx columns (24-48-byte row
// segments), one buffer twice or four times as wide.
template <typename T, int N, int MODE, int S>
__host__ __device__ constexpr int col_nbuf() {
    return col_two<T, N, MODE, S>() ? 1 : ((S == 1 && N >= 1024) ? 1 : 2);
}
template <typename T, int N, int MODE, int S>
__host__ __device__ constexpr int col_tkx() {
    return col_two<T, N, MODE, S>() ? col_tkx_sel<T, N, MODE>(1, SMEM_BUDGET / col_ctas<T, N, MODE, S>())
                                 : col_tkx_sel<T, N, MODE>(col_nbuf<T, N, MODE, S>(), SMEM_BUDGET);
}
template <typename T, int N, int MODE, int S>
__host__ __device__ constexpr int col_pitch() {
    return col_pitch_for<T, col_nb(MODE)>(col_tkx<T, N, MODE, S>());
}
template <typename T, int N, int MODE, int S>
__host__ __device__ constexpr size_t col_smem_bytes() {
    return col_bytes_nb<T, N, MODE>(col_tkx<T, N, MODE, S>(), col_nbuf<T, N, MODE, S>());
}

template <int N>
__device__ __forceinline__ double kwrap(int i, double dk) {
    return dk * (double)(i <= N / 2 ? i : i - N);
}

// i k x a  (vorticity_equation.cpp:323-336)
template <typename A>
__device__ __forceinline__ void curl(A kx, A ky, A kz, const cpx<A>* a, cpx<A>* t) {
    t[0] = mk<A>(-(ky * a[2].y - kz * a[1].y), (ky * a[2].x - kz * a[1].x));
    t[1] = mk<A>(-(kz * a[0].y - kx * a[2].y), (kz * a[0].x - kx * a[2].x));
    t[2] = mk<A>(-(kx * a[1].y - ky * a[0].y), (kx * a[1].x - ky * a[0].x));
}

// kspace::force_divfree on one mode (kspace.cpp:487-519), k2 > 0
template <typename A>
__device__ __forceinline__ void divfree(A kx, A ky, A kz, A inv_k2, cpx<A>* a) {
    const A tr = (kx * a[0].x + ky * a[1].x + kz * a[2].x) * inv_k2;
    const A ti = (kx * a[0].y + ky * a[1].y + kz * a[2].y) * inv_k2;
    a[0].x -= tr * kx; a[0].y -= ti * kx;
    a[1].x -= tr * ky; a[1].y -= ti * ky;
    a[2].x -= tr * kz; a[2].y -= ti * kz;
}

template <typename T>
__device__ __forceinline__ cpx<T> zero_c() { return mk<T>((T)0, (T)0); }

// 1 / k^2 in the storage precision: correctly rounded in FP64; in FP32 the
// reciprocal of k^2 rounded to FP32 (within an FP32 ulp of the FP64 value
// rounded, without the FP64 reciprocal sequence)
template <typename T>
__device__ __forceinline__ T inv_k2(double k2) {
    if constexpr (sizeof(T) == 4) return __frcp_rn(__double2float_rn(k2));
    else return (T)__drcp_rn(k2);
}

__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// global row of tile row l (input side) / lo (output side) for a pass mode
template <int N, int MODE>
__device__ __forceinline__ size_t col_in_row(int a, int l) {
    if (MODE == CM_IZ_VEL || MODE == CM_IZ_PLAIN || MODE == CM_IZ_U) return (size_t)a * N + l;  // S[ky=a][kz=l]
    if (MODE >= CM_FZ_RK1 && MODE <= CM_FZ_PLAIN) return (size_t)l * N + a;                   // W[z=l][ky=a]
    return (size_t)a * N + l;                                                                // W[z=a][y=l]
}
template <int N, int MODE>
__device__ __forceinline__ size_t col_out_row(int a, int lo) {
    if (MODE == CM_IZ_VEL || MODE == CM_IZ_PLAIN || MODE == CM_IZ_U) return (size_t)lo * N + a;  // W[z=lo][ky=a]
    return (size_t)a * N + lo;                                                                 // S or W[z=a]
}

// ---------------------------------------------------------------------------
// Strided-axis pass.  Persistent CTAs (grid = SMs x CTAs per SM) walk the
// tiles t = (a, kx-tile), kx-tile fastest; each tile (N rows x TKX kx
// columns x 3 components x NB buffers) is streamed into shared memory with
// 16-byte cp.async, while the other CTA on the SM (schedule 0) or the other
// tile buffer (schedule 1) keeps the SM busy.  (One TMA bulk copy per tile
// row, 96-192 bytes each, measured slower: IY 1.60 -> 1.81 ms at 512^3.)
// fac: per-axis integrating-factor tables, 3 factors x (NXV + N + N):
//      [f][0..NXV) kx, [f][NXV..NXV+N) ky, [f][NXV+N..NXV+2N) kz, where
//      f = 0: exp(-nu k^2 dt), 1: exp(-nu k^2 dt/2), 2: exp(+nu k^2 dt/2)
//      per axis (their product over the axes is the factor of k^2).
// FZ epilogue for one mode (l = kz, ix): dealias, i k x, forcing,
// force_divfree, RK update of stage MODE (vorticity_equation.cpp:290-437)
// What an epilogue mode needs from its kx column and the tile's ky: computed
// once per column (a thread keeps one column over its modes).
template <typename T>
struct FzCol {
    double kx, ky, kxy2;  // kx, ky, kx^2 + ky^2
    T kxT, kyT;
    T fxy0, fxy1;         // kx and ky parts of the integrating factors
    double lo, hi;        // forcing band on k2 (see fz_point)
};
template <typename T, int N, int MODE>
__device__ __forceinline__ FzCol<T> fz_col(const KParams& kp, const T* __restrict__ fac, int a,
                                           int ix, double ky) {
    FzCol<T> fc;
    fc.kx = (double)ix * kp.dkx;
    fc.ky = ky;
    fc.kxy2 = fc.kx * fc.kx + ky * ky;
    fc.kxT = (T)fc.kx;
    fc.kyT = (T)ky;
    const int nxv = kp.nxv, nfac = nxv + 2 * N;
    const int s0 = MODE == CM_FZ_RK1 ? 0 : 1;
    fc.fxy0 = fac[s0 * nfac + ix] * fac[s0 * nfac + nxv + a];
    fc.fxy1 = MODE == CM_FZ_RK2 ? fac[2 * nfac + ix] * fac[2 * nfac + nxv + a] : (T)0;
    // the band test on |k| = sqrt(k2), taken only where k2 is near the band
    // (the margin keeps every mode the exact test accepts)
    fc.lo = kp.fk0 > 0.0 ? kp.fk0 * kp.fk0 * (1.0 - 1e-12) : -1.0;
    fc.hi = kp.fk1 * kp.fk1 * (1.0 + 1e-12);
    return fc;
}

template <typename T, int N, int MODE, int S>
__device__ __forceinline__ void fz_point(const KParams& kp, const cpx<T>* tile, int PR, int a, int l,
                                         int ix, int col, const FzCol<T>& fc, const cpx<T>* v0,
                                         const cpx<T>* vp, size_t pt, const T* __restrict__ filt,
                                         const T* __restrict__ fac, const cpx<T>* __restrict__ fsrc,
                                         cpx<T>* out0) {
    const int nxv = kp.nxv;
    const double kz = kwrap<N>(l, kp.dkz);
    const double kx = fc.kx, ky = fc.ky;
    const double k2 = fc.kxy2 + kz * kz;
    const int p = dif_position<N, col_mr<T, MODE, S>()>(l);
    cpx<T> nl[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) nl[c] = tile[p * PR + col * 3 + c];
    // dealias (kspace.cpp:461-485)
    if (kp.dealias == 1) {
        int key = (int)rint(k2 * kp.inv_dk2);
        key = key < kp.nfilt ? key : kp.nfilt - 1;
        const T f = filt[key];
#pragma unroll
        for (int c = 0; c < 3; ++c) nl[c] = scale(nl[c], f);
    } else if (k2 >= kp.kM2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) nl[c] = zero_c<T>();
    }
    // i k x (vorticity_equation.cpp:323-350)
    cpx<T> tt[3];
    const T kzT = (T)kz;
    curl<T>(fc.kxT, fc.kyT, kzT, nl, tt);
    // forcing (vorticity_equation.cpp:241-288), factor 1
    if (kp.forcing == 1) {
        if (k2 >= fc.lo && k2 <= fc.hi && kp.fk0 <= sqrt(k2) && kp.fk1 >= sqrt(k2)) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const cpx<T> fv = fsrc[pt * 3 + c];
                tt[c].x += (T)(kp.famp * (double)fv.x);
                tt[c].y += (T)(kp.famp * (double)fv.y);
            }
        }
    } else if (kp.forcing == 2) {
        if (ix == 0 && l == 0) {
            if (a == kp.fmode) tt[2].x -= (T)(kp.famp / 2);
            if (a == N - kp.fmode) tt[2].x -= (T)(kp.famp / 2);
        }
    }
    // force_divfree on the nonlinear term; zero mode cleared
    const bool kzero = (a == 0 && l == 0 && ix == 0);
    const T ik2 = inv_k2<T>(k2);
    if (k2 > 0.0) divfree<T>(fc.kxT, fc.kyT, kzT, ik2, tt);
    if (kzero) {
#pragma unroll
        for (int c = 0; c < 3; ++c) tt[c] = zero_c<T>();
    }
    // RK update (vorticity_equation.cpp:366-434), only for k2 <= kM2.  The
    // RK operands are read only where they are used: outside kM2 stages 1-2
    // write zero and stage 3 keeps v0 (about half of the modes, and the
    // whole of many tiles' rows, lie outside the smooth filter's sphere)
    const bool inside = k2 <= kp.kM2;
    const T dt = (T)kp.dt;
    cpx<T> o[3];
    const int nfac = nxv + 2 * N;
    if (MODE == CM_FZ_RK1) {
        if (inside) {
            const T f0 = fc.fxy0 * fac[nxv + N + l];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const cpx<T> a0 = v0[c];
                o[c] = mk<T>((a0.x + dt * tt[c].x) * f0, (a0.y + dt * tt[c].y) * f0);
            }
        } else {
#pragma unroll
            for (int c = 0; c < 3; ++c) o[c] = zero_c<T>();
        }
    } else if (MODE == CM_FZ_RK2) {
        if (inside) {
            const T f0 = fc.fxy0 * fac[nfac + nxv + N + l];
            const T f1 = fc.fxy1 * fac[2 * nfac + nxv + N + l];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const cpx<T> a0 = v0[c], ap = vp[c];
                o[c] = mk<T>((3 * a0.x * f0 + (ap.x + dt * tt[c].x) * f1) * (T)0.25,
                             (3 * a0.y * f0 + (ap.y + dt * tt[c].y) * f1) * (T)0.25);
            }
        } else {
#pragma unroll
            for (int c = 0; c < 3; ++c) o[c] = zero_c<T>();
        }
    } else {
        const T third = (T)(1.0 / 3.0);  // the division by 3 as a product (within one rounding)
        if (inside) {
            const T f0 = fc.fxy0 * fac[nfac + nxv + N + l];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const cpx<T> a0 = v0[c], ap = vp[c];
                o[c] = mk<T>((a0.x * f0 + 2 * (ap.x + dt * tt[c].x)) * f0 * third,
                             (a0.y * f0 + 2 * (ap.y + dt * tt[c].y)) * f0 * third);
            }
        } else {
#pragma unroll
            for (int c = 0; c < 3; ++c) o[c] = v0[c];
        }
        // final force_divfree of the state (vorticity_equation.cpp:436)
        if (k2 > 0.0) divfree<T>(fc.kxT, fc.kyT, kzT, ik2, o);
        if (kzero) {
#pragma unroll
            for (int c = 0; c < 3; ++c) o[c] = zero_c<T>();
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) out0[pt * 3 + c] = o[c];
}

// An RK tile of the FZ pass (one ky, kx columns kx0..) whose every mode lies
// outside kM2 (kx0^2 + ky^2 > kM2): its epilogue writes zero (stages 1-2) or
// keeps v0 (stage 3) without reading the transformed product, so neither the
// product's load nor its transform is needed (about a fifth of the tiles
// with the smooth filter's kM = N/2 - 1).
template <int N, int MODE>
__device__ __forceinline__ bool fz_tile_outside(const KParams& kp, int a, int kx0) {
    if constexpr (MODE >= CM_FZ_RK1 && MODE <= CM_FZ_RK3) {
        const double ky = kwrap<N>(a, kp.dky), kx = (double)kx0 * kp.dkx;
        return kx * kx + ky * ky > kp.kM2;
    } else {
        return false;
    }
}

template <typename T, int N, int MODE, int S>
__device__ __forceinline__ void col_issue_load(cpx<T>* tile, const cpx<T>* in0,
                                               const cpx<T>* in1, int a, int kx0, int ncol,
                                               size_t nxp3, int tid) {
    constexpr int NB = col_nb(MODE);
    constexpr int NBIN = col_nbin(MODE);
    constexpr int TKX = col_tkx<T, N, MODE, S>();
    constexpr int W = 3 * TKX;
    constexpr int PR = col_pitch<T, N, MODE, S>();
    constexpr int VB = ((W * (int)sizeof(cpx<T>)) % 16 == 0) ? 16 : 8;
    constexpr int VPE = VB / (int)sizeof(cpx<T>) > 0 ? VB / (int)sizeof(cpx<T>) : 1;  // complex per copy
    constexpr int WV = W / VPE;
    const int nvalid = (3 * ncol + VPE - 1) / VPE;
    for (int e = tid; e < N * NBIN * WV; e += col_threads<T, N, MODE, S>()) {
        const int v = e % WV;
        const int r = e / WV;
        const int b = r % NBIN;
        const int l = r / NBIN;
        if (v >= nvalid) continue;
        const cpx<T>* src = ((b == 0) ? in0 : in1) + col_in_row<N, MODE>(a, l) * nxp3 +
                            (size_t)kx0 * 3 + v * VPE;
        const int bdst = (MODE == CM_IZ_VEL) ? 1 : b;  // w^ goes to slot 1
        cp_async<VB>(&tile[l * PR + bdst * W + v * VPE], src);
    }
}

// Dynamic tile scheduling: CTAs take tile numbers from a counter in global
// memory (tctr[0]), so an SM that runs slower takes fewer tiles instead of
// holding up the end of the pass.  Used for every launch with at least 8
// tiles per CTA (the exit protocol costs a few microseconds per CTA, so short
// launches keep the static order); measured at 512^3 FP32 against the static
// order: IY 1.59 -> 1.42, FY 0.754 -> 0.684, FZ 1.70 -> 1.56 ms (its tiles
// wholly outside kM cost a fraction of the others), IZ faster as well.  The
// last CTA to leave resets both words,
// so the next launch on the stream (or the next replay of a graph) starts
// from zero without a host-side reset.
// With no counter (tctr null) the k-th ticket of a CTA is the static
// blockIdx.x + k gridDim.x.
__device__ __forceinline__ int tile_ticket(int* tctr, int k) {
    return tctr ? atomicAdd(tctr, 1) : (int)blockIdx.x + k * (int)gridDim.x;
}
__device__ __forceinline__ void tile_tickets_done(int* tctr, int tid) {
    if (tctr && tid == 0) {
        __threadfence();
        if (atomicAdd(tctr + 1, 1) == (int)gridDim.x - 1) {
            tctr[0] = 0;
            tctr[1] = 0;
            __threadfence();
        }
    }
}

// Last FFT stage of a column pass fused with the store: block b of R
// positions holds frequencies f(b) + (N/R) q; lanes take consecutive pencils,
// i.e. consecutive complex numbers of one output row chunk.  NYQ: the tile
// holds the Nyquist column only and PP counts its pencils (3 per buffer).
template <typename T, int N, int MODE, int S, int PP, bool NYQ>
__device__ __forceinline__ void col_last_store(const cpx<T>* tile, int tid, const Member<T>& mb,
                                               const Roles& rl, int a, int kx0, int ncol) {
    constexpr int NT = col_threads<T, N, MODE, S>();
    constexpr int TKX = col_tkx<T, N, MODE, S>();
    constexpr int W = 3 * TKX;
    constexpr int PR = col_pitch<T, N, MODE, S>();
    constexpr bool INV = col_inverse(MODE);
    constexpr int MR = col_mr<T, MODE, S>();
    constexpr int NST = plan_nstages(N, MR);
    constexpr int R = plan_radix(N, NST - 1, MR);
    constexpr int NW = PP * (N / R);
    constexpr size_t nxp3 = (size_t)(N / 2 + 4) * 3;
    const int nval = 3 * ncol;
    for (int w = tid; w < NW; w += NT) {
        const int pn = w % PP;
        const int bb = w / PP;
        const int pp = NYQ ? (pn / 3) * W + pn % 3 : pn;
        cpx<T> v[R];
#pragma unroll
        for (int m = 0; m < R; ++m) v[m] = tile[pp + (bb * R + m) * PR];
        dft<T, INV, R>(v);
        const int bufi = pp / W, q = pp % W;
        if (q >= nval) continue;
        cpx<T>* dst = mbuf(mb, (bufi == 0) ? rl.out0 : rl.out1) + (size_t)kx0 * 3 + q;
        const int f0 = dif_frequency<N, MR>(bb * R);
#pragma unroll
        for (int m = 0; m < R; ++m) dst[col_out_row<N, MODE>(a, f0 + (N / R) * m) * nxp3] = v[m];
    }
}

template <typename T, int N, int MODE, int S>
__global__ void __launch_bounds__(col_threads<T, N, MODE, S>(), col_ctas<T, N, MODE, S>())
col_pass(const Member<T>* __restrict__ mem, const Roles rl, const cpx<T>* __restrict__ tw_g,
         int ntx, int tiles_per, int ntiles, int* __restrict__ tctr) {
    constexpr int NT = col_threads<T, N, MODE, S>();
    constexpr int NBUF = col_nbuf<T, N, MODE, S>();
    constexpr int NB = col_nb(MODE);
    constexpr int TKX = col_tkx<T, N, MODE, S>();
    constexpr int W = 3 * TKX;                     // complex per row per buffer
    constexpr int PR = col_pitch<T, N, MODE, S>();    // tile row pitch
    constexpr int TILE = N * PR;
    constexpr bool INV = col_inverse(MODE);
    constexpr int NRK = col_nrk(MODE);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* bufs = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* tw = bufs + NBUF * TILE;

    constexpr int NXV = N / 2 + 1;
    constexpr size_t nxp3 = (size_t)(N / 2 + 4) * 3;
    const int tid = threadIdx.x;
    for (int i = tid; i < N; i += NT) tw[i] = tw_g[i];

    // tile t: member t / tiles_per, then (a, kx-tile) with the kx-tile fastest
    // tiles: this one (t) and, with two buffers, the next one (tnext)
    __shared__ int s_tk[2];
    int nk = 0;  // tickets drawn (thread 0)
    if (tid == 0) {
        s_tk[0] = tile_ticket(tctr, nk++);
        s_tk[1] = NBUF == 2 ? tile_ticket(tctr, nk++) : 0;
    }
    __syncthreads();
    int t = s_tk[0];
    int tnext = s_tk[1];
    if (t < ntiles) {
        const int m = t / tiles_per, tl = t - m * tiles_per;
        const int kx0 = (tl % ntx) * TKX;
        if (!fz_tile_outside<N, MODE>(mem[m].kp, tl / ntx, kx0))
            col_issue_load<T, N, MODE, S>(bufs, mbuf(mem[m], rl.in0), mbuf(mem[m], rl.in1), tl / ntx,
                                          kx0, min(TKX, NXV - kx0), nxp3, tid);
    }
    cp_async_commit();
    __shared__ Member<T> mb;  // this tile's member, read once per tile
    for (int it = 0; t < ntiles; ++it) {
        cpx<T>* tile = bufs + (NBUF == 2 ? (it & 1) * TILE : 0);
        const int m = t / tiles_per, tl = t - m * tiles_per;
        {
            // the previous tile ended with a barrier: nobody reads mb now
            constexpr int NWORDS = (int)(sizeof(Member<T>) / sizeof(int));
            const int* src = reinterpret_cast<const int*>(&mem[m]);
            int* dst = reinterpret_cast<int*>(&mb);
            for (int i = tid; i < NWORDS; i += NT) dst[i] = src[i];
        }
        if constexpr (NRK > 0) {
            // RK operands of this tile, rows S[ky=a][kz=l][kx0..kx0+TKX): into
            // L2 while the tile is transformed, read by the epilogue; only
            // rows with a mode inside kM2, except v0 in stage 3, which the
            // epilogue also reads outside
            const int a = tl / ntx;
            const int kx0 = (tl % ntx) * TKX;
            const cpx<T>* rk_v0 = mbuf(mem[m], rl.v0);  // mb is not yet visible to all
            const cpx<T>* rk_vp = NRK > 1 ? mbuf(mem[m], rl.vp) : rk_v0;
            const KParams& gkp = mem[m].kp;
            const double kyv = kwrap<N>(a, gkp.dky), kxv = (double)kx0 * gkp.dkx;
            const double room = gkp.kM2 - (kxv * kxv + kyv * kyv);  // kz^2 left inside
            constexpr int LINES = (3 * TKX * (int)sizeof(cpx<T>) + 127) / 128 + 1;
            const int nbytes = 3 * min(TKX, NXV - kx0) * (int)sizeof(cpx<T>);
            for (int e = tid; e < N * NRK * LINES; e += NT) {
                const int q = e % LINES;
                const int r = e / LINES;
                const int arr = r % NRK;
                const int l = r / NRK;
                const double kz = kwrap<N>(l, gkp.dkz);
                const bool used = (MODE == CM_FZ_RK3 && arr == 0) || kz * kz <= room;
                if (!used) continue;
                const char* row = reinterpret_cast<const char*>(
                    ((arr == 0) ? rk_v0 : rk_vp) + ((size_t)a * N + l) * nxp3 + (size_t)kx0 * 3);
                if (128 * q < nbytes) prefetch_l2(row + 128 * q);
            }
        }
        if constexpr (NBUF == 2) {
            // the next tile streams into the other buffer while this one is transformed
            const int tn = tnext;
            if (tn < ntiles) {
                const int mn = tn / tiles_per, tln = tn - mn * tiles_per;
                const int kx0n = (tln % ntx) * TKX;
                if (!fz_tile_outside<N, MODE>(mem[mn].kp, tln / ntx, kx0n))
                    col_issue_load<T, N, MODE, S>(bufs + ((it + 1) & 1) * TILE, mbuf(mem[mn], rl.in0),
                                                  mbuf(mem[mn], rl.in1), tln / ntx, kx0n,
                                                  min(TKX, NXV - kx0n), nxp3, tid);
            }
            cp_async_commit();
        }
        if constexpr (NBUF == 2) cp_async_wait<1>();
        else cp_async_wait<0>();
        __syncthreads();
        // ticket for the tile after the prefetched one (two buffers) or for
        // the next one (one buffer); read after the barrier ending this tile
        if (tid == 0) s_tk[0] = tile_ticket(tctr, nk++);
        const int a = tl / ntx;
        const int kx0 = (tl % ntx) * TKX;
        const int ncol = min(TKX, NXV - kx0);
        const KParams& kp = mb.kp;

        // ---- prologue: u^ = i k x w^ / k^2 for 0 < k^2 <= kM^2 -----------
        if constexpr (MODE == CM_IZ_VEL || MODE == CM_IZ_U) {
            constexpr int WSRC = (MODE == CM_IZ_VEL) ? W : 0;  // slot holding w^
            const double ky = kwrap<N>(a, kp.dky);
            // one point: kx, kx^2 + ky^2 and the storage-precision kx, ky of its
            // column given
            // compute_velocity ends with field::symmetrize (field.cpp:903-978),
            // which on the kx = 0 plane replaces every row ky = N - yy
            // (0 < yy < N/2) by the conjugate of row yy, kz reversed.  The
            // modes computed here already agree with that except on the kz =
            // N/2 line, whose wavenumber +N/2 dkz does not change sign with
            // ky (it matters where that line lies inside kM, e.g. for dk
            // larger along y than along z): there u is taken from the mirror
            // mode (N - ky, N/2), read from the source field.
            const bool mirror_row = kx0 == 0 && a > N / 2;
            auto point = [&](int col, int l, double kxy2, T kxT, T kyT) {
                const double kz = kwrap<N>(l, kp.dkz);
                const double k2 = kxy2 + kz * kz;
                cpx<T>* w = &tile[l * PR + WSRC + col * 3];
                cpx<T> u[3];
                if (k2 <= kp.kM2 && k2 > 0.0) {
                    const T ik2 = inv_k2<T>(k2);
                    cpx<T> wv[3] = {w[0], w[1], w[2]};
                    const bool mirror = mirror_row && col == 0 && l == N / 2;
                    if (mirror) {
                        const cpx<T>* src = mbuf(mb, rl.in0) +
                                            ((size_t)(N - a) * N + N / 2) * (N / 2 + 4) * 3;
#pragma unroll
                        for (int c = 0; c < 3; ++c) wv[c] = src[c];
                    }
                    curl<T>(kxT, mirror ? (T)kwrap<N>(N - a, kp.dky) : kyT, (T)kz, wv, u);
#pragma unroll
                    for (int c = 0; c < 3; ++c) u[c] = scale(u[c], ik2);
                    if (mirror) {
#pragma unroll
                        for (int c = 0; c < 3; ++c) u[c] = conjg(u[c]);
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < 3; ++c) u[c] = zero_c<T>();
                }
#pragma unroll
                for (int c = 0; c < 3; ++c) tile[l * PR + col * 3 + c] = u[c];
            };
            if constexpr (NT % TKX == 0) {
                // a thread keeps one column.  In FP32, with a tile pitch of
                // 2 modulo 4, each half-warp takes eight consecutive rows of
                // two columns: the 8-byte accesses PR l + 3 col (+ c) then
                // fall on sixteen distinct banks (with the column fastest
                // they met two-way)
                constexpr bool ROWS8 = sizeof(T) == 4 && TKX >= 2 && PR % 4 == 2 && NT % (8 * TKX) == 0;
                const int col = ROWS8 ? (tid >> 3) % TKX : tid % TKX;
                const int l0 = ROWS8 ? (tid & 7) + 8 * (tid / (8 * TKX)) : tid / TKX;
                if (col < ncol) {
                    const double kx = (double)(kx0 + col) * kp.dkx;
                    const double kxy2 = kx * kx + ky * ky;
                    for (int l = l0; l < N; l += NT / TKX) point(col, l, kxy2, (T)kx, (T)ky);
                }
            } else {
                for (int e = tid; e < N * TKX; e += NT) {
                    const int col = e % TKX;
                    const int l = e / TKX;
                    if (col >= ncol) continue;
                    const double kx = (double)(kx0 + col) * kp.dkx;
                    point(col, l, kx * kx + ky * ky, (T)kx, (T)ky);
                }
            }
            __syncthreads();
        }

        // ---- FFT along l: NB*W pencils, pencil stride 1, element stride PR --
        using LY = Lay<1, 1, 0, PR>;
        constexpr int P = NB * W;
        // the tile holding only the Nyquist column transforms just its pencils
        using LYN = Lay<3, W, 1, PR>;
        constexpr int PN = NB * 3;
        constexpr int MR = col_mr<T, MODE, S>();
        constexpr int NST = plan_nstages(N, MR);
        if constexpr (MODE >= CM_FZ_RK1 && MODE <= CM_FZ_RK3) {
            // a tile wholly outside kM2 was not loaded: its epilogue reads
            // only the RK operands (fz_tile_outside)
            if (!fz_tile_outside<N, MODE>(kp, a, kx0)) {
                if (ncol == TKX) dif<T, N, INV, P, LY, 1, N, MR>(tile, tw, tid, NT);
                else dif<T, N, INV, PN, LYN, 1, N, MR>(tile, tw, tid, NT);
            }
            __syncthreads();
            // ---- epilogue: one thread per mode (kz = l, kx = kx0 + col)
            const double ky = kwrap<N>(a, kp.dky);
            auto mode = [&](int col, int l, const FzCol<T>& fc) {
                const size_t pt = ((size_t)a * N + l) * (N / 2 + 4) + kx0 + col;  // S[ky=a][kz=l][kx]
                const cpx<T>* v0 = mbuf(mb, rl.v0) + pt * 3;
                const cpx<T>* vp = NRK > 1 ? mbuf(mb, rl.vp) + pt * 3 : v0;
                fz_point<T, N, MODE, S>(kp, tile, PR, a, l, kx0 + col, col, fc, v0, vp, pt, mb.filt,
                                     mb.fac, mbuf(mb, rl.fsrc), mbuf(mb, rl.out0));
            };
            if constexpr (NT % TKX == 0) {
                // a thread keeps one column: its constants once per tile
                const int col = tid % TKX;
                if (col < ncol) {
                    const FzCol<T> fc = fz_col<T, N, MODE>(kp, mb.fac, a, kx0 + col, ky);
                    for (int l = tid / TKX; l < N; l += NT / TKX) mode(col, l, fc);
                }
            } else {
                for (int e = tid; e < N * TKX; e += NT) {
                    const int col = e % TKX;
                    const int l = e / TKX;
                    if (col >= ncol) continue;
                    mode(col, l, fz_col<T, N, MODE>(kp, mb.fac, a, kx0 + col, ky));
                }
            }
        } else {
            if (ncol == TKX) {
                dif_range<T, N, 0, NST - 1, INV, P, LY, 1, N, MR>(tile, tw, tid, NT);
                col_last_store<T, N, MODE, S, P, false>(tile, tid, mb, rl, a, kx0, ncol);
            } else {
                dif_range<T, N, 0, NST - 1, INV, PN, LYN, 1, N, MR>(tile, tw, tid, NT);
                col_last_store<T, N, MODE, S, PN, true>(tile, tid, mb, rl, a, kx0, ncol);
            }
        }
        __syncthreads();  // this buffer is refilled by the next load
        if constexpr (NBUF == 1) {
            const int tn = s_tk[0];
            if (tn < ntiles) {
                const int mn = tn / tiles_per, tln = tn - mn * tiles_per;
                const int kx0n = (tln % ntx) * TKX;
                if (!fz_tile_outside<N, MODE>(mem[mn].kp, tln / ntx, kx0n))
                    col_issue_load<T, N, MODE, S>(bufs, mbuf(mem[mn], rl.in0), mbuf(mem[mn], rl.in1),
                                                  tln / ntx, kx0n, min(TKX, NXV - kx0n), nxp3, tid);
            }
            cp_async_commit();
            t = tn;
        } else {
            const int t2 = s_tk[0];
            t = tnext;
            tnext = t2;
        }
    }
    cp_async_wait<0>();
    tile_tickets_done(tctr, tid);
}

// ---------------------------------------------------------------------------
enum RowMode {
    RM_NONLIN = 0,     // (u^, w^) rows -> R2C(u x w / N^3) into out, opt. real u
    RM_C2R = 1,        // complex rows -> real rows
    RM_R2C = 2,        // real rows -> complex rows
};
constexpr int ROW_THREADS = 512;
constexpr int ROW_CTAS = 1;  // resident CTAs per SM
constexpr int ROW_BUDGET = SMEM_BUDGET / ROW_CTAS - 2048;

template <int N>
__host__ __device__ constexpr int row_rl() { return (N / 2 + 4) * 3; }  // padded row, complex
template <int N>
__host__ __device__ constexpr int row_pl() { return N / 2 + 1; }  // odd pencil pitch
// radix cap of the x transforms (length M = N/2): 8 (a cap of 16, two
// stages at M = 256, left most threads of a tile idle in the mirror-paired
// and last-stage phases and measured 30 % slower at 512^3)
#ifndef BFG_ROW_MR_F32
#define BFG_ROW_MR_F32 8
#endif
template <typename T, int M>
__host__ __device__ constexpr int row_max_radix() {
    return (sizeof(T) == 4 && M >= 64) ? BFG_ROW_MR_F32 : 8;
}
// shared memory for R rows: staging (two alternating buffers of interleaved
// rows as they sit in HBM), pencils (one per component, odd pitch), output
// rows (R2C only), twiddles and the digit-reversal table
template <typename T, int N, int MODE>
__host__ __device__ constexpr size_t row_bytes_for(int R) {
    return (size_t)((MODE == RM_R2C) ? 2 * R * (N * 3 / 2) + R * row_rl<N>()
                                     : 2 * R * (MODE == RM_NONLIN ? 2 : 1) * row_rl<N>()) *
               sizeof(cpx<T>) +
           (size_t)((MODE == RM_NONLIN ? 6 : 3) * R * row_pl<N>() + N) * sizeof(cpx<T>) +
           (size_t)(N / 2) * 4;
}
template <typename T, int N, int MODE>
__host__ __device__ constexpr int row_rows_from(int R) {
    return (R <= 1 || (row_bytes_for<T, N, MODE>(R) <= (size_t)ROW_BUDGET && R <= (N * N) / 296))
               ? (R < 1 ? 1 : R)
               : row_rows_from<T, N, MODE>(R / 2);
}
template <typename T, int N, int MODE>
__host__ __device__ constexpr int row_rows() {
    return row_rows_from<T, N, MODE>(16);
}
template <typename T, int N, int MODE>
__host__ __device__ constexpr size_t row_smem_bytes() {
    return row_bytes_for<T, N, MODE>(row_rows<T, N, MODE>());
}

// C2R pre-processing (pairs k, M-k; X[0] and X[M] enter with their real
// parts only), reading X from an interleaved row (stride 3) and writing Z to
// a contiguous pencil.
template <typename T, int N>
__device__ __forceinline__ void c2r_pre(const cpx<T>* x, cpx<T>* z, const cpx<T>* tw, int k) {
    constexpr int M = N / 2;
    if (k == 0) {
        const T x0 = x[0].x, xm = x[3 * M].x;
        z[0] = mk<T>(x0 + xm, x0 - xm);
        return;
    }
    const cpx<T> a = x[3 * k], b = x[3 * (M - k)];
    const cpx<T> w = tw[k];  // exp(-2 pi i k / N)
    // Z[k] = (a + conj b) + i conj(w) (a - conj b)
    {
        const cpx<T> sp = a + conjg(b), dm = a - conjg(b);
        const cpx<T> e = cmulc(dm, w);  // dm * conj(w)
        z[k] = mk<T>(sp.x - e.y, sp.y + e.x);
    }
    if (k != M - k) {
        // Z[M-k] = (b + conj a) - i w (b - conj a)
        const cpx<T> sp = b + conjg(a), dm = b - conjg(a);
        const cpx<T> e = cmul(dm, w);
        z[M - k] = mk<T>(sp.x + e.y, sp.y - e.x);
    }
}

// R2C post-processing: natural-order Z from a contiguous pencil, X[0..M]
// written into an interleaved row (stride 3).
template <typename T, int N>
__device__ __forceinline__ void r2c_post(const cpx<T>* z, cpx<T>* x, const cpx<T>* tw, int k) {
    constexpr int M = N / 2;
    const T h = (T)0.5;
    if (k == 0) {
        const cpx<T> z0 = z[0];
        x[0] = mk<T>(z0.x + z0.y, (T)0);
        x[3 * M] = mk<T>(z0.x - z0.y, (T)0);
        return;
    }
    const cpx<T> zk = z[k], zm = z[M - k];
    const cpx<T> w = tw[k];
    {
        const cpx<T> e = scale(zk + conjg(zm), h);
        const cpx<T> d = zk - conjg(zm);
        const cpx<T> o = mk<T>(d.y * h, -d.x * h);  // d / (2i)
        x[3 * k] = e + cmul(w, o);
    }
    if (k != M - k) {
        // exp(-2 pi i (M-k)/N) = -conj(w)
        const cpx<T> e = scale(zm + conjg(zk), h);
        const cpx<T> d = zm - conjg(zk);
        const cpx<T> o = mk<T>(d.y * h, -d.x * h);
        x[3 * (M - k)] = e - cmul(conjg(w), o);
    }
}

// Row pass over (z, y) rows of W.  Persistent CTAs walk tiles of ROWS
// consecutive rows; a tile's rows are contiguous in HBM and are streamed
// with cp.async into one of two staging buffers while the previous tile is
// transformed.  The C2R pre-processing moves each component of each row into
// its own pencil (odd pitch PL, so that lanes on consecutive pencils or
// consecutive elements hit distinct banks); the R2C post-processing moves the
// result back into the interleaved staging rows, which are stored with
// 16-byte vectors.
template <typename T, int N, int MODE>
__device__ __forceinline__ void row_issue_load(cpx<T>* stage, const cpx<T>* wu, const cpx<T>* ww,
                                               const T* rin, size_t row0, int tid) {
    constexpr int ROWS = row_rows<T, N, MODE>();
    constexpr int VPE = 16 / (int)sizeof(cpx<T>);
    if constexpr (MODE == RM_R2C) {
        constexpr int NV = ROWS * N * 3 / 2 / VPE;  // 16-byte vectors of the real rows
        const cpx<T>* src = reinterpret_cast<const cpx<T>*>(rin + row0 * N * 3);
        for (int v = tid; v < NV; v += ROW_THREADS) cp_async16(&stage[v * VPE], &src[v * VPE]);
    } else {
        constexpr int NBIN = (MODE == RM_NONLIN) ? 2 : 1;
        constexpr int RL = row_rl<N>();
        constexpr int NV = ROWS * RL / VPE;  // per buffer
        for (int e = tid; e < NBIN * NV; e += ROW_THREADS) {
            const int v = e % NV;
            const int b = e / NV;
            const cpx<T>* src = ((b == 0) ? wu : ww) + row0 * RL;
            cp_async16(&stage[b * ROWS * RL + v * VPE], &src[v * VPE]);
        }
    }
}

template <typename T, int N, int MODE, bool WRITE_RU>
__global__ void __launch_bounds__(ROW_THREADS, ROW_CTAS)
row_pass(const Member<T>* __restrict__ mem, const Roles rl, const cpx<T>* __restrict__ tw_g,
         int tiles_per, int ntiles) {
    constexpr int M = N / 2;
    constexpr int ROWS = row_rows<T, N, MODE>();
    constexpr int RL = row_rl<N>();
    constexpr int PL = row_pl<N>();
    constexpr int NBIN = (MODE == RM_NONLIN) ? 2 : 1;
    constexpr int VPE = 16 / (int)sizeof(cpx<T>);
    constexpr int STAGE = (MODE == RM_R2C) ? ROWS * N * 3 / 2 : ROWS * NBIN * RL;
    constexpr int NP = NBIN * 3 * ROWS;  // pencils of the inverse transform
    using LP = Lay<1, PL, 0, 1>;          // contiguous pencils, odd pitch
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* stage0 = reinterpret_cast<cpx<T>*>(smem_raw);
    cpx<T>* outr = stage0 + 2 * STAGE;                               // R2C output rows
    cpx<T>* S = outr + ((MODE == RM_R2C) ? ROWS * RL : 0);           // pencils
    cpx<T>* tw = S + ((MODE == RM_NONLIN) ? 6 : 3) * ROWS * PL;
    int* posn = reinterpret_cast<int*>(tw + N);                      // DIF position of n
    const int tid = threadIdx.x;

    for (int i = tid; i < N; i += ROW_THREADS) tw[i] = tw_g[i];
    constexpr int MRR = row_max_radix<T, M>();
    for (int i = tid; i < M; i += ROW_THREADS) posn[i] = dif_position<M, MRR>(i);
    if constexpr (MODE == RM_R2C) {
        // padding columns of the output rows are written out: start them at 0
        for (int i = tid; i < ROWS * RL; i += ROW_THREADS) outr[i] = zero_c<T>();
    }

    // tile t: member t / tiles_per, then ROWS consecutive rows
    int t = blockIdx.x;
    if (t < ntiles) {
        const int m = t / tiles_per, tl = t - m * tiles_per;
        row_issue_load<T, N, MODE>(stage0, mbuf(mem[m], rl.in0), mbuf(mem[m], rl.in1),
                                   mreal(mem[m], rl.rin), (size_t)tl * ROWS, tid);
    }
    cp_async_commit();
    for (int it = 0; t < ntiles; ++it, t += gridDim.x) {
        cpx<T>* st = stage0 + (it & 1) * STAGE;
        {
            const int tn = t + gridDim.x;
            if (tn < ntiles) {
                const int mn = tn / tiles_per, tln = tn - mn * tiles_per;
                row_issue_load<T, N, MODE>(stage0 + ((it + 1) & 1) * STAGE, mbuf(mem[mn], rl.in0),
                                           mbuf(mem[mn], rl.in1), mreal(mem[mn], rl.rin),
                                           (size_t)tln * ROWS, tid);
            }
            cp_async_commit();
        }
        cp_async_wait<1>();
        __syncthreads();
        const int m = t / tiles_per, tl = t - m * tiles_per;
        const size_t row0 = (size_t)tl * ROWS;
        T* rout = mreal(mem[m], rl.rout);
        cpx<T>* wout = mbuf(mem[m], rl.out0);

        if constexpr (MODE == RM_R2C) {
            // real rows -> digit-reversed complex pencils z_c[n] = (x[2n][c], x[2n+1][c])
            const T* rs = reinterpret_cast<const T*>(st);
            for (int e = tid; e < ROWS * 3 * M; e += ROW_THREADS) {
                const int n = e % M;
                const int p = e / M;  // = r*3 + c
                const int c = p % 3, r = p / 3;
                const T* src = rs + (r * N + 2 * n) * 3 + c;
                S[p * PL + posn[n]] = mk<T>(src[0], src[3]);
            }
            __syncthreads();
        } else {
            // C2R pre-processing, interleaved rows -> pencils
            for (int e = tid; e < NP * (M / 2 + 1); e += ROW_THREADS) {
                const int k = e % (M / 2 + 1);
                const int p = e / (M / 2 + 1);  // = (b*ROWS + r)*3 + c
                c2r_pre<T, N>(st + (p / 3) * RL + (p % 3), S + p * PL, tw, k);
            }
            __syncthreads();
            dif<T, M, true, NP, LP, 2, N, MRR>(S, tw, tid, ROW_THREADS);

            if constexpr (MODE == RM_C2R || WRITE_RU) {
                // real u (pencils of buffer 0) to rout in natural x order
                for (int e = tid; e < ROWS * N * 3; e += ROW_THREADS) {
                    const int c = e % 3;
                    const int r2 = e / 3;
                    const int x = r2 % N;
                    const int r = r2 / N;
                    const cpx<T> z = S[(r * 3 + c) * PL + posn[x >> 1]];
                    rout[(row0 + r) * (N * 3) + x * 3 + c] = (x & 1) ? z.y : z.x;
                }
            }
            if constexpr (MODE == RM_C2R) {
                __syncthreads();
                continue;
            }
            if constexpr (WRITE_RU) __syncthreads();
            if constexpr (MODE == RM_NONLIN) {
                // u x w / npoints at each position (two grid points per position)
                const T inv_np = (T)1 / ((T)N * (T)N * (T)N);
                for (int e = tid; e < ROWS * M; e += ROW_THREADS) {
                    const int p = e % M;
                    const int r = e / M;
                    cpx<T> u[3], w[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        u[c] = S[(r * 3 + c) * PL + p];
                        w[c] = S[(3 * ROWS + r * 3 + c) * PL + p];
                    }
#pragma unroll
                    for (int cc = 0; cc < 3; ++cc) {
                        const int c1 = (cc + 1) % 3, c2 = (cc + 2) % 3;
                        const T tx = u[c1].x * w[c2].x - u[c2].x * w[c1].x;
                        const T ty = u[c1].y * w[c2].y - u[c2].y * w[c1].y;
                        S[(r * 3 + cc) * PL + p] = mk<T>(tx * inv_np, ty * inv_np);
                    }
                }
                __syncthreads();
            }
        }
        // forward: digit-reversed -> natural, then R2C post-processing into
        // interleaved rows (the staging rows of u, or the R2C output rows)
        dit<T, M, false, 3 * ROWS, LP, 2, N, MRR>(S, tw, tid, ROW_THREADS);
        cpx<T>* orow = (MODE == RM_R2C) ? outr : st;
        for (int e = tid; e < 3 * ROWS * (M / 2 + 1); e += ROW_THREADS) {
            const int k = e % (M / 2 + 1);
            const int p = e / (M / 2 + 1);  // = r*3 + c
            r2c_post<T, N>(S + p * PL, orow + (p / 3) * RL + (p % 3), tw, k);
        }
        __syncthreads();
        // padded rows out (padding columns carry zeros), 16-byte vectors
        {
            const float4* src = reinterpret_cast<const float4*>(orow);
            float4* dst = reinterpret_cast<float4*>(wout + row0 * RL);
            for (int v = tid; v < ROWS * RL / VPE; v += ROW_THREADS) dst[v] = src[v];
        }
        __syncthreads();
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// Fused nonlinear row pass (the X pass of every RK stage, N >= 32).
//
// Same result as row_pass<RM_NONLIN> with fewer shared-memory round trips:
//   A  C2R pre-processing fused with DIF stage 0: a work unit takes the
//      butterflies j and S0 - j of stage 0 (span S0), whose inputs are each
//      other's mirror partners k, M - k, straight from the staging rows;
//   B  the middle DIF stages;
//   C  the last DIF stage (span 1) of the six pencils of a row, u x w / N^3
//      and the first DIT stage, in registers, per block of the last radix;
//   D  the middle DIT stages;
//   E  DIT stage 0 fused with the R2C post-processing, again on mirror
//      pairs, writing interleaved output rows.
// One staging buffer: the rows of the next tile stream in (cp.async) from
// the end of phase A, while B..E and the store of this tile run.  Per row
// the pencil region holds the u pencils (overwritten by the output row in
// phase E) and the w pencils (which receive the product).  Pitches: the
// region length RG is odd (-1 modulo the banks a wavefront spans), the
// pencil pitch PL and the w offset W are multiples of the rows per tile
// modulo that count, so that lanes on (pencil, row) or (block, row) pairs
// hit distinct banks.
template <typename T>
__host__ __device__ constexpr int nslot() { return 128 / (int)sizeof(cpx<T>); }
// smallest x >= v with x = res (mod md)
__host__ __device__ constexpr int at_least_mod(int v, int md, int res) {
    return v + (((res - v) % md) + md) % md;
}
template <typename T, int N>
__host__ __device__ constexpr int rnl_pl(int R) {
    return at_least_mod(N / 2 + 1, nslot<T>(), R % nslot<T>());
}
template <typename T, int N>
__host__ __device__ constexpr int rnl_w(int R) {
    return at_least_mod(row_rl<N>() > 2 * rnl_pl<T, N>(R) + N / 2 ? row_rl<N>()
                                                                  : 2 * rnl_pl<T, N>(R) + N / 2,
                        nslot<T>(), (3 * R) % nslot<T>());
}
template <typename T, int N>
__host__ __device__ constexpr int rnl_rg(int R) {
    return at_least_mod(rnl_w<T, N>(R) + 3 * rnl_pl<T, N>(R), nslot<T>(), nslot<T>() - 1);
}
template <typename T, int N>
__host__ __device__ constexpr int rnl_tw0() {
    return (N / 2) / plan_radix(N / 2, 0, row_max_radix<T, N / 2>()) *
           (plan_radix(N / 2, 0, row_max_radix<T, N / 2>()) - 1);
}
template <typename T, int N>
__host__ __device__ constexpr size_t rnl_bytes_for(int R) {
    return (size_t)(2 * R * row_rl<N>() + R * rnl_rg<T, N>(R) + N + rnl_tw0<T, N>()) *
               sizeof(cpx<T>) +
           (size_t)(N / 2) * 4;
}
// at most N^2/296 rows per tile (a single instance then still has a tile for
// each of two CTAs on every SM), but up to 16 on small grids, whose passes
// are launched over many instances at once and pay per-tile overheads
template <int N>
__host__ __device__ constexpr int rnl_row_cap() { return (N * N) / 296 > 16 ? (N * N) / 296 : 16; }
// rows per tile within a shared-memory budget
template <typename T, int N>
__host__ __device__ constexpr int rnl_rows_fit(int R, size_t budget) {
    return (R <= 1 || (rnl_bytes_for<T, N>(R) <= budget && R <= rnl_row_cap<N>()))
               ? (R < 1 ? 1 : R)
               : rnl_rows_fit<T, N>(R / 2, budget);
}
// CTAs per SM of the fused row pass: two 256-thread CTAs where each still
// holds at least 4 rows (slightly faster: one CTA's barriers are covered by
// the other), else one 512-thread CTA
template <typename T, int N>
__host__ __device__ constexpr int rnl_ctas() {
    return rnl_rows_fit<T, N>(16, SMEM_BUDGET / 2 - 2048) >= 4 ? 2 : 1;
}
template <typename T, int N>
__host__ __device__ constexpr int rnl_threads() { return 512 / rnl_ctas<T, N>(); }
template <typename T, int N>
__host__ __device__ constexpr int rnl_rows_from(int R) {
    return rnl_rows_fit<T, N>(R, SMEM_BUDGET / rnl_ctas<T, N>() - 2048);
}
template <typename T, int N>
__host__ __device__ constexpr int rnl_rows() { return rnl_rows_from<T, N>(16); }
template <typename T, int N>
__host__ __device__ constexpr size_t rnl_smem_bytes() {
    return rnl_bytes_for<T, N>(rnl_rows<T, N>());
}
template <typename T, int N>
__host__ __device__ constexpr bool rnl_fused() {
    return plan_nstages(N / 2, row_max_radix<T, N / 2>()) >= 2;
}

// pencil p = c6 * ROWS + r: c6 < 3 the u pencils, c6 >= 3 the w pencils
template <int ROWS, int RG, int PL, int W>
struct LayNL6 {
    static constexpr int ES = 1;
    __device__ __forceinline__ static int base(int p) {
        const int c6 = p / ROWS, r = p - c6 * ROWS;
        return r * RG + (c6 < 3 ? c6 * PL : W + (c6 - 3) * PL);
    }
};
// the w pencils only: p = c * ROWS + r
template <int ROWS, int RG, int PL, int W>
struct LayNLW {
    static constexpr int ES = 1;
    __device__ __forceinline__ static int base(int p) {
        const int c = p / ROWS, r = p - c * ROWS;
        return r * RG + W + c * PL;
    }
};

// C2R pre-processing of one mirror pair held in registers: a = X[k],
// b = X[M-k] become Z[k], Z[M-k] (w = exp(-2 pi i k / N)); the formulas of
// c2r_pre.
template <typename T>
__device__ __forceinline__ cpx<T> c2r_lo(cpx<T> a, cpx<T> b, cpx<T> w) {
    const cpx<T> sp = a + conjg(b), dm = a - conjg(b);
    const cpx<T> e = cmulc(dm, w);
    return mk<T>(sp.x - e.y, sp.y + e.x);
}
template <typename T>
__device__ __forceinline__ cpx<T> c2r_hi(cpx<T> a, cpx<T> b, cpx<T> w) {
    const cpx<T> sp = b + conjg(a), dm = b - conjg(a);
    const cpx<T> e = cmul(dm, w);
    return mk<T>(sp.x + e.y, sp.y - e.x);
}
// R2C post-processing of one mirror pair: zk = Z[k], zm = Z[M-k] give X[k]
// and X[M-k]; the formulas of r2c_post.
template <typename T>
__device__ __forceinline__ cpx<T> r2c_lo(cpx<T> zk, cpx<T> zm, cpx<T> w) {
    const T h = (T)0.5;
    const cpx<T> e = scale(zk + conjg(zm), h);
    const cpx<T> d = zk - conjg(zm);
    const cpx<T> o = mk<T>(d.y * h, -d.x * h);
    return e + cmul(w, o);
}
template <typename T>
__device__ __forceinline__ cpx<T> r2c_hi(cpx<T> zk, cpx<T> zm, cpx<T> w) {
    const T h = (T)0.5;
    const cpx<T> e = scale(zm + conjg(zk), h);
    const cpx<T> d = zm - conjg(zk);
    const cpx<T> o = mk<T>(d.y * h, -d.x * h);
    return e - cmul(conjg(w), o);
}

template <typename T, int N, bool WRITE_RU>
__global__ void __launch_bounds__(rnl_threads<T, N>(), rnl_ctas<T, N>())
row_nonlin(const Member<T>* __restrict__ mem, const Roles rl, const cpx<T>* __restrict__ tw_g,
           int tiles_per, int ntiles) {
    constexpr int RNL_THREADS = rnl_threads<T, N>();
    constexpr int M = N / 2;
    constexpr int MRR = row_max_radix<T, M>();
    constexpr int NS = plan_nstages(M, MRR);
    constexpr int R0 = plan_radix(M, 0, MRR);
    constexpr int S0 = M / R0;                      // span of stage 0
    constexpr int H0 = S0 / 2;                      // mirror-paired units per pencil
    constexpr int RZ = plan_radix(M, NS - 1, MRR);  // radix of the last stage (span 1)
    constexpr int NBZ = M / RZ;
    constexpr int ROWS = rnl_rows<T, N>();
    constexpr int RL = row_rl<N>();
    constexpr int PL = rnl_pl<T, N>(ROWS);
    constexpr int W = rnl_w<T, N>(ROWS);
    constexpr int RG = rnl_rg<T, N>(ROWS);
    constexpr int VPE = 16 / (int)sizeof(cpx<T>);
    constexpr int NV = ROWS * RL / VPE;        // 16-byte vectors per input buffer
    constexpr int G = (ROWS % RZ == 0) ? RZ : ROWS;  // rows across lanes in phase C
    constexpr bool SPLIT = RZ * 6 * (int)sizeof(cpx<T>) > 192;  // w's last stage apart
    using L6 = LayNL6<ROWS, RG, PL, W>;
    using LW = LayNLW<ROWS, RG, PL, W>;
    static_assert(NS >= 2 && H0 >= 2, "fused row pass needs two stages");
    static_assert(W >= RL && W >= 2 * PL + M && (RG & 1), "region layout");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T>* st = reinterpret_cast<cpx<T>*>(smem_raw);  // u rows, then w rows
    cpx<T>* P = st + 2 * ROWS * RL;                     // ROWS regions of RG
    cpx<T>* tw = P + ROWS * RG;
    cpx<T>* tw0 = tw + N;  // stage-0 twiddles [j][q-1] = tw[2 j q]
    int* posn = reinterpret_cast<int*>(tw0 + rnl_tw0<T, N>());
    const int tid = threadIdx.x;

    for (int i = tid; i < N; i += RNL_THREADS) tw[i] = tw_g[i];
    for (int i = tid; i < rnl_tw0<T, N>(); i += RNL_THREADS) {
        const int j = i / (R0 - 1), q = i - j * (R0 - 1) + 1;
        tw0[i] = tw_g[2 * j * q];
    }
    if constexpr (WRITE_RU)
        for (int i = tid; i < M; i += RNL_THREADS) posn[i] = dif_position<M, MRR>(i);

    auto issue = [&](int tt) {
        const int mm = tt / tiles_per, tl = tt - mm * tiles_per;
        const cpx<T>* su = mbuf(mem[mm], rl.in0) + (size_t)tl * ROWS * RL;
        const cpx<T>* sw = mbuf(mem[mm], rl.in1) + (size_t)tl * ROWS * RL;
        for (int e = tid; e < 2 * NV; e += RNL_THREADS) {
            const int b = e >= NV ? 1 : 0;
            const int v = e - b * NV;
            cp_async16(&st[b * ROWS * RL + v * VPE], &(b ? sw : su)[v * VPE]);
        }
    };
    int t = blockIdx.x;
    if (t < ntiles) issue(t);
    cp_async_commit();
    for (; t < ntiles; t += gridDim.x) {
        cp_async_wait<0>();
        __syncthreads();
        const int m = t / tiles_per, tl = t - m * tiles_per;
        const size_t row0 = (size_t)tl * ROWS;

        // A: C2R pre-processing + DIF stage 0, staging rows -> pencils
        for (int e = tid; e < 6 * ROWS * H0; e += RNL_THREADS) {
            const int u = e % H0;
            const int p = e / H0;  // = r * 6 + c6
            const int r = p / 6, c6 = p - 6 * r;
            const int b = c6 >= 3 ? 1 : 0, c = c6 - 3 * b;
            const cpx<T>* x = st + (b * ROWS + r) * RL + c;
            cpx<T>* z = P + r * RG + (b ? W : 0) + c * PL;
            const int ja = u, jb = u == 0 ? H0 : S0 - u;
            cpx<T> va[R0], vb[R0];
#pragma unroll
            for (int q = 0; q < R0; ++q) {
                va[q] = x[3 * (ja + S0 * q)];
                vb[q] = x[3 * (jb + S0 * q)];
            }
            if (u != 0) {
                // k = u + S0 q pairs with M - k = jb + S0 (R0 - 1 - q)
#pragma unroll
                for (int q = 0; q < R0 / 2; ++q) {
                    const cpx<T> a0 = va[q], b0 = vb[R0 - 1 - q];
                    const cpx<T> a1 = va[R0 - 1 - q], b1 = vb[q];
                    const cpx<T> w0 = tw[ja + S0 * q], w1 = tw[ja + S0 * (R0 - 1 - q)];
                    va[q] = c2r_lo(a0, b0, w0);
                    vb[R0 - 1 - q] = c2r_hi(a0, b0, w0);
                    va[R0 - 1 - q] = c2r_lo(a1, b1, w1);
                    vb[q] = c2r_hi(a1, b1, w1);
                }
            } else {
                // item 0: k = S0 q pairs with S0 (R0 - q); X[0] with X[M]
                const T x0 = va[0].x, xm = x[3 * M].x;
                va[0] = mk<T>(x0 + xm, x0 - xm);
#pragma unroll
                for (int q = 1; q < R0 / 2; ++q) {
                    const cpx<T> a0 = va[q], b0 = va[R0 - q];
                    const cpx<T> w0 = tw[S0 * q];
                    va[q] = c2r_lo(a0, b0, w0);
                    va[R0 - q] = c2r_hi(a0, b0, w0);
                }
                va[R0 / 2] = c2r_lo(va[R0 / 2], va[R0 / 2], tw[S0 * (R0 / 2)]);
                // item S0/2: k = H0 + S0 q pairs with H0 + S0 (R0 - 1 - q)
#pragma unroll
                for (int q = 0; q < R0 / 2; ++q) {
                    const cpx<T> a0 = vb[q], b0 = vb[R0 - 1 - q];
                    const cpx<T> w0 = tw[H0 + S0 * q];
                    vb[q] = c2r_lo(a0, b0, w0);
                    vb[R0 - 1 - q] = c2r_hi(a0, b0, w0);
                }
            }
            dft<T, true, R0>(va);
            dft<T, true, R0>(vb);
#pragma unroll
            for (int q = 1; q < R0; ++q) {
                va[q] = cmulc(va[q], tw0[ja * (R0 - 1) + q - 1]);
                vb[q] = cmulc(vb[q], tw0[jb * (R0 - 1) + q - 1]);
            }
#pragma unroll
            for (int q = 0; q < R0; ++q) {
                z[ja + S0 * q] = va[q];
                z[jb + S0 * q] = vb[q];
            }
        }
        __syncthreads();
        // the staging rows are free: stream in the next tile
        if (t + (int)gridDim.x < ntiles) issue(t + gridDim.x);
        cp_async_commit();

        // B: middle DIF stages over the six pencils of each row
        dif_range<T, M, 1, NS - 1, true, 6 * ROWS, L6, 2, N, MRR>(P, tw, tid, RNL_THREADS);
        if constexpr (SPLIT) {
            dif_stage<T, M, NS - 1, true, 3 * ROWS, LW, 2, N, MRR>(P, tw, tid, RNL_THREADS);
            __syncthreads();
        }

        // C: last DIF stage, u x w / N^3, first DIT stage (product -> w pencils)
        {
            const T inv_np = (T)1 / ((T)N * (T)N * (T)N);
            for (int e = tid; e < ROWS * NBZ; e += RNL_THREADS) {
                const int rlo = e % G;
                const int t2 = e / G;
                const int bb = t2 % NBZ;
                const int r = (t2 / NBZ) * G + rlo;
                cpx<T>* reg = P + r * RG + bb * RZ;
                cpx<T> uu[3][RZ];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
#pragma unroll
                    for (int q = 0; q < RZ; ++q) uu[c][q] = reg[c * PL + q];
                    dft<T, true, RZ>(uu[c]);
                }
                if constexpr (WRITE_RU) {
#pragma unroll
                    for (int c = 0; c < 3; ++c)
#pragma unroll
                        for (int q = 0; q < RZ; ++q) reg[c * PL + q] = uu[c][q];
                }
                if constexpr (SPLIT) {
#pragma unroll
                    for (int q = 0; q < RZ; ++q) {
                        cpx<T> w3[3];
#pragma unroll
                        for (int c = 0; c < 3; ++c) w3[c] = reg[W + c * PL + q];
                        cpx<T> pr[3];
#pragma unroll
                        for (int cc = 0; cc < 3; ++cc) {
                            const int c1 = (cc + 1) % 3, c2 = (cc + 2) % 3;
                            const T tx = uu[c1][q].x * w3[c2].x - uu[c2][q].x * w3[c1].x;
                            const T ty = uu[c1][q].y * w3[c2].y - uu[c2][q].y * w3[c1].y;
                            pr[cc] = mk<T>(tx * inv_np, ty * inv_np);
                        }
#pragma unroll
                        for (int c = 0; c < 3; ++c) uu[c][q] = pr[c];
                    }
                } else {
                    cpx<T> ww[3][RZ];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
#pragma unroll
                        for (int q = 0; q < RZ; ++q) ww[c][q] = reg[W + c * PL + q];
                        dft<T, true, RZ>(ww[c]);
                    }
#pragma unroll
                    for (int q = 0; q < RZ; ++q) {
                        cpx<T> pr[3];
#pragma unroll
                        for (int cc = 0; cc < 3; ++cc) {
                            const int c1 = (cc + 1) % 3, c2 = (cc + 2) % 3;
                            const T tx = uu[c1][q].x * ww[c2][q].x - uu[c2][q].x * ww[c1][q].x;
                            const T ty = uu[c1][q].y * ww[c2][q].y - uu[c2][q].y * ww[c1][q].y;
                            pr[cc] = mk<T>(tx * inv_np, ty * inv_np);
                        }
#pragma unroll
                        for (int c = 0; c < 3; ++c) uu[c][q] = pr[c];
                    }
                }
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    dft<T, false, RZ>(uu[c]);
#pragma unroll
                    for (int q = 0; q < RZ; ++q) reg[W + c * PL + q] = uu[c][q];
                }
            }
        }
        __syncthreads();
        if constexpr (WRITE_RU) {
            // real u (u pencils after the inverse transform) in natural x
            // order: complex word posn[j] of component c's pencil holds
            // u(2j, c) and u(2j+1, c), so a thread takes four x (two words
            // per component) and writes their 12 values [x][c] as 16-byte
            // vectors of the (contiguous) output row
            T* rout = mreal(mem[m], rl.rout) + row0 * (N * 3);
            constexpr int QR = N / 4;  // four-x groups per row
            for (int v = tid; v < ROWS * QR; v += RNL_THREADS) {
                const int r = v / QR;
                const int k = v - r * QR;
                const int p0 = posn[2 * k], p1 = posn[2 * k + 1];
                T val[12];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const cpx<T> lo = P[r * RG + c * PL + p0];
                    const cpx<T> hi = P[r * RG + c * PL + p1];
                    val[c] = lo.x;
                    val[3 + c] = lo.y;
                    val[6 + c] = hi.x;
                    val[9 + c] = hi.y;
                }
                T* dst = rout + (size_t)r * (N * 3) + (size_t)k * 12;
                if constexpr (sizeof(T) == 4) {
#pragma unroll
                    for (int q = 0; q < 3; ++q)
                        reinterpret_cast<float4*>(dst)[q] =
                            make_float4(val[4 * q], val[4 * q + 1], val[4 * q + 2], val[4 * q + 3]);
                } else {
#pragma unroll
                    for (int q = 0; q < 6; ++q)
                        reinterpret_cast<double2*>(dst)[q] = make_double2(val[2 * q], val[2 * q + 1]);
                }
            }
            if constexpr (NS == 2) __syncthreads();  // phase E overwrites the u pencils
        }

        // D: middle DIT stages over the w pencils
        dit_range<T, M, NS - 2, 1, false, 3 * ROWS, LW, 2, N, MRR>(P, tw, tid, RNL_THREADS);

        // E: DIT stage 0 + R2C post-processing, w pencils -> output rows
        for (int e = tid; e < 3 * ROWS * H0; e += RNL_THREADS) {
            const int u = e % H0;
            const int p = e / H0;  // = r * 3 + c
            const int r = p / 3, c = p - 3 * r;
            const cpx<T>* z = P + r * RG + W + c * PL;
            cpx<T>* x = P + r * RG + c;
            const int ja = u, jb = u == 0 ? H0 : S0 - u;
            cpx<T> va[R0], vb[R0];
#pragma unroll
            for (int q = 0; q < R0; ++q) {
                va[q] = z[ja + S0 * q];
                vb[q] = z[jb + S0 * q];
            }
#pragma unroll
            for (int q = 1; q < R0; ++q) {
                va[q] = cmul(va[q], tw0[ja * (R0 - 1) + q - 1]);
                vb[q] = cmul(vb[q], tw0[jb * (R0 - 1) + q - 1]);
            }
            dft<T, false, R0>(va);
            dft<T, false, R0>(vb);
            if (u != 0) {
#pragma unroll
                for (int q = 0; q < R0; ++q) {
                    const int k = ja + S0 * q;
                    const cpx<T> w0 = tw[k];
                    x[3 * k] = r2c_lo(va[q], vb[R0 - 1 - q], w0);
                    x[3 * (M - k)] = r2c_hi(va[q], vb[R0 - 1 - q], w0);
                }
            } else {
                const cpx<T> z0 = va[0];
                x[0] = mk<T>(z0.x + z0.y, (T)0);
                x[3 * M] = mk<T>(z0.x - z0.y, (T)0);
#pragma unroll
                for (int q = 1; q < R0 / 2; ++q) {
                    const int k = S0 * q;
                    const cpx<T> w0 = tw[k];
                    x[3 * k] = r2c_lo(va[q], va[R0 - q], w0);
                    x[3 * (M - k)] = r2c_hi(va[q], va[R0 - q], w0);
                }
                x[3 * (M / 2)] = r2c_lo(va[R0 / 2], va[R0 / 2], tw[M / 2]);
#pragma unroll
                for (int q = 0; q < R0 / 2; ++q) {
                    const int k = H0 + S0 * q;
                    const cpx<T> w0 = tw[k];
                    x[3 * k] = r2c_lo(vb[q], vb[R0 - 1 - q], w0);
                    x[3 * (M - k)] = r2c_hi(vb[q], vb[R0 - 1 - q], w0);
                }
            }
        }
        // padding points of the output rows carry zeros
        for (int i = tid; i < ROWS * (RL - 3 * (M + 1)); i += RNL_THREADS) {
            const int r = i / (RL - 3 * (M + 1));
            P[r * RG + 3 * (M + 1) + (i - r * (RL - 3 * (M + 1)))] = zero_c<T>();
        }
        __syncthreads();
        // output rows out with 16-byte vectors
        {
            cpx<T>* wout = mbuf(mem[m], rl.out0) + row0 * RL;
            float4* dst = reinterpret_cast<float4*>(wout);
            for (int v = tid; v < NV; v += RNL_THREADS) {
                const int r = v / (RL / VPE);
                const cpx<T>* s = P + r * RG + (v - r * (RL / VPE)) * VPE;
                float4 val;
                if constexpr (VPE == 2) {
                    const cpx<T> a = s[0], b = s[1];
                    val = make_float4(a.x, a.y, b.x, b.y);
                } else {
                    val = *reinterpret_cast<const float4*>(s);
                }
                dst[v] = val;
            }
        }
        __syncthreads();
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// field::symmetrize on the kx = 0 plane of a state-layout buffer
// (field.cpp:903-978).  One thread per (ky, kz) of the plane.
template <typename T, int N>
__global__ void symmetrize_kernel(const Member<T>* __restrict__ mem, int bufi) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= N * N) return;
    cpx<T>* s = mem[blockIdx.y].buf[bufi];
    const int nxp = N / 2 + 4;
    const int ky = e / N, kz = e % N;
    const size_t P = (size_t)nxp;
    auto at = [&](int y, int z) -> cpx<T>* { return s + ((size_t)y * N + z) * P * 3; };
    if (ky == 0) {
        if (kz == 0) {
            cpx<T>* d = at(0, 0);
#pragma unroll
            for (int c = 0; c < 3; ++c) d[c].y = (T)0;
        } else if (kz > N / 2) {
            // a[0][N-ii] = conj(a[0][ii]), ii = N - kz in 1..N/2-1
            const cpx<T>* src = at(0, N - kz);
            cpx<T>* d = at(0, kz);
#pragma unroll
            for (int c = 0; c < 3; ++c) d[c] = conjg(src[c]);
        }
    } else if (ky > N / 2) {
        const int yy = N - ky;  // 1..N/2-1
        const int src_kz = (kz == 0) ? 0 : N - kz;
        const cpx<T>* src = at(yy, src_kz);
        cpx<T>* d = at(ky, kz);
#pragma unroll
        for (int c = 0; c < 3; ++c) d[c] = conjg(src[c]);
    }
}

// pointwise k-space kernels over the state layout ----------------------------
// compute_velocity (vorticity_equation.cpp:206-239), without the symmetrize
template <typename T, int N>
__global__ void velocity_kernel(const KParams kp, const cpx<T>* __restrict__ w, cpx<T>* u) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t npts = (size_t)N * N * kp.nxv;
    if (e >= npts) return;
    const int ix = (int)(e % kp.nxv);
    const size_t r = e / kp.nxv;
    const int kz_i = (int)(r % N), ky_i = (int)(r / N);
    const double kx = ix * kp.dkx, ky = kwrap<N>(ky_i, kp.dky), kz = kwrap<N>(kz_i, kp.dkz);
    const double k2 = (kx * kx + ky * ky) + kz * kz;
    const size_t pt = r * kp.nxp + ix;
    cpx<T> o[3];
    if (k2 <= kp.kM2 && k2 > 0.0) {
        cpx<T> wv[3] = {w[pt * 3], w[pt * 3 + 1], w[pt * 3 + 2]};
        curl<T>((T)kx, (T)ky, (T)kz, wv, o);
        const T ik2 = (T)__drcp_rn(k2);
#pragma unroll
        for (int c = 0; c < 3; ++c) o[c] = scale(o[c], ik2);
    } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) o[c] = zero_c<T>();
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) u[pt * 3 + c] = o[c];
}

// low_pass(kM) + force_divfree (vorticity_equation.hpp:121-126)
template <typename T, int N>
__global__ void lowpass_divfree_kernel(const KParams kp, cpx<T>* a) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t npts = (size_t)N * N * kp.nxv;
    if (e >= npts) return;
    const int ix = (int)(e % kp.nxv);
    const size_t r = e / kp.nxv;
    const int kz_i = (int)(r % N), ky_i = (int)(r / N);
    const double kx = ix * kp.dkx, ky = kwrap<N>(ky_i, kp.dky), kz = kwrap<N>(kz_i, kp.dkz);
    const double k2 = (kx * kx + ky * ky) + kz * kz;
    const size_t pt = r * kp.nxp + ix;
    cpx<T> v[3] = {a[pt * 3], a[pt * 3 + 1], a[pt * 3 + 2]};
    if (k2 >= kp.kM2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = zero_c<T>();
    }
    if (k2 > 0.0) divfree<T>((T)kx, (T)ky, (T)kz, (T)__drcp_rn(k2), v);
    if (e == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = zero_c<T>();
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) a[pt * 3 + c] = v[c];
}

}  // namespace bfg
