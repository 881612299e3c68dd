// Shared-memory FFT building blocks for the sm_100a NSVE kernels.
//
// All transforms here are power-of-two, in place, on "pencils" that live in
// shared memory.  A pencil of length L is addressed as
//     s[p * PS + e * ES]      (pencil p, element e)
// so the same code serves the strided-axis passes (pencils side by side,
// ES = row pitch, PS = 1) and the row pass (pencils contiguous, ES = 1).
//
// Two in-place forms are used:
//   * DIF (Gentleman-Sande): natural-order input, digit-reversed output;
//   * DIT (Cooley-Tukey):    digit-reversed input, natural-order output.
// The digit order of a length-L transform with stage radices R1, R2, ... is
//   position(k) = q1*(L/R1) + q2*(L/(R1*R2)) + ...,  k = q1 + R1*(q2 + R2*(...)).
// Radices are 8, then 4 or 2 for the remainder (plan_step below).
//
// Twiddles come from one table tw[m] = exp(-2*pi*i*m/TAB), m < TAB, built on
// the host in long double and rounded once to the working precision; any
// transform length L dividing TAB indexes it with stride TAB/L.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bfg {

template <typename T>
struct __align__(2 * sizeof(T)) cpx {
    T x, y;
};

template <typename T>
__device__ __forceinline__ cpx<T> mk(T a, T b) {
    cpx<T> r;
    r.x = a;
    r.y = b;
    return r;
}
template <typename T>
__device__ __forceinline__ cpx<T> operator+(cpx<T> a, cpx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T>
__device__ __forceinline__ cpx<T> operator-(cpx<T> a, cpx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T>
__device__ __forceinline__ cpx<T> cmul(cpx<T> a, cpx<T> b) {
    return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T>
__device__ __forceinline__ cpx<T> cmulc(cpx<T> a, cpx<T> b) {  // a * conj(b)
    return mk<T>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename T>
__device__ __forceinline__ cpx<T> conjg(cpx<T> a) { return mk<T>(a.x, -a.y); }
template <typename T>
__device__ __forceinline__ cpx<T> scale(cpx<T> a, T s) { return mk<T>(a.x * s, a.y * s); }
// multiply by -i (forward sign) or +i (inverse sign)
template <typename T, bool INV>
__device__ __forceinline__ cpx<T> rot90(cpx<T> a) {
    return INV ? mk<T>(-a.y, a.x) : mk<T>(a.y, -a.x);
}

// ------------------------------------------------------ async copies --
// cp.async (global -> shared, bypassing registers), PTX ISA 7.0+.
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND) : "memory");
}
// copy of VB bytes (16 or 8)
template <int VB>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
    if constexpr (VB == 16) cp_async16(dst, src);
    else cp_async8(dst, src);
}
template <int VB>
struct vec_of;
template <>
struct vec_of<16> {
    using type = float4;
};
template <>
struct vec_of<8> {
    using type = float2;
};

// ---------------------------------------------------------------- plans --
__host__ __device__ constexpr int plan_step(int L) {
    return (L % 8 == 0 && L / 8 != 2) ? 8 : ((L % 4 == 0) ? 4 : 2);
}
__host__ __device__ constexpr int plan_nstages(int L) {
    return L <= 1 ? 0 : 1 + plan_nstages(L / plan_step(L));
}
// radix of stage s
__host__ __device__ constexpr int plan_radix(int L, int s) {
    return s == 0 ? plan_step(L) : plan_radix(L / plan_step(L), s - 1);
}
// block length at stage s (L at s = 0, divided by the earlier radices)
__host__ __device__ constexpr int plan_block(int L, int s) {
    return s == 0 ? L : plan_block(L / plan_step(L), s - 1);
}

// position of frequency k after a DIF of length L
template <int L>
__device__ __forceinline__ int dif_position(int k) {
    int pos = 0;
    int rem = k;
    int Lr = L;
#pragma unroll
    for (int s = 0; s < plan_nstages(L); ++s) {
        const int R = plan_step(Lr);
        const int q = rem % R;
        rem /= R;
        Lr /= R;
        pos += q * Lr;
    }
    return pos;
}

// ------------------------------------------------------- small DFTs --
template <typename T, bool INV>
__device__ __forceinline__ void dft2(cpx<T>* v) {
    cpx<T> t = v[0] - v[1];
    v[0] = v[0] + v[1];
    v[1] = t;
}
template <typename T, bool INV>
__device__ __forceinline__ void dft4(cpx<T>* v) {
    cpx<T> s02 = v[0] + v[2], d02 = v[0] - v[2];
    cpx<T> s13 = v[1] + v[3], d13 = rot90<T, INV>(v[1] - v[3]);
    v[0] = s02 + s13;
    v[2] = s02 - s13;
    v[1] = d02 + d13;
    v[3] = d02 - d13;
}
template <typename T, bool INV>
__device__ __forceinline__ void dft8(cpx<T>* v) {
    cpx<T> e[4] = {v[0], v[2], v[4], v[6]};
    cpx<T> o[4] = {v[1], v[3], v[5], v[7]};
    dft4<T, INV>(e);
    dft4<T, INV>(o);
    const T h = (T)0.70710678118654752440084436210484903928;  // 1/sqrt(2)
    // o[q] *= exp(-+ 2 pi i q / 8)
    o[1] = INV ? mk<T>(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
               : mk<T>(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    o[2] = rot90<T, INV>(o[2]);
    o[3] = INV ? mk<T>(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
               : mk<T>(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        v[q] = e[q] + o[q];
        v[q + 4] = e[q] - o[q];
    }
}
template <typename T, bool INV, int R>
__device__ __forceinline__ void dft(cpx<T>* v) {
    if constexpr (R == 2) dft2<T, INV>(v);
    else if constexpr (R == 4) dft4<T, INV>(v);
    else dft8<T, INV>(v);
}

template <typename T, bool INV>
__device__ __forceinline__ cpx<T> twiddle(const cpx<T>* tw, int idx) {
    cpx<T> t = tw[idx];
    if (INV) t.y = -t.y;
    return t;
}

// ----------------------------------------------------------- stages --
// Pencil layout in shared memory: pencil p starts at
//   base(p) = (p / PG) * GS + (p % PG) * PS
// and its element e sits at base(p) + e * ES.  Examples: pencils side by side
// in a tile row (PG = 1, GS = 1, ES = row pitch); contiguous pencils
// (PG = 1, GS = pitch, ES = 1); the three components of interleaved rows
// (PG = 3, GS = row length, PS = 1, ES = 3).
template <int PG_, int GS_, int PS_, int ES_>
struct Lay {
    static constexpr int PG = PG_, GS = GS_, PS = PS_, ES = ES_;
    __device__ __forceinline__ static int base(int p) {
        return PG == 1 ? p * GS : (p / PG) * GS + (p % PG) * PS;
    }
};

// MAP (thread -> butterfly order): 1 = consecutive threads take consecutive
// pencils; 0 = consecutive threads take consecutive elements; 2 = elements
// while a stage's butterfly span is >= 32, pencils below.
__host__ __device__ constexpr bool map_pencil_fast(int MAP, int span) {
    return MAP == 1 || (MAP == 2 && span < 32);
}

// decode work item w of stage (P pencils, NBLK blocks, span) into (p, b, j)
template <int P, int NBLK, int span, bool PF>
__device__ __forceinline__ void stage_item(int w, int& p, int& b, int& j) {
    if (PF) {
        p = w % P;
        const int r = w / P;
        j = r % span;
        b = r / span;
    } else {
        j = w % span;
        const int r = w / span;
        b = r % NBLK;
        p = r / NBLK;
    }
}

// One DIF stage S of a length-L transform over P pencils.
template <typename T, int L, int S, bool INV, int P, class LAY, int MAP, int TAB>
__device__ __forceinline__ void dif_stage(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    constexpr int R = plan_radix(L, S);
    constexpr int Ls = plan_block(L, S);
    constexpr int span = Ls / R;
    constexpr int NBLK = L / Ls;
    constexpr int NW = P * NBLK * span;
    constexpr int ES = LAY::ES;
    for (int w = tid; w < NW; w += nthr) {
        int p, b, j;
        stage_item<P, NBLK, span, map_pencil_fast(MAP, span)>(w, p, b, j);
        const int base = LAY::base(p) + (b * Ls + j) * ES;
        cpx<T> v[R];
#pragma unroll
        for (int m = 0; m < R; ++m) v[m] = s[base + m * span * ES];
        dft<T, INV, R>(v);
        if (span > 1) {
#pragma unroll
            for (int q = 1; q < R; ++q) v[q] = cmul(v[q], twiddle<T, INV>(tw, j * q * (TAB / Ls)));
        }
#pragma unroll
        for (int q = 0; q < R; ++q) s[base + q * span * ES] = v[q];
    }
}

// One DIT stage S (stages run from the last DIF stage back to stage 0).
template <typename T, int L, int S, bool INV, int P, class LAY, int MAP, int TAB>
__device__ __forceinline__ void dit_stage(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    constexpr int R = plan_radix(L, S);
    constexpr int Ls = plan_block(L, S);
    constexpr int span = Ls / R;
    constexpr int NBLK = L / Ls;
    constexpr int NW = P * NBLK * span;
    constexpr int ES = LAY::ES;
    for (int w = tid; w < NW; w += nthr) {
        int p, b, j;
        stage_item<P, NBLK, span, map_pencil_fast(MAP, span)>(w, p, b, j);
        const int base = LAY::base(p) + (b * Ls + j) * ES;
        cpx<T> v[R];
#pragma unroll
        for (int m = 0; m < R; ++m) v[m] = s[base + m * span * ES];
        if (span > 1) {
#pragma unroll
            for (int m = 1; m < R; ++m) v[m] = cmul(v[m], twiddle<T, INV>(tw, j * m * (TAB / Ls)));
        }
        dft<T, INV, R>(v);
#pragma unroll
        for (int q = 0; q < R; ++q) s[base + q * span * ES] = v[q];
    }
}

// DIF stages [S, SEND), each followed by a barrier.
template <typename T, int L, int S, int SEND, bool INV, int P, class LAY, int MAP, int TAB>
__device__ __forceinline__ void dif_range(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    if constexpr (S < SEND) {
        dif_stage<T, L, S, INV, P, LAY, MAP, TAB>(s, tw, tid, nthr);
        __syncthreads();
        dif_range<T, L, S + 1, SEND, INV, P, LAY, MAP, TAB>(s, tw, tid, nthr);
    }
}
// Full DIF transform: natural in, digit-reversed out.  Ends with a barrier.
template <typename T, int L, bool INV, int P, class LAY, int MAP, int TAB>
__device__ __forceinline__ void dif(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    dif_range<T, L, 0, plan_nstages(L), INV, P, LAY, MAP, TAB>(s, tw, tid, nthr);
}

template <typename T, int L, int S, bool INV, int P, class LAY, int MAP, int TAB>
__device__ __forceinline__ void dit_down(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    if constexpr (S >= 0) {
        dit_stage<T, L, S, INV, P, LAY, MAP, TAB>(s, tw, tid, nthr);
        __syncthreads();
        dit_down<T, L, S - 1, INV, P, LAY, MAP, TAB>(s, tw, tid, nthr);
    }
}
// DIT stages S down to SLO (inclusive), each followed by a barrier.
template <typename T, int L, int S, int SLO, bool INV, int P, class LAY, int MAP, int TAB>
__device__ __forceinline__ void dit_range(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    if constexpr (S >= SLO) {
        dit_stage<T, L, S, INV, P, LAY, MAP, TAB>(s, tw, tid, nthr);
        __syncthreads();
        dit_range<T, L, S - 1, SLO, INV, P, LAY, MAP, TAB>(s, tw, tid, nthr);
    }
}
// Full DIT transform: digit-reversed in, natural out.  Ends with a barrier.
template <typename T, int L, bool INV, int P, class LAY, int MAP, int TAB>
__device__ __forceinline__ void dit(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    dit_down<T, L, plan_nstages(L) - 1, INV, P, LAY, MAP, TAB>(s, tw, tid, nthr);
}

// frequency held at DIF output position p of a length-L transform
template <int L>
__device__ __forceinline__ int dif_frequency(int p) {
    int k = 0, mult = 1, Lr = L, rem = p;
#pragma unroll
    for (int s = 0; s < plan_nstages(L); ++s) {
        const int R = plan_step(Lr);
        Lr /= R;
        const int q = rem / Lr;
        rem -= q * Lr;
        k += q * mult;
        mult *= R;
    }
    return k;
}

}  // namespace bfg
