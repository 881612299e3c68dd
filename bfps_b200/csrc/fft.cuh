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
// A plan uses the largest power-of-two radix up to a cap MR (8, 16 or 32)
// that does not leave a lone radix-2 stage (plan_step below); the 16- and
// 32-point butterflies are two-level register transforms (dft_2l).
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
__host__ __device__ __forceinline__ cpx<T> mk(T a, T b) {
    cpx<T> r;
    r.x = a;
    r.y = b;
    return r;
}
// FP32 complex sums and scalings can use the paired FP32 instructions of
// sm_100 (__fadd2_rn / __fmul2_rn: one instruction for both parts, each part
// rounded as the scalar operation would be) with BFG_PACKED_F32=1; measured
// within 1 % of the scalar form on the passes (they are not bound by FP32
// issue), so it is off by default.
#ifndef BFG_PACKED_F32
#define BFG_PACKED_F32 0
#endif
template <typename T>
__host__ __device__ __forceinline__ cpx<T> operator+(cpx<T> a, cpx<T> b) {
#if defined(__CUDA_ARCH__) && BFG_PACKED_F32
    if constexpr (sizeof(T) == 4) {
        const float2 r = __fadd2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
        return mk<T>(r.x, r.y);
    }
#endif
    return mk<T>(a.x + b.x, a.y + b.y);
}
template <typename T>
__host__ __device__ __forceinline__ cpx<T> operator-(cpx<T> a, cpx<T> b) {
#if defined(__CUDA_ARCH__) && BFG_PACKED_F32
    if constexpr (sizeof(T) == 4) {
        const float2 r = __fadd2_rn(make_float2(a.x, a.y), make_float2(-b.x, -b.y));
        return mk<T>(r.x, r.y);
    }
#endif
    return mk<T>(a.x - b.x, a.y - b.y);
}
template <typename T>
__host__ __device__ __forceinline__ cpx<T> cmul(cpx<T> a, cpx<T> b) {
    return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T>
__host__ __device__ __forceinline__ cpx<T> cmulc(cpx<T> a, cpx<T> b) {  // a * conj(b)
    return mk<T>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename T>
__host__ __device__ __forceinline__ cpx<T> conjg(cpx<T> a) { return mk<T>(a.x, -a.y); }
template <typename T>
__host__ __device__ __forceinline__ cpx<T> scale(cpx<T> a, T s) {
#if defined(__CUDA_ARCH__) && BFG_PACKED_F32
    if constexpr (sizeof(T) == 4) {
        const float2 r = __fmul2_rn(make_float2(a.x, a.y), make_float2(s, s));
        return mk<T>(r.x, r.y);
    }
#endif
    return mk<T>(a.x * s, a.y * s);
}
// multiply by -i (forward sign) or +i (inverse sign)
template <typename T, bool INV>
__host__ __device__ __forceinline__ cpx<T> rot90(cpx<T> a) {
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
// radix of the first stage of a length-L transform with radices up to MR
__host__ __device__ constexpr int plan_step(int L, int MR) {
    return (L <= MR) ? L
                     : ((L % MR == 0 && L / MR != 2) ? MR : plan_step(L, MR / 2));
}
__host__ __device__ constexpr int plan_nstages(int L, int MR) {
    return L <= 1 ? 0 : 1 + plan_nstages(L / plan_step(L, MR), MR);
}
// radix of stage s
__host__ __device__ constexpr int plan_radix(int L, int s, int MR) {
    return s == 0 ? plan_step(L, MR) : plan_radix(L / plan_step(L, MR), s - 1, MR);
}
// block length at stage s (L at s = 0, divided by the earlier radices)
__host__ __device__ constexpr int plan_block(int L, int s, int MR) {
    return s == 0 ? L : plan_block(L / plan_step(L, MR), s - 1, MR);
}
// radix cap of a strided-axis transform: 32 in FP32 where the schedule asks
// for wide butterflies, 8 otherwise and always in FP64 (twice the registers
// per value)
template <typename T, bool WIDE>
__host__ __device__ constexpr int col_max_radix() {
    return (sizeof(T) == 4 && WIDE) ? 32 : 8;
}

// position of frequency k after a DIF of length L
template <int L, int MR>
__host__ __device__ __forceinline__ int dif_position(int k) {
    int pos = 0;
    int rem = k;
    int Lr = L;
#pragma unroll
    for (int s = 0; s < plan_nstages(L, MR); ++s) {
        const int R = plan_step(Lr, MR);
        const int q = rem % R;
        rem /= R;
        Lr /= R;
        pos += q * Lr;
    }
    return pos;
}

// ------------------------------------------------------- small DFTs --
template <typename T, bool INV>
__host__ __device__ __forceinline__ void dft2(cpx<T>* v) {
    cpx<T> t = v[0] - v[1];
    v[0] = v[0] + v[1];
    v[1] = t;
}
template <typename T, bool INV>
__host__ __device__ __forceinline__ void dft4(cpx<T>* v) {
    cpx<T> s02 = v[0] + v[2], d02 = v[0] - v[2];
    cpx<T> s13 = v[1] + v[3], d13 = rot90<T, INV>(v[1] - v[3]);
    v[0] = s02 + s13;
    v[2] = s02 - s13;
    v[1] = d02 + d13;
    v[3] = d02 - d13;
}
template <typename T, bool INV>
__host__ __device__ __forceinline__ void dft8(cpx<T>* v) {
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
// cos(2 pi j / 32) and sin(2 pi j / 32) for any integer j (compile-time
// constants once the butterfly loops are unrolled)
__host__ __device__ constexpr double cos_q8(int j) {  // cos(2 pi j / 32), 0 <= j <= 8
    return j == 0 ? 1.0
         : j == 1 ? 0.98078528040323044912618223613424
         : j == 2 ? 0.92387953251128675612818318939679
         : j == 3 ? 0.83146961230254523707878837761791
         : j == 4 ? 0.70710678118654752440084436210485
         : j == 5 ? 0.55557023301960222474283081394853
         : j == 6 ? 0.38268343236508977172845998403040
         : j == 7 ? 0.19509032201612826784828486847702
                  : 0.0;
}
__host__ __device__ constexpr double cos32(int j) {
    return (j & 31) <= 8 ? cos_q8(j & 31)
         : (j & 31) <= 16 ? -cos_q8(16 - (j & 31))
         : (j & 31) <= 24 ? -cos_q8((j & 31) - 16)
                          : cos_q8(32 - (j & 31));
}
__host__ __device__ constexpr double sin32(int j) { return cos32(j - 8); }

// v * W_R^m with W_R = exp(-+ 2 pi i / R) (forward / inverse), R | 32
template <typename T, bool INV, int R>
__host__ __device__ __forceinline__ cpx<T> mul_wr(cpx<T> v, int m) {
    const int j = ((m % R) + R) % R * (32 / R);  // angle in units of 2 pi / 32
    if (j == 0) return v;
    if (j == 16) return mk<T>(-v.x, -v.y);
    if (j == 8) return rot90<T, INV>(v);
    if (j == 24) return rot90<T, !INV>(v);
    const T c = (T)cos32(j), s = (T)sin32(j);
    // forward: v (c - i s); inverse: v (c + i s)
    return INV ? mk<T>(v.x * c - v.y * s, v.y * c + v.x * s)
               : mk<T>(v.x * c + v.y * s, v.y * c - v.x * s);
}

template <typename T, bool INV, int R>
__host__ __device__ __forceinline__ void dft(cpx<T>* v);

// Two-level DFT of R = R1 R2 points in registers, natural order in and out:
// R2 DFTs of R1 points (stride R2), twiddles W_R^(n2 k1), R1 DFTs of R2
// points.
template <typename T, bool INV, int R1, int R2>
__host__ __device__ __forceinline__ void dft_2l(cpx<T>* v) {
    constexpr int R = R1 * R2;
    cpx<T> t[R];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) {
        cpx<T> a[R1];
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) a[n1] = v[n1 * R2 + n2];
        dft<T, INV, R1>(a);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) t[k1 * R2 + n2] = mul_wr<T, INV, R>(a[k1], n2 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
        cpx<T> b[R2];
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) b[n2] = t[k1 * R2 + n2];
        dft<T, INV, R2>(b);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = b[k2];
    }
}

template <typename T, bool INV, int R>
__host__ __device__ __forceinline__ void dft(cpx<T>* v) {
    if constexpr (R == 1) return;
    else if constexpr (R == 2) dft2<T, INV>(v);
    else if constexpr (R == 4) dft4<T, INV>(v);
    else if constexpr (R == 8) dft8<T, INV>(v);
    else if constexpr (R == 16) dft_2l<T, INV, 4, 4>(v);
    else dft_2l<T, INV, 4, 8>(v);  // 32
}

template <typename T, bool INV>
__host__ __device__ __forceinline__ cpx<T> twiddle(const cpx<T>* tw, int idx) {
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
    __host__ __device__ __forceinline__ static int base(int p) {
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
__host__ __device__ __forceinline__ void stage_item(int w, int& p, int& b, int& j) {
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

// One DIF stage S of a length-L transform over P pencils (radices up to MR).
template <typename T, int L, int S, bool INV, int P, class LAY, int MAP, int TAB, int MR>
__host__ __device__ __forceinline__ void dif_stage(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    constexpr int R = plan_radix(L, S, MR);
    constexpr int Ls = plan_block(L, S, MR);
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
template <typename T, int L, int S, bool INV, int P, class LAY, int MAP, int TAB, int MR>
__host__ __device__ __forceinline__ void dit_stage(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    constexpr int R = plan_radix(L, S, MR);
    constexpr int Ls = plan_block(L, S, MR);
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
template <typename T, int L, int S, int SEND, bool INV, int P, class LAY, int MAP, int TAB, int MR>
__device__ __forceinline__ void dif_range(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    if constexpr (S < SEND) {
        dif_stage<T, L, S, INV, P, LAY, MAP, TAB, MR>(s, tw, tid, nthr);
        __syncthreads();
        dif_range<T, L, S + 1, SEND, INV, P, LAY, MAP, TAB, MR>(s, tw, tid, nthr);
    }
}
// Full DIF transform: natural in, digit-reversed out.  Ends with a barrier.
template <typename T, int L, bool INV, int P, class LAY, int MAP, int TAB, int MR>
__device__ __forceinline__ void dif(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    dif_range<T, L, 0, plan_nstages(L, MR), INV, P, LAY, MAP, TAB, MR>(s, tw, tid, nthr);
}

// DIT stages S down to SLO (inclusive), each followed by a barrier.
template <typename T, int L, int S, int SLO, bool INV, int P, class LAY, int MAP, int TAB, int MR>
__device__ __forceinline__ void dit_range(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    if constexpr (S >= SLO) {
        dit_stage<T, L, S, INV, P, LAY, MAP, TAB, MR>(s, tw, tid, nthr);
        __syncthreads();
        dit_range<T, L, S - 1, SLO, INV, P, LAY, MAP, TAB, MR>(s, tw, tid, nthr);
    }
}
// Full DIT transform: digit-reversed in, natural out.  Ends with a barrier.
template <typename T, int L, bool INV, int P, class LAY, int MAP, int TAB, int MR>
__device__ __forceinline__ void dit(cpx<T>* s, const cpx<T>* tw, int tid, int nthr) {
    dit_range<T, L, plan_nstages(L, MR) - 1, 0, INV, P, LAY, MAP, TAB, MR>(s, tw, tid, nthr);
}

// frequency held at DIF output position p of a length-L transform
template <int L, int MR>
__host__ __device__ __forceinline__ int dif_frequency(int p) {
    int k = 0, mult = 1, Lr = L, rem = p;
#pragma unroll
    for (int s = 0; s < plan_nstages(L, MR); ++s) {
        const int R = plan_step(Lr, MR);
        Lr /= R;
        const int q = rem / Lr;
        rem -= q * Lr;
        k += q * mult;
        mult *= R;
    }
    return k;
}

}  // namespace bfg
