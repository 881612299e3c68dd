// Field statistics of NSVE::do_stats as device reductions.
//
// * co-spectrum (kspace::cospectrum, bfps/cpp/kspace.cpp:521-598):
//   spec[int(|k|/dk)][i][j] += w * (Re a_i Re a_j + Im a_i Im a_j) over
//   k^2 <= kM^2, w = 1 on the kx = 0 plane and 2 elsewhere.  Summed in a
//   fixed order (per-warp shell arrays filled by segmented scans, warps
//   added in order, block partials added in order): deterministic.
// * real-space moments and histograms (field::compute_rspace_stats,
//   bfps/cpp/field.cpp:661-889): min / <v^n>, n = 1..8 / max of the three
//   components and the magnitude, with the reference's initial values (0 for
//   the component extrema, max_estimate for the magnitude minimum).  Each
//   block writes its partials; one block reduces them in block order, so
//   the moments are deterministic.  Histogram counts are integer atomics.
#pragma once
#include "fft.cuh"
#include "passes.cuh"

namespace bfg {

constexpr int STATS_BLOCKS = 1184;  // 8 x 148 SMs
constexpr int STATS_THREADS = 256;
constexpr int NQ = 40;  // 10 moments x 4 values

// Co-spectrum with a fixed order of summation (the result does not depend
// on scheduling: the same field gives the same bits, alone or beside other
// work).  Block b takes the ky planes b, b + grid, ...; warp w of a block the
// kz rows w, w + SPEC_WARPS, ...; lanes take 32 consecutive kx of a row.
// Along a row the shell index int(|k|/dk) does not decrease with kx, so the
// lanes of one shell form a contiguous run: a segmented inclusive scan
// (shuffles in a fixed pattern) sums each run, and the run's last lane adds
// it to its warp's own shell array in shared memory (no two lanes of a warp
// touch the same shell at once, and a warp's additions come in a fixed
// order).  The block then adds its warps' arrays in warp order into its
// partial, and spectrum_final adds the partials in block order.
constexpr int SPEC_BLOCKS = 148;
constexpr int SPEC_WARPS_MAX = 4;

__device__ __forceinline__ double shfl_up_d(double v, int o) {
    return __shfl_up_sync(0xffffffffu, v, o);
}

template <typename T, int N>
__global__ void __launch_bounds__(SPEC_WARPS_MAX * 32)
spectrum_kernel(const KParams kp, const cpx<T>* __restrict__ f, int nshells, double dk,
                double* __restrict__ partial) {
    extern __shared__ double sh[];  // warps x nshells x 9
    const int nwarps = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int ns9 = nshells * 9;
    for (int i = threadIdx.x; i < nwarps * ns9; i += blockDim.x) sh[i] = 0.0;
    __syncthreads();
    double* mine = sh + (size_t)wid * ns9;
    const int nxv = kp.nxv;
    for (int ky_i = blockIdx.x; ky_i < N; ky_i += gridDim.x) {
        const double ky = kwrap<N>(ky_i, kp.dky);
        for (int kz_i = wid; kz_i < N; kz_i += nwarps) {
            const double kz = kwrap<N>(kz_i, kp.dkz);
            const size_t r = (size_t)ky_i * N + kz_i;
            for (int x0 = 0; x0 < nxv; x0 += 32) {
                const int ix = x0 + lane;
                int sidx = -1;
                double v[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) v[q] = 0.0;
                if (ix < nxv) {
                    const double kx = ix * kp.dkx;
                    const double k2 = (kx * kx + ky * ky) + kz * kz;
                    if (k2 <= kp.kM2) {
                        sidx = (int)(sqrt(k2) / dk);
                        const double w = ix == 0 ? 1.0 : 2.0;
                        const size_t pt = r * kp.nxp + ix;
                        double re[3], im[3];
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const cpx<T> a = f[pt * 3 + c];
                            re[c] = (double)a.x;
                            im[c] = (double)a.y;
                        }
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int j = 0; j < 3; ++j) v[i * 3 + j] = w * (re[i] * re[j] + im[i] * im[j]);
                    }
                }
                // segmented inclusive scan over runs of equal shell index
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int so = __shfl_up_sync(0xffffffffu, sidx, o);
                    const bool take = lane >= o && so == sidx;
#pragma unroll
                    for (int q = 0; q < 9; ++q) {
                        const double u = shfl_up_d(v[q], o);
                        if (take) v[q] += u;
                    }
                }
                const int snext = __shfl_down_sync(0xffffffffu, sidx, 1);
                const bool tail = lane == 31 || snext != sidx;
                if (tail && sidx >= 0) {
#pragma unroll
                    for (int q = 0; q < 9; ++q) mine[sidx * 9 + q] += v[q];
                }
                __syncwarp();
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ns9; i += blockDim.x) {
        double acc = sh[i];
        for (int w = 1; w < nwarps; ++w) acc += sh[(size_t)w * ns9 + i];
        partial[(size_t)blockIdx.x * ns9 + i] = acc;
    }
}

// the block partials added in block order
__global__ void spectrum_final(const double* __restrict__ partial, int nblocks, int ns9,
                               double* __restrict__ spec) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns9) return;
    double acc = partial[i];
    for (int b = 1; b < nblocks; ++b) acc += partial[(size_t)b * ns9 + i];
    spec[i] = acc;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// partial layout per block: [q] with q = moment*4 + value
template <typename T>
__global__ void __launch_bounds__(STATS_THREADS)
moments_kernel(const T* __restrict__ r, size_t npts, double me0, double me1, double me2,
               double me3, int nbins, double* __restrict__ partial,
               unsigned long long* __restrict__ hist) {
    extern __shared__ unsigned int shist[];  // nbins * 4
    __shared__ double red[STATS_THREADS / 32][NQ];
    for (int i = threadIdx.x; i < nbins * 4; i += blockDim.x) shist[i] = 0;
    __syncthreads();
    const double me[4] = {me0, me1, me2, me3};
    double binsize[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) binsize[i] = 2 * me[i] / nbins;
    double mn[4] = {0.0, 0.0, 0.0, me3};
    double mx[4] = {0.0, 0.0, 0.0, 0.0};
    double sm[8][4];
#pragma unroll
    for (int n = 0; n < 8; ++n)
#pragma unroll
        for (int i = 0; i < 4; ++i) sm[n][i] = 0.0;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < npts;
         e += (size_t)gridDim.x * blockDim.x) {
        double v[4];
        v[3] = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            v[i] = (double)r[e * 3 + i];
            v[3] += v[i] * v[i];
        }
        v[3] = sqrt(v[3]);
        {
            const int b = (int)floor(v[3] * 2 / binsize[3]);
            if (b >= 0 && b < nbins) atomicAdd(&shist[b * 4 + 3], 1u);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int b = (int)floor((v[i] + me[i]) / binsize[i]);
            if (b >= 0 && b < nbins) atomicAdd(&shist[b * 4 + i], 1u);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            mn[i] = fmin(mn[i], v[i]);
            mx[i] = fmax(mx[i], v[i]);
            double p = 1.0;
#pragma unroll
            for (int n = 0; n < 8; ++n) {
                p = v[i] * p;
                sm[n][i] += p;
            }
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double a = warp_min(mn[i]);
        double b = warp_max(mx[i]);
        if (lane == 0) {
            red[wid][0 * 4 + i] = a;
            red[wid][9 * 4 + i] = b;
        }
#pragma unroll
        for (int n = 0; n < 8; ++n) {
            double s = warp_sum(sm[n][i]);
            if (lane == 0) red[wid][(n + 1) * 4 + i] = s;
        }
    }
    __syncthreads();
    if (threadIdx.x < NQ) {
        const int q = threadIdx.x;
        double acc = red[0][q];
        for (int w = 1; w < STATS_THREADS / 32; ++w) {
            const double v = red[w][q];
            if (q < 4) acc = fmin(acc, v);
            else if (q >= 36) acc = fmax(acc, v);
            else acc += v;
        }
        partial[(size_t)blockIdx.x * NQ + q] = acc;
    }
    for (int i = threadIdx.x; i < nbins * 4; i += blockDim.x)
        if (shist[i]) atomicAdd(&hist[i], (unsigned long long)shist[i]);
}

__global__ void moments_final(const double* __restrict__ partial, int nblocks, double inv_npts,
                              double* __restrict__ out) {
    const int q = threadIdx.x;
    if (q >= NQ) return;
    double acc = partial[q];
    for (int b = 1; b < nblocks; ++b) {
        const double v = partial[(size_t)b * NQ + q];
        if (q < 4) acc = fmin(acc, v);
        else if (q >= 36) acc = fmax(acc, v);
        else acc += v;
    }
    if (q >= 4 && q < 36) acc *= inv_npts;
    out[q] = acc;
}

// count of non-finite values in a buffer (bfg_check_finite)
template <typename T>
__global__ void nonfinite_kernel(const T* __restrict__ a, size_t n,
                                 unsigned long long* __restrict__ count) {
    unsigned long long local = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        if (!isfinite(a[i])) ++local;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

}  // namespace bfg
