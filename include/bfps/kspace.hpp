/*
 * kspace.hpp -- drop-in replacement for bfps/cpp/kspace.hpp (bfps_b200).
 *
 * kspace<be, dt> with the reference's public members (kspace.hpp:43-110):
 * wavenumber tables kx, ky, kz; kM, dk, nshells, kshell, nshell; the smooth
 * dealiasing filter keyed by round(k2 / dk2); and the CLOOP, CLOOP_K2,
 * CLOOP_K2_NXMODES loops (kspace.hpp:117-192) over the complex layout, plus
 * low_pass, dealias and force_divfree on host arrays (kspace.cpp:235-253,
 * 461-519).  The tables are built on the host in the reference's order
 * (kspace.cpp:34-167; the filter entry written last in CLOOP order wins, as
 * with one OpenMP thread).  The solver's own k-space work runs on the GPU
 * inside include/bfps_b200.h; these host methods serve code that works on
 * a field's host copy.
 */
#ifndef BFPS_B200_KSPACE_HPP
#define BFPS_B200_KSPACE_HPP

#include <cmath>
#include <unordered_map>
#include <vector>

#include "field_layout.hpp"

enum kspace_dealias_type { TWO_THIRDS, SMOOTH };

template <typename rnumber>
struct fftw_interface {
    typedef rnumber complex[2];
};

template <field_backend be, kspace_dealias_type dt>
class kspace {
  public:
    field_layout<ONE>* layout;
    double dkx, dky, dkz, dk, dk2;
    double kMx, kMy, kMz, kM, kM2;
    std::vector<double> kx, ky, kz;
    std::unordered_map<int, double> dealias_filter;
    std::vector<double> kshell;
    std::vector<int64_t> nshell;
    int nshells;

    template <field_components fc>
    kspace(const field_layout<fc>* source_layout, const double DKX = 1.0, const double DKY = 1.0,
           const double DKZ = 1.0) {
        layout = new field_layout<ONE>(source_layout->sizes, source_layout->subsizes,
                                       source_layout->starts, source_layout->comm);
        dkx = DKX;
        dky = DKY;
        dkz = DKZ;
        const hsize_t s0 = layout->sizes[0], s1 = layout->sizes[1], s2 = layout->sizes[2];
        kx.resize(s2);
        ky.resize(s0);
        kz.resize(s1);
        for (hsize_t i = 0; i < s2; ++i) kx[i] = (double)i * dkx;
        // kspace.cpp:60-74: ky wraps at sizes[1] / 2, kz at sizes[0] / 2
        for (hsize_t i = 0; i < s0; ++i)
            ky[i] = (i <= s1 / 2) ? dky * (double)i : dky * ((double)i - (double)s1);
        for (hsize_t i = 0; i < s1; ++i)
            kz[i] = (i <= s0 / 2) ? dkz * (double)i : dkz * ((double)i - (double)s0);
        if (dt == TWO_THIRDS) {  // kspace.cpp:75-93
            kMx = dkx * (int(2 * (s2 - 1) / 3) - 1);
            kMy = dky * (int(s0 / 3) - 1);
            kMz = dkz * (int(s1 / 3) - 1);
        } else {
            kMx = dkx * (int(s2 - 2));
            kMy = dky * (int(s0 / 2) - 1);
            kMz = dkz * (int(s1 / 2) - 1);
        }
        kM = kMx;
        if (kM < kMy) kM = kMy;
        if (kM < kMz) kM = kMz;
        kM2 = kM * kM;
        dk = dkx;
        if (dk > dky) dk = dky;
        if (dk > dkz) dk = dkz;
        dk2 = dk * dk;
        nshells = int(kM / dk) + 2;
        kshell.assign(nshells, 0.0);
        nshell.assign(nshells, 0);
        CLOOP_K2_NXMODES([&](ptrdiff_t, ptrdiff_t, ptrdiff_t, ptrdiff_t, double k2, int nxmodes) {
            if (k2 < kM2) {
                const double knorm = std::sqrt(k2);
                kshell[int(knorm / dk)] += nxmodes * knorm;
                nshell[int(knorm / dk)] += nxmodes;
            }
            if (dt == SMOOTH)
                dealias_filter[int(std::round(k2 / dk2))] = std::exp(-36.0 * std::pow(k2 / kM2, 18.));
        });
        for (int n = 0; n < nshells; ++n)
            if (nshell[n] != 0) kshell[n] /= nshell[n];
    }
    ~kspace() { delete layout; }
    kspace(const kspace&) = delete;
    kspace& operator=(const kspace&) = delete;

    template <class func_type>
    void CLOOP(func_type expression) {
        for (hsize_t yindex = 0; yindex < layout->subsizes[0]; yindex++)
            for (hsize_t zindex = 0; zindex < layout->subsizes[1]; zindex++) {
                ptrdiff_t cindex = (yindex * layout->subsizes[1] + zindex) * layout->subsizes[2];
                for (hsize_t xindex = 0; xindex < layout->subsizes[2]; xindex++)
                    expression(cindex++, xindex, yindex, zindex);
            }
    }
    template <class func_type>
    void CLOOP_K2(func_type expression) {
        CLOOP([&](ptrdiff_t cindex, ptrdiff_t xindex, ptrdiff_t yindex, ptrdiff_t zindex) {
            const double k2 =
                kx[xindex] * kx[xindex] + ky[yindex] * ky[yindex] + kz[zindex] * kz[zindex];
            expression(cindex, xindex, yindex, zindex, k2);
        });
    }
    template <class func_type>
    void CLOOP_K2_NXMODES(func_type expression) {
        CLOOP([&](ptrdiff_t cindex, ptrdiff_t xindex, ptrdiff_t yindex, ptrdiff_t zindex) {
            const double k2 =
                kx[xindex] * kx[xindex] + ky[yindex] * ky[yindex] + kz[zindex] * kz[zindex];
            expression(cindex, xindex, yindex, zindex, k2, xindex == 0 ? 1 : 2);
        });
    }

    /* kspace.cpp:235-253: zero every mode with k2 >= kmax^2 */
    template <typename rnumber, field_components fc>
    void low_pass(typename fftw_interface<rnumber>::complex* __restrict__ a, const double kmax) {
        const double km2 = kmax * kmax;
        CLOOP_K2([&](ptrdiff_t cindex, ptrdiff_t, ptrdiff_t, ptrdiff_t, double k2) {
            if (k2 >= km2)
                for (unsigned t = 0; t < 2 * ncomp(fc); ++t) ((rnumber*)a)[2 * ncomp(fc) * cindex + t] = 0;
        });
    }
    /* kspace.cpp:461-485 */
    template <typename rnumber, field_components fc>
    void dealias(typename fftw_interface<rnumber>::complex* __restrict__ a) {
        if (dt == TWO_THIRDS) {
            low_pass<rnumber, fc>(a, kM);
            return;
        }
        CLOOP_K2([&](ptrdiff_t cindex, ptrdiff_t, ptrdiff_t, ptrdiff_t, double k2) {
            const double tval = dealias_filter[int(std::round(k2 / dk2))];
            for (unsigned t = 0; t < 2 * ncomp(fc); ++t) ((rnumber*)a)[2 * ncomp(fc) * cindex + t] *= tval;
        });
    }
    /* kspace.cpp:487-519, then the zero mode */
    template <typename rnumber>
    void force_divfree(typename fftw_interface<rnumber>::complex* __restrict__ a) {
        CLOOP_K2([&](ptrdiff_t cindex, ptrdiff_t xindex, ptrdiff_t yindex, ptrdiff_t zindex, double k2) {
            if (k2 > 0) {
                rnumber* v = (rnumber*)a + 6 * cindex;
                const double kk[3] = {kx[xindex], ky[yindex], kz[zindex]};
                double tr = 0, ti = 0;
                for (int c = 0; c < 3; ++c) {
                    tr += kk[c] * v[2 * c];
                    ti += kk[c] * v[2 * c + 1];
                }
                tr /= k2;
                ti /= k2;
                for (int c = 0; c < 3; ++c) {
                    v[2 * c] -= (rnumber)(tr * kk[c]);
                    v[2 * c + 1] -= (rnumber)(ti * kk[c]);
                }
            }
        });
        for (int t = 0; t < 6; ++t) ((rnumber*)a)[t] = 0;
    }
};

#endif
