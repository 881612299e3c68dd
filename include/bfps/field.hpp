/*
 * field.hpp -- drop-in replacement for bfps/cpp/field.hpp (bfps_b200).
 *
 * field<rnumber, be, fc> with the reference's public interface
 * (field.hpp:53-289): npoints, real_space_representation, the layouts
 * clayout / rlayout / rmemlayout, dft / ift / normalize / symmetrize,
 * get_rdata / get_cdata / rval / cval, assignment from arrays, RLOOP,
 * get_cindex / get_rindex, impose_zero_mode, and compute_stats.
 *
 * The data lives on the host in the reference's in-place layout (real
 * (nz, ny, nx+2, ncomp), complex (ny, nz, nx/2+1, ncomp)).  A field that
 * belongs to a vorticity_equation (cvorticity, cvelocity) is also backed by
 * that solver's device buffers: a coherence flag says which copy is current
 * (host, device or both); the solver's methods run on the device copy and
 * the first host access afterwards downloads it (a non-const access marks
 * the host copy as the current one, so the next device method uploads it).
 * Transforms and statistics of 3-component fields run on the GPU through
 * the C-ABI (bfg_ift / bfg_dft / bfg_field_stats, on host memory, through a
 * shared context per grid); 1- and 9-component fields keep their host data
 * and accessors, and their transforms report an error (the device engine
 * transforms 3-vectors).
 */
#ifndef BFPS_B200_FIELD_HPP
#define BFPS_B200_FIELD_HPP

#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "bfps_b200.h"
#include "field_layout.hpp"
#include "kspace.hpp"

namespace bfps_b200_compat {

inline void check(int rc, const bfg_ctx* ctx, const char* what) {
    if (rc != BFG_OK)
        throw std::runtime_error(std::string(what) + ": " + (ctx ? bfg_last_error(ctx) : "") +
                                 " (code " + std::to_string(rc) + ")");
}

// one context per (grid, precision, dk, dealiasing) for the transforms and
// statistics of fields that do not belong to a solver; kept for the process
inline bfg_ctx* shared_ctx(int nx, int ny, int nz, int real_bytes, double dkx = 1.0,
                           double dky = 1.0, double dkz = 1.0, int dealias = BFG_SMOOTH) {
    typedef std::tuple<int, int, int, int, double, double, double, int> key_t;
    static std::map<key_t, std::unique_ptr<bfg_ctx, void (*)(bfg_ctx*)>> ctxs;
    const key_t k(nx, ny, nz, real_bytes, dkx, dky, dkz, dealias);
    auto it = ctxs.find(k);
    if (it != ctxs.end()) return it->second.get();
    bfg_ctx* c = nullptr;
    check(bfg_ctx_create(&c, nx, ny, nz, dkx, dky, dkz, real_bytes, dealias, 0), nullptr,
          "bfg_ctx_create");
    ctxs.emplace(k, std::unique_ptr<bfg_ctx, void (*)(bfg_ctx*)>(c, bfg_ctx_destroy));
    return c;
}

enum where_t { ON_HOST, ON_DEVICE, ON_BOTH };

}  // namespace bfps_b200_compat

template <typename rnumber, field_backend be, field_components fc>
class field {
  private:
    mutable std::vector<rnumber> data_;
    // device link: the solver context and its field id (-1: none)
    bfg_ctx* link_ctx_ = nullptr;
    int link_id_ = -1;
    mutable bfps_b200_compat::where_t where_ = bfps_b200_compat::ON_HOST;
    int nx_, ny_, nz_;

  public:
    hsize_t npoints;
    bool real_space_representation;
    int myrank, nprocs;
    MPI_Comm comm;
    field_layout<fc>*clayout, *rlayout, *rmemlayout;
    unsigned fftw_plan_rigor;

    field(const int nx, const int ny, const int nz, const MPI_Comm COMM_TO_USE,
          const unsigned FFTW_PLAN_RIGOR = DEFAULT_FFTW_FLAG)
        : nx_(nx), ny_(ny), nz_(nz), myrank(0), nprocs(1), comm(COMM_TO_USE),
          fftw_plan_rigor(FFTW_PLAN_RIGOR) {
        // field.cpp:85-104 with one process holding every slab
        hsize_t sizes[3], starts[3] = {0, 0, 0};
        sizes[0] = nz; sizes[1] = ny; sizes[2] = nx;
        rlayout = new field_layout<fc>(sizes, sizes, starts, comm);
        npoints = rlayout->full_size / ncomp(fc);
        sizes[0] = nz; sizes[1] = ny; sizes[2] = nx + 2;
        rmemlayout = new field_layout<fc>(sizes, sizes, starts, comm);
        sizes[0] = ny; sizes[1] = nz; sizes[2] = nx / 2 + 1;
        clayout = new field_layout<fc>(sizes, sizes, starts, comm);
        data_.assign(rmemlayout->local_size, (rnumber)0);
        real_space_representation = true;
    }
    ~field() {
        delete clayout;
        delete rlayout;
        delete rmemlayout;
    }
    field(const field&) = delete;
    field& operator=(const field&) = delete;

    /* essential FFT stuff (field.cpp:144-175) */
    void dft() {
        require3("dft");
        host_sync();
        bfg_ctx* c = bfps_b200_compat::shared_ctx(nx_, ny_, nz_, (int)sizeof(rnumber));
        bfps_b200_compat::check(bfg_dft(c, data_.data(), data_.data()), c, "field::dft");
        real_space_representation = false;
        where_ = bfps_b200_compat::ON_HOST;
    }
    void ift() {
        require3("ift");
        if (link_id_ == BFG_FIELD_VELOCITY && !real_space_representation &&
            where_ != bfps_b200_compat::ON_HOST) {
            // the solver's velocity: transformed where it lives
            bfps_b200_compat::check(bfg_field_ift(link_ctx_, BFG_FIELD_VELOCITY), link_ctx_,
                                    "field::ift");
            real_space_representation = true;
            where_ = bfps_b200_compat::ON_DEVICE;
            return;
        }
        host_sync();
        bfg_ctx* c = bfps_b200_compat::shared_ctx(nx_, ny_, nz_, (int)sizeof(rnumber));
        bfps_b200_compat::check(bfg_ift(c, data_.data(), data_.data()), c, "field::ift");
        real_space_representation = true;
        where_ = bfps_b200_compat::ON_HOST;
    }
    void normalize() {
        host_sync();
        const double inv = 1.0 / (double)npoints;
        for (auto& v : data_) v = (rnumber)(v * inv);
        where_ = bfps_b200_compat::ON_HOST;
    }
    /* field.cpp:903-978 on the kx = 0 plane */
    void symmetrize() {
        host_sync();
        const hsize_t nc = ncomp(fc);
        const hsize_t s1 = clayout->sizes[1], s0 = clayout->sizes[0], s2 = clayout->sizes[2];
        rnumber* d = data_.data();
        auto at = [&](hsize_t y, hsize_t z, hsize_t c, int im) -> rnumber& {
            return d[(((y * s1 + z) * s2) * nc + c) * 2 + im];
        };
        for (hsize_t c = 0; c < nc; ++c) at(0, 0, c, 1) = 0;
        for (hsize_t ii = 1; ii < s1 / 2; ++ii)
            for (hsize_t c = 0; c < nc; ++c) {
                at(0, s1 - ii, c, 0) = at(0, ii, c, 0);
                at(0, s1 - ii, c, 1) = -at(0, ii, c, 1);
            }
        std::vector<rnumber> buf(s1 * nc * 2);
        for (hsize_t yy = 1; yy < s0 / 2; ++yy) {
            for (hsize_t z = 0; z < s1; ++z)
                for (hsize_t c = 0; c < nc; ++c) {
                    buf[(z * nc + c) * 2] = at(yy, z, c, 0);
                    buf[(z * nc + c) * 2 + 1] = at(yy, z, c, 1);
                }
            for (hsize_t ii = 1; ii < s1; ++ii)
                for (hsize_t c = 0; c < nc; ++c) {
                    at(s0 - yy, ii, c, 0) = buf[((s1 - ii) * nc + c) * 2];
                    at(s0 - yy, ii, c, 1) = -buf[((s1 - ii) * nc + c) * 2 + 1];
                }
            for (hsize_t c = 0; c < nc; ++c) {
                at(s0 - yy, 0, c, 0) = buf[c * 2];
                at(s0 - yy, 0, c, 1) = -buf[c * 2 + 1];
            }
        }
        where_ = bfps_b200_compat::ON_HOST;
    }

    /* access data: a non-const access makes the host copy the current one */
    rnumber* __restrict__ get_rdata() {
        host_sync();
        where_ = bfps_b200_compat::ON_HOST;
        return data_.data();
    }
    const rnumber* __restrict__ get_rdata() const {
        host_sync();
        return data_.data();
    }
    typename fftw_interface<rnumber>::complex* __restrict__ get_cdata() {
        return (typename fftw_interface<rnumber>::complex*)get_rdata();
    }
    const typename fftw_interface<rnumber>::complex* __restrict__ get_cdata() const {
        return (const typename fftw_interface<rnumber>::complex*)get_rdata();
    }
    rnumber& rval(ptrdiff_t rindex, unsigned int component = 0) {
        return get_rdata()[rindex * ncomp(fc) + component];
    }
    const rnumber& rval(ptrdiff_t rindex, unsigned int component = 0) const {
        return get_rdata()[rindex * ncomp(fc) + component];
    }
    rnumber& rval(ptrdiff_t rindex, int comp1, int comp0) {
        return get_rdata()[(rindex * 3 + comp1) * 3 + comp0];
    }
    rnumber& cval(ptrdiff_t cindex, int imag) { return get_rdata()[cindex * 2 + imag]; }
    rnumber& cval(ptrdiff_t cindex, int component, int imag) {
        return get_rdata()[(cindex * ncomp(fc) + component) * 2 + imag];
    }
    const rnumber& cval(ptrdiff_t cindex, int component, int imag) const {
        return get_rdata()[(cindex * ncomp(fc) + component) * 2 + imag];
    }
    rnumber& cval(ptrdiff_t cindex, int comp1, int comp0, int imag) {
        return get_rdata()[((cindex * 3 + comp1) * 3 + comp0) * 2 + imag];
    }

    field& operator=(const typename fftw_interface<rnumber>::complex* __restrict__ source) {
        std::memcpy(get_rdata(), source, sizeof(rnumber) * 2 * clayout->local_size);
        real_space_representation = false;
        return *this;
    }
    field& operator=(const rnumber* __restrict__ source) {
        std::memcpy(get_rdata(), source, sizeof(rnumber) * rmemlayout->local_size);
        real_space_representation = true;
        return *this;
    }
    field& operator=(const rnumber value) {
        rnumber* d = get_rdata();
        std::fill(d, d + rmemlayout->local_size, value);
        return *this;
    }

    /* field::compute_stats (field.cpp:984-1040) of a 3-component complex
     * field, computed on the GPU: co-spectrum (nshells, 3, 3), moments
     * (10, 4), histograms (nbins, 4); the arrays the reference writes to its
     * statistics group */
    template <kspace_dealias_type dt>
    void compute_stats(kspace<be, dt>* kk, std::vector<double>& spectrum,
                       std::vector<double>& moments, std::vector<int64_t>& histograms,
                       const double max_estimate, const int nbins = 256) {
        require3("compute_stats");
        if (real_space_representation)
            throw std::runtime_error("field::compute_stats needs the Fourier representation");
        host_sync();
        bfg_ctx* c = link_ctx_ ? link_ctx_
                               : bfps_b200_compat::shared_ctx(nx_, ny_, nz_, (int)sizeof(rnumber),
                                                              kk->dkx, kk->dky, kk->dkz,
                                                              dt == SMOOTH ? BFG_SMOOTH
                                                                           : BFG_TWO_THIRDS);
        spectrum.assign((size_t)kk->nshells * 9, 0.0);
        moments.assign(40, 0.0);
        histograms.assign((size_t)nbins * 4, 0);
        bfps_b200_compat::check(bfg_field_stats(c, data_.data(), max_estimate, nbins,
                                                spectrum.data(), moments.data(), histograms.data()),
                                c, "field::compute_stats");
    }

    inline void impose_zero_mode() {
        if (!real_space_representation) {
            rnumber* d = get_rdata();
            std::fill_n(d, 2 * ncomp(fc), (rnumber)0);
        }
    }
    template <class func_type>
    void RLOOP(func_type expression) {
        for (hsize_t zindex = 0; zindex < rlayout->subsizes[0]; zindex++)
            for (hsize_t yindex = 0; yindex < rlayout->subsizes[1]; yindex++) {
                ptrdiff_t rindex = (zindex * rlayout->subsizes[1] + yindex) * rmemlayout->subsizes[2];
                for (hsize_t xindex = 0; xindex < rlayout->subsizes[2]; xindex++)
                    expression(rindex++, xindex, yindex, zindex);
            }
    }
    ptrdiff_t get_cindex(ptrdiff_t xindex, ptrdiff_t yindex, ptrdiff_t zindex) {
        return ((yindex * clayout->subsizes[1] + zindex) * clayout->subsizes[2] + xindex);
    }
    ptrdiff_t get_rindex(ptrdiff_t xindex, ptrdiff_t yindex, ptrdiff_t zindex) const {
        return ((zindex * rmemlayout->subsizes[1] + yindex) * rmemlayout->subsizes[2] + xindex);
    }
    ptrdiff_t get_rindex_from_global(const ptrdiff_t x, const ptrdiff_t y, const ptrdiff_t z) const {
        return get_rindex(x, y, z);
    }

    /* ---- device link (used by vorticity_equation and the particle system) */
    void bfg_link(bfg_ctx* ctx, int field_id) {
        link_ctx_ = ctx;
        link_id_ = field_id;
    }
    bfg_ctx* bfg_linked_ctx() const { return link_ctx_; }
    int bfg_linked_id() const { return link_id_; }
    /* the device copy became the current one (a solver method wrote it) */
    void bfg_mark_device(bool real_rep) {
        real_space_representation = real_rep;
        where_ = bfps_b200_compat::ON_DEVICE;
    }
    /* upload the host copy if it is the current one */
    void bfg_device_sync() {
        if (!link_ctx_ || where_ != bfps_b200_compat::ON_HOST) return;
        const int id = (link_id_ == BFG_FIELD_VELOCITY && real_space_representation)
                           ? BFG_FIELD_RVELOCITY
                           : link_id_;
        bfps_b200_compat::check(bfg_field_upload(link_ctx_, id, data_.data()), link_ctx_,
                                "field upload");
        where_ = bfps_b200_compat::ON_BOTH;
    }
    /* download the device copy if it is the current one */
    void host_sync() const {
        if (!link_ctx_ || where_ != bfps_b200_compat::ON_DEVICE) return;
        const int id = (link_id_ == BFG_FIELD_VELOCITY && real_space_representation)
                           ? BFG_FIELD_RVELOCITY
                           : link_id_;
        bfps_b200_compat::check(bfg_field_download(link_ctx_, id, data_.data()), link_ctx_,
                                "field download");
        where_ = bfps_b200_compat::ON_BOTH;
    }

  private:
    void require3(const char* what) const {
        if (fc != THREE)
            throw std::runtime_error(std::string("field::") + what +
                                     ": the device engine transforms 3-component fields");
    }
};

#endif
