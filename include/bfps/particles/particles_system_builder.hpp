/*
 * particles_system_builder.hpp -- drop-in replacement for
 * bfps/cpp/particles/particles_system_builder.hpp (bfps_b200).
 *
 * particles_system_builder(...) with the reference's template parameters
 * and runtime (interpolation size, spline mode) dispatch
 * (particles_system_builder.hpp:238-257) returns an
 * abstract_particles_system whose tracers live on the GPU, in the context
 * of the solver that owns the velocity field passed in: completeLoop
 * samples that context's real velocity (cvelocity after ift(), as
 * NSVEparticles::step leaves it) and advances the tracers with
 * Adams-Bashforth, all on the device (bfg_particles_*).  The reference
 * reads the initial state from an HDF5 file; this builder takes the state
 * (nparticles, 3) and rhs history (nsteps, nparticles, 3) arrays the caller
 * read (NULL rhs: zeros), with the same coherency checks.  Host getters
 * download the state on demand.  compute / move / redistribute /
 * inc_step_idx / shift_rhs_vectors exist only as the fused completeLoop on
 * the device and report an error when called alone; sample_compute_field
 * samples the velocity field the system was built on.
 */
#ifndef BFPS_B200_PARTICLES_SYSTEM_BUILDER_HPP
#define BFPS_B200_PARTICLES_SYSTEM_BUILDER_HPP

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../field.hpp"
#include "../kspace.hpp"
#include "abstract_particles_system.hpp"

namespace bfps_b200_compat {

template <class partsize_t, class real_number, class field_rnumber>
class device_particles_system : public abstract_particles_system<partsize_t, real_number> {
    static_assert(sizeof(real_number) == 8, "tracer state is double precision");

  public:
    device_particles_system(field<field_rnumber, FFTW, THREE>* velocity, int nsteps,
                            partsize_t nparticles, const double* state, const double* rhs,
                            int interpolation_size, int spline_mode, int current_iteration)
        : vel_(velocity), ctx_(velocity->bfg_linked_ctx()), n_(nparticles), nrhs_(nsteps) {
        if (!ctx_ || velocity->bfg_linked_id() != BFG_FIELD_VELOCITY)
            throw std::runtime_error("particles_system_builder: the field must be a solver's cvelocity");
        check(bfg_particles_create(ctx_, &p_, (int64_t)nparticles, interpolation_size, spline_mode,
                                   nsteps, state, rhs, nullptr, current_iteration),
              ctx_, "particles_system_builder");
    }
    ~device_particles_system() override { bfg_particles_destroy(p_); }

    void completeLoop(const real_number dt) override {
        vel_->bfg_device_sync();
        check(bfg_particles_complete_loop(p_, dt), ctx_, "completeLoop");
        stale_ = true;
    }
    void compute() override { alone("compute"); }
    void move(const real_number) override { alone("move"); }
    void redistribute() override { alone("redistribute"); }
    void inc_step_idx() override { alone("inc_step_idx"); }
    void shift_rhs_vectors() override { alone("shift_rhs_vectors"); }

    const real_number* getParticlesPositions() const override {
        fetch();
        return pos_.data();
    }
    const std::unique_ptr<real_number[]>* getParticlesRhs() const override {
        fetch();
        return rhs_.data();
    }
    const partsize_t* getParticlesIndexes() const override {
        fetch();
        return idx_.data();
    }
    partsize_t getLocalNbParticles() const override { return n_; }
    partsize_t getGlobalNbParticles() const override { return n_; }
    int getNbRhs() const override { return nrhs_; }
    int get_step_idx() const override {
        int s = 0;
        check(bfg_particles_info(p_, nullptr, nullptr, &s), ctx_, "get_step_idx");
        return s;
    }

    void sample_compute_field(const field<float, FFTW, ONE>&, real_number[]) override {
        unsupported();
    }
    void sample_compute_field(const field<float, FFTW, THREE>& f, real_number out[]) override {
        sample(static_cast<const void*>(&f), out);
    }
    void sample_compute_field(const field<float, FFTW, THREExTHREE>&, real_number[]) override {
        unsupported();
    }
    void sample_compute_field(const field<double, FFTW, ONE>&, real_number[]) override {
        unsupported();
    }
    void sample_compute_field(const field<double, FFTW, THREE>& f, real_number out[]) override {
        sample(static_cast<const void*>(&f), out);
    }
    void sample_compute_field(const field<double, FFTW, THREExTHREE>&, real_number[]) override {
        unsupported();
    }

  private:
    field<field_rnumber, FFTW, THREE>* vel_;
    bfg_ctx* ctx_;
    bfg_pctx* p_ = nullptr;
    partsize_t n_;
    int nrhs_;
    mutable bool stale_ = true;
    mutable std::vector<real_number> pos_;
    mutable std::vector<std::unique_ptr<real_number[]>> rhs_;
    mutable std::vector<partsize_t> idx_;

    void fetch() const {
        if (!stale_) return;
        pos_.resize((size_t)n_ * 3);
        std::vector<double> rhs((size_t)nrhs_ * n_ * 3);
        std::vector<int64_t> idx((size_t)n_);
        check(bfg_particles_download(p_, pos_.data(), rhs.data(), idx.data()), ctx_,
              "particles download");
        rhs_.clear();
        for (int s = 0; s < nrhs_; ++s) {
            rhs_.emplace_back(new real_number[(size_t)n_ * 3]);
            std::copy(rhs.begin() + (size_t)s * n_ * 3, rhs.begin() + (size_t)(s + 1) * n_ * 3,
                      rhs_.back().get());
        }
        idx_.assign(idx.begin(), idx.end());
        stale_ = false;
    }
    void sample(const void* f, real_number out[]) {
        if (f != static_cast<const void*>(vel_) || !vel_->real_space_representation)
            throw std::runtime_error(
                "sample_compute_field: the velocity field the system was built on, in real space");
        vel_->bfg_device_sync();
        check(bfg_particles_sample_velocity(p_, out), ctx_, "sample_compute_field");
    }
    [[noreturn]] static void alone(const char* what) {
        throw std::runtime_error(std::string(what) +
                                 ": runs only inside completeLoop on the device");
    }
    [[noreturn]] static void unsupported() {
        throw std::runtime_error("sample_compute_field: 3-component fields only");
    }
};

}  // namespace bfps_b200_compat

template <class partsize_t, class field_rnumber, field_backend be, field_components fc,
          class particles_rnumber = double>
inline std::unique_ptr<abstract_particles_system<partsize_t, particles_rnumber>>
particles_system_builder(const field<field_rnumber, be, fc>* fs_field,
                         const kspace<be, SMOOTH>* fs_kk, const int nsteps,
                         const partsize_t nparticles, const double* state, const double* rhs,
                         const int interpolation_size, const int spline_mode, MPI_Comm mpi_comm,
                         const int in_current_iteration) {
    static_assert(fc == THREE, "tracers sample a 3-component velocity");
    (void)fs_kk;  // the box (2 pi / dk) and spacing come from the solver's context
    (void)mpi_comm;
    return std::unique_ptr<abstract_particles_system<partsize_t, particles_rnumber>>(
        new bfps_b200_compat::device_particles_system<partsize_t, particles_rnumber, field_rnumber>(
            const_cast<field<field_rnumber, be, fc>*>(fs_field), nsteps, nparticles, state, rhs,
            interpolation_size, spline_mode, in_current_iteration));
}

#endif
