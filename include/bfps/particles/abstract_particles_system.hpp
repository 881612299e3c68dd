/*
 * abstract_particles_system.hpp -- drop-in replacement for
 * bfps/cpp/particles/abstract_particles_system.hpp (bfps_b200): the same
 * pure interface (abstract_particles_system.hpp:12-55).
 */
#ifndef BFPS_B200_ABSTRACT_PARTICLES_SYSTEM_HPP
#define BFPS_B200_ABSTRACT_PARTICLES_SYSTEM_HPP

#include <memory>

#include "../field.hpp"

template <class partsize_t, class real_number>
class abstract_particles_system {
  public:
    virtual ~abstract_particles_system() {}
    virtual void compute() = 0;
    virtual void move(const real_number dt) = 0;
    virtual void redistribute() = 0;
    virtual void inc_step_idx() = 0;
    virtual void shift_rhs_vectors() = 0;
    virtual void completeLoop(const real_number dt) = 0;
    virtual const real_number* getParticlesPositions() const = 0;
    virtual const std::unique_ptr<real_number[]>* getParticlesRhs() const = 0;
    virtual const partsize_t* getParticlesIndexes() const = 0;
    virtual partsize_t getLocalNbParticles() const = 0;
    virtual partsize_t getGlobalNbParticles() const = 0;
    virtual int getNbRhs() const = 0;
    virtual int get_step_idx() const = 0;
    virtual void sample_compute_field(const field<float, FFTW, ONE>& sample_field,
                                      real_number sample_rhs[]) = 0;
    virtual void sample_compute_field(const field<float, FFTW, THREE>& sample_field,
                                      real_number sample_rhs[]) = 0;
    virtual void sample_compute_field(const field<float, FFTW, THREExTHREE>& sample_field,
                                      real_number sample_rhs[]) = 0;
    virtual void sample_compute_field(const field<double, FFTW, ONE>& sample_field,
                                      real_number sample_rhs[]) = 0;
    virtual void sample_compute_field(const field<double, FFTW, THREE>& sample_field,
                                      real_number sample_rhs[]) = 0;
    virtual void sample_compute_field(const field<double, FFTW, THREExTHREE>& sample_field,
                                      real_number sample_rhs[]) = 0;
};

#endif
