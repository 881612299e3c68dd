/*
 * vorticity_equation.hpp -- drop-in replacement for
 * bfps/cpp/vorticity_equation.hpp (bfps_b200).
 *
 * vorticity_equation<rnumber, be> with the reference's constructor
 * (NAME, nx, ny, nz, DKX, DKY, DKZ, FFTW_PLAN_RIGOR) and public members
 * (vorticity_equation.hpp:46-134): name, iteration, checkpoint,
 * checkpoints_per_file, cvorticity, cvelocity, kk, u, v[4], nu, fmode,
 * famplitude, fk0, fk1, forcing_type.  The solver runs on the GPU through
 * include/bfps_b200.h: cvorticity and cvelocity are backed by the
 * context's device buffers (see field.hpp for the host / device coherence);
 * step, compute_velocity and the particle loop never leave the device.
 * The physical members are read at every solver call, as in the reference.
 *
 * The RK fields v[1], v[2] and rvorticity live only inside the device
 * step and are null here; v[0] = v[3] = cvorticity, u = cvelocity.  The
 * FFTW plan rigor is accepted and unused (the transforms are this
 * library's own).  Checkpoint files: this header carries no HDF5 code (the
 * Python launcher bfps_b200.dns reads and writes bfps' files); a C++ caller
 * reads vorticity/complex/<iteration> into cvorticity->get_cdata() with its
 * own HDF5 calls and then calls io_checkpoint_read_host(), the read-time
 * steps of io_checkpoint.
 */
#ifndef BFPS_B200_VORTICITY_EQUATION_HPP
#define BFPS_B200_VORTICITY_EQUATION_HPP

#include <cassert>
#include <cstring>
#include <string>

#include "field.hpp"
#include "kspace.hpp"

template <typename rnumber, field_backend be>
class vorticity_equation {
  public:
    char name[256];
    int iteration;
    int checkpoint;
    int checkpoints_per_file;

    field<rnumber, be, THREE>*cvorticity, *cvelocity;
    field<rnumber, be, THREE>* rvorticity;
    kspace<be, SMOOTH>* kk;
    field<rnumber, be, THREE>*u, *v[4];

    double nu;
    int fmode;
    double famplitude;
    double fk0, fk1;
    char forcing_type[128];

    vorticity_equation(const char* NAME, int nx, int ny, int nz, double DKX = 1.0,
                       double DKY = 1.0, double DKZ = 1.0,
                       unsigned FFTW_PLAN_RIGOR = FFTW_MEASURE) {
        std::strncpy(name, NAME ? NAME : "", sizeof(name) - 1);
        name[sizeof(name) - 1] = 0;
        bfps_b200_compat::check(bfg_ctx_create(&ctx_, nx, ny, nz, DKX, DKY, DKZ,
                                               (int)sizeof(rnumber), BFG_SMOOTH, 0),
                                nullptr, "vorticity_equation");
        cvorticity = new field<rnumber, be, THREE>(nx, ny, nz, MPI_COMM_WORLD, FFTW_PLAN_RIGOR);
        cvelocity = new field<rnumber, be, THREE>(nx, ny, nz, MPI_COMM_WORLD, FFTW_PLAN_RIGOR);
        cvorticity->bfg_link(ctx_, BFG_FIELD_VORTICITY);
        cvelocity->bfg_link(ctx_, BFG_FIELD_VELOCITY);
        cvorticity->real_space_representation = false;
        cvelocity->real_space_representation = false;
        rvorticity = nullptr;
        u = cvelocity;
        v[0] = cvorticity;
        v[1] = nullptr;
        v[2] = nullptr;
        v[3] = cvorticity;
        kk = new kspace<be, SMOOTH>(cvorticity->clayout, DKX, DKY, DKZ);
        // defaults of the reference constructor (vorticity_equation.cpp:150-155)
        iteration = 0;
        checkpoint = 0;
        checkpoints_per_file = 1;
        nu = 0.1;
        fmode = 1;
        famplitude = 1.0;
        fk0 = 2.0;
        fk1 = 4.0;
        std::strncpy(forcing_type, "none", sizeof(forcing_type));
    }
    ~vorticity_equation() {
        delete kk;
        delete cvorticity;
        delete cvelocity;
        bfg_ctx_destroy(ctx_);
    }
    vorticity_equation(const vorticity_equation&) = delete;
    vorticity_equation& operator=(const vorticity_equation&) = delete;

    bfg_ctx* handle() const { return ctx_; }

    /* vorticity_equation::step (vorticity_equation.cpp:358-439) */
    void step(double dt) {
        cvorticity->bfg_device_sync();
        push();
        bfps_b200_compat::check(bfg_step(ctx_, dt, 1), ctx_, "vorticity_equation::step");
        bfps_b200_compat::check(bfg_get_iteration(ctx_, &iteration), ctx_, "step");
        cvorticity->bfg_mark_device(false);
        cvelocity->bfg_mark_device(false);  // the step uses it as scratch, as the reference does
    }
    /* compute_velocity (vorticity_equation.cpp:206-239) of the state */
    void compute_velocity(field<rnumber, be, THREE>* vorticity) {
        if (vorticity != cvorticity)
            throw std::runtime_error(
                "vorticity_equation::compute_velocity: the device solver takes cvorticity");
        cvorticity->bfg_device_sync();
        push();
        bfps_b200_compat::check(bfg_compute_velocity(ctx_), ctx_, "compute_velocity");
        cvelocity->bfg_mark_device(false);
    }
    /* impose_zero_modes (vorticity_equation.cpp:110-120): the zero mode of
     * the state and of the velocity */
    void impose_zero_modes() {
        cvorticity->impose_zero_mode();
        cvelocity->impose_zero_mode();
    }
    /* compute_pressure (vorticity_equation.cpp:441-514) of the state's
     * velocity into a 1-component field (Fourier representation) */
    void compute_pressure(field<rnumber, be, ONE>* pressure) {
        cvorticity->bfg_device_sync();
        push();
        bfps_b200_compat::check(bfg_compute_pressure(ctx_, pressure->get_cdata()), ctx_,
                                "compute_pressure");
        pressure->real_space_representation = false;
        cvelocity->bfg_mark_device(true);  // left in real space by the pressure solve
    }
    /* compute_Lagrangian_acceleration (vorticity_equation.cpp:516-578) */
    void compute_Lagrangian_acceleration(field<rnumber, be, THREE>* acceleration) {
        cvorticity->bfg_device_sync();
        push();
        bfps_b200_compat::check(bfg_lagrangian_acceleration(ctx_, acceleration->get_cdata()), ctx_,
                                "compute_Lagrangian_acceleration");
        acceleration->real_space_representation = false;
        cvelocity->bfg_mark_device(false);
    }

    /* I/O (vorticity_equation.hpp:99-128) */
    inline std::string get_current_fname() {
        return std::string(name) + std::string("_checkpoint_") + std::to_string(checkpoint) +
               std::string(".h5");
    }
    /* the read-time steps of io_checkpoint after field::io has filled the
     * host copy: symmetrize (field.cpp:340), low_pass(kM), force_divfree */
    void io_checkpoint_read_host() {
        cvorticity->real_space_representation = false;
        cvorticity->symmetrize();
        kk->template low_pass<rnumber, THREE>(cvorticity->get_cdata(), kk->kM);
        kk->template force_divfree<rnumber>(cvorticity->get_cdata());
    }

  private:
    bfg_ctx* ctx_ = nullptr;
    void push() {
        const int f = std::strcmp(forcing_type, "linear") == 0       ? BFG_FORCING_LINEAR
                      : std::strcmp(forcing_type, "Kolmogorov") == 0 ? BFG_FORCING_KOLMOGOROV
                                                                     : BFG_FORCING_NONE;
        bfps_b200_compat::check(bfg_set_physics(ctx_, nu, f, famplitude, fk0, fk1, fmode), ctx_,
                                "set_physics");
        bfps_b200_compat::check(bfg_set_iteration(ctx_, iteration), ctx_, "set_iteration");
    }
};

#endif
