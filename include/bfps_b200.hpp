/*
 * bfps_b200.hpp — C++ host mirror of bfps' building blocks over the C-ABI
 * (bfps_b200.h), header only.
 *
 *   bfps_b200::vorticity_equation<rnumber>   vorticity_equation<rnumber, FFTW>
 *                                            (bfps/cpp/vorticity_equation.hpp:46-134)
 *   bfps_b200::particles_system              abstract_particles_system<long long, double>
 *                                            (bfps/cpp/particles/abstract_particles_system.hpp:12-55)
 *   bfps_b200::NSVEparticles_step            NSVEparticles::step
 *                                            (bfps/cpp/full_code/NSVEparticles.cpp:33-41)
 *   bfps_b200::ensemble                      batched form over bfg_ens_* (no
 *                                            counterpart in the reference)
 *
 * The public physical members (nu, fmode, famplitude, fk0, fk1,
 * forcing_type) are plain data as in the reference and are read whenever a
 * method needs them; iteration follows the device state.  Fields stay on
 * the GPU; host access goes through get_/set_ methods in the reference's
 * host layouts.  Failures throw bfps_b200::error (std::runtime_error), the
 * exception the reference's particle code throws (particles_utils.hpp:18-20).
 */
#ifndef BFPS_B200_HPP
#define BFPS_B200_HPP

#include <algorithm>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "bfps_b200.h"

namespace bfps_b200 {

class error : public std::runtime_error {
  public:
    error(const std::string& what, int code) : std::runtime_error(what), code(code) {}
    int code;
};

inline void check(int rc, const bfg_ctx* ctx, const char* what) {
    if (rc != BFG_OK)
        throw error(std::string(what) + ": " + (ctx ? bfg_last_error(ctx) : "") + " (code " +
                        std::to_string(rc) + ")",
                    rc);
}

template <typename rnumber>
class vorticity_equation {
    static_assert(sizeof(rnumber) == 4 || sizeof(rnumber) == 8, "float or double");

  public:
    using cnumber = std::complex<rnumber>;

    char name[256];
    int iteration = 0;
    /* physical parameters, defaults of the reference constructor
     * (vorticity_equation.cpp:150-155) */
    double nu = 0.1;
    int fmode = 1;
    double famplitude = 1.0;
    double fk0 = 2.0, fk1 = 4.0;
    char forcing_type[128] = "none";

    const int nx, ny, nz;

    vorticity_equation(const char* NAME, int nx_, int ny_, int nz_, double DKX = 1.0,
                       double DKY = 1.0, double DKZ = 1.0, int dealias = BFG_SMOOTH,
                       int device = 0)
        : nx(nx_), ny(ny_), nz(nz_) {
        std::strncpy(name, NAME ? NAME : "", sizeof(name) - 1);
        name[sizeof(name) - 1] = 0;
        check(bfg_ctx_create(&ctx, nx, ny, nz, DKX, DKY, DKZ, (int)sizeof(rnumber), dealias,
                             device),
              nullptr, "bfg_ctx_create");
    }
    ~vorticity_equation() { bfg_ctx_destroy(ctx); }
    vorticity_equation(const vorticity_equation&) = delete;
    vorticity_equation& operator=(const vorticity_equation&) = delete;

    bfg_ctx* handle() const { return ctx; }

    /* sizes of the host layouts (elements) */
    size_t complex_size() const { return (size_t)ny * nz * (nx / 2 + 1) * 3; }
    size_t real_size() const { return (size_t)nz * ny * (nx + 2) * 3; }

    /* vorticity_equation::step (vorticity_equation.cpp:358-439) */
    void step(double dt) {
        push_physics();
        check(bfg_step(ctx, dt, 1), ctx, "step");
        pull_iteration();
    }
    /* compute_velocity(cvorticity) (vorticity_equation.cpp:206-239) */
    void compute_velocity() {
        push_physics();
        check(bfg_compute_velocity(ctx), ctx, "compute_velocity");
    }
    /* compute_velocity + cvelocity->ift() (NSVEparticles.cpp:35-36) */
    void compute_velocity_rspace() {
        push_physics();
        check(bfg_velocity_rspace(ctx), ctx, "compute_velocity_rspace");
    }
    /* compute_pressure (vorticity_equation.cpp:441-514): (ny, nz, nx/2+1) */
    void compute_pressure(cnumber* pressure) {
        push_physics();
        check(bfg_compute_pressure(ctx, pressure), ctx, "compute_pressure");
    }
    /* compute_Lagrangian_acceleration (vorticity_equation.cpp:516-578) */
    void compute_Lagrangian_acceleration(cnumber* acceleration) {
        push_physics();
        check(bfg_lagrangian_acceleration(ctx, acceleration), ctx,
              "compute_Lagrangian_acceleration");
    }

    /* the state (cvorticity) and derived fields in the host layouts */
    void set_cvorticity(const cnumber* host) {
        check(bfg_field_upload(ctx, BFG_FIELD_VORTICITY, host), ctx, "set_cvorticity");
    }
    void get_cvorticity(cnumber* host) const {
        check(bfg_field_download(ctx, BFG_FIELD_VORTICITY, host), ctx, "get_cvorticity");
    }
    void get_cvelocity(cnumber* host) const {
        check(bfg_field_download(ctx, BFG_FIELD_VELOCITY, host), ctx, "get_cvelocity");
    }
    void get_rvelocity(rnumber* host) const {
        check(bfg_field_download(ctx, BFG_FIELD_RVELOCITY, host), ctx, "get_rvelocity");
    }
    /* io_checkpoint(read = true) after field::io has filled host
     * (vorticity_equation.hpp:107-128): symmetrize, low_pass, force_divfree */
    void io_checkpoint_read(const cnumber* host, int it) {
        set_cvorticity(host);
        check(bfg_read_checkpoint_fixup(ctx), ctx, "io_checkpoint_read");
        iteration = it;
        check(bfg_set_iteration(ctx, it), ctx, "io_checkpoint_read");
    }

    void push_physics() {
        const int f = std::strcmp(forcing_type, "linear") == 0       ? BFG_FORCING_LINEAR
                      : std::strcmp(forcing_type, "Kolmogorov") == 0 ? BFG_FORCING_KOLMOGOROV
                                                                     : BFG_FORCING_NONE;
        check(bfg_set_physics(ctx, nu, f, famplitude, fk0, fk1, fmode), ctx, "set_physics");
        check(bfg_set_iteration(ctx, iteration), ctx, "set_iteration");
    }
    void pull_iteration() { check(bfg_get_iteration(ctx, &iteration), ctx, "get_iteration"); }

  private:
    bfg_ctx* ctx = nullptr;
};

/* particles_system_builder + particles_system (particles_system_builder.hpp:
 * 238-257): tracers of one vorticity_equation, state in global index order */
class particles_system {
  public:
    template <typename rnumber>
    particles_system(vorticity_equation<rnumber>& fs, long long nparticles, int neighbours,
                     int smoothness, int nsteps, const double* state, const double* rhs,
                     const long long* indexes, int step_idx)
        : ctx(fs.handle()), n(nparticles), nrhs(nsteps) {
        static_assert(sizeof(long long) == sizeof(int64_t), "index type");
        check(bfg_particles_create(ctx, &p, nparticles, neighbours, smoothness, nsteps, state,
                                   rhs, reinterpret_cast<const int64_t*>(indexes), step_idx),
              ctx, "particles_system");
    }
    ~particles_system() { bfg_particles_destroy(p); }
    particles_system(const particles_system&) = delete;
    particles_system& operator=(const particles_system&) = delete;

    bfg_pctx* handle() const { return p; }

    /* completeLoop (particles_system.hpp:210-217) on the context's current
     * real velocity */
    void completeLoop(double dt) {
        check(bfg_particles_complete_loop(p, dt), ctx, "completeLoop");
    }
    long long getLocalNbParticles() const { return n; }
    long long getGlobalNbParticles() const { return n; }
    int getNbRhs() const { return nrhs; }
    int get_step_idx() const {
        int s = 0;
        check(bfg_particles_info(p, nullptr, nullptr, &s), ctx, "get_step_idx");
        return s;
    }
    /* positions (n, 3), rhs history (nsteps, n, 3) and indexes (n), each may
     * be null, in global index order */
    void get_state(double* positions, double* rhs, long long* indexes) const {
        check(bfg_particles_download(p, positions, rhs, reinterpret_cast<int64_t*>(indexes)),
              ctx, "get_state");
    }
    /* sample_compute_field of the velocity (after compute_velocity_rspace)
     * and of the Lagrangian acceleration (NSVEparticles.cpp:70-98), (n, 3) */
    void sample_velocity(double* out) {
        check(bfg_particles_sample_velocity(p, out), ctx, "sample_velocity");
    }
    void sample_acceleration(double* out) {
        check(bfg_particles_sample_acceleration(p, out), ctx, "sample_acceleration");
    }

  private:
    bfg_ctx* ctx;
    bfg_pctx* p = nullptr;
    long long n;
    int nrhs;
};

/* NSVEparticles::step (NSVEparticles.cpp:33-41): velocity of the current
 * state, tracers advanced on it, then the fluid step; iteration += 1 */
template <typename rnumber>
inline void NSVEparticles_step(vorticity_equation<rnumber>& fs, particles_system& ps, double dt) {
    fs.push_physics();
    check(bfg_nsveparticles_step(fs.handle(), ps.handle(), dt, 1), fs.handle(),
          "NSVEparticles_step");
    fs.pull_iteration();
}

/* Members of any sizes advanced together, one launch per pass and RK stage
 * for each grid size; a member keeps its state and API but is stepped only
 * through the ensemble while it belongs to it. */
class ensemble {
  public:
    explicit ensemble(int device = 0) {
        if (bfg_ens_create(&e, device) != BFG_OK) throw error("bfg_ens_create", BFG_ECUDA);
    }
    ~ensemble() { bfg_ens_destroy(e); }
    ensemble(const ensemble&) = delete;
    ensemble& operator=(const ensemble&) = delete;

    template <typename rnumber>
    void add(vorticity_equation<rnumber>& fs, double dt, particles_system* ps = nullptr) {
        fs.push_physics();
        chk(bfg_ens_add(e, fs.handle(), ps ? ps->handle() : nullptr, dt), "ensemble::add");
        members.emplace_back(fs.handle(), [&fs] { fs.pull_iteration(); });
    }
    template <typename rnumber>
    void remove(vorticity_equation<rnumber>& fs) {
        chk(bfg_ens_remove(e, fs.handle()), "ensemble::remove");
        members.erase(std::remove_if(members.begin(), members.end(),
                                     [&fs](const auto& m) { return m.first == fs.handle(); }),
                      members.end());
    }
    /* nsteps NSVEparticles steps of every member (enqueued; the members'
     * iteration counters advance at once) */
    void step(int nsteps) {
        chk(bfg_ens_step(e, nsteps), "ensemble::step");
        for (auto& m : members) m.second();
    }
    /* true once the last step() has finished, false if still running after
     * timeout_ms */
    bool wait(double timeout_ms) {
        int done = 0;
        chk(bfg_ens_wait(e, timeout_ms, &done), "ensemble::wait");
        return done != 0;
    }
    double last_ms() {
        double ms = 0;
        chk(bfg_ens_last_ms(e, &ms), "ensemble::last_ms");
        return ms;
    }
    int count() const {
        int n = 0;
        chk(bfg_ens_count(e, &n), "ensemble::count");
        return n;
    }

  private:
    void chk(int rc, const char* what) const {
        if (rc != BFG_OK)
            throw error(std::string(what) + ": " + bfg_ens_last_error(e) + " (code " +
                            std::to_string(rc) + ")",
                        rc);
    }
    bfg_ens* e = nullptr;
    std::vector<std::pair<bfg_ctx*, std::function<void()>>> members;
};

}  // namespace bfps_b200

#endif
