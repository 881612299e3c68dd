/*
 * bfps_b200 — single-GPU (B200, sm_100a) engine for bfps' pseudospectral
 * vorticity-equation DNS step and Lagrangian tracer step.
 *
 * C ABI: plain pointers and sizes only; no exceptions cross it.  Every entry
 * point returns 0 on success or a negative BFG_E* code; the message of the
 * most recent failure on a context is kept until the next call
 * (bfg_last_error).  One host thread drives a context (the reference is
 * MPI_THREAD_FUNNELED with OpenMP inside calls, main_code.hpp:74-96);
 * distinct contexts may be driven from distinct threads.
 *
 * Memory layouts at the boundary are exactly the reference's host layouts
 * (bfps/cpp/field.cpp:85-101):
 *   complex 3-vector field: [ky][kz][kx][c][re,im], kx in 0..nx/2
 *                           ("transposed out", shape (ny, nz, nx/2+1, 3))
 *   real 3-vector field:    [z][y][x][c] with x padded to nx+2
 *                           (shape (nz, ny, nx+2, 3); the pad is written as 0)
 *   tracers:                positions (n, 3) f64, rhs history (nsteps, n, 3)
 *                           f64, indices (n) i64, in global index order
 *                           (particles_output_hdf5.hpp).
 * Scalars are float when real_bytes == 4 and double when real_bytes == 8.
 */
#ifndef BFPS_B200_H
#define BFPS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bfg_ctx bfg_ctx;
typedef struct bfg_pctx bfg_pctx;

/* error codes */
#define BFG_OK 0
#define BFG_EINVAL -1     /* bad argument */
#define BFG_ECUDA -2      /* CUDA runtime error */
#define BFG_ENOMEM -3     /* device allocation failed */
#define BFG_EUNSUP -4     /* configuration the library does not support */
#define BFG_ESTATE -5     /* call not valid in the current state */

/* dealiasing (bfps/cpp/kspace.hpp:40, enum kspace_dealias_type) */
#define BFG_TWO_THIRDS 0
#define BFG_SMOOTH 1

/* forcing_type (bfps/cpp/vorticity_equation.cpp:241-288) */
#define BFG_FORCING_NONE 0
#define BFG_FORCING_LINEAR 1
#define BFG_FORCING_KOLMOGOROV 2

/* field ids for upload / download */
#define BFG_FIELD_VORTICITY 0   /* complex state, vorticity_equation::cvorticity */
#define BFG_FIELD_VELOCITY 1    /* complex, vorticity_equation::cvelocity */
#define BFG_FIELD_RVELOCITY 2   /* real velocity, cvelocity after ift() */

/* Library version string. */
const char* bfg_version(void);

/* Create a solver context: replaces the constructors of
 * vorticity_equation<rnumber, FFTW> (bfps/cpp/vorticity_equation.cpp:110-156)
 * with its five field<rnumber, FFTW, THREE> buffers (field.cpp:37-121) and
 * kspace<FFTW, dt> (kspace.cpp:34-167).  Grids are cubic, nx = ny = nz = n,
 * n a power of two in [16, 1024].  real_bytes selects rnumber (4 or 8).
 * The state starts at zero with iteration 0 and the reference constructor's
 * physical defaults (nu 0.1, forcing none). */
int bfg_ctx_create(bfg_ctx** out, int nx, int ny, int nz, double dkx, double dky,
                   double dkz, int real_bytes, int dealias_type, int device);
void bfg_ctx_destroy(bfg_ctx* ctx);
const char* bfg_last_error(const bfg_ctx* ctx);

/* Physical parameters: the public members nu, forcing_type, famplitude,
 * fk0, fk1, fmode of vorticity_equation (vorticity_equation.hpp:46-134). */
int bfg_set_physics(bfg_ctx* ctx, double nu, int forcing_type, double famplitude,
                    double fk0, double fk1, int fmode);

/* kspace information (kspace.hpp:43-60): kM, dk, nshells; kshell / nshell
 * arrays of length nshells may be NULL. */
int bfg_kspace_info(const bfg_ctx* ctx, double* kM, double* dk, int* nshells,
                    double* kshell, int64_t* nshell);

/* Host <-> device copies in the reference layouts above.
 * Upload of BFG_FIELD_VORTICITY replaces the state; it does NOT apply the
 * checkpoint-read transformations (use bfg_read_checkpoint_fixup). */
int bfg_field_upload(bfg_ctx* ctx, int field_id, const void* host);
int bfg_field_download(bfg_ctx* ctx, int field_id, void* host);

/* io_checkpoint(read) post-processing of the state
 * (vorticity_equation.hpp:107-128 with field::io's symmetrize at
 * field.cpp:340): symmetrize, low_pass(kM), force_divfree. */
int bfg_read_checkpoint_fixup(bfg_ctx* ctx);

/* vorticity_equation::step (vorticity_equation.cpp:358-439), nsteps times:
 * one IF-RK3 step each, iteration += 1 each. */
int bfg_step(bfg_ctx* ctx, double dt, int nsteps);

/* vorticity_equation::compute_velocity(cvorticity)
 * (vorticity_equation.cpp:206-239): fills BFG_FIELD_VELOCITY. */
int bfg_compute_velocity(bfg_ctx* ctx);

/* compute_velocity(cvorticity) followed by cvelocity->ift()
 * (NSVEparticles.cpp:35-36): fills BFG_FIELD_RVELOCITY. */
int bfg_velocity_rspace(bfg_ctx* ctx);

/* vorticity_equation::compute_pressure (vorticity_equation.cpp:441-514) of
 * the velocity of the current state (compute_velocity + ift first, as
 * compute_Lagrangian_acceleration does at :528-531).  If host is not NULL
 * the pressure is written there in the reference complex layout
 * (ny, nz, nx/2+1) of one component.  Leaves BFG_FIELD_RVELOCITY set. */
int bfg_compute_pressure(bfg_ctx* ctx, void* host);

/* vorticity_equation::compute_Lagrangian_acceleration
 * (vorticity_equation.cpp:516-578) of the current state, in Fourier space;
 * written to host (reference layout (ny, nz, nx/2+1, 3)) if not NULL. */
int bfg_lagrangian_acceleration(bfg_ctx* ctx, void* host);

/* field::ift / field::dft (field.cpp:144-162) on a 3-vector field, using
 * caller device buffers in the reference layouts (complex: (n, n, n/2+1, 3),
 * real: (n, n, n+2, 3)); unnormalised like FFTW.  in may equal out; host
 * or device memory (unified addressing).  Where either buffer is device
 * memory the call first waits for all work queued on the device (the
 * caller's kernels on any stream), and it returns once the output is
 * complete. */
int bfg_ift(bfg_ctx* ctx, const void* dev_complex_in, void* dev_real_out);
int bfg_dft(bfg_ctx* ctx, const void* dev_real_in, void* dev_complex_out);

/* field::ift of the context's velocity (cvelocity->ift(), as
 * NSVEparticles::step calls it after compute_velocity, NSVEparticles.cpp:
 * 35-36): the C2R of BFG_FIELD_VELOCITY into BFG_FIELD_RVELOCITY; the
 * complex velocity is kept.  Other field ids: BFG_EINVAL. */
int bfg_field_ift(bfg_ctx* ctx, int field_id);

/* field::compute_stats (field.cpp:984-1040) of any complex 3-vector field
 * in the reference layout (ny, nz, nx/2+1, 3), in host or device memory:
 * co-spectrum (nshells, 3, 3), real-space moments (10, 4) and histograms
 * (nbins, 4) with max_estimate per component (max_estimate sqrt(3) for the
 * magnitude, field.cpp:1001-1004).  Uses the context's free RK buffer; the
 * state and the velocity are untouched.  Outputs may be NULL.  A field in
 * device memory is read after all work queued on the device. */
int bfg_field_stats(bfg_ctx* ctx, const void* field, double max_estimate, int nbins,
                    double* spec, double* mom, int64_t* hist);

/* No counterpart in the reference: returns a context to the state of a new
 * one of the same grid (every field buffer zero, iteration 0), keeping its
 * device memory, physics members and tables, so that a server can reuse it
 * for the next solve of that size without freeing and allocating. */
int bfg_ctx_reset(bfg_ctx* ctx);

/* iteration counter (vorticity_equation::iteration). */
int bfg_get_iteration(const bfg_ctx* ctx, int* iteration);
int bfg_set_iteration(bfg_ctx* ctx, int iteration);

/* Field statistics of NSVE::do_stats (bfps/cpp/full_code/NSVE.cpp:101-135)
 * for the current state: co-spectra (kspace::cospectrum, kspace.cpp:521-598)
 * of vorticity and velocity, (nshells, 3, 3) f64 each, and real-space
 * moments (10, 4) f64 and histograms (nbins, 4) i64
 * (field::compute_rspace_stats, field.cpp:661-889).  max_*_estimate are the
 * parameters of the same names; any output pointer may be NULL. */
int bfg_stats(bfg_ctx* ctx, double max_velocity_estimate, double max_vorticity_estimate,
              int nbins, double* spec_vel, double* spec_vort, double* mom_vel,
              double* mom_vort, int64_t* hist_vel, int64_t* hist_vort);

/* Number of non-finite values (NaN or +-Inf, real and imaginary parts
 * counted separately) in a field on the device, written to *nonfinite.
 * Stands in for the floating-point-exception trapping the reference enables
 * in its host code (bfps/cpp/full_code/main_code.hpp:48-52), which cannot
 * see device arithmetic: a run checks its state with it and stops instead
 * of writing a corrupted checkpoint.  field_id as for bfg_field_download. */
int bfg_check_finite(bfg_ctx* ctx, int field_id, int64_t* nonfinite);

/* ---------------------------------------------------------- tracers ---- */

/* particles_system_builder (bfps/cpp/particles/particles_system_builder.hpp:
 * 111-257) + particles_system::init (particles_system.hpp:81-121):
 * n tracers, interpolation (neighbours 1..5, smoothness 0..2; 0 = Lagrange),
 * nsteps >= 1 Adams-Bashforth history slots, step_idx = iteration + 1 of the
 * run that resumes (NSVEparticles.cpp:23).  pos is (n, 3), rhs is
 * (nsteps, n, 3) (may be NULL for zeros), idx is (n) (NULL for 0..n-1). */
int bfg_particles_create(bfg_ctx* ctx, bfg_pctx** out, int64_t n, int neighbours,
                         int smoothness, int nsteps, const double* pos,
                         const double* rhs, const int64_t* idx, int step_idx);
void bfg_particles_destroy(bfg_pctx* p);

/* particles_system::completeLoop(dt) (particles_system.hpp:210-217) using
 * the context's real velocity field (BFG_FIELD_RVELOCITY). */
int bfg_particles_complete_loop(bfg_pctx* p, double dt);

/* NSVEparticles::step (bfps/cpp/full_code/NSVEparticles.cpp:33-41):
 * velocity at time t -> tracers advance -> fluid IF-RK3 step, nsteps times.
 * p may be NULL (then this is NSVE::step). */
int bfg_nsveparticles_step(bfg_ctx* ctx, bfg_pctx* p, double dt, int nsteps);

/* Sample the context's real velocity field at the tracer positions
 * (particles_system::sample_compute, particles_system.hpp:134-170) into
 * out (n, 3) in global index order. */
int bfg_particles_sample_velocity(bfg_pctx* p, double* out);

/* The acceleration half of NSVEparticles::do_stats (NSVEparticles.cpp:
 * 84-91): compute_Lagrangian_acceleration of the current state, ift, and
 * sample it at the tracer positions into out (n, 3) in global index order
 * (the context's real velocity field is left untouched). */
int bfg_particles_sample_acceleration(bfg_pctx* p, double* out);

/* Replace positions (n, 3) and the rhs history (nsteps, n, 3, NULL for
 * zeros) of existing tracers, in the order given at creation, and set
 * step_idx (checkpoint read, particles_input_hdf5.hpp:61-279). */
int bfg_particles_upload(bfg_pctx* p, const double* pos, const double* rhs, int step_idx);

/* State in global index order: pos (n, 3), rhs (nsteps, n, 3), idx (n);
 * any pointer may be NULL. */
int bfg_particles_download(bfg_pctx* p, double* pos, double* rhs, int64_t* idx);
int bfg_particles_info(const bfg_pctx* p, int64_t* n, int* nsteps, int* step_idx);

/* ------------------------------------------------------ ensembles ---- */

/* Batched form (no counterpart in the single-instance reference; each
 * member's step is vorticity_equation::step / NSVEparticles::step): many
 * independent contexts of any sizes, viscosities and seeds, advanced
 * together.  Members of equal grid size share one persistent launch per
 * pass and RK stage; the fluid launches are replayed from CUDA graphs;
 * tracers advance after stage 1 of the step, as in NSVEparticles::step.
 * Members keep
 * their state and API; while in an ensemble they must be stepped only
 * through it.  All members share one device and one precision. */
typedef struct bfg_ens bfg_ens;
int bfg_ens_create(bfg_ens** out, int device);
void bfg_ens_destroy(bfg_ens* e);
const char* bfg_ens_last_error(const bfg_ens* e);
/* add a member with its fixed time step (and optional tracers) */
int bfg_ens_add(bfg_ens* e, bfg_ctx* member, bfg_pctx* tracers_or_null, double dt);
int bfg_ens_remove(bfg_ens* e, bfg_ctx* member);
int bfg_ens_count(const bfg_ens* e, int* members);
/* nsteps NSVEparticles steps of every member */
int bfg_ens_step(bfg_ens* e, int nsteps);
/* device time of the last bfg_ens_step call (synchronises) */
int bfg_ens_last_ms(bfg_ens* e, double* ms);
/* poll with a timeout: *done = 1 once the work of the last bfg_ens_step
 * call has finished, 0 if it is still running after timeout_ms (0 polls
 * once); the host waits, the device is not blocked.  The serving loop's
 * "poll with timeout" (bfps' request loop has no counterpart: new) */
int bfg_ens_wait(bfg_ens* e, double timeout_ms, int* done);
/* replay the fluid launches from CUDA graphs (default 1) or launch directly */
int bfg_ens_use_graphs(bfg_ens* e, int enable);
/* kernels launched by bfg_ens_step since creation (the nodes of replayed
 * graphs included) */
int bfg_ens_kernel_launches(const bfg_ens* e, int64_t* count);

/* ------------------------------------------------------ measurement ---- */

/* Synchronise the context's stream and return the device time of the last
 * bfg_step / bfg_nsveparticles_step call in milliseconds (CUDA events). */
int bfg_last_step_ms(bfg_ctx* ctx, double* ms);

/* Per-kernel device timing.  With profiling on, every launch on the
 * context's stream is bracketed by CUDA events and its duration is added to
 * its kind: 0 IZ (inverse over kz, fused compute_velocity), 1 IY (inverse
 * over ky), 2 X (row pass: C2R, u x w, R2C), 3 FY (forward over y),
 * 4 FZ (forward over z, fused dealias / curl / forcing / divfree / RK),
 * 5 small k-space kernels, 6 tracers, 7 statistics.  bfg_profile_read
 * synchronises, returns the accumulated milliseconds and launch count of a
 * kind, and bfg_profile(ctx, 1) also clears the accumulators. */
#define BFG_NKINDS 8
int bfg_profile(bfg_ctx* ctx, int enable);
int bfg_profile_read(bfg_ctx* ctx, int kind, double* total_ms, int64_t* launches);

/* Autotuner of the column passes (no counterpart in the reference, whose
 * FFTW plans are chosen by FFTW's own planner rigor, bfps/cpp/
 * fftw_interface.hpp:30-35).  Every pass over z or y (kinds 0 IZ, 1 IY,
 * 3 FY, 4 FZ) is built in two schedules: 0, two 256-thread CTAs per SM with
 * one tile buffer each and 32-point butterflies in FP32; 1, one 512-thread
 * CTA with two tile buffers and radix-8 butterflies.  The choice is kept per
 * device, grid size, precision and members per launch (1 for a lone
 * context; the size of an ensemble's group of equal grids otherwise), since
 * the better schedule depends on how many tiles one launch holds.
 * bfg_autotune times both on this context's buffers (reps launches each,
 * after one warm-up; only the work buffers are written, so the complex and
 * real velocity of the context are lost) for one member per launch.
 * bfg_ens_autotune does the same for every size group of an ensemble, as
 * bfg_ens_step launches it (all members of the group in one launch), and
 * re-captures the ensemble's graphs at its next step.  Schedule 1 is chosen
 * only when it is more than 2% faster than schedule 0 (10% for the groups of
 * an ensemble that holds several grid sizes, whose launches run
 * concurrently: schedule 1 holds all of an SM's shared memory).  Where the environment
 * variable BFPS_B200_TUNE_CACHE names a file, the choices are appended to it
 * and read back by later processes on a device of the same name.  A key
 * never tuned uses schedule 0.  bfg_tune_get reads the choice for a member
 * count and its measured times (0 when not measured), bfg_tune_set imposes
 * one. */
int bfg_autotune(bfg_ctx* ctx, int reps);
int bfg_ens_autotune(bfg_ens* e, int reps);
int bfg_tune_get(const bfg_ctx* ctx, int kind, int members, int* schedule, double* ms0, double* ms1);
int bfg_tune_set(bfg_ctx* ctx, int kind, int members, int schedule);

/* No counterpart in the reference: exercises the error path of the
 * library's bounded waits.  Kernels that wait on their own TMA bulk copies
 * (mbarrier waits) give up after a bound, set a device status word and
 * return; the next synchronising call (bfg_last_step_ms, a download) reads
 * the word and fails with BFG_ECUDA and a message.  This call launches one
 * warp whose wait, on an mbarrier that nothing arms, runs out after a short
 * bound, and returns what that check reports: BFG_ECUDA, with the status
 * word cleared and the context still usable. */
int bfg_selftest_wait(bfg_ctx* ctx);

/* Count of kernels the library launched since the context was created. */
int bfg_kernel_launches(const bfg_ctx* ctx, int64_t* count);

/* ------------------------------------------------- no-allocation stats ---- */

/* No counterpart in the reference: an extra entry point for callers that
 * cannot call cudaMalloc (device memory already owned or reserved by another
 * framework's allocator, a footprint fixed at start-up, or a loop that
 * cannot afford cudaMalloc's device-wide synchronisation).
 *
 * Computes the real-space moments (10, 4) f64 and histogram (nbins, 4) i64 of
 * field::compute_rspace_stats (field.cpp:661-889) for a real 3-vector field
 * in the reference layout (nz, ny, nx+2, 3) (float if real_bytes == 4, else
 * double).  max_estimate is the per-component estimate (the magnitude uses
 * max_estimate * sqrt(3)).  All pointers are device pointers supplied by the
 * caller; the work is queued on `stream` (NULL: the default stream) and the
 * call returns without waiting for it.
 *
 * Allocates nothing: the per-block partial sums live in a fixed 370 KiB
 * device array inside the library, present on every GPU that loads it until
 * the library is unloaded.  The first call in each device context (and the
 * first after a device reset, which creates a new context) looks up that
 * array's device address (with the device current) and should come before
 * any stream capture.  Rows are 2 (nx/2 + 1) values apart (nx + 2 for even
 * nx).  All calls share the array, so calls that overlap on
 * the GPU (for example on two streams at once) race; order them.  The
 * histogram output is cleared by the call itself.  nbins above
 * BFG_NOALLOC_MAX_BINS returns BFG_EUNSUP. */
#define BFG_NOALLOC_MAX_BINS 2048
int bfg_rspace_stats_noalloc(const void* dev_field, int nx, int ny, int nz, int real_bytes,
                             double max_estimate, int nbins, double* dev_moments,
                             int64_t* dev_hist, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BFPS_B200_H */
