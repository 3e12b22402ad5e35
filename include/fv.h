/*
 * fv.h -- C-ABI of the B200 (sm_100a) finite-volume solver for the 2D compressible Euler equations.
 *
 * This is the drop-in boundary for the solver step of GusGus2004/neural-pde-surrogate.  The
 * reference's in-process interface is the C++ class e2d::Solver
 *     Solver(const Grid&, FluxFn, Limiter, double cfl)       solver/src/solver2d.hpp:61-64
 *     double compute_dt(const std::vector<Conserved>& U)     solver/src/solver2d.hpp:67-83
 *     void   step(std::vector<Conserved>& U, double dt)      solver/src/solver2d.hpp:86-103
 * with the plug-in points FluxFn (riemann2d.hpp:8) and Limiter (limiters.hpp:5) chosen by name in
 * the driver (main2d.cpp:145-155), the grid of make_grid (grid2d.hpp:30-39), the driver's frame
 * loop (main2d.cpp:224-246) and TrajectoryWriter::add (trajectory.hpp:31-51).  Each entry point
 * below names the piece it replaces.
 *
 * Conventions
 *  - Plain C types only.  Every function returns an int status (FV_OK or an FV_ERR_* code) and never
 *    exits the process; fv_last_error() gives a message for the calling thread's last failure.
 *  - State layout: interior cells only, row-major, 4 doubles per cell (rho, rho*u, rho*v, E), i.e.
 *    U[(j*nx + i)*4 + q] -- the reference's std::vector<Conserved> without the 2-cell ghost ring.
 *    Ghost cells are never stored: boundaries are applied inside the kernels.
 *  - Host buffers are owned by the caller; device buffers by the library.  Functions whose name
 *    ends in _device take device pointers (no host copies).
 *  - One handle must not be used from two threads at once (the reference Solver is not reentrant
 *    either: shared scratch, solver2d.hpp:110-113).  All work runs on the handle's stream.
 *  - Results are bit-identical to the reference's CPU solver for every tile shape and grid size.
 */
#ifndef FV_H
#define FV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FV_OK 0
#define FV_ERR_ARG 1         /* invalid argument (the driver's "must be positive" / unknown-name errors) */
#define FV_ERR_CUDA 2        /* CUDA runtime error, or no usable GPU */
#define FV_ERR_NONPHYSICAL 3 /* !(rho > 0) || !(p > 0) in a cell (solver2d.hpp:75); the reference exits(1) */
#define FV_ERR_TIMEOUT 4     /* a bounded device-side wait gave up */
#define FV_ERR_STATE 5       /* call out of order (e.g. no state set) */

/* boundary conditions (grid2d.hpp:7) */
#define FV_BC_TRANSMISSIVE 0
#define FV_BC_PERIODIC 1
/* flux schemes (main2d.cpp:145-148) */
#define FV_FLUX_RUSANOV 0
#define FV_FLUX_HLLC 1
/* limiters (main2d.cpp:150-155) */
#define FV_LIM_NONE 0
#define FV_LIM_UNLIMITED 1
#define FV_LIM_MINMOD 2
#define FV_LIM_VANLEER 3

typedef struct fv_solver fv_solver;

/* First non-physical cell in row-major order (report_bad_cell, solver2d.hpp:116-126). */
typedef struct {
    int i, j;
    double rho, p;
} fv_bad_cell;

/* Replaces make_grid (grid2d.hpp:30-39) + Solver::Solver (solver2d.hpp:61-64).  Allocates the state
 * and scratch on the current CUDA device once.  stream: a cudaStream_t, or NULL for a stream the
 * library creates. */
int fv_create(int nx, int ny, double x_min, double x_max, double y_min, double y_max, int bc_x, int bc_y,
              int flux, int limiter, double cfl, void* stream, fv_solver** out);
int fv_destroy(fv_solver* s);

/* Conserved state in/out (interior cells, layout above).  Setting the state resets t and the step
 * count to 0 unless fv_set_time is called after it. */
int fv_set_state(fv_solver* s, const double* U);
int fv_get_state(fv_solver* s, double* U);
int fv_set_state_device(fv_solver* s, const double* dU);
int fv_get_state_device(fv_solver* s, double* dU);
/* Primitive (rho, u, v, p), each an (ny, nx) array, converted with to_conserved (state2d.hpp:16-19)
 * as read_initial_condition does (io_hdf5.hpp:197-204).  Returns FV_ERR_ARG if any rho or p is not
 * positive (io_hdf5.hpp:201-202) and leaves the state unchanged. */
int fv_set_primitive(fv_solver* s, const double* rho, const double* u, const double* v, const double* p);

/* Simulation time and step count kept on the device by fv_advance_to. */
int fv_set_time(fv_solver* s, double t);
int fv_get_time(fv_solver* s, double* t, long long* steps);

/* Replaces Solver::compute_dt (solver2d.hpp:67-83): dt = cfl / (sx/dx + sy/dy).  On a non-physical
 * cell returns FV_ERR_NONPHYSICAL and fills *bad (may be NULL) instead of exiting. */
int fv_compute_dt(fv_solver* s, double* dt, fv_bad_cell* bad);

/* Replaces Solver::step (solver2d.hpp:86-103): one SSP-RK2 step with the given dt.  Like the
 * reference's step it does not advance the simulation time (the driver does); it does count the step. */
int fv_step(fv_solver* s, double dt);

/* The driver's inner loop (main2d.cpp:237-242): while (t < t_next) { dt = min(compute_dt(U),
 * t_next - t); step(U, dt); t += dt; } -- run on the device, with dt never leaving the GPU.  Returns
 * FV_ERR_NONPHYSICAL (and *bad) where compute_dt would have exited; the state is then the one that
 * failed the check.  t and steps (may be NULL) receive the new time and total step count. */
int fv_advance_to(fv_solver* s, double t_next, double* t, long long* steps, fv_bad_cell* bad);

/* Replaces TrajectoryWriter::add for one storage level (trajectory.hpp:31-51): f x f block sums in
 * FP64 (j-outer, i-inner) times 1/(f*f), cast to float, layout (4, ny/f, nx/f).  f must divide nx
 * and ny (trajectory.hpp:19-28), else FV_ERR_ARG. */
int fv_block_average(fv_solver* s, int factor, float* out);
int fv_block_average_device(fv_solver* s, int factor, float* d_out);

/* Whole trajectory in one call (main2d.cpp:224-246 in --traj mode): spin up silently to t_start,
 * record frame 0, then nout frames at t_start + (t_end - t_start)*k/nout, each block-averaged to
 * every size in sizes[0..nsizes-1] (a size m means factor nx/m, trajectory.hpp:19-28).  out[l]
 * receives (nout+1, 4, ny/f, nx/f) floats for level l; times (may be NULL) receives nout+1 doubles.
 * *steps (may be NULL) receives the total step count. */
int fv_run_trajectory(fv_solver* s, double t_start, double t_end, int nout, const int* sizes, int nsizes,
                      float** out, double* times, long long* steps, fv_bad_cell* bad);

/* ---- Batched ensemble --------------------------------------------------------------------------
 * Many independent grids ("members", uneven sizes allowed) with one flux and limiter, each keeping
 * its own CFL dt, time and step count, advanced together: one persistent launch per RK stage covers
 * the tiles of every running member, and batches of steps replay a captured CUDA graph.  Replaces
 * running the driver once per trajectory (data/generate.py:60-105, solver_baseline.py:116-117).
 * Every member is bit-identical to its own fv_advance_to run.
 * bounds: 4*count doubles (x_min, x_max, y_min, y_max per member) or NULL for [0,1]^2. */
typedef struct fv_ensemble fv_ensemble;
int fv_ensemble_create(int count, const int* nx, const int* ny, const double* bounds, const int* bc_x,
                       const int* bc_y, int flux, int limiter, double cfl, void* stream, fv_ensemble** out);
int fv_ensemble_destroy(fv_ensemble* e);
/* Member state in/out (interior layout above); setting resets the member's time and step count. */
int fv_ensemble_set_state(fv_ensemble* e, int member, const double* U);
int fv_ensemble_set_state_device(fv_ensemble* e, int member, const double* dU);
int fv_ensemble_get_state(fv_ensemble* e, int member, double* U);
/* All members' states at once, from/to one device buffer holding them back to back in member order
 * (sum of nx*ny*4 doubles); setting resets every member's time and step count. */
int fv_ensemble_set_all_device(fv_ensemble* e, const double* dU);
int fv_ensemble_get_all_device(fv_ensemble* e, double* dU);
/* Device address of a member's state (owned by the ensemble). */
int fv_ensemble_state_device(fv_ensemble* e, int member, double** dU);
/* Every member runs the driver loop (main2d.cpp:237-242) to its own t_next[member].  t, steps and
 * status (each count entries, may be NULL) receive the members' times, step counts and statuses
 * (0 or FV_ERR_NONPHYSICAL); a member that fails stops where compute_dt would have exited while the
 * others continue, and the call then returns FV_ERR_NONPHYSICAL. */
int fv_ensemble_advance_to(fv_ensemble* e, const double* t_next, double* t, long long* steps, int* status);
int fv_ensemble_launch_count(fv_ensemble* e, long long* launches);
/* The ensemble's cudaStream_t (see fv_get_stream). */
int fv_ensemble_get_stream(fv_ensemble* e, void** stream);

/* Face fluxes of n face pairs evaluated on the GPU by the same device code the stage kernels use:
 * the FluxFn (riemann2d.hpp:8; rusanov_flux :11-15, hllc_flux :27-39) for y_face = 0, or
 * flux_y_face (riemann2d.hpp:42-44) for y_face = 1.  UL, UR, F: host arrays of n x 4 doubles.
 * Inspection hook for the Riemann solvers (the reference's test_riemann2d.cpp calls them directly). */
int fv_riemann_flux(int flux, int y_face, int n, const double* UL, const double* UR, double* F);

/* q[k] = a[k] / b[k] for n host doubles, computed on the GPU by the division the stage kernels use
 * at every general division site: IEEE division in libfv.so; in the tolerance build (libfv_tol.so)
 * a Newton-Raphson reciprocal with Markstein's correction.  Checks the tolerance build's division
 * against IEEE on chosen operands. */
int fv_eval_division(int n, const double* a, const double* b, double* q);

/* Division sequences of the stage kernels, for checking them against IEEE division (the reference
 * divides with the IEEE `/` of its CPU build).  Where the parity build replaces `/` it is by a
 * sequence that returns the same correctly rounded quotient:
 *   FV_DIV_GENERAL  a / b at every general division site (IEEE `/` in libfv.so; a Newton-Raphson
 *                   reciprocal with Markstein's correction in libfv_tol.so)
 *   FV_DIV_GM1      a / (GAMMA - 1) (to_conserved, state2d.hpp:17); b is ignored and may be NULL
 *   FV_DIV_ZERO     a / b with a fast path for a zero numerator (to_primitive, state2d.hpp:22-23)
 *   FV_DIV_BACK     RN(RN(a*b) / a): with a = rho and b = u, the velocity to_primitive recovers from
 *                   a face state's momentum (riemann2d.hpp:12,28 on to_conserved(edge), solver2d.hpp:145-148)
 * fv_eval_division_kind evaluates one kind on n host operand pairs.  fv_division_sweep draws n
 * operand pairs on the device (normal numbers near 1 and across the exponent range, zeros,
 * subnormals, infinities, edge mantissas; seeded) and counts the quotients that differ in any bit from
 * IEEE division, with the largest difference in ulps (max_ulps may be NULL).  No reference
 * counterpart (the reference's divisions are its compiler's). */
#define FV_DIV_GENERAL 0
#define FV_DIV_GM1 1
#define FV_DIV_ZERO 2
#define FV_DIV_BACK 3
int fv_eval_division_kind(int kind, int n, const double* a, const double* b, double* q);
int fv_division_sweep(int kind, long long n, unsigned long long seed, long long* mismatches, long long* max_ulps);

/* The (ny+4) x (nx+4) ghosted array that apply_bcs (grid2d.hpp:43-66) builds from the interior
 * state U, produced on the GPU with the boundary mapping the stage kernels use (no ghost ring is
 * stored by the solver itself).  Ug: host array of (ny+4)*(nx+4)*4 doubles. */
int fv_fill_ghosts(int nx, int ny, int bc_x, int bc_y, const double* U, double* Ug);

/* The persistent stepper's dependency lists for an nx x ny grid of tx x ty tiles (host code, no GPU
 * needed): for tile t (row-major over tiles), idx[off[t] .. off[t+1]) are the tiles holding a cell of
 * its halo box [i0-2, i0+tx+1] x [j0-2, j0+ty+1] once mapped through the boundary conditions
 * (grid2d.hpp:43-66), and the tiles whose halo box holds one of its cells, itself included, sorted.
 * *nnz receives the number of entries; off (ntiles + 1 entries) and idx are filled when their
 * capacities suffice.  Inspection hook; no reference counterpart. */
int fv_stepper_dependencies(int nx, int ny, int bc_x, int bc_y, int tx, int ty, int* off, int off_cap, int* idx,
                            int idx_cap, int* nnz);

/* Tile shapes.  The stage kernels exist for several CTA tile shapes (fv_tile_variant enumerates
 * them: tile width, height, threads); all give bit-identical results.  A handle picks the fastest
 * for its grid by timing each on a copy of its state the first time it steps (the autotuner; the
 * choice is cached per device, grid size, flux and limiter for the process).  FV_TILE=<index> in
 * the environment fixes the shape instead, FV_AUTOTUNE=0 keeps the default.  fv_autotune re-times
 * now (steps per variant, <= 0 for the default) and returns the chosen index. */
int fv_autotune(fv_solver* s, int steps, int* variant);
int fv_set_tile(fv_solver* s, int variant);
int fv_get_tile(fv_solver* s, int* variant);
int fv_tile_variant(int variant, int* tx, int* ty, int* threads);

/* Kernel timing (the reference's --profile, solver2d.hpp:29-52, main2d.cpp:261): while enabled,
 * CUDA events bracket every stage-kernel launch of the handle; fv_profile_read returns the mean
 * duration in ms of stage-1 and stage-2 launches and the number of steps timed since enabling. */
int fv_profile(fv_solver* s, int enable);
int fv_profile_read(fv_solver* s, double* ms_stage1, double* ms_stage2, long long* steps_timed);
/* The same, per whole step and for both kernel paths: fv_advance_to runs on the persistent stepper
 * (one cooperative launch per batch of steps, FV_STEPPER=0 in the environment to use the per-stage
 * kernels instead), whose stages have no launches of their own.  ms_per_step: mean device time per
 * step of every timed launch since fv_profile(s, 1); steps: steps timed; launches: stepper launches
 * timed.  Any pointer may be NULL. */
int fv_profile_steps(fv_solver* s, double* ms_per_step, long long* steps, long long* launches);
/* The tile shape the handle's persistent stepper uses (0s before its first fv_advance_to, or when the
 * stepper is switched off).  Chosen like the per-stage kernels' shape, by timing each on a copy of
 * the state; FV_STEPPER_TILE=<index> fixes it. */
int fv_stepper_tile(fv_solver* s, int* tx, int* ty, int* threads);
/* The stepper shape's index (what FV_STEPPER_TILE takes) and its launch: CTAs per SM and CTAs in
 * all; -1 and 0s before the first fv_advance_to or with the stepper switched off.  Any pointer may
 * be NULL. */
int fv_stepper_launch(fv_solver* s, int* variant, int* ctas_per_sm, int* ctas);

/* Self-test of the library's bounded waits: runs the wait used for every TMA copy and tensor-core
 * batch on a barrier that nothing arrives at, with a 10 ms limit.  Returns FV_ERR_TIMEOUT when the
 * wait gave up and reported it (the expected outcome; the context stays usable), FV_ERR_STATE if it
 * did not, FV_ERR_CUDA on a CUDA error.  No reference counterpart (the reference has no GPU code). */
int fv_wait_selftest(void);

/* Self-test of the persistent stepper's bounded waits: its wait for a step's publication and its
 * wait for neighbour tiles' flags, each run against a control block and a flag that nothing ever
 * publishes, with a 10 ms limit, plus a second CTA waiting with the default limit that must leave as
 * soon as the first has recorded the timeout.  Returns FV_ERR_TIMEOUT when every wait gave up and
 * reported it (the expected outcome; the context stays usable), FV_ERR_STATE if not, FV_ERR_CUDA on
 * a CUDA error.  No reference counterpart. */
int fv_stepper_wait_selftest(void);

/* Measured FP64 FMA throughput of the current device (DFMA per second, one FMA = 2 flops): the
 * denominator of the FP64-pipe roofline the stage kernels are reported against.  No reference
 * counterpart (the reference has no GPU code). */
int fv_fp64_peak(double* dfma_per_second);

/* One SSP-RK2 step with a fixed dt (Solver::step semantics, bit-identical to fv_step) on a
 * caller-owned device state d_U (interior layout above, updated in place), that allocates no device
 * memory: for callers that cannot call cudaMalloc at that point -- a host running inside another
 * framework's memory pool, or a driver loop that forbids allocation after start-up.  Its scratch is
 * a fixed array compiled into the library (about 1.5 MB, held by every GPU that loads the library
 * until exit), so grids are limited to FV_NOALLOC_MAX_CELLS cells (larger ones return FV_ERR_ARG).
 * All calls on a device share that scratch: calls that overlap on the GPU race and must be
 * serialised by the caller.  The first call on a device sets up the scratch address; make it before
 * any stream capture, and do not use this entry point across cudaDeviceReset (the set-up is cached
 * for the process).  d_U must be 16-byte aligned, as cudaMalloc'd memory is: the kernels move each
 * cell with two 16-byte accesses, and a misaligned pointer returns FV_ERR_ARG with nothing launched.
 * stream: a cudaStream_t or NULL.  No counterpart in the reference. */
#define FV_NOALLOC_MAX_CELLS (128 * 128)
int fv_step_noalloc(int nx, int ny, double x_min, double x_max, double y_min, double y_max, int bc_x, int bc_y,
                    int flux, int limiter, double* d_U, double dt, void* stream);

/* Number of kernels the handle has launched since it was created. */
int fv_launch_count(fv_solver* s, long long* launches);

/* Blocks until all work queued on the handle's stream is done. */
int fv_synchronize(fv_solver* s);

/* The cudaStream_t the handle's work is queued on (the one given to fv_create, or the library's own
 * non-blocking stream).  The *_device entry points read and write caller memory in this stream's
 * order: a caller that produces or consumes those buffers on another stream orders the two streams
 * itself (events), e.g. the Python mirror against torch's current stream.  No reference counterpart
 * (the reference is CPU code). */
int fv_get_stream(fv_solver* s, void** stream);

/* Message for the calling thread's last failing call ("" if none). */
const char* fv_last_error(void);

/* Library version string. */
const char* fv_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FV_H */
