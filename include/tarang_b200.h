/*
 * tarang_b200.h -- C ABI of libtarang_b200.so, the sm_100a implementation of
 * Tarang.jl's IMEX timestep hot path for RealFourier(x) x ChebyshevT(z) tau
 * problems (2D Boussinesq Rayleigh-Benard convection).
 *
 * Every entry point returns a tb_status; nothing throws or aborts across the
 * ABI.  Pointers are borrowed for the duration of the call only.  Device
 * buffers are owned by the library.  Calls on one plan are not thread-safe
 * (one CUDA stream per plan); distinct plans may be used concurrently.
 *
 * Array conventions (identical to the reference's column-major storage):
 *   grid field        real    (Nx, Nz) column-major  -> element (x, z) at x + z*Nx
 *   coefficient field complex (Nx/2+1, Nz) column-major, interleaved (re, im)
 *                     -> element (k, n) at 2*(k + n*(Nx/2+1))
 *   tau field         complex (Nx/2+1) per tau variable
 */
#ifndef TARANG_B200_H
#define TARANG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int tb_status;
enum {
  TB_OK = 0,
  TB_EINVAL = 1,        /* bad argument, shape or descriptor                  */
  TB_ENOMEM = 2,        /* device allocation failed                           */
  TB_ESINGULAR = 3,     /* a tau system is singular; tb_last_error names mode */
  TB_ETIMEOUT = 4,      /* a bounded device wait gave up                      */
  TB_ECUDA = 5,         /* CUDA runtime error (message in tb_last_error)      */
  TB_ENOTSUPPORTED = 6, /* size/feature outside what the kernels implement    */
  TB_EBUDGET = 7,       /* request exceeds the HBM budget of a server         */
  TB_ESTATE = 8         /* call order violated (e.g. solve before factor)     */
};

typedef struct tb_context tb_context;
typedef struct tb_plan tb_plan;

/* Where a host-visible pointer lives. */
enum { TB_HOST = 0, TB_DEVICE = 1 };
/* OR'ed into `where` of tb_set_state / tb_set_states: the write keeps the
 * multistep (SBDF) history.  For a caller that mirrors the plan's state in its
 * own field arrays and writes them back before every step (the Julia
 * extension's per-step sync): the reference keeps its history across writes
 * into a live state field (timestepper_data, src/core/timesteppers/state.jl:47-91),
 * and a plain write restarts the history at SBDF1. */
enum { TB_KEEP_HISTORY = 0x10 };
/* OR'ed into where of tb_set_states: return once the copies are queued on the
 * plan's stream instead of waiting for them (cudaMemcpyAsync semantics).  A
 * pinned host source must then stay unchanged until the plan's next wait
 * (tb_step, tb_get_states, tb_plan_wait, tb_synchronize); a pageable source
 * is consumed before the call returns (the runtime stages it).  The next
 * step or read-back queues behind the copies.  tb_get_states refuses it
 * (TB_EINVAL): its data is read by the caller after the return. */
enum { TB_NO_WAIT = 0x20 };

/* Time steppers (src/core/timesteppers/types.jl:49-167, 217). */
enum { TB_RK222 = 0, TB_RK443 = 1, TB_SBDF1 = 2, TB_SBDF2 = 3 };

/* Equation programs.  TB_PROGRAM_RBC is the Boussinesq system of
 * test/test_subproblem_rk.jl:50-57 (first-order tau formulation with
 * lift(., -1) on the last ChebyshevT mode).  TB_PROGRAM_TURB2D is the doubly
 * periodic vorticity-streamfunction system of
 * examples/2d_decaying_turbulence_gpu.jl (dq/dt - nu Lap q = -u.grad q,
 * Lap psi = q with zero-mean gauge, u = skew(grad psi)) stepped with
 * DiagonalIMEX_SBDF2 in FP32 (uses Nx, Ny, Lx, Ly, nu). */
enum { TB_PROGRAM_RBC = 0, TB_PROGRAM_TURB2D = 1 };

/* Arithmetic of the step. */
enum { TB_PREC_F64 = 0, TB_PREC_MIXED = 1 };

/* Field selectors for tb_set_state / tb_get_state.  3D plans (ndim 3) hold
 * coefficient fields complex (Nx/2+1, Ny, Nz) column-major (kx fastest, ky in
 * FFT order) and 9 taus of (Nx/2+1, Ny): tau_p, tau_b1, tau_b2, tau_u1x,
 * tau_u1y, tau_u1z, tau_u2x, tau_u2y, tau_u2z. */
enum {
  TB_FIELD_B = 0, TB_FIELD_UX = 1, TB_FIELD_UZ = 2, TB_FIELD_P = 3,
  TB_FIELD_TAU = 4, /* 2D: 7 x (Nx/2+1) complex: tau_p, tau_b1, tau_b2, tau_u1x, tau_u1z, tau_u2x, tau_u2z */
  TB_FIELD_UY = 5   /* 3D only */
};

typedef struct tb_problem_desc {
  int ndim;          /* 2, or 3 (RealFourier y, RK222 / RK443, even Nz)          */
  int Nx, Ny, Nz;    /* grid sizes (Ny ignored in 2D)                            */
  double Lx, Ly, Lz; /* x in [0,Lx), y in [0,Ly), z in [0,Lz]                    */
  double dealias;    /* 3/2 padding factor along Fourier axes                    */
  int precision;     /* TB_PREC_*                                                */
  int timestepper;   /* TB_RK222 ...                                             */
  int program;       /* TB_PROGRAM_RBC or TB_PROGRAM_TURB2D                      */
  double kappa, nu;  /* b diffusivity, kinematic viscosity                       */
  double b_bottom;   /* value of b at z = 0   (BC "b(z=0) = ...")               */
  double b_top;      /* value of b at z = Lz  (BC "b(z=Lz) = ...")              */
} tb_problem_desc;

/* -------------------------------------------------------------------------
 * Context and errors.  Replaces the device selection the reference does
 * through CUDA.jl when arch=GPU() (src/core/architectures.jl:107).
 * ---------------------------------------------------------------------- */
tb_status tb_context_create(int device, tb_context** out);
tb_status tb_context_destroy(tb_context* ctx);
const char* tb_last_error(const tb_context* ctx);
const char* tb_status_string(tb_status s);
int tb_version(void);

/* -------------------------------------------------------------------------
 * Timestep plan.  Replaces InitialValueSolver(problem, ts; dt) for arch=GPU()
 * (src/core/solvers/solver_types.jl:468-573, 993): builds the per-Fourier-mode
 * tau operators that build_matrices! assembles
 * (src/core/subsystems/subproblem_matrix_build.jl:11-309) in the library's own
 * banded form and allocates all device state.
 * ---------------------------------------------------------------------- */
tb_status tb_plan_create(tb_context* ctx, const tb_problem_desc* desc, tb_plan** out);
tb_status tb_plan_destroy(tb_plan* plan);

/* Coefficient-space state I/O (the fields' coefficient layout, :c).
 * where = TB_HOST or TB_DEVICE.  Replaces get_coeff_data/set on state fields.
 * A set restarts the multistep history unless TB_KEEP_HISTORY is OR'ed into
 * where. */
tb_status tb_set_state(tb_plan* plan, int field, const void* data, int where);
tb_status tb_get_state(tb_plan* plan, int field, void* data, int where);
/* Several fields in one call: data[i] holds field fields[i] (2D plans).  The
 * copies are queued back to back on the plan's stream and the call returns
 * once all of them are done (one wait instead of one per field), so a caller
 * that moves the whole state every step (b, u_x, u_z, p, taus) pays one
 * host/device round trip each way.  Fields adjacent in the device state
 * (b, u_x, u_z, p, taus in that order) whose buffers are also adjacent in the
 * caller's memory go as one copy.  Same layouts and ownership as
 * tb_set_state / tb_get_state; a bad selector fails before any copy. */
tb_status tb_set_states(tb_plan* plan, int nfields, const int* fields, const void* const* data, int where);
tb_status tb_get_states(tb_plan* plan, int nfields, const int* fields, void* const* data, int where);

/* Advance nsteps steps of size dt.  Replaces step!(solver, dt)
 * (src/core/solvers/solver_stepping.jl:24-38) through
 * _dispatch_step! -> step_subproblem_rk! / step_subproblem_multistep!
 * (src/core/timesteppers/dispatch.jl:22-230).  The first call for a new dt
 * factors the tau systems (once per (dt, a_ii)); later calls replay a CUDA
 * graph of one step. */
tb_status tb_step(tb_plan* plan, double dt, int nsteps);
tb_status tb_sim_time(const tb_plan* plan, double* t, long long* iteration);
/* Wait for the plan's stream (the step is asynchronous otherwise). */
tb_status tb_synchronize(tb_plan* plan);

/* Device-side timing of the last tb_step call in milliseconds (CUDA events on
 * the plan's stream). */
tb_status tb_last_step_ms(const tb_plan* plan, float* ms);
/* Per-kernel timing (the library's own tracing, standing in for the
 * reference's opt-in transform counters, transform_fourier.jl:49-65).  With
 * profiling on, tb_step launches the step eagerly (no graph replay) with CUDA
 * events around every kernel and accumulates (total ms, launches) per kernel
 * name; entries are listed in name order. */
tb_status tb_set_profiling(tb_plan* plan, int on);
tb_status tb_profile_count(const tb_plan* plan, int* n);
tb_status tb_profile_entry(const tb_plan* plan, int i, char* name, int name_len, double* ms_total,
                           long long* launches);
tb_status tb_profile_reset(tb_plan* plan);
/* Host-only query of the banded layout the plan compiler builds for the RBC
 * tau system (no GPU needed): info4 = {band rows n, border size nb, kl, ku}
 * for parity class cls (0 or 1). */
tb_status tb_tau_layout_query(int Nz, double Lx, double Lz, int cls, int* info4);
/* Number of kernels one step launches (for launch accounting). */
tb_status tb_kernels_per_step(const tb_plan* plan, int* n);

/* Dynamic wall values of b (time- and space-dependent boundary conditions
 * b(z=0) = f(x[, y], t), b(z=Lz) = g(x[, y], t)).  Replaces the per-stage BC
 * refresh and ALG_F re-gather of the reference (step_subproblem_rk.jl:547-560,
 * subproblem_rhs.jl:523-607): wall 0 is z = 0, wall 1 is z = Lz; value are the
 * coefficients of the wall profile (the unnormalised transform of its grid
 * values: complex Nx/2+1 in 2D, (Nx/2+1, Ny) kx fastest in 3D) at the plan's
 * current time, rate their time derivative (NULL: constant), so each stage
 * solve sees value + rate (t_stage - now); rk stage times are t_n + c_i dt,
 * SBDF solves t_{n+1}.  A time dependence other than linear is followed by
 * calling this between steps.  The first call replaces the descriptor's
 * constant b_bottom / b_top (the other wall keeps its constant until set). */
tb_status tb_set_wall_values(tb_plan* plan, int wall, const double* value, const double* rate, int where);

/* Checkpoints (save_state / load_state!, src/tools/solver_checkpoint.jl:88-194).
 * tb_checkpoint_stage transforms the state to the grid on the device - fields
 * b, u_x, (u_y,) u_z, p, each real (Nx, Nz) or (Nx, Ny, Nz) column-major,
 * back to back - and copies them to host_grid (capacity in doubles) on a side
 * stream: the call returns at once, the plan may step on, and
 * tb_checkpoint_wait completes the copy (host_grid should be pinned for the
 * copy to overlap).  clock = {sim_time, iteration, last dt}.
 * tb_checkpoint_load sets the state from such grid fields and the clock; the
 * taus are cleared (no later step reads them) and the multistep history
 * restarts, as the reference drops its timestepper state on load. */
tb_status tb_checkpoint_stage(tb_plan* plan, double* host_grid, size_t capacity, double* clock);
tb_status tb_checkpoint_wait(tb_plan* plan);
tb_status tb_checkpoint_load(tb_plan* plan, const double* grid, int where, const double* clock);

/* Kernel shapes of a plan (the library's own autotuning; the reference tunes
 * FFTW plans instead, transform_fourier.jl plan cache):
 *   tau_parts  row partitions of each 4-mode group's tau solves: 16 (one
 *              per half-warp, eight warps), 8 (one per half-warp, four
 *              warps) or 4 (one per warp) - partitioned, the shortest
 *              latency for one plan - or 1 (no response records, the least
 *              device work per solve); needs npad/12 >= parts;
 *   xrows      3D: padded y rows per x-pass CTA, 1, 2 or 4; 2D (Float64
 *              and mixed plans): the x-products kernel, 1 = the three
 *              gradient transforms one after another, 2 = all inverse and
 *              forward transforms of a row batched through shared passes,
 *              3 = batched and in place (decimation in frequency for the
 *              inverse, in time for the forward transforms; half the shared
 *              memory of 2).
 * 0 keeps a setting.  A change drops the plan's factors and step graphs; the
 * next step rebuilds them.  tb_plan_tune times trial_steps steps of every
 * feasible combination from the current state (the state is restored after
 * each trial and at the end) and keeps the fastest; *tau_parts / *xrows get
 * the choice.  It then times at least 10 steps with and without the step's
 * independent kernels (M X, L X, the SBDF history copies) overlapped on a
 * second stream beside the right-hand side and keeps the faster; untuned
 * plans run them in line.  Mixed plans with a tensor-core form of their
 * transform GEMMs (tb_plan_set_gemm_path) get the faster GEMM path the same
 * way. */
tb_status tb_plan_set_variant(tb_plan* plan, int tau_parts, int xrows);
tb_status tb_plan_get_variant(const tb_plan* plan, int* tau_parts, int* xrows);
tb_status tb_plan_tune(tb_plan* plan, double dt, int trial_steps, int* tau_parts, int* xrows);
/* FP32 Chebyshev transform GEMMs of a mixed-precision plan: tensor_cores = 1
 * runs them on the tcgen05 tensor cores in TF32 with three products per term
 * (FP32 accuracy), 0 on the SIMT FP32 kernel.  2D: tensor cores wherever
 * Nz <= 256 (the backward transform of even Nz on the plane form, the rest on
 * the operand-image form), SIMT by default.  3D: the streaming tensor-core
 * kernel (TMA tiles of the raw planes) wherever Nz <= 128, and there it is
 * the default; SIMT above.  tb_plan_tune picks the faster path.  No counterpart in the reference, whose GPU Chebyshev transforms
 * are cuFFT DCT-Is (ext/cuda/cheb_deriv.jl:503-596).  A change drops the
 * plan's step graphs. */
tb_status tb_plan_set_gemm_path(tb_plan* plan, int tensor_cores);
tb_status tb_plan_get_gemm_path(const tb_plan* plan, int* tensor_cores);

/* -------------------------------------------------------------------------
 * Transform backend.  Replaces Tarang._gpu_forward_transform_backend! /
 * _gpu_backward_transform_backend!(::GPU, field)
 * (src/core/transforms/transform_gpu.jl:181-205; implemented by the CUDA
 * extension at ext/cuda/transforms.jl:234-243,510 and
 * ext/cuda/mixed_transforms.jl:229-424).  Forward: grid (Nx,Nz) real ->
 * coefficients (Nx/2+1,Nz) complex: unnormalised rfft along x, DCT-I along z
 * scaled 1/(Nz-1) with halved endpoints and flipped odd degrees
 * (transform_chebyshev.jl:135-244).  Backward is the exact inverse of that
 * chain (irfft ignores Im of the DC/Nyquist bins).  Pointers are device
 * pointers.  nfields fields stored back to back.
 * ---------------------------------------------------------------------- */
tb_status tb_transform_forward(tb_plan* plan, const double* grid, double* coeff, int nfields);
tb_status tb_transform_backward(tb_plan* plan, const double* coeff, double* grid, int nfields);

/* 3/2-dealiased product of two grid fields on the plan's (Nx, Nz) grid.
 * Replaces evaluate_transform_multiply -> evaluate_padded_multiply
 * (src/core/nonlinear/nonlinear_evaluation.jl:115-213,
 * src/core/nonlinear/nonlinear_padding.jl:359-443).  Device pointers. */
tb_status tb_dealiased_multiply(tb_plan* plan, const double* a_grid, const double* b_grid, double* out_grid);

/* The same 3/2-dealiased product without a plan and without allocating any
 * device memory (no counterpart in the reference).  For callers that must not
 * let a library call cudaMalloc -- a host runtime that owns a device memory
 * pool, or a process whose device footprint is fixed after start-up.  a_grid,
 * b_grid, out_grid: the caller's device buffers, Nz rows of Nx doubles.  The
 * FFT twiddles live in a static device array of the library (80 KiB per GPU,
 * held until exit), so Nx <= 2048 (else TB_ENOTSUPPORTED).  Calls share that
 * array: calls that overlap on the GPU race.  The first call on a device
 * resolves the array's address (once per device); make it before any stream
 * capture.  Runs on the legacy default stream, which does not wait for
 * non-blocking streams (CUDA.jl task streams, torch side streams): synchronise
 * the stream that wrote a_grid and b_grid before calling.  Returns when
 * out_grid is written. */
tb_status tb_dealiased_multiply_noalloc(int device, int Nx, int Nz, const double* a_grid, const double* b_grid,
                                        double* out_grid);

/* RHS program: F = -(u.grad) f for f in (b, ux, uz), coefficient space in and
 * out.  Replaces execute_lazy_rhs_buffered! for the RBC program
 * (src/core/solvers/lazy_rhs.jl:1542-1561).  in: 3 coefficient fields
 * (b, ux, uz) back to back; out: 3 coefficient fields.  Device pointers. */
tb_status tb_rhs_advection(tb_plan* plan, const double* coeff_in, double* coeff_out);

/* -------------------------------------------------------------------------
 * Batched dense complex LU, one n x n matrix per slice.  Replaces
 * BatchedDenseLU batched_factor!/batched_solve!
 * (src/tools/batched_matsolvers.jl:57-123; CUDA getrf/getrs strided batched at
 * ext/cuda/batched_matsolvers.jl:80-125).  A: device, column-major n x n
 * complex128 per slice, overwritten by the factors; piv: device int32 n*batch.
 * On a singular slice returns TB_ESINGULAR and writes the first singular
 * slice index to *bad_slice (the reference names the mode and raises).
 * ---------------------------------------------------------------------- */
tb_status tb_batched_lu_factor(tb_context* ctx, int n, int batch, double* A, int* piv, int* bad_slice);
tb_status tb_batched_lu_solve(tb_context* ctx, int n, int batch, const double* A, const int* piv,
                              double* B /* n x batch complex, overwritten by X */);

/* -------------------------------------------------------------------------
 * Asynchronous stepping.  The reference's step!/run! (solver_stepping.jl:24-38,
 * 115-205) return when the step is done; these calls let a caller (or the
 * ensemble runner and the request server below) keep several plans in flight.
 * tb_step_async enqueues nsteps steps on the plan's stream, as CUDA graphs of
 * up to graph_steps steps each, and returns; tb_plan_query reports whether the
 * plan's stream is idle, tb_plan_wait waits for it.  tb_plan_device_bytes:
 * device memory the plan holds (state, work arrays, constants, factors).
 * ---------------------------------------------------------------------- */
tb_status tb_step_async(tb_plan* plan, double dt, int nsteps, int graph_steps);
tb_status tb_plan_query(tb_plan* plan, int* idle);
tb_status tb_plan_wait(tb_plan* plan);
tb_status tb_plan_device_bytes(const tb_plan* plan, size_t* bytes);

/* -------------------------------------------------------------------------
 * Ensembles: many independent plans (uneven sizes, own parameters and dt)
 * stepped together.  Counterpart of the reference's batched ensemble path
 * (mode_batch.jl:23-668, step_subproblem_rk_batched.jl:838-1006), which steps
 * instances in turn.  Members are borrowed plans of one context; a run steps
 * every member nsteps at its own dt (dt[i]), spreading the members' step graphs
 * over worker streams.  tb_ensemble_tune times candidate (streams, steps per
 * graph, tau-solve partitions of the members) settings on the members from a
 * snapshot of their state, restores the state and keeps the fastest setting
 * (the partitioning is applied to the member plans: tb_plan_get_variant).  member_ms[i]: time from the run's start
 * until member i finished (device clock); total_ms: the run.
 * ---------------------------------------------------------------------- */
typedef struct tb_ensemble tb_ensemble;
tb_status tb_ensemble_create(tb_context* ctx, int n, tb_plan* const* members, tb_ensemble** out);
tb_status tb_ensemble_destroy(tb_ensemble* ens);
tb_status tb_ensemble_tune(tb_ensemble* ens, const double* dt, int trial_steps, int* streams, int* graph_steps);
tb_status tb_ensemble_set_config(tb_ensemble* ens, int streams, int graph_steps);
tb_status tb_ensemble_config(const tb_ensemble* ens, int* streams, int* graph_steps);
/* Form of a run: 0 per member (each member's step graphs on worker streams),
 * 1 fused: members of one shape (Nx, Nz, domain, walls, RK222/RK443, FP64)
 * at one dt are stacked along the mode axis into one plan per shape, so each
 * kernel of a step covers the whole group in one launch (state gathered into
 * and scattered from the group plan around a run); other members step per
 * member.  tb_ensemble_tune chooses the form; groups reports the stacked plans. */
tb_status tb_ensemble_set_form(tb_ensemble* ens, int fused);
tb_status tb_ensemble_get_form(const tb_ensemble* ens, int* fused, int* groups);
tb_status tb_ensemble_run(tb_ensemble* ens, const double* dt, int nsteps, float* member_ms, float* total_ms);

/* -------------------------------------------------------------------------
 * 2D decaying turbulence, FP32.  Replaces the reference's DiagonalIMEX_SBDF2
 * step (desc->timestepper TB_SBDF2; src/core/timesteppers/
 * step_diagonal_imex.jl:329-388, 674-689) or DiagonalIMEX_RK222 / RK443 step
 * (TB_RK222 / TB_RK443; _step_diagonal_imex_rk_impl!, :183-296, with the full
 * ESDIRK tableau) for a doubly periodic RealFourier x RealFourier problem, with the
 * spectral Poisson and velocity refresh (state_utils.jl:1059-1104) and the
 * 3/2-padded products with symmetric Nyquist split/fold
 * (nonlinear_padding.jl:182-443).  q0_spec: initial vorticity coefficients,
 * complex128 (Nx/2+1, Ny), x fastest, unnormalised rfft along x and fft along
 * y (the reference's coefficient layout).  Nx, Ny even, 2^a 3^b, <= 2048.
 * ---------------------------------------------------------------------- */
typedef struct tb_turb tb_turb;
tb_status tb_turb_create(tb_context* ctx, const tb_problem_desc* desc, const double* q0_spec, tb_turb** out);
tb_status tb_turb_destroy(tb_turb* turb);
tb_status tb_turb_step(tb_turb* turb, double dt, int nsteps);
tb_status tb_turb_get_vorticity(tb_turb* turb, double* q_spec_host);

/* Doubly periodic transforms in FP64 for a PeriodicDomain (RealFourier x,
 * RealFourier y; src/extras/quick_domains.jl:33-58), the grid <-> coefficient
 * conversion of field["g"] (transform_fourier.jl:473-590): forward
 * c = fft_y(rfft_x(g)) unnormalised, backward g = irfft_x(ifft_y(c)) with
 * 1/(Nx Ny), ignoring Im of the kx = 0 and Nyquist bins.  grid (Ny, Nx) real,
 * x fastest; coeff (Ny, Nx/2+1) complex128, kx fastest, ky in FFT order.
 * where = TB_HOST or TB_DEVICE.  Nx, Ny even, 2^a 3^b, <= 2048. */
typedef struct tb_periodic tb_periodic;
tb_status tb_periodic_create(tb_context* ctx, int Nx, int Ny, tb_periodic** out);
tb_status tb_periodic_destroy(tb_periodic* p);
tb_status tb_periodic_forward(tb_periodic* p, const double* grid, double* coeff, int where);
tb_status tb_periodic_backward(tb_periodic* p, const double* coeff, double* grid, int where);
/* Replace the vorticity (same layout as tb_turb_create's q0_spec); the next
 * step starts afresh (SBDF2: with its SBDF1 step). */
tb_status tb_turb_set_vorticity(tb_turb* turb, const double* q_spec_host);

/* -------------------------------------------------------------------------
 * Request server (continuous batching).  No counterpart in the reference,
 * which runs one solver per process.  A worker thread admits requests in
 * arrival order while their estimated device bytes fit the budget and a run
 * slot is free, gives each its own plan and stream, and keeps every running
 * request's next chunk of steps in flight, so requests of different programs
 * and sizes overlap on the device and new ones join as memory frees up.
 * init_grid: RBC - the initial buoyancy on the (Nz, Nx) grid (x fastest,
 * real); TURB2D - the initial vorticity coefficients as for tb_turb_create.
 * Results: RBC fields 0..2 = b, u_x, u_z coefficients (Nx/2+1, Nz) complex128;
 * TURB2D field 0 = vorticity coefficients (Nx/2+1, Ny) complex128.
 * Time to solution = completion - submission (host clock, ms).
 * ---------------------------------------------------------------------- */
enum { TB_REQ_QUEUED = 0, TB_REQ_RUNNING = 1, TB_REQ_DONE = 2, TB_REQ_FAILED = 3 };
typedef struct tb_request {
  tb_problem_desc desc;
  double dt;
  int nsteps;
  const double* init_grid;
} tb_request;
typedef struct tb_server_stats {
  long long submitted, completed, failed, running, queued;
  double elapsed_ms;   /* first submission to last completion            */
  double solves_per_s; /* completed requests per second of elapsed time  */
  double steps_per_s;  /* completed request steps per second             */
  double p50_ms, p99_ms, mean_wait_ms;
  size_t peak_bytes, budget_bytes;
  int peak_running;
  double mean_setup_ms; /* admission to ready: plan build, factors, graph capture */
  int peak_cohort;      /* most requests that ran as one stacked plan (1: none stacked) */
  long long cohort_requests; /* requests that completed as members of a stacked run */
} tb_server_stats;
typedef struct tb_server tb_server;
tb_status tb_server_create(tb_context* ctx, size_t budget_bytes, int max_running, int chunk_steps, tb_server** out);
/* Cohorts: RBC requests of one shape (grid, box, walls, stepper, precision)
 * and one dt, with step counts within 25 % of each other, queued together
 * are admitted as one run of a stacked plan (the ensemble's fused form), up
 * to max_members (1..64; 1, the default, runs every request alone).  Each
 * member leaves the run with its result when its own step count is reached.  A member's result equals its solo run to rounding
 * (the stacked kernels sum in a different order); with max_members = 1 it is
 * bitwise the solo result. */
tb_status tb_server_set_cohort(tb_server* srv, int max_members);
tb_status tb_server_submit(tb_server* srv, const tb_request* req, long long* id);
tb_status tb_server_poll(tb_server* srv, long long id, int* state, double* tts_ms);
tb_status tb_server_result(tb_server* srv, long long id, int field, double* host_out, size_t* ndoubles);
tb_status tb_server_wait_all(tb_server* srv);
tb_status tb_server_get_stats(tb_server* srv, tb_server_stats* out);
tb_status tb_server_destroy(tb_server* srv);

#ifdef __cplusplus
}
#endif
#endif /* TARANG_B200_H */
