// Plan object of the C ABI and the internal driver entry points shared by the
// C ABI (tb_capi.cu), the ensemble runner (tb_ensemble.cu) and the request
// server (tb_server.cu).  Not part of the public interface.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "tb_internal.h"
#include "tb_kernels.cuh"

namespace tb {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  void alloc(size_t b) {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = b;
    if (b == 0) return;
    cudaError_t e = cudaMalloc(&p, b);
    if (e != cudaSuccess) {
      p = nullptr;
      throw Error{TB_ENOMEM, std::string("cudaMalloc(") + std::to_string(b) + "): " + cudaGetErrorString(e)};
    }
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Stream-ordered scratch: allocated from the device's memory pool in the order
// of one stream and released in that order, so that dropping it does not wait
// for the whole device the way cudaFree does (a request server builds plans
// while other requests' steps run).
struct StreamBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  StreamBuf() = default;
  StreamBuf(const StreamBuf&) = delete;
  StreamBuf& operator=(const StreamBuf&) = delete;
  ~StreamBuf() {
    if (p) cudaFreeAsync(p, st);
  }
  void alloc(size_t b, cudaStream_t s) {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    bytes = b;
    st = s;
    if (b == 0) return;
    cudaError_t e = cudaMallocAsync(&p, b, s);
    if (e != cudaSuccess) {
      p = nullptr;
      throw Error{TB_ENOMEM, std::string("cudaMallocAsync(") + std::to_string(b) + "): " + cudaGetErrorString(e)};
    }
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Non-owning window into a DevBuf.
struct DevView {
  void* p = nullptr;
  size_t bytes = 0;
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

template <class T>
void upload(DevBuf& d, const std::vector<T>& h) {
  d.alloc(h.size() * sizeof(T));
  if (!h.empty()) TB_CUDA_TRY(cudaMemcpy(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
}

struct ClassTables {
  DevBuf row_eq, row_k, col_unk, col_k, left_unk, left_k, bc_rhs, band, bord, c2_z, c2_nz, c1_z, c1_nz;
  DevBuf col_code, left_code;  // store targets of the band columns / border unknowns
};

struct FactorSet {
  double alpha = 0, beta = 0;
  DevBuf FR, BR, SI;  // solve-layout factor records (see tb_kernels.cuh)
  DevBuf PP;          // partition transfer matrices of the solve
  DevBuf HR;          // per-row backward responses of the partitioned solve
};

// One family of per-mode banded tau systems: the coupled Boussinesq system
// (system 0) or, in 3D, the decoupled cross-wavevector velocity (system 1).
struct TauSystem {
  TauLayout lay;
  ClassTables ct[2];
  DevBuf rhs_off;  // [row][class] right-hand-side codes
  DevBuf xcode;    // [row][class] store targets of the band columns, 16-bit (TauArgs::xcode)
  std::vector<DevBuf> mband, mbord;  // stacked instances: band / border coefficients [instance][class]
  std::vector<std::unique_ptr<FactorSet>> factors;
  int tau_parts = 1;  // partitions of the solve (kTauParts16, kTauParts8, kTauParts or 1)
  int npad = 0;       // band rows padded to a multiple of kTauRowPad
};

struct Tableau {
  int s;
  double AE[4][4], AI[4][4], bE[4], bI[4];
};

Tableau tableau(int ts);

// Host twiddle tables: exp(-2 pi i k/n), k < n (row FFT kernels), and the
// per-pass tables of a Stockham plan (CTA FFTs with per-pass twiddles).
std::vector<double2> host_twiddles(int n);
std::vector<double2> host_pass_twiddles(const FftPlan& fp);
// FFT along y of each kx column of a [y][kx] array (length Ny, in place):
// sign -1 forward (unnormalised), +1 inverse (scaled by 1/Ny).
void periodic_ycols(double2* a, int Ny, int Kx, const FftPlan& fp, const double2* ptw, int sign, cudaStream_t st);

// Graph of `steps` consecutive steps of one kind at one dt.
struct StepGraph {
  double dt = -1.0;
  int kind = -1, steps = 0;
  cudaGraphExec_t exec = nullptr;
};

}  // namespace tb

struct tb_plan {
  using DevBuf = tb::DevBuf;
  using DevView = tb::DevView;
  using ClassTables = tb::ClassTables;
  using FactorSet = tb::FactorSet;
  using TauLayout = tb::TauLayout;
  using TauSystem = tb::TauSystem;
  using FftPlan = tb::FftPlan;
  tb_context* ctx = nullptr;
  tb_problem_desc d{};
  int Nx = 0, Nz = 0, Nk = 0, M = 0;
  double k0 = 0, s = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  size_t plane = 0;  // Nz * Nk complex entries
  // 3D (ndim 3): Fourier modes m = ix * Ny + iy over Kx = Nx/2+1 x-modes and Ny
  // y-modes (ky in FFT order), Nk = Kx * Ny; the horizontal velocity is held as
  // (u_par, u_perp) along / across the wavevector (u_par in the u_x slot)
  int ndim = 2, Ny = 1, Kx = 0, My = 0;
  // stacked instances (the fused ensemble form): B plans of one shape share the
  // mode axis, instance b owning modes b Nkm .. (b+1) Nkm - 1 of Nk = B Nkm;
  // their kappa / nu per instance (B = 1: a single plan, Nkm = Nk)
  int B = 1, Nkm = 0;
  DevBuf kappa_m, nu_m;
  int nplanes = 4;  // state planes before the taus: b, u_x|u_par, u_z, p (, u_perp)
  int ntau = 7;     // tau rows
  int nf = 3;       // velocity-like fields with a time derivative
  double k0y = 0;
  // state and work arrays
  // X holds the state planes followed by the tau rows (tau views its tail),
  // so one 32-bit element offset from X addresses every unknown of the solve
  DevBuf X, G, H, MX0, FP[4], LXP[4], Fprev, MXprev, Rsb, tmpgrid;
  DevView tau;
  // 3D RHS program (element type of the RHS precision): Cartesian copy of the
  // state, Chebyshev half planes, y-transformed factors, x-pass products,
  // y-forward output, per-pass twiddles of the padded x / y plans
  DevBuf kmag, Xc, G3, mix3, pm3, H3, ptwX, ptwY;
  FftPlan fpMy{};
  // 3D field transforms and state I/O: plan and per-pass twiddles of the Ny
  // transform, one complex plane of scratch
  FftPlan fpNy{};
  DevBuf ptwNy, tmp3;
  int xrows = 1;  // padded y rows per x-pass CTA (a tuned shape)
  bool tc32 = false;  // mixed precision: FP32 transform GEMMs on the tensor cores (2D opt-in; the 3D default where supported)
  // transform constants
  DevBuf bwd, fwd, s3, twM, twN, ptwM, iptwM;
  // parity halves of the Chebyshev matrices (H = ceil(Nz/2) rows/cols)
  DevBuf bEv, bOv, bEd, bOd, fE, fO, sfE, sfO;
  int Hz = 0, Ke = 0, Ko = 0;  // Hz = ceil(Nz/2)
  FftPlan fpM{}, fpN{};
  // the padded length's passes in the order of the in-place x-products kernels
  // (x-products form 3; the order with the fewest shared-memory bank conflicts)
  FftPlan fpMip{};
  // tau systems
  TauSystem sys[2];
  int nsys = 1;
  DevBuf err_mode;
  DevBuf solve_scratch;  // y columns of one-partition tau solves (shared by the systems)
  // dynamic wall values of b (tb_set_wall_values): [bottom value, bottom rate,
  // top value, top rate][mode] on the device, and the time since they were
  // set (advanced on the device at the end of each step, so graphs replay)
  bool bc_dynamic = false;
  DevBuf bcdyn, t_dev;
  std::vector<double2> bc_host;
  double bc_tref = 0.0;
  // checkpoint staging: grid copies of the fields on the device, copied to the
  // caller's host buffer on a side stream while the plan steps on
  DevBuf stage_grid;
  cudaStream_t io_st = nullptr;
  // side stream of the step: work independent of the RHS chain (L X
  // finalisation, M X, the SBDF history copies) forks onto it and joins back
  // before its results are used, inside the captured step graphs
  cudaStream_t st2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool overlap = false;  // use the side stream (chosen by tb_plan_tune; a change drops the step graphs)
  cudaEvent_t io_ready = nullptr, io_done = nullptr;
  // stepping state
  double last_dt = 0.0;
  double sim_time = 0.0;
  long long iteration = 0;
  int ms_history = 0;  // SBDF: number of stored history levels
  double graph_dt = -1.0;
  int graph_kind = -1;
  cudaGraphExec_t gexec = nullptr;
  tb::StepGraph multi;  // graph of several steps (asynchronous / batched stepping)
  int kernels_per_step = 0;
  // mixed precision (TB_PREC_MIXED): FP32 copies for the RHS program
  bool mixed = false;
  DevBuf X32, G32, H32, bEv32, bOv32, bEd32, bOd32, fE32, fO32, sfE32, sfO32, ptwM32, iptwM32;
  // tensor-core transform GEMMs: TF32 hi/lo images of the eight matrices above
  // (empty when the shapes exceed one tensor-core tile) and the per-call
  // scratch of the B-operand images
  DevBuf tcAimg, tcBimg;
  // 3D: the streaming tensor-core form of the z transforms (A operands and
  // the tensor maps of the two input plane sets), when the shapes allow it
  bool tc3 = false;
  DevBuf tc3img;
  // 2D: the plane form's A operands (empty when the shapes do not allow it),
  // and whether its forward transform runs on it too (the C^(2) rows)
  DevBuf tc2img;
  bool tc2fwd = true;
  tb::TmaDesc tc3Xc, tc3H3;
  // profiling: eager launches bracketed by events, accumulated per kernel name
  bool profiling = false;
  struct ProfRec {
    std::string name;
    cudaEvent_t a, b;
  };
  std::vector<ProfRec> pending;
  std::vector<cudaEvent_t> event_pool;
  std::map<std::string, std::pair<double, long long>> prof;  // name -> (ms, launches)

  ~tb_plan() {
    for (auto e : event_pool) cudaEventDestroy(e);
    for (auto& r : pending) {
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    if (gexec) cudaGraphExecDestroy(gexec);
    if (multi.exec) cudaGraphExecDestroy(multi.exec);
    if (st2) {
      cudaStreamSynchronize(st2);
      cudaStreamDestroy(st2);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (io_st) {
      cudaStreamSynchronize(io_st);
      cudaStreamDestroy(io_st);
    }
    if (io_ready) cudaEventDestroy(io_ready);
    if (io_done) cudaEventDestroy(io_done);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (st) cudaStreamDestroy(st);
  }

  double2* Xp(int f) const { return X.as<double2>() + (size_t)f * plane; }
};

namespace tb {

// Build a plan (tb_plan_create) or, for B > 1, one plan of B stacked 2D
// instances of one shape (descs[0..B-1], differing only in kappa / nu).
void build_plan(tb_plan* P, tb_context* ctx, const tb_problem_desc* descs, int B);

// Device bytes the plan holds (state, work arrays, constants, factors).
size_t plan_device_bytes(const tb_plan* P);
// Kind of the next step: 0 RK, 1 SBDF1, 2 SBDF2.
int plan_next_kind(const tb_plan* P);
// Enqueue nsteps steps on stream s (the plan's own stream if s is null), using
// cached CUDA graphs of up to graph_steps steps; factors and graphs are built
// on first use of a (dt, kind).  Returns without waiting for the GPU.
void plan_launch_steps(tb_plan* P, double dt, int nsteps, cudaStream_t s, int graph_steps);
// Factors and step graphs for the next steps at dt, built ahead of the first
// launch (so that a caller can overlap this host work with other plans' steps).
void plan_prepare(tb_plan* P, double dt, int graph_steps);
// Snapshot / restore of the stepping state (X, history, counters) in device scratch.
struct PlanSnapshot {
  DevBuf X, Fprev, MXprev;
  double t_dev = 0.0;  // time of the dynamic wall values
  double sim_time = 0.0;
  long long iteration = 0;
  int ms_history = 0;
};
void plan_snapshot(tb_plan* P, PlanSnapshot* snap);
void plan_restore(tb_plan* P, const PlanSnapshot& snap);

// Profiling hook: runs fn (which enqueues one kernel) and, with profiling on,
// brackets it with events collected after the step (recorded as event nodes
// when the profiled steps are captured into a graph).
inline cudaEvent_t take_event(tb_plan* P) {
  if (!P->event_pool.empty()) {
    cudaEvent_t e = P->event_pool.back();
    P->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  TB_CUDA_TRY(cudaEventCreate(&e));
  return e;
}
template <class F>
void timed(tb_plan* P, const char* name, F&& fn) {
  if (!P->profiling) {
    fn();
    return;
  }
  cudaEvent_t a = take_event(P), b = take_event(P);
  TB_CUDA_TRY(cudaEventRecordWithFlags(a, P->st, cudaEventRecordExternal));
  fn();
  TB_CUDA_TRY(cudaEventRecordWithFlags(b, P->st, cudaEventRecordExternal));
  P->pending.push_back({name, a, b});
}

// 3D program (tb_rbc3d.cu): constants and work arrays of a new plan, the RHS
// F = -(u.grad) f for f = b, u_x, u_y, u_z written as the b, u_par, u_z, u_perp
// momentum rows (C^(2) space, 4 planes from out4), and the L delta correction
// of the stage L X for the Hermitian projection of the kx = 0 and Nyquist planes.
void rbc3d_setup(tb_plan* P);
void rbc3d_enqueue_rhs(tb_plan* P, const double2* Xin, double2* out4);
bool rbc3d_xrows_ok(const tb_plan* P, int rows);
// Tunable kernel shapes of a plan: tau-solve partitions (1, 4, 8 or 16, for
// every tau system) and, in 3D, x-pass rows per CTA (1, 2, 4).  Changing one
// drops the plan's factors and step graphs (rebuilt on the next step).
bool plan_tau_parts_ok(const tb_plan* P, int parts);
void plan_set_variant(tb_plan* P, int tau_parts, int xrows);
void rbc3d_lx_project(tb_plan* P, double2* LX, double beta, cudaStream_t st = nullptr);  // null: the plan's stream
void rbc3d_mx_project(tb_plan* P, double2* MX, cudaStream_t st = nullptr);
size_t rbc3d_device_bytes(const tb_plan* P);
// 3D transforms between grid (Nz, Ny, Nx) real and coefficients (Nz, Ny, Nx/2+1)
// complex (kx fastest), device pointers, one field.
void rbc3d_transform_forward(tb_plan* P, const double* grid, double2* coeff);
void rbc3d_transform_backward(tb_plan* P, const double2* coeff, double* grid);
// State I/O between the public layout (device pointer) and the plan's planes:
// field TB_FIELD_* (Cartesian velocity), or the 9 taus.
void rbc3d_state_get(tb_plan* P, int field, double2* dst);
void rbc3d_state_set(tb_plan* P, int field, const double2* src);

// Error plumbing shared by the C ABI translation units.
void record_error(tb_context* ctx, const Error& e);
template <class F>
tb_status guarded(tb_context* ctx, F&& fn) {
  try {
    fn();
    return TB_OK;
  } catch (const Error& e) {
    record_error(ctx, e);
    return e.code;
  } catch (const std::bad_alloc&) {
    record_error(ctx, Error{TB_ENOMEM, "host allocation failed"});
    return TB_ENOMEM;
  } catch (...) {
    record_error(ctx, Error{TB_EINVAL, "unexpected internal error"});
    return TB_EINVAL;
  }
}

}  // namespace tb
