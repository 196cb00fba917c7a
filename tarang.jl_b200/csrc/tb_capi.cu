// C ABI of libtarang_b200: contexts, plans, state I/O and the timestep driver.
//
// The driver mirrors the reference's step loop for a GPU plan:
//   RK222 / RK443 : step_subproblem_rk!          (step_subproblem_rk.jl:393-739)
//   SBDF1 / SBDF2 : step_subproblem_multistep!   (step_subproblem_multistep.jl:197-405),
//                   SBDF2 starting with one SBDF1 step (step_multistep.jl:341-356)
// One step is captured once per dt as a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>

#include "tb_internal.h"
#include "tb_kernels.cuh"
#include "tb_plan.h"

using namespace tb;

namespace tb {
Tableau tableau(int ts) {
  Tableau t{};
  if (ts == TB_RK222) {
    const double g = 1.0 - 1.0 / std::sqrt(2.0);
    t.s = 3;
    double AE[3][3] = {{0, 0, 0}, {g, 0, 0}, {g, 1 - g, 0}};
    double AI[3][3] = {{0, 0, 0}, {0, g, 0}, {0, 1 - g, g}};
    double b[3] = {0, 1 - g, g};
    for (int i = 0; i < 3; ++i) {
      t.bE[i] = b[i];
      t.bI[i] = b[i];
      for (int j = 0; j < 3; ++j) {
        t.AE[i][j] = AE[i][j];
        t.AI[i][j] = AI[i][j];
      }
    }
  } else {
    const double g = 0.4358665215084590;
    t.s = 4;
    double AE[4][4] = {{0, 0, 0, 0},
                       {0.4358665215084590, 0, 0, 0},
                       {0.3212788860285571, 0.3966543747256624, 0, 0},
                       {-0.105858296071263, 0.5529291479590279, 0.5529291481122351, 0}};
    double AI[4][4] = {{0, 0, 0, 0}, {0, g, 0, 0}, {0, 0.2820667392457805, g, 0},
                       {0, 1.208496649176010, -0.6443631706844688, g}};
    double bE[4] = {0.0, 1.208496649176010, -0.6443631706844688, 0.4358665215084590};
    double bI[4] = {0.0, 1.208496649176010, -0.6443631706844688, g};
    for (int i = 0; i < 4; ++i) {
      t.bE[i] = bE[i];
      t.bI[i] = bI[i];
      for (int j = 0; j < 4; ++j) {
        t.AE[i][j] = AE[i][j];
        t.AI[i][j] = AI[i][j];
      }
    }
  }
  return t;
}

}  // namespace tb


namespace {

thread_local std::string g_err;

}  // namespace

void tb::set_thread_error(const std::string& msg) { g_err = msg; }
void tb::set_context_error(tb_context* ctx, const std::string& msg) {
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->last_error = msg;
}

namespace {

tb_status fail(tb_context* ctx, const Error& e) {
  if (ctx) set_context_error(ctx, e.msg);
  g_err = e.msg;
  return e.code;
}

}  // namespace

void tb::record_error(tb_context* ctx, const Error& e) { fail(ctx, e); }

namespace {

template <class F>
tb_status guard(tb_context* ctx, F&& fn) {
  try {
    fn();
    return TB_OK;
  } catch (const Error& e) {
    return fail(ctx, e);
  } catch (const std::bad_alloc&) {
    return fail(ctx, Error{TB_ENOMEM, "host allocation failed"});
  } catch (...) {
    return fail(ctx, Error{TB_EINVAL, "unexpected internal error"});
  }
}

void check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw Error{TB_ECUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

void collect_profile(tb_plan* P) {
  TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  for (auto& r : P->pending) {
    float ms = 0.f;
    TB_CUDA_TRY(cudaEventElapsedTime(&ms, r.a, r.b));
    auto& acc = P->prof[r.name];
    acc.first += ms;
    acc.second += 1;
    P->event_pool.push_back(r.a);
    P->event_pool.push_back(r.b);
  }
  P->pending.clear();
}

inline int pad16k(int k) { return (k + 15) / 16 * 16; }

// Per-pass twiddle tables of a Stockham plan: pass s (stride Ns, radix R)
// contributes exp(-2 pi i j n/(Ns R) / n) for j < Ns, passes concatenated.
std::vector<double2> pass_twiddles(const FftPlan& fp) {
  std::vector<double2> t;
  const long double pi = 3.141592653589793238462643383279502884L;
  int Ns = 1;
  for (int s = 0; s < fp.nstages; ++s) {
    const int R = fp.radix[s];
    const int tstride = fp.n / (Ns * R);
    for (int j = 0; j < Ns; ++j) {
      long double a = -2.0L * pi * (long double)(j * tstride) / (long double)fp.n;
      t.push_back(make_double2((double)cosl(a), (double)sinl(a)));
    }
    Ns *= R;
  }
  return t;
}

// In-place (DIF/DIT) twiddles: per pass s, exp(-2 pi i j / L_s) for j < L_s / R_s,
// L_s = n / (R_0 ... R_{s-1}) (the layout fftg::fft_ip_dif / fft_ip_dit read)
std::vector<double2> ip_twiddles(const FftPlan& fp) {
  std::vector<double2> t;
  const long double pi = 3.141592653589793238462643383279502884L;
  int L = fp.n;
  for (int s = 0; s < fp.nstages; ++s) {
    const int m = L / fp.radix[s];
    for (int j = 0; j < m; ++j) {
      const long double a = -2.0L * pi * (long double)j / (long double)L;
      t.push_back(make_double2((double)cosl(a), (double)sinl(a)));
    }
    L = m;
  }
  return t;
}

// Shared-memory wavefronts of the in-place passes of plan fp (fftg::pass_ip:
// item = thread + k * blockDim over NA arrays Ms = n apart, a warp = 32
// consecutive items, lane element base + r m at the XOR-swizzled index
// fidx), summed over the DIF inverse (4 arrays) and DIT forward (2 arrays)
// transforms of the x-products kernel.  Elements of esz bytes: 16 (double2,
// four 8-lane phases over 8 bank quads) or 8 (float2, two 16-lane phases
// over 16 bank pairs); a phase costs as many wavefronts as the most distinct
// addresses on one bank group.
long long ip_wavefronts(const FftPlan& fp, int esz) {
  const int n = fp.n, lanes = esz == 16 ? 8 : 16, banks = esz == 16 ? 8 : 16;
  auto swz = [](int i) { return i ^ ((i >> 3) & 7); };
  long long wf = 0;
  for (int t = 0; t < 2; ++t) {
    const int NA = t == 0 ? 4 : 2;
    int L = n;
    for (int s = 0; s < fp.nstages; ++s) {
      const int R = fp.radix[s], m = L / R, nb = n / R, total = NA * nb;
      for (int w0 = 0; w0 < total; w0 += 32)
        for (int r = 0; r < R; ++r)
          for (int ph = w0; ph < w0 + 32 && ph < total; ph += lanes) {
            std::vector<std::vector<int>> grp(banks);
            int worst = 0;
            for (int item = ph; item < ph + lanes && item < total; ++item) {
              const int arr = item / nb, b = item - arr * nb, base = (b / m) * L + b % m;
              const int addr = arr * n + swz(base + r * m);
              auto& g = grp[addr % banks];
              if (std::find(g.begin(), g.end(), addr) == g.end()) g.push_back(addr);
              worst = std::max(worst, (int)g.size());
            }
            wf += worst;
          }
      L = m;
    }
  }
  return wf;
}

// The order of fp's passes with the fewest in-place wavefronts (ties keep the
// earlier order in lexicographic sequence, starting from fp's own).
FftPlan best_ip_order(const FftPlan& fp, int esz) {
  FftPlan best = fp, cand = fp;
  long long bw = ip_wavefronts(fp, esz);
  std::sort(cand.radix, cand.radix + cand.nstages);
  do {
    const long long w = ip_wavefronts(cand, esz);
    if (w < bw) {
      bw = w;
      best = cand;
    }
  } while (std::next_permutation(cand.radix, cand.radix + cand.nstages));
  return best;
}

std::vector<double2> twiddles(int n) {
  std::vector<double2> t(n);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int k = 0; k < n; ++k) {
    long double a = -2.0L * pi * (long double)k / (long double)n;
    t[k] = make_double2((double)cosl(a), (double)sinl(a));
  }
  return t;
}

ClassDev class_dev(tb_plan* P, int sy, int c, FactorSet* f) {
  ClassDev cd{};
  const ClassLayout& L = P->sys[sy].lay.cls[c];
  ClassTables& T = P->sys[sy].ct[c];
  cd.n = L.n;
  cd.nb = L.nb;
  cd.kl = L.kl;
  cd.ku = L.ku;
  cd.row_eq = T.row_eq.as<short>();
  cd.row_k = T.row_k.as<short>();
  cd.col_unk = T.col_unk.as<short>();
  cd.col_k = T.col_k.as<short>();
  cd.left_unk = T.left_unk.as<short>();
  cd.left_k = T.left_k.as<short>();
  cd.bc_rhs = T.bc_rhs.as<double>();
  cd.band = T.band.as<Coef>();
  cd.bord = T.bord.as<Coef>();
  cd.c2_z = T.c2_z.as<double>();
  cd.c2_nz = T.c2_nz.as<double>();
  cd.c1_z = T.c1_z.as<double>();
  cd.c1_nz = T.c1_nz.as<double>();
  cd.col_code = T.col_code.as<int>();
  cd.left_code = T.left_code.as<int>();
  if (f) {
    cd.FR = f->FR.as<double>();
    cd.BR = f->BR.as<double>();
    cd.SI = f->SI.as<double>();
  }
  return cd;
}

TauArgs tau_args(tb_plan* P, int sy, FactorSet* f, const double2* rhsP) {
  TauArgs a{};
  a.cls[0] = class_dev(P, sy, 0, f);
  a.cls[1] = class_dev(P, sy, 1, f);
  a.Nz = P->Nz;
  a.Nk = P->Nk;
  a.Nx = P->Nx;
  a.k0 = P->k0;
  a.kmag = P->kmag.as<double>();
  a.alpha = f ? f->alpha : 0.0;
  a.beta = f ? f->beta : 0.0;
  a.X = P->X.as<double2>();
  a.tau = P->tau.as<double2>();
  a.rhsP = rhsP;
  a.npad = P->sys[sy].npad;
  a.PP = f ? f->PP.as<double>() : nullptr;
  a.HR = f ? f->HR.as<double>() : nullptr;
  a.rhs_off = P->sys[sy].rhs_off.as<int>();
  a.xcode = P->sys[sy].xcode.as<short>();
  a.err_mode = P->err_mode.as<int>();
  a.ysave = P->solve_scratch.as<double>();
  a.Nkm = P->Nkm;
  a.mode0 = 0;
  return a;
}

void drop_graph(tb_plan* P);

// Destroys both cached step graphs (the single-step one and the multi-step
// one); the next launch recaptures.  A graph still executing is released by
// CUDA when it completes.
void drop_step_graphs(tb_plan* P) {
  drop_graph(P);
  if (P->multi.exec) cudaGraphExecDestroy(P->multi.exec);
  P->multi = StepGraph{};
}

FactorSet* get_factors(tb_plan* P, int sy, double alpha, double beta) {
  TauSystem& S = P->sys[sy];
  for (auto& f : S.factors)
    if (f->alpha == alpha && f->beta == beta) return f.get();
  // keep at most two sets (SBDF needs the SBDF1 and SBDF2 left-hand sides);
  // a new (alpha, beta) takes over the oldest set's device buffers, so a dt
  // change frees and allocates nothing (cudaFree would wait for the whole
  // device).  A captured graph bakes in the device pointers of the set it was
  // captured against, and its cache key (dt, kind, steps) cannot tell that
  // those buffers now hold another dt's factors, so every cached step graph
  // is dropped here and the caller recaptures before its next launch.
  std::unique_ptr<FactorSet> fs;
  if (S.factors.size() >= 2) {
    fs = std::move(S.factors.front());
    S.factors.erase(S.factors.begin());
    drop_step_graphs(P);
  } else {
    fs = std::make_unique<FactorSet>();
  }
  fs->alpha = alpha;
  fs->beta = beta;
  const int Nk = P->Nk;
  const size_t groups = (size_t)(Nk + kSolveModes - 1) / kSolveModes;
  const size_t n = S.npad;
  auto fit = [](DevBuf& b, size_t bytes) {
    if (b.bytes != bytes) b.alloc(bytes);
  };
  fit(fs->FR, groups * n * 2 * kFwdRec * kSolveModes * sizeof(double));
  fit(fs->BR, groups * n * 2 * kBwdRec * kSolveModes * sizeof(double));
  fit(fs->SI, groups * 2 * 16 * kSolveModes * sizeof(double));
  fit(fs->PP, tau_transfer_doubles(Nk, S.tau_parts) * sizeof(double));
  fit(fs->HR, tau_response_doubles(Nk, (int)n, S.tau_parts) * sizeof(double));
  TB_CUDA_TRY(cudaMemsetAsync(fs->FR.p, 0, fs->FR.bytes, P->st));
  TB_CUDA_TRY(cudaMemsetAsync(fs->BR.p, 0, fs->BR.bytes, P->st));
  TB_CUDA_TRY(cudaMemsetAsync(fs->SI.p, 0, fs->SI.bytes, P->st));
  int neg = 0x7fffffff;
  TB_CUDA_TRY(cudaMemcpyAsync(P->err_mode.p, &neg, sizeof(int), cudaMemcpyHostToDevice, P->st));
  TauArgs a = tau_args(P, sy, fs.get(), nullptr);
  for (int b = 0; b < P->B; ++b) {  // one factor launch per stacked instance (its own kappa, nu)
    TauArgs ab = a;
    ab.mode0 = b * P->Nkm;
    if (P->B > 1)
      for (int c = 0; c < 2; ++c) {
        ab.cls[c].band = S.mband[2 * b + c].as<Coef>();
        ab.cls[c].bord = S.mbord[2 * b + c].as<Coef>();
      }
    launch_tau_factor(ab, S.tau_parts, P->st);
  }
  launch_tau_transfer(a, S.tau_parts, P->st);
  check_launch("tau factor");
  int bad = 0;
  TB_CUDA_TRY(cudaMemcpyAsync(&bad, P->err_mode.p, sizeof(int), cudaMemcpyDeviceToHost, P->st));
  TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  if (bad != neg) {
    std::string where = P->ndim == 3 ? " (kx index " + std::to_string(bad / P->Ny) + ", ky index " +
                                           std::to_string(bad % P->Ny) + ")"
                                     : " (kx = " + std::to_string(bad * P->k0) + ")";
    throw Error{TB_ESINGULAR, "singular tau system at Fourier mode " + std::to_string(bad) + where};
  }
  S.factors.push_back(std::move(fs));
  return S.factors.back().get();
}

// F = -(u.grad) f in C^(2) rows (sfwd) or T coefficients (fwd) for f = b, ux, uz.
// TF32 operand image of the mixed plan's transform matrix m (0..3 backward
// even/odd values and derivatives, 4/5 forward to T rows, 6/7 forward to
// C^(2) rows), or null when the plan has none (shapes past the tensor-core tile)
const float* tc32_image(const tb_plan* P, int m) {
  if (P->tcAimg.bytes < (size_t)(m + 1) * tc32_a_image_floats() * sizeof(float)) return nullptr;
  return P->tcAimg.as<float>() + (size_t)m * tc32_a_image_floats();
}

// Mixed 2D plans: the stage solves also write the FP32 copy of the b, u_x,
// u_z planes that the next right-hand side reads (its rounding pass skipped).
void set_x32(const tb_plan* P, TauArgs* a) {
  if (P->mixed && P->ndim == 2) {
    a->X32 = P->X32.as<float>();
    a->x32_lim = 3LL * (long long)P->plane * 2;
  }
}

// Mixed precision: the same RHS program on FP32 data; F is written in FP64.
void enqueue_rhs_mixed(tb_plan* P, const double2* Xin, double2* out3, bool c2rows, bool x32_fresh) {
  const int N = P->Nz, H = P->Hz;
  const int ncol = 2 * P->Nk;
  const size_t hplane = (size_t)H * P->Nk;
  float2* X32 = P->X32.as<float2>();
  float2* G = P->G32.as<float2>();
  auto gp = [&](int f, int w) { return G + (size_t)(4 * f + w) * hplane; };
  if (!x32_fresh) timed(P, "round_f32", [&] { launch_round_f32(Xin, X32, 3LL * (long long)P->plane, P->st); });
  GemmBatch32 bt{};
  int nb = 0;
  for (int f = 0; f < 3; ++f) {
    const float* in = reinterpret_cast<const float*>(X32 + (size_t)f * P->plane);
    const float* Am[4] = {P->bEv32.as<float>(), P->bOv32.as<float>(), P->bEd32.as<float>(), P->bOd32.as<float>()};
    for (int w = 0; w < 4; ++w) {
      bt.item[nb] = GemmItem32{Am[w], in, gp(f, w), H, (w & 1) ? P->Ko : P->Ke, pad16k((w & 1) ? P->Ko : P->Ke),
                               GEMM_PARITY, w & 1};
      bt.item[nb++].Aimg = tc32_image(P, w);
    }
  }
  float* bsc = P->tcBimg.as<float>();
  const size_t bscn = P->tcBimg.bytes / sizeof(float);
  // tensor cores: the plane form where its A operands exist (the C^(2) rows
  // of the step; the plain forward rows keep the image form)
  const bool plane = P->tc32 && P->tc2img.p != nullptr;
  if (plane)
    timed(P, "z_backward_gemm", [&] {
      launch_tc32p(true, reinterpret_cast<const float*>(X32), P->tc2img.as<float>(), G, 3, N, ncol, P->st);
    });
  else
    timed(P, "z_backward_gemm",
          [&] { launch_gemm_f32_path(bt, nb, ncol, ncol, ncol, N, false, P->st, P->tc32, bsc, bscn); });
  XProdArgs32 xa{};
  for (int f = 0; f < 3; ++f) {
    xa.ev[f] = gp(f, 0);
    xa.ov[f] = gp(f, 1);
    xa.ed[f] = gp(f, 2);
    xa.od[f] = gp(f, 3);
    xa.out[f] = P->H32.as<float2>() + (size_t)f * P->plane;
  }
  xa.ptw = P->ptwM32.as<float2>();
  xa.nptw = (int)(P->ptwM32.bytes / sizeof(float2));
  xa.fp = P->xrows == 3 ? P->fpMip : P->fpM;  // the in-place kernels run their own pass order
  xa.Nx = P->Nx;
  xa.Nk = P->Nkm;
  xa.ld = P->Nk;
  xa.instances = P->B;
  xa.M = P->M;
  xa.Nz = N;
  xa.k0 = (float)P->k0;
  xa.iptw = P->iptwM32.as<float2>();
  xa.niptw = (int)(P->iptwM32.bytes / sizeof(float2));
  timed(P, "x_fft_products", [&] {
    if (P->xrows == 3)
      launch_xprod32_ip(xa, P->st);  // transforms in place (DIF / DIT)
    else if (P->xrows == 2)
      launch_xprod32_b(xa, P->st);  // transforms batched through shared passes
    else
      launch_xprod32(xa, P->st);
  });
  GemmBatch32 bf{};
  nb = 0;
  for (int f = 0; f < 3; ++f) {
    const float* in = reinterpret_cast<const float*>(P->H32.as<float2>() + (size_t)f * P->plane);
    double* out = reinterpret_cast<double*>(out3 + (size_t)f * P->plane);
    bf.item[nb] = GemmItem32{c2rows ? P->sfE32.as<float>() : P->fE32.as<float>(), in, out, P->Ke, H, pad16k(H),
                             GEMM_MIRROR, 0};
    bf.item[nb++].Aimg = tc32_image(P, c2rows ? 6 : 4);
    if (P->Ko > 0) {
      bf.item[nb] = GemmItem32{c2rows ? P->sfO32.as<float>() : P->fO32.as<float>(), in, out, P->Ko, H, pad16k(H),
                               GEMM_MIRROR, 1};
      bf.item[nb++].Aimg = tc32_image(P, c2rows ? 7 : 5);
    }
  }
  if (plane && c2rows && P->tc2fwd)
    timed(P, "z_forward_gemm", [&] {
      launch_tc32p(false, reinterpret_cast<const float*>(P->H32.as<float2>()), P->tc2img.as<float>(), out3, 3, N,
                   ncol, P->st);
    });
  else
    timed(P, "z_forward_gemm",
          [&] { launch_gemm_f32_path(bf, nb, ncol, ncol, ncol, N, true, P->st, P->tc32, bsc, bscn); });
}

// x32_fresh: the FP32 copy of Xin's planes is current (written by the solve
// that produced Xin), so the mixed program skips its rounding pass.
void enqueue_rhs(tb_plan* P, const double2* Xin, double2* out3, bool c2rows, bool x32_fresh = false) {
  if (P->mixed) {
    enqueue_rhs_mixed(P, Xin, out3, c2rows, x32_fresh);
    return;
  }
  const int N = P->Nz, H = P->Hz;
  const int ncol = 2 * P->Nk;
  const size_t hplane = (size_t)H * P->Nk;
  double2* G = P->G.as<double2>();
  auto gp = [&](int f, int w) { return G + (size_t)(4 * f + w) * hplane; };  // w: 0 ev, 1 ov, 2 ed, 3 od
  GemmBatch bt{};
  int nb = 0;
  for (int f = 0; f < 3; ++f) {
    const double* in = reinterpret_cast<const double*>(Xin + (size_t)f * P->plane);
    const double* Am[4] = {P->bEv.as<double>(), P->bOv.as<double>(), P->bEd.as<double>(), P->bOd.as<double>()};
    for (int w = 0; w < 4; ++w)
      bt.item[nb++] = GemmItem{Am[w], in, reinterpret_cast<double*>(gp(f, w)), H, (w & 1) ? P->Ko : P->Ke,
                               pad16k((w & 1) ? P->Ko : P->Ke), GEMM_PARITY, w & 1};
  }
  timed(P, "z_backward_gemm", [&] { launch_gemm_f64(bt, nb, ncol, ncol, ncol, N, P->st); });
  XProdArgs xa{};
  for (int f = 0; f < 3; ++f) {
    xa.ev[f] = gp(f, 0);
    xa.ov[f] = gp(f, 1);
    xa.ed[f] = gp(f, 2);
    xa.od[f] = gp(f, 3);
    xa.out[f] = P->H.as<double2>() + (size_t)f * P->plane;
  }
  xa.ptw = P->ptwM.as<double2>();
  xa.nptw = (int)(P->ptwM.bytes / sizeof(double2));
  xa.fp = P->xrows == 3 ? P->fpMip : P->fpM;  // the in-place kernels run their own pass order
  xa.Nx = P->Nx;
  xa.Nk = P->Nkm;
  xa.ld = P->Nk;
  xa.instances = P->B;
  xa.M = P->M;
  xa.Nz = N;
  xa.k0 = P->k0;
  xa.iptw = P->iptwM.as<double2>();
  xa.niptw = (int)(P->iptwM.bytes / sizeof(double2));
  timed(P, "x_fft_products", [&] {
    if (P->xrows == 3)
      launch_xprod_ip(xa, P->st);  // transforms in place (DIF / DIT)
    else if (P->xrows == 2)
      launch_xprod_b(xa, P->st);  // transforms batched through shared passes
    else
      launch_xprod(xa, P->st);
  });
  GemmBatch bf{};
  nb = 0;
  for (int f = 0; f < 3; ++f) {
    const double* in = reinterpret_cast<const double*>(P->H.as<double2>() + (size_t)f * P->plane);
    double* out = reinterpret_cast<double*>(out3 + (size_t)f * P->plane);
    bf.item[nb++] = GemmItem{c2rows ? P->sfE.as<double>() : P->fE.as<double>(), in, out, P->Ke, H, pad16k(H), GEMM_MIRROR, 0};
    if (P->Ko > 0)
      bf.item[nb++] =
          GemmItem{c2rows ? P->sfO.as<double>() : P->fO.as<double>(), in, out, P->Ko, H, pad16k(H), GEMM_MIRROR, 1};
  }
  timed(P, "z_forward_gemm", [&] { launch_gemm_f64(bf, nb, ncol, ncol, ncol, N, P->st); });
}

// The side stream: side(P) is the stream for work forked off the step's main
// chain when the plan overlaps (the plan's own stream otherwise, and when
// profiling, so that every kernel's events bracket it alone); fork_side
// orders it after everything enqueued so far, join_side makes the main stream
// wait for it.  Whether overlapping pays depends on the size: the small
// latency-bound steps gain, the large ones lose a little to the concurrent
// kernel, so tb_plan_tune decides.
bool use_side(const tb_plan* P) { return P->overlap && !P->profiling; }
cudaStream_t side(const tb_plan* P) { return use_side(P) ? P->st2 : P->st; }
void fork_side(tb_plan* P) {
  if (!use_side(P)) return;
  TB_CUDA_TRY(cudaEventRecord(P->ev_fork, P->st));
  TB_CUDA_TRY(cudaStreamWaitEvent(P->st2, P->ev_fork, 0));
}
void join_side(tb_plan* P) {
  if (!use_side(P)) return;
  TB_CUDA_TRY(cudaEventRecord(P->ev_join, P->st2));
  TB_CUDA_TRY(cudaStreamWaitEvent(P->st, P->ev_join, 0));
}

void enqueue_rk_step(tb_plan* P, double dt) {
  const Tableau T = tableau(P->d.timestepper);
  const double gamma = T.AI[1][1];
  const double beta = dt * gamma;
  FactorSet* fs = get_factors(P, 0, 1.0, beta);  // done before capture by the caller
  FactorSet* fs2 = P->nsys > 1 ? get_factors(P, 1, 1.0, beta) : nullptr;
  const long long cnt = (long long)P->nplanes * (long long)P->plane;
  double2* X = P->X.as<double2>();
  const bool d3 = P->ndim == 3;
  // M X_0 on the side stream, beside the first right-hand side
  fork_side(P);
  timed(P, "mass_apply", [&] {
    launch_mass_apply(X, P->MX0.as<double2>(), P->s3.as<double>(), P->Nz, P->Nk, P->Nx, 0, P->nf, side(P), P->Nkm);
  });
  int nk = 1;
  for (int i = 0; i < T.s; ++i) {
    if (i > 0) {
      LinComb lc{};
      lc.in[lc.n] = P->MX0.as<double2>();
      lc.w[lc.n++] = 1.0;
      for (int j = 0; j < i; ++j) {
        if (std::fabs(dt * T.AE[i][j]) > 1e-14) {
          lc.in[lc.n] = P->FP[j].as<double2>();
          lc.w[lc.n++] = dt * T.AE[i][j];
        }
        if (std::fabs(dt * T.AI[i][j]) > 1e-14) {
          lc.in[lc.n] = P->LXP[j].as<double2>();
          lc.w[lc.n++] = -dt * T.AI[i][j];
        }
      }
      timed(P, "stage_lincomb", [&] { launch_lincomb(lc, P->LXP[i].as<double2>(), cnt, P->st); });
      TauArgs a = tau_args(P, 0, fs, P->LXP[i].as<double2>());
      set_x32(P, &a);
      if (P->bc_dynamic) {  // wall values at the stage time t_n + c_i dt
        double ci = 0.0;
        for (int j = 0; j < i; ++j) ci += T.AE[i][j];
        a.bcdyn = P->bcdyn.as<double2>();
        a.t_dev = P->t_dev.as<double>();
        a.bc_toff = ci * dt;
      }
      timed(P, "tau_solve", [&] { launch_tau_solve(a, P->sys[0].tau_parts, P->st); });
      if (fs2) {
        TauArgs a2 = tau_args(P, 1, fs2, P->LXP[i].as<double2>());
        timed(P, "tau_solve_perp", [&] { launch_tau_solve(a2, P->sys[1].tau_parts, P->st); });
        ++nk;
      }
      // L X_i = (rhs - M X_i) / beta on the side stream, beside F(X_i)
      fork_side(P);
      timed(P, "lx_finalize", [&] {
        launch_lx_finalize(P->LXP[i].as<double2>(), X, P->s3.as<double>(), P->Nz, P->Nk, d3 ? 0 : P->Nx, P->k0, P->s,
                           P->d.kappa, P->d.nu, beta, P->nf, side(P), P->Nkm, P->kappa_m.as<double>(),
                           P->nu_m.as<double>());
      });
      nk += 3;
      if (d3) {
        rbc3d_lx_project(P, P->LXP[i].as<double2>(), beta, side(P));
        ++nk;
      }
    }
    if (d3) {
      rbc3d_enqueue_rhs(P, X, P->FP[i].as<double2>() + P->plane);
      nk += P->mixed ? 6 : 5;
    } else {
      // the stage solve (i > 0) has written the FP32 copy of X_i
      enqueue_rhs(P, X, P->FP[i].as<double2>() + P->plane, true, i > 0);
      nk += P->mixed && i == 0 ? 4 : 3;
    }
    join_side(P);  // M X_0 or L X_i is in place before the next combination
  }
  LinComb lc{};
  lc.in[lc.n] = P->MX0.as<double2>();
  lc.w[lc.n++] = 1.0;
  for (int j = 0; j < T.s; ++j) {
    if (std::fabs(dt * T.bE[j]) > 1e-14) {
      lc.in[lc.n] = P->FP[j].as<double2>();
      lc.w[lc.n++] = dt * T.bE[j];
    }
    if (std::fabs(dt * T.bI[j]) > 1e-14) {
      lc.in[lc.n] = P->LXP[j].as<double2>();
      lc.w[lc.n++] = -dt * T.bI[j];
    }
  }
  timed(P, "rk_final", [&] {
    launch_rk_final(lc, X, P->tau.as<double2>(), P->s3.as<double>(), P->Nz, P->Nk, P->nf, P->ntau, P->st);
  });
  nk += 1;
  if (P->bc_dynamic) {
    launch_advance_time(P->t_dev.as<double>(), dt, P->st);
    nk += 1;
  }
  P->kernels_per_step = nk;
}

// SBDF1/SBDF2 coefficients for constant dt (step_subproblem_multistep.jl:536-553).
struct SbdfCoefs {
  double a0, a1, a2, c1, c2;
};
SbdfCoefs sbdf_coefs(int order, double dt) {
  SbdfCoefs k{};
  if (order == 1) {
    k.a0 = 1.0 / dt;
    k.a1 = -1.0 / dt;
    k.c1 = 1.0;
  } else {
    const double w1 = 1.0;
    k.a0 = (1.0 + 2.0 * w1) / ((1.0 + w1) * dt);
    k.a1 = -(1.0 + w1) / dt;
    k.a2 = w1 * w1 / ((1.0 + w1) * dt);
    k.c1 = 1.0 + w1;
    k.c2 = -w1;
  }
  return k;
}

// One SBDF step of the given order (1 or 2); history of (F, MX) in Fprev/MXprev.
void enqueue_sbdf_step(tb_plan* P, double dt, int order) {
  const SbdfCoefs K = sbdf_coefs(order, dt);
  const double a0 = K.a0, a1 = K.a1, a2 = K.a2, c1 = K.c1, c2 = K.c2;
  FactorSet* fs = get_factors(P, 0, a0, 1.0);
  FactorSet* fs2 = P->nsys > 1 ? get_factors(P, 1, a0, 1.0) : nullptr;
  const long long cnt = (long long)P->nplanes * (long long)P->plane;
  double2* X = P->X.as<double2>();
  double2* Fcur = P->FP[0].as<double2>();
  double2* MXcur = P->MX0.as<double2>();
  const bool d3 = P->ndim == 3;
  int extra = 0;
  // M X of the projected fields (2D drops Im at the DC / Nyquist modes; 3D
  // subtracts M delta on the kx = 0 / Nyquist planes) on the side stream,
  // beside the right-hand side
  fork_side(P);
  timed(P, "mass_apply", [&] {
    launch_mass_apply(X, MXcur, P->s3.as<double>(), P->Nz, P->Nk, P->Nx, d3 ? 0 : 1, P->nf, side(P), P->Nkm);
  });
  if (d3) {
    rbc3d_mx_project(P, MXcur, side(P));
    ++extra;
  }
  if (d3)
    rbc3d_enqueue_rhs(P, X, Fcur + P->plane);
  else
    enqueue_rhs(P, X, Fcur + P->plane, true);
  join_side(P);
  LinComb lc{};
  lc.in[lc.n] = Fcur;
  lc.w[lc.n++] = c1;
  lc.in[lc.n] = MXcur;
  lc.w[lc.n++] = -a1;
  if (order == 2) {
    lc.in[lc.n] = P->Fprev.as<double2>();
    lc.w[lc.n++] = c2;
    lc.in[lc.n] = P->MXprev.as<double2>();
    lc.w[lc.n++] = -a2;
  }
  timed(P, "stage_lincomb", [&] { launch_lincomb(lc, P->Rsb.as<double2>(), cnt, P->st); });
  // the history for the next step (read by the combination above) is copied
  // on the side stream while the tau systems are solved
  fork_side(P);
  TB_CUDA_TRY(cudaMemcpyAsync(P->Fprev.p, Fcur, sizeof(double2) * cnt, cudaMemcpyDeviceToDevice, side(P)));
  TB_CUDA_TRY(cudaMemcpyAsync(P->MXprev.p, MXcur, sizeof(double2) * cnt, cudaMemcpyDeviceToDevice, side(P)));
  TauArgs a = tau_args(P, 0, fs, P->Rsb.as<double2>());
  if (P->bc_dynamic) {  // wall values at t_{n+1}
    a.bcdyn = P->bcdyn.as<double2>();
    a.t_dev = P->t_dev.as<double>();
    a.bc_toff = dt;
  }
  timed(P, "tau_solve", [&] { launch_tau_solve(a, P->sys[0].tau_parts, P->st); });
  if (fs2) {
    TauArgs a2 = tau_args(P, 1, fs2, P->Rsb.as<double2>());
    timed(P, "tau_solve_perp", [&] { launch_tau_solve(a2, P->sys[1].tau_parts, P->st); });
    ++extra;
  }
  join_side(P);
  P->kernels_per_step = (d3 ? (P->mixed ? 6 : 5) : (P->mixed ? 4 : 3)) + 1 + 1 + 1 + extra;
  if (P->bc_dynamic) {
    launch_advance_time(P->t_dev.as<double>(), dt, P->st);
    P->kernels_per_step += 1;
  }
}

void drop_graph(tb_plan* P) {
  if (P->gexec) cudaGraphExecDestroy(P->gexec);
  P->gexec = nullptr;
  P->graph_dt = -1.0;
  P->graph_kind = -1;
}

// Capture one step of `kind` (0 = RK, 1 = SBDF1, 2 = SBDF2) for dt.
// Captures `steps` consecutive steps of one kind (the plan's stream must be idle).
cudaGraphExec_t capture_steps(tb_plan* P, double dt, int kind, int steps) {
  cudaGraph_t g = nullptr;
  TB_CUDA_TRY(cudaStreamBeginCapture(P->st, cudaStreamCaptureModeThreadLocal));
  try {
    for (int i = 0; i < steps; ++i) {
      if (kind == 0)
        enqueue_rk_step(P, dt);
      else
        enqueue_sbdf_step(P, dt, kind);
    }
  } catch (...) {
    cudaStreamEndCapture(P->st, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  TB_CUDA_TRY(cudaStreamEndCapture(P->st, &g));
  cudaGraphExec_t exec = nullptr;
  cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) throw Error{TB_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
  return exec;
}

void capture_step(tb_plan* P, double dt, int kind) {
  drop_graph(P);
  P->gexec = capture_steps(P, dt, kind, 1);
  P->graph_dt = dt;
  P->graph_kind = kind;
}

// Factors for the next step of the given kind (built once per dt).
void prepare_kind(tb_plan* P, double dt, int kind) {
  for (int sy = 0; sy < P->nsys; ++sy) {
    if (kind == 0) {
      const Tableau T = tableau(P->d.timestepper);
      get_factors(P, sy, 1.0, dt * T.AI[1][1]);
    } else {
      get_factors(P, sy, sbdf_coefs(kind, dt).a0, 1.0);
    }
  }
}

void advance_counters(tb_plan* P, double dt, int kind, int steps) {
  P->last_dt = dt;
  P->sim_time += dt * steps;
  P->iteration += steps;
  if (kind != 0) P->ms_history = 1;
}

}  // namespace

namespace tb {
std::vector<double2> host_twiddles(int n) { return twiddles(n); }
std::vector<double2> host_pass_twiddles(const FftPlan& fp) { return pass_twiddles(fp); }
}  // namespace tb

int tb::plan_next_kind(const tb_plan* P) {
  const int ts = P->d.timestepper;
  if (ts == TB_SBDF1) return 1;
  if (ts == TB_SBDF2) return (P->ms_history >= 1) ? 2 : 1;
  return 0;
}

void tb::plan_launch_steps(tb_plan* P, double dt, int nsteps, cudaStream_t s, int graph_steps) {
  if (!s) s = P->st;
  if (graph_steps < 1) graph_steps = 1;
  int left = nsteps;
  while (left > 0) {
    const int kind = plan_next_kind(P);
    // SBDF2's first step is SBDF1 and stands alone; every other step repeats
    const bool uniform = !(P->d.timestepper == TB_SBDF2 && kind == 1);
    const int chunk = uniform ? std::min(left, graph_steps) : 1;
    prepare_kind(P, dt, kind);
    if (P->profiling) {
      // The profiled steps run as a graph of their own in which an event
      // record node brackets every kernel, so a kernel's time is its device
      // time between its neighbours, without the host's launch latency that
      // eager launches would add to the short kernels.
      if (s != P->st) throw Error{TB_EINVAL, "profiled steps run on the plan's own stream"};
      TB_CUDA_TRY(cudaStreamSynchronize(P->st));
      cudaGraphExec_t ex = nullptr;
      try {
        ex = capture_steps(P, dt, kind, chunk);
      } catch (...) {
        for (auto& r : P->pending) {
          P->event_pool.push_back(r.a);
          P->event_pool.push_back(r.b);
        }
        P->pending.clear();
        throw;
      }
      const cudaError_t e = cudaGraphLaunch(ex, P->st);
      cudaGraphExecDestroy(ex);
      if (e != cudaSuccess) throw Error{TB_ECUDA, std::string("profiled step: ") + cudaGetErrorString(e)};
      check_launch("profiled step");
    } else if (chunk < graph_steps || chunk == 1) {
      // single steps (also for a partial last chunk, so the graph of
      // graph_steps steps is kept)
      if (!(P->gexec && P->graph_dt == dt && P->graph_kind == kind)) {
        TB_CUDA_TRY(cudaStreamSynchronize(P->st));
        capture_step(P, dt, kind);
      }
      for (int i = 0; i < chunk; ++i) TB_CUDA_TRY(cudaGraphLaunch(P->gexec, s));
    } else {
      StepGraph& mg = P->multi;
      if (!(mg.exec && mg.dt == dt && mg.kind == kind && mg.steps == chunk)) {
        if (mg.exec) cudaGraphExecDestroy(mg.exec);
        mg.exec = nullptr;
        TB_CUDA_TRY(cudaStreamSynchronize(P->st));
        mg.exec = capture_steps(P, dt, kind, chunk);
        mg.dt = dt;
        mg.kind = kind;
        mg.steps = chunk;
      }
      TB_CUDA_TRY(cudaGraphLaunch(mg.exec, s));
    }
    advance_counters(P, dt, kind, chunk);
    left -= chunk;
  }
}

// The 2D x-products kernel of form 2 (batched, ping-pong) or 3 (batched, in
// place) fits shared memory (F64, or the FP32 kernel of a mixed plan).
static bool xprod2d_form_fits(const tb_plan* P, int form) {
  if (form == 1) return true;
  if (P->mixed)
    return form == 2 ? xprod32_b_fits(P->M, (int)(P->ptwM32.bytes / sizeof(float2)))
                     : xprod32_ip_fits(P->M, (int)(P->iptwM32.bytes / sizeof(float2)));
  return form == 2 ? xprod_b_fits(P->M, (int)(P->ptwM.bytes / sizeof(double2)))
                   : xprod_ip_fits(P->M, (int)(P->iptwM.bytes / sizeof(double2)));
}

bool tb::plan_tau_parts_ok(const tb_plan* P, int parts) {
  if (parts != 1 && parts != kTauParts && parts != kTauParts8 && parts != kTauParts16) return false;
  for (int sy = 0; sy < P->nsys; ++sy) {
    if (tau_solve_smem_bytes(P->sys[sy].npad, parts) > 227 * 1024) return false;
    if (P->sys[sy].npad / kBwdWin < parts) return false;  // every partition at least one window
  }
  return true;
}

void tb::plan_set_variant(tb_plan* P, int tau_parts, int xrows) {
  bool changed = false;
  if (tau_parts > 0) {
    TB_REQUIRE(plan_tau_parts_ok(P, tau_parts), TB_ENOTSUPPORTED, "tau solve partitions must be 1, 4, 8 or 16 and fit");
    for (int sy = 0; sy < P->nsys; ++sy) {
      TauSystem& S = P->sys[sy];
      if (S.tau_parts == tau_parts) continue;
      TB_CUDA_TRY(cudaStreamSynchronize(P->st));
      S.tau_parts = tau_parts;
      S.factors.clear();  // record layouts differ between the two forms
      const size_t ys = tau_solve_scratch_doubles(P->Nk, S.npad, tau_parts) * sizeof(double);
      if (ys > P->solve_scratch.bytes) P->solve_scratch.alloc(ys);
      changed = true;
    }
  }
  if (xrows > 0 && xrows != P->xrows) {
    if (P->ndim == 3)
      TB_REQUIRE(rbc3d_xrows_ok(P, xrows), TB_ENOTSUPPORTED, "x-pass rows must be 1, 2 or 4 and fit");
    else
      TB_REQUIRE(xrows >= 1 && xrows <= 3 && xprod2d_form_fits(P, xrows), TB_ENOTSUPPORTED,
                 "2D x-products form must be 1 (per field), 2 (batched) or 3 (batched in place) and fit");
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
    P->xrows = xrows;
    changed = true;
  }
  if (changed) drop_step_graphs(P);
}

void tb::plan_prepare(tb_plan* P, double dt, int graph_steps) {
  TB_CUDA_TRY(cudaSetDevice(P->ctx->device));
  const int kind = plan_next_kind(P);
  prepare_kind(P, dt, kind);
  TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  if (!(P->gexec && P->graph_dt == dt && P->graph_kind == kind)) capture_step(P, dt, kind);
  const bool uniform = !(P->d.timestepper == TB_SBDF2 && kind == 1);
  if (uniform && graph_steps > 1) {
    StepGraph& mg = P->multi;
    if (!(mg.exec && mg.dt == dt && mg.kind == kind && mg.steps == graph_steps)) {
      if (mg.exec) cudaGraphExecDestroy(mg.exec);
      mg.exec = capture_steps(P, dt, kind, graph_steps);
      mg.dt = dt;
      mg.kind = kind;
      mg.steps = graph_steps;
    }
  }
}

size_t tb::plan_device_bytes(const tb_plan* P) {
  size_t b = 0;
  const DevBuf* bufs[] = {&P->X,   &P->G,   &P->H,    &P->MX0,  &P->Fprev, &P->MXprev, &P->Rsb, &P->tmpgrid,
                          &P->bwd, &P->fwd, &P->s3,   &P->twM,  &P->twN,   &P->ptwM,   &P->bEv, &P->bOv,
                          &P->bEd, &P->bOd, &P->fE,   &P->fO,   &P->sfE,   &P->sfO,    &P->err_mode,
                          &P->solve_scratch, &P->bcdyn,  &P->t_dev};
  for (const DevBuf* d : bufs) b += d->bytes;
  for (int i = 0; i < 4; ++i) b += P->FP[i].bytes + P->LXP[i].bytes;
  for (int sy = 0; sy < P->nsys; ++sy) {
    const TauSystem& S = P->sys[sy];
    b += S.rhs_off.bytes + S.xcode.bytes;
    for (int c = 0; c < 2; ++c) {
      const ClassTables& t = S.ct[c];
      const DevBuf* tb_[] = {&t.row_eq, &t.row_k, &t.col_unk, &t.col_k, &t.left_unk, &t.left_k, &t.bc_rhs, &t.band,
                             &t.bord,   &t.c2_z,  &t.c2_nz,   &t.c1_z,  &t.c1_nz,    &t.col_code, &t.left_code};
      for (const DevBuf* d : tb_) b += d->bytes;
    }
    for (const auto& f : S.factors) b += f->FR.bytes + f->BR.bytes + f->SI.bytes + f->PP.bytes + f->HR.bytes;
  }
  b += rbc3d_device_bytes(P) + P->kappa_m.bytes + P->nu_m.bytes;
  for (const DevBuf& d : P->sys[0].mband) b += d.bytes;
  for (const DevBuf& d : P->sys[0].mbord) b += d.bytes;
  const DevBuf* m32[] = {&P->X32,  &P->G32,  &P->H32,  &P->bEv32, &P->bOv32,  &P->bEd32, &P->bOd32,
                         &P->fE32, &P->fO32, &P->sfE32, &P->sfO32, &P->ptwM32, &P->tcAimg, &P->tcBimg, &P->tc2img};
  for (const DevBuf* d : m32) b += d->bytes;
  return b;
}

void tb::plan_snapshot(tb_plan* P, PlanSnapshot* snap) {
  snap->X.alloc(P->X.bytes);
  TB_CUDA_TRY(cudaMemcpyAsync(snap->X.p, P->X.p, P->X.bytes, cudaMemcpyDeviceToDevice, P->st));
  if (P->Fprev.bytes) {
    snap->Fprev.alloc(P->Fprev.bytes);
    snap->MXprev.alloc(P->MXprev.bytes);
    TB_CUDA_TRY(cudaMemcpyAsync(snap->Fprev.p, P->Fprev.p, P->Fprev.bytes, cudaMemcpyDeviceToDevice, P->st));
    TB_CUDA_TRY(cudaMemcpyAsync(snap->MXprev.p, P->MXprev.p, P->MXprev.bytes, cudaMemcpyDeviceToDevice, P->st));
  }
  if (P->bc_dynamic)
    TB_CUDA_TRY(cudaMemcpyAsync(&snap->t_dev, P->t_dev.p, sizeof(double), cudaMemcpyDeviceToHost, P->st));
  snap->sim_time = P->sim_time;
  snap->iteration = P->iteration;
  snap->ms_history = P->ms_history;
  TB_CUDA_TRY(cudaStreamSynchronize(P->st));
}

void tb::plan_restore(tb_plan* P, const PlanSnapshot& snap) {
  TB_CUDA_TRY(cudaMemcpyAsync(P->X.p, snap.X.p, P->X.bytes, cudaMemcpyDeviceToDevice, P->st));
  if (snap.Fprev.bytes) {
    TB_CUDA_TRY(cudaMemcpyAsync(P->Fprev.p, snap.Fprev.p, P->Fprev.bytes, cudaMemcpyDeviceToDevice, P->st));
    TB_CUDA_TRY(cudaMemcpyAsync(P->MXprev.p, snap.MXprev.p, P->MXprev.bytes, cudaMemcpyDeviceToDevice, P->st));
  }
  if (P->bc_dynamic)
    TB_CUDA_TRY(cudaMemcpyAsync(P->t_dev.p, &snap.t_dev, sizeof(double), cudaMemcpyHostToDevice, P->st));
  P->sim_time = snap.sim_time;
  P->iteration = snap.iteration;
  P->ms_history = snap.ms_history;
  TB_CUDA_TRY(cudaStreamSynchronize(P->st));
}

namespace {

void validate_desc(const tb_problem_desc* d) {
  TB_REQUIRE(d != nullptr, TB_EINVAL, "null problem descriptor");
  TB_REQUIRE(d->ndim == 2 || d->ndim == 3, TB_ENOTSUPPORTED, "ndim must be 2 or 3");
  TB_REQUIRE(d->program == TB_PROGRAM_RBC, TB_ENOTSUPPORTED, "unknown equation program");
  TB_REQUIRE(d->Nx >= 6 && d->Nx % 2 == 0, TB_EINVAL, "Nx must be even and >= 6");
  if (d->ndim == 3) {
    TB_REQUIRE(d->Ny >= 6 && d->Ny % 2 == 0, TB_EINVAL, "Ny must be even and >= 6");
    TB_REQUIRE(d->Ly > 0, TB_EINVAL, "domain lengths must be positive");
    TB_REQUIRE(d->Nz % 2 == 0, TB_ENOTSUPPORTED, "3D plans need an even Nz");

  }
  TB_REQUIRE(d->Nz >= 8 && d->Nz <= 32767, TB_EINVAL, "Nz must be in [8, 32767]");
  TB_REQUIRE(d->Lx > 0 && d->Lz > 0, TB_EINVAL, "domain lengths must be positive");
  TB_REQUIRE(std::fabs(d->dealias - 1.5) < 1e-12, TB_ENOTSUPPORTED, "only dealias = 3/2 is implemented");
  TB_REQUIRE(d->timestepper >= TB_RK222 && d->timestepper <= TB_SBDF2, TB_EINVAL, "unknown timestepper");
  TB_REQUIRE(d->precision == TB_PREC_F64 || d->precision == TB_PREC_MIXED, TB_EINVAL, "unknown precision mode");
  TB_REQUIRE(d->kappa > 0 && d->nu > 0, TB_EINVAL, "kappa and nu must be positive");
}

// Store code of unknown (unk, k) of tau system sy: 2 * (element offset of its
// row for mode 0 from X) + 1 when the unknown is i times the solved real column
// (u_x / u_par and its two taus).  System 0 taus occupy tau rows 0..6, the
// decoupled system's tau_1 / tau_2 rows 7 / 8.
long long store_code(const tb_plan* P, int sy, int unk, int k) {
  const long long Nk = P->Nk, taub = (long long)P->nplanes * (long long)P->plane;
  if (sy == 0) {
    if (unk < UK_TAU0) return 2 * ((long long)unk * P->Nz + k) * Nk + (unk == UK_UX ? 1 : 0);
    const int t = unk - UK_TAU0;
    return 2 * (taub + t * Nk) + ((t == 3 || t == 5) ? 1 : 0);
  }
  if (unk < UK_TAU0) return 2 * ((long long)4 * P->Nz + k) * Nk;
  return 2 * (taub + (long long)(6 + unk - UK_TAU0) * Nk);
}

// Right-hand-side code of a band row: 2 * (element offset of its row in a stage
// vector) + 1 for a u_x / u_par momentum row (scaled by -i on load).
long long rhs_code(const tb_plan* P, int sy, int eq, int k) {
  if (sy == 0) return 2 * ((long long)eq * P->Nz + k) * P->Nk + (eq == EQ_MX ? 1 : 0);
  return 2 * ((long long)4 * P->Nz + k) * P->Nk;
}

// Pad a class's band template to the compiled (kTauKL, kTauKU) shape.
void pad_band(ClassLayout& L) {
  TB_REQUIRE(L.kl <= kTauKL && L.ku <= kTauKU && L.nb <= 4, TB_ENOTSUPPORTED, "unexpected tau band shape");
  if (L.kl == kTauKL && L.ku == kTauKU) return;
  const int WC = kTauKL + kTauKU + 1;
  std::vector<Coef> band((size_t)L.n * WC, Coef{0, 0, 0, 0});
  for (int r = 0; r < L.n; ++r)
    for (int d = 0; d < L.kl + L.ku + 1; ++d)
      band[(size_t)r * WC + (d - L.kl + kTauKL)] = L.band[(size_t)r * (L.kl + L.ku + 1) + d];
  L.band = band;
  L.kl = kTauKL;
  L.ku = kTauKU;
}

void install_system(tb_plan* P, int sy, TauLayout lay) {
  TauSystem& S = P->sys[sy];
  auto to_int = [](long long v) {
    TB_REQUIRE(v >= -1 && v < 0x7fffffffLL, TB_ENOTSUPPORTED, "plan too large for 32-bit solve addressing");
    return (int)v;
  };
  for (int c = 0; c < 2; ++c) {
    ClassLayout& L = lay.cls[c];
    pad_band(L);
    auto to_short = [](const std::vector<int>& v) { return std::vector<short>(v.begin(), v.end()); };
    std::vector<int> cc(L.n), lc(L.nb);
    for (int j = 0; j < L.n; ++j) cc[j] = to_int(store_code(P, sy, L.col_unk[j], L.col_k[j]));
    for (int b = 0; b < L.nb; ++b) lc[b] = to_int(store_code(P, sy, L.left_unk[b], L.left_k[b]));
    ClassTables& T = S.ct[c];
    upload(T.row_eq, to_short(L.row_eq));
    upload(T.row_k, to_short(L.row_k));
    upload(T.col_unk, to_short(L.col_unk));
    upload(T.col_k, to_short(L.col_k));
    upload(T.left_unk, to_short(L.left_unk));
    upload(T.left_k, to_short(L.left_k));
    upload(T.bc_rhs, L.bc_rhs);
    upload(T.band, L.band);
    upload(T.bord, L.bord);
    upload(T.c2_z, L.c2_z);
    upload(T.c2_nz, L.c2_nz);
    upload(T.c1_z, L.c1_z);
    upload(T.c1_nz, L.c1_nz);
    upload(T.col_code, cc);
    upload(T.left_code, lc);
  }
  TB_REQUIRE(lay.cls[0].n == lay.cls[1].n, TB_ENOTSUPPORTED, "parity classes of unequal size");
  const int n = lay.cls[0].n;
  S.npad = (n + kTauRowPad - 1) / kTauRowPad * kTauRowPad;
  // partitioned solve (kTauParts warps per mode group) when its shared memory
  // fits and the modes alone do not fill the GPU, else one warp per group
  const bool many_groups = (P->Nk + kSolveModes - 1) / kSolveModes >= 4 * 148;
  S.tau_parts = (!many_groups && tau_solve_smem_bytes(S.npad, kTauParts) <= 227 * 1024) ? kTauParts : 1;
  TB_REQUIRE(tau_solve_smem_bytes(S.npad, S.tau_parts) <= 227 * 1024, TB_ENOTSUPPORTED,
             "Nz too large for the staged tau solve");
  const size_t ys = tau_solve_scratch_doubles(P->Nk, S.npad, S.tau_parts) * sizeof(double);
  if (ys > P->solve_scratch.bytes) P->solve_scratch.alloc(ys);
  // per (band row, class) right-hand-side code, -1 for the padding rows
  std::vector<int> ro((size_t)2 * S.npad, -1);
  for (int j = 0; j < n; ++j)
    for (int c = 0; c < 2; ++c) ro[2 * j + c] = to_int(rhs_code(P, sy, lay.cls[c].row_eq[j], lay.cls[c].row_k[j]));
  upload(S.rhs_off, ro);
  // per (band row, class) store target in 16 bits: the code is 2 * R * Nk +
  // flag for the element row R of the unknown, kept as 2 R + flag
  std::vector<short> xc((size_t)2 * S.npad, (short)-1);
  for (int j = 0; j < n; ++j)
    for (int c = 0; c < 2; ++c) {
      const long long code = store_code(P, sy, lay.cls[c].col_unk[j], lay.cls[c].col_k[j]);
      const long long R = (code >> 1) / P->Nk;
      TB_REQUIRE((code >> 1) % P->Nk == 0 && 2 * R + 1 < 0x7fff, TB_ENOTSUPPORTED, "store code outside 16 bits");
      xc[2 * j + c] = (short)(2 * R + (code & 1));
    }
  upload(S.xcode, xc);
  S.lay = std::move(lay);
}

// 3D state I/O: the layout change and the rotation of the horizontal velocity
// run on the device (rbc3d_state_get / _set) through one plane of scratch.
void state3d_io(tb_plan* P, int field, void* data, int where, bool set) {
  TB_REQUIRE(field >= TB_FIELD_B && field <= TB_FIELD_UY, TB_EINVAL, "bad field selector");
  const size_t count = field == TB_FIELD_TAU ? 9 * (size_t)P->Nk : P->plane;
  double2* dev = where == TB_DEVICE ? static_cast<double2*>(data) : P->tmp3.as<double2>();
  if (set) {
    if (where != TB_DEVICE)
      TB_CUDA_TRY(cudaMemcpyAsync(dev, data, count * sizeof(double2), cudaMemcpyHostToDevice, P->st));
    rbc3d_state_set(P, field, dev);
  } else {
    rbc3d_state_get(P, field, dev);
    if (where != TB_DEVICE)
      TB_CUDA_TRY(cudaMemcpyAsync(data, dev, count * sizeof(double2), cudaMemcpyDeviceToHost, P->st));
  }
  check_launch("3D state I/O");
  TB_CUDA_TRY(cudaStreamSynchronize(P->st));
}

}  // namespace

extern "C" {

int tb_version(void) { return 1; }

const char* tb_status_string(tb_status s) {
  switch (s) {
    case TB_OK: return "ok";
    case TB_EINVAL: return "invalid argument";
    case TB_ENOMEM: return "out of device memory";
    case TB_ESINGULAR: return "singular tau system";
    case TB_ETIMEOUT: return "device wait timed out";
    case TB_ECUDA: return "CUDA error";
    case TB_ENOTSUPPORTED: return "not supported";
    case TB_EBUDGET: return "over HBM budget";
    case TB_ESTATE: return "invalid call order";
    default: return "unknown status";
  }
}

tb_status tb_context_create(int device, tb_context** out) {
  if (!out) return TB_EINVAL;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    g_err = std::string("no CUDA device: ") + cudaGetErrorString(e);
    return TB_ECUDA;
  }
  if (device < 0 || device >= ndev) {
    g_err = "device index out of range";
    return TB_EINVAL;
  }
  e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    g_err = cudaGetErrorString(e);
    return TB_ECUDA;
  }
  tb_context* c = new (std::nothrow) tb_context();
  if (!c) return TB_ENOMEM;
  c->device = device;
  // Stream-ordered scratch (factorisation work arrays, staging of initial
  // states) returns to the device's default pool; keep up to 256 MB of it
  // mapped so that a later plan reuses it without a new mapping.
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    unsigned long long keep = 256ull << 20;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  *out = c;
  return TB_OK;
}

tb_status tb_context_destroy(tb_context* ctx) {
  delete ctx;
  return TB_OK;
}

const char* tb_last_error(const tb_context* ctx) {
  if (!ctx) return g_err.c_str();
  // a per-thread copy, so another thread's failure cannot move the string
  // under the caller
  thread_local std::string copy;
  std::lock_guard<std::mutex> lk(ctx->mu);
  copy = ctx->last_error;
  return copy.c_str();
}

}  // extern "C"

void tb::build_plan(tb_plan* P, tb_context* ctx, const tb_problem_desc* descs, int B) {
  const tb_problem_desc* desc = descs;
  TB_REQUIRE(B >= 1, TB_EINVAL, "no instances");
  for (int b = 1; b < B; ++b)
    TB_REQUIRE(descs[b].ndim == 2 && descs[0].ndim == 2 && descs[b].Nx == descs[0].Nx && descs[b].Nz == descs[0].Nz &&
                   descs[b].Lx == descs[0].Lx && descs[b].Lz == descs[0].Lz &&
                   descs[b].timestepper == descs[0].timestepper && descs[b].precision == descs[0].precision &&
                   descs[b].b_bottom == descs[0].b_bottom && descs[b].b_top == descs[0].b_top,
               TB_EINVAL, "stacked instances must share the 2D shape, walls, stepper and precision");
    validate_desc(desc);
    TB_CUDA_TRY(cudaSetDevice(ctx->device));
    P->ctx = ctx;
    P->d = *desc;
    P->ndim = desc->ndim;
    P->Nx = desc->Nx;
    P->Nz = desc->Nz;
    P->Kx = desc->Nx / 2 + 1;
    P->Ny = desc->ndim == 3 ? desc->Ny : 1;
    P->B = B;
    P->Nkm = P->Kx * P->Ny;
    P->Nk = P->Nkm * B;
    int M = (int)std::ceil(1.5 * desc->Nx);
    if (M % 2) ++M;
    P->M = M;
    P->k0 = 2.0 * M_PI / desc->Lx;
    P->s = 2.0 / desc->Lz;
    P->plane = (size_t)P->Nz * P->Nk;
    if (desc->ndim == 3) {
      int My = (int)std::ceil(1.5 * desc->Ny);
      if (My % 2) ++My;
      P->My = My;
      P->k0y = 2.0 * M_PI / desc->Ly;
      P->nplanes = 5;
      P->ntau = 9;
      P->nf = 4;
    }
    TB_REQUIRE(make_fft_plan(P->M, &P->fpM) && make_fft_plan(P->Nx, &P->fpN), TB_ENOTSUPPORTED,
               "Nx must be of the form 2^a 3^b");
    if (desc->ndim == 2)
      TB_REQUIRE(xprod_smem_bytes(P->M, P->Nk, (int)pass_twiddles(P->fpM).size()) <= 227 * 1024, TB_ENOTSUPPORTED,
                 "Nx too large for the fused x kernel");
    // the step's main chain on a work stream, the work forked off it on a
    // side stream of least priority (create_work_stream)
    TB_CUDA_TRY(create_work_stream(&P->st));
    TB_CUDA_TRY(create_work_stream(&P->st2, true));
    TB_CUDA_TRY(cudaEventCreateWithFlags(&P->ev_fork, cudaEventDisableTiming));
    TB_CUDA_TRY(cudaEventCreateWithFlags(&P->ev_join, cudaEventDisableTiming));
    TB_CUDA_TRY(cudaEventCreate(&P->ev0));
    TB_CUDA_TRY(cudaEventCreate(&P->ev1));
    TB_CUDA_TRY(set_transform_smem_limits(227 * 1024));
    TB_CUDA_TRY(set_tau_smem_limits(227 * 1024));
    TB_CUDA_TRY(set_tc32_smem_limits());
    // transforms
    ChebMats cm = build_cheb_mats(P->Nz, desc->Lz);
    const int N = P->Nz;
    P->Hz = (N + 1) / 2;
    P->Ke = (N + 1) / 2;
    P->Ko = N / 2;
    auto pad16 = [](int k) { return (k + 15) / 16 * 16; };
    auto cols_of = [&](const std::vector<double>& m, int par) {  // rows j < H, columns n = 2k + par
      const int K = par ? P->Ko : P->Ke, Kp = pad16(K);
      std::vector<double> o((size_t)P->Hz * Kp, 0.0);
      for (int j = 0; j < P->Hz; ++j)
        for (int k = 0; k < K; ++k) o[(size_t)j * Kp + k] = m[(size_t)j * N + 2 * k + par];
      return o;
    };
    auto rows_of = [&](const std::vector<double>& m, int par) {  // rows n = 2r + par, columns j < H
      const int R = par ? P->Ko : P->Ke, Kp = pad16(P->Hz);
      std::vector<double> o((size_t)R * Kp, 0.0);
      for (int r = 0; r < R; ++r)
        for (int j = 0; j < P->Hz; ++j) o[(size_t)r * Kp + j] = m[(size_t)(2 * r + par) * N + j];
      return o;
    };
    std::vector<double> bwdp((size_t)N * pad16(N), 0.0);
    for (int j = 0; j < N; ++j)
      for (int n = 0; n < N; ++n) bwdp[(size_t)j * pad16(N) + n] = cm.bwd[(size_t)j * N + n];
    upload(P->bEv, cols_of(cm.bwd, 0));
    upload(P->bOv, cols_of(cm.bwd, 1));
    upload(P->bEd, cols_of(cm.bwd_d, 0));
    upload(P->bOd, cols_of(cm.bwd_d, 1));
    upload(P->fE, rows_of(cm.fwd, 0));
    upload(P->fO, rows_of(cm.fwd, 1));
    upload(P->sfE, rows_of(cm.sfwd, 0));
    upload(P->sfO, rows_of(cm.sfwd, 1));
    upload(P->bwd, bwdp);
    upload(P->s3, cm.s3);
    upload(P->twM, twiddles(P->M));
    upload(P->ptwM, pass_twiddles(P->fpM));
    P->mixed = desc->precision == TB_PREC_MIXED;
    P->fpMip = best_ip_order(P->fpM, P->mixed ? 8 : 16);
    upload(P->iptwM, ip_twiddles(P->fpMip));
    upload(P->twN, twiddles(P->Nx));
    if (P->mixed) {
      auto f32 = [](const std::vector<double>& v) {
        std::vector<float> o(v.size());
        for (size_t i = 0; i < v.size(); ++i) o[i] = (float)v[i];
        return o;
      };
      upload(P->bEv32, f32(cols_of(cm.bwd, 0)));
      upload(P->bOv32, f32(cols_of(cm.bwd, 1)));
      upload(P->bEd32, f32(cols_of(cm.bwd_d, 0)));
      upload(P->bOd32, f32(cols_of(cm.bwd_d, 1)));
      upload(P->fE32, f32(rows_of(cm.fwd, 0)));
      upload(P->fO32, f32(rows_of(cm.fwd, 1)));
      upload(P->sfE32, f32(rows_of(cm.sfwd, 0)));
      upload(P->sfO32, f32(rows_of(cm.sfwd, 1)));
      const std::vector<double2> pt = pass_twiddles(P->fpM);
      std::vector<float2> pt32(pt.size());
      for (size_t i = 0; i < pt.size(); ++i) pt32[i] = make_float2((float)pt[i].x, (float)pt[i].y);
      upload(P->ptwM32, pt32);
      const std::vector<double2> it = ip_twiddles(P->fpMip);
      std::vector<float2> it32(it.size());
      for (size_t i = 0; i < it.size(); ++i) it32[i] = make_float2((float)it[i].x, (float)it[i].y);
      upload(P->iptwM32, it32);
      TB_REQUIRE(xprod32_smem_bytes(P->M, (int)pt32.size()) <= 227 * 1024, TB_ENOTSUPPORTED,
                 "Nx too large for the FP32 x kernel");
      // TF32 operand images of the eight transform matrices for the 2D
      // tensor-core GEMMs, and the scratch of their per-call B images (six
      // distinct inputs per GEMM), when the shapes fit one tensor-core tile
      // (3D plans stream their planes through the form made in rbc3d_setup)
      if (P->ndim == 2 && P->Hz <= 128 && pad16(P->Ke) <= 128) {
        const size_t fa = tc32_a_image_floats();
        P->tcAimg.alloc(8 * fa * sizeof(float));
        const DevBuf* mats[8] = {&P->bEv32, &P->bOv32, &P->bEd32, &P->bOd32, &P->fE32, &P->fO32, &P->sfE32, &P->sfO32};
        const int rows[8] = {P->Hz, P->Hz, P->Hz, P->Hz, P->Ke, P->Ko, P->Ke, P->Ko};
        const int kps[8] = {pad16(P->Ke), pad16(P->Ko), pad16(P->Ke), pad16(P->Ko),
                            pad16(P->Hz), pad16(P->Hz), pad16(P->Hz), pad16(P->Hz)};
        for (int m = 0; m < 8; ++m)
          if (rows[m] > 0) make_tc32_a_image(mats[m]->as<float>(), rows[m], kps[m], P->tcAimg.as<float>() + m * fa, P->st);
        TB_CUDA_TRY(cudaGetLastError());
        TB_CUDA_TRY(cudaStreamSynchronize(P->st));
        P->tcBimg.alloc(tc32_b_scratch_floats(2 * P->Nk, 6) * sizeof(float));
      }
      // the plane form (A in tensor memory, tiles read from the planes)
      if (P->ndim == 2 && tc32p_supported(N, 2 * P->Nk)) {
        P->tc2img.alloc(tc32p_image_floats() * sizeof(float));
        make_tc32p_images(P->bEv32.as<float>(), P->bOv32.as<float>(), P->bEd32.as<float>(), P->bOd32.as<float>(),
                          pad16(P->Ke), pad16(P->Ko), P->sfE32.as<float>(), P->sfO32.as<float>(), pad16(P->Hz), N,
                          P->tc2img.as<float>(), P->st);
        TB_CUDA_TRY(cudaGetLastError());
        TB_CUDA_TRY(cudaStreamSynchronize(P->st));
      }
      TB_CUDA_TRY(set_mixed_smem_limits(227 * 1024));
    }
    // tau systems: the coupled Boussinesq system (with |k| per mode in 3D) and,
    // in 3D, the decoupled cross-wavevector velocity
    const bool d3 = P->ndim == 3;
    install_system(P, 0,
                   build_rbc_layout(P->Nz, d3 ? desc->Lx * desc->Ly : desc->Lx, desc->Lz, desc->kappa, desc->nu,
                                    d3 ? (double)desc->Nx * desc->Ny : (double)desc->Nx, desc->b_bottom, desc->b_top));
    if (B > 1) {
      // instances differ only in kappa / nu: their band and border coefficients
      P->sys[0].mband = std::vector<DevBuf>(2 * B);
      P->sys[0].mbord = std::vector<DevBuf>(2 * B);
      std::vector<double> km(B), nm(B);
      for (int b = 0; b < B; ++b) {
        TauLayout lb = build_rbc_layout(P->Nz, descs[b].Lx, descs[b].Lz, descs[b].kappa, descs[b].nu,
                                        (double)descs[b].Nx, descs[b].b_bottom, descs[b].b_top);
        for (int c = 0; c < 2; ++c) {
          pad_band(lb.cls[c]);
          upload(P->sys[0].mband[2 * b + c], lb.cls[c].band);
          upload(P->sys[0].mbord[2 * b + c], lb.cls[c].bord);
        }
        km[b] = descs[b].kappa;
        nm[b] = descs[b].nu;
      }
      upload(P->kappa_m, km);
      upload(P->nu_m, nm);
    }
    if (d3) install_system(P, 1, build_helmholtz_layout(P->Nz, desc->Lz, desc->nu));
    P->nsys = d3 ? 2 : 1;
    TB_REQUIRE(rk_final_smem_bytes(P->Nz) <= 227 * 1024, TB_ENOTSUPPORTED, "Nz too large for the final RK update");
    P->err_mode.alloc(sizeof(int));
    // state and work arrays
    const size_t pb = P->plane * sizeof(double2);
    P->X.alloc(P->nplanes * pb + (size_t)P->ntau * P->Nk * sizeof(double2));
    P->tau.p = static_cast<char*>(P->X.p) + P->nplanes * pb;
    P->tau.bytes = (size_t)P->ntau * P->Nk * sizeof(double2);
    if (!d3) {
      P->G.alloc(12 * (size_t)((P->Nz + 1) / 2) * P->Nk * sizeof(double2));
      P->H.alloc(3 * pb);
      if (P->mixed) {
        P->X32.alloc(3 * P->plane * sizeof(float2));
        P->G32.alloc(12 * (size_t)((P->Nz + 1) / 2) * P->Nk * sizeof(float2));
        P->H32.alloc(3 * P->plane * sizeof(float2));
      }
      P->tmpgrid.alloc(P->plane * sizeof(double2));
    } else {
      rbc3d_setup(P);
    }
    P->MX0.alloc(P->nplanes * pb);
    const int nst = tableau(desc->timestepper).s;
    const int nstage = (desc->timestepper == TB_SBDF1 || desc->timestepper == TB_SBDF2) ? 1 : nst;
    for (int i = 0; i < nstage; ++i) {
      P->FP[i].alloc(P->nplanes * pb);
      P->LXP[i].alloc(P->nplanes * pb);
    }
    const bool sbdf = desc->timestepper == TB_SBDF1 || desc->timestepper == TB_SBDF2;
    if (sbdf) {
      P->Fprev.alloc(P->nplanes * pb);
      P->MXprev.alloc(P->nplanes * pb);
      P->Rsb.alloc(P->nplanes * pb);
    }
    TB_CUDA_TRY(cudaMemsetAsync(P->X.p, 0, P->X.bytes, P->st));
    TB_CUDA_TRY(cudaMemsetAsync(P->MX0.p, 0, P->MX0.bytes, P->st));
    for (int i = 0; i < nstage; ++i) {
      TB_CUDA_TRY(cudaMemsetAsync(P->FP[i].p, 0, P->FP[i].bytes, P->st));
      TB_CUDA_TRY(cudaMemsetAsync(P->LXP[i].p, 0, P->LXP[i].bytes, P->st));
    }
    if (sbdf) {
      TB_CUDA_TRY(cudaMemsetAsync(P->Fprev.p, 0, P->Fprev.bytes, P->st));
      TB_CUDA_TRY(cudaMemsetAsync(P->MXprev.p, 0, P->MXprev.bytes, P->st));
    }
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
}

extern "C" {

tb_status tb_plan_create(tb_context* ctx, const tb_problem_desc* desc, tb_plan** out) {
  if (!ctx || !out) return TB_EINVAL;
  *out = nullptr;
  std::unique_ptr<tb_plan> P(new (std::nothrow) tb_plan());
  if (!P) return TB_ENOMEM;
  tb_status s = guard(ctx, [&] { build_plan(P.get(), ctx, desc, 1); });
  if (s != TB_OK) return s;
  *out = P.release();
  return TB_OK;
}

tb_status tb_plan_destroy(tb_plan* plan) {
  if (!plan) return TB_OK;
  cudaStreamSynchronize(plan->st);
  delete plan;
  return TB_OK;
}

tb_status tb_set_state(tb_plan* P, int field, const void* data, int where) {
  if (!P || !data) return TB_EINVAL;
  const bool keep = (where & TB_KEEP_HISTORY) != 0;
  where &= ~TB_KEEP_HISTORY;
  if (P->ndim == 3)
    return guard(P->ctx, [&] {
      state3d_io(P, field, const_cast<void*>(data), where, true);
      if (!keep) P->ms_history = 0;
    });
  return guard(P->ctx, [&] {
    TB_REQUIRE(field >= TB_FIELD_B && field <= TB_FIELD_TAU, TB_EINVAL, "bad field selector");
    void* dst = field == TB_FIELD_TAU ? P->tau.p : (void*)P->Xp(field);
    size_t bytes = field == TB_FIELD_TAU ? P->tau.bytes : P->plane * sizeof(double2);
    TB_CUDA_TRY(cudaMemcpyAsync(dst, data, bytes, where == TB_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                P->st));
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
    if (!keep) P->ms_history = 0;  // a new state restarts multistep history
  });
}

tb_status tb_get_state(tb_plan* P, int field, void* data, int where) {
  if (!P || !data) return TB_EINVAL;
  if (P->ndim == 3) return guard(P->ctx, [&] { state3d_io(P, field, data, where, false); });
  return guard(P->ctx, [&] {
    TB_REQUIRE(field >= TB_FIELD_B && field <= TB_FIELD_TAU, TB_EINVAL, "bad field selector");
    const void* src = field == TB_FIELD_TAU ? P->tau.p : (const void*)P->Xp(field);
    size_t bytes = field == TB_FIELD_TAU ? P->tau.bytes : P->plane * sizeof(double2);
    TB_CUDA_TRY(cudaMemcpyAsync(data, src, bytes, where == TB_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                P->st));
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  });
}

}  // extern "C"

namespace {
// Copies of several 2D state fields on the plan's stream, one wait.  Fields
// that are neighbours in the device state (b, u_x, u_z, p, then the taus, one
// allocation) and whose caller buffers are neighbours too go as one copy.
void copy_state_fields(tb_plan* P, int nfields, const int* fields, void* const* data, int where, bool to_device,
                       bool wait = true) {
  TB_REQUIRE(P->ndim == 2, TB_ENOTSUPPORTED, "multi-field state I/O is for 2D plans (use the single-field call in 3D)");
  for (int i = 0; i < nfields; ++i) {
    TB_REQUIRE(fields[i] >= TB_FIELD_B && fields[i] <= TB_FIELD_TAU, TB_EINVAL, "bad field selector");
    TB_REQUIRE(data[i] != nullptr, TB_EINVAL, "null field buffer");
  }
  auto dev = [&](int f) -> char* { return static_cast<char*>(f == TB_FIELD_TAU ? P->tau.p : (void*)P->Xp(f)); };
  auto len = [&](int f) -> size_t { return f == TB_FIELD_TAU ? P->tau.bytes : P->plane * sizeof(double2); };
  const cudaMemcpyKind kind = where == TB_DEVICE ? cudaMemcpyDeviceToDevice
                                                 : (to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost);
  for (int i = 0; i < nfields;) {
    char* d0 = dev(fields[i]);
    char* h0 = static_cast<char*>(data[i]);
    size_t bytes = len(fields[i]);
    int k = i + 1;
    while (k < nfields && dev(fields[k]) == d0 + bytes && static_cast<char*>(data[k]) == h0 + bytes) {
      bytes += len(fields[k]);
      ++k;
    }
    if (to_device)
      TB_CUDA_TRY(cudaMemcpyAsync(d0, h0, bytes, kind, P->st));
    else
      TB_CUDA_TRY(cudaMemcpyAsync(h0, d0, bytes, kind, P->st));
    i = k;
  }
  if (wait) TB_CUDA_TRY(cudaStreamSynchronize(P->st));
}
}  // namespace

extern "C" {

tb_status tb_set_states(tb_plan* P, int nfields, const int* fields, const void* const* data, int where) {
  if (!P || nfields < 0 || (nfields > 0 && (!fields || !data))) return TB_EINVAL;
  const bool keep = (where & TB_KEEP_HISTORY) != 0, nowait = (where & TB_NO_WAIT) != 0;
  where &= ~(TB_KEEP_HISTORY | TB_NO_WAIT);
  return guard(P->ctx, [&] {
    copy_state_fields(P, nfields, fields, const_cast<void* const*>(data), where, true, !nowait);
    if (!keep) P->ms_history = 0;  // a new state restarts multistep history
  });
}

tb_status tb_get_states(tb_plan* P, int nfields, const int* fields, void* const* data, int where) {
  if (!P || nfields < 0 || (nfields > 0 && (!fields || !data)) || (where & TB_NO_WAIT)) return TB_EINVAL;
  return guard(P->ctx, [&] { copy_state_fields(P, nfields, fields, data, where, false); });
}

tb_status tb_step(tb_plan* P, double dt, int nsteps) {
  if (!P) return TB_EINVAL;
  return guard(P->ctx, [&] {
    TB_REQUIRE(dt > 0 && std::isfinite(dt), TB_EINVAL, "dt must be positive and finite");
    TB_REQUIRE(nsteps >= 0, TB_EINVAL, "nsteps must be >= 0");
    TB_CUDA_TRY(cudaSetDevice(P->ctx->device));
    TB_CUDA_TRY(cudaEventRecord(P->ev0, P->st));
    plan_launch_steps(P, dt, nsteps, P->st, 1);
    TB_CUDA_TRY(cudaEventRecord(P->ev1, P->st));
    TB_CUDA_TRY(cudaEventSynchronize(P->ev1));
    TB_CUDA_TRY(cudaEventElapsedTime(&P->last_ms, P->ev0, P->ev1));
    TB_CUDA_TRY(cudaGetLastError());
    if (P->mixed && P->tc32 && tc32_status() == 1)
      throw Error{TB_ETIMEOUT, "a tensor-core transform GEMM gave up waiting for its MMAs (results not stored)"};
    if (P->profiling) collect_profile(P);
  });
}

tb_status tb_step_async(tb_plan* P, double dt, int nsteps, int graph_steps) {
  if (!P) return TB_EINVAL;
  return guard(P->ctx, [&] {
    TB_REQUIRE(dt > 0 && std::isfinite(dt), TB_EINVAL, "dt must be positive and finite");
    TB_REQUIRE(nsteps >= 0 && graph_steps >= 1, TB_EINVAL, "nsteps must be >= 0 and graph_steps >= 1");
    TB_REQUIRE(!P->profiling, TB_ESTATE, "profiling runs through tb_step");
    TB_CUDA_TRY(cudaSetDevice(P->ctx->device));
    plan_launch_steps(P, dt, nsteps, P->st, graph_steps);
    check_launch("asynchronous steps");
  });
}

tb_status tb_plan_query(tb_plan* P, int* idle) {
  if (!P || !idle) return TB_EINVAL;
  return guard(P->ctx, [&] {
    TB_CUDA_TRY(cudaSetDevice(P->ctx->device));
    const cudaError_t e = cudaStreamQuery(P->st);
    if (e == cudaSuccess) {
      *idle = 1;
    } else if (e == cudaErrorNotReady) {
      cudaGetLastError();
      *idle = 0;
    } else {
      throw Error{TB_ECUDA, std::string("plan stream: ") + cudaGetErrorString(e)};
    }
  });
}

tb_status tb_plan_wait(tb_plan* P) {
  if (!P) return TB_EINVAL;
  return guard(P->ctx, [&] {
    TB_CUDA_TRY(cudaSetDevice(P->ctx->device));
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  });
}

tb_status tb_plan_device_bytes(const tb_plan* P, size_t* bytes) {
  if (!P || !bytes) return TB_EINVAL;
  *bytes = plan_device_bytes(P);
  return TB_OK;
}

tb_status tb_sim_time(const tb_plan* P, double* t, long long* it) {
  if (!P) return TB_EINVAL;
  if (t) *t = P->sim_time;
  if (it) *it = P->iteration;
  return TB_OK;
}

tb_status tb_synchronize(tb_plan* P) {
  if (!P) return TB_EINVAL;
  return guard(P->ctx, [&] { TB_CUDA_TRY(cudaStreamSynchronize(P->st)); });
}

tb_status tb_last_step_ms(const tb_plan* P, float* ms) {
  if (!P || !ms) return TB_EINVAL;
  *ms = P->last_ms;
  return TB_OK;
}

tb_status tb_set_profiling(tb_plan* P, int on) {
  if (!P) return TB_EINVAL;
  P->profiling = on != 0;
  return TB_OK;
}

tb_status tb_profile_count(const tb_plan* P, int* n) {
  if (!P || !n) return TB_EINVAL;
  *n = (int)P->prof.size();
  return TB_OK;
}

tb_status tb_profile_entry(const tb_plan* P, int i, char* name, int name_len, double* ms_total, long long* launches) {
  if (!P || i < 0 || i >= (int)P->prof.size() || !name || name_len < 1) return TB_EINVAL;
  auto it = P->prof.begin();
  std::advance(it, i);
  std::snprintf(name, (size_t)name_len, "%s", it->first.c_str());
  if (ms_total) *ms_total = it->second.first;
  if (launches) *launches = it->second.second;
  return TB_OK;
}

tb_status tb_profile_reset(tb_plan* P) {
  if (!P) return TB_EINVAL;
  P->prof.clear();
  return TB_OK;
}

tb_status tb_tau_layout_query(int Nz, double Lx, double Lz, int cls, int* info4) {
  if (!info4 || cls < 0 || cls > 1) return TB_EINVAL;
  if (Nz < 8 || Nz > 32767 || !(Lx > 0) || !(Lz > 0)) return TB_EINVAL;
  try {
    TauLayout L = build_rbc_layout(Nz, Lx, Lz, 1.0, 1.0, 1.0, 0.0, 0.0);
    info4[0] = L.cls[cls].n;
    info4[1] = L.cls[cls].nb;
    info4[2] = L.cls[cls].kl;
    info4[3] = L.cls[cls].ku;
    return TB_OK;
  } catch (const Error& e) {
    g_err = e.msg;
    return e.code;
  }
}

tb_status tb_plan_set_variant(tb_plan* P, int tau_parts, int xrows) {
  if (!P) return TB_EINVAL;
  return guard(P->ctx, [&] {
    TB_CUDA_TRY(cudaSetDevice(P->ctx->device));
    plan_set_variant(P, tau_parts, xrows);
  });
}

tb_status tb_plan_set_gemm_path(tb_plan* P, int tensor_cores) {
  if (!P || (tensor_cores != 0 && tensor_cores != 1)) return TB_EINVAL;
  return guard(P->ctx, [&] {
    TB_CUDA_TRY(cudaSetDevice(P->ctx->device));
    if (P->tc32 != (tensor_cores == 1)) {
      TB_CUDA_TRY(cudaStreamSynchronize(P->st));
      P->tc32 = tensor_cores == 1;
      drop_step_graphs(P);  // the captured steps launch the other kernel
    }
  });
}

tb_status tb_plan_get_gemm_path(const tb_plan* P, int* tensor_cores) {
  if (!P || !tensor_cores) return TB_EINVAL;
  *tensor_cores = P->tc32 ? 1 : 0;
  return TB_OK;
}

tb_status tb_plan_get_variant(const tb_plan* P, int* tau_parts, int* xrows) {
  if (!P) return TB_EINVAL;
  if (tau_parts) *tau_parts = P->sys[0].tau_parts;
  if (xrows) *xrows = P->xrows;
  return TB_OK;
}

tb_status tb_plan_tune(tb_plan* P, double dt, int trial_steps, int* tau_parts, int* xrows) {
  if (!P || trial_steps < 1) return TB_EINVAL;
  return guard(P->ctx, [&] {
    TB_REQUIRE(dt > 0 && std::isfinite(dt), TB_EINVAL, "dt must be positive and finite");
    TB_REQUIRE(!P->profiling, TB_ESTATE, "tuning runs without profiling");
    TB_CUDA_TRY(cudaSetDevice(P->ctx->device));
    PlanSnapshot snap;
    plan_snapshot(P, &snap);
    std::vector<int> parts_c, rows_c;
    for (int p : {kTauParts16, kTauParts8, kTauParts, 1})
      if (plan_tau_parts_ok(P, p)) parts_c.push_back(p);
    if (P->ndim == 3) {
      for (int r : {1, 2, 4})
        if (rbc3d_xrows_ok(P, r)) rows_c.push_back(r);
    } else {
      for (int form : {1, 2, 3})  // per field, batched, batched in place
        if (xprod2d_form_fits(P, form)) rows_c.push_back(form);
    }
    float best = 1e30f;
    int bp = P->sys[0].tau_parts, br = P->xrows;
    for (int pc : parts_c)
      for (int rc : rows_c) {
        plan_set_variant(P, pc, rc);
        // first launches factor the tau systems and capture the graphs
        plan_launch_steps(P, dt, std::min(trial_steps, 2), P->st, 1);
        TB_CUDA_TRY(cudaStreamSynchronize(P->st));
        plan_restore(P, snap);
        TB_CUDA_TRY(cudaEventRecord(P->ev0, P->st));
        plan_launch_steps(P, dt, trial_steps, P->st, 1);
        TB_CUDA_TRY(cudaEventRecord(P->ev1, P->st));
        TB_CUDA_TRY(cudaEventSynchronize(P->ev1));
        float ms = 0.f;
        TB_CUDA_TRY(cudaEventElapsedTime(&ms, P->ev0, P->ev1));
        plan_restore(P, snap);
        if (ms < best) {
          best = ms;
          bp = pc;
          br = rc;
        }
      }
    plan_set_variant(P, bp, br);
    // then the side stream on or off, on a longer trial (the difference is a
    // few percent)
    const int ov_steps = std::max(trial_steps, 10);
    float ov_ms[2] = {1e30f, 1e30f};  // best of two alternating trials each
    for (int t = 0; t < 4; ++t) {
      const int ov = t & 1;
      if (P->overlap != (ov == 1)) {
        P->overlap = ov == 1;
        drop_step_graphs(P);
      }
      plan_launch_steps(P, dt, 2, P->st, 1);
      TB_CUDA_TRY(cudaStreamSynchronize(P->st));
      plan_restore(P, snap);
      TB_CUDA_TRY(cudaEventRecord(P->ev0, P->st));
      plan_launch_steps(P, dt, ov_steps, P->st, 1);
      TB_CUDA_TRY(cudaEventRecord(P->ev1, P->st));
      TB_CUDA_TRY(cudaEventSynchronize(P->ev1));
      float ms = 0.f;
      TB_CUDA_TRY(cudaEventElapsedTime(&ms, P->ev0, P->ev1));
      ov_ms[ov] = std::min(ov_ms[ov], ms);
      plan_restore(P, snap);
    }
    const bool ov_best = ov_ms[1] < ov_ms[0];
    if (P->overlap != ov_best) {
      P->overlap = ov_best;
      drop_step_graphs(P);
    }
    // mixed plans with a tensor-core form of their transforms: that form or
    // the SIMT kernel, whichever is faster at this size
    if (P->mixed && (P->tc2img.p != nullptr || P->tc3)) {
      float tc_ms[2] = {1e30f, 1e30f};
      for (int t = 0; t < 4; ++t) {
        const int tc = t & 1;
        if (P->tc32 != (tc == 1)) {
          P->tc32 = tc == 1;
          drop_step_graphs(P);
        }
        plan_launch_steps(P, dt, 2, P->st, 1);
        TB_CUDA_TRY(cudaStreamSynchronize(P->st));
        plan_restore(P, snap);
        TB_CUDA_TRY(cudaEventRecord(P->ev0, P->st));
        plan_launch_steps(P, dt, ov_steps, P->st, 1);
        TB_CUDA_TRY(cudaEventRecord(P->ev1, P->st));
        TB_CUDA_TRY(cudaEventSynchronize(P->ev1));
        float ms = 0.f;
        TB_CUDA_TRY(cudaEventElapsedTime(&ms, P->ev0, P->ev1));
        tc_ms[tc] = std::min(tc_ms[tc], ms);
        plan_restore(P, snap);
      }
      const bool tc_best = tc_ms[1] < tc_ms[0];
      if (P->tc32 != tc_best) {
        P->tc32 = tc_best;
        drop_step_graphs(P);
      }
    }
    plan_restore(P, snap);
    if (tau_parts) *tau_parts = bp;
    if (xrows) *xrows = br;
  });
}

tb_status tb_set_wall_values(tb_plan* P, int wall, const double* value, const double* rate, int where) {
  if (!P || !value || (wall != 0 && wall != 1)) return TB_EINVAL;
  return guard(P->ctx, [&] {
    TB_REQUIRE(P->d.program == TB_PROGRAM_RBC, TB_ENOTSUPPORTED, "wall values belong to the RBC program");
    TB_CUDA_TRY(cudaSetDevice(P->ctx->device));
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
    const size_t nm = P->Nk;
    auto fetch = [&](const double* src, std::vector<double2>& dst) {
      dst.assign(nm, make_double2(0.0, 0.0));
      if (!src) return;
      std::vector<double2> pub(nm);
      if (where == TB_DEVICE)
        TB_CUDA_TRY(cudaMemcpy(pub.data(), src, nm * sizeof(double2), cudaMemcpyDeviceToHost));
      else
        std::memcpy(pub.data(), src, nm * sizeof(double2));
      for (size_t m = 0; m < nm; ++m) {  // public (kx fastest) -> plan mode order (ky fastest in 3D)
        const size_t ix = m / P->Ny, iy = m % P->Ny;
        dst[m] = pub[ix + (size_t)P->Kx * iy];
      }
      for (const double2& v : dst)
        TB_REQUIRE(std::isfinite(v.x) && std::isfinite(v.y), TB_EINVAL, "wall values must be finite");
    };
    std::vector<double2> v0, v1;
    fetch(value, v0);
    fetch(rate, v1);
    if (!P->bc_dynamic) {
      // start from the plan's constant wall values: b at the DC mode, times the
      // unnormalised transform of a constant (Nx, or Nx Ny)
      const double scale = (double)P->Nx * (double)P->Ny;
      P->bc_host.assign(4 * nm, make_double2(0.0, 0.0));
      P->bc_host[0] = make_double2(P->d.b_bottom * scale, 0.0);
      P->bc_host[2 * nm] = make_double2(P->d.b_top * scale, 0.0);
      P->bcdyn.alloc(4 * nm * sizeof(double2));
      P->t_dev.alloc(sizeof(double));
      P->bc_tref = P->sim_time;
      P->bc_dynamic = true;
      drop_step_graphs(P);  // step graphs gain the wall-time update
    }
    // re-reference both walls to the current time, then replace this wall
    const double el = P->sim_time - P->bc_tref;
    for (int w = 0; w < 2; ++w)
      for (size_t m = 0; m < nm; ++m) {
        double2& a = P->bc_host[(2 * w) * nm + m];
        const double2 r = P->bc_host[(2 * w + 1) * nm + m];
        a = make_double2(a.x + r.x * el, a.y + r.y * el);
      }
    for (size_t m = 0; m < nm; ++m) {
      P->bc_host[(2 * wall) * nm + m] = v0[m];
      P->bc_host[(2 * wall + 1) * nm + m] = v1[m];
    }
    P->bc_tref = P->sim_time;
    const double zero = 0.0;
    TB_CUDA_TRY(cudaMemcpy(P->bcdyn.p, P->bc_host.data(), 4 * nm * sizeof(double2), cudaMemcpyHostToDevice));
    TB_CUDA_TRY(cudaMemcpy(P->t_dev.p, &zero, sizeof(double), cudaMemcpyHostToDevice));
  });
}

}  // extern "C"

namespace {

// Grid fields of a checkpoint, in order: b, u_x, (u_y), u_z, p.
int checkpoint_fields(const tb_plan* P) { return P->ndim == 3 ? 5 : 4; }
size_t grid_points(const tb_plan* P) { return (size_t)P->Nz * P->Ny * P->Nx; }

// 2D: coefficient plane (Nz, Nx/2+1) -> grid (Nz, Nx) on the plan's stream.
void grid_of_plane_2d(tb_plan* P, const double2* coeff, double* grid) {
  double2* mixed = P->tmpgrid.as<double2>();
  GemmBatch bt{};
  bt.item[0] = GemmItem{P->bwd.as<double>(), reinterpret_cast<const double*>(coeff), reinterpret_cast<double*>(mixed),
                        P->Nz, P->Nz, pad16k(P->Nz), GEMM_PLAIN, 0};
  launch_gemm_f64(bt, 1, 2 * P->Nk, 2 * P->Nk, 2 * P->Nk, P->Nz, P->st);
  launch_x_irfft(mixed, grid, P->Nz, P->Nx, P->fpN, P->twN.as<double2>(), P->st);
}

void plane_of_grid_2d(tb_plan* P, const double* grid, double2* coeff) {
  double2* mixed = P->tmpgrid.as<double2>();
  launch_x_rfft(grid, mixed, P->Nz, P->Nx, P->fpN, P->twN.as<double2>(), P->st);
  GemmBatch bt{};
  bt.item[0] = GemmItem{P->fE.as<double>(), reinterpret_cast<const double*>(mixed), reinterpret_cast<double*>(coeff),
                        P->Ke, P->Hz, pad16k(P->Hz), GEMM_MIRROR, 0};
  bt.item[1] = GemmItem{P->fO.as<double>(), reinterpret_cast<const double*>(mixed), reinterpret_cast<double*>(coeff),
                        P->Ko, P->Hz, pad16k(P->Hz), GEMM_MIRROR, 1};
  launch_gemm_f64(bt, P->Ko > 0 ? 2 : 1, 2 * P->Nk, 2 * P->Nk, 2 * P->Nk, P->Nz, P->st);
}

}  // namespace

extern "C" {

tb_status tb_checkpoint_stage(tb_plan* P, double* host_grid, size_t capacity, double* clock3) {
  if (!P || !host_grid) return TB_EINVAL;
  return guard(P->ctx, [&] {
    TB_REQUIRE(P->d.program == TB_PROGRAM_RBC, TB_ENOTSUPPORTED, "checkpoints of RBC plans");
    const int nf = checkpoint_fields(P);
    const size_t g = grid_points(P);
    TB_REQUIRE(capacity >= (size_t)nf * g, TB_EINVAL, "host buffer smaller than the checkpoint's grid fields");
    TB_CUDA_TRY(cudaSetDevice(P->ctx->device));
    if (!P->io_st) {
      TB_CUDA_TRY(cudaStreamCreateWithFlags(&P->io_st, cudaStreamNonBlocking));
      TB_CUDA_TRY(cudaEventCreateWithFlags(&P->io_ready, cudaEventDisableTiming));
      TB_CUDA_TRY(cudaEventCreateWithFlags(&P->io_done, cudaEventDisableTiming));
      TB_CUDA_TRY(cudaEventRecord(P->io_done, P->io_st));
    }
    if (P->stage_grid.bytes < (size_t)nf * g * sizeof(double)) {
      TB_CUDA_TRY(cudaStreamSynchronize(P->io_st));
      P->stage_grid.alloc((size_t)nf * g * sizeof(double));
    }
    double* stage = P->stage_grid.as<double>();
    // the previous checkpoint's copy must have left the staging buffer
    TB_CUDA_TRY(cudaStreamWaitEvent(P->st, P->io_done, 0));
    if (P->ndim == 3) {
      const int fields[5] = {TB_FIELD_B, TB_FIELD_UX, TB_FIELD_UY, TB_FIELD_UZ, TB_FIELD_P};
      for (int f = 0; f < nf; ++f) {
        rbc3d_state_get(P, fields[f], P->tmp3.as<double2>());
        rbc3d_transform_backward(P, P->tmp3.as<double2>(), stage + f * g);
      }
    } else {
      const int planes[4] = {0, 1, 2, 3};  // b, u_x, u_z, p
      for (int f = 0; f < nf; ++f) grid_of_plane_2d(P, P->Xp(planes[f]), stage + f * g);
    }
    check_launch("checkpoint staging");
    TB_CUDA_TRY(cudaEventRecord(P->io_ready, P->st));
    TB_CUDA_TRY(cudaStreamWaitEvent(P->io_st, P->io_ready, 0));
    TB_CUDA_TRY(cudaMemcpyAsync(host_grid, stage, (size_t)nf * g * sizeof(double), cudaMemcpyDeviceToHost,
                                P->io_st));
    TB_CUDA_TRY(cudaEventRecord(P->io_done, P->io_st));
    if (clock3) {
      clock3[0] = P->sim_time;
      clock3[1] = (double)P->iteration;
      clock3[2] = P->last_dt;
    }
  });
}

tb_status tb_checkpoint_wait(tb_plan* P) {
  if (!P) return TB_EINVAL;
  return guard(P->ctx, [&] {
    if (P->io_st) TB_CUDA_TRY(cudaStreamSynchronize(P->io_st));
  });
}

tb_status tb_checkpoint_load(tb_plan* P, const double* grid, int where, const double* clock3) {
  if (!P || !grid || !clock3) return TB_EINVAL;
  return guard(P->ctx, [&] {
    TB_REQUIRE(P->d.program == TB_PROGRAM_RBC, TB_ENOTSUPPORTED, "checkpoints of RBC plans");
    TB_REQUIRE(std::isfinite(clock3[0]) && clock3[1] >= 0, TB_EINVAL, "checkpoint clock must be finite");
    TB_CUDA_TRY(cudaSetDevice(P->ctx->device));
    const int nf = checkpoint_fields(P);
    const size_t g = grid_points(P);
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
    if (P->stage_grid.bytes < (size_t)nf * g * sizeof(double)) P->stage_grid.alloc((size_t)nf * g * sizeof(double));
    if (P->io_st) TB_CUDA_TRY(cudaStreamSynchronize(P->io_st));
    double* stage = P->stage_grid.as<double>();
    TB_CUDA_TRY(cudaMemcpy(stage, grid, (size_t)nf * g * sizeof(double),
                           where == TB_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
    // the taus and pressure history never enter a later step through M X, and
    // the multistep history restarts (the reference drops its timestepper state)
    TB_CUDA_TRY(cudaMemsetAsync(P->tau.p, 0, P->tau.bytes, P->st));
    if (P->ndim == 3) {
      const int fields[5] = {TB_FIELD_B, TB_FIELD_UX, TB_FIELD_UY, TB_FIELD_UZ, TB_FIELD_P};
      TB_CUDA_TRY(cudaMemsetAsync(P->X.p, 0, (size_t)P->nplanes * P->plane * sizeof(double2), P->st));
      for (int f = 0; f < nf; ++f) {
        rbc3d_transform_forward(P, stage + f * g, P->tmp3.as<double2>());
        rbc3d_state_set(P, fields[f], P->tmp3.as<double2>());
      }
    } else {
      for (int f = 0; f < nf; ++f) plane_of_grid_2d(P, stage + f * g, P->Xp(f));
    }
    check_launch("checkpoint load");
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
    P->sim_time = clock3[0];
    P->iteration = (long long)clock3[1];
    P->last_dt = clock3[2];
    P->ms_history = 0;
  });
}

tb_status tb_kernels_per_step(const tb_plan* P, int* n) {
  if (!P || !n) return TB_EINVAL;
  *n = P->kernels_per_step;
  return TB_OK;
}

tb_status tb_transform_forward(tb_plan* P, const double* grid, double* coeff, int nfields) {
  if (!P || !grid || !coeff || nfields < 1) return TB_EINVAL;
  if (P->ndim == 3)
    return guard(P->ctx, [&] {
      const size_t g = (size_t)P->Nz * P->Ny * P->Nx;
      for (int f = 0; f < nfields; ++f)
        rbc3d_transform_forward(P, grid + f * g, reinterpret_cast<double2*>(coeff) + f * P->plane);
      check_launch("transform forward");
      TB_CUDA_TRY(cudaStreamSynchronize(P->st));
    });
  return guard(P->ctx, [&] {
    const size_t gsz = (size_t)P->Nz * P->Nx;
    for (int f = 0; f < nfields; ++f) {
      double2* mixed = P->tmpgrid.as<double2>();
      launch_x_rfft(grid + f * gsz, mixed, P->Nz, P->Nx, P->fpN, P->twN.as<double2>(), P->st);
      GemmBatch bt{};
      bt.item[0] = GemmItem{P->fE.as<double>(), reinterpret_cast<const double*>(mixed), coeff + f * 2 * P->plane, P->Ke,
                            P->Hz, pad16k(P->Hz), GEMM_MIRROR, 0};
      bt.item[1] = GemmItem{P->fO.as<double>(), reinterpret_cast<const double*>(mixed), coeff + f * 2 * P->plane, P->Ko,
                            P->Hz, pad16k(P->Hz), GEMM_MIRROR, 1};
      launch_gemm_f64(bt, P->Ko > 0 ? 2 : 1, 2 * P->Nk, 2 * P->Nk, 2 * P->Nk, P->Nz, P->st);
      check_launch("transform forward");
    }
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  });
}

tb_status tb_transform_backward(tb_plan* P, const double* coeff, double* grid, int nfields) {
  if (!P || !grid || !coeff || nfields < 1) return TB_EINVAL;
  if (P->ndim == 3)
    return guard(P->ctx, [&] {
      const size_t g = (size_t)P->Nz * P->Ny * P->Nx;
      for (int f = 0; f < nfields; ++f)
        rbc3d_transform_backward(P, reinterpret_cast<const double2*>(coeff) + f * P->plane, grid + f * g);
      check_launch("transform backward");
      TB_CUDA_TRY(cudaStreamSynchronize(P->st));
    });
  return guard(P->ctx, [&] {
    const size_t gsz = (size_t)P->Nz * P->Nx;
    for (int f = 0; f < nfields; ++f) {
      double2* mixed = P->tmpgrid.as<double2>();
      GemmBatch bt{};
      bt.item[0] = GemmItem{P->bwd.as<double>(), coeff + f * 2 * P->plane, reinterpret_cast<double*>(mixed), P->Nz,
                            P->Nz, pad16k(P->Nz), GEMM_PLAIN, 0};
      launch_gemm_f64(bt, 1, 2 * P->Nk, 2 * P->Nk, 2 * P->Nk, P->Nz, P->st);
      launch_x_irfft(mixed, grid + f * gsz, P->Nz, P->Nx, P->fpN, P->twN.as<double2>(), P->st);
      check_launch("transform backward");
    }
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  });
}

tb_status tb_dealiased_multiply(tb_plan* P, const double* a, const double* b, double* out) {
  if (!P || !a || !b || !out) return TB_EINVAL;
  return guard(P->ctx, [&] {
    TB_REQUIRE(P->ndim == 2, TB_ENOTSUPPORTED, "2D plans only");
    launch_x_dealias_mul(a, b, out, P->Nz, P->Nx, P->M, P->fpN, P->twN.as<double2>(), P->fpM,
                         P->twM.as<double2>(), P->st);
    check_launch("dealiased multiply");
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  });
}

tb_status tb_rhs_advection(tb_plan* P, const double* coeff_in, double* coeff_out) {
  if (!P || !coeff_in || !coeff_out) return TB_EINVAL;
  return guard(P->ctx, [&] {
    TB_REQUIRE(P->ndim == 2, TB_ENOTSUPPORTED, "2D plans only");
    enqueue_rhs(P, reinterpret_cast<const double2*>(coeff_in), reinterpret_cast<double2*>(coeff_out), false);
    check_launch("rhs advection");
    TB_CUDA_TRY(cudaStreamSynchronize(P->st));
  });
}

}  // extern "C"
