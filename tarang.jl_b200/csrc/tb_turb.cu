// 2D decaying turbulence in FP32: vorticity q with streamfunction psi and
// velocity u = skew(grad psi), DiagonalIMEX_SBDF2 (examples/
// 2d_decaying_turbulence_gpu.jl; src/core/timesteppers/step_diagonal_imex.jl).
//
// Coefficients q^(kx, ky): rfft along x (kx = 0..Nx/2, Nyquist +Nx/2), fft
// along y in FFT order (ky = 0..Ny/2-1, -Ny/2..-1), unnormalised
// (basis_wavenumbers.jl:68-108).  Stored on the device transposed,
// [kx][ky] with ky fastest, so that the y transforms read whole columns.
//
// One RHS  F = -(u d_x q + v d_y q)  follows the reference's chain:
//   psi^ = -q^/k^2 (0 at k = 0)                  state_utils.jl:1059-1075
//   u^ = -i ky psi^, v^ = i kx psi^, d_x q^ = i kx q^, d_y q^ = i ky q^
//                                                lazy_rhs.jl:1190-1238
//   grid round trip of each factor: the kx = 0 and kx = Nx/2 columns lose
//   their non-Hermitian part in ky (irfft drops Im of DC and Nyquist)
//   3/2 padding in x and y with the even-N Nyquist split X/2 at +-N/2, product
//   on the padded grid, forward transform, fold of the -N/2 images into +N/2
//   and truncation                                nonlinear_padding.jl:182-443
// DiagonalIMEX_SBDF2 (step_diagonal_imex.jl:674-689, constant dt, L^ = nu k^2):
//   first step  q1 = (q0 + dt F0) / (1 + dt L^)
//   then        q_{n+1} = (2 q_n - q_{n-1}/2 + dt (2 F_n - F_{n-1})) / (3/2 + dt L^)
// DiagonalIMEX_RK222 / RK443 (_step_diagonal_imex_rk_impl!,
// step_diagonal_imex.jl:183-296; the full ESDIRK tableau, types.jl:511-620):
//   Y_s = q_n + dt sum_{j<s} (AE_sj F_j - AI_sj L^ Y_j),  Y_s /= 1 + dt AI_ss L^
//   F_s = RHS(Y_s);  q_{n+1} = q_n + dt sum_s (bE_s F_s - bI_s L^ Y_s)
// (a stage RHS whose weights are all zero, the first stage's, is skipped).
//
// Kernels per step: k_turb_yinv (per kx column: derived fields, projection,
// y padding, 4 inverse FFTs along y), transpose, k_turb_xpass (per padded y
// row: 2 packed inverse real FFTs along x, product, forward FFT, x
// truncation), transpose, k_turb_yfwd (per kx column: forward FFT along y,
// folds, truncation, SBDF update).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "tb_fft.cuh"
#include "tb_internal.h"
#include "tb_plan.h"
#include "tb_turb.h"

using namespace tb;
namespace F = tb::fftg;

struct tb_turb {
  tb_context* ctx = nullptr;
  int Nx = 0, Ny = 0, Mx = 0, My = 0, Kx = 0;
  double Lx = 0, Ly = 0, nu = 0;
  FftPlan fpMx{}, fpMy{};
  int nptx = 0, npty = 0;
  cudaStream_t st = nullptr;
  DevBuf Q[2], Fb;         // q_n / q_{n-1} (roles alternate), F_{n-1} (updated in place); [Kx][Ny] complex64
  DevBuf mix, mixT;        // 4 x [Kx][My] and 4 x [My][Kx]
  DevBuf pm, pmT;          // [My][Kx] and [Kx][My]
  DevBuf ptx, pty;         // per-pass twiddles (FP32) of the Mx and My plans
  // DiagonalIMEX RK (rk true): tableau and per-stage states / right-hand sides
  bool rk = false;
  int stages = 0;
  double AE[4][4] = {}, AI[4][4] = {}, bE[4] = {}, bI[4] = {};
  bool f_used[4] = {};
  DevBuf Ys[4], Fs[4];     // Y_s (s >= 1; Y_0 is q_n) and F_s where used
  int cur = 0;             // Q[cur] holds q_n
  long long iteration = 0;
  double graph_dt = -1.0;
  cudaGraphExec_t g[2] = {nullptr, nullptr};  // steady step with q_n in Q[0] / Q[1]

  ~tb_turb() {
    for (auto& e : g)
      if (e) cudaGraphExecDestroy(e);
    if (st) cudaStreamDestroy(st);
  }
};

namespace {

constexpr int kTurbThreads = 256;

struct TurbArgs {
  int Nx, Ny, Mx, My, Kx;
  float kx0, ky0, nu;
  FftPlan fpx, fpy;
  int nptx, npty;
  const float2* ptx;
  const float2* pty;
};

__device__ __forceinline__ float ky_of(int ky, int Ny) { return (float)(ky < Ny / 2 ? ky : ky - Ny); }

// Stage combination of the diagonal IMEX RK step over [kx][ky]:
//   out = (base + sum_t w_t (L^ if isL_t) src_t) / (1 + dgam L^),  L^ = nu k^2.
constexpr int kCombMax = 8;
struct TurbComb {
  const float2* base;
  const float2* src[kCombMax];
  float w[kCombMax];
  int isL[kCombMax];
  int n;
  float dgam;
  float2* out;
};

__global__ void __launch_bounds__(256) k_turb_combine(TurbArgs a, TurbComb c) {
  const size_t total = (size_t)a.Kx * a.Ny;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int kx = (int)(e / a.Ny), ky = (int)(e % a.Ny);
    const float kxv = a.kx0 * kx, kyv = a.ky0 * ky_of(ky, a.Ny);
    const float L = a.nu * (kxv * kxv + kyv * kyv);
    float2 acc = c.base[e];
#pragma unroll
    for (int t = 0; t < kCombMax; ++t) {
      if (t < c.n) {
        const float2 v = c.src[t][e];
        const float wt = c.isL[t] ? c.w[t] * L : c.w[t];
        acc = F::mk<float2>(fmaf(wt, v.x, acc.x), fmaf(wt, v.y, acc.y));
      }
    }
    if (c.dgam != 0.f) {
      const float den = 1.0f / (1.0f + c.dgam * L);
      acc = F::mk<float2>(acc.x * den, acc.y * den);
    }
    c.out[e] = acc;
  }
}

// Per kx column: the four factors u, v, d_x q, d_y q of the products, with the
// grid round trip's projection, the x Nyquist split and the y padding, inverse
// FFT along y; out: mix[f][kx][y], f = u, v, qx, qy.
__global__ void __launch_bounds__(kTurbThreads) k_turb_yinv(TurbArgs a, const float2* __restrict__ q,
                                                            float2* __restrict__ mix) {
  extern __shared__ float2 sm[];
  const int My = a.My, Ny = a.Ny, kx = blockIdx.x;
  const int Ms = (My + 7) & ~7;
  float2* A = sm;
  float2* B = sm + Ms;
  float2* qs = sm + 2 * Ms;        // the q^ column
  float2* pt = qs + Ny;            // twiddles of the My plan
  for (int t = threadIdx.x; t < a.npty; t += blockDim.x) pt[t] = a.pty[t];
  for (int t = threadIdx.x; t < Ny; t += blockDim.x) qs[t] = q[(size_t)kx * Ny + t];
  __syncthreads();
  const float kxv = a.kx0 * kx;
  const bool edge = (kx == 0) || (2 * kx == a.Nx);  // columns whose grid round trip is real
  const float xs = (2 * kx == a.Nx) ? 0.5f : 1.0f;  // even-N Nyquist split along x
  // q^ of the grid round trip: the kx = 0 / Nyquist columns lose their
  // non-Hermitian part before any derivative is taken
  auto qproj = [&](int ky) -> float2 {
    const float2 c = qs[ky];
    if (!edge) return c;
    const float2 w = qs[(Ny - ky) % Ny];
    return F::mk<float2>(0.5f * (c.x + w.x), 0.5f * (c.y - w.y));
  };
  auto factor = [&](int f, int ky) -> float2 {
    const float kyv = a.ky0 * ky_of(ky, Ny);
    const float2 c = qproj(ky);
    const float k2 = kxv * kxv + kyv * kyv;
    float2 psi = k2 > 1e-12f ? F::mk<float2>(-c.x / k2, -c.y / k2) : F::mk<float2>(0.f, 0.f);
    // i k z = (-k z.y, k z.x)
    if (f == 0) return F::mk<float2>(kyv * psi.y, -kyv * psi.x);   // -i ky psi
    if (f == 1) return F::mk<float2>(-kxv * psi.y, kxv * psi.x);   //  i kx psi
    if (f == 2) return F::mk<float2>(-kxv * c.y, kxv * c.x);       //  i kx q
    return F::mk<float2>(-kyv * c.y, kyv * c.x);                    //  i ky q
  };
  for (int f = 0; f < 4; ++f) {
    for (int y = threadIdx.x; y < My; y += blockDim.x) A[F::fidx<true>(y)] = F::mk<float2>(0.f, 0.f);
    __syncthreads();
    for (int ky = threadIdx.x; ky < Ny; ky += blockDim.x) {
      float2 v = factor(f, ky);
      v = F::scale(v, xs);
      if (2 * ky < Ny) {
        A[F::fidx<true>(ky)] = v;
      } else if (2 * ky == Ny) {
        const float2 h = F::scale(v, 0.5f);
        A[F::fidx<true>(Ny / 2)] = h;
        A[F::fidx<true>(My - Ny / 2)] = h;
      } else {
        A[F::fidx<true>(My - Ny + ky)] = v;
      }
    }
    __syncthreads();
    float2* R = F::fft<true>(A, B, a.fpy, pt, +1);
    float2* out = mix + ((size_t)f * a.Kx + kx) * My;
    for (int y = threadIdx.x; y < My; y += blockDim.x) out[y] = R[F::fidx<true>(y)];
    __syncthreads();
  }
}

// Batched transpose: in[b][R][C] -> out[b][C][R] (32 x 32 tiles).
__global__ void __launch_bounds__(256) k_transpose_c64(const float2* __restrict__ in, float2* __restrict__ out, int R,
                                                        int C) {
  __shared__ float2 tile[32][33];
  const size_t boff = (size_t)blockIdx.z * R * C;
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    if (r < R && c < C) tile[i][threadIdx.x] = in[boff + (size_t)r * C + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (r < R && c < C) out[boff + (size_t)c * R + r] = tile[threadIdx.x][i];
  }
}

// Per padded y row: u, v, d_x q, d_y q on the padded x grid (two packed inverse
// real FFTs), the product u d_x q + v d_y q, its forward FFT, bins 0..Nx/2.
__global__ void __launch_bounds__(kTurbThreads) k_turb_xpass(TurbArgs a, const float2* __restrict__ mixT,
                                                             float2* __restrict__ pm) {
  extern __shared__ float2 sm[];
  const int Mx = a.Mx, Kx = a.Kx, My = a.My, y = blockIdx.x;
  const int Ms = (Mx + 7) & ~7;
  float2* Z1 = sm;
  float2* Z2 = sm + Ms;
  float2* S1 = sm + 2 * Ms;
  float2* S2 = sm + 3 * Ms;
  float2* pt = sm + 4 * Ms;
  for (int t = threadIdx.x; t < a.nptx; t += blockDim.x) pt[t] = a.ptx[t];
  auto row = [&](int f) { return mixT + ((size_t)f * My + y) * Kx; };
  const float2 *ru = row(0), *rv = row(1), *rqx = row(2), *rqy = row(3);
  // half-spectrum bin k of a factor (zero past the data; DC and Nyquist kept
  // real, as the factor's own irfft on Nx points does)
  auto bin = [&](const float2* r, int k) -> float2 {
    if (k >= Kx) return F::mk<float2>(0.f, 0.f);
    float2 v = r[k];
    if (k == 0 || 2 * k == a.Nx) v.y = 0.f;
    return v;
  };
  for (int k = threadIdx.x; k <= Mx / 2; k += blockDim.x) {
    const float2 U = bin(ru, k), V = bin(rv, k), QX = bin(rqx, k), QY = bin(rqy, k);
    // spectrum of a + i b: A + i B at k, conj(A) + i conj(B) at Mx - k
    Z1[F::fidx<true>(k)] = F::mk<float2>(U.x - V.y, U.y + V.x);
    Z2[F::fidx<true>(k)] = F::mk<float2>(QX.x - QY.y, QX.y + QY.x);
    if (k > 0 && k < Mx / 2) {
      Z1[F::fidx<true>(Mx - k)] = F::mk<float2>(U.x + V.y, -U.y + V.x);
      Z2[F::fidx<true>(Mx - k)] = F::mk<float2>(QX.x + QY.y, -QX.y + QY.x);
    }
  }
  __syncthreads();
  float2* z1 = F::fft<true>(Z1, S1, a.fpx, pt, +1);
  float2* z2 = F::fft<true>(Z2, S2, a.fpx, pt, +1);
  float2* P = (z1 == Z1) ? S1 : Z1;
  float2* W = (z2 == Z2) ? S2 : Z2;
  for (int x = threadIdx.x; x < Mx; x += blockDim.x) {
    const int i = F::fidx<true>(x);
    const float2 s = z1[i], t = z2[i];
    P[i] = F::mk<float2>(s.x * t.x + s.y * t.y, 0.f);
  }
  __syncthreads();
  float2* C = F::fft<true>(P, W, a.fpx, pt, -1);
  for (int k = threadIdx.x; k < Kx; k += blockDim.x) pm[(size_t)y * Kx + k] = C[F::fidx<true>(k)];
}

// Per kx column: forward FFT along y, the Nyquist folds and truncation to Ny,
// F = -(...) / (Nx Ny Mx My), and the SBDF1 / SBDF2 update in place.
//   qn: q_n [Kx][Ny];  qo: q_{n-1} on entry, q_{n+1} on exit;  Fp: F_{n-1} on
//   entry, F_n on exit.  first: 1 SBDF1 startup (q_{n+1} written to qo),
//   0 SBDF2, 2 the right-hand side alone (Fp = F; qn and qo untouched).
__global__ void __launch_bounds__(kTurbThreads) k_turb_yfwd(TurbArgs a, const float2* __restrict__ pmT,
                                                            const float2* __restrict__ qn, float2* __restrict__ qo,
                                                            float2* __restrict__ Fp, float dt, int first) {
  extern __shared__ float2 sm[];
  const int My = a.My, Ny = a.Ny, kx = blockIdx.x;
  const int Ms = (My + 7) & ~7;
  float2* A = sm;
  float2* B = sm + Ms;
  float2* pt = sm + 2 * Ms;
  for (int t = threadIdx.x; t < a.npty; t += blockDim.x) pt[t] = a.pty[t];
  const float2* col = pmT + (size_t)kx * My;
  for (int y = threadIdx.x; y < My; y += blockDim.x) A[F::fidx<true>(y)] = col[y];
  __syncthreads();
  const float2* Q = F::fft<true>(A, B, a.fpy, pt, -1);
  const bool xnyq = (2 * kx == a.Nx);
  // Q'(y) with the x fold: Q(Nx/2, y) + conj(Q(Nx/2, -y))
  auto qf = [&](int yy) -> float2 {
    float2 v = Q[F::fidx<true>(yy)];
    if (xnyq) {
      const float2 w = Q[F::fidx<true>((My - yy) % My)];
      v = F::mk<float2>(v.x + w.x, v.y - w.y);
    }
    return v;
  };
  const float sc = -1.0f / ((float)a.Nx * (float)Ny * (float)a.Mx * (float)My);
  const float kxv = a.kx0 * kx;
  for (int ky = threadIdx.x; ky < Ny; ky += blockDim.x) {
    float2 r;
    if (2 * ky < Ny) {
      r = qf(ky);
    } else if (2 * ky == Ny) {
      r = F::add(qf(Ny / 2), qf(My - Ny / 2));
    } else {
      r = qf(My - Ny + ky);
    }
    const float2 Fn = F::scale(r, sc);
    const size_t e = (size_t)kx * Ny + ky;
    if (first == 2) {
      Fp[e] = Fn;
      continue;
    }
    const float kyv = a.ky0 * ky_of(ky, Ny);
    const float L = a.nu * (kxv * kxv + kyv * kyv);
    const float2 q0 = qn[e];
    float2 q1;
    if (first) {
      const float den = 1.0f / (1.0f + dt * L);
      q1 = F::mk<float2>((q0.x + dt * Fn.x) * den, (q0.y + dt * Fn.y) * den);
    } else {
      const float2 qm = qo[e], Fm = Fp[e];
      const float den = 1.0f / (1.5f + dt * L);
      q1 = F::mk<float2>((2.0f * q0.x - 0.5f * qm.x + dt * (2.0f * Fn.x - Fm.x)) * den,
                         (2.0f * q0.y - 0.5f * qm.y + dt * (2.0f * Fn.y - Fm.y)) * den);
    }
    qo[e] = q1;
    Fp[e] = Fn;
  }
}

size_t yinv_smem(const tb_turb* T) {
  const size_t Ms = (T->My + 7) & ~7;
  return (2 * Ms + T->Ny + T->npty) * sizeof(float2);
}
size_t xpass_smem(const tb_turb* T) {
  const size_t Ms = (T->Mx + 7) & ~7;
  return (4 * Ms + T->nptx) * sizeof(float2);
}
size_t yfwd_smem(const tb_turb* T) {
  const size_t Ms = (T->My + 7) & ~7;
  return (2 * Ms + T->npty) * sizeof(float2);
}

TurbArgs args_of(const tb_turb* T) {
  TurbArgs a{};
  a.Nx = T->Nx;
  a.Ny = T->Ny;
  a.Mx = T->Mx;
  a.My = T->My;
  a.Kx = T->Kx;
  a.kx0 = (float)(2.0 * M_PI / T->Lx);
  a.ky0 = (float)(2.0 * M_PI / T->Ly);
  a.nu = (float)T->nu;
  a.fpx = T->fpMx;
  a.fpy = T->fpMy;
  a.nptx = T->nptx;
  a.npty = T->npty;
  a.ptx = T->ptx.as<float2>();
  a.pty = T->pty.as<float2>();
  return a;
}

// The RHS chain on q, ending in k_turb_yfwd with mode first (see there).
void enqueue_rhs(tb_turb* T, const float2* q, float2* qo, float2* Fp, double dt, int first) {
  const TurbArgs a = args_of(T);
  float2* mix = T->mix.as<float2>();
  float2* mixT = T->mixT.as<float2>();
  k_turb_yinv<<<T->Kx, kTurbThreads, yinv_smem(T), T->st>>>(a, q, mix);
  dim3 tb(32, 8);
  k_transpose_c64<<<dim3((T->My + 31) / 32, (T->Kx + 31) / 32, 4), tb, 0, T->st>>>(mix, mixT, T->Kx, T->My);
  k_turb_xpass<<<T->My, kTurbThreads, xpass_smem(T), T->st>>>(a, mixT, T->pm.as<float2>());
  k_transpose_c64<<<dim3((T->Kx + 31) / 32, (T->My + 31) / 32, 1), tb, 0, T->st>>>(T->pm.as<float2>(),
                                                                                   T->pmT.as<float2>(), T->My, T->Kx);
  k_turb_yfwd<<<T->Kx, kTurbThreads, yfwd_smem(T), T->st>>>(a, T->pmT.as<float2>(), q, qo, Fp, (float)dt, first);
}

void launch_combine(tb_turb* T, const TurbComb& c) {
  const size_t total = (size_t)T->Kx * T->Ny;
  int blocks = (int)((total + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_turb_combine<<<blocks, 256, 0, T->st>>>(args_of(T), c);
}

// One DiagonalIMEX RK step from Q[cur] into Q[1 - cur].
void enqueue_rk_step(tb_turb* T, double dt) {
  float2* qn = T->Q[T->cur].as<float2>();
  float2* qo = T->Q[1 - T->cur].as<float2>();
  const float2* Y[4] = {qn, nullptr, nullptr, nullptr};
  auto add = [&](TurbComb& c, const float2* src, double w, int isL) {
    if (c.n >= kCombMax) throw Error{TB_EINVAL, "too many stage terms"};
    c.src[c.n] = src;
    c.w[c.n] = (float)w;
    c.isL[c.n] = isL;
    ++c.n;
  };
  const int s = T->stages;
  for (int i = 0; i < s; ++i) {
    if (i > 0) {
      TurbComb c{};
      c.base = qn;
      for (int j = 0; j < i; ++j) {
        if (std::fabs(T->AE[i][j]) > 1e-14) add(c, T->Fs[j].as<float2>(), dt * T->AE[i][j], 0);
        if (std::fabs(T->AI[i][j]) > 1e-14) add(c, Y[j], -dt * T->AI[i][j], 1);
      }
      c.dgam = std::fabs(T->AI[i][i]) > 1e-14 ? (float)(dt * T->AI[i][i]) : 0.f;
      c.out = T->Ys[i].as<float2>();
      launch_combine(T, c);
      Y[i] = T->Ys[i].as<float2>();
    }
    if (T->f_used[i]) enqueue_rhs(T, Y[i], nullptr, T->Fs[i].as<float2>(), dt, 2);
  }
  TurbComb c{};
  c.base = qn;
  for (int i = 0; i < s; ++i) {
    if (std::fabs(T->bE[i]) > 1e-14) add(c, T->Fs[i].as<float2>(), dt * T->bE[i], 0);
    if (std::fabs(T->bI[i]) > 1e-14) add(c, Y[i], -dt * T->bI[i], 1);
  }
  c.dgam = 0.f;
  c.out = qo;
  launch_combine(T, c);
}

void enqueue_step(tb_turb* T, double dt, int first) {
  if (T->rk) {
    enqueue_rk_step(T, dt);
    return;
  }
  float2* qn = T->Q[T->cur].as<float2>();
  float2* qo = T->Q[1 - T->cur].as<float2>();
  enqueue_rhs(T, qn, qo, T->Fb.as<float2>(), dt, first);
}

std::vector<float2> pass_twiddles_f(const FftPlan& fp) {
  std::vector<float2> t;
  const long double pi = 3.141592653589793238462643383279502884L;
  int Ns = 1;
  for (int s = 0; s < fp.nstages; ++s) {
    const int R = fp.radix[s];
    const int tstride = fp.n / (Ns * R);
    for (int j = 0; j < Ns; ++j) {
      const long double ang = -2.0L * pi * (long double)(j * tstride) / (long double)fp.n;
      t.push_back(make_float2((float)cosl(ang), (float)sinl(ang)));
    }
    Ns *= R;
  }
  return t;
}

int padded_len(int n) {
  int m = (int)std::ceil(1.5 * n);
  return (m % 2) ? m + 1 : m;
}

cudaGraphExec_t capture(tb_turb* T, double dt) {
  cudaGraph_t g = nullptr;
  TB_CUDA_TRY(cudaStreamBeginCapture(T->st, cudaStreamCaptureModeThreadLocal));
  enqueue_step(T, dt, 0);
  TB_CUDA_TRY(cudaStreamEndCapture(T->st, &g));
  cudaGraphExec_t ex = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) throw Error{TB_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
  return ex;
}

}  // namespace

size_t tb::turb_estimate_bytes(int Nx, int Ny, int timestepper) {
  const size_t Kx = Nx / 2 + 1, Mx = padded_len(Nx), My = padded_len(Ny);
  (void)Mx;
  // SBDF2: q_n, q_{n-1}, F_{n-1}; RK: q_n, q_{n+1} and up to 3 stage states
  // and 3 stage right-hand sides (4 stages, the first state and RHS not kept)
  const size_t specs = timestepper == TB_SBDF2 ? 3 : (timestepper == TB_RK222 ? 6 : 8);
  return sizeof(float2) * (specs * Kx * Ny + 8 * Kx * My + 2 * Kx * My) + (4u << 20);
}

tb_turb* tb::turb_create(tb_context* ctx, const tb_problem_desc& d, const double* q0) {
  TB_REQUIRE(d.program == TB_PROGRAM_TURB2D, TB_EINVAL, "not a turbulence descriptor");
  TB_REQUIRE(d.Nx >= 8 && d.Ny >= 8 && d.Nx % 2 == 0 && d.Ny % 2 == 0, TB_EINVAL, "Nx, Ny must be even and >= 8");
  TB_REQUIRE(d.Nx <= 2048 && d.Ny <= 2048, TB_ENOTSUPPORTED, "Nx, Ny above 2048");
  TB_REQUIRE(d.Lx > 0 && d.Ly > 0 && d.nu >= 0, TB_EINVAL, "bad lengths or viscosity");
  TB_REQUIRE(std::fabs(d.dealias - 1.5) < 1e-12, TB_ENOTSUPPORTED, "only dealias = 3/2 is implemented");
  TB_REQUIRE(q0 != nullptr, TB_EINVAL, "null initial vorticity");
  TB_REQUIRE(d.timestepper == TB_SBDF2 || d.timestepper == TB_RK222 || d.timestepper == TB_RK443, TB_ENOTSUPPORTED,
             "turbulence steps: DiagonalIMEX SBDF2, RK222 or RK443");
  auto T = std::make_unique<tb_turb>();
  if (d.timestepper != TB_SBDF2) {
    const Tableau tb_ = tableau(d.timestepper);
    T->rk = true;
    T->stages = tb_.s;
    for (int i = 0; i < tb_.s; ++i) {
      T->bE[i] = tb_.bE[i];
      T->bI[i] = tb_.bI[i];
      for (int j = 0; j < tb_.s; ++j) {
        T->AE[i][j] = tb_.AE[i][j];
        T->AI[i][j] = tb_.AI[i][j];
      }
    }
    // F_s is computed only where a later stage or the update weighs it
    for (int i = 0; i < tb_.s; ++i) {
      bool used = std::fabs(tb_.bE[i]) > 1e-14;
      for (int k = i + 1; k < tb_.s; ++k) used = used || std::fabs(tb_.AE[k][i]) > 1e-14;
      T->f_used[i] = used;
    }
  }
  T->ctx = ctx;
  T->Nx = d.Nx;
  T->Ny = d.Ny;
  T->Mx = padded_len(d.Nx);
  T->My = padded_len(d.Ny);
  T->Kx = d.Nx / 2 + 1;
  T->Lx = d.Lx;
  T->Ly = d.Ly;
  T->nu = d.nu;
  TB_REQUIRE(make_fft_plan(T->Mx, &T->fpMx) && make_fft_plan(T->My, &T->fpMy), TB_ENOTSUPPORTED,
             "Nx, Ny must be of the form 2^a 3^b");
  TB_CUDA_TRY(cudaSetDevice(ctx->device));
  TB_CUDA_TRY(create_work_stream(&T->st));
  const size_t spec = (size_t)T->Kx * T->Ny * sizeof(float2);
  for (auto& b : T->Q) b.alloc(spec);
  if (T->rk) {
    for (int i = 1; i < T->stages; ++i) T->Ys[i].alloc(spec);
    for (int i = 0; i < T->stages; ++i)
      if (T->f_used[i]) T->Fs[i].alloc(spec);
  } else {
    T->Fb.alloc(spec);
  }
  T->mix.alloc(4 * (size_t)T->Kx * T->My * sizeof(float2));
  T->mixT.alloc(T->mix.bytes);
  T->pm.alloc((size_t)T->Kx * T->My * sizeof(float2));
  T->pmT.alloc(T->pm.bytes);
  upload(T->ptx, pass_twiddles_f(T->fpMx));
  upload(T->pty, pass_twiddles_f(T->fpMy));
  T->nptx = F::pass_twiddle_count(T->fpMx);
  T->npty = F::pass_twiddle_count(T->fpMy);
  TB_REQUIRE(xpass_smem(T.get()) <= 227 * 1024 && yinv_smem(T.get()) <= 227 * 1024, TB_ENOTSUPPORTED,
             "turbulence grid too large for the shared-memory transforms");
  TB_CUDA_TRY(cudaFuncSetAttribute(k_turb_yinv, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  TB_CUDA_TRY(cudaFuncSetAttribute(k_turb_xpass, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  TB_CUDA_TRY(cudaFuncSetAttribute(k_turb_yfwd, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  turb_set(T.get(), q0);
  return T.release();
}

// Vorticity coefficients from the reference layout (Kx, Ny), x fastest, into
// Q[0] = q_n (device [kx][ky]); the step history restarts.  Everything runs on
// the plan's own (non-blocking) stream, so the next step is ordered after it.
void tb::turb_set(tb_turb* T, const double* q0) {
  const size_t spec = (size_t)T->Kx * T->Ny * sizeof(float2);
  std::vector<float2> h((size_t)T->Kx * T->Ny);
  for (int ky = 0; ky < T->Ny; ++ky)
    for (int kx = 0; kx < T->Kx; ++kx) {
      const size_t s = (size_t)ky * T->Kx + kx;
      h[(size_t)kx * T->Ny + ky] = make_float2((float)q0[2 * s], (float)q0[2 * s + 1]);
    }
  TB_CUDA_TRY(cudaStreamSynchronize(T->st));  // no step still reads the buffers
  TB_CUDA_TRY(cudaMemcpyAsync(T->Q[0].p, h.data(), spec, cudaMemcpyHostToDevice, T->st));
  TB_CUDA_TRY(cudaMemsetAsync(T->Q[1].p, 0, spec, T->st));
  if (T->Fb.p) TB_CUDA_TRY(cudaMemsetAsync(T->Fb.p, 0, spec, T->st));
  TB_CUDA_TRY(cudaStreamSynchronize(T->st));
  T->cur = 0;
  T->iteration = 0;
}

void tb::turb_destroy(tb_turb* T) { delete T; }

cudaStream_t tb::turb_stream(const tb_turb* T) { return T->st; }

void tb::turb_prepare(tb_turb* T, double dt) {
  if (T->graph_dt == dt) return;
  TB_CUDA_TRY(cudaSetDevice(T->ctx->device));
  TB_CUDA_TRY(cudaStreamSynchronize(T->st));
  for (auto& e : T->g)
    if (e) cudaGraphExecDestroy(e), e = nullptr;
  const int keep = T->cur;
  for (int c = 0; c < 2; ++c) {
    T->cur = c;
    T->g[c] = capture(T, dt);
  }
  T->cur = keep;
  T->graph_dt = dt;
}

void tb::turb_launch_steps(tb_turb* T, double dt, int steps) {
  for (int i = 0; i < steps; ++i) {
    if (T->iteration == 0) {
      enqueue_step(T, dt, 1);
    } else {
      turb_prepare(T, dt);
      TB_CUDA_TRY(cudaGraphLaunch(T->g[T->cur], T->st));
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw Error{TB_ECUDA, std::string("turbulence step: ") + cudaGetErrorString(e)};
    T->cur = 1 - T->cur;
    T->iteration += 1;
  }
}

size_t tb::turb_device_bytes(const tb_turb* T) {
  size_t b = T->Q[0].bytes + T->Q[1].bytes + T->Fb.bytes + T->mix.bytes + T->mixT.bytes + T->pm.bytes +
             T->pmT.bytes + T->ptx.bytes + T->pty.bytes;
  for (int i = 0; i < 4; ++i) b += T->Ys[i].bytes + T->Fs[i].bytes;
  return b;
}

size_t tb::turb_field_doubles(const tb_turb* T) { return 2 * (size_t)T->Kx * T->Ny; }

void tb::turb_fetch(tb_turb* T, double* host) {
  std::vector<float2> h((size_t)T->Kx * T->Ny);
  TB_CUDA_TRY(cudaMemcpyAsync(h.data(), T->Q[T->cur].p, h.size() * sizeof(float2), cudaMemcpyDeviceToHost, T->st));
  TB_CUDA_TRY(cudaStreamSynchronize(T->st));
  for (int ky = 0; ky < T->Ny; ++ky)
    for (int kx = 0; kx < T->Kx; ++kx) {
      const float2 v = h[(size_t)kx * T->Ny + ky];
      const size_t s = (size_t)ky * T->Kx + kx;
      host[2 * s] = v.x;
      host[2 * s + 1] = v.y;
    }
}

extern "C" {

tb_status tb_turb_create(tb_context* ctx, const tb_problem_desc* desc, const double* q0_spec, tb_turb** out) {
  if (!ctx || !desc || !out) return TB_EINVAL;
  *out = nullptr;
  return guarded(ctx, [&] { *out = turb_create(ctx, *desc, q0_spec); });
}

tb_status tb_turb_destroy(tb_turb* T) {
  if (!T) return TB_EINVAL;
  cudaStreamSynchronize(T->st);
  turb_destroy(T);
  return TB_OK;
}

tb_status tb_turb_step(tb_turb* T, double dt, int nsteps) {
  if (!T) return TB_EINVAL;
  return guarded(T->ctx, [&] {
    TB_REQUIRE(dt > 0 && std::isfinite(dt) && nsteps >= 0, TB_EINVAL, "dt must be positive, nsteps >= 0");
    TB_CUDA_TRY(cudaSetDevice(T->ctx->device));
    turb_launch_steps(T, dt, nsteps);
    TB_CUDA_TRY(cudaStreamSynchronize(T->st));
  });
}

tb_status tb_turb_set_vorticity(tb_turb* T, const double* host) {
  if (!T || !host) return TB_EINVAL;
  return guarded(T->ctx, [&] {
    TB_CUDA_TRY(cudaSetDevice(T->ctx->device));
    turb_set(T, host);
  });
}

tb_status tb_turb_get_vorticity(tb_turb* T, double* host) {
  if (!T || !host) return TB_EINVAL;
  return guarded(T->ctx, [&] { turb_fetch(T, host); });
}

}  // extern "C"
