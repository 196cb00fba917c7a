// Tau-system kernels: factorisation of the per-mode bordered banded systems,
// the batched solve, and the fused stage updates of the IMEX steppers.
//
// Stage algebra (src/core/timesteppers/step_subproblem_rk.jl:393-739):
//   rhs_i = M X_n + dt sum_j (aE_ij F_j - aI_ij L X_j);  rhs_i[bc] = dt aI_ii F_alg
//   (M + dt aI_ii L) X_i = rhs_i   (a_ii = 0: min-norm mass solve)
//   X_{n+1} = pinv(M) (M X_n + dt sum_s (bE_s F_s - bI_s L X_s))
// All stage vectors are held in C^(2) row space (the bulk rows left-multiplied
// by S = S1 S0).  L X_i is recovered from the solve itself,
//   L X_i = (rhs_i - M X_i) / (dt aI_ii)
// minus L applied to the imaginary DC/Nyquist parts that the reference's
// grid round trip discards before it re-gathers X_i
// (step_subproblem_rk_batched.jl:33-37).
#include <cuda_runtime.h>

#include "tb_kernels.cuh"

namespace tb {

namespace {

constexpr int NBMAX = 4;

__device__ __forceinline__ double coef_val(const Coef& c, double alpha, double beta, double kx) {
  return alpha * c.m + beta * (c.l0 + kx * c.l1 + kx * kx * c.l2);
}

__device__ __forceinline__ double2 cfma(double a, double2 x, double2 acc) {
  return make_double2(fma(a, x.x, acc.x), fma(a, x.y, acc.y));
}

__device__ __forceinline__ bool realified(int unk) {
  return unk == UK_UX || unk == UK_TAU0 + 3 || unk == UK_TAU0 + 5;
}

// ---------------------------------------------------------------------------
// Factorisation: one thread per (mode, class).  Banded LU with partial
// pivoting restricted to the band of the bulk rows; the boundary rows are
// eliminated alongside as a dense border and leave an nb x nb Schur
// complement, inverted explicitly.
// ---------------------------------------------------------------------------
template <int KL, int KU>
__global__ void __launch_bounds__(64) k_tau_factor(TauArgs a, int nmax) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (m >= a.Nk) return;
  const ClassDev& C = a.cls[c];
  const int n = C.n, nb = C.nb;
  constexpr int WW = 2 * KL + KU + 1;
  constexpr int W1 = KL + KU + 1;
  const int Nk = a.Nk;
  const double kx = a.k0 * m;
  const bool zmode = (m == 0);
  const size_t per = (size_t)nmax * WW + (size_t)nmax * NBMAX + (size_t)NBMAX * nmax + NBMAX * NBMAX;
  double* W = a.scratch + ((size_t)c * Nk + m) * per;
  double* Bd = W + (size_t)nmax * WW;
  double* Cr = Bd + (size_t)nmax * NBMAX;
  double* C1 = Cr + (size_t)NBMAX * nmax;
  const int cw = C.kl + C.ku + 1;
  for (int r = 0; r < n; ++r) {
    for (int d = 0; d < WW; ++d) W[(size_t)r * WW + d] = 0.0;
    for (int d = 0; d < cw; ++d) {
      int col = r + d - C.kl;
      if (col < 0 || col >= n) continue;
      W[(size_t)r * WW + (col - r + KL)] = coef_val(C.band[(size_t)r * cw + d], a.alpha, a.beta, kx);
    }
    for (int b = 0; b < nb; ++b) Bd[(size_t)r * NBMAX + b] = coef_val(C.bord[(size_t)r * nb + b], a.alpha, a.beta, kx);
  }
  for (int q = 0; q < nb; ++q) {
    for (int col = 0; col < n; ++col)
      Cr[(size_t)q * nmax + col] = a.beta * (zmode ? C.c2_z : C.c2_nz)[(size_t)q * n + col];
    for (int b = 0; b < nb; ++b) C1[q * NBMAX + b] = a.beta * (zmode ? C.c1_z : C.c1_nz)[q * nb + b];
  }
  for (int j = 0; j < n; ++j) {
    const int ilast = min(j + KL, n - 1);
    const int clast = min(j + KL + KU, n - 1);
    int p = j;
    double best = fabs(W[(size_t)j * WW + KL]);
    for (int i = j + 1; i <= ilast; ++i) {
      double v = fabs(W[(size_t)i * WW + (j - i + KL)]);
      if (v > best) {
        best = v;
        p = i;
      }
    }
    if (!(best > 0.0) || !isfinite(best)) {
      atomicMin(a.err_mode, m);
      return;
    }
    if (p != j) {
      for (int cc = j; cc <= clast; ++cc) {
        double t = W[(size_t)j * WW + (cc - j + KL)];
        W[(size_t)j * WW + (cc - j + KL)] = W[(size_t)p * WW + (cc - p + KL)];
        W[(size_t)p * WW + (cc - p + KL)] = t;
      }
      for (int b = 0; b < nb; ++b) {
        double t = Bd[(size_t)j * NBMAX + b];
        Bd[(size_t)j * NBMAX + b] = Bd[(size_t)p * NBMAX + b];
        Bd[(size_t)p * NBMAX + b] = t;
      }
    }
    C.piv[(size_t)j * Nk + m] = (unsigned char)(p - j);
    const double dinv = 1.0 / W[(size_t)j * WW + KL];
    for (int t = 0; t < KL; ++t) {
      const int i = j + 1 + t;
      double l = 0.0;
      if (i <= ilast) {
        l = W[(size_t)i * WW + (j - i + KL)] * dinv;
        W[(size_t)i * WW + (j - i + KL)] = 0.0;
        for (int cc = j + 1; cc <= clast; ++cc)
          W[(size_t)i * WW + (cc - i + KL)] -= l * W[(size_t)j * WW + (cc - j + KL)];
        for (int b = 0; b < nb; ++b) Bd[(size_t)i * NBMAX + b] -= l * Bd[(size_t)j * NBMAX + b];
      }
      C.Lm[((size_t)j * KL + t) * Nk + m] = l;
    }
    for (int q = 0; q < nb; ++q) {
      const double cq = Cr[(size_t)q * nmax + j] * dinv;
      Cr[(size_t)q * nmax + j] = 0.0;
      for (int cc = j + 1; cc <= clast; ++cc) Cr[(size_t)q * nmax + cc] -= cq * W[(size_t)j * WW + (cc - j + KL)];
      for (int b = 0; b < nb; ++b) C1[q * NBMAX + b] -= cq * Bd[(size_t)j * NBMAX + b];
      C.Cm[((size_t)j * nb + q) * Nk + m] = cq;
    }
    C.U[((size_t)j * W1 + 0) * Nk + m] = dinv;
    for (int t = 1; t < W1; ++t)
      C.U[((size_t)j * W1 + t) * Nk + m] = (j + t < n) ? W[(size_t)j * WW + KL + t] : 0.0;
    for (int b = 0; b < nb; ++b) C.Bd[((size_t)j * nb + b) * Nk + m] = Bd[(size_t)j * NBMAX + b];
  }
  // invert the nb x nb Schur complement (Gauss-Jordan, partial pivoting)
  double Aug[NBMAX][2 * NBMAX];
  for (int q = 0; q < NBMAX; ++q)
    for (int b = 0; b < 2 * NBMAX; ++b) Aug[q][b] = 0.0;
  for (int q = 0; q < nb; ++q) {
    for (int b = 0; b < nb; ++b) Aug[q][b] = C1[q * NBMAX + b];
    Aug[q][NBMAX + q] = 1.0;
  }
  double scale = 0.0;
  for (int q = 0; q < nb; ++q)
    for (int b = 0; b < nb; ++b) scale = fmax(scale, fabs(Aug[q][b]));
  for (int col = 0; col < nb; ++col) {
    int p = col;
    for (int q = col + 1; q < nb; ++q)
      if (fabs(Aug[q][col]) > fabs(Aug[p][col])) p = q;
    if (!(fabs(Aug[p][col]) > 1e-14 * scale) || !isfinite(Aug[p][col])) {
      atomicMin(a.err_mode, m);
      return;
    }
    if (p != col)
      for (int b = 0; b < 2 * NBMAX; ++b) {
        double t = Aug[col][b];
        Aug[col][b] = Aug[p][b];
        Aug[p][b] = t;
      }
    const double inv = 1.0 / Aug[col][col];
    for (int b = 0; b < 2 * NBMAX; ++b) Aug[col][b] *= inv;
    for (int q = 0; q < nb; ++q) {
      if (q == col) continue;
      const double f = Aug[q][col];
      if (f != 0.0)
        for (int b = 0; b < 2 * NBMAX; ++b) Aug[q][b] -= f * Aug[col][b];
    }
  }
  for (int q = 0; q < nb; ++q)
    for (int b = 0; b < nb; ++b) C.Sinv[((size_t)q * nb + b) * Nk + m] = Aug[q][NBMAX + b];
}

// ---------------------------------------------------------------------------
// Solve: one thread per (mode, class); the real and imaginary parts of the
// right-hand side are the two columns of a double2.
// ---------------------------------------------------------------------------
template <int KL, int KU>
__global__ void __launch_bounds__(128) k_tau_solve(TauArgs a) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (m >= a.Nk) return;
  const ClassDev& C = a.cls[c];
  const int n = C.n, nb = C.nb;
  const int Nk = a.Nk, Nz = a.Nz;
  constexpr int W1 = KL + KU + 1;
  auto addr = [&](int unk, int k) -> double2* {
    return unk < 4 ? a.X + ((size_t)unk * Nz + k) * Nk + m : a.tau + (size_t)(unk - UK_TAU0) * Nk + m;
  };
  auto load_rhs = [&](int r) -> double2 {
    const int e = C.row_eq[r], k = C.row_k[r];
    double2 v = a.rhsP[((size_t)e * Nz + k) * Nk + m];
    if (e == EQ_MX) v = make_double2(v.y, -v.x);  // row scaled by -i
    return v;
  };
  double2 y[KL + 1];
#pragma unroll
  for (int t = 0; t <= KL; ++t) y[t] = (t < n) ? load_rhs(t) : make_double2(0.0, 0.0);
  double2 z[NBMAX];
#pragma unroll
  for (int b = 0; b < NBMAX; ++b) z[b] = make_double2((b < nb && m == 0) ? a.beta * C.bc_rhs[b] : 0.0, 0.0);
  for (int j = 0; j < n; ++j) {
    const int p = C.piv[(size_t)j * Nk + m];
    double2 yj = y[0];
#pragma unroll
    for (int t = 1; t <= KL; ++t)
      if (t == p) {
        yj = y[t];
        y[t] = y[0];
      }
    *addr(C.col_unk[j], C.col_k[j]) = yj;
#pragma unroll
    for (int t = 1; t <= KL; ++t) y[t] = cfma(-C.Lm[((size_t)j * KL + (t - 1)) * Nk + m], yj, y[t]);
#pragma unroll
    for (int b = 0; b < NBMAX; ++b)
      if (b < nb) z[b] = cfma(-C.Cm[((size_t)j * nb + b) * Nk + m], yj, z[b]);
#pragma unroll
    for (int t = 0; t < KL; ++t) y[t] = y[t + 1];
    y[KL] = (j + KL + 1 < n) ? load_rhs(j + KL + 1) : make_double2(0.0, 0.0);
  }
  double2 x1[NBMAX];
#pragma unroll
  for (int q = 0; q < NBMAX; ++q) {
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int b = 0; b < NBMAX; ++b)
      if (q < nb && b < nb) acc = cfma(C.Sinv[((size_t)q * nb + b) * Nk + m], z[b], acc);
    x1[q] = acc;
  }
  double2 xw[W1];
#pragma unroll
  for (int t = 0; t < W1; ++t) xw[t] = make_double2(0.0, 0.0);
  for (int j = n - 1; j >= 0; --j) {
    const int unk = C.col_unk[j];
    double2* ptr = addr(unk, C.col_k[j]);
    double2 s = *ptr;
#pragma unroll
    for (int t = 1; t < W1; ++t) s = cfma(-C.U[((size_t)j * W1 + t) * Nk + m], xw[t], s);
#pragma unroll
    for (int b = 0; b < NBMAX; ++b)
      if (b < nb) s = cfma(-C.Bd[((size_t)j * nb + b) * Nk + m], x1[b], s);
    const double dinv = C.U[((size_t)j * W1) * Nk + m];
    const double2 xj = make_double2(s.x * dinv, s.y * dinv);
    *ptr = realified(unk) ? make_double2(-xj.y, xj.x) : xj;
#pragma unroll
    for (int t = W1 - 1; t >= 2; --t) xw[t] = xw[t - 1];
    xw[1] = xj;
  }
  for (int b = 0; b < nb; ++b) {
    const int unk = C.left_unk[b];
    const double2 v = x1[b];
    *addr(unk, C.left_k[b]) = realified(unk) ? make_double2(-v.y, v.x) : v;
  }
}

__global__ void k_lincomb(LinComb lc, double2* __restrict__ out, long long count) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    double2 acc = make_double2(0.0, 0.0);
    for (int t = 0; t < lc.n; ++t) acc = cfma(lc.w[t], lc.in[t][i], acc);
    out[i] = acc;
  }
}

__device__ __forceinline__ double2 proj(double2 v, bool p) { return p ? make_double2(v.x, 0.0) : v; }

__global__ void k_mass_apply(const double2* __restrict__ X, double2* __restrict__ MX, const double* __restrict__ s3,
                             int Nz, int Nk, int Nx, int project) {
  const long long total = (long long)Nz * Nk;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / Nk), m = (int)(i % Nk);
    const bool pj = project && (m == 0 || 2 * m == Nx);
    const double s0 = s3[3 * k], s1 = s3[3 * k + 1], s2 = s3[3 * k + 2];
    MX[i] = make_double2(0.0, 0.0);
    for (int f = 0; f < 3; ++f) {
      const double2* Xf = X + (size_t)f * Nz * Nk;
      double2 acc = make_double2(0.0, 0.0);
      acc = cfma(s0, proj(Xf[(size_t)k * Nk + m], pj), acc);
      if (k + 2 < Nz) acc = cfma(s1, proj(Xf[(size_t)(k + 2) * Nk + m], pj), acc);
      if (k + 4 < Nz) acc = cfma(s2, proj(Xf[(size_t)(k + 4) * Nk + m], pj), acc);
      MX[(size_t)(1 + f) * Nz * Nk + i] = acc;
    }
  }
}

__global__ void k_lx_finalize(double2* __restrict__ LX, const double2* __restrict__ X, const double* __restrict__ s3,
                              int Nz, int Nk, int Nx, double k0, double s, double kappa, double nu, double beta) {
  const long long total = (long long)Nz * Nk;
  const double ib = 1.0 / beta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i / Nk), m = (int)(i % Nk);
    const double s0 = s3[3 * k], s1 = s3[3 * k + 1], s2 = s3[3 * k + 2];
    auto xf = [&](int f, int kk) -> double2 {
      return (kk < Nz) ? X[((size_t)f * Nz + kk) * Nk + m] : make_double2(0.0, 0.0);
    };
    auto Sx = [&](int f) -> double2 {
      double2 acc = make_double2(0.0, 0.0);
      acc = cfma(s0, xf(f, k), acc);
      acc = cfma(s1, xf(f, k + 2), acc);
      acc = cfma(s2, xf(f, k + 4), acc);
      return acc;
    };
    const size_t plane = (size_t)Nz * Nk;
    double2 out[4];
    for (int e = 0; e < 4; ++e) {
      double2 r = LX[(size_t)e * plane + i];
      if (e > 0) {
        double2 mx = Sx(e - 1);
        r.x -= mx.x;
        r.y -= mx.y;
      }
      out[e] = make_double2(r.x * ib, r.y * ib);
    }
    if (m == 0 || 2 * m == Nx) {
      // L applied to delta = i Im(X) of b, ux, uz (the part a grid round trip drops)
      const double kx = k0 * m, kx2 = kx * kx;
      auto dl = [&](int f, int kk) -> double { return (kk < Nz) ? X[((size_t)f * Nz + kk) * Nk + m].y : 0.0; };
      auto Sd = [&](int f) -> double { return s0 * dl(f, k) + s1 * dl(f, k + 2) + s2 * dl(f, k + 4); };
      const double d2 = 2.0 * (k + 2) * s * s;
      // every term is i * (real coefficient) * Im(X): subtract from the imaginary part
      // cont: i kx S d_ux + SD d_uz ; i kx * (i a) = -kx a is real
      double cont_re = -kx * Sd(UK_UX);
      double cont_im = s * (dl(UK_UZ, k + 1) - dl(UK_UZ, k + 3));
      out[0].x -= cont_re;
      out[0].y -= cont_im;
      out[1].y -= kappa * kx2 * Sd(UK_B) - kappa * d2 * dl(UK_B, k + 2);
      out[2].y -= nu * kx2 * Sd(UK_UX) - nu * d2 * dl(UK_UX, k + 2);
      out[3].y -= nu * kx2 * Sd(UK_UZ) - nu * d2 * dl(UK_UZ, k + 2) - Sd(UK_B);
    }
    for (int e = 0; e < 4; ++e) LX[(size_t)e * plane + i] = out[e];
  }
}

__global__ void k_rk_final(LinComb lc, double2* __restrict__ X, const double* __restrict__ s3, int Nz, int Nk) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y >> 1, par = blockIdx.y & 1;
  if (m >= Nk) return;
  const size_t plane = (size_t)Nz * Nk;
  int k = Nz - 1;
  if ((k & 1) != par) --k;
  double2 x2 = make_double2(0.0, 0.0), x4 = make_double2(0.0, 0.0);  // x_{k+2}, x_{k+4}
  for (; k >= 0; k -= 2) {
    const size_t i = (size_t)(1 + f) * plane + (size_t)k * Nk + m;
    double2 y = make_double2(0.0, 0.0);
    for (int t = 0; t < lc.n; ++t) y = cfma(lc.w[t], lc.in[t][i], y);
    y = cfma(-s3[3 * k + 1], x2, y);
    y = cfma(-s3[3 * k + 2], x4, y);
    const double inv = 1.0 / s3[3 * k];
    const double2 x = make_double2(y.x * inv, y.y * inv);
    X[(size_t)f * plane + (size_t)k * Nk + m] = x;
    x4 = x2;
    x2 = x;
  }
}

template <int KL, int KU>
void factor_impl(const TauArgs& a, cudaStream_t st) {
  int nmax = a.cls[0].n > a.cls[1].n ? a.cls[0].n : a.cls[1].n;
  dim3 grid((a.Nk + 63) / 64, 2);
  k_tau_factor<KL, KU><<<grid, 64, 0, st>>>(a, nmax);
}

template <int KL, int KU>
void solve_impl(const TauArgs& a, cudaStream_t st) {
  dim3 grid((a.Nk + 127) / 128, 2);
  k_tau_solve<KL, KU><<<grid, 128, 0, st>>>(a);
}

}  // namespace

size_t tau_factor_scratch_doubles(int nmax, int Nk);

// Supported band shape: the RBC layout gives kl = 4, ku = 8 for every Nz >= 8
// (narrower layouts are zero-padded to it by the plan).
void launch_tau_factor(const TauArgs& a, cudaStream_t st) { factor_impl<kTauKL, kTauKU>(a, st); }
void launch_tau_solve(const TauArgs& a, cudaStream_t st) { solve_impl<kTauKL, kTauKU>(a, st); }

size_t tau_factor_scratch_doubles(int nmax, int Nk) {
  const int KL = kTauKL, KU = kTauKU, WW = 2 * KL + KU + 1;
  const size_t per = (size_t)nmax * WW + (size_t)nmax * NBMAX + (size_t)NBMAX * nmax + NBMAX * NBMAX;
  return per * 2 * (size_t)Nk;
}

void launch_lincomb(const LinComb& lc, double2* out, long long count, cudaStream_t st) {
  int blocks = (int)((count + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  k_lincomb<<<blocks, 256, 0, st>>>(lc, out, count);
}

void launch_mass_apply(const double2* X, double2* MX, const double* s3, int Nz, int Nk, int Nx, int project,
                       cudaStream_t st) {
  long long total = (long long)Nz * Nk;
  int blocks = (int)((total + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_mass_apply<<<blocks, 256, 0, st>>>(X, MX, s3, Nz, Nk, Nx, project);
}

void launch_lx_finalize(double2* LX, const double2* X, const double* s3, int Nz, int Nk, int Nx, double k0,
                        double s, double kappa, double nu, double beta, cudaStream_t st) {
  long long total = (long long)Nz * Nk;
  int blocks = (int)((total + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_lx_finalize<<<blocks, 256, 0, st>>>(LX, X, s3, Nz, Nk, Nx, k0, s, kappa, nu, beta);
}

void launch_rk_final(const LinComb& lc, double2* X, double2* tau, const double* s3, int Nz, int Nk,
                     cudaStream_t st) {
  dim3 grid((Nk + 127) / 128, 6);
  k_rk_final<<<grid, 128, 0, st>>>(lc, X, s3, Nz, Nk);
  cudaMemsetAsync(X + (size_t)3 * Nz * Nk, 0, sizeof(double2) * (size_t)Nz * Nk, st);
  cudaMemsetAsync(tau, 0, sizeof(double2) * 7 * (size_t)Nk, st);
}

}  // namespace tb
