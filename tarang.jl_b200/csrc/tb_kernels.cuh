// Device kernels of libtarang_b200 (sm_100a) and their launch wrappers.
#pragma once

#include <cuda_runtime.h>

#include "tb_internal.h"

namespace tb {

// Up to this many inputs (and 2x outputs) per batched GEMM launch.
constexpr int kGemmMaxBatch = 6;

struct GemmBatch {
  const double* in[kGemmMaxBatch];
  double* out[2 * kGemmMaxBatch];
};

// C[r][c] = sum_k A[r][k] * B[k][c] for each batch entry.  A: Mo x K
// row-major (shared), B: K x ncol (ldb), output row r goes to
// out[b*nsplit + r/rows_per_out] at row r % rows_per_out (ldc).
void launch_gemm_f64(const double* A, int Mo, int K, const GemmBatch& bt, int nbatch, int ncol, int ldb,
                     int ldc, int rows_per_out, int nsplit, cudaStream_t st);

struct XProdArgs {
  // mixed-space inputs (Nz x Nk complex): values and z-derivatives of b, ux, uz
  const double2* val[3];
  const double2* dz[3];
  double2* out[3];       // mixed-space products -(u.grad f) (Nz x Nk complex)
  const double2* tw;     // exp(-2 pi i t / M), t < M
  FftPlan fp;            // length M plan
  int Nx, Nk, M, Nz;
  double k0;             // 2 pi / Lx
};
void launch_xprod(const XProdArgs& a, cudaStream_t st);
size_t xprod_smem_bytes(int M);
// Raise the dynamic shared-memory limit of the transform kernels (once per plan).
cudaError_t set_transform_smem_limits(int bytes);
// Scratch (doubles) the factorisation needs for nmax band rows and Nk modes.
size_t tau_factor_scratch_doubles(int nmax, int Nk);

// Standalone x transforms on rows: forward rfft (grid rows -> half spectra) and
// backward irfft (half spectra -> grid rows), unnormalised / 1/N like FFTW.
void launch_x_rfft(const double* grid, double2* spec, int nrows, int Nx, const FftPlan& fp, const double2* tw,
                   cudaStream_t st);
void launch_x_irfft(const double2* spec, double* grid, int nrows, int Nx, const FftPlan& fp, const double2* tw,
                    cudaStream_t st);
// Standalone 3/2-dealiased product of two grid fields (rows of length Nx).
void launch_x_dealias_mul(const double* a, const double* b, double* out, int nrows, int Nx, int M,
                          const FftPlan& fpN, const double2* twN, const FftPlan& fpM, const double2* twM,
                          cudaStream_t st);

// ---- tau system kernels ----
// Compiled band shape of the per-class tau systems (lower / upper bandwidth).
constexpr int kTauKL = 4, kTauKU = 8;
struct ClassDev {
  int n, nb, kl, ku;
  const short* row_eq;
  const short* row_k;
  const short* col_unk;
  const short* col_k;
  const short* left_unk;
  const short* left_k;
  const double* bc_rhs;
  const Coef* band;   // n x (kl+ku+1)
  const Coef* bord;   // n x nb
  const double* c2_z; // nb x n
  const double* c2_nz;
  const double* c1_z; // nb x nb
  const double* c1_nz;
  // factors (mode fastest)
  unsigned char* piv;  // n x Nk
  double* Lm;          // n x kl x Nk
  double* U;           // n x (kl+ku+1) x Nk ; U[j][0] = 1/diag
  double* Bd;          // n x nb x Nk
  double* Cm;          // n x nb x Nk
  double* Sinv;        // nb x nb x Nk
};

struct TauArgs {
  ClassDev cls[2];
  int Nz, Nk, Nx;
  double k0;           // 2 pi / Lx
  double alpha, beta;  // LHS = alpha M + beta L
  // state (T space): X[4][Nz][Nk] (b, ux, uz, p), tau[7][Nk]
  double2* X;
  double2* tau;
  // P-space right-hand side (cont, b, mx, mz) x Nz x Nk
  const double2* rhsP;
  double* scratch;     // factor workspace
  int* err_mode;       // first singular mode, or -1
};
void launch_tau_factor(const TauArgs& a, cudaStream_t st);
void launch_tau_solve(const TauArgs& a, cudaStream_t st);

struct LinComb {
  const double2* in[12];
  double w[12];
  int n;
};
// out[i] = sum_t w_t in_t[i] over count complex entries
void launch_lincomb(const LinComb& lc, double2* out, long long count, cudaStream_t st);

// MX[e][k][m] = S X_f (e = 1+f), cont rows zero; optional DC/Nyquist projection.
void launch_mass_apply(const double2* X, double2* MX, const double* s3, int Nz, int Nk, int Nx, int project,
                       cudaStream_t st);
// LX (in place over rhsP) = (rhsP - PM X)/beta - PL delta at the DC/Nyquist modes.
void launch_lx_finalize(double2* LX, const double2* X, const double* s3, int Nz, int Nk, int Nx, double k0,
                        double s, double kappa, double nu, double beta, cudaStream_t st);
// X_f = S^{-1} (lincomb)[1+f] for f = b, ux, uz; p and taus zeroed.
void launch_rk_final(const LinComb& lc, double2* X, double2* tau, const double* s3, int Nz, int Nk,
                     cudaStream_t st);

}  // namespace tb
