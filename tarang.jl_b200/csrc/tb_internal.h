// Internal declarations shared by the libtarang_b200 translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tarang_b200.h"

struct tb_context {
  int device = 0;
  // message of the context's last failure; written under mu (several threads
  // may use plans of one context), read through tb_last_error
  std::string last_error;
  mutable std::mutex mu;
};

namespace tb {

// Work streams of the library (plans, turbulence plans, ensemble workers) are
// created at the device's greatest priority, all alike, so that the only
// streams that yield are the plans' step side streams (least priority): the
// forked kernels of a step fill the SMs its main chain leaves idle, while the
// plans of an ensemble or a server compete on equal terms.
inline cudaError_t create_work_stream(cudaStream_t* s, bool side = false) {
  int least = 0, greatest = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (e != cudaSuccess) return e;
  return cudaStreamCreateWithPriority(s, cudaStreamNonBlocking, side ? least : greatest);
}

// ---------------------------------------------------------------------------
// Error plumbing: every failure becomes a tb_status plus a message stored in
// the context; nothing escapes the C ABI as an exception.
// ---------------------------------------------------------------------------
struct Error {
  tb_status code;
  std::string msg;
};

#define TB_CUDA_TRY(expr)                                                         \
  do {                                                                            \
    cudaError_t _e = (expr);                                                      \
    if (_e != cudaSuccess)                                                        \
      throw ::tb::Error{TB_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)}; \
  } while (0)

#define TB_REQUIRE(cond, code, msg)                        \
  do {                                                     \
    if (!(cond)) throw ::tb::Error{(code), std::string(msg)}; \
  } while (0)

// ---------------------------------------------------------------------------
// Per-parity-class banded layout of one Fourier mode's tau system.
//
// The reference assembles, per Fourier mode, a dense-D complex system in the
// ChebyshevT basis (subproblem_matrix_build.jl).  The library left-multiplies
// every bulk equation block by the T->C^(2) conversion S = S1 S0 (an
// invertible row operation, so the solution is unchanged), which makes every
// derivative and lift operator banded; scales u_x and its taus by i so that
// the system becomes real; and splits the unknowns by Chebyshev parity into
// two independent classes.  Each class is a bordered banded system:
//   [ B2  B1 ] [x2]   [r_B]     B2: bulk rows x band columns (banded kl/ku)
//   [ C2  C1 ] [x1] = [r_C]     C : boundary rows (dense), x1: border unknowns
// ---------------------------------------------------------------------------
enum Eq : int { EQ_CONT = 0, EQ_B = 1, EQ_MX = 2, EQ_MZ = 3 };
// Unknown codes: 0 b, 1 u_x (stored; real-ified as v_x = -i u_x), 2 u_z, 3 p,
// 4 + t for tau t in (tau_p, tau_b1, tau_b2, tau_u1x, tau_u1z, tau_u2x, tau_u2z).
enum Unk : int { UK_B = 0, UK_UX = 1, UK_UZ = 2, UK_P = 3, UK_TAU0 = 4 };

struct Coef {  // value = alpha*m + beta*(l0 + kx*l1 + kx^2*l2)
  double m, l0, l1, l2;
};

struct ClassLayout {
  int n = 0;    // number of band rows (= band columns) = bulk rows
  int nb = 0;   // border size (boundary rows = border unknowns)
  int kl = 0, ku = 0;
  std::vector<int> row_eq, row_k;      // band row j -> (equation, C2 index)
  std::vector<int> col_unk, col_k;     // band column j -> (unknown, T index)
  std::vector<int> left_unk, left_k;   // border unknown b -> (unknown, T index)
  // band entries: row j, column j + d - kl (d in [0, kl+ku]); (n x (kl+ku+1))
  std::vector<Coef> band;
  // border entries of bulk rows: (n x nb)
  std::vector<Coef> bord;
  // boundary rows: C2 (nb x n) and C1 (nb x nb); value = beta * (kx==0 ? z : nz)
  std::vector<double> c2_z, c2_nz, c1_z, c1_nz;
  // boundary row right-hand sides at kx = 0 (times beta); zero at kx != 0
  std::vector<double> bc_rhs;
};

struct TauLayout {
  int Nz = 0;
  ClassLayout cls[2];
};

// Records the message of a failure in the context (under its mutex).
void set_context_error(tb_context* ctx, const std::string& msg);
// Records a message for tb_last_error(NULL) on the calling thread.
void set_thread_error(const std::string& msg);

// Builds the banded layout for the RBC program (host, once per plan).
TauLayout build_rbc_layout(int Nz, double Lx, double Lz, double kappa, double nu, double Nx_scale,
                           double b_bottom, double b_top);

// Banded layout of the decoupled velocity component of the 3D program
// (Helmholtz tau system with two lifts and two no-slip walls); needs even Nz.
TauLayout build_helmholtz_layout(int Nz, double Lz, double nu);

// Chebyshev transform matrices (row-major, N x N) built in extended precision.
struct ChebMats {
  std::vector<double> bwd;     // grid_j = sum_n bwd[j][n] c_n
  std::vector<double> bwd_d;   // (d/dz) grid_j = sum_n bwd_d[j][n] c_n
  std::vector<double> fwd;     // c_n = sum_j fwd[n][j] g_j
  std::vector<double> sfwd;    // (S fwd): C^(2) coefficients of the forward transform
  std::vector<double> s3;      // S[k][k], S[k][k+2], S[k][k+4]  (N x 3)
};
ChebMats build_cheb_mats(int N, double Lz);

// FFT plan for lengths 2^a 3^b (Stockham, radices 4, 2, 3).
struct FftPlan {
  int n = 0;
  int nstages = 0;
  int radix[16];
};
bool make_fft_plan(int n, FftPlan* out);

}  // namespace tb
