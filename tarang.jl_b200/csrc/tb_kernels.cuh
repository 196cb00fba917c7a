// Device kernels of libtarang_b200 (sm_100a) and their launch wrappers.
#pragma once

#include <cuda_runtime.h>

#include "tb_internal.h"

namespace tb {

// Batched Chebyshev-direction GEMM (see tb_transforms.cu for the row maps).
enum { GEMM_PLAIN = 0, GEMM_PARITY = 1, GEMM_MIRROR = 2 };
constexpr int kGemmMaxBatch = 16;
struct GemmItem {
  const double* A;  // M x Kpad row-major, columns K..Kpad-1 zero (Kpad a multiple of 16)
  const double* B;  // input rows (ldb doubles apart; ldb even)
  double* C;        // output rows (ldc)
  int M, K, Kpad, mode, par;
};
struct GemmBatch {
  GemmItem item[kGemmMaxBatch];
};
void launch_gemm_f64(const GemmBatch& bt, int nbatch, int ncol, int ldb, int ldc, int Nrows, cudaStream_t st);

// FP32 twins for the mixed-precision RHS (same row maps; C is float or double).
struct GemmItem32 {
  const float* A;  // M x Kpad row-major, zero padded
  const float* B;  // input rows (ldb floats apart; ldb even)
  void* C;         // output rows (ldc elements)
  int M, K, Kpad, mode, par;
  // tensor-core path: A's TF32 hi/lo operand image (make_tc32_a_image; null:
  // SIMT only) and, set by launch_gemm_tc32, the item's B' tile images
  const float* Aimg = nullptr;
  const float* Bimg = nullptr;
};
struct GemmBatch32 {
  GemmItem32 item[kGemmMaxBatch];
};
void launch_gemm_f32(const GemmBatch32& bt, int nbatch, int ncol, int ldb, int ldc, int Nrows, bool out_f64,
                     cudaStream_t st);
// The same GEMMs on the tcgen05 tensor cores (TF32, three products per term;
// tb_tc32.cu) for items with M <= 128 and K <= 128.  The operands reach the
// tensor cores as images of their shared-memory tiles (TF32 hi and lo parts,
// 128-byte swizzled, K-major), copied in by bulk copies: A's once per plan
// (make_tc32_a_image, tc32_a_image_floats floats each), B's per call by a
// staging kernel into scratch (tc32_b_scratch_floats floats for up to
// kGemmMaxBatch distinct inputs of ncol columns).
bool gemm_tc32_supported(const GemmBatch32& bt, int nbatch);
size_t tc32_a_image_floats();
size_t tc32_b_scratch_floats(int ncol, int nimages);
void make_tc32_a_image(const float* A, int M, int Kpad, float* image, cudaStream_t st);
// false (nothing launched) when an item has no A image or the scratch is too small
bool launch_gemm_tc32(const GemmBatch32& bt, int nbatch, int ncol, int ldb, int ldc, int Nrows, bool out_f64,
                      cudaStream_t st, float* bscratch, size_t bscratch_floats);
cudaError_t set_tc32_smem_limits();
// Streaming form for the 3D z transforms (even N <= 128 rows, ncol a multiple
// of 4): the raw FP32 planes of nfields fields (N x ncol each, contiguous) are
// read through a TMA tensor map, the row maps live in the A operands
// (tc32s_image_floats floats, made once per plan by make_tc32s_images from
// the eight FP32 transform matrices).  Backward: C_w (N/2 x ncol) of field f
// at out + (4 f + w) N/2 ncol, w = parity + 2 derivative; forward: FP64 rows
// of field f at out + f N ncol.
struct alignas(64) TmaDesc {
  unsigned char bytes[128];
};
bool tc32s_supported(int N, int ncol);
size_t tc32s_image_floats();
void make_tc32s_images(const float* Ev, const float* Ov, const float* Ed, const float* Od, int kpe, int kpo,
                       const float* sfE, const float* sfO, int kph, int N, float* images, cudaStream_t st);
bool make_tc32s_tmap(TmaDesc* d, const float* planes, int nfields, int N, int ncol);  // false: unsupported
void launch_tc32s(bool backward, const TmaDesc& d, const float* images, void* out, int nfields, int N, int ncol,
                  cudaStream_t st);
// Plane form for the 2D z transforms (even N <= 256 rows, even ncol): the same
// products with each CTA serving one A operand held in tensor memory (4
// backward roles, 2 forward), the tiles read straight from the planes (whose
// rows need not be 16-byte aligned).  Same outputs as launch_tc32s for
// nfields fields; A parts from make_tc32p_images (tc32p_image_floats floats).
bool tc32p_supported(int N, int ncol);
size_t tc32p_image_floats();
void make_tc32p_images(const float* Ev, const float* Ov, const float* Ed, const float* Od, int kpe, int kpo,
                       const float* sfE, const float* sfO, int kph, int N, float* images, cudaStream_t st);
void launch_tc32p(bool backward, const float* in, const float* images, void* out, int nfields, int N, int ncol,
                  cudaStream_t st);
int tc32_status();  // 1 once a tensor-core GEMM's bounded wait gave up, -1 if unreadable
// tensor cores when asked for and the shapes fit, else SIMT
inline void launch_gemm_f32_path(const GemmBatch32& bt, int nbatch, int ncol, int ldb, int ldc, int Nrows,
                                 bool out_f64, cudaStream_t st, bool tensor_cores, float* bscratch = nullptr,
                                 size_t bscratch_floats = 0) {
  if (tensor_cores && gemm_tc32_supported(bt, nbatch) &&
      launch_gemm_tc32(bt, nbatch, ncol, ldb, ldc, Nrows, out_f64, st, bscratch, bscratch_floats))
    return;
  launch_gemm_f32(bt, nbatch, ncol, ldb, ldc, Nrows, out_f64, st);
}
void launch_round_f32(const double2* in, float2* out, long long n, cudaStream_t st);
struct XProdArgs32 {
  const float2* ev[3];
  const float2* ov[3];
  const float2* ed[3];
  const float2* od[3];
  float2* out[3];
  const float2* ptw;  // per-pass FP32 twiddles of the length-M plan
  int nptw;
  FftPlan fp;
  int Nx, Nk, M, Nz;
  float k0;
  int ld;         // row stride of the planes (Nk, or instances x Nk in a stacked plan)
  int instances;  // instances stacked along the mode axis (grid.y)
  const float2* iptw;  // in-place (DIF/DIT) FP32 twiddles of the length-M plan
  int niptw;
};
void launch_xprod32(const XProdArgs32& a, cudaStream_t st);
void launch_xprod32_ip(const XProdArgs32& a, cudaStream_t st);  // transforms in place (fftg::k_xprod_ip)
bool xprod32_ip_fits(int M, int niptw);
void launch_xprod32_b(const XProdArgs32& a, cudaStream_t st);  // transforms batched (as launch_xprod_b)
bool xprod32_b_fits(int M, int nptw);
size_t xprod32_smem_bytes(int M, int nptw);
cudaError_t set_mixed_smem_limits(int bytes);

struct XProdArgs {
  // mixed-space inputs as even/odd Chebyshev half planes (ceil(Nz/2) x Nk
  // complex) of the values (ev, ov) and z-derivatives (ed, od) of b, ux, uz
  const double2* ev[3];
  const double2* ov[3];
  const double2* ed[3];
  const double2* od[3];
  double2* out[3];       // mixed-space products -(u.grad f) (Nz x Nk complex)
  const double2* ptw;    // per-pass twiddle tables of the length-M plan (pass_twiddle_count entries)
  int nptw;
  FftPlan fp;            // length M plan
  int Nx, Nk, M, Nz;
  double k0;             // 2 pi / Lx
  int ld;                // row stride of the planes (Nk, or instances x Nk in a batched plan)
  int instances;         // instances stacked along the mode axis (grid.y)
  const double2* iptw;   // in-place (DIF/DIT) twiddles of the length-M plan (fftg::ip_twiddle_count)
  int niptw;
};
void launch_xprod(const XProdArgs& a, cudaStream_t st);
// The same products with the transforms in place: DIF inverse passes,
// pointwise products, DIT forward passes (four arrays of shared memory).
void launch_xprod_ip(const XProdArgs& a, cudaStream_t st);
bool xprod_ip_fits(int M, int niptw);
size_t xprod_smem_bytes(int M, int Nk, int nptw);
// The same products with the inverse and forward transforms batched through
// shared passes (two 4-array blocks of shared memory).
void launch_xprod_b(const XProdArgs& a, cudaStream_t st);
bool xprod_b_fits(int M, int nptw);
// Raise the dynamic shared-memory limit of the transform kernels (once per plan).
cudaError_t set_transform_smem_limits(int bytes);
// Scratch (doubles) the factorisation needs for nmax band rows and Nk modes.

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
// The solve streams per-row factor records of kSolveModes consecutive Fourier
// modes: forward record = pivot offset, kTauKL multipliers, 4 boundary-row
// multipliers; backward record = 1/diag, kTauKL+kTauKU U entries, 4 border
// entries, the encoded store target of the band column and the 4 responses of
// the row's y to its partition's starting window (one contiguous record per
// mode, an even number of doubles so a lane reads it 16 bytes at a time).
constexpr int kSolveModes = 4;
// forward: pivot, multipliers, border, rotation flag of the row entering the window
constexpr int kFwdRec = 1 + kTauKL + 4 + 1;
constexpr int kFwdRot = kFwdRec - 1;
// backward: 1/diag, U entries, border, store code, 4 forward responses G
constexpr int kBwdCode = 1 + kTauKL + kTauKU + 4;
constexpr int kBwdG = kBwdCode + 1;
constexpr int kBwdRec = kBwdG + 4;
// per-row backward responses H of the partitioned solve: 12 entries (the
// rows' store codes come from the per-row table TauArgs::xcode)
constexpr int kHRec = kTauKL + kTauKU;
// Register windows of the solve sweeps.  The solve splits the band rows into
// partitions (one warp each), each a whole number of backward windows; rows
// are padded with identity rows to a multiple of kTauParts * kBwdWin
// (kTauRowPad), so kTauParts partitions are equal.  kTauParts8 partitions
// take the same rows, as evenly as whole windows go (tau_part_row0).
constexpr int kFwdWin = kTauKL + 2;
constexpr int kBwdWin = kTauKL + kTauKU;
constexpr int kTauParts = 4;
constexpr int kTauParts8 = 8;
constexpr int kTauRowPad = kTauParts * kBwdWin;
// First band row of partition k (0 <= k <= P) of a P-partition solve over
// np rows (np a multiple of kBwdWin): windows spread as evenly as they go,
// the spare ones to the upper partitions (the backward carry starts at the
// bottom, so the lighter lower partitions begin it while the upper ones
// still sweep).  With two partitions per warp (ppw = 2, np a multiple of
// 2 kBwdWin) the two partitions of a warp get equal row counts, so the warp's
// halves sweep in step: warp w takes pairs of windows spread the same way.
__host__ __device__ inline int tau_part_row0(int np, int P, int k, int ppw = 1) {
  auto first = [](int n, int parts, int i) {  // first unit of part i of n units, spares to the first parts
    const int q = n / parts, r = n % parts;
    return i * q + (i < r ? i : r);
  };
  if (ppw == 1) return kBwdWin * first(np / kBwdWin, P, k);
  const int nw = P / 2, pairs = np / (2 * kBwdWin);
  const int w = k / 2, h = k % 2;
  const int b0 = first(pairs, nw, w), b1 = first(pairs, nw, w + 1);
  return 2 * kBwdWin * b0 + h * kBwdWin * (b1 - b0);
}
// Partitions per warp of the 8- and 16-partition solves (two: each half-warp
// sweeps one).  The 16-partition form (eight warps per group) streams its
// records in stages of 3 rows and keeps y and the particular unknowns in
// global scratch (prefetched with the records), so that 16 rings fit one SM.
constexpr int kTau8PerWarp = 2;
constexpr int kTauParts16 = 16;
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
  // store targets (element offset of the unknown's row for mode 0, times 2,
  // plus 1 when the unknown is i times the solved real column): band column
  // j -> col_code[j], border unknown b -> left_code[b]
  const int* col_code;
  const int* left_code;
  // factors, shared by both classes (set on cls[0]):
  //   FR[group][row][class][kSolveModes][kFwdRec], BR[group][row][class][kSolveModes][kBwdRec],
  //   SI[group][class][4][4][kSolveModes]
  double* FR;
  double* BR;
  double* SI;
};

struct TauArgs {
  ClassDev cls[2];
  int Nz, Nk, Nx;
  int npad;            // band rows padded to a multiple of kTauRowPad
  double k0;           // 2 pi / Lx
  const double* kmag;  // per-mode horizontal wavenumber |k| (3D), or null for k0 * m
  double alpha, beta;  // LHS = alpha M + beta L
  // state (T space): X[4][Nz][Nk] (b, ux, uz, p) directly followed by tau[7][Nk]
  double2* X;
  double2* tau;
  // P-space right-hand side (cont, b, mx, mz) x Nz x Nk
  const double2* rhsP;
  // [row][class] over npad rows: 2 * (element offset of band row j's right-hand
  // side in rhsP) + 1 for a u_x momentum row, -1 for none
  const int* rhs_off;
  // [row][class] over npad rows: store target of band column j packed in 16
  // bits, 2 * (its element offset / Nk) + (1 if the unknown is i times the
  // solved column), -1 for none (the store code is 2 * offset + flag)
  const short* xcode;
  // optional FP32 copy of the first x32_lim doubles of X (mixed 2D plans: the
  // b, u_x, u_z planes), written beside X by the solve; null for none
  float* X32;
  long long x32_lim;
  // partition responses of the solve, written by the factorisation:
  // PP[group][partition][class][mode] = Phi (4x4), Psi (12x12), Gz (4x4);
  // HR[group][row][class][mode][kHRec] = H (12)
  double* PP;
  double* HR;
  double* ysave;       // one-partition solve: [group][row][lane] y scratch (tau_solve_scratch_doubles)
  // modes per instance (batched plans stack instances along the mode axis:
  // mode m belongs to instance m / Nkm, its own mode m % Nkm); the
  // factorisation runs per instance on modes mode0 .. mode0 + Nkm - 1
  int Nkm, mode0;
  // dynamic wall values of b (null: constant BCs from bc_rhs): [bottom value,
  // bottom rate, top value, top rate][mode] at time *t_dev + bc_toff
  const double2* bcdyn;
  const double* t_dev;
  double bc_toff;
  int* err_mode;       // first singular mode, or -1
};
// parts: kTauParts, kTauParts8 or kTauParts16 (partitioned solve, needs a.PP)
// or 1 (one warp per group).
// launch_tau_factor factors modes a.mode0 .. a.mode0 + a.Nkm - 1; the
// partition responses (launch_tau_transfer) are then computed for all modes.
void launch_tau_factor(const TauArgs& a, int parts, cudaStream_t st);
void launch_tau_transfer(const TauArgs& a, int parts, cudaStream_t st);
void launch_tau_solve(const TauArgs& a, int parts, cudaStream_t st);
cudaError_t set_tau_smem_limits(int bytes);
size_t tau_solve_smem_bytes(int npad, int parts);
size_t tau_transfer_doubles(int Nk, int parts);
size_t tau_response_doubles(int Nk, int npad, int parts);
size_t tau_solve_scratch_doubles(int Nk, int npad, int parts);

struct LinComb {
  const double2* in[12];
  double w[12];
  int n;
};
// out[i] = sum_t w_t in_t[i] over count complex entries
void launch_lincomb(const LinComb& lc, double2* out, long long count, cudaStream_t st);

void launch_advance_time(double* t, double dt, cudaStream_t st);

// Velocity-like fields of a stage vector: nf = 3 (2D: b, u_x, u_z in X planes
// 0..2, equation planes 1..3) or 4 (3D adds u_perp in X plane 4 with its
// momentum rows in equation plane 4).
// MX[e][k][m] = S X_f, cont rows zero; optional DC/Nyquist projection (2D).
void launch_mass_apply(const double2* X, double2* MX, const double* s3, int Nz, int Nk, int Nx, int project,
                       int nf, cudaStream_t st, int Nkm = 0);
// LX (in place over rhsP) = (rhsP - PM X)/beta, minus PL delta at the 2D
// DC/Nyquist modes when Nx > 0 (3D passes Nx = 0 and corrects separately).
// Batched plans: Nkm modes per instance, per-instance kappa / nu (null: the scalars).
void launch_lx_finalize(double2* LX, const double2* X, const double* s3, int Nz, int Nk, int Nx, double k0,
                        double s, double kappa, double nu, double beta, int nf, cudaStream_t st, int Nkm = 0,
                        const double* kappa_m = nullptr, const double* nu_m = nullptr);
// X_f = S^{-1} (lincomb)[eq(f)] for the nf velocity-like fields; p and the ntau taus zeroed.
void launch_rk_final(const LinComb& lc, double2* X, double2* tau, const double* s3, int Nz, int Nk, int nf,
                     int ntau, cudaStream_t st);
size_t rk_final_smem_bytes(int Nz);

}  // namespace tb
