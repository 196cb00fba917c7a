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

#ifdef TB_SOLVE_CLOCKS
// Phase clocks of the tau solve (a separate build, `make clocks`): SM cycle
// counter of lane 0 of every partition at the start of F1, F2, the border
// solve (B1), B2, B3 and the end, [group][partition][8].
constexpr int kSolveClockSlots = 1 << 16;
__device__ long long g_solve_clocks[kSolveClockSlots];
#define TB_SOLVE_CLOCK(ph)                                                           \
  do {                                                                             \
    if (tl == 0 && (g * P + pid) * 8 + (ph) < kSolveClockSlots)                    \
      g_solve_clocks[(g * P + pid) * 8 + (ph)] = clock64();                        \
  } while (0)
#else
#define TB_SOLVE_CLOCK(ph) \
  do {                     \
  } while (0)
#endif

namespace {

constexpr int NBMAX = 4;

__device__ __forceinline__ double coef_val(const Coef& c, double alpha, double beta, double kx) {
  return alpha * c.m + beta * (c.l0 + kx * c.l1 + kx * kx * c.l2);
}

__device__ __forceinline__ double2 cfma(double a, double2 x, double2 acc) {
  return make_double2(fma(a, x.x, acc.x), fma(a, x.y, acc.y));
}

// Solve-layout factor records: for group g = m / kSolveModes and band row j the
// records of both classes and the group's modes are contiguous,
// FR[g][j][class][mode % kSolveModes][kFwdRec] (and BR likewise), so one lane
// reads its own record with 16-byte loads and the group's rows stream as a block.
__device__ __forceinline__ double* fwd_record(double* FR, int npad, int m, int j, int c) {
  const int g = m / kSolveModes, mm = m % kSolveModes;
  return FR + ((((size_t)g * npad + j) * 2 + c) * kSolveModes + mm) * kFwdRec;
}
__device__ __forceinline__ double* bwd_record(double* BR, int npad, int m, int j, int c) {
  const int g = m / kSolveModes, mm = m % kSolveModes;
  return BR + ((((size_t)g * npad + j) * 2 + c) * kSolveModes + mm) * kBwdRec;
}

// ---------------------------------------------------------------------------
// Factorisation: one warp per (mode, class).  Banded LU with partial pivoting
// restricted to the band of the bulk rows; the boundary rows are eliminated
// alongside as a dense border and leave an nb x nb Schur complement, inverted
// explicitly.
//
// Only a window of the elimination is live at step j: rows j..j+KL of the
// band and columns j..j+KL+KU of the boundary rows.  The window sits in the
// warp's shared memory; a row enters (its coefficients evaluated from the
// band tables and |k|) when step j = row - KL first updates it, a boundary-
// row column when step j = column - KL - KU does (ring slots: row i at
// i % (KL+1), column c at c % (KL+KU+1)).  At each step the lanes take the
// columns: lane t < KL+KU updates column j+1+t of the KL rows below and of
// the boundary rows, lanes KL+KU.. the border entries.  Every element gets the
// same operations in the same order as a sequential elimination, so the
// factors do not depend on the lane split; the pivot scan (KL+1 candidates)
// and the Schur inverse run on lane 0.
// ---------------------------------------------------------------------------
constexpr int kFactorWarps = 4;  // systems (warps) per CTA of the factorisation

// Window doubles per system: rows (KL+1) x (band slots + border), boundary-row
// columns NBMAX x (KL+KU+1), the NBMAX^2 border block.
template <int KL, int KU>
__host__ __device__ constexpr int factor_window_doubles() {
  return (KL + 1) * ((2 * KL + KU + 1) + NBMAX) + NBMAX * (KL + KU + 1) + NBMAX * NBMAX;
}
template <int KL, int KU>
__host__ __device__ constexpr size_t factor_smem_bytes() {
  return (size_t)factor_window_doubles<KL, KU>() * kFactorWarps * sizeof(double);
}

template <int KL, int KU>
__global__ void __launch_bounds__(32 * kFactorWarps) k_tau_factor(TauArgs a) {
  static_assert(KL + KU + NBMAX <= 32 && kFwdRec <= 32 && kBwdCode < 32, "one lane per column and record slot");
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int ml = blockIdx.x * kFactorWarps + warp;  // mode within this instance
  const int c = blockIdx.y;
  if (ml >= a.Nkm) return;  // whole warps leave together
  const int m = a.mode0 + ml;
  const ClassDev& C = a.cls[c];
  const int n = C.n, nb = C.nb;
  constexpr int WW = 2 * KL + KU + 1;
  constexpr int W1 = KL + KU + 1;
  constexpr int RR = KL + 1, CW = KL + KU + 1;
  const double kx = a.kmag ? a.kmag[m] : a.k0 * ml;
  const bool zmode = (ml == 0);
  extern __shared__ double fsm[];
  double* win = fsm + (size_t)warp * factor_window_doubles<KL, KU>();
  auto Wr = [&](int i, int d) -> double& { return win[(i % RR) * WW + d]; };
  auto Bd = [&](int i, int b) -> double& { return win[RR * WW + (i % RR) * NBMAX + b]; };
  auto Cr = [&](int q, int col) -> double& { return win[RR * (WW + NBMAX) + q * CW + col % CW]; };
  auto C1 = [&](int q, int b) -> double& { return win[RR * (WW + NBMAX) + NBMAX * CW + q * NBMAX + b]; };
  const int cw = C.kl + C.ku + 1;
  // row r enters: lane s < WW fills band slot s, lanes < nb the border
  auto init_row = [&](int r) {
    if (lane < WW) {
      double v = 0.0;
      const int d = lane + C.kl - KL;  // band-table entry of slot lane
      const int col = r + lane - KL;
      if (d >= 0 && d < cw && col >= 0 && col < n) v = coef_val(C.band[(size_t)r * cw + d], a.alpha, a.beta, kx);
      Wr(r, lane) = v;
    }
    if (lane < nb) Bd(r, lane) = coef_val(C.bord[(size_t)r * nb + lane], a.alpha, a.beta, kx);
  };
  auto init_col = [&](int col) {
    if (lane < nb) Cr(lane, col) = a.beta * (zmode ? C.c2_z : C.c2_nz)[(size_t)lane * n + col];
  };
  for (int r = 0; r <= KL && r < n; ++r) init_row(r);
  for (int col = 0; col < CW && col < n; ++col) init_col(col);
  if (lane < nb * nb) {
    const int q = lane / nb, b = lane % nb;
    C1(q, b) = a.beta * (zmode ? C.c1_z : C.c1_nz)[q * nb + b];
  }
  __syncwarp();
  for (int j = 0; j < n; ++j) {
    // rows / columns entering the window at this step (their slots held row /
    // column j-1, finished at the previous step)
    if (j >= 1 && j + KL < n) init_row(j + KL);
    if (j >= 1 && j + CW - 1 < n) init_col(j + CW - 1);
    __syncwarp();
    const int ilast = min(j + KL, n - 1);
    const int clast = min(j + KL + KU, n - 1);
    // pivot: the first largest |entry| of column j among rows j..ilast
    int p = j;
    bool bad = false;
    if (lane == 0) {
      double best = fabs(Wr(j, KL));
      for (int i = j + 1; i <= ilast; ++i) {
        double v = fabs(Wr(i, j - i + KL));
        if (v > best) {
          best = v;
          p = i;
        }
      }
      bad = !(best > 0.0) || !isfinite(best);
    }
    p = __shfl_sync(0xffffffffu, p, 0);
    if (__shfl_sync(0xffffffffu, (int)bad, 0)) {
      if (lane == 0) atomicMin(a.err_mode, m);
      return;
    }
    if (p != j) {
      const int cc = j + lane;
      if (cc <= clast) {
        double t = Wr(j, cc - j + KL);
        Wr(j, cc - j + KL) = Wr(p, cc - p + KL);
        Wr(p, cc - p + KL) = t;
      }
      if (lane < nb) {
        double t = Bd(j, lane);
        Bd(j, lane) = Bd(p, lane);
        Bd(p, lane) = t;
      }
      __syncwarp();
    }
    const double dinv = 1.0 / Wr(j, KL);
    // multipliers of the rows below and of the boundary rows, read by every
    // lane before lane 0 clears their column-j entries
    double l[KL], cqv[NBMAX];
#pragma unroll
    for (int t = 0; t < KL; ++t) {
      const int i = j + 1 + t;
      l[t] = (i <= ilast) ? Wr(i, j - i + KL) * dinv : 0.0;
    }
#pragma unroll
    for (int q = 0; q < NBMAX; ++q) cqv[q] = (q < nb) ? Cr(q, j) * dinv : 0.0;
    __syncwarp();
    if (lane == 0) {
      for (int t = 0; t < KL; ++t)
        if (j + 1 + t <= ilast) Wr(j + 1 + t, j - (j + 1 + t) + KL) = 0.0;
      for (int q = 0; q < nb; ++q) Cr(q, j) = 0.0;
    }
    if (lane < KL + KU) {
      const int cc = j + 1 + lane;
      if (cc <= clast) {
        const double wj = Wr(j, cc - j + KL);
#pragma unroll
        for (int t = 0; t < KL; ++t) {
          const int i = j + 1 + t;
          if (i <= ilast) Wr(i, cc - i + KL) -= l[t] * wj;
        }
#pragma unroll
        for (int q = 0; q < NBMAX; ++q)
          if (q < nb) Cr(q, cc) -= cqv[q] * wj;
      }
    } else if (lane - (KL + KU) < nb) {
      const int b = lane - (KL + KU);
      const double bj = Bd(j, b);
#pragma unroll
      for (int t = 0; t < KL; ++t) {
        const int i = j + 1 + t;
        if (i <= ilast) Bd(i, b) -= l[t] * bj;
      }
#pragma unroll
      for (int q = 0; q < NBMAX; ++q)
        if (q < nb) C1(q, b) -= cqv[q] * bj;
    }
    // records of row j (row j itself is final after the swap)
    double* fr = fwd_record(C.FR, a.npad, m, j, c);
    double* br = bwd_record(C.BR, a.npad, m, j, c);
    if (lane == 0) {
      fr[0] = __longlong_as_double((long long)(p - j));  // pivot offset, integer bits
    } else if (lane <= KL) {
      fr[lane] = l[lane - 1];
    } else if (lane <= KL + NBMAX) {
      fr[lane] = cqv[lane - 1 - KL];  // 0 past nb
    } else if (lane == kFwdRot) {
      // 1 when the right-hand side of row j + kFwdWin (the row entering the
      // forward window at this row) is a u_x momentum row, scaled by -i on load
      const int jn = j + kFwdWin;
      fr[kFwdRot] = __longlong_as_double((jn < n && C.row_eq[jn] == EQ_MX) ? 1LL : 0LL);
    }
    if (lane == 0) {
      br[0] = dinv;
    } else if (lane < W1) {
      br[lane] = (j + lane < n) ? Wr(j, KL + lane) : 0.0;
    } else if (lane < W1 + NBMAX) {
      const int b = lane - W1;
      br[lane] = (b < nb) ? Bd(j, b) : 0.0;
    } else if (lane == kBwdCode) {
      // store target of this band column (element offset of its row * 2 + the i flag), bit-cast
      br[kBwdCode] = __longlong_as_double((long long)C.col_code[j]);
    }
    __syncwarp();  // row j's slot is refilled at the next step
  }
  // padding rows n..npad-1: identity rows with no right-hand side and no store
  for (int j = n + lane; j < a.npad; j += 32) {
    double* fr = fwd_record(C.FR, a.npad, m, j, c);
    double* br = bwd_record(C.BR, a.npad, m, j, c);
    for (int t = 0; t < kFwdRec; ++t) fr[t] = 0.0;
    br[0] = 1.0;
    for (int t = 1; t < kBwdCode; ++t) br[t] = 0.0;
    br[kBwdCode] = __longlong_as_double(-1LL);
  }
  if (lane != 0) return;
  // invert the nb x nb Schur complement (Gauss-Jordan, partial pivoting)
  double Aug[NBMAX][2 * NBMAX];
  for (int q = 0; q < NBMAX; ++q)
    for (int b = 0; b < 2 * NBMAX; ++b) Aug[q][b] = 0.0;
  for (int q = 0; q < nb; ++q) {
    for (int b = 0; b < nb; ++b) Aug[q][b] = C1(q, b);
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
  {
    const int g = m / kSolveModes, mm = m % kSolveModes;
    double* si = C.SI + (((size_t)g * 2 + c) * NBMAX * NBMAX) * kSolveModes + mm;
    for (int q = 0; q < NBMAX; ++q)
      for (int b = 0; b < NBMAX; ++b)
        si[(q * NBMAX + b) * kSolveModes] = (q < nb && b < nb) ? Aug[q][NBMAX + b] : 0.0;
  }
}

// ---------------------------------------------------------------------------
// Solve: one CTA of P warps per group of kSolveModes Fourier modes.  Lane
// (c, part, mm) of a warp runs the sweeps of parity class c for mode
// g*kSolveModes + mm on the real (part 0) or imaginary (part 1) column; lanes
// NL..31 mirror lanes 0..NL-1 (same arithmetic, so the unrolled sweeps stay
// branch free) and only the owner lanes store.
//
// The npad band rows are split into P partitions of whole backward windows
// (tau_part_row0: equal for P = 4, as even as windows go for P = 8), warp w
// owning partition w.  Both triangular sweeps are linear
// recurrences whose state crossing a partition boundary is small: the 4
// pending entries of the forward window and the 12 latest unknowns of the
// backward window.  Every warp sweeps its own rows from a guessed boundary
// state (the raw right-hand side forward, zeros backward), which is exact for
// the first (forward) and last (backward) warp, and the error of the guess is
// removed with responses precomputed by the factorisation:
//   F1  forward sweep of every partition; publish the exit window;
//   F2  warp w >= 1 composes its true starting window with the 4x4 transfer
//       matrices Phi of the partitions above it; the border accumulators get
//       the 4x4 response Gz, and each y of the partition the 4-vector
//       response G (held in the backward record, applied when y is read);
//   B1  backward sweep of every partition from a zero window (the last warp
//       stores X; the others keep their unknowns in shared memory);
//   B2  the true incoming windows are carried up from the last partition,
//       T_{P-2} = Xhat_{P-1}, T_{k-1} = Xhat_k + Psi_k T_k (warp k applies
//       its 12x12 transfer matrix Psi_k, one barrier per partition);
//   B3  warp w < P-1 adds the 12-vector response H of each of its unknowns
//       (one streamed pass, no recurrence) and stores X; the last warp's
//       unknowns are final after B1 and are stored there.
// Each sequential chain is about 2 npad/P rows long.  Factor records stream
// through a per-warp shared-memory ring (cp.async, ring_doubles<P>() doubles
// split into as many stages of kPartRows rows as each phase's records fill);
// each lane pulls its records of a stage into registers with 16-byte loads
// before the stage's arithmetic.
// ---------------------------------------------------------------------------
constexpr int kPartRows = 6;    // rows per ring stage (the forward window)
constexpr int kPartStages = 4;  // ring depth in stages of the largest record (1 and 4 partitions)
// exchange doubles per (warp, lane): D(4) Z(4) Xhat(12), padded to 21 so that
// the 16 lanes of a warp read distinct banks
constexpr int kXch = 21;
// per (partition, class, mode): Phi (4x4), Psi (12x12), Gz (4x4)
constexpr int kTrPhi = 0, kTrPsi = 16, kTrGz = 160, kTransfer = 176;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = valid ? 16 : 0;  // src-size 0 zero-fills the destination
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Rows per ring stage: one forward window (6) with up to 8 partitions, half
// of one (3) with 16, whose sixteen rings share one SM's shared memory.
template <int P>
__host__ __device__ constexpr int part_rows() {
  return P > kTauParts8 ? kPartRows / 2 : kPartRows;
}
// With 1 and 16 partitions the y column of a group and the particular
// unknowns live in global scratch (L2) and are prefetched with the records;
// with 4 and 8 they stay in shared memory.
template <int P>
__host__ __device__ constexpr bool ys_global() {
  return P == 1 || P > kTauParts8;
}
// Doubles per ring stage (the largest of the three phases): forward records
// and right-hand sides; backward records (+ the stage's y values with y in
// global scratch); H records (+ the stage's particular unknowns with 16).
template <int P>
__host__ __device__ constexpr size_t part_stage_doubles() {
  constexpr size_t MP = kSolveModes, R = part_rows<P>(), NL = 4 * MP;
  constexpr size_t F = R * (2 * MP * kFwdRec + 2 * 2 * MP);
  constexpr size_t B = R * (2 * MP * kBwdRec + (ys_global<P>() ? NL : 0));
  constexpr size_t H = R * (2 * MP * kHRec + (P > kTauParts8 ? NL : 0));
  return F > B ? (F > H ? F : H) : (B > H ? B : H);
}
// Doubles of one partition's ring: kPartStages of the largest stage (1 and 4
// partitions), two (8: eight rings and the y store share one SM's 227 KB),
// two or the 12x12 Psi of the group's slots if larger (16).
template <int P>
__host__ __device__ constexpr size_t ring_doubles() {
  if (P > kTauParts8) {
    constexpr size_t b2 = 2 * part_stage_doubles<P>(), psi = 2 * kSolveModes * (kBwdWin * kBwdWin + 2);
    return b2 > psi ? b2 : psi;
  }
  return (P > kTauParts ? 2 : kPartStages) * part_stage_doubles<P>();
}
// Ring stages of each phase: the ring split into stages of that phase's
// records.  Forward: as many (record, right-hand side) stage pairs as fit;
// backward: the fixed depth kPartStages (1 and 4 partitions) or two; H: six
// stages (1 and 4 partitions) or as many as fit.
template <int P>
__host__ __device__ constexpr int fwd_stages() {
  constexpr size_t F = part_rows<P>() * (2 * kSolveModes * kFwdRec + 2 * 2 * kSolveModes);
  return (int)(ring_doubles<P>() / F);
}
template <int P>
__host__ __device__ constexpr int bwd_stages() {
  return P > kTauParts ? 2 : kPartStages;
}
template <int P>
__host__ __device__ constexpr int h_stages() {
  constexpr size_t H =
      part_rows<P>() * (2 * kSolveModes * kHRec + (P > kTauParts8 ? 4 * kSolveModes : 0));
  return P > kTauParts ? (int)(ring_doubles<P>() / H) : 6;
}

// X (the state planes) and the tau rows are one allocation, so a 32-bit
// element offset from X addresses both; code = 2 * offset + (1 if the unknown is i
// times the solved real-ified column), -1 for no store.  u_x = i v gives
// re(u_x) = -v_im (part-1 lane) and im(u_x) = v_re (part-0 lane).
// With X32 non-null the value also goes, rounded, to the FP32 copy of the
// first x32_lim doubles of X (the b, u_x, u_z planes the mixed RHS reads), so
// that no rounding pass has to run before the stage's right-hand side.
__device__ __forceinline__ void store_unknown(double* Xd, int code, int m, int part, double x, bool on,
                                              float* X32 = nullptr, long long x32_lim = 0) {
  if (on && code >= 0) {
    const int rl = code & 1;
    const size_t i = 2 * ((size_t)(code >> 1) + m) + (part ^ rl);
    const double v = (rl & part) ? -x : x;
    Xd[i] = v;
    if (X32 != nullptr && (long long)i < x32_lim) X32[i] = (float)v;
  }
}

template <int KL, int KU, int P, int PPW>
__global__ void __launch_bounds__(32 * P / PPW) k_tau_solve(TauArgs a) {
  static_assert(KL + 2 == kFwdWin && KL + KU == kBwdWin, "window sizes follow the band shape");
  constexpr int R = part_rows<P>();  // rows per ring stage
  static_assert(kFwdWin % R == 0 && kBwdWin % R == 0, "whole stages per forward window and per backward block");
  static_assert(kFwdRec == KL + NBMAX + 2 && kFwdRot == kFwdRec - 1 && kFwdRec % 2 == 0,
                "forward record: pivot, l, border, rotation flag of the entering row");
  static_assert(kBwdCode == KL + KU + 1 + NBMAX && kBwdG == kBwdCode + 1 && kBwdRec == kBwdG + 4 && kBwdRec % 2 == 0,
                "backward record: 1/d, u, border, code, G");
  static_assert(kHRec == kBwdWin && kHRec % 2 == 0, "H record: the 12 responses");
  constexpr int MP = kSolveModes;
  constexpr int W1 = KL + KU + 1;
  constexpr int FREC = 2 * MP * kFwdRec;  // doubles per forward row (both classes)
  constexpr int BREC = 2 * MP * kBwdRec;  // doubles per backward row
  constexpr int HREC = 2 * MP * kHRec;    // doubles per H row
  constexpr int RREC = 2 * MP;            // double2 rhs entries per row (class, mode)
  constexpr int FV = kFwdRec / 2, BV = kBwdRec / 2, HV = kHRec / 2;  // 16-byte words per record
  constexpr int NL = 4 * MP;  // distinct lanes of a partition
  constexpr int TPL = 32 / PPW;  // threads per partition (a warp, or a half-warp)
  constexpr int BSUB = 3;     // backward rows whose records are held in registers at once
  constexpr int RING = (int)ring_doubles<P>();  // doubles of one partition's ring
  constexpr bool YG = ys_global<P>();  // y and particular unknowns in global scratch
  constexpr int NSF = fwd_stages<P>(), NSB = bwd_stages<P>(), NSH = h_stages<P>();
  constexpr int WS = kFwdWin / R;      // ring stages per forward window
  constexpr int KB = kBwdWin / R;      // ring stages per backward block
  constexpr int FRS = R * FREC;        // forward stage: records,
  constexpr int FHS = R * 2 * RREC;    // and right-hand sides (separate slots)
  constexpr int BST = R * (BREC + (YG ? NL : 0));  // backward stage (+ y)
  static_assert(NSF >= 2 * WS && NSF * (FRS + FHS) <= RING && NSB >= 2 && NSB * BST <= RING, "ring stages");
  static_assert(NL <= TPL && TPL % NL == 0 && P % PPW == 0 && (PPW == 1 || PPW == 2), "lane layout");
  static_assert(R % BSUB == 0, "backward sub-blocks");
  extern __shared__ __align__(16) double smem[];
  const int np = a.npad;
  const int Nk = a.Nk;
  const int g = blockIdx.x;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  // partition pid of this thread: the warp's own (PPW = 1, lanes NL.. mirror
  // lanes 0..NL-1), or one per half-warp (PPW = 2); tl = lane within it
  const int pid = warp * PPW + lane / TPL, tl = lane % TPL;
  const int row0 = tau_part_row0(np, P, pid, PPW), Lp = tau_part_row0(np, P, pid + 1, PPW) - row0;
  const int nst = Lp / R;  // ring stages of this partition's rows (even: Lp is whole backward windows)
  const int ln = lane % NL;
  const int c = ln / (2 * MP), part = (ln / MP) & 1, mm = ln % MP;
  const int slot = c * MP + mm;
  const bool owner = tl < NL;
  const int m = g * MP + mm;
  const bool live = owner && m < Nk;
  double* ring = smem + (size_t)pid * RING;
  // [row][ln]: y, then (rows of partitions < P-1) particular x.  With 1 and 16
  // partitions the group's column lives in global scratch (written by F1 and
  // B1 and read back, through the rings, by B1 and B3 of the same CTA while it
  // is still in L2), which leaves the shared memory to the rings.
  double* ysave = YG ? a.ysave + (size_t)g * np * NL : smem + (size_t)P * RING;
  double* xch = smem + (size_t)P * RING + (YG ? 0 : (size_t)np * NL);  // [partition][ln][kXch]
  int* rofs = reinterpret_cast<int*>(xch + (size_t)P * NL * kXch);
  // [row][class] right-hand-side code: 2 * element offset + (1 for a u_x momentum
  // row, scaled by -i on load), -1 for none
  for (int q = threadIdx.x; q < np / 2; q += blockDim.x) cp_async16(rofs + 4 * q, a.rhs_off + 4 * q, true);
  // [row][class] 16-bit store targets of the H pass (2 R + flag, -1 for none)
  short* xcs = reinterpret_cast<short*>(rofs + 2 * np);
  for (int q = threadIdx.x; q < np / 4; q += blockDim.x) cp_async16(xcs + 8 * q, a.xcode + 8 * q, true);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  TB_SOLVE_CLOCK(0);
  const double* FRg = a.cls[0].FR + (size_t)g * np * FREC;
  const double* BRg = a.cls[0].BR + (size_t)g * np * BREC;
  const double* HRg = a.HR + (size_t)g * np * HREC;
  double* Xd = reinterpret_cast<double*>(a.X);

  // ---- F1: forward sweep over this partition's rows: y = L^-1 P r, boundary rows accumulate z ----
  double y[kFwdWin];
  double z[NBMAX];
  // Ring: NSF record slots, then NSF right-hand-side slots.  Group k (k >= -WS)
  // loads the records of stage k (0 <= k < nst) and the right-hand sides of
  // stage k + WS (rows past the partition are the next partition's first rows,
  // zero-filled past the last row): a window's records arrive with the
  // right-hand sides of the rows that enter the window as it is swept.
  auto frec = [&](int st) { return ring + (size_t)(st % NSF) * FRS; };
  auto frhs = [&](int st) { return ring + (size_t)NSF * FRS + (size_t)(st % NSF) * FHS; };
  auto issue_fwd = [&](int k) {
    if (k >= 0 && k < nst) {
      double* dst = frec(k);
      const double* src = FRg + (size_t)(row0 + k * R) * FREC;
      for (int q = tl; q < FRS / 2; q += TPL) cp_async16(dst + 2 * q, src + 2 * q, true);
    }
    if (k < nst) {
      const int r0 = row0 + (k + WS) * R;
      double2* rdst = reinterpret_cast<double2*>(frhs(k + WS));
      for (int q = tl; q < R * RREC; q += TPL) {
        const int r = q / RREC, cc = (q / MP) % 2, md = q % MP;
        const int mq = g * MP + md;
        const int code = (r0 + r < np) ? rofs[2 * (r0 + r) + cc] : -1;
        const bool ok = code >= 0 && mq < Nk;
        cp_async16(rdst + q, a.rhsP + (ok ? (size_t)(code >> 1) + mq : 0), ok);
      }
    }
    cp_async_commit();
  };
  // right-hand side of row row0 + rr for this lane (0 past the last row);
  // u_x momentum rows are scaled by -i, i.e. (re, im) -> (im, -re)
  auto rhs_at = [&](int rr) -> double {
    const int j = row0 + rr;
    if (j >= np) return 0.0;
    const double* rb = frhs(rr / R) + (size_t)((rr % R) * RREC + slot) * 2;
    const int rot = rofs[2 * j + c] & 1;
    const double v = rb[part ^ rot];
    return (rot & part) ? -v : v;
  };
#pragma unroll
  for (int b = 0; b < NBMAX; ++b)
    z[b] = (pid == 0 && part == 0 && m < Nk && m % a.Nkm == 0 && b < a.cls[c].nb) ? a.beta * a.cls[c].bc_rhs[b]
                                                                                  : 0.0;
  if (a.bcdyn != nullptr && pid == 0 && m < Nk) {
    // dynamic wall values of b: boundary row 0 of class c is the parity-c
    // combination of the walls, (top + bottom)/2 (c = 0) or (top - bottom)/2,
    // with both walls at the stage time (value + rate * t)
    const double t = *a.t_dev + a.bc_toff;
    const double2 v0b = a.bcdyn[m], v1b = a.bcdyn[Nk + m], v0t = a.bcdyn[2 * (size_t)Nk + m],
                  v1t = a.bcdyn[3 * (size_t)Nk + m];
    const double bot = part ? fma(v1b.y, t, v0b.y) : fma(v1b.x, t, v0b.x);
    const double top = part ? fma(v1t.y, t, v0t.y) : fma(v1t.x, t, v0t.x);
    z[0] = a.beta * 0.5 * (c == 0 ? top + bot : top - bot);
  }
  for (int k = -WS; k < NSF - WS; ++k) issue_fwd(k);
  cp_async_wait<NSF - WS>();  // groups -WS..-1: the right-hand sides of the first window
  __syncwarp();
#pragma unroll
  for (int t = 0; t < kFwdWin; ++t) y[t] = rhs_at(t);
  __syncwarp();  // those slots are refilled next
  for (int s = 0; s < nst; s += WS) {
    for (int k = s + NSF - WS; k < s + NSF; ++k) issue_fwd(k);  // the previous window's slots
    cp_async_wait<NSF - WS>();  // groups up to s + WS - 1 are resident
    __syncwarp();
    double2 rv[kFwdWin][FV];
#pragma unroll
    for (int u = 0; u < kFwdWin; ++u) {
      const double2* st =
          reinterpret_cast<const double2*>(frec(s + u / R) + (size_t)(u % R) * FREC + (size_t)slot * kFwdRec);
#pragma unroll
      for (int v = 0; v < FV; ++v) rv[u][v] = st[v];
    }
    // right-hand sides of the rows entering the window (zero-filled past the
    // last row), -i applied to u_x momentum rows by the record's flag
    double incoming[kFwdWin];
#pragma unroll
    for (int u = 0; u < kFwdWin; ++u) {
      const double* rb = frhs(s + WS + u / R) + (size_t)((u % R) * RREC + slot) * 2;
      const int rot = __double2loint(rv[u][FV - 1].y);
      const double v = rb[part ^ rot];
      incoming[u] = (rot & part) ? -v : v;
    }
    double* ys = ysave + (size_t)(row0 + s * R) * NL + ln;
#pragma unroll
    for (int u = 0; u < kFwdWin; ++u) {
      auto rec = [&](int k) -> double { return (k & 1) ? rv[u][k >> 1].y : rv[u][k >> 1].x; };
      const int p = __double2loint(rv[u][0].x);
      double yj = y[u];
#pragma unroll
      for (int t = 1; t <= KL; ++t) {
        const bool sw = (t == p);
        const double yt = y[(u + t) % kFwdWin];
        y[(u + t) % kFwdWin] = sw ? yj : yt;
        yj = sw ? yt : yj;
      }
      ys[u * NL] = yj;
#pragma unroll
      for (int t = 1; t <= KL; ++t) y[(u + t) % kFwdWin] = fma(-rec(t), yj, y[(u + t) % kFwdWin]);
#pragma unroll
      for (int b = 0; b < NBMAX; ++b) z[b] = fma(-rec(1 + KL + b), yj, z[b]);
      y[u] = incoming[u];
    }
    __syncwarp();  // the window's slots are refilled next
  }
  TB_SOLVE_CLOCK(1);
  double* myx = xch + ((size_t)pid * NL + ln) * kXch;
  // exit window minus the raw right-hand side of the next partition's first rows (the
  // ring still holds those right-hand sides)
#pragma unroll
  for (int t = 0; t < 4; ++t) myx[t] = y[t] - rhs_at(Lp + t);
  cp_async_wait<0>();
  if constexpr (YG) __threadfence();  // y stores of all lanes reach L2 before their cp.async reloads
  __syncwarp();
  // The ring is free: stage the Schur inverse of the group and this partition's
  // forward transfer data while the other partitions finish their sweeps:
  // Phi_k for k < pid and Gz_pid (up to 8 partitions: each partition composes
  // its own starting window), or its own Phi_pid and Gz_pid (16 partitions:
  // the windows are carried down one partition at a time).
  constexpr bool CARRY = P > kTauParts8;
  constexpr int TRF = 32;  // Phi (16) + Gz (16) per (partition, record slot)
  // shared-memory stride of a staged (partition, slot) record: 34 doubles, so
  // that the 8 slots a warp reads at once fall in distinct banks
  constexpr int TRS = TRF + 2;
  static_assert(2 * NBMAX * NBMAX * MP + (CARRY ? 1 : P - 1) * 2 * MP * TRS <= RING,
                "Schur inverse and Phi fit the ring");
  double* sSI = ring;                         // [class][4][4][mode], 2*16*MP doubles
  double* sTR = ring + 2 * NBMAX * NBMAX * MP;  // [k-1][slot][TRS] (carry: [slot][TRS] of Phi_pid)
  {
    const double* SIg = a.cls[0].SI + (size_t)g * 2 * NBMAX * NBMAX * MP;
    for (int q = tl; q < NBMAX * NBMAX * MP; q += TPL) cp_async16(sSI + 2 * q, SIg + 2 * q, true);
    if (P > 1 && pid > 0) {
      const int k1 = CARRY ? pid : 1;  // first staged partition (slot 0)
      for (int q = tl; q < (pid - k1 + 1) * 2 * MP * (TRF / 2); q += TPL) {
        const int k = k1 + q / (2 * MP * (TRF / 2)), rs = (q / (TRF / 2)) % (2 * MP), h = q % (TRF / 2);
        const double* rec = a.PP + (((size_t)g * P + k) * 2 * MP + rs) * kTransfer;
        const double* src = (h < 8) ? rec + kTrPhi + 2 * h : rec + kTrGz + 2 * (h - 8);
        cp_async16(sTR + ((size_t)(k - k1) * 2 * MP + rs) * TRS + 2 * h, src, true);
      }
    }
    cp_async_commit();
  }

  // ---- F2: true starting window of this partition, border accumulators ----
  double d[4] = {0.0, 0.0, 0.0, 0.0};  // starting-window correction (0 for partition 0)
  if constexpr (P > 1) {
    __syncthreads();
    cp_async_wait<0>();
    __syncwarp();
    if constexpr (CARRY) {
      // delta_1 = D_0, delta_{k+1} = D_k + Phi_k delta_k: partition k reads
      // delta_k (published by k-1 in the exchange slots of its Xhat, free
      // until B2), publishes delta_{k+1}, one barrier per partition
      for (int k = 1; k < P; ++k) {
        if (pid == k) {
          const double* src = xch + ((size_t)(k - 1) * NL + ln) * kXch + (k == 1 ? 0 : 8);
#pragma unroll
          for (int t = 0; t < 4; ++t) d[t] = src[t];
          if (k < P - 1) {
            const double* phi = sTR + (size_t)slot * TRS;
            const double* Dk = xch + ((size_t)k * NL + ln) * kXch;
            double nd[4];
#pragma unroll
            for (int o = 0; o < 4; ++o) {
              double acc = Dk[o];
#pragma unroll
              for (int i = 0; i < 4; ++i) acc = fma(phi[o * 4 + i], d[i], acc);
              nd[o] = acc;
            }
#pragma unroll
            for (int o = 0; o < 4; ++o) myx[8 + o] = nd[o];
          }
        }
        __syncthreads();
      }
      if (pid > 0) {
        const double* gz = sTR + (size_t)slot * TRS + 16;
#pragma unroll
        for (int b = 0; b < NBMAX; ++b)
#pragma unroll
          for (int i = 0; i < 4; ++i) z[b] = fma(gz[b * 4 + i], d[i], z[b]);
      }
    } else if (pid > 0) {
#pragma unroll
      for (int t = 0; t < 4; ++t) d[t] = xch[(size_t)ln * kXch + t];  // delta_1 = D_0
      for (int k = 1; k < pid; ++k) {
        const double2* phi = reinterpret_cast<const double2*>(sTR + ((size_t)(k - 1) * 2 * MP + slot) * TRS);
        const double* Dk = xch + ((size_t)k * NL + ln) * kXch;
        double nd[4];
#pragma unroll
        for (int o = 0; o < 4; ++o) {
          const double2 w0 = phi[2 * o], w1 = phi[2 * o + 1];
          double acc = Dk[o];
          acc = fma(w0.x, d[0], acc);
          acc = fma(w0.y, d[1], acc);
          acc = fma(w1.x, d[2], acc);
          acc = fma(w1.y, d[3], acc);
          nd[o] = acc;
        }
#pragma unroll
        for (int o = 0; o < 4; ++o) d[o] = nd[o];
      }
      const double* gz = sTR + ((size_t)(pid - 1) * 2 * MP + slot) * TRS + 16;
#pragma unroll
      for (int b = 0; b < NBMAX; ++b)
#pragma unroll
        for (int i = 0; i < 4; ++i) z[b] = fma(gz[b * 4 + i], d[i], z[b]);
    }
#pragma unroll
    for (int b = 0; b < NBMAX; ++b) myx[4 + b] = z[b];
    __syncthreads();
#pragma unroll
    for (int b = 0; b < NBMAX; ++b) {
      double acc = 0.0;
      for (int k = 0; k < P; ++k) acc += xch[((size_t)k * NL + ln) * kXch + 4 + b];
      z[b] = acc;
    }
  } else {
    cp_async_wait<0>();
    __syncwarp();
  }

  // ---- border unknowns from the Schur complement ----
  TB_SOLVE_CLOCK(2);
  double x1[NBMAX];
  {
    const double* si = sSI + (size_t)c * NBMAX * NBMAX * MP + mm;
#pragma unroll
    for (int q = 0; q < NBMAX; ++q) {
      double acc = 0.0;
#pragma unroll
      for (int b = 0; b < NBMAX; ++b) acc = fma(si[(q * NBMAX + b) * MP], z[b], acc);
      x1[q] = acc;
    }
  }
  __syncwarp();  // the ring is reused by B1

  // ---- B1: backward sweep over this partition's rows, x = U^-1 (y - B x1), from a zero window ----
  // (the particular unknowns replace y in shared memory; B3 completes and stores them)
  double xw[kBwdWin];  // x_j lives in slot j % kBwdWin
#pragma unroll
  for (int t = 0; t < kBwdWin; ++t) xw[t] = 0.0;
  auto issue_bwd = [&](int s) {  // local stage s from the bottom: rows row0 + Lp - (s+1) R ..
    if (s < nst) {
      double* dst = ring + (size_t)(s % NSB) * BST;
      const int lo = row0 + Lp - (s + 1) * R;
      for (int q = tl; q < R * BREC / 2; q += TPL) cp_async16(dst + 2 * q, BRg + (size_t)lo * BREC + 2 * q, true);
      if constexpr (YG)
        for (int q = tl; q < R * NL / 2; q += TPL)
          cp_async16(dst + R * BREC + 2 * q, ysave + (size_t)lo * NL + 2 * q, true);
    }
    cp_async_commit();
  };
  for (int s = 0; s < NSB - 1; ++s) issue_bwd(s);
  for (int s0 = 0; s0 < nst; s0 += KB) {
    const int q0 = row0 + Lp - (s0 + KB) * R;  // block rows q0 .. q0 + kBwdWin - 1, q0 % kBwdWin == 0
#pragma unroll
    for (int hs = 0; hs < KB; ++hs) {
      const int s = s0 + hs;
      issue_bwd(s + NSB - 1);
      cp_async_wait<NSB - 1>();  // stage s is resident
      __syncwarp();
      const double2* st = reinterpret_cast<const double2*>(ring + (size_t)(s % NSB) * BST + (size_t)slot * kBwdRec);
#pragma unroll
      for (int h = 0; h < R / BSUB; ++h) {
        // rows q0 + kBwdWin - 1 - u for u = hs R + h BSUB + w; stage row index R - 1 - (h BSUB + w)
        double2 rv[BSUB][BV];
#pragma unroll
        for (int w = 0; w < BSUB; ++w)
#pragma unroll
          for (int v = 0; v < BV; ++v) rv[w][v] = st[(R - 1 - (h * BSUB + w)) * (BREC / 2) + v];
#pragma unroll
        for (int w = 0; w < BSUB; ++w) {
          const int u = hs * R + h * BSUB + w;
          const int j = q0 + kBwdWin - 1 - u;  // j % kBwdWin == kBwdWin-1-u
          auto rec = [&](int k) -> double { return (k & 1) ? rv[w][k >> 1].y : rv[w][k >> 1].x; };
          double* yx = ysave + (size_t)j * NL + ln;
          double acc0;
          if constexpr (YG)
            acc0 = ring[(size_t)(s % NSB) * BST + R * BREC + (R - 1 - (h * BSUB + w)) * NL + ln];
          else
            acc0 = *yx;
          double acc1 = 0.0, acc2 = 0.0;
#pragma unroll
          for (int i = 0; i < 4; ++i) acc2 = fma(rec(kBwdG + i), d[i], acc2);  // y correction G d
#pragma unroll
          for (int b = 0; b < NBMAX; ++b) acc1 = fma(-rec(W1 + b), x1[b], acc1);
#pragma unroll
          for (int t = kBwdWin; t >= 2; --t) {
            const int sl = (kBwdWin - 1 - u + t) % kBwdWin;
            if (t % 3 == 0)
              acc0 = fma(-rec(t), xw[sl], acc0);
            else if (t % 3 == 1)
              acc1 = fma(-rec(t), xw[sl], acc1);
            else
              acc2 = fma(-rec(t), xw[sl], acc2);
          }
          const double sacc = fma(-rec(1), xw[(kBwdWin - u) % kBwdWin], acc0 + (acc1 + acc2));
          const double xj = sacc * rec(0);
          xw[(kBwdWin - 1 - u) % kBwdWin] = xj;
          if (P == 1 || pid == P - 1)
            store_unknown(Xd, __double2loint(rec(kBwdCode)), m, part, xj, live, a.X32,
                          a.x32_lim);  // final: no correction
          else
            *yx = xj;
        }
      }
      __syncwarp();  // the slot of stage s is refilled next
    }
  }
  cp_async_wait<0>();
  if constexpr (YG && P > 1) __threadfence();  // particular x of all lanes reach L2 before B3 reloads them
  __syncwarp();

  // ---- B2: true incoming window T of this partition (zero for the last) ----
  TB_SOLVE_CLOCK(3);
  const bool last = (pid == P - 1);
  double T[kBwdWin];
#pragma unroll
  for (int t = 0; t < kBwdWin; ++t) T[t] = 0.0;
  // B3's H ring: NSH slots of R rows (+ the particular x with y in global scratch)
  constexpr int SLOT3 = R * HREC + (YG ? R * NL : 0);
  static_assert(P == 1 || (NSH >= 2 && NSH * SLOT3 <= RING), "H ring fits the partition's ring");
  const int nst3 = last ? 0 : nst;  // H stages this partition streams
  auto issue_h = [&](int s) {
    if (s < nst3) {
      double* dst = ring + (size_t)(s % NSH) * SLOT3;
      const int lo = row0 + s * R;
      for (int q = tl; q < R * HREC / 2; q += TPL) cp_async16(dst + 2 * q, HRg + (size_t)lo * HREC + 2 * q, true);
      if constexpr (YG)
        for (int q = tl; q < R * NL / 2; q += TPL)
          cp_async16(dst + R * HREC + 2 * q, ysave + (size_t)lo * NL + 2 * q, true);
    }
    cp_async_commit();
  };
  // Psi sits at the end of the ring, so the first H stages of B3 (the ring's
  // front) stream in while the windows are carried
  constexpr int PS = kBwdWin * kBwdWin + 2;
  constexpr int PSI = 2 * MP * PS;
  constexpr int NPRE = (RING - PSI) / SLOT3 < NSH - 1 ? (RING - PSI) / SLOT3 : NSH - 1;  // H stages prefetched
  if constexpr (P > 1) {
    // Carry from the bottom: T_{P-2} = Xhat_{P-1} (the last partition's top
    // window is exact), T_{k-1} = Xhat_k + Psi_k T_k.  Partition k (1 <= k <=
    // P-2) stages its own Psi_k (transposed: row i holds the responses of the
    // 12 outputs to input i) in its ring, [slot][PS] with the stride PS = 146
    // doubles putting the 8 slots read at once in distinct banks, and
    // overwrites its published Xhat_k with T_{k-1}, which partition k-1 reads.
    // The carry runs warp by warp from the bottom as soon as each warp has
    // finished B1: within a warp the hand-over is a __syncwarp, between warps
    // w and w-1 the named barrier w (64 threads: w arrives after writing its
    // lowest partition's output, w-1 before reading it), so the lower warps
    // carry while the upper ones still sweep, and each partition starts B3 as
    // soon as it has its window.
    static_assert(PSI <= RING, "Psi fits the ring");
    static_assert(P / PPW <= 16, "one named barrier per pair of adjacent warps");
    double* sPsi = ring + (RING - PSI);
    if (pid >= 1 && pid <= P - 2) {
      for (int q = tl; q < 2 * MP * 72; q += TPL) {
        const int rs = q / 72, h = q % 72;
        const double* rec = a.PP + (((size_t)g * P + pid) * 2 * MP + rs) * kTransfer + kTrPsi;
        cp_async16(sPsi + (size_t)rs * PS + 2 * h, rec + 2 * h, true);
      }
    }
    cp_async_commit();
    for (int s = 0; s < NPRE; ++s) issue_h(s);
    double* myxh = myx + 8;
#pragma unroll
    for (int t = 0; t < kBwdWin; ++t) myxh[t] = xw[t];
    cp_async_wait<NPRE>();  // Psi (the H stages may still be in flight)
    __syncwarp();
    constexpr int NW = P / PPW;  // warps of the CTA
#pragma unroll
    for (int h = PPW - 1; h >= 0; --h) {
      const int k = warp * PPW + h;  // the partition of this warp whose window is carried now
      if (k < P - 1) {
        // its window T_k is the output of partition k + 1: the warp below
        // (named barrier warp + 1) or the other half of this warp
        if (h == PPW - 1) {
          __syncwarp();  // the whole warp reaches the barrier together
          if (warp < NW - 1) asm volatile("bar.sync %0, %1;" ::"r"(warp + 1), "r"(64) : "memory");
        } else {
          __syncwarp();
        }
        if (pid == k) {
          const double* Xn = xch + ((size_t)(k + 1) * NL + ln) * kXch + 8;
#pragma unroll
          for (int t = 0; t < kBwdWin; ++t) T[t] = Xn[t];
          if (k >= 1) {
            // twelve independent accumulators, input by input (16-byte rows of
            // Psi^T); each output still sums its inputs in order 0..11
            const double2* psi = reinterpret_cast<const double2*>(sPsi + (size_t)slot * PS);
            double nt[kBwdWin];
#pragma unroll
            for (int o = 0; o < kBwdWin; ++o) nt[o] = xw[o];
#pragma unroll
            for (int i = 0; i < kBwdWin; ++i)
#pragma unroll
              for (int o = 0; o < kBwdWin; o += 2) {
                const double2 w = psi[(i * kBwdWin + o) / 2];
                nt[o] = fma(w.x, T[i], nt[o]);
                nt[o + 1] = fma(w.y, T[i], nt[o + 1]);
              }
#pragma unroll
            for (int o = 0; o < kBwdWin; ++o) myxh[o] = nt[o];  // lanes ln and ln + NL write the same values
          }
        }
      }
      // this warp's lowest partition has written its output: hand it up
      __syncwarp();
      if (h == 0 && warp >= 1) asm volatile("bar.sync %0, %1;" ::"r"(warp), "r"(64) : "memory");
    }
    __syncwarp();  // the ring is reused by B3
  }

  // ---- B3: x_j = particular + H_j . T over the rows of this partition, stored to X ----
  TB_SOLVE_CLOCK(4);
  // (the last partition stored its unknowns in B1: its threads run the loop
  // without loads or stores, so the warp-wide syncs see every lane)
  if constexpr (P > 1) {
    constexpr int LG = TPL / NL;  // lane groups: each takes every LG-th row of a stage
    const int grp = tl / NL;
    const int nloop = __shfl_sync(0xffffffffu, nst3, 0) > __shfl_sync(0xffffffffu, nst3, 31)
                          ? __shfl_sync(0xffffffffu, nst3, 0)
                          : __shfl_sync(0xffffffffu, nst3, 31);  // the warp's trip count
    for (int s = NPRE; s < NSH - 1; ++s) issue_h(s);
    for (int s = 0; s < nloop; ++s) {
      issue_h(s + NSH - 1);
      cp_async_wait<NSH - 1>();
      __syncwarp();
      if (s < nst3) {
        const double2* st =
            reinterpret_cast<const double2*>(ring + (size_t)(s % NSH) * SLOT3 + (size_t)slot * kHRec);
        // no recurrence here: the lane groups take interleaved rows
#pragma unroll
        for (int q = 0; q < (R + LG - 1) / LG; ++q) {
          const int u = q * LG + grp;
          if (u >= R) break;
          double2 hv[HV];
#pragma unroll
          for (int v = 0; v < HV; ++v) hv[v] = st[u * (HREC / 2) + v];
          const int j = row0 + s * R + u;
          double acc0 = YG ? ring[(size_t)(s % NSH) * SLOT3 + R * HREC + u * NL + ln] : ysave[(size_t)j * NL + ln];
          double acc1 = 0.0;
#pragma unroll
          for (int i = 0; i < kBwdWin; i += 2) {
            acc0 = fma(hv[i / 2].x, T[i], acc0);
            acc1 = fma(hv[i / 2].y, T[i + 1], acc1);
          }
          const int xc = xcs[2 * j + c];  // 2 R + flag -> store code 2 R Nk + flag
          store_unknown(Xd, xc < 0 ? -1 : 2 * (xc >> 1) * Nk + (xc & 1), m, part, acc0 + acc1, m < Nk, a.X32,
                        a.x32_lim);
        }
      }
      __syncwarp();
    }
    cp_async_wait<0>();
  }
  TB_SOLVE_CLOCK(5);
  // border unknowns
  if (pid == 0) {
#pragma unroll
    for (int b = 0; b < NBMAX; ++b) {
      if (live && b < a.cls[c].nb)
        store_unknown(Xd, a.cls[c].left_code[b], m, part, x1[b], true, a.X32, a.x32_lim);
    }
  }
}

// ---------------------------------------------------------------------------
// Partition responses of the solve, one thread per (mode, class, partition,
// unit vector), from the factor records (the arithmetic of the sweeps in
// k_tau_solve).  Partition k owns rows [r0, r1) = [tau_part_row0(k),
// tau_part_row0(k + 1)).  For k >= 1
// (forward, started from unit pending entry i of the window and a zero
// right-hand side):
//   G of row j (backward record slots kBwdG..) = y_j,
//   Phi_k[o][i] = exit pending entry o,  Gz_k[b][i] = border accumulator b.
// For k <= P-2 (backward from unit window entry i, row r1 + i, with zero
// y and border unknowns):
//   H of row j (H record) = x_j,  Psi_k[o][i] = x of row r0 + o (stored
//   transposed, [i][o], so the carry reads it by input).
// ---------------------------------------------------------------------------
template <int KL, int KU, int P, int PPW>
__global__ void __launch_bounds__(128) k_tau_transfer(TauArgs a) {
  // one thread per (mode, class, partition, unit): forward unit i < 4,
  // backward unit i - 4 < 12
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y & 1, k = blockIdx.y >> 1;
  const int i = blockIdx.z;
  if (m >= a.Nk) return;
  const int np = a.npad;
  const int g = m / kSolveModes, mm = m % kSolveModes;
  // Phi, Gz, Psi exist only for P > 1 (a.PP is null otherwise)
  double* tr = P > 1 ? a.PP + ((((size_t)g * P + k) * 2 + c) * kSolveModes + mm) * kTransfer : nullptr;
  const int r0 = tau_part_row0(np, P, k, PPW), r1 = tau_part_row0(np, P, k + 1, PPW);
  if (i < 4) {
    if (k < 1) return;
    double y[kFwdWin], z[NBMAX] = {0.0, 0.0, 0.0, 0.0};
    for (int t = 0; t < kFwdWin; ++t) y[t] = (t == i) ? 1.0 : 0.0;
    for (int j = r0; j < r1; ++j) {
      const double* fr = fwd_record(a.cls[0].FR, np, m, j, c);
      const int u = (j - r0) % kFwdWin;
      const int p = __double2loint(fr[0]);
      double yj = y[u];
      for (int t = 1; t <= KL; ++t) {
        if (t == p) {
          const double yt = y[(u + t) % kFwdWin];
          y[(u + t) % kFwdWin] = yj;
          yj = yt;
        }
      }
      bwd_record(a.cls[0].BR, np, m, j, c)[kBwdG + i] = yj;
      for (int t = 1; t <= KL; ++t) y[(u + t) % kFwdWin] = fma(-fr[t], yj, y[(u + t) % kFwdWin]);
      for (int b = 0; b < NBMAX; ++b) z[b] = fma(-fr[1 + KL + b], yj, z[b]);
      y[u] = 0.0;
    }
    for (int o = 0; o < 4; ++o) tr[kTrPhi + o * 4 + i] = y[o];
    for (int b = 0; b < NBMAX; ++b) tr[kTrGz + b * 4 + i] = z[b];
    return;
  }
  const int ib = i - 4;
  if (k == P - 1) return;  // the last partition's unknowns need no correction (stored by its backward sweep)
  double xw[kBwdWin];
  for (int t = 0; t < kBwdWin; ++t) xw[t] = (t == ib) ? 1.0 : 0.0;
  for (int j = r1 - 1; j >= r0; --j) {
    const double* br = bwd_record(a.cls[0].BR, np, m, j, c);
    double acc = 0.0;
    for (int t = 1; t <= KL + KU; ++t) acc = fma(-br[t], xw[(j + t) % kBwdWin], acc);
    xw[j % kBwdWin] = acc * br[0];
    double* hr = a.HR + ((((size_t)g * np + j) * 2 + c) * kSolveModes + mm) * kHRec;
    hr[ib] = xw[j % kBwdWin];
  }
  for (int o = 0; o < kBwdWin; ++o) tr[kTrPsi + ib * kBwdWin + o] = xw[o];  // Psi^T: row ib
}

template <int N>
__global__ void k_lincomb(LinComb lc, double2* __restrict__ out, long long count) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    double2 v[N];
#pragma unroll
    for (int t = 0; t < N; ++t) v[t] = lc.in[t][i];  // all loads in flight before the sums
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int t = 0; t < N; ++t) acc = cfma(lc.w[t], v[t], acc);
    out[i] = acc;
  }
}

__device__ __forceinline__ double2 proj(double2 v, bool p) { return p ? make_double2(v.x, 0.0) : v; }

// State plane and equation plane of velocity-like field q (b, u_x / u_par,
// u_z, then u_perp in 3D).
__device__ __forceinline__ int xplane_of(int q) { return q < 3 ? q : 4; }
__device__ __forceinline__ int eplane_of(int q) { return q < 3 ? 1 + q : 4; }

// One thread per (row k, mode m): grid (ceil(Nk / 128), Nz).
// Advance the device time of dynamic wall values by dt (end of a step).
__global__ void k_advance_time(double* t, double dt) { *t += dt; }

__global__ void __launch_bounds__(128) k_mass_apply(const double2* __restrict__ X, double2* __restrict__ MX,
                                                    const double* __restrict__ s3, int Nz, int Nk, int Nx,
                                                    int project, int nf, int Nkm) {
  const int k = blockIdx.y, m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= Nk) return;
  const size_t i = (size_t)k * Nk + m;
  const int ml = m % Nkm;  // mode within its instance
  const bool pj = project && (ml == 0 || 2 * ml == Nx);
  const double s0 = s3[3 * k], s1 = s3[3 * k + 1], s2 = s3[3 * k + 2];
  MX[i] = make_double2(0.0, 0.0);
  for (int f = 0; f < nf; ++f) {
    const double2* Xf = X + (size_t)xplane_of(f) * Nz * Nk;
    double2 acc = make_double2(0.0, 0.0);
    acc = cfma(s0, proj(Xf[i], pj), acc);
    if (k + 2 < Nz) acc = cfma(s1, proj(Xf[i + 2 * (size_t)Nk], pj), acc);
    if (k + 4 < Nz) acc = cfma(s2, proj(Xf[i + 4 * (size_t)Nk], pj), acc);
    MX[(size_t)eplane_of(f) * Nz * Nk + i] = acc;
  }
}

// One thread per (row k, mode m): grid (ceil(Nk / 128), Nz).
__global__ void __launch_bounds__(128) k_lx_finalize(double2* __restrict__ LX, const double2* __restrict__ X,
                                                     const double* __restrict__ s3, int Nz, int Nk, int Nx, double k0,
                                                     double s, double kappa, double nu, double beta, int nf, int Nkm,
                                                     const double* __restrict__ kappa_m,
                                                     const double* __restrict__ nu_m) {
  const double ib = 1.0 / beta;
  {
    const int k = blockIdx.y, m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= Nk) return;
    const size_t i = (size_t)k * Nk + m;
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
    if (nf > 3) {  // u_perp rows (3D): the equation plane after the pressure
      double2 r = LX[4 * plane + i];
      const double2 mx = Sx(4);
      LX[4 * plane + i] = make_double2((r.x - mx.x) * ib, (r.y - mx.y) * ib);
    }
    const int ml = m % Nkm;  // mode within its instance
    if (Nx > 0 && (ml == 0 || 2 * ml == Nx)) {
      // L applied to delta = i Im(X) of b, ux, uz (the part a grid round trip drops)
      const double kx = k0 * ml, kx2 = kx * kx;
      if (kappa_m) {
        kappa = kappa_m[m / Nkm];
        nu = nu_m[m / Nkm];
      }
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

// Final RK update X_f = S^{-1} y for f = b, ux, uz, where y is the stage
// combination of the b / u_x / u_z equation rows (C^(2) space).  S is upper
// triangular with offsets 0, +2, +4, so each (field, parity, mode) column is a
// short backward recurrence.  A CTA owns kFinalModes modes of one (field,
// parity): its 256 threads form y for all rows into shared memory (every
// input of a row in flight at once), together with the S entries of those
// rows and the reciprocal diagonal; the first kFinalModes threads run the
// recurrences out of shared memory, and all threads write X back.
constexpr int kFinalModes = 8;
template <int N>
__global__ void __launch_bounds__(256) k_rk_final(LinComb lc, double2* __restrict__ X, const double* __restrict__ s3,
                                                  int Nz, int Nk) {
  extern __shared__ double2 ys[];  // [rows of this parity][kFinalModes], then 3 doubles per row
  constexpr int MB = kFinalModes, RG = 256 / MB;  // modes per CTA, row groups
  const int f = blockIdx.y >> 1, par = blockIdx.y & 1;
  const int mm = threadIdx.x % MB, ks = threadIdx.x / MB;
  const int m = blockIdx.x * MB + mm;
  const size_t plane = (size_t)Nz * Nk;
  const int K = (Nz - par + 1) / 2;  // rows k = par + 2 ri
  double* sk = reinterpret_cast<double*>(ys + (size_t)K * MB);  // [ri][3]: 1/S_kk, S_k,k+2, S_k,k+4
  for (int q = threadIdx.x; q < K; q += blockDim.x) {
    const int k = par + 2 * q;
    sk[3 * q] = 1.0 / s3[3 * k];
    sk[3 * q + 1] = s3[3 * k + 1];
    sk[3 * q + 2] = s3[3 * k + 2];
  }
  const size_t base = (size_t)eplane_of(f) * plane;  // equation rows of field f
  const int mc = m < Nk ? m : Nk - 1;           // clamped column: loads stay in bounds
  for (int r0 = ks; r0 < K; r0 += 2 * RG) {
    const int r1 = (r0 + RG < K) ? r0 + RG : r0;
    const size_t e0 = base + (size_t)(par + 2 * r0) * Nk + mc;
    const size_t e1 = base + (size_t)(par + 2 * r1) * Nk + mc;
    double2 v0[N], v1[N];
#pragma unroll
    for (int t = 0; t < N; ++t) {
      v0[t] = lc.in[t][e0];
      v1[t] = lc.in[t][e1];
    }
    double2 a0 = make_double2(0.0, 0.0), a1 = make_double2(0.0, 0.0);
#pragma unroll
    for (int t = 0; t < N; ++t) {
      a0 = cfma(lc.w[t], v0[t], a0);
      a1 = cfma(lc.w[t], v1[t], a1);
    }
    ys[r0 * MB + mm] = a0;
    if (r0 + RG < K) ys[(r0 + RG) * MB + mm] = a1;
  }
  __syncthreads();
  if (threadIdx.x < MB) {
    double2 x2 = make_double2(0.0, 0.0), x4 = make_double2(0.0, 0.0);
    for (int ri = K - 1; ri >= 0; --ri) {
      double2 y = ys[ri * MB + mm];
      y = cfma(-sk[3 * ri + 1], x2, y);
      y = cfma(-sk[3 * ri + 2], x4, y);
      const double inv = sk[3 * ri];
      const double2 x = make_double2(y.x * inv, y.y * inv);
      ys[ri * MB + mm] = x;
      x4 = x2;
      x2 = x;
    }
  }
  __syncthreads();
  if (m < Nk)
    for (int ri = ks; ri < K; ri += RG)
      X[(size_t)xplane_of(f) * plane + (size_t)(par + 2 * ri) * Nk + m] = ys[ri * MB + mm];
}

template <int KL, int KU>
void factor_impl(const TauArgs& a, int parts, cudaStream_t st) {
  (void)parts;
  dim3 grid((a.Nkm + kFactorWarps - 1) / kFactorWarps, 2);
  k_tau_factor<KL, KU><<<grid, 32 * kFactorWarps, factor_smem_bytes<KL, KU>(), st>>>(a);
}

template <int KL, int KU>
void transfer_impl(const TauArgs& a, int parts, cudaStream_t st) {
  // one partition: the sweeps need no transfer responses (B1 stores x directly)
  const int tgx = (a.Nk + 127) / 128;
  if (parts == kTauParts) k_tau_transfer<KL, KU, kTauParts, 1><<<dim3(tgx, 2 * kTauParts, 16), 128, 0, st>>>(a);
  if (parts == kTauParts8)
    k_tau_transfer<KL, KU, kTauParts8, kTau8PerWarp><<<dim3(tgx, 2 * kTauParts8, 16), 128, 0, st>>>(a);
  if (parts == kTauParts16)
    k_tau_transfer<KL, KU, kTauParts16, kTau8PerWarp><<<dim3(tgx, 2 * kTauParts16, 16), 128, 0, st>>>(a);
}

template <int P>
size_t solve_smem_bytes(int npad) {
  constexpr size_t NL = 4 * kSolveModes;
  const size_t ys = ys_global<P>() ? 0 : (size_t)npad * NL;  // 1 and 16 partitions keep y in global scratch
  return ((size_t)P * ring_doubles<P>() + ys + (size_t)P * NL * kXch) * sizeof(double) +
         (size_t)npad * 2 * (sizeof(int) + sizeof(short));
}

template <int KL, int KU>
void solve_impl(const TauArgs& a, int parts, cudaStream_t st) {
  const int groups = (a.Nk + kSolveModes - 1) / kSolveModes;
  if (parts == kTauParts16)
    k_tau_solve<KL, KU, kTauParts16, kTau8PerWarp>
        <<<groups, 32 * kTauParts16 / kTau8PerWarp, solve_smem_bytes<kTauParts16>(a.npad), st>>>(a);
  else if (parts == kTauParts8)
    k_tau_solve<KL, KU, kTauParts8, kTau8PerWarp>
        <<<groups, 32 * kTauParts8 / kTau8PerWarp, solve_smem_bytes<kTauParts8>(a.npad), st>>>(a);
  else if (parts == kTauParts)
    k_tau_solve<KL, KU, kTauParts, 1><<<groups, 32 * kTauParts, solve_smem_bytes<kTauParts>(a.npad), st>>>(a);
  else
    k_tau_solve<KL, KU, 1, 1><<<groups, 32, solve_smem_bytes<1>(a.npad), st>>>(a);
}

}  // namespace


cudaError_t set_tau_smem_limits(int bytes) {
  cudaError_t e =
      cudaFuncSetAttribute(k_tau_solve<kTauKL, kTauKU, 1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_tau_solve<kTauKL, kTauKU, kTauParts, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           bytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_tau_solve<kTauKL, kTauKU, kTauParts8, kTau8PerWarp>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_tau_solve<kTauKL, kTauKU, kTauParts16, kTau8PerWarp>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  const void* fns[] = {(const void*)k_rk_final<1>,  (const void*)k_rk_final<2>,  (const void*)k_rk_final<3>,
                       (const void*)k_rk_final<4>,  (const void*)k_rk_final<5>,  (const void*)k_rk_final<6>,
                       (const void*)k_rk_final<7>,  (const void*)k_rk_final<8>,  (const void*)k_rk_final<9>,
                       (const void*)k_rk_final<10>, (const void*)k_rk_final<11>, (const void*)k_rk_final<12>};
  for (const void* fn : fns) {
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

size_t tau_solve_smem_bytes(int npad, int parts) {
  if (parts == kTauParts16) return solve_smem_bytes<kTauParts16>(npad);
  if (parts == kTauParts8) return solve_smem_bytes<kTauParts8>(npad);
  return parts == kTauParts ? solve_smem_bytes<kTauParts>(npad) : solve_smem_bytes<1>(npad);
}

size_t tau_transfer_doubles(int Nk, int parts) {
  if (parts <= 1) return 0;
  const size_t groups = (size_t)(Nk + kSolveModes - 1) / kSolveModes;
  return groups * (size_t)parts * 2 * kSolveModes * kTransfer;
}

size_t tau_solve_scratch_doubles(int Nk, int npad, int parts) {
  if (parts != 1 && parts != kTauParts16) return 0;
  const size_t groups = (size_t)(Nk + kSolveModes - 1) / kSolveModes;
  return groups * (size_t)npad * 4 * kSolveModes;
}

size_t tau_response_doubles(int Nk, int npad, int parts) {
  if (parts <= 1) return 0;
  const size_t groups = (size_t)(Nk + kSolveModes - 1) / kSolveModes;
  return groups * (size_t)npad * 2 * kSolveModes * kHRec;
}

// Supported band shape: the RBC layout gives kl = 4, ku = 8 for every Nz >= 8
// (narrower layouts are zero-padded to it by the plan).
void launch_tau_factor(const TauArgs& a, int parts, cudaStream_t st) { factor_impl<kTauKL, kTauKU>(a, parts, st); }
void launch_tau_transfer(const TauArgs& a, int parts, cudaStream_t st) {
  transfer_impl<kTauKL, kTauKU>(a, parts, st);
}
void launch_tau_solve(const TauArgs& a, int parts, cudaStream_t st) { solve_impl<kTauKL, kTauKU>(a, parts, st); }


void launch_lincomb(const LinComb& lc, double2* out, long long count, cudaStream_t st) {
  int blocks = (int)((count + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
#define TB_LINCOMB_CASE(N) \
  case N:                    \
    k_lincomb<N><<<blocks, 256, 0, st>>>(lc, out, count); \
    break;
  switch (lc.n) {
    TB_LINCOMB_CASE(1) TB_LINCOMB_CASE(2) TB_LINCOMB_CASE(3) TB_LINCOMB_CASE(4) TB_LINCOMB_CASE(5) TB_LINCOMB_CASE(6)
    TB_LINCOMB_CASE(7) TB_LINCOMB_CASE(8) TB_LINCOMB_CASE(9) TB_LINCOMB_CASE(10) TB_LINCOMB_CASE(11) TB_LINCOMB_CASE(12)
    default:
      throw Error{TB_EINVAL, "linear combination of more than 12 stage vectors"};
  }
#undef TB_LINCOMB_CASE
}

void launch_advance_time(double* t, double dt, cudaStream_t st) { k_advance_time<<<1, 1, 0, st>>>(t, dt); }

void launch_mass_apply(const double2* X, double2* MX, const double* s3, int Nz, int Nk, int Nx, int project,
                       int nf, cudaStream_t st, int Nkm) {
  dim3 grid((Nk + 127) / 128, Nz);
  k_mass_apply<<<grid, 128, 0, st>>>(X, MX, s3, Nz, Nk, Nx, project, nf, Nkm > 0 ? Nkm : Nk);
}

void launch_lx_finalize(double2* LX, const double2* X, const double* s3, int Nz, int Nk, int Nx, double k0,
                        double s, double kappa, double nu, double beta, int nf, cudaStream_t st, int Nkm,
                        const double* kappa_m, const double* nu_m) {
  dim3 grid((Nk + 127) / 128, Nz);
  k_lx_finalize<<<grid, 128, 0, st>>>(LX, X, s3, Nz, Nk, Nx, k0, s, kappa, nu, beta, nf, Nkm > 0 ? Nkm : Nk, kappa_m,
                                      nu_m);
}

void launch_rk_final(const LinComb& lc, double2* X, double2* tau, const double* s3, int Nz, int Nk, int nf,
                     int ntau, cudaStream_t st) {
  dim3 grid((Nk + kFinalModes - 1) / kFinalModes, 2 * nf);
  const size_t smem = rk_final_smem_bytes(Nz);
#define TB_RKFINAL_CASE(N) \
  case N:                   \
    k_rk_final<N><<<grid, 256, smem, st>>>(lc, X, s3, Nz, Nk); \
    break;
  switch (lc.n) {
    TB_RKFINAL_CASE(1) TB_RKFINAL_CASE(2) TB_RKFINAL_CASE(3) TB_RKFINAL_CASE(4) TB_RKFINAL_CASE(5) TB_RKFINAL_CASE(6)
    TB_RKFINAL_CASE(7) TB_RKFINAL_CASE(8) TB_RKFINAL_CASE(9) TB_RKFINAL_CASE(10) TB_RKFINAL_CASE(11) TB_RKFINAL_CASE(12)
    default:
      throw Error{TB_EINVAL, "linear combination of more than 12 stage vectors"};
  }
#undef TB_RKFINAL_CASE
  cudaMemsetAsync(X + (size_t)3 * Nz * Nk, 0, sizeof(double2) * (size_t)Nz * Nk, st);
  cudaMemsetAsync(tau, 0, sizeof(double2) * (size_t)ntau * Nk, st);
}

size_t rk_final_smem_bytes(int Nz) {
  const size_t K = (size_t)(Nz + 1) / 2;
  return K * kFinalModes * sizeof(double2) + K * 3 * sizeof(double);
}

}  // namespace tb

#ifdef TB_SOLVE_CLOCKS
// Copies the first n phase clocks of the last tau solves to host memory.
extern "C" int tb_solve_clocks(long long* out, int n) {
  if (!out || n < 0 || n > tb::kSolveClockSlots) return 1;
  return cudaMemcpyFromSymbol(out, tb::g_solve_clocks, sizeof(long long) * (size_t)n) == cudaSuccess ? 0 : 1;
}
#endif
