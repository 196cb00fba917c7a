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
    const int g = m / kSolveModes, mm = m % kSolveModes;
    double* fr = C.FR + ((((size_t)g * a.npad + j) * 2 + c) * kFwdRec) * kSolveModes + mm;
    double* br = C.BR + ((((size_t)g * a.npad + j) * 2 + c) * kBwdRec) * kSolveModes + mm;
    // pivot offset, plus 16 when this band row's right-hand side is a u_x momentum
    // row (scaled by -i on load)
    fr[0] = (double)(p - j) + (C.row_eq[j] == EQ_MX ? 16.0 : 0.0);
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
      fr[(1 + t) * kSolveModes] = l;
    }
    for (int q = 0; q < nb; ++q) {
      const double cq = Cr[(size_t)q * nmax + j] * dinv;
      Cr[(size_t)q * nmax + j] = 0.0;
      for (int cc = j + 1; cc <= clast; ++cc) Cr[(size_t)q * nmax + cc] -= cq * W[(size_t)j * WW + (cc - j + KL)];
      for (int b = 0; b < nb; ++b) C1[q * NBMAX + b] -= cq * Bd[(size_t)j * NBMAX + b];
      fr[(1 + KL + q) * kSolveModes] = cq;
    }
    for (int q = nb; q < NBMAX; ++q) fr[(1 + KL + q) * kSolveModes] = 0.0;
    br[0] = dinv;
    for (int t = 1; t < W1; ++t) br[t * kSolveModes] = (j + t < n) ? W[(size_t)j * WW + KL + t] : 0.0;
    for (int b = 0; b < NBMAX; ++b) br[(W1 + b) * kSolveModes] = (b < nb) ? Bd[(size_t)j * NBMAX + b] : 0.0;
    {
      // store target of this band column: element offset (per mode) into X or the tau
      // array, encoded as offset*2 + (1 if the unknown is scaled by i), bit-cast
      const int unk = C.col_unk[j], kk = C.col_k[j];
      const long long off = unk < 4 ? ((long long)unk * a.Nz + kk) * Nk : (long long)4 * a.Nz * Nk + (long long)(unk - UK_TAU0) * Nk;
      br[(W1 + NBMAX) * kSolveModes] = __longlong_as_double(2 * off + (realified(unk) ? 1 : 0));
    }
  }
  // padding rows n..npad-1: identity rows with no right-hand side and no store
  for (int j = n; j < a.npad; ++j) {
    const int g = m / kSolveModes, mm = m % kSolveModes;
    double* fr = C.FR + ((((size_t)g * a.npad + j) * 2 + c) * kFwdRec) * kSolveModes + mm;
    double* br = C.BR + ((((size_t)g * a.npad + j) * 2 + c) * kBwdRec) * kSolveModes + mm;
    for (int t = 0; t < kFwdRec; ++t) fr[t * kSolveModes] = 0.0;
    br[0] = 1.0;
    for (int t = 1; t < kBwdRec - 1; ++t) br[t * kSolveModes] = 0.0;
    br[(kBwdRec - 1) * kSolveModes] = __longlong_as_double(-1LL);
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
  {
    const int g = m / kSolveModes, mm = m % kSolveModes;
    double* si = C.SI + (((size_t)g * 2 + c) * NBMAX * NBMAX) * kSolveModes + mm;
    for (int q = 0; q < NBMAX; ++q)
      for (int b = 0; b < NBMAX; ++b)
        si[(q * NBMAX + b) * kSolveModes] = (q < nb && b < nb) ? Aug[q][NBMAX + b] : 0.0;
  }
}

// ---------------------------------------------------------------------------
// Solve: one warp per group of kSolveModes Fourier modes.  Lane (c, mm) with
// c = lane / kSolveModes < 2 runs the forward and backward sweeps of parity
// class c for mode g*kSolveModes + mm (real and imaginary parts together as a
// double2).  The factor rows of the group are contiguous records that the
// whole warp streams into a shared-memory ring with cp.async, kRowsPerStage
// rows per stage and kStages stages deep; the forward sweep's intermediate y
// stays in shared memory for the backward sweep.
// ---------------------------------------------------------------------------
constexpr int kRowsPerStage = 12;  // a multiple of the forward and backward window lengths
constexpr int kStages = 6;

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

template <int KL, int KU>
__global__ void __launch_bounds__(32) k_tau_solve(TauArgs a) {
  static_assert(KL + 2 == kFwdWin && KL + KU == kBwdWin, "window sizes follow the band shape");
  constexpr int MP = kSolveModes;
  constexpr int W1 = KL + KU + 1;
  constexpr int FREC = 2 * kFwdRec * MP;  // doubles per forward row (both classes)
  constexpr int BREC = 2 * kBwdRec * MP;  // doubles per backward row
  constexpr int RREC = 2 * MP;            // double2 rhs entries per row (class, mode)
  constexpr int R = kRowsPerStage;
  constexpr int NL = 4 * MP;              // distinct lanes; lanes NL..31 mirror lanes 0..NL-1
  static_assert(NL <= 32 && 32 % NL == 0, "lane layout");
  extern __shared__ __align__(16) double smem[];
  const int np = a.npad;
  const int Nk = a.Nk;
  const int g = blockIdx.x;
  const int lane = threadIdx.x;
  const int ln = lane % NL;
  // ln = c*2*MP + part*MP + mm : class c, real (part 0) / imaginary (part 1) column, mode mm.
  // Mirror lanes repeat the same arithmetic (so the unrolled sweeps stay branch free) and
  // only the owner lanes store.
  const int c = ln / (2 * MP), part = (ln / MP) & 1, mm = ln % MP;
  const bool owner = lane < NL;
  const int m = g * MP + mm;
  const bool live = owner && m < Nk;
  constexpr int FSTAGE = R * (FREC + 2 * RREC);
  constexpr int BSTAGE = R * BREC;
  constexpr int STAGE = FSTAGE > BSTAGE ? FSTAGE : BSTAGE;
  double* ring = smem;
  double* ysave = smem + (size_t)kStages * STAGE;                  // [row][ln]
  int* rofs = reinterpret_cast<int*>(ysave + (size_t)np * NL);  // [row][class] rhs offset, -1: none
  for (int q = lane; q < 2 * np; q += 32) rofs[q] = (q < 2 * a.cls[0].n) ? a.rhs_off[q] : -1;
  __syncwarp();
  const double* FRg = a.cls[0].FR + (size_t)g * np * FREC;
  const double* BRg = a.cls[0].BR + (size_t)g * np * BREC;
  const int nstage = np / R;

  // ---- forward sweep: y = L^-1 P r (rows 0..np-1), boundary rows accumulate z ----
  auto issue_fwd = [&](int s) {
    if (s < nstage) {
      double* dst = ring + (size_t)(s % kStages) * STAGE;
      const int r0 = s * R;
      for (int q = lane; q < R * FREC / 2; q += 32) cp_async16(dst + 2 * q, FRg + (size_t)r0 * FREC + 2 * q, true);
      double2* rdst = reinterpret_cast<double2*>(dst + R * FREC);
      for (int q = lane; q < R * RREC; q += 32) {
        const int r = q / RREC, cc = (q / MP) % 2, md = q % MP;
        const int mq = g * MP + md;
        const int off = rofs[2 * (r0 + r) + cc];
        const bool ok = off >= 0 && mq < Nk;
        cp_async16(rdst + q, a.rhsP + (ok ? (size_t)off + mq : 0), ok);
      }
    }
    cp_async_commit();
  };
  for (int s = 0; s < kStages - 1; ++s) issue_fwd(s);
  // right-hand side of row j (j < np) for this lane: u_x momentum rows are
  // scaled by -i, i.e. (re, im) -> (im, -re)
  auto rhs_row = [&](int j) -> double {
    const int s = j / R, r = j % R;
    const double* base = ring + (size_t)(s % kStages) * STAGE;
    const double* rb = base + R * FREC + (size_t)(r * RREC + c * MP + mm) * 2;
    const bool rot = base[(size_t)r * FREC + c * kFwdRec * MP + mm] >= 8.0;
    const double v = rb[part ^ (rot ? 1 : 0)];
    return (rot && part) ? -v : v;
  };
  double y[kFwdWin];
  double z[NBMAX];
#pragma unroll
  for (int b = 0; b < NBMAX; ++b) z[b] = (part == 0 && m == 0 && b < a.cls[c].nb) ? a.beta * a.cls[c].bc_rhs[b] : 0.0;
  for (int j0 = 0; j0 < np; j0 += kFwdWin) {
    const int s = j0 / R;
    if (j0 % R == 0) {
      issue_fwd(s + kStages - 1);
      cp_async_wait<kStages - 2>();  // stages s and s+1 are resident
      __syncwarp();
      if (s == 0) {
#pragma unroll
        for (int t = 0; t < kFwdWin; ++t) y[t] = rhs_row(t);
      }
    }
    const double* st = ring + (size_t)(s % kStages) * STAGE + (size_t)(j0 - s * R) * FREC + c * kFwdRec * MP + mm;
    // rows j0 .. j0+kFwdWin-1; the right-hand sides entering the window are rows
    // j0+kFwdWin .. j0+2 kFwdWin-1, resident in stage s or s+1 (or past the end)
    double incoming[kFwdWin];
#pragma unroll
    for (int u = 0; u < kFwdWin; ++u) {
      const int jn = j0 + kFwdWin + u;
      incoming[u] = (jn < np) ? rhs_row(jn < np ? jn : 0) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kFwdWin; ++u) {
      const int j = j0 + u;
      const double* rec = st + (size_t)u * FREC;
      const double pf = rec[0];
      const int p = (int)(pf >= 8.0 ? pf - 16.0 : pf);
      double yj = y[u % kFwdWin];
#pragma unroll
      for (int t = 1; t <= KL; ++t) {
        const bool sw = (t == p);
        const double yt = y[(u + t) % kFwdWin];
        y[(u + t) % kFwdWin] = sw ? yj : yt;
        yj = sw ? yt : yj;
      }
      ysave[(size_t)j * NL + ln] = yj;
#pragma unroll
      for (int t = 1; t <= KL; ++t) y[(u + t) % kFwdWin] = fma(-rec[t * MP], yj, y[(u + t) % kFwdWin]);
#pragma unroll
      for (int b = 0; b < NBMAX; ++b) z[b] = fma(-rec[(1 + KL + b) * MP], yj, z[b]);
      y[u % kFwdWin] = incoming[u];
    }
    if ((j0 + kFwdWin) % R == 0) __syncwarp();  // the ring slot of stage s may be refilled next
  }
  cp_async_wait<0>();
  __syncwarp();

  // ---- border unknowns from the Schur complement ----
  double x1[NBMAX];
  {
    const double* si = a.cls[0].SI + ((size_t)g * 2 + c) * NBMAX * NBMAX * MP + mm;
#pragma unroll
    for (int q = 0; q < NBMAX; ++q) {
      double acc = 0.0;
#pragma unroll
      for (int b = 0; b < NBMAX; ++b) acc = fma(si[(q * NBMAX + b) * MP], z[b], acc);
      x1[q] = acc;
    }
  }

  // ---- backward sweep: x = U^-1 (y - B x1), rows np-1..0 ----
  auto issue_bwd = [&](int s) {
    if (s < nstage) {
      double* dst = ring + (size_t)(s % kStages) * STAGE;
      const int lo = np - (s + 1) * R;
      for (int q = lane; q < R * BREC / 2; q += 32) cp_async16(dst + 2 * q, BRg + (size_t)lo * BREC + 2 * q, true);
    }
    cp_async_commit();
  };
  for (int s = 0; s < kStages - 1; ++s) issue_bwd(s);
  double xw[kBwdWin];  // x_{j+t} lives in slot (j+t) % kBwdWin
#pragma unroll
  for (int t = 0; t < kBwdWin; ++t) xw[t] = 0.0;
  const size_t xplanes = (size_t)4 * a.Nz * Nk;
  double* Xd = reinterpret_cast<double*>(a.X);
  double* Td = reinterpret_cast<double*>(a.tau);
  static_assert(kBwdWin == R, "one backward block per stage");
  for (int s = 0; s < nstage; ++s) {
    issue_bwd(s + kStages - 1);
    cp_async_wait<kStages - 1>();
    __syncwarp();
    const int q0 = np - (s + 1) * R;  // rows q0+R-1 .. q0, q0 % kBwdWin == 0
    const double* st = ring + (size_t)(s % kStages) * STAGE + c * kBwdRec * MP + mm;
    double xs[kBwdWin];
#pragma unroll
    for (int u = 0; u < kBwdWin; ++u) {
      const int j = q0 + kBwdWin - 1 - u;  // j % kBwdWin == kBwdWin-1-u
      const double* rec = st + (size_t)(kBwdWin - 1 - u) * BREC;
      double acc0 = ysave[(size_t)j * NL + ln];
      double acc1 = 0.0, acc2 = 0.0;
#pragma unroll
      for (int b = 0; b < NBMAX; ++b) acc1 = fma(-rec[(W1 + b) * MP], x1[b], acc1);
#pragma unroll
      for (int t = kBwdWin; t >= 2; --t) {
        const int sl = (kBwdWin - 1 - u + t) % kBwdWin;
        if (t % 3 == 0)
          acc0 = fma(-rec[t * MP], xw[sl], acc0);
        else if (t % 3 == 1)
          acc1 = fma(-rec[t * MP], xw[sl], acc1);
        else
          acc2 = fma(-rec[t * MP], xw[sl], acc2);
      }
      const double sacc = fma(-rec[1 * MP], xw[(kBwdWin - u) % kBwdWin], acc0 + (acc1 + acc2));
      const double xj = sacc * rec[0];
      xw[(kBwdWin - 1 - u) % kBwdWin] = xj;
      xs[u] = xj;
    }
    // stores for the block, undoing the i-scaling of u_x and its taus
    // (ux = i vx: re = -vx_im, im = vx_re)
#pragma unroll
    for (int u = 0; u < kBwdWin; ++u) {
      const double* rec = st + (size_t)(kBwdWin - 1 - u) * BREC;
      const double partner = __shfl_xor_sync(0xffffffffu, xs[u], MP);
      const long long code = __double_as_longlong(rec[(kBwdRec - 1) * MP]);
      const size_t off = (size_t)(code >> 1);
      const double v = (code & 1) ? (part ? partner : -partner) : xs[u];
      double* dst = off < xplanes ? Xd + 2 * (off + m) : Td + 2 * (off - xplanes + m);
      if (live && code >= 0) dst[part] = v;
    }
    __syncwarp();
  }
  cp_async_wait<0>();
  // border unknowns
#pragma unroll
  for (int b = 0; b < NBMAX; ++b) {
    const double partner = __shfl_xor_sync(0xffffffffu, x1[b], MP);
    if (live && b < a.cls[c].nb) {
      const int unk = a.cls[c].left_unk[b];
      const int k = a.cls[c].left_k[b];
      const double v = realified(unk) ? (part ? partner : -partner) : x1[b];
      double* dst = unk < 4 ? Xd + 2 * (((size_t)unk * a.Nz + k) * Nk + m) : Td + 2 * ((size_t)(unk - UK_TAU0) * Nk + m);
      dst[part] = v;
    }
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

// Final RK update X_f = S^{-1} y, y = linear combination of the stage vectors
// in C^(2) rows.  S is upper triangular with offsets 0, +2, +4, so each
// (field, parity, mode) column is a short backward recurrence.  The CTA first
// forms y for all rows of its 32 modes in shared memory (256 threads, loads
// independent), then warp 0 runs the recurrences from shared memory.
__global__ void __launch_bounds__(256) k_rk_final(LinComb lc, double2* __restrict__ X, const double* __restrict__ s3,
                                                  int Nz, int Nk) {
  extern __shared__ double2 ys[];  // [rows of this parity][32]
  const int f = blockIdx.y >> 1, par = blockIdx.y & 1;
  const int m0 = blockIdx.x * 32;
  const int mm = threadIdx.x % 32, ks = threadIdx.x / 32;
  const int m = m0 + mm;
  const size_t plane = (size_t)Nz * Nk;
  const int K = (Nz - par + 1) / 2;  // rows k = par + 2 ri
  for (int ri = ks; ri < K; ri += 8) {
    const int k = par + 2 * ri;
    double2 y = make_double2(0.0, 0.0);
    if (m < Nk) {
      const size_t i = (size_t)(1 + f) * plane + (size_t)k * Nk + m;
      for (int t = 0; t < lc.n; ++t) y = cfma(lc.w[t], lc.in[t][i], y);
    }
    ys[ri * 32 + mm] = y;
  }
  __syncthreads();
  if (ks == 0) {
    double2 x2 = make_double2(0.0, 0.0), x4 = make_double2(0.0, 0.0);
    for (int ri = K - 1; ri >= 0; --ri) {
      const int k = par + 2 * ri;
      double2 y = ys[ri * 32 + mm];
      y = cfma(-s3[3 * k + 1], x2, y);
      y = cfma(-s3[3 * k + 2], x4, y);
      const double inv = 1.0 / s3[3 * k];
      const double2 x = make_double2(y.x * inv, y.y * inv);
      ys[ri * 32 + mm] = x;
      x4 = x2;
      x2 = x;
    }
  }
  __syncthreads();
  if (m < Nk)
    for (int ri = ks; ri < K; ri += 8) X[(size_t)f * plane + (size_t)(par + 2 * ri) * Nk + m] = ys[ri * 32 + mm];
}

template <int KL, int KU>
void factor_impl(const TauArgs& a, cudaStream_t st) {
  int nmax = a.cls[0].n > a.cls[1].n ? a.cls[0].n : a.cls[1].n;
  dim3 grid((a.Nk + 63) / 64, 2);
  k_tau_factor<KL, KU><<<grid, 64, 0, st>>>(a, nmax);
}

size_t solve_smem_bytes(int npad) {
  constexpr int MP = kSolveModes;
  const size_t FREC = 2 * kFwdRec * MP, BREC = 2 * kBwdRec * MP, RREC = 2 * MP;
  const size_t FSTAGE = kRowsPerStage * (FREC + 2 * RREC), BSTAGE = kRowsPerStage * BREC;
  const size_t STAGE = FSTAGE > BSTAGE ? FSTAGE : BSTAGE;
  return (kStages * STAGE) * sizeof(double) + (size_t)npad * 4 * MP * sizeof(double) + (size_t)npad * 2 * sizeof(int);
}

template <int KL, int KU>
void solve_impl(const TauArgs& a, cudaStream_t st) {
  const int groups = (a.Nk + kSolveModes - 1) / kSolveModes;
  const size_t smem = solve_smem_bytes(a.npad);
  k_tau_solve<KL, KU><<<groups, 32, smem, st>>>(a);
}

}  // namespace

size_t tau_factor_scratch_doubles(int nmax, int Nk);

cudaError_t set_tau_smem_limits(int bytes) {
  cudaError_t e = cudaFuncSetAttribute(k_tau_solve<kTauKL, kTauKU>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_rk_final, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

size_t tau_solve_smem_bytes(int n) { return solve_smem_bytes(n); }

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
  dim3 grid((Nk + 31) / 32, 6);
  const size_t smem = (size_t)((Nz + 1) / 2) * 32 * sizeof(double2);
  k_rk_final<<<grid, 256, smem, st>>>(lc, X, s3, Nz, Nk);
  cudaMemsetAsync(X + (size_t)3 * Nz * Nk, 0, sizeof(double2) * (size_t)Nz * Nk, st);
  cudaMemsetAsync(tau, 0, sizeof(double2) * 7 * (size_t)Nk, st);
}

}  // namespace tb
