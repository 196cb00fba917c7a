// Transform kernels: the ChebyshevT direction as a batched FP64 GEMM against
// precomputed N x N matrices, and the RealFourier direction as a Stockham FFT
// in shared memory fused with the 3/2-dealiased advection products.
//
// Reference semantics reproduced here:
//   rfft unnormalised / irfft 1/N ignoring Im of DC and Nyquist
//     (src/core/transforms/transform_fourier.jl:7-31,287-313)
//   DCT-I REDFT00 with 1/(N-1), halved endpoints, odd flip
//     (src/core/transforms/transform_chebyshev.jl:135-244)
//   3/2 padding M = ceil(3N/2) even, Nyquist split X/2 at +-N/2 and folded back,
//   output scaled so the product lands on the N grid
//     (src/core/nonlinear/nonlinear_padding.jl:103-108,182-226,294-346,359-443)
#include <cuda_runtime.h>

#include "tb_fft.cuh"
#include "tb_kernels.cuh"

namespace tb {

// ---------------------------------------------------------------------------
// FP64 batched GEMM for the Chebyshev direction on the FP64 tensor cores
// (mma.sync m8n8k4 .f64).  CTA tile 64 x 64 (4 warps, 32 x 32 each), 16-deep
// K slices double-buffered in shared memory with cp.async.  Each batch entry
// carries its own A (rows padded to a multiple of 16 doubles) and a B-row map:
//   GEMM_PLAIN   : B row k = in[k]
//   GEMM_PARITY  : B row k = in[2k + par]              (even / odd coefficients)
//   GEMM_MIRROR  : B row j = in[j] + sgn in[N-1-j]     (grid rows folded about
//                  the mid-plane; sgn = +1 for par 0, -1 for par 1; the middle
//                  row of odd N counts once / not at all)
// and an output-row map (row r -> out row r, or 2r + par for GEMM_MIRROR).
// ---------------------------------------------------------------------------
namespace {
constexpr int GBM = 64, GBN = 64, GBK = 16, GTH = 128;
constexpr int ASTR = GBK + 4;  // padded shared row strides (doubles)
constexpr int BSTR = GBN + 8;
constexpr size_t kGemmSmem = (2 * GBM * ASTR + 4 * GBK * BSTR) * sizeof(double);

__device__ __forceinline__ void g_cp16(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void g_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void g_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void g_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// SPLITK = false: CTA tile 64 x 64, warp (wm, wn) owns rows wm*32.., cols wn*32..
// SPLITK = true:  CTA tile 32 x 64 (twice the CTAs for short M), warp (wk, wn)
//                 owns cols wn*32.. and the k-steps ks = 2 wk, 2 wk + 1 of every
//                 16-deep slice; the two k halves are summed through shared memory.
template <bool SPLITK>
__global__ void __launch_bounds__(GTH) k_gemm_f64(GemmBatch bt, int ncol, int ldb, int ldc, int Nrows) {
  constexpr int TM = SPLITK ? GBM / 2 : GBM;  // CTA tile rows
  extern __shared__ __align__(16) double gsm[];
  double (*As)[GBM * ASTR] = reinterpret_cast<double (*)[GBM * ASTR]>(gsm);
  double (*Bs)[GBK * BSTR] = reinterpret_cast<double (*)[GBK * BSTR]>(gsm + 2 * GBM * ASTR);
  double (*Bm)[GBK * BSTR] = reinterpret_cast<double (*)[GBK * BSTR]>(gsm + 2 * GBM * ASTR + 2 * GBK * BSTR);  // mirror partners
  const GemmItem& it = bt.item[blockIdx.z];
  const double* __restrict__ A = it.A;
  const double* __restrict__ B = it.B;
  const int Mo = it.M, K = it.K, Kp = it.Kpad, mode = it.mode, par = it.par;
  const int row0 = blockIdx.y * TM, col0 = blockIdx.x * GBN;
  if (row0 >= Mo) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = SPLITK ? 0 : (warp >> 1), wk = SPLITK ? (warp >> 1) : 0, wn = warp & 1;
  const int gid = lane >> 2, tig = lane & 3;
  const bool mirror = mode == GEMM_MIRROR;
  const int ntiles = (K + GBK - 1) / GBK;

  auto load_tile = [&](int t, int buf) {
    const int k0 = t * GBK;
    // A: TM rows x 16 doubles = TM*8 chunks of 16 B
#pragma unroll
    for (int q = 0; q < TM * 8 / GTH; ++q) {
      const int ch = tid + q * GTH;
      const int r = ch >> 3, kc = (ch & 7) * 2;
      const int gr = row0 + r;
      const bool ok = gr < Mo;
      g_cp16(&As[buf][r * ASTR + kc], A + (size_t)(ok ? gr : 0) * Kp + k0 + kc, ok);
    }
    // B: 16 rows x 64 doubles = 512 chunks, 4 per thread (8 with the mirror partner)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int ch = tid + q * GTH;
      const int kk = ch >> 5, cc = (ch & 31) * 2;
      const int gk = k0 + kk, gc = col0 + cc;
      const bool ok = gk < K && gc < ncol;
      int srow = gk;
      if (mode == GEMM_PARITY) srow = 2 * gk + par;
      g_cp16(&Bs[buf][kk * BSTR + cc], B + (size_t)(ok ? srow : 0) * ldb + (ok ? gc : 0), ok);
      if (mirror) {
        const int jm = Nrows - 1 - gk;
        const bool okm = ok && jm != gk;  // the middle row of odd N has no partner
        g_cp16(&Bm[buf][kk * BSTR + cc], B + (size_t)(okm ? jm : 0) * ldb + (okm ? gc : 0), okm);
      }
    }
    g_commit();
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const double sgn = par ? -1.0 : 1.0;
  // the middle row of odd N contributes once to the even sum and not at all to the odd one
  const int midk = (mirror && (Nrows & 1)) ? (Nrows - 1) / 2 : -1;

  load_tile(0, 0);
  for (int t = 0; t < ntiles; ++t) {
    const int buf = t & 1;
    if (t + 1 < ntiles)
      load_tile(t + 1, buf ^ 1);
    else
      g_commit();
    g_wait1();
    __syncthreads();
    if (mirror) {
      // fold the mirror partners into the B slice once, in place: row j of
      // B' = in[j] + sgn in[N-1-j] (the middle row of odd N once / not at all)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int ch = tid + q * GTH;
        const int kk = ch >> 5, cc = (ch & 31) * 2;
        const int gk = t * GBK + kk;
        double2* bp = reinterpret_cast<double2*>(&Bs[buf][kk * BSTR + cc]);
        const double2 v = *bp, w = *reinterpret_cast<const double2*>(&Bm[buf][kk * BSTR + cc]);
        *bp = (gk == midk) ? (par ? make_double2(0.0, 0.0) : v)
                           : make_double2(fma(sgn, w.x, v.x), fma(sgn, w.y, v.y));
      }
      __syncthreads();
    }
    const double* as = As[buf];
    const double* bs = Bs[buf];
#pragma unroll
    for (int kq = 0; kq < (SPLITK ? GBK / 8 : GBK / 4); ++kq) {
      const int ks = SPLITK ? 2 * wk + kq : kq;
      const int kk = ks * 4 + tig;
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = as[(wm * 32 + i * 8 + gid) * ASTR + kk];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = bs[kk * BSTR + wn * 32 + j * 8 + gid];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    __syncthreads();
  }
  g_wait0();
  if constexpr (SPLITK) {
    // the upper k half hands its partial tile to the lower half (buffers are free)
    double* red = gsm + (size_t)wn * 32 * 32;
    if (wk == 1) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          red[((i * 4 + j) * 2 + 0) * 32 + lane] = acc[i][j][0];
          red[((i * 4 + j) * 2 + 1) * 32 + lane] = acc[i][j][1];
        }
    }
    __syncthreads();
    if (wk == 1) return;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        acc[i][j][0] += red[((i * 4 + j) * 2 + 0) * 32 + lane];
        acc[i][j][1] += red[((i * 4 + j) * 2 + 1) * 32 + lane];
      }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gr = row0 + wm * 32 + i * 8 + gid;
    if (gr >= Mo) continue;
    const int orow = mirror ? 2 * gr + par : gr;
    double* C = it.C + (size_t)orow * ldc;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gc = col0 + wn * 32 + j * 8 + tig * 2;
      if (gc + 1 < ncol) {
        *reinterpret_cast<double2*>(C + gc) = make_double2(acc[i][j][0], acc[i][j][1]);
      } else if (gc < ncol) {
        C[gc] = acc[i][j][0];
      }
    }
  }
}
}  // namespace

void launch_gemm_f64(const GemmBatch& bt, int nbatch, int ncol, int ldb, int ldc, int Nrows, cudaStream_t st) {
  int mmax = 0;
  for (int b = 0; b < nbatch; ++b) mmax = bt.item[b].M > mmax ? bt.item[b].M : mmax;
  const int ncx = (ncol + GBN - 1) / GBN;
  const long long ctas = (long long)ncx * ((mmax + GBM - 1) / GBM) * nbatch;
  if (ctas < 2LL * 148) {
    // too few 64-row tiles to fill the SMs: halve the tile rows and split K inside the CTA
    dim3 grid(ncx, (mmax + GBM / 2 - 1) / (GBM / 2), nbatch);
    k_gemm_f64<true><<<grid, GTH, kGemmSmem, st>>>(bt, ncol, ldb, ldc, Nrows);
  } else {
    dim3 grid(ncx, (mmax + GBM - 1) / GBM, nbatch);
    k_gemm_f64<false><<<grid, GTH, kGemmSmem, st>>>(bt, ncol, ldb, ldc, Nrows);
  }
}

// ---------------------------------------------------------------------------
// Stockham FFT in shared memory, executed by the whole CTA.
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// Logical -> physical index of an FFT buffer.  With SW the low three bits are
// XORed with the next three, so the stride-R stores of a Stockham pass
// (R <= 8 consecutive elements per thread) and the unit-stride loads both hit
// eight distinct 16-byte bank groups per quarter warp.  Buffers are sized to a
// multiple of 8 elements so the permutation stays inside them.
template <bool SW>
__device__ __forceinline__ int fidx(int i) {
  return SW ? (i ^ ((i >> 3) & 7)) : i;
}

// exp(sign 2 pi i t / n) for 0 <= t < n from a table of exp(-2 pi i t / n),
// t < n/2 (the upper half is the negated lower half).
__device__ __forceinline__ double2 twid(const double2* tw, int t, int h, int sign) {
  const bool hi = t >= h;
  double2 w = tw[hi ? t - h : t];
  if (hi) w = make_double2(-w.x, -w.y);
  if (sign > 0) w.y = -w.y;
  return w;
}

// multiply by exp(sign i pi/2): -i for the forward transform, +i for the inverse
__device__ __forceinline__ double2 rot4(double2 d, int sign) {
  return (sign < 0) ? make_double2(d.y, -d.x) : make_double2(-d.y, d.x);
}

__device__ __forceinline__ void dft4(double2& x0, double2& x1, double2& x2, double2& x3, int sign) {
  const double2 t0 = cadd(x0, x2), t1 = csub(x0, x2), t2 = cadd(x1, x3), t3 = rot4(csub(x1, x3), sign);
  x0 = cadd(t0, t2);
  x1 = cadd(t1, t3);
  x2 = csub(t0, t2);
  x3 = csub(t1, t3);
}

// In-register DFT of length R (unnormalised, exponent sign), natural order.
template <int R>
__device__ __forceinline__ void dft_small(double2 (&v)[R], int sign) {
  if constexpr (R == 2) {
    const double2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (R == 3) {
    const double h = 0.86602540378443864676372317075294;  // sqrt(3)/2
    const double2 sm = cadd(v[1], v[2]), df = csub(v[1], v[2]);
    const double2 base = make_double2(v[0].x - 0.5 * sm.x, v[0].y - 0.5 * sm.y);
    const double2 rot = make_double2(-sign * h * df.y, sign * h * df.x);  // i sign h df
    v[0] = cadd(v[0], sm);
    v[1] = cadd(base, rot);
    v[2] = csub(base, rot);
  } else if constexpr (R == 4) {
    dft4(v[0], v[1], v[2], v[3], sign);
  } else {  // R == 8, one radix-2 decimation-in-frequency step then two DFT-4
    const double r = 0.70710678118654752440084436210485;  // 1/sqrt(2)
    const double s = (double)sign;
    double2 a[4], b[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      a[n] = cadd(v[n], v[n + 4]);
      b[n] = csub(v[n], v[n + 4]);
    }
    // b_n *= exp(sign 2 pi i n / 8)
    b[1] = make_double2(r * (b[1].x - s * b[1].y), r * (b[1].y + s * b[1].x));
    b[2] = rot4(b[2], sign);
    b[3] = make_double2(r * (-b[3].x - s * b[3].y), r * (-b[3].y + s * b[3].x));
    dft4(a[0], a[1], a[2], a[3], sign);
    dft4(b[0], b[1], b[2], b[3], sign);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[2 * k] = a[k];
      v[2 * k + 1] = b[k];
    }
  }
}

// One Stockham pass of radix R (Govindaraju et al. formulation: read
// in[idx + r n/R], twiddle by w^(j r n/(Ns R)), R-point DFT, write
// out[(idx/Ns) Ns R + idx%Ns + r Ns]).  Output ends in natural order.
template <int R, bool SW>
__device__ __forceinline__ void fft_pass(const double2* __restrict__ in, double2* __restrict__ out, int n, int Ns,
                                         const double2* __restrict__ tw, int sign) {
  const int nR = n / R;
  const int tstride = n / (Ns * R);
  const int h = n >> 1;
  for (int idx = threadIdx.x; idx < nR; idx += blockDim.x) {
    const int j = idx % Ns, k = idx / Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = in[fidx<SW>(idx + r * nR)];
    if (Ns > 1) {
      const int e = j * tstride;  // r e < n for every r < R
      if constexpr (R == 8) {
        const double2 w1 = twid(tw, e, h, sign), w2 = twid(tw, 2 * e, h, sign), w4 = twid(tw, 4 * e, h, sign);
        const double2 w3 = cmul(w1, w2);
        v[1] = cmul(v[1], w1);
        v[2] = cmul(v[2], w2);
        v[3] = cmul(v[3], w3);
        v[4] = cmul(v[4], w4);
        v[5] = cmul(v[5], cmul(w1, w4));
        v[6] = cmul(v[6], cmul(w2, w4));
        v[7] = cmul(v[7], cmul(w3, w4));
      } else {
#pragma unroll
        for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twid(tw, r * e, h, sign));
      }
    }
    dft_small<R>(v, sign);
    const int ob = k * Ns * R + j;
#pragma unroll
    for (int r = 0; r < R; ++r) out[fidx<SW>(ob + r * Ns)] = v[r];
  }
}

// Returns the buffer holding the result (a or b).  sign = -1 forward, +1 inverse
// (both unnormalised).  tw[t] = exp(-2 pi i t / n) for t < n/2 (a longer table
// works too).
template <bool SW = false>
__device__ double2* fft_cta(double2* a, double2* b, const FftPlan& fp, const double2* __restrict__ tw, int sign) {
  const int n = fp.n;
  int Ns = 1;
  double2* in = a;
  double2* out = b;
  for (int s = 0; s < fp.nstages; ++s) {
    const int R = fp.radix[s];
    if (R == 8)
      fft_pass<8, SW>(in, out, n, Ns, tw, sign);
    else if (R == 4)
      fft_pass<4, SW>(in, out, n, Ns, tw, sign);
    else if (R == 2)
      fft_pass<2, SW>(in, out, n, Ns, tw, sign);
    else
      fft_pass<3, SW>(in, out, n, Ns, tw, sign);
    __syncthreads();
    double2* t = in;
    in = out;
    out = t;
    Ns *= R;
  }
  return in;
}

// Stockham pass as fft_pass, with the twiddles of this pass from its own table
// pt[j] = exp(-2 pi i j tstride / n), j < Ns (consecutive threads read
// consecutive entries: no bank conflicts); w^r for r > 1 by products of w.
template <int R, bool SW>
__device__ __forceinline__ void fft_pass_pt(const double2* __restrict__ in, double2* __restrict__ out, int n, int Ns,
                                            const double2* __restrict__ pt, int sign) {
  const int nR = n / R;
  for (int idx = threadIdx.x; idx < nR; idx += blockDim.x) {
    const int j = idx % Ns, k = idx / Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = in[fidx<SW>(idx + r * nR)];
    if (Ns > 1) {
      double2 w1 = pt[j];
      if (sign > 0) w1.y = -w1.y;
      if constexpr (R == 8) {
        const double2 w2 = cmul(w1, w1), w4 = cmul(w2, w2), w3 = cmul(w1, w2);
        v[1] = cmul(v[1], w1);
        v[2] = cmul(v[2], w2);
        v[3] = cmul(v[3], w3);
        v[4] = cmul(v[4], w4);
        v[5] = cmul(v[5], cmul(w1, w4));
        v[6] = cmul(v[6], cmul(w2, w4));
        v[7] = cmul(v[7], cmul(w3, w4));
      } else if constexpr (R == 4) {
        const double2 w2 = cmul(w1, w1);
        v[1] = cmul(v[1], w1);
        v[2] = cmul(v[2], w2);
        v[3] = cmul(v[3], cmul(w1, w2));
      } else if constexpr (R == 3) {
        v[1] = cmul(v[1], w1);
        v[2] = cmul(v[2], cmul(w1, w1));
      } else {
        v[1] = cmul(v[1], w1);
      }
    }
    dft_small<R>(v, sign);
    const int ob = k * Ns * R + j;
#pragma unroll
    for (int r = 0; r < R; ++r) out[fidx<SW>(ob + r * Ns)] = v[r];
  }
}

// fft_cta with per-pass twiddle tables: pass s reads pt + (sum of Ns of the
// passes before it), the layout written by pass_twiddles() on the host.
template <bool SW>
__device__ double2* fft_cta_pt(double2* a, double2* b, const FftPlan& fp, const double2* __restrict__ pt, int sign) {
  const int n = fp.n;
  int Ns = 1;
  double2* in = a;
  double2* out = b;
  for (int s = 0; s < fp.nstages; ++s) {
    const int R = fp.radix[s];
    if (R == 8)
      fft_pass_pt<8, SW>(in, out, n, Ns, pt, sign);
    else if (R == 4)
      fft_pass_pt<4, SW>(in, out, n, Ns, pt, sign);
    else if (R == 2)
      fft_pass_pt<2, SW>(in, out, n, Ns, pt, sign);
    else
      fft_pass_pt<3, SW>(in, out, n, Ns, pt, sign);
    __syncthreads();
    double2* t = in;
    in = out;
    out = t;
    pt += Ns;
    Ns *= R;
  }
  return in;
}

// Half-spectrum entry H_k of a row whose unnormalised rfft bins are g (length
// Nk = N/2+1), as an operand of the padded product: DC and Nyquist are real
// (irfft ignores their imaginary parts) and the Nyquist bin is split in half.
__device__ __forceinline__ double2 half_bin(const double2* __restrict__ g, int k, int N) {
  const int h = N / 2;
  if (k == 0) return make_double2(g[0].x, 0.0);
  if (k < h) return g[k];
  if (k == h) return make_double2(0.5 * g[h].x, 0.0);
  return make_double2(0.0, 0.0);
}

// Full length-M spectrum of two real signals a + i b from their half spectra.
__device__ __forceinline__ double2 pack2(double2 A, double2 B) { return make_double2(A.x - B.y, A.y + B.x); }
__device__ __forceinline__ double2 pack2_mirror(double2 A, double2 B) {
  // conj(A) + i conj(B)
  return make_double2(A.x + B.y, -A.y + B.x);
}

// Row-wise advection products on the 3/2-padded x grid.  One CTA per grid row
// z (two CTAs per SM): four swizzled FFT buffers of M complex entries and the
// half twiddle table live in shared memory; the six mixed-space input rows are
// read straight from the even/odd Chebyshev half planes (L2-resident after
// the z GEMM), each entry once per spectrum it feeds.
//   1. U = ifft(ux + i uz)                      (velocity on the padded grid)
//   2. for f in b, ux, uz: G = ifft(d_x f + i d_z f); prod_f = -(u G.x + w G.y)
//   3. fft(prod_b + i prod_ux), fft(prod_uz), unpacked and truncated to Nk bins
__global__ void __launch_bounds__(256, 2) k_xprod(XProdArgs a) {
  extern __shared__ double2 sm[];
  const int M = a.M, N = a.Nx, Nk = a.Nk;
  const int Ms = (M + 7) & ~7;
  double2* S0 = sm;
  double2* S1 = sm + Ms;
  double2* S2 = sm + 2 * Ms;
  double2* S3 = sm + 3 * Ms;
  double2* tw = sm + 4 * Ms;  // per-pass twiddle tables of the length-M plan
  const int hN = N / 2;
  for (int t = threadIdx.x; t < a.nptw; t += blockDim.x) tw[t] = a.ptw[t];
  // Grid row z from the even/odd Chebyshev half planes: rows z < H are E + O,
  // mirrored rows N-1-z are E - O for values and -E + O for z-derivatives.
  const int z = blockIdx.x;
  const int zm = a.Nz - 1 - z;
  const bool lower = z <= zm;
  // instance blockIdx.y of a batched plan: its Nk modes start at column y * Nk
  const size_t ld = a.ld > 0 ? (size_t)a.ld : (size_t)Nk, col0 = (size_t)blockIdx.y * Nk;
  const size_t rr = (size_t)(lower ? z : zm) * ld + col0;
  auto value = [&](int f, int q) -> double2 {
    const double2 e = a.ev[f][rr + q], o = a.ov[f][rr + q];
    return lower ? make_double2(e.x + o.x, e.y + o.y) : make_double2(e.x - o.x, e.y - o.y);
  };
  auto deriv = [&](int f, int q) -> double2 {
    const double2 e = a.ed[f][rr + q], o = a.od[f][rr + q];
    return lower ? make_double2(e.x + o.x, e.y + o.y) : make_double2(o.x - e.x, o.y - e.y);
  };
  // padded operand bin q of a half spectrum value v (DC / Nyquist real, Nyquist halved)
  auto hbin = [&](double2 v, int q) -> double2 {
    if (q == 0) return make_double2(v.x, 0.0);
    if (q == hN) return make_double2(0.5 * v.x, 0.0);
    return v;
  };
  // spectrum of A + i B on the padded grid from half spectra A_q, B_q (q <= N/2)
  auto put2 = [&](double2* dst, int q, double2 A, double2 B) {
    dst[fidx<true>(q)] = pack2(A, B);
    if (q > 0) dst[fidx<true>(M - q)] = pack2_mirror(A, B);
  };
  auto zero_gap = [&](double2* dst) {  // bins N/2 < k < M - N/2 are zero
    for (int k = hN + 1 + threadIdx.x; k < M - hN; k += blockDim.x) dst[fidx<true>(k)] = make_double2(0.0, 0.0);
  };
  // Inputs are read in batches of QB bins per thread with every load issued
  // before the first is used, so a thread waits for memory once per batch
  // rather than once per bin.
  constexpr int QB = 3;
  // 1. velocity spectrum
  for (int q0 = threadIdx.x; q0 <= hN; q0 += QB * blockDim.x) {
    double2 vx[QB], vz[QB];
#pragma unroll
    for (int i = 0; i < QB; ++i) {
      const int q = q0 + i * blockDim.x;
      if (q <= hN) {
        vx[i] = value(1, q);
        vz[i] = value(2, q);
      }
    }
#pragma unroll
    for (int i = 0; i < QB; ++i) {
      const int q = q0 + i * blockDim.x;
      if (q <= hN) put2(S0, q, hbin(vx[i], q), hbin(vz[i], q));
    }
  }
  zero_gap(S0);
  __syncthreads();
  double2* U = fft_cta_pt<true>(S0, S1, a.fp, tw, +1);
  double2* P = (U == S0) ? S1 : S0;  // prod_b + i prod_ux
  double2* Q = nullptr;              // prod_uz (real parts)
  // 2. gradients of each field and the advection products
  for (int f = 0; f < 3; ++f) {
    for (int q0 = threadIdx.x; q0 <= hN; q0 += QB * blockDim.x) {
      double2 gv[QB], dv[QB];
#pragma unroll
      for (int i = 0; i < QB; ++i) {
        const int q = q0 + i * blockDim.x;
        if (q <= hN) {
          gv[i] = value(f, q);
          dv[i] = deriv(f, q);
        }
      }
#pragma unroll
      for (int i = 0; i < QB; ++i) {
        const int q = q0 + i * blockDim.x;
        if (q <= hN) {
          double2 Ax = make_double2(0.0, 0.0);
          if (q > 0 && q < hN) {
            const double kk = a.k0 * q;
            Ax = make_double2(-kk * gv[i].y, kk * gv[i].x);  // i k g
          }
          put2(S2, q, Ax, hbin(dv[i], q));
        }
      }
    }
    zero_gap(S2);
    __syncthreads();
    double2* G = fft_cta_pt<true>(S2, S3, a.fp, tw, +1);
    double2* Gf = (G == S2) ? S3 : S2;  // the pass buffer left free
    for (int p = threadIdx.x; p < M; p += blockDim.x) {
      const int ps = fidx<true>(p);
      const double2 u = U[ps], g = G[ps];
      const double pr = -(u.x * g.x + u.y * g.y);
      if (f == 0)
        P[ps].x = pr;
      else if (f == 1)
        P[ps].y = pr;
      else
        Gf[ps] = make_double2(pr, 0.0);
    }
    if (f == 2) {
      Q = Gf;
      // the gradient buffer G is free from here on
      __syncthreads();
      // 3a. forward transform of prod_b + i prod_ux into G's buffer pair
      double2* C1 = fft_cta_pt<true>(P, G, a.fp, tw, -1);
      // 3b. forward transform of prod_uz, ping-ponging with U's buffer (free now);
      // it touches neither C1 nor P's partner, so both proceed before one barrier
      double2* C2 = fft_cta_pt<true>(Q, U, a.fp, tw, -1);
      const double sc = 1.0 / ((double)M * (double)N);
      const size_t ro = (size_t)z * ld + col0;
      for (int k = threadIdx.x; k < Nk; k += blockDim.x) {
        const double2 c = C1[fidx<true>(k)];
        const double2 cm = C1[fidx<true>((M - k) % M)];
        // b: (c + conj(cm))/2 ; ux: (c - conj(cm))/(2i)
        const double2 sb = make_double2(0.5 * (c.x + cm.x), 0.5 * (c.y - cm.y));
        const double2 su = make_double2(0.5 * (c.y + cm.y), -0.5 * (c.x - cm.x));
        const double2 c2 = C2[fidx<true>(k)];
        double2 ob, ou, oz;
        if (k == 0) {
          ob = make_double2(sb.x * sc, 0.0);
          ou = make_double2(su.x * sc, 0.0);
          oz = make_double2(c2.x * sc, 0.0);
        } else if (k == hN) {
          ob = make_double2(2.0 * sb.x * sc, 0.0);
          ou = make_double2(2.0 * su.x * sc, 0.0);
          oz = make_double2(2.0 * c2.x * sc, 0.0);
        } else {
          ob = cscale(sb, sc);
          ou = cscale(su, sc);
          oz = cscale(c2, sc);
        }
        a.out[0][ro + k] = ob;
        a.out[1][ro + k] = ou;
        a.out[2][ro + k] = oz;
      }
    } else {
      __syncthreads();
    }
  }
}

// One Stockham pass over NA arrays of length n stored Ms apart: the
// (array, butterfly) pairs are spread over the CTA, so the arrays share the
// pass's barrier.  Same arithmetic as fft_pass_pt for each array.
template <int R>
__device__ __forceinline__ void fft_pass_multi(const double2* __restrict__ in, double2* __restrict__ out, int NA,
                                               int Ms, int n, int Ns, const double2* __restrict__ pt, int sign) {
  const int nR = n / R, total = NA * nR;
  for (int item = threadIdx.x; item < total; item += blockDim.x) {
    const int arr = item / nR, idx = item - arr * nR;
    const double2* ia = in + (size_t)arr * Ms;
    double2* oa = out + (size_t)arr * Ms;
    const int j = idx % Ns, k = idx / Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = ia[fidx<true>(idx + r * nR)];
    if (Ns > 1) {
      double2 w1 = pt[j];
      if (sign > 0) w1.y = -w1.y;
      if constexpr (R == 8) {
        const double2 w2 = cmul(w1, w1), w4 = cmul(w2, w2), w3 = cmul(w1, w2);
        v[1] = cmul(v[1], w1);
        v[2] = cmul(v[2], w2);
        v[3] = cmul(v[3], w3);
        v[4] = cmul(v[4], w4);
        v[5] = cmul(v[5], cmul(w1, w4));
        v[6] = cmul(v[6], cmul(w2, w4));
        v[7] = cmul(v[7], cmul(w3, w4));
      } else if constexpr (R == 4) {
        const double2 w2 = cmul(w1, w1);
        v[1] = cmul(v[1], w1);
        v[2] = cmul(v[2], w2);
        v[3] = cmul(v[3], cmul(w1, w2));
      } else if constexpr (R == 3) {
        v[1] = cmul(v[1], w1);
        v[2] = cmul(v[2], cmul(w1, w1));
      } else {
        v[1] = cmul(v[1], w1);
      }
    }
    dft_small<R>(v, sign);
    const int ob = k * Ns * R + j;
#pragma unroll
    for (int r = 0; r < R; ++r) oa[fidx<true>(ob + r * Ns)] = v[r];
  }
}

// NA length-fp.n transforms at a[arr * Ms], ping-ponging with b[arr * Ms];
// returns the block (a or b) holding the results.
__device__ double2* fft_cta_multi(double2* a, double2* b, int NA, int Ms, const FftPlan& fp,
                                  const double2* __restrict__ pt, int sign) {
  const int n = fp.n;
  int Ns = 1;
  double2* in = a;
  double2* out = b;
  for (int s = 0; s < fp.nstages; ++s) {
    const int R = fp.radix[s];
    if (R == 8)
      fft_pass_multi<8>(in, out, NA, Ms, n, Ns, pt, sign);
    else if (R == 4)
      fft_pass_multi<4>(in, out, NA, Ms, n, Ns, pt, sign);
    else if (R == 2)
      fft_pass_multi<2>(in, out, NA, Ms, n, Ns, pt, sign);
    else
      fft_pass_multi<3>(in, out, NA, Ms, n, Ns, pt, sign);
    __syncthreads();
    double2* t = in;
    in = out;
    out = t;
    pt += Ns;
    Ns *= R;
  }
  return in;
}

// The same row products as k_xprod with the transforms batched: the velocity
// and the three gradient spectra are built in one sweep over the half-plane
// inputs (each value and z-derivative bin read once), go through one set of
// inverse passes together (4 arrays, one barrier per pass), the products
// are formed for all three fields at once, and the two forward transforms
// share their passes too: about 10 barriers per row instead of 27.  Shared
// memory: two blocks of 4 arrays (ping-pong) and the per-pass twiddles.
template <int NT>
__global__ void __launch_bounds__(NT, NT == 256 ? 2 : 1) k_xprod_b(XProdArgs a) {
  extern __shared__ double2 sm[];
  const int M = a.M, N = a.Nx, Nk = a.Nk;
  const int Ms = (M + 7) & ~7;
  double2* A = sm;           // 4 arrays: U spectrum, then gradient spectra of b, ux, uz
  double2* Bk = sm + 4 * Ms;  // ping-pong partner block
  double2* tw = sm + 8 * Ms;
  const int hN = N / 2;
  for (int t = threadIdx.x; t < a.nptw; t += blockDim.x) tw[t] = a.ptw[t];
  const int z = blockIdx.x;
  const int zm = a.Nz - 1 - z;
  const bool lower = z <= zm;
  const size_t ld = a.ld > 0 ? (size_t)a.ld : (size_t)Nk, col0 = (size_t)blockIdx.y * Nk;
  const size_t rr = (size_t)(lower ? z : zm) * ld + col0;
  auto hbin = [&](double2 v, int q) -> double2 {
    if (q == 0) return make_double2(v.x, 0.0);
    if (q == hN) return make_double2(0.5 * v.x, 0.0);
    return v;
  };
  auto put2 = [&](double2* dst, int q, double2 P, double2 Q) {
    dst[fidx<true>(q)] = pack2(P, Q);
    if (q > 0) dst[fidx<true>(M - q)] = pack2_mirror(P, Q);
  };
  // 1. all four inverse-transform inputs from one read of the six rows
  for (int q = threadIdx.x; q <= hN; q += blockDim.x) {
    double2 g[3], d[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const double2 e = a.ev[f][rr + q], o = a.ov[f][rr + q];
      const double2 ed = a.ed[f][rr + q], od = a.od[f][rr + q];
      g[f] = lower ? make_double2(e.x + o.x, e.y + o.y) : make_double2(e.x - o.x, e.y - o.y);
      d[f] = lower ? make_double2(ed.x + od.x, ed.y + od.y) : make_double2(od.x - ed.x, od.y - ed.y);
    }
    put2(A, q, hbin(g[1], q), hbin(g[2], q));
    const double kk = a.k0 * q;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      double2 Ax = make_double2(0.0, 0.0);
      if (q > 0 && q < hN) Ax = make_double2(-kk * g[f].y, kk * g[f].x);  // i k g
      put2(A + (size_t)(1 + f) * Ms, q, Ax, hbin(d[f], q));
    }
  }
  for (int k = hN + 1 + threadIdx.x; k < M - hN; k += blockDim.x)  // bins N/2 < k < M - N/2 are zero
#pragma unroll
    for (int arr = 0; arr < 4; ++arr) A[(size_t)arr * Ms + fidx<true>(k)] = make_double2(0.0, 0.0);
  __syncthreads();
  double2* Rb = fft_cta_multi(A, Bk, 4, Ms, a.fp, tw, +1);
  double2* Fb = (Rb == A) ? Bk : A;  // the free block
  // 2. products -(u d_x f + w d_z f) for f = b, ux, uz: (b + i ux) and (uz) spectra inputs
  for (int p = threadIdx.x; p < M; p += blockDim.x) {
    const int ps = fidx<true>(p);
    const double2 u = Rb[ps];
    double pr[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const double2 gg = Rb[(size_t)(1 + f) * Ms + ps];
      pr[f] = -(u.x * gg.x + u.y * gg.y);
    }
    Fb[ps] = make_double2(pr[0], pr[1]);
    Fb[(size_t)Ms + ps] = make_double2(pr[2], 0.0);
  }
  __syncthreads();
  // 3. both forward transforms through the same passes (Rb's first two arrays are free)
  double2* Cb = fft_cta_multi(Fb, Rb, 2, Ms, a.fp, tw, -1);
  const double2* C1 = Cb;
  const double2* C2 = Cb + Ms;
  const double sc = 1.0 / ((double)M * (double)N);
  const size_t ro = (size_t)z * ld + col0;
  for (int k = threadIdx.x; k < Nk; k += blockDim.x) {
    const double2 c = C1[fidx<true>(k)];
    const double2 cm = C1[fidx<true>((M - k) % M)];
    const double2 sb = make_double2(0.5 * (c.x + cm.x), 0.5 * (c.y - cm.y));
    const double2 su = make_double2(0.5 * (c.y + cm.y), -0.5 * (c.x - cm.x));
    const double2 c2 = C2[fidx<true>(k)];
    double2 ob, ou, oz;
    if (k == 0) {
      ob = make_double2(sb.x * sc, 0.0);
      ou = make_double2(su.x * sc, 0.0);
      oz = make_double2(c2.x * sc, 0.0);
    } else if (k == hN) {
      ob = make_double2(2.0 * sb.x * sc, 0.0);
      ou = make_double2(2.0 * su.x * sc, 0.0);
      oz = make_double2(2.0 * c2.x * sc, 0.0);
    } else {
      ob = cscale(sb, sc);
      ou = cscale(su, sc);
      oz = cscale(c2, sc);
    }
    a.out[0][ro + k] = ob;
    a.out[1][ro + k] = ou;
    a.out[2][ro + k] = oz;
  }
}

// rfft of real rows (unnormalised), via a complex FFT of the row.
__global__ void __launch_bounds__(256) k_x_rfft(const double* __restrict__ grid, double2* __restrict__ spec,
                                                int Nx, FftPlan fp, const double2* __restrict__ tw) {
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* B = sm + Nx;
  const int row = blockIdx.x;
  const int Nk = Nx / 2 + 1;
  for (int p = threadIdx.x; p < Nx; p += blockDim.x) A[p] = make_double2(grid[(size_t)row * Nx + p], 0.0);
  __syncthreads();
  double2* R = fft_cta(A, B, fp, tw, -1);
  for (int k = threadIdx.x; k < Nk; k += blockDim.x) {
    double2 v = R[k];
    if (k == 0 || 2 * k == Nx) v.y = 0.0;
    spec[(size_t)row * Nk + k] = v;
  }
}

// irfft (1/N) of half-spectrum rows, ignoring Im of DC and Nyquist.
__global__ void __launch_bounds__(256) k_x_irfft(const double2* __restrict__ spec, double* __restrict__ grid,
                                                 int Nx, FftPlan fp, const double2* __restrict__ tw) {
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* B = sm + Nx;
  const int row = blockIdx.x;
  const int Nk = Nx / 2 + 1;
  const double2* g = spec + (size_t)row * Nk;
  for (int k = threadIdx.x; k < Nx; k += blockDim.x) {
    double2 v;
    if (k < Nk) {
      v = g[k];
      if (k == 0 || 2 * k == Nx) v.y = 0.0;
    } else {
      v = cconj(g[Nx - k]);
    }
    A[k] = v;
  }
  __syncthreads();
  double2* R = fft_cta(A, B, fp, tw, +1);
  const double inv = 1.0 / Nx;
  for (int p = threadIdx.x; p < Nx; p += blockDim.x) grid[(size_t)row * Nx + p] = R[p].x * inv;
}

// Dealiased product of two real rows: pad both to M, multiply, truncate back.
__global__ void __launch_bounds__(256) k_x_dealias_mul(const double* __restrict__ a, const double* __restrict__ b,
                                                       double* __restrict__ out, int Nx, int M, FftPlan fpN,
                                                       const double2* __restrict__ twN, FftPlan fpM,
                                                       const double2* __restrict__ twM) {
  extern __shared__ double2 sm[];
  double2* A = sm;
  double2* B = sm + M;
  const int row = blockIdx.x;
  const int Nk = Nx / 2 + 1, half = M / 2, h = Nx / 2;
  // spectra of a + i b on the N grid
  for (int p = threadIdx.x; p < Nx; p += blockDim.x)
    A[p] = make_double2(a[(size_t)row * Nx + p], b[(size_t)row * Nx + p]);
  __syncthreads();
  double2* S = fft_cta(A, B, fpN, twN, -1);
  double2* T = (S == A) ? B : A;
  // unpack into half spectra (stored in T[0..Nk) and T[Nk..2Nk))
  for (int k = threadIdx.x; k < Nk; k += blockDim.x) {
    double2 c = S[k], cm = S[(Nx - k) % Nx];
    T[k] = make_double2(0.5 * (c.x + cm.x), 0.5 * (c.y - cm.y));
    T[Nk + k] = make_double2(0.5 * (c.y + cm.y), -0.5 * (c.x - cm.x));
  }
  __syncthreads();
  // move half spectra into registers-free scratch: copy to S then build padded
  for (int k = threadIdx.x; k < 2 * Nk; k += blockDim.x) S[k] = T[k];
  __syncthreads();
  double2* ha = S;
  double2* hb = S + Nk;
  // Build padded spectrum in T (length M); note S holds only 2*Nk <= M entries.
  // To avoid aliasing S and T, write to T after all reads of S are done per k.
  for (int k = threadIdx.x; k < M; k += blockDim.x) {
    int q = (k <= half) ? k : M - k;
    double2 A1 = half_bin(ha, q, Nx), B1 = half_bin(hb, q, Nx);
    T[k] = (k <= half) ? pack2(A1, B1) : pack2_mirror(A1, B1);
  }
  __syncthreads();
  double2* G = fft_cta(T, S, fpM, twM, +1);
  double2* H = (G == T) ? S : T;
  for (int p = threadIdx.x; p < M; p += blockDim.x) H[p] = make_double2(G[p].x * G[p].y, 0.0);
  __syncthreads();
  double2* C = fft_cta(H, G, fpM, twM, -1);
  double2* D = (C == H) ? G : H;
  // truncated half spectrum, scaled by 1/(M N) relative to the N-grid rfft, then irfft (1/N)
  const double sc = 1.0 / ((double)M * (double)Nx);
  for (int k = threadIdx.x; k < Nx; k += blockDim.x) {
    int q = (k < Nk) ? k : Nx - k;
    double2 c = C[q];
    double2 v;
    if (q == 0)
      v = make_double2(c.x * sc, 0.0);
    else if (q == h)
      v = make_double2(2.0 * c.x * sc, 0.0);
    else
      v = cscale(c, sc);
    D[k] = (k < Nk) ? v : cconj(v);
  }
  __syncthreads();
  double2* E = fft_cta(D, C, fpN, twN, +1);
  const double inv = 1.0 / Nx;
  for (int p = threadIdx.x; p < Nx; p += blockDim.x) out[(size_t)row * Nx + p] = E[p].x * inv;
}

}  // namespace

cudaError_t set_transform_smem_limits(int bytes) {
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(k_gemm_f64<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem)) !=
      cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(k_gemm_f64<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem)) !=
      cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(k_xprod, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_xprod_b<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(k_xprod_b<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(fftg::k_xprod_ip<256, double2, XProdArgs>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                bytes)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(fftg::k_xprod_ip<512, double2, XProdArgs>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                bytes)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(k_x_rfft, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_x_irfft, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_x_dealias_mul, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

size_t xprod_smem_bytes(int M, int Nk, int nptw) {
  (void)Nk;
  const size_t Ms = (size_t)((M + 7) & ~7);
  return (4 * Ms + (size_t)nptw) * sizeof(double2);
}

void launch_xprod(const XProdArgs& a, cudaStream_t st) {
  size_t smem = xprod_smem_bytes(a.M, a.Nk, a.nptw);
  k_xprod<<<dim3(a.Nz, a.instances > 0 ? a.instances : 1), 256, smem, st>>>(a);
}

size_t xprod_b_smem_bytes(int M, int nptw) {
  const size_t Ms = (size_t)((M + 7) & ~7);
  return (8 * Ms + (size_t)nptw) * sizeof(double2);
}

bool xprod_b_fits(int M, int nptw) { return xprod_b_smem_bytes(M, nptw) <= 227 * 1024; }

bool xprod_ip_fits(int M, int niptw) { return fftg::xprod_ip_smem_bytes<double2>(M, niptw) <= 227 * 1024; }

void launch_xprod_ip(const XProdArgs& a, cudaStream_t st) {
  const size_t smem = fftg::xprod_ip_smem_bytes<double2>(a.M, a.niptw);
  const dim3 grid(a.Nz, a.instances > 0 ? a.instances : 1);
  if (2 * smem <= 227 * 1024)  // two CTAs of 256 threads per SM while both fit
    fftg::k_xprod_ip<256, double2, XProdArgs><<<grid, 256, smem, st>>>(a);
  else
    fftg::k_xprod_ip<512, double2, XProdArgs><<<grid, 512, smem, st>>>(a);
}

void launch_xprod_b(const XProdArgs& a, cudaStream_t st) {
  const size_t smem = xprod_b_smem_bytes(a.M, a.nptw);
  const dim3 grid(a.Nz, a.instances > 0 ? a.instances : 1);
  // two CTAs of 256 threads per SM while both fit, else one of 512
  if (2 * smem <= 227 * 1024)
    k_xprod_b<256><<<grid, 256, smem, st>>>(a);
  else
    k_xprod_b<512><<<grid, 512, smem, st>>>(a);
}

void launch_x_rfft(const double* grid, double2* spec, int nrows, int Nx, const FftPlan& fp, const double2* tw,
                   cudaStream_t st) {
  size_t smem = 2 * (size_t)Nx * sizeof(double2);
  k_x_rfft<<<nrows, 256, smem, st>>>(grid, spec, Nx, fp, tw);
}

void launch_x_irfft(const double2* spec, double* grid, int nrows, int Nx, const FftPlan& fp, const double2* tw,
                    cudaStream_t st) {
  size_t smem = 2 * (size_t)Nx * sizeof(double2);
  k_x_irfft<<<nrows, 256, smem, st>>>(spec, grid, Nx, fp, tw);
}

void launch_x_dealias_mul(const double* a, const double* b, double* out, int nrows, int Nx, int M,
                          const FftPlan& fpN, const double2* twN, const FftPlan& fpM, const double2* twM,
                          cudaStream_t st) {
  size_t smem = 2 * (size_t)M * sizeof(double2);
  k_x_dealias_mul<<<nrows, 256, smem, st>>>(a, b, out, Nx, M, fpN, twN, fpM, twM);
}

}  // namespace tb
