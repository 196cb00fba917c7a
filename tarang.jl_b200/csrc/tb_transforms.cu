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

__global__ void __launch_bounds__(GTH) k_gemm_f64(GemmBatch bt, int ncol, int ldb, int ldc, int Nrows) {
  extern __shared__ __align__(16) double gsm[];
  double (*As)[GBM * ASTR] = reinterpret_cast<double (*)[GBM * ASTR]>(gsm);
  double (*Bs)[GBK * BSTR] = reinterpret_cast<double (*)[GBK * BSTR]>(gsm + 2 * GBM * ASTR);
  double (*Bm)[GBK * BSTR] = reinterpret_cast<double (*)[GBK * BSTR]>(gsm + 2 * GBM * ASTR + 2 * GBK * BSTR);  // mirror partners
  const GemmItem& it = bt.item[blockIdx.z];
  const double* __restrict__ A = it.A;
  const double* __restrict__ B = it.B;
  const int Mo = it.M, K = it.K, Kp = it.Kpad, mode = it.mode, par = it.par;
  const int row0 = blockIdx.y * GBM, col0 = blockIdx.x * GBN;
  if (row0 >= Mo) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int gid = lane >> 2, tig = lane & 3;
  const bool mirror = mode == GEMM_MIRROR;
  const int ntiles = (K + GBK - 1) / GBK;

  auto load_tile = [&](int t, int buf) {
    const int k0 = t * GBK;
    // A: 64 rows x 16 doubles = 512 chunks of 16 B, 4 per thread
#pragma unroll
    for (int q = 0; q < 4; ++q) {
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
    const double* as = As[buf];
    const double* bs = Bs[buf];
    const double* bm = Bm[buf];
#pragma unroll
    for (int ks = 0; ks < GBK / 4; ++ks) {
      const int kk = ks * 4 + tig;
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = as[(wm * 32 + i * 8 + gid) * ASTR + kk];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int cidx = kk * BSTR + wn * 32 + j * 8 + gid;
        double v = bs[cidx];
        if (mirror) {
          const int gk = t * GBK + kk;
          v = (gk == midk) ? (par ? 0.0 : v) : fma(sgn, bm[cidx], v);
        }
        b[j] = v;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    __syncthreads();
  }
  g_wait0();
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
  dim3 grid((ncol + GBN - 1) / GBN, (mmax + GBM - 1) / GBM, nbatch);
  k_gemm_f64<<<grid, GTH, kGemmSmem, st>>>(bt, ncol, ldb, ldc, Nrows);
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

// One Stockham pass of radix R (Govindaraju et al. formulation: read
// in[idx + r n/R], twiddle by w^(j r n/(Ns R)), R-point DFT, write
// out[(idx/Ns) Ns R + idx%Ns + r Ns]).  Output ends in natural order.
template <int R>
__device__ __forceinline__ void fft_pass(const double2* __restrict__ in, double2* __restrict__ out, int n, int Ns,
                                         const double2* __restrict__ tw, int sign) {
  const int nR = n / R;
  const int tstride = n / (Ns * R);
  for (int idx = threadIdx.x; idx < nR; idx += blockDim.x) {
    const int j = idx % Ns, k = idx / Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      double2 x = in[idx + r * nR];
      if (r > 0) {
        double2 w = tw[j * r * tstride];
        if (sign > 0) w.y = -w.y;
        x = cmul(x, w);
      }
      v[r] = x;
    }
    const int ob = k * Ns * R + j;
    if (R == 2) {
      out[ob] = cadd(v[0], v[1]);
      out[ob + Ns] = csub(v[0], v[1]);
    } else if (R == 4) {
      double2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
      double2 t2 = cadd(v[1], v[3]), d = csub(v[1], v[3]);
      // forward: -i d ; inverse: +i d
      double2 t3 = (sign < 0) ? make_double2(d.y, -d.x) : make_double2(-d.y, d.x);
      out[ob] = cadd(t0, t2);
      out[ob + Ns] = cadd(t1, t3);
      out[ob + 2 * Ns] = csub(t0, t2);
      out[ob + 3 * Ns] = csub(t1, t3);
    } else {  // R == 3
      const double h = 0.86602540378443864676372317075294;  // sqrt(3)/2
      double2 sm = cadd(v[1], v[2]), df = csub(v[1], v[2]);
      double2 base = make_double2(v[0].x - 0.5 * sm.x, v[0].y - 0.5 * sm.y);
      double2 rot = make_double2(-sign * h * df.y, sign * h * df.x);  // i sign h df
      out[ob] = cadd(v[0], sm);
      out[ob + Ns] = cadd(base, rot);
      out[ob + 2 * Ns] = csub(base, rot);
    }
  }
}

// Returns the buffer holding the result (a or b).  sign = -1 forward, +1 inverse
// (both unnormalised).  tw[t] = exp(-2 pi i t / n).
__device__ double2* fft_cta(double2* a, double2* b, const FftPlan& fp, const double2* __restrict__ tw, int sign) {
  const int n = fp.n;
  int Ns = 1;
  double2* in = a;
  double2* out = b;
  for (int s = 0; s < fp.nstages; ++s) {
    const int R = fp.radix[s];
    if (R == 4)
      fft_pass<4>(in, out, n, Ns, tw, sign);
    else if (R == 2)
      fft_pass<2>(in, out, n, Ns, tw, sign);
    else
      fft_pass<3>(in, out, n, Ns, tw, sign);
    __syncthreads();
    double2* t = in;
    in = out;
    out = t;
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

__global__ void __launch_bounds__(256) k_xprod(XProdArgs a) {
  extern __shared__ double2 sm[];
  const int M = a.M, N = a.Nx, Nk = a.Nk;
  double2* X = sm;          // velocity on the padded grid: ux + i uz
  double2* Y = sm + M;
  double2* W = sm + 2 * M;
  double2* P = sm + 3 * M;  // prod_b + i prod_ux
  double* Puz = reinterpret_cast<double*>(sm + 4 * M);  // after the products are formed
  double2* Rrows = sm + 4 * M + (M + 1) / 2;              // the 6 combined input rows (6 Nk entries)
  const int z = blockIdx.x;
  const size_t ro = (size_t)z * Nk;
  const int half = M / 2;
  // Grid row z from the even/odd Chebyshev half planes: rows z < H are E + O,
  // mirrored rows N-1-z are E - O for values and -E + O for z-derivatives.
  double2* R = Rrows;
  {
    const int Nz = a.Nz;
    const int zm = Nz - 1 - z;
    const bool lower = z <= zm;
    const int zr = lower ? z : zm;
    const size_t rr = (size_t)zr * Nk;
    for (int k = threadIdx.x; k < Nk; k += blockDim.x)
      for (int f = 0; f < 3; ++f) {
        const double2 ev = a.ev[f][rr + k], ov = a.ov[f][rr + k];
        const double2 ed = a.ed[f][rr + k], od = a.od[f][rr + k];
        R[(2 * f) * Nk + k] = lower ? make_double2(ev.x + ov.x, ev.y + ov.y) : make_double2(ev.x - ov.x, ev.y - ov.y);
        R[(2 * f + 1) * Nk + k] = lower ? make_double2(ed.x + od.x, ed.y + od.y) : make_double2(od.x - ed.x, od.y - ed.y);
      }
  }
  __syncthreads();
  // 1. velocity spectrum
  {
    const double2* gx = R + 2 * Nk;
    const double2* gz = R + 4 * Nk;
    for (int k = threadIdx.x; k < M; k += blockDim.x) {
      double2 v;
      if (k <= half) {
        v = pack2(half_bin(gx, k, N), half_bin(gz, k, N));
      } else {
        int q = M - k;
        v = pack2_mirror(half_bin(gx, q, N), half_bin(gz, q, N));
      }
      X[k] = v;
    }
  }
  __syncthreads();
  double2* U = fft_cta(X, Y, a.fp, a.tw, +1);
  double2* F0 = (U == X) ? Y : X;  // free buffers: F0 and W
  // 2. gradients of each field and the advection products
  for (int f = 0; f < 3; ++f) {
    const double2* gv = R + (2 * f) * Nk;
    const double2* gd = R + (2 * f + 1) * Nk;
    for (int k = threadIdx.x; k < M; k += blockDim.x) {
      int q = (k <= half) ? k : M - k;
      double2 Ax = make_double2(0.0, 0.0);
      if (q > 0 && q < N / 2) {
        double kk = a.k0 * q;
        double2 g = gv[q];
        Ax = make_double2(-kk * g.y, kk * g.x);  // i k g
      }
      double2 Az = half_bin(gd, q, N);
      F0[k] = (k <= half) ? pack2(Ax, Az) : pack2_mirror(Ax, Az);
    }
    __syncthreads();
    double2* G = fft_cta(F0, W, a.fp, a.tw, +1);
    for (int p = threadIdx.x; p < M; p += blockDim.x) {
      double2 u = U[p], g = G[p];
      double pr = -(u.x * g.x + u.y * g.y);
      if (f == 0)
        P[p].x = pr;
      else if (f == 1)
        P[p].y = pr;
      else
        Puz[p] = pr;
    }
    __syncthreads();
  }
  // 3. forward transforms of the products
  double2* C1 = fft_cta(P, F0, a.fp, a.tw, -1);
  // Save the two unpacked spectra for k <= N/2 into the free buffer W... then FFT Puz.
  const double sc = 1.0 / ((double)M * (double)N);
  const int h = N / 2;
  for (int k = threadIdx.x; k < Nk; k += blockDim.x) {
    double2 c = C1[k];
    double2 cm = C1[(M - k) % M];
    // b: (c + conj(cm))/2 ; ux: (c - conj(cm))/(2i)
    double2 sb = make_double2(0.5 * (c.x + cm.x), 0.5 * (c.y - cm.y));
    double2 su = make_double2(0.5 * (c.y + cm.y), -0.5 * (c.x - cm.x));
    double2 ob, ou;
    if (k == 0) {
      ob = make_double2(sb.x * sc, 0.0);
      ou = make_double2(su.x * sc, 0.0);
    } else if (k == h) {
      ob = make_double2(2.0 * sb.x * sc, 0.0);
      ou = make_double2(2.0 * su.x * sc, 0.0);
    } else {
      ob = cscale(sb, sc);
      ou = cscale(su, sc);
    }
    a.out[0][ro + k] = ob;
    a.out[1][ro + k] = ou;
  }
  __syncthreads();
  double2* B1 = (C1 == P) ? F0 : P;
  for (int p = threadIdx.x; p < M; p += blockDim.x) B1[p] = make_double2(Puz[p], 0.0);
  __syncthreads();
  double2* B2 = (B1 == P) ? F0 : P;
  double2* C2 = fft_cta(B1, B2, a.fp, a.tw, -1);
  for (int k = threadIdx.x; k < Nk; k += blockDim.x) {
    double2 c = C2[k];
    double2 o;
    if (k == 0)
      o = make_double2(c.x * sc, 0.0);
    else if (k == h)
      o = make_double2(2.0 * c.x * sc, 0.0);
    else
      o = cscale(c, sc);
    a.out[2][ro + k] = o;
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
  if ((e = cudaFuncSetAttribute(k_gemm_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem)) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(k_xprod, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_x_rfft, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
  if ((e = cudaFuncSetAttribute(k_x_irfft, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_x_dealias_mul, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

size_t xprod_smem_bytes(int M, int Nk) {
  return (size_t)M * 4 * sizeof(double2) + (size_t)((M + 1) / 2) * sizeof(double2) + (size_t)6 * Nk * sizeof(double2);
}

void launch_xprod(const XProdArgs& a, cudaStream_t st) {
  size_t smem = xprod_smem_bytes(a.M, a.Nk);
  k_xprod<<<a.Nz, 256, smem, st>>>(a);
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
