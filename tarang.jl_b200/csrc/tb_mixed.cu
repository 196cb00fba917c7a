// FP32 right-hand side of the mixed-precision RBC step (TB_PREC_MIXED).
//
// The transforms and the dealiased products of the RHS program run in FP32:
// the state is rounded to FP32, the Chebyshev backward transform (even/odd
// halves, values and z-derivatives), the per-row Fourier FFTs and products and
// the forward transform to C^(2) rows all run on float data, and the forward
// GEMM writes the FP64 stage vector F directly from its FP32 accumulators.
// The tau LU, its solves and the stage algebra stay FP64.
//
// Kernels: k_round_f32 (state planes to FP32), k_gemm_f32<OutT> (SIMT FP32
// GEMM with the row maps of the FP64 transform GEMM), k_xprod32 (per z row:
// packed inverse FFTs, products, forward FFTs, as k_xprod).
#include <cuda_runtime.h>

#include "tb_fft.cuh"
#include "tb_kernels.cuh"

namespace tb {

namespace {

namespace F = tb::fftg;

__global__ void k_round_f32(const double2* __restrict__ in, float2* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 v = in[i];
    out[i] = make_float2((float)v.x, (float)v.y);
  }
}

// C (M x ncol) = A (M x K, row stride Kpad) . B' (K x ncol), B' rows mapped as
// in the FP64 transform GEMM: GEMM_PLAIN row k = B[k], GEMM_PARITY row k =
// B[2k + par], GEMM_MIRROR row j = B[j] + sgn B[N-1-j] (middle row of odd N
// once / not at all) with output row 2r + par.  CTA tile 64 x 64, K slices of
// 16 through shared memory (next slice prefetched in registers), 256 threads
// with 4 x 4 outputs each.
constexpr int SBM = 64, SBN = 64, SBK = 16, STH = 256;

template <class OutT>
__global__ void __launch_bounds__(STH) k_gemm_f32(GemmBatch32 bt, int ncol, int ldb, int ldc, int Nrows) {
  __shared__ __align__(16) float As[2][SBK][SBM];  // transposed A tile
  __shared__ __align__(16) float Bs[2][SBK][SBN];
  const GemmItem32& it = bt.item[blockIdx.z];
  const float* __restrict__ A = it.A;
  const float* __restrict__ B = it.B;
  const int Mo = it.M, K = it.K, Kp = it.Kpad, mode = it.mode, par = it.par;
  const int row0 = blockIdx.y * SBM, col0 = blockIdx.x * SBN;
  if (row0 >= Mo) return;
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  const bool mirror = mode == GEMM_MIRROR;
  const float sgn = par ? -1.f : 1.f;
  const int midk = (mirror && (Nrows & 1)) ? (Nrows - 1) / 2 : -1;
  const int ntiles = (K + SBK - 1) / SBK;
  // staging registers: A one float4 (row ar, k 4ak..), B two float2 (row bk, cols bc, bc + 32)
  const int ar = tid / 4, ak = (tid % 4) * 4;
  const int bk = tid / 16, bc = (tid % 16) * 2;
  float4 ra;
  float2 rb[2];
  auto fetch = [&](int t) {
    const int k0 = t * SBK;
    const int gr = row0 + ar;
    ra = (gr < Mo) ? *reinterpret_cast<const float4*>(A + (size_t)gr * Kp + k0 + ak) : make_float4(0.f, 0.f, 0.f, 0.f);
    const int gk = k0 + bk;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int gc = col0 + bc + 32 * h;
      float2 v = make_float2(0.f, 0.f);
      if (gk < K && gc < ncol) {
        int srow = gk;
        if (mode == GEMM_PARITY) srow = 2 * gk + par;
        v = *reinterpret_cast<const float2*>(B + (size_t)srow * ldb + gc);
        if (mirror) {
          const int jm = Nrows - 1 - gk;
          if (gk == midk) {
            if (par) v = make_float2(0.f, 0.f);
          } else {
            const float2 w = *reinterpret_cast<const float2*>(B + (size_t)jm * ldb + gc);
            v = make_float2(fmaf(sgn, w.x, v.x), fmaf(sgn, w.y, v.y));
          }
        }
      }
      rb[h] = v;
    }
  };
  auto stash = [&](int buf) {
    As[buf][ak + 0][ar] = ra.x;
    As[buf][ak + 1][ar] = ra.y;
    As[buf][ak + 2][ar] = ra.z;
    As[buf][ak + 3][ar] = ra.w;
    *reinterpret_cast<float2*>(&Bs[buf][bk][bc]) = rb[0];
    *reinterpret_cast<float2*>(&Bs[buf][bk][bc + 32]) = rb[1];
  };
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
  fetch(0);
  stash(0);
  __syncthreads();
  for (int t = 0; t < ntiles; ++t) {
    const int buf = t & 1;
    if (t + 1 < ntiles) fetch(t + 1);
#pragma unroll
    for (int k = 0; k < SBK; ++k) {
      const float4 a = *reinterpret_cast<const float4*>(&As[buf][k][ty * 4]);
      // columns tx*2 + {0,1} and tx*2 + 32 + {0,1}
      const float2 b0 = *reinterpret_cast<const float2*>(&Bs[buf][k][tx * 2]);
      const float2 b1 = *reinterpret_cast<const float2*>(&Bs[buf][k][tx * 2 + 32]);
      const float av[4] = {a.x, a.y, a.z, a.w};
      const float bv[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    if (t + 1 < ntiles) stash(buf ^ 1);
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gr = row0 + ty * 4 + i;
    if (gr >= Mo) continue;
    const int orow = mirror ? 2 * gr + par : gr;
    OutT* C = reinterpret_cast<OutT*>(it.C) + (size_t)orow * ldc;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int gc = col0 + tx * 2 + 32 * h;
      if (gc < ncol) C[gc] = (OutT)acc[i][2 * h];
      if (gc + 1 < ncol) C[gc + 1] = (OutT)acc[i][2 * h + 1];
    }
  }
}

__device__ __forceinline__ float2 half_bin32(const float2* __restrict__ g, int k, int N) {
  const int h = N / 2;
  if (k == 0) return make_float2(g[0].x, 0.f);
  if (k < h) return g[k];
  if (k == h) return make_float2(0.5f * g[h].x, 0.f);
  return make_float2(0.f, 0.f);
}

// FP32 twin of k_xprod (same data flow, float2 buffers and twiddles).
__global__ void __launch_bounds__(256, 2) k_xprod32(XProdArgs32 a) {
  extern __shared__ float2 sm32[];
  const int M = a.M, N = a.Nx, Nk = a.Nk;
  const int Ms = (M + 7) & ~7;
  float2* S0 = sm32;
  float2* S1 = sm32 + Ms;
  float2* S2 = sm32 + 2 * Ms;
  float2* S3 = sm32 + 3 * Ms;
  float2* tw = sm32 + 4 * Ms;
  const int hN = N / 2;
  for (int t = threadIdx.x; t < a.nptw; t += blockDim.x) tw[t] = a.ptw[t];
  const int z = blockIdx.x;
  const int zm = a.Nz - 1 - z;
  const bool lower = z <= zm;
  const size_t ld = a.ld > 0 ? (size_t)a.ld : (size_t)Nk, col0 = (size_t)blockIdx.y * Nk;
  const size_t rr = (size_t)(lower ? z : zm) * ld + col0;
  auto value = [&](int f, int q) -> float2 {
    const float2 e = a.ev[f][rr + q], o = a.ov[f][rr + q];
    return lower ? make_float2(e.x + o.x, e.y + o.y) : make_float2(e.x - o.x, e.y - o.y);
  };
  auto deriv = [&](int f, int q) -> float2 {
    const float2 e = a.ed[f][rr + q], o = a.od[f][rr + q];
    return lower ? make_float2(e.x + o.x, e.y + o.y) : make_float2(o.x - e.x, o.y - e.y);
  };
  auto hbin = [&](float2 v, int q) -> float2 {
    if (q == 0) return make_float2(v.x, 0.f);
    if (q == hN) return make_float2(0.5f * v.x, 0.f);
    return v;
  };
  auto put2 = [&](float2* dst, int q, float2 A, float2 B) {
    dst[F::fidx<true>(q)] = make_float2(A.x - B.y, A.y + B.x);
    if (q > 0) dst[F::fidx<true>(M - q)] = make_float2(A.x + B.y, -A.y + B.x);
  };
  auto zero_gap = [&](float2* dst) {
    for (int k = hN + 1 + threadIdx.x; k < M - hN; k += blockDim.x) dst[F::fidx<true>(k)] = make_float2(0.f, 0.f);
  };
  // inputs in batches of QB bins per thread, every load issued before the
  // first is used (one wait for memory per batch)
  constexpr int QB = 3;
  for (int q0 = threadIdx.x; q0 <= hN; q0 += QB * blockDim.x) {
    float2 vx[QB], vz[QB];
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
  float2* U = F::fft<true>(S0, S1, a.fp, tw, +1);
  float2* P = (U == S0) ? S1 : S0;
  for (int f = 0; f < 3; ++f) {
    for (int q0 = threadIdx.x; q0 <= hN; q0 += QB * blockDim.x) {
      float2 gv[QB], dv[QB];
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
          float2 Ax = make_float2(0.f, 0.f);
          if (q > 0 && q < hN) {
            const float kk = a.k0 * q;
            Ax = make_float2(-kk * gv[i].y, kk * gv[i].x);
          }
          put2(S2, q, Ax, hbin(dv[i], q));
        }
      }
    }
    zero_gap(S2);
    __syncthreads();
    float2* G = F::fft<true>(S2, S3, a.fp, tw, +1);
    float2* Gf = (G == S2) ? S3 : S2;
    for (int p = threadIdx.x; p < M; p += blockDim.x) {
      const int ps = F::fidx<true>(p);
      const float2 u = U[ps], g = G[ps];
      const float pr = -(u.x * g.x + u.y * g.y);
      if (f == 0)
        P[ps].x = pr;
      else if (f == 1)
        P[ps].y = pr;
      else
        Gf[ps] = make_float2(pr, 0.f);
    }
    __syncthreads();
    if (f == 2) {
      float2* C1 = F::fft<true>(P, G, a.fp, tw, -1);
      float2* C2 = F::fft<true>(Gf, U, a.fp, tw, -1);
      const float sc = 1.0f / ((float)M * (float)N);
      const size_t ro = (size_t)z * ld + col0;
      for (int k = threadIdx.x; k < Nk; k += blockDim.x) {
        const float2 c = C1[F::fidx<true>(k)];
        const float2 cm = C1[F::fidx<true>((M - k) % M)];
        const float2 sb = make_float2(0.5f * (c.x + cm.x), 0.5f * (c.y - cm.y));
        const float2 su = make_float2(0.5f * (c.y + cm.y), -0.5f * (c.x - cm.x));
        const float2 c2 = C2[F::fidx<true>(k)];
        float2 ob, ou, oz;
        if (k == 0) {
          ob = make_float2(sb.x * sc, 0.f);
          ou = make_float2(su.x * sc, 0.f);
          oz = make_float2(c2.x * sc, 0.f);
        } else if (k == hN) {
          ob = make_float2(2.f * sb.x * sc, 0.f);
          ou = make_float2(2.f * su.x * sc, 0.f);
          oz = make_float2(2.f * c2.x * sc, 0.f);
        } else {
          ob = make_float2(sb.x * sc, sb.y * sc);
          ou = make_float2(su.x * sc, su.y * sc);
          oz = make_float2(c2.x * sc, c2.y * sc);
        }
        a.out[0][ro + k] = ob;
        a.out[1][ro + k] = ou;
        a.out[2][ro + k] = oz;
      }
    }
  }
}

// k_xprod32 with the transforms batched (as k_xprod_b): the velocity and the
// three gradient spectra from one read of the inputs, one set of inverse
// passes for the four, the three products at once, one set of forward passes
// for the two product spectra.
template <int NT>
__global__ void __launch_bounds__(NT, NT == 256 ? 2 : 1) k_xprod32_b(XProdArgs32 a) {
  extern __shared__ float2 sm32b[];
  const int M = a.M, N = a.Nx, Nk = a.Nk;
  const int Ms = (M + 7) & ~7;
  float2* A = sm32b;
  float2* Bk = sm32b + 4 * Ms;
  float2* tw = sm32b + 8 * Ms;
  const int hN = N / 2;
  for (int t = threadIdx.x; t < a.nptw; t += blockDim.x) tw[t] = a.ptw[t];
  const int z = blockIdx.x;
  const int zm = a.Nz - 1 - z;
  const bool lower = z <= zm;
  const size_t ld = a.ld > 0 ? (size_t)a.ld : (size_t)Nk, col0 = (size_t)blockIdx.y * Nk;
  const size_t rr = (size_t)(lower ? z : zm) * ld + col0;
  auto hbin = [&](float2 v, int q) -> float2 {
    if (q == 0) return make_float2(v.x, 0.f);
    if (q == hN) return make_float2(0.5f * v.x, 0.f);
    return v;
  };
  auto put2 = [&](float2* dst, int q, float2 P, float2 Q) {
    dst[F::fidx<true>(q)] = make_float2(P.x - Q.y, P.y + Q.x);
    if (q > 0) dst[F::fidx<true>(M - q)] = make_float2(P.x + Q.y, -P.y + Q.x);
  };
  for (int q = threadIdx.x; q <= hN; q += blockDim.x) {
    float2 g[3], d[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const float2 e = a.ev[f][rr + q], o = a.ov[f][rr + q];
      const float2 ed = a.ed[f][rr + q], od = a.od[f][rr + q];
      g[f] = lower ? make_float2(e.x + o.x, e.y + o.y) : make_float2(e.x - o.x, e.y - o.y);
      d[f] = lower ? make_float2(ed.x + od.x, ed.y + od.y) : make_float2(od.x - ed.x, od.y - ed.y);
    }
    put2(A, q, hbin(g[1], q), hbin(g[2], q));
    const float kk = a.k0 * q;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      float2 Ax = make_float2(0.f, 0.f);
      if (q > 0 && q < hN) Ax = make_float2(-kk * g[f].y, kk * g[f].x);
      put2(A + (size_t)(1 + f) * Ms, q, Ax, hbin(d[f], q));
    }
  }
  for (int k = hN + 1 + threadIdx.x; k < M - hN; k += blockDim.x)
#pragma unroll
    for (int arr = 0; arr < 4; ++arr) A[(size_t)arr * Ms + F::fidx<true>(k)] = make_float2(0.f, 0.f);
  __syncthreads();
  float2* Rb = F::fft_multi<true>(A, Bk, 4, Ms, a.fp, tw, +1);
  float2* Fb = (Rb == A) ? Bk : A;
  for (int p = threadIdx.x; p < M; p += blockDim.x) {
    const int ps = F::fidx<true>(p);
    const float2 u = Rb[ps];
    float pr[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const float2 gg = Rb[(size_t)(1 + f) * Ms + ps];
      pr[f] = -(u.x * gg.x + u.y * gg.y);
    }
    Fb[ps] = make_float2(pr[0], pr[1]);
    Fb[(size_t)Ms + ps] = make_float2(pr[2], 0.f);
  }
  __syncthreads();
  float2* Cb = F::fft_multi<true>(Fb, Rb, 2, Ms, a.fp, tw, -1);
  const float2* C1 = Cb;
  const float2* C2 = Cb + Ms;
  const float sc = 1.0f / ((float)M * (float)N);
  const size_t ro = (size_t)z * ld + col0;
  for (int k = threadIdx.x; k < Nk; k += blockDim.x) {
    const float2 c = C1[F::fidx<true>(k)];
    const float2 cm = C1[F::fidx<true>((M - k) % M)];
    const float2 sb = make_float2(0.5f * (c.x + cm.x), 0.5f * (c.y - cm.y));
    const float2 su = make_float2(0.5f * (c.y + cm.y), -0.5f * (c.x - cm.x));
    const float2 c2 = C2[F::fidx<true>(k)];
    float2 ob, ou, oz;
    if (k == 0) {
      ob = make_float2(sb.x * sc, 0.f);
      ou = make_float2(su.x * sc, 0.f);
      oz = make_float2(c2.x * sc, 0.f);
    } else if (k == hN) {
      ob = make_float2(2.f * sb.x * sc, 0.f);
      ou = make_float2(2.f * su.x * sc, 0.f);
      oz = make_float2(2.f * c2.x * sc, 0.f);
    } else {
      ob = make_float2(sb.x * sc, sb.y * sc);
      ou = make_float2(su.x * sc, su.y * sc);
      oz = make_float2(c2.x * sc, c2.y * sc);
    }
    a.out[0][ro + k] = ob;
    a.out[1][ro + k] = ou;
    a.out[2][ro + k] = oz;
  }
}

}  // namespace

void launch_round_f32(const double2* in, float2* out, long long n, cudaStream_t st) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_round_f32<<<blocks, 256, 0, st>>>(in, out, n);
}

void launch_gemm_f32(const GemmBatch32& bt, int nbatch, int ncol, int ldb, int ldc, int Nrows, bool out_f64,
                     cudaStream_t st) {
  int mmax = 0;
  for (int b = 0; b < nbatch; ++b) mmax = bt.item[b].M > mmax ? bt.item[b].M : mmax;
  dim3 grid((ncol + SBN - 1) / SBN, (mmax + SBM - 1) / SBM, nbatch);
  if (out_f64)
    k_gemm_f32<double><<<grid, STH, 0, st>>>(bt, ncol, ldb, ldc, Nrows);
  else
    k_gemm_f32<float><<<grid, STH, 0, st>>>(bt, ncol, ldb, ldc, Nrows);
}

size_t xprod32_smem_bytes(int M, int nptw) {
  const size_t Ms = (size_t)((M + 7) & ~7);
  return (4 * Ms + (size_t)nptw) * sizeof(float2);
}

cudaError_t set_mixed_smem_limits(int bytes) {
  cudaError_t e = cudaFuncSetAttribute(k_xprod32, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(F::k_xprod_ip<256, float2, XProdArgs32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           bytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(F::k_xprod_ip<512, float2, XProdArgs32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           bytes);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_xprod32_b<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_xprod32_b<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

void launch_xprod32(const XProdArgs32& a, cudaStream_t st) {
  k_xprod32<<<dim3(a.Nz, a.instances > 0 ? a.instances : 1), 256, xprod32_smem_bytes(a.M, a.nptw), st>>>(a);
}

size_t xprod32_b_smem_bytes(int M, int nptw) {
  const size_t Ms = (size_t)((M + 7) & ~7);
  return (8 * Ms + (size_t)nptw) * sizeof(float2);
}

bool xprod32_b_fits(int M, int nptw) { return xprod32_b_smem_bytes(M, nptw) <= 227 * 1024; }

bool xprod32_ip_fits(int M, int niptw) { return F::xprod_ip_smem_bytes<float2>(M, niptw) <= 227 * 1024; }

void launch_xprod32_ip(const XProdArgs32& a, cudaStream_t st) {
  const size_t smem = F::xprod_ip_smem_bytes<float2>(a.M, a.niptw);
  const dim3 grid(a.Nz, a.instances > 0 ? a.instances : 1);
  if (2 * smem <= 227 * 1024)
    F::k_xprod_ip<256, float2, XProdArgs32><<<grid, 256, smem, st>>>(a);
  else
    F::k_xprod_ip<512, float2, XProdArgs32><<<grid, 512, smem, st>>>(a);
}

void launch_xprod32_b(const XProdArgs32& a, cudaStream_t st) {
  const size_t smem = xprod32_b_smem_bytes(a.M, a.nptw);
  const dim3 grid(a.Nz, a.instances > 0 ? a.instances : 1);
  if (2 * smem <= 227 * 1024)
    k_xprod32_b<256><<<grid, 256, smem, st>>>(a);
  else
    k_xprod32_b<512><<<grid, 512, smem, st>>>(a);
}

}  // namespace tb
