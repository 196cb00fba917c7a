// Batched dense complex LU with partial pivoting, one CTA per matrix.
//
// Drop-in for BatchedDenseLU (src/tools/batched_matsolvers.jl:57-123), whose
// CUDA methods call getrf/getrs strided-batched
// (ext/cuda/batched_matsolvers.jl:80-125): A is column-major n x n complex128
// per slice and is overwritten by L (unit, below the diagonal) and U; ipiv is
// 1-based LAPACK style (row i was swapped with row ipiv[i]).  A slice with an
// exactly zero pivot is reported, never silently solved.
//
// Blocked right-looking factorisation (n <= kLuBlockedMaxN; larger slices use
// the unblocked kernel below), panels of kLuNb columns:
//   1. the panel (rows j0..n-1) is factored in shared memory: per column a
//      block-wide pivot search (largest |re| + |im|, lowest row on ties, as
//      izamax), the row swap inside the panel, the scaling by the pivot's
//      reciprocal and the rank-1 update of the panel's later columns;
//   2. the panel's swaps are applied to the columns left and right of it (one
//      thread per column, the swaps in order);
//   3. U12 = L11^-1 A12 (unit lower triangular, one thread per column), kept
//      in shared memory and written back;
//   4. A22 -= L21 U12 with L21 and U12 from shared memory, each thread a 4 x 4
//      complex tile of A22 read from and written to global memory (L2), the
//      16-deep inner product in registers.
// Shared memory per slice: the panel (n x 16) and U12 (16 x n), 2 * 16 * 16 n
// bytes (135 KB at n = 263).
#include <cuda_runtime.h>

#include <mutex>

#include "tb_internal.h"

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
// acc -= a * b
__device__ __forceinline__ void cfms(double2& acc, double2 a, double2 b) {
  acc.x = fma(-a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(-a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}

constexpr int kLuNb = 16;            // panel width
constexpr int kLuThreads = 256;
constexpr int kLuBlockedMaxN = 440;  // 2 * 16 * 16 * n bytes of shared memory <= 227 KB

size_t lu_blocked_smem(int n) { return (size_t)2 * kLuNb * n * sizeof(double2) + 64; }

__global__ void __launch_bounds__(kLuThreads) k_dense_getrf_blocked(int n, double2* __restrict__ Ab,
                                                                    int* __restrict__ pivb, int* __restrict__ bad) {
  extern __shared__ __align__(16) double2 lsm[];
  __shared__ double rv[kLuThreads / 32];
  __shared__ int ri[kLuThreads / 32];
  __shared__ int sp;
  __shared__ double2 sinv;
  const int s = blockIdx.x;
  double2* A = Ab + (size_t)s * n * n;
  int* piv = pivb + (size_t)s * n;
  const int tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
  double2* Pn = lsm;                      // panel, column-major, leading dimension n
  double2* U = lsm + (size_t)kLuNb * n;   // U12, [k][column], leading dimension n
  for (int j0 = 0; j0 < n; j0 += kLuNb) {
    const int jb = min(kLuNb, n - j0), m = n - j0;
    // 1. panel rows j0..n-1, columns j0..j0+jb-1 into shared memory
    for (int q = tid; q < jb * m; q += kLuThreads) {
      const int c = q / m, r = q % m;
      Pn[(size_t)c * n + r] = A[(size_t)(j0 + c) * n + j0 + r];
    }
    __syncthreads();
    for (int c = 0; c < jb; ++c) {
      double best = -1.0;
      int bi = c;
      for (int r = c + tid; r < m; r += kLuThreads) {
        const double2 v = Pn[(size_t)c * n + r];
        const double a = fabs(v.x) + fabs(v.y);
        if (a > best) {
          best = a;
          bi = r;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (lane == 0) {
        rv[warp] = best;
        ri[warp] = bi;
      }
      __syncthreads();
      if (tid == 0) {
        double b = rv[0];
        int i = ri[0];
        for (int w = 1; w < kLuThreads / 32; ++w)
          if (rv[w] > b || (rv[w] == b && ri[w] < i)) {
            b = rv[w];
            i = ri[w];
          }
        sp = (b > 0.0) ? i : -1;
        piv[j0 + c] = j0 + (b > 0.0 ? i : c) + 1;
        if (!(b > 0.0)) atomicMin(bad, s);
      }
      __syncthreads();
      const int p = sp;
      if (p < 0) return;  // singular: reported, the slice is left as it is
      if (p != c && tid < jb) {
        const double2 t = Pn[(size_t)tid * n + c];
        Pn[(size_t)tid * n + c] = Pn[(size_t)tid * n + p];
        Pn[(size_t)tid * n + p] = t;
      }
      __syncthreads();
      if (tid == 0) sinv = cdiv(make_double2(1.0, 0.0), Pn[(size_t)c * n + c]);
      __syncthreads();
      const double2 inv = sinv;
      for (int r = c + 1 + tid; r < m; r += kLuThreads) Pn[(size_t)c * n + r] = cmul(Pn[(size_t)c * n + r], inv);
      __syncthreads();
      const int mr = m - c - 1, mc = jb - c - 1;
      for (int q = tid; q < mr * mc; q += kLuThreads) {
        const int cc = c + 1 + q / mr, r = c + 1 + q % mr;
        cfms(Pn[(size_t)cc * n + r], Pn[(size_t)c * n + r], Pn[(size_t)cc * n + c]);
      }
      __syncthreads();
    }
    // panel back to global memory
    for (int q = tid; q < jb * m; q += kLuThreads) {
      const int c = q / m, r = q % m;
      A[(size_t)(j0 + c) * n + j0 + r] = Pn[(size_t)c * n + r];
    }
    // 2. the panel's row swaps on the other columns, one thread per column
    for (int col = tid; col < n - jb; col += kLuThreads) {
      const int cg = col < j0 ? col : col + jb;
      double2* Ac = A + (size_t)cg * n;
      for (int c = 0; c < jb; ++c) {
        const int p = piv[j0 + c] - 1;
        if (p != j0 + c) {
          const double2 t = Ac[j0 + c];
          Ac[j0 + c] = Ac[p];
          Ac[p] = t;
        }
      }
    }
    __syncthreads();
    const int n2 = n - j0 - jb;  // columns (and rows) of the trailing matrix
    if (n2 <= 0) break;
    // 3. U12 = L11^-1 A12, one thread per column
    for (int col = tid; col < n2; col += kLuThreads) {
      double2* Ac = A + (size_t)(j0 + jb + col) * n + j0;
      double2 u[kLuNb];
#pragma unroll
      for (int k = 0; k < kLuNb; ++k) u[k] = k < jb ? Ac[k] : make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < kLuNb; ++k)
#pragma unroll
        for (int i = k + 1; i < kLuNb; ++i)
          if (i < jb) cfms(u[i], Pn[(size_t)k * n + i], u[k]);
#pragma unroll
      for (int k = 0; k < kLuNb; ++k)
        if (k < jb) {
          Ac[k] = u[k];
          U[(size_t)k * n + col] = u[k];
        }
    }
    __syncthreads();
    // 4. A22 -= L21 U12 in 64 x 64 tiles, a 4 x 4 complex block per thread
    const int ti = tid % 16, tj = tid / 16;
    for (int r0 = 0; r0 < n2; r0 += 64)
      for (int c0 = 0; c0 < n2; c0 += 64) {
        const int rb = r0 + 4 * ti, cb = c0 + 4 * tj;
        if (rb >= n2 || cb >= n2) continue;
        double2 acc[4][4];
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
          for (int a = 0; a < 4; ++a)
            acc[b][a] = (rb + a < n2 && cb + b < n2) ? A[(size_t)(j0 + jb + cb + b) * n + j0 + jb + rb + a]
                                                     : make_double2(0.0, 0.0);
        for (int k = 0; k < jb; ++k) {
          double2 l[4], u[4];
#pragma unroll
          for (int a = 0; a < 4; ++a) l[a] = rb + a < n2 ? Pn[(size_t)k * n + jb + rb + a] : make_double2(0.0, 0.0);
#pragma unroll
          for (int b = 0; b < 4; ++b) u[b] = cb + b < n2 ? U[(size_t)k * n + cb + b] : make_double2(0.0, 0.0);
#pragma unroll
          for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int a = 0; a < 4; ++a) cfms(acc[b][a], l[a], u[b]);
        }
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
          for (int a = 0; a < 4; ++a)
            if (rb + a < n2 && cb + b < n2) A[(size_t)(j0 + jb + cb + b) * n + j0 + jb + rb + a] = acc[b][a];
      }
    __syncthreads();
  }
}

// Unblocked form (slices larger than the blocked form's shared memory): per
// column the pivot search, the swap across the row, the scaling and the
// rank-1 update of the trailing matrix, all in global memory.
__global__ void __launch_bounds__(256) k_dense_getrf(int n, double2* __restrict__ Ab, int* __restrict__ pivb,
                                                     int* __restrict__ bad) {
  const int s = blockIdx.x;
  double2* A = Ab + (size_t)s * n * n;
  int* piv = pivb + (size_t)s * n;
  __shared__ double sv[256];
  __shared__ int si[256];
  __shared__ int sp;
  __shared__ double2 sd;
  for (int j = 0; j < n; ++j) {
    // pivot search over rows j..n-1 of column j
    double best = -1.0;
    int bi = j;
    for (int i = j + threadIdx.x; i < n; i += blockDim.x) {
      double2 v = A[(size_t)j * n + i];
      double a = fabs(v.x) + fabs(v.y);
      if (a > best) {
        best = a;
        bi = i;
      }
    }
    sv[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) {
        if (sv[threadIdx.x + w] > sv[threadIdx.x] ||
            (sv[threadIdx.x + w] == sv[threadIdx.x] && si[threadIdx.x + w] < si[threadIdx.x])) {
          sv[threadIdx.x] = sv[threadIdx.x + w];
          si[threadIdx.x] = si[threadIdx.x + w];
        }
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      sp = si[0];
      piv[j] = sp + 1;
      if (!(sv[0] > 0.0)) atomicMin(bad, s);
    }
    __syncthreads();
    const int p = sp;
    if (!(sv[0] > 0.0)) return;
    if (p != j)
      for (int c = threadIdx.x; c < n; c += blockDim.x) {
        double2 t = A[(size_t)c * n + j];
        A[(size_t)c * n + j] = A[(size_t)c * n + p];
        A[(size_t)c * n + p] = t;
      }
    __syncthreads();
    if (threadIdx.x == 0) sd = A[(size_t)j * n + j];
    __syncthreads();
    const double2 d = sd;
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) A[(size_t)j * n + i] = cdiv(A[(size_t)j * n + i], d);
    __syncthreads();
    const int m = n - j - 1;
    for (long long q = threadIdx.x; q < (long long)m * m; q += blockDim.x) {
      const int c = j + 1 + (int)(q / m), i = j + 1 + (int)(q % m);
      double2 l = A[(size_t)j * n + i], u = A[(size_t)c * n + j];
      double2 pr = cmul(l, u);
      double2& t = A[(size_t)c * n + i];
      t.x -= pr.x;
      t.y -= pr.y;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_dense_getrs(int n, const double2* __restrict__ Ab,
                                                     const int* __restrict__ pivb, double2* __restrict__ Bb) {
  const int s = blockIdx.x;
  const double2* A = Ab + (size_t)s * n * n;
  const int* piv = pivb + (size_t)s * n;
  double2* b = Bb + (size_t)s * n;
  if (threadIdx.x == 0)
    for (int j = 0; j < n; ++j) {
      int p = piv[j] - 1;
      if (p != j) {
        double2 t = b[j];
        b[j] = b[p];
        b[p] = t;
      }
    }
  __syncthreads();
  for (int j = 0; j < n; ++j) {  // L y = b (unit lower)
    const double2 bj = b[j];
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      double2 pr = cmul(A[(size_t)j * n + i], bj);
      b[i].x -= pr.x;
      b[i].y -= pr.y;
    }
    __syncthreads();
  }
  for (int j = n - 1; j >= 0; --j) {  // U x = y
    __shared__ double2 xj;
    if (threadIdx.x == 0) {
      xj = cdiv(b[j], A[(size_t)j * n + j]);
      b[j] = xj;
    }
    __syncthreads();
    const double2 x = xj;
    for (int i = threadIdx.x; i < j; i += blockDim.x) {
      double2 pr = cmul(A[(size_t)j * n + i], x);
      b[i].x -= pr.x;
      b[i].y -= pr.y;
    }
    __syncthreads();
  }
}

// first singular slice of the last factorisation (INT_MAX: none); factor
// calls are synchronous and serialised by g_lu_mutex, so one flag per device
// serves every call
__device__ int g_lu_bad;
std::mutex g_lu_mutex;

}  // namespace

extern "C" {

tb_status tb_batched_lu_factor(tb_context* ctx, int n, int batch, double* A, int* piv, int* bad_slice) {
  if (!ctx || !A || !piv || n < 1 || batch < 1) return TB_EINVAL;
  std::lock_guard<std::mutex> lock(g_lu_mutex);
  const int init = 0x7fffffff;
  int* dbad = nullptr;
  cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&dbad), g_lu_bad);
  if (e == cudaSuccess) e = cudaMemcpy(dbad, &init, sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    if (n <= kLuBlockedMaxN) {
      const size_t smem = lu_blocked_smem(n);
      e = cudaFuncSetAttribute(k_dense_getrf_blocked, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess)
        k_dense_getrf_blocked<<<batch, kLuThreads, smem>>>(n, reinterpret_cast<double2*>(A), piv, dbad);
    } else {
      k_dense_getrf<<<batch, 256>>>(n, reinterpret_cast<double2*>(A), piv, dbad);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  int bad = init;
  if (e == cudaSuccess) e = cudaMemcpy(&bad, dbad, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    tb::set_context_error(ctx, std::string("batched LU factor: ") + cudaGetErrorString(e));
    return TB_ECUDA;
  }
  if (bad != init) {
    if (bad_slice) *bad_slice = bad;
    tb::set_context_error(ctx, "singular matrix in batched LU at slice " + std::to_string(bad));
    return TB_ESINGULAR;
  }
  if (bad_slice) *bad_slice = -1;
  return TB_OK;
}

tb_status tb_batched_lu_solve(tb_context* ctx, int n, int batch, const double* A, const int* piv, double* B) {
  if (!ctx || !A || !piv || !B || n < 1 || batch < 1) return TB_EINVAL;
  k_dense_getrs<<<batch, 256>>>(n, reinterpret_cast<const double2*>(A), piv, reinterpret_cast<double2*>(B));
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    tb::set_context_error(ctx, std::string("batched LU solve: ") + cudaGetErrorString(e));
    return TB_ECUDA;
  }
  return TB_OK;
}

}  // extern "C"
