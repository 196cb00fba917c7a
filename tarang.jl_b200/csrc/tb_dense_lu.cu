// Batched dense complex LU with partial pivoting, one CTA per matrix.
//
// Drop-in for BatchedDenseLU (src/tools/batched_matsolvers.jl:57-123), whose
// CUDA methods call getrf/getrs strided-batched
// (ext/cuda/batched_matsolvers.jl:80-125): A is column-major n x n complex128
// per slice and is overwritten by L (unit, below the diagonal) and U; ipiv is
// 1-based LAPACK style (row i was swapped with row ipiv[i]).  A slice with an
// exactly zero pivot is reported, never silently solved.
#include <cuda_runtime.h>

#include "tb_internal.h"

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

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

}  // namespace

extern "C" {

tb_status tb_batched_lu_factor(tb_context* ctx, int n, int batch, double* A, int* piv, int* bad_slice) {
  if (!ctx || !A || !piv || n < 1 || batch < 1) return TB_EINVAL;
  int* dbad = nullptr;
  if (cudaMalloc(&dbad, sizeof(int)) != cudaSuccess) return TB_ENOMEM;
  int init = 0x7fffffff;
  cudaMemcpy(dbad, &init, sizeof(int), cudaMemcpyHostToDevice);
  k_dense_getrf<<<batch, 256>>>(n, reinterpret_cast<double2*>(A), piv, dbad);
  cudaError_t e = cudaGetLastError();
  int bad = init;
  if (e == cudaSuccess) e = cudaMemcpy(&bad, dbad, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(dbad);
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
