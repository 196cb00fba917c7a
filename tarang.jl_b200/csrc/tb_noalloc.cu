// Plan-free 3/2-dealiased product that allocates no device memory.
//
// Who needs this: callers that own every device buffer themselves and may not
// call cudaMalloc from a foreign library -- a host runtime with its own device
// memory pool (CUDA.jl's allocator, a framework's caching allocator) or a
// process that must not grow its device footprint after start-up.  They pass
// their own input and output buffers; the only other device memory the
// product needs, the FFT twiddle tables, lives in the file-scope array below.
//
// Limits and sharing:
//   * the array holds kNoAllocTwiddles complex entries (80 KiB), enough for
//     Nx <= 2048 (twiddles of length Nx and of the padded length M <= 3072);
//     larger Nx is rejected with TB_ENOTSUPPORTED;
//   * every GPU that loads the library holds one copy until the process exits;
//   * all calls share it and each call rewrites it for its own Nx, so calls
//     that overlap on the GPU (from several host threads or streams) race;
//   * the first call on a device resolves the array's device address with
//     that device current (once per device); make that first call before any
//     stream capture;
//   * the kernels run on the legacy default stream, which does not wait for
//     work on non-blocking streams (CUDA.jl task streams, a framework's side
//     streams): the caller synchronises the stream that wrote a_grid and
//     b_grid before the call.  The call returns when out_grid is written.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "tb_internal.h"
#include "tb_kernels.cuh"

namespace {

constexpr int kNoAllocMaxNx = 2048;
constexpr int kNoAllocMaxM = 3072;
constexpr int kNoAllocTwiddles = kNoAllocMaxNx + kNoAllocMaxM;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double2 g_noalloc_twiddles[kNoAllocTwiddles];

std::mutex g_setup_mu;
double2* g_twiddle_ptr[kMaxDevices] = {};

// tw[t] = exp(-2 pi i t / n), t < n (same table the plan path uploads)
__global__ void k_noalloc_twiddles(double2* tw, int n) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(-2.0 * (double)t / (double)n, &s, &c);
    tw[t] = make_double2(c, s);
  }
}

tb_status setup_device(int device, double2** out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (g_twiddle_ptr[device]) {
    *out = g_twiddle_ptr[device];
    return TB_OK;
  }
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_twiddles);
  if (e != cudaSuccess) {
    tb::set_thread_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    return TB_ECUDA;
  }
  e = tb::set_transform_smem_limits(227 * 1024);
  if (e != cudaSuccess) {
    tb::set_thread_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    return TB_ECUDA;
  }
  g_twiddle_ptr[device] = static_cast<double2*>(p);
  *out = g_twiddle_ptr[device];
  return TB_OK;
}

}  // namespace

extern "C" {

tb_status tb_dealiased_multiply_noalloc(int device, int Nx, int Nz, const double* a_grid, const double* b_grid,
                                        double* out_grid) {
  if (!a_grid || !b_grid || !out_grid) {
    tb::set_thread_error("a_grid, b_grid and out_grid must be non-null device pointers");
    return TB_EINVAL;
  }
  if (Nz < 1) {
    tb::set_thread_error("Nz must be >= 1");
    return TB_EINVAL;
  }
  if (device < 0 || device >= kMaxDevices) {
    tb::set_thread_error("device index out of range");
    return TB_EINVAL;
  }
  if (Nx < 6 || Nx % 2) {
    tb::set_thread_error("Nx must be even and >= 6");
    return TB_EINVAL;
  }
  int M = (int)std::ceil(1.5 * Nx);
  if (M % 2) ++M;
  if (Nx > kNoAllocMaxNx || M > kNoAllocMaxM) {
    tb::set_thread_error("Nx above the no-allocation limit of 2048");
    return TB_ENOTSUPPORTED;
  }
  tb::FftPlan fpN{}, fpM{};
  if (!tb::make_fft_plan(Nx, &fpN) || !tb::make_fft_plan(M, &fpM)) {
    tb::set_thread_error("Nx must be of the form 2^a 3^b");
    return TB_ENOTSUPPORTED;
  }
  int prev = 0;
  cudaGetDevice(&prev);
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    tb::set_thread_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return TB_ECUDA;
  }
  double2* tw = nullptr;
  tb_status st = setup_device(device, &tw);
  if (st == TB_OK) {
    double2* twN = tw;
    double2* twM = tw + kNoAllocMaxNx;
    k_noalloc_twiddles<<<(Nx + 255) / 256, 256>>>(twN, Nx);
    k_noalloc_twiddles<<<(M + 255) / 256, 256>>>(twM, M);
    tb::launch_x_dealias_mul(a_grid, b_grid, out_grid, Nz, Nx, M, fpN, twN, fpM, twM, 0);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
      tb::set_thread_error(std::string("dealiased multiply: ") + cudaGetErrorString(e));
      st = TB_ECUDA;
    }
  }
  cudaSetDevice(prev);
  return st;
}

}  // extern "C"
