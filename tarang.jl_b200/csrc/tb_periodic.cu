// Transforms of a doubly periodic RealFourier x RealFourier domain in FP64,
// the grid <-> coefficient conversion behind field["g"] on a PeriodicDomain
// (src/extras/quick_domains.jl:33-58; conventions of
// src/core/transforms/transform_fourier.jl:473-590):
//   forward  c = fft_y(rfft_x(g)), unnormalised;
//   backward g = irfft_x(ifft_y(c)) with 1/(Nx Ny), the irfft ignoring the
//            imaginary parts of the kx = 0 and Nyquist bins.
// Grid (Ny, Nx) real, x fastest; coefficients (Ny, Nx/2+1) complex, kx fastest,
// ky in FFT order.  The row transforms are the library's x-direction kernels
// and the column FFT the y-direction kernel of the 3D path.
#include <cuda_runtime.h>

#include <memory>

#include "tb_internal.h"
#include "tb_plan.h"

using namespace tb;

struct tb_periodic {
  tb_context* ctx = nullptr;
  int Nx = 0, Ny = 0, Kx = 0;
  FftPlan fpN{}, fpNy{};
  DevBuf twN, ptwNy;   // x row twiddles, per-pass twiddles of the Ny plan
  DevBuf grid, coeff;  // device staging for host callers
  cudaStream_t st = nullptr;
  ~tb_periodic() {
    if (st) cudaStreamDestroy(st);
  }
};

namespace {

void forward(tb_periodic* T, const double* grid, double2* coeff) {
  launch_x_rfft(grid, coeff, T->Ny, T->Nx, T->fpN, T->twN.as<double2>(), T->st);
  periodic_ycols(coeff, T->Ny, T->Kx, T->fpNy, T->ptwNy.as<double2>(), -1, T->st);
}

void backward(tb_periodic* T, const double2* coeff, double* grid) {
  // the column FFT runs in place, so it works on a copy of the caller's data
  double2* t = T->coeff.as<double2>();
  if (t != coeff)
    TB_CUDA_TRY(cudaMemcpyAsync(t, coeff, T->coeff.bytes, cudaMemcpyDeviceToDevice, T->st));
  periodic_ycols(t, T->Ny, T->Kx, T->fpNy, T->ptwNy.as<double2>(), +1, T->st);
  launch_x_irfft(t, grid, T->Ny, T->Nx, T->fpN, T->twN.as<double2>(), T->st);
}

}  // namespace

extern "C" {

tb_status tb_periodic_create(tb_context* ctx, int Nx, int Ny, tb_periodic** out) {
  if (!ctx || !out) return TB_EINVAL;
  *out = nullptr;
  return guarded(ctx, [&] {
    TB_REQUIRE(Nx >= 8 && Ny >= 8 && Nx % 2 == 0 && Ny % 2 == 0, TB_EINVAL, "Nx, Ny must be even and >= 8");
    TB_REQUIRE(Nx <= 2048 && Ny <= 2048, TB_ENOTSUPPORTED, "Nx, Ny above 2048");
    auto T = std::make_unique<tb_periodic>();
    T->ctx = ctx;
    T->Nx = Nx;
    T->Ny = Ny;
    T->Kx = Nx / 2 + 1;
    TB_REQUIRE(make_fft_plan(Nx, &T->fpN) && make_fft_plan(Ny, &T->fpNy), TB_ENOTSUPPORTED,
               "Nx, Ny must be of the form 2^a 3^b");
    TB_CUDA_TRY(cudaSetDevice(ctx->device));
    TB_CUDA_TRY(set_transform_smem_limits(227 * 1024));
    TB_CUDA_TRY(create_work_stream(&T->st));
    upload(T->twN, host_twiddles(Nx));
    upload(T->ptwNy, host_pass_twiddles(T->fpNy));
    T->grid.alloc((size_t)Ny * Nx * sizeof(double));
    T->coeff.alloc((size_t)Ny * T->Kx * sizeof(double2));
    *out = T.release();
  });
}

tb_status tb_periodic_destroy(tb_periodic* T) {
  if (!T) return TB_OK;
  cudaStreamSynchronize(T->st);
  delete T;
  return TB_OK;
}

tb_status tb_periodic_forward(tb_periodic* T, const double* grid, double* coeff, int where) {
  if (!T || !grid || !coeff) return TB_EINVAL;
  return guarded(T->ctx, [&] {
    TB_CUDA_TRY(cudaSetDevice(T->ctx->device));
    if (where == TB_DEVICE) {
      forward(T, grid, reinterpret_cast<double2*>(coeff));
    } else {
      TB_CUDA_TRY(cudaMemcpyAsync(T->grid.p, grid, T->grid.bytes, cudaMemcpyHostToDevice, T->st));
      forward(T, T->grid.as<double>(), T->coeff.as<double2>());
      TB_CUDA_TRY(cudaMemcpyAsync(coeff, T->coeff.p, T->coeff.bytes, cudaMemcpyDeviceToHost, T->st));
    }
    TB_CUDA_TRY(cudaGetLastError());
    TB_CUDA_TRY(cudaStreamSynchronize(T->st));
  });
}

tb_status tb_periodic_backward(tb_periodic* T, const double* coeff, double* grid, int where) {
  if (!T || !grid || !coeff) return TB_EINVAL;
  return guarded(T->ctx, [&] {
    TB_CUDA_TRY(cudaSetDevice(T->ctx->device));
    if (where == TB_DEVICE) {
      backward(T, reinterpret_cast<const double2*>(coeff), grid);
    } else {
      TB_CUDA_TRY(cudaMemcpyAsync(T->coeff.p, coeff, T->coeff.bytes, cudaMemcpyHostToDevice, T->st));
      backward(T, T->coeff.as<double2>(), T->grid.as<double>());
      TB_CUDA_TRY(cudaMemcpyAsync(grid, T->grid.p, T->grid.bytes, cudaMemcpyDeviceToHost, T->st));
    }
    TB_CUDA_TRY(cudaGetLastError());
    TB_CUDA_TRY(cudaStreamSynchronize(T->st));
  });
}

}  // extern "C"
