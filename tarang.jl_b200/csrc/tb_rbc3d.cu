// 3D Rayleigh-Benard program: RealFourier x, RealFourier y, ChebyshevT z
// (ChannelDomain3D, src/extras/quick_domains.jl:124-143), equations of
// test/test_subproblem_rk.jl:50-57 with a 3-component velocity.
//
// Fourier modes m = ix * Ny + iy: kx = 2 pi/Lx ix (ix = 0..Nx/2, Nyquist
// +Nx/2), ky = 2 pi/Ly [0..Ny/2-1, -Ny/2..-1] (basis_wavenumbers.jl:68-108).
// The horizontal velocity is held along / across the wavevector,
//   u_par = (kx u_x + ky u_y)/|k|,  u_perp = (-ky u_x + kx u_y)/|k|
// (u_par = u_x, u_perp = u_y at k = 0); the momentum rows rotate the same way.
// Then the pressure and continuity couple only (b, u_par, u_z, p), which is the
// 2D system with kx replaced by |k|, and u_perp is a Helmholtz problem of its
// own; both are exact row/column rotations of the reference's per-mode
// Cartesian system (subproblem_matrix_build.jl:11-309), so the solution is
// unchanged.
//
// RHS  F_f = -(u_x d_x f + u_y d_y f + u_z d_z f),  f = b, u_x, u_y, u_z,
// following the lazy evaluator (lazy_rhs.jl:712-1336) and the 3/2 padded
// product along both Fourier axes (nonlinear_padding.jl:86-103, 164-443):
//   k3_prep   state -> Cartesian b, u_x, u_y, u_z (RHS precision)
//   GEMM      Chebyshev backward: values and z-derivatives as even/odd half
//             planes over the z grid (tensor-core DMMA in FP64, SIMT in FP32)
//   k3_yinv   per (kx, z pair): value, d_y and d_z of each field with the grid
//             round trip's Hermitian projection of the kx = 0 / Nyquist columns,
//             the x Nyquist split, y padding with the Nyquist split, 12 inverse
//             FFTs along y
//   k3_xpass  per (y rows, z): d_x from the x bins, 15 real inverse FFTs along
//             x (8 packed), the 4 products, 2 packed forward FFTs, x truncation
//             with the Nyquist fold
//   k3_yfwd   per (kx, z): 4 forward FFTs along y, Nyquist fold, truncation,
//             scale, rotation of the momentum rows
//   GEMM      Chebyshev forward into C^(2) rows (S fwd) of the stage vector.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "tb_fft.cuh"
#include "tb_internal.h"
#include "tb_kernels.cuh"
#include "tb_plan.h"

namespace tb {
namespace {

namespace F = tb::fftg;

constexpr int kR3Threads = 256;

struct R3Args {
  int Nx, Ny, Nz, Kx, Mx, My, Nk, H;
  double kx0, ky0;
  FftPlan fpx, fpy;
  int nptx, npty;
};

__device__ __forceinline__ int ky_index(int iy, int Ny) { return iy < Ny / 2 ? iy : iy - Ny; }

// Rotation (cx, cy) = (kx, ky)/|k| of mode (ix, iy); (1, 0) at k = 0.
__device__ __forceinline__ void rot_of(const R3Args& a, int ix, int iy, double& cx, double& cy) {
  const double kx = a.kx0 * ix, ky = a.ky0 * ky_index(iy, a.Ny);
  const double kk = sqrt(kx * kx + ky * ky);
  if (kk > 0.0) {
    cx = kx / kk;
    cy = ky / kk;
  } else {
    cx = 1.0;
    cy = 0.0;
  }
}

// State (b, u_par, u_z, p, u_perp planes) -> Cartesian (b, u_x, u_y, u_z) in
// the RHS precision.  Grid (ceil(Nk/256), Nz).
template <class C>
__global__ void __launch_bounds__(256) k3_prep(R3Args a, const double2* __restrict__ X, C* __restrict__ Xc) {
  using T = typename F::Real<C>::type;
  const int z = blockIdx.y, m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.Nk) return;
  const size_t plane = (size_t)a.Nz * a.Nk, i = (size_t)z * a.Nk + m;
  double cx, cy;
  rot_of(a, m / a.Ny, m % a.Ny, cx, cy);
  const double2 b = X[i], up = X[plane + i], uz = X[2 * plane + i], uq = X[4 * plane + i];
  Xc[i] = F::mk<C>((T)b.x, (T)b.y);
  Xc[plane + i] = F::mk<C>((T)(cx * up.x - cy * uq.x), (T)(cx * up.y - cy * uq.y));
  Xc[2 * plane + i] = F::mk<C>((T)(cy * up.x + cx * uq.x), (T)(cy * up.y + cx * uq.y));
  Xc[3 * plane + i] = F::mk<C>((T)uz.x, (T)uz.y);
}

// The FP32 kernels at the 384-point padded length run the two-pass register
// transform (natural-order buffers, kLen384Buf apart, twiddle table w^k for
// k < 384); other compiled lengths the Stockham plan with constant strides,
// the rest the runtime plan (both on swizzled buffers, per-pass twiddles).
template <class C, int M>
constexpr bool kReg384 = std::is_same<C, float2>::value && M == 384;

template <class C, int M>
__device__ __forceinline__ int bidx(int i) {
  if constexpr (kReg384<C, M>)
    return i;
  else
    return F::sidx<C>(i);
}

template <class C, int M>
__host__ __device__ constexpr int buf_len(int m) {
  return kReg384<C, M> ? F::kLen384Buf : F::pad_swz<C>(m);
}

// Batched FFT of nb buffers.
template <int N, class C>
__device__ __forceinline__ C* fftb(C* a, C* b, int nb, int stride, const FftPlan& fp, const C* __restrict__ pt,
                                   int sign) {
  if constexpr (kReg384<C, N>)
    return F::fft384_batch(a, b, nb, stride, pt, sign);
  else if constexpr (N > 0)
    return F::fft_batch_ct<N>(a, b, nb, stride, pt, sign);
  else
    return F::fft_batch<true>(a, b, nb, stride, fp, pt, sign);
}

// Per (kx column ix, z pair j / Nz-1-j).  G: 16 half planes (field f, w) at
// G + (4 f + w) hplane, w = 0 even values, 1 odd values, 2 even d_z, 3 odd d_z,
// element (j, m).  Output mix[z][q][ix][y], q = 3 f + kind (value, d_y, d_z).
template <class C, int MY>
__global__ void __launch_bounds__(kR3Threads) k3_yinv(R3Args a, const C* __restrict__ G, const C* __restrict__ pty,
                                                       C* __restrict__ mix) {
  using T = typename F::Real<C>::type;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C* sm = reinterpret_cast<C*>(sm_raw);
  const int Ny = a.Ny, My = MY > 0 ? MY : a.My, ix = blockIdx.x, j = blockIdx.y;
  const int Ms = buf_len<C, MY>(My);
  C* stg = sm;                    // [16][Ny]
  C* A = stg + 16 * Ny;           // [12][Ms]
  C* B = A + 12 * Ms;             // [12][Ms]
  C* pt = B + 12 * Ms;            // [npty]
  const size_t hplane = (size_t)a.H * a.Nk;
  for (int t = threadIdx.x; t < a.npty; t += blockDim.x) pt[t] = pty[t];
  for (int t = threadIdx.x; t < 16 * Ny; t += blockDim.x) {
    const int q = t / Ny, iy = t - q * Ny;
    stg[t] = G[(size_t)q * hplane + (size_t)j * a.Nk + (size_t)ix * Ny + iy];
  }
  __syncthreads();
  const bool edge = (ix == 0) || (2 * ix == a.Nx);  // columns whose grid round trip is Hermitian
  const T xs = (2 * ix == a.Nx) ? (T)0.5 : (T)1.0;  // even-N Nyquist split along x
  const int hy = Ny / 2, gap = My - Ny - 1;          // y bins hy+1 .. My-hy-1 stay zero
  for (int lev = 0; lev < 2; ++lev) {
    const int zl = lev ? a.Nz - 1 - j : j;
    // value (kind 0, 1) or z-derivative (kind 2) of field f at grid level zl
    auto base = [&](int f, int kind, int iy) -> C {
      const C e = stg[(4 * f + (kind == 2 ? 2 : 0)) * Ny + iy];
      const C o = stg[(4 * f + (kind == 2 ? 3 : 1)) * Ny + iy];
      if (kind == 2) return lev ? F::sub(o, e) : F::add(e, o);
      return lev ? F::sub(e, o) : F::add(e, o);
    };
    for (int t = threadIdx.x; t < 12 * gap; t += blockDim.x) {
      const int q = t / gap, y = hy + 1 + (t - q * gap);
      A[(size_t)q * Ms + bidx<C, MY>(y)] = F::mk<C>((T)0, (T)0);
    }
    for (int t = threadIdx.x; t < 12 * Ny; t += blockDim.x) {
      const int q = t / Ny, iy = t - q * Ny;
      const int f = q / 3, kind = q - 3 * f;
      // the factor is a derivative of the field's grid round trip, so the
      // projection comes first (it differs from projecting i ky v at the
      // self-paired ky = -Ny/2 mode)
      C v = base(f, kind, iy);
      if (edge) {
        const C w = base(f, kind, (Ny - iy) % Ny);
        v = F::mk<C>((T)0.5 * (v.x + w.x), (T)0.5 * (v.y - w.y));
      }
      if (kind == 1) {
        const T kyv = (T)(a.ky0 * ky_index(iy, Ny));
        v = F::mk<C>(-kyv * v.y, kyv * v.x);  // i ky v
      }
      v = F::scale(v, xs);
      C* col = A + (size_t)q * Ms;
      if (iy < hy) {
        col[bidx<C, MY>(iy)] = v;
      } else if (iy == hy) {
        const C h = F::scale(v, (T)0.5);
        col[bidx<C, MY>(hy)] = h;
        col[bidx<C, MY>(My - hy)] = h;
      } else {
        col[bidx<C, MY>(My - Ny + iy)] = v;
      }
    }
    __syncthreads();
    C* R = fftb<MY>(A, B, 12, Ms, a.fpy, pt, +1);
    for (int t = threadIdx.x; t < 12 * My; t += blockDim.x) {
      const int q = t / My, y = t - q * My;
      mix[(((size_t)zl * 12 + q) * a.Kx + ix) * My + y] = R[(size_t)q * Ms + bidx<C, MY>(y)];
    }
    __syncthreads();
  }
}

// Per (RR consecutive padded y rows, z level).  mix[z][q][kx][y] ->
// pm[z][f][kx][y] (f = b, u_x, u_y, u_z; kx < Kx, Nyquist folded).
// Factors on the x grid (15 real, packed in pairs a + i b): 0 u_x, 1 u_y,
// 2 u_z, 3..6 d_x f, 7..10 d_y f, 11..14 d_z f (f = b, u_x, u_y, u_z).
template <class C, int RR, int MX>
__global__ void __launch_bounds__(RR == 4 ? 2 * kR3Threads : kR3Threads) k3_xpass(R3Args a, const C* __restrict__ mix, const C* __restrict__ ptx,
                                                        C* __restrict__ pm) {
  using T = typename F::Real<C>::type;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C* sm = reinterpret_cast<C*>(sm_raw);
  const int Mx = MX > 0 ? MX : a.Mx, Kx = a.Kx, My = a.My, hN = a.Nx / 2;
  const int y0 = blockIdx.x * RR, z = blockIdx.y;
  const int Ms = buf_len<C, MX>(Mx);
  constexpr int NB = 8 * RR;
  C* Z = sm;              // [NB][Ms]
  C* S = Z + NB * Ms;     // [NB][Ms]
  C* pt = S + NB * Ms;    // [nptx]
  for (int t = threadIdx.x; t < a.nptx; t += blockDim.x) pt[t] = ptx[t];
  // 1. half spectra of the 15 factors, [r][factor][k < Kx], staged in S (DC and
  // Nyquist kept real, as the factors' own irfft on Nx points does)
  C* hs = S;
  for (int t = threadIdx.x; t < 12 * Kx * RR; t += blockDim.x) {
    const int r = t % RR, rest = t / RR;
    const int k = rest % Kx, q = rest / Kx;
    C v = mix[(((size_t)z * 12 + q) * Kx + k) * My + y0 + r];
    const bool edge = (k == 0 || k == hN);
    if (edge) v.y = (T)0;
    const int f = q / 3, kind = q - 3 * f;
    C* row = hs + (size_t)r * 15 * Kx;
    if (kind == 0) {
      if (f > 0) row[(size_t)(f - 1) * Kx + k] = v;
      const T kk = (T)(a.kx0 * k);
      row[(size_t)(3 + f) * Kx + k] = edge ? F::mk<C>((T)0, (T)0) : F::mk<C>(-kk * v.y, kk * v.x);  // i kx v
    } else {
      row[(size_t)((kind == 1 ? 7 : 11) + f) * Kx + k] = v;
    }
  }
  __syncthreads();
  // 2. packed spectra: Z[p] = spectrum of factor 2p + i factor 2p+1 on Mx points
  const int nh = Mx / 2 + 1;
  for (int t = threadIdx.x; t < RR * 8 * nh; t += blockDim.x) {
    const int r = t % RR, rest = t / RR;
    const int k = rest % nh, p = rest / nh;
    const C* row = hs + (size_t)r * 15 * Kx;
    const C A = k < Kx ? row[(size_t)(2 * p) * Kx + k] : F::mk<C>((T)0, (T)0);
    const C B = (k < Kx && p < 7) ? row[(size_t)(2 * p + 1) * Kx + k] : F::mk<C>((T)0, (T)0);
    C* dst = Z + (size_t)(r * 8 + p) * Ms;
    // spectrum of a + i b: A + i B at k, conj(A) + i conj(B) at Mx - k
    dst[bidx<C, MX>(k)] = F::mk<C>(A.x - B.y, A.y + B.x);
    if (k > 0 && k < Mx / 2) dst[bidx<C, MX>(Mx - k)] = F::mk<C>(A.x + B.y, -A.y + B.x);
  }
  __syncthreads();
  C* Rg = fftb<MX>(Z, S, NB, Ms, a.fpx, pt, +1);
  C* W = (Rg == Z) ? S : Z;
  for (int t = threadIdx.x; t < RR * Mx; t += blockDim.x) {
    const int r = t / Mx, x = t - r * Mx;
    const int i = bidx<C, MX>(x);
    const C* g = Rg + (size_t)r * 8 * Ms;
    const C z0 = g[i], z1 = g[Ms + i], z2 = g[2 * Ms + i], z3 = g[3 * Ms + i];
    const C z4 = g[4 * Ms + i], z5 = g[5 * Ms + i], z6 = g[6 * Ms + i], z7 = g[7 * Ms + i];
    const T ux = z0.x, uy = z0.y, uz = z1.x;
    const T pb = ux * z1.y + uy * z3.y + uz * z5.y;   // d_x b, d_y b, d_z b
    const T pu = ux * z2.x + uy * z4.x + uz * z6.x;   // d_x u_x, d_y u_x, d_z u_x
    const T pv = ux * z2.y + uy * z4.y + uz * z6.y;   // d_x u_y, d_y u_y, d_z u_y
    const T pw = ux * z3.x + uy * z5.x + uz * z7.x;   // d_x u_z, d_y u_z, d_z u_z
    W[(size_t)(2 * r) * Ms + i] = F::mk<C>(pb, pu);
    W[(size_t)(2 * r + 1) * Ms + i] = F::mk<C>(pv, pw);
  }
  __syncthreads();
  C* Fq = fftb<MX>(W, Rg, 2 * RR, Ms, a.fpx, pt, -1);
  for (int t = threadIdx.x; t < RR * 2 * Kx; t += blockDim.x) {
    const int r = t % RR, rest = t / RR;
    const int k = rest % Kx, h = rest / Kx;
    const C* buf = Fq + (size_t)(2 * r + h) * Ms;
    const C c = buf[bidx<C, MX>(k)], cm = buf[bidx<C, MX>((Mx - k) % Mx)];
    // first: (c + conj(cm))/2, second: (c - conj(cm))/(2i)
    C o1 = F::mk<C>((T)0.5 * (c.x + cm.x), (T)0.5 * (c.y - cm.y));
    C o2 = F::mk<C>((T)0.5 * (c.y + cm.y), (T)-0.5 * (c.x - cm.x));
    if (k == 0) {
      o1.y = (T)0;
      o2.y = (T)0;
    } else if (k == hN) {  // fold of the -Nx/2 image: 2 Re
      o1 = F::mk<C>((T)2 * o1.x, (T)0);
      o2 = F::mk<C>((T)2 * o2.x, (T)0);
    }
    pm[(((size_t)z * 4 + 2 * h) * Kx + k) * My + y0 + r] = o1;
    pm[(((size_t)z * 4 + 2 * h + 1) * Kx + k) * My + y0 + r] = o2;
  }
}

// Per (kx column ix, z level): forward FFTs along y of the 4 products, y
// Nyquist fold and truncation, F = -P / (Nx Ny Mx My), rotation of the
// horizontal momentum rows; out[f][z][m] for f = b, u_par, u_z, u_perp.
template <class C, int MY>
__global__ void __launch_bounds__(kR3Threads) k3_yfwd(R3Args a, const C* __restrict__ pm, const C* __restrict__ pty,
                                                       C* __restrict__ out) {
  using T = typename F::Real<C>::type;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C* sm = reinterpret_cast<C*>(sm_raw);
  const int Ny = a.Ny, My = MY > 0 ? MY : a.My, ix = blockIdx.x, z = blockIdx.y;
  const int Ms = buf_len<C, MY>(My);
  C* A = sm;
  C* B = A + 4 * Ms;
  C* pt = B + 4 * Ms;
  for (int t = threadIdx.x; t < a.npty; t += blockDim.x) pt[t] = pty[t];
  for (int t = threadIdx.x; t < 4 * My; t += blockDim.x) {
    const int f = t / My, y = t - f * My;
    A[(size_t)f * Ms + bidx<C, MY>(y)] = pm[(((size_t)z * 4 + f) * a.Kx + ix) * My + y];
  }
  __syncthreads();
  const C* Q = fftb<MY>(A, B, 4, Ms, a.fpy, pt, -1);
  const double sc = -1.0 / ((double)a.Nx * (double)Ny * (double)a.Mx * (double)My);
  const size_t plane = (size_t)a.Nz * a.Nk;
  for (int iy = threadIdx.x; iy < Ny; iy += blockDim.x) {
    double2 v[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const C* col = Q + (size_t)f * Ms;
      C r;
      if (2 * iy < Ny) {
        r = col[bidx<C, MY>(iy)];
      } else if (2 * iy == Ny) {
        r = F::add(col[bidx<C, MY>(Ny / 2)], col[bidx<C, MY>(My - Ny / 2)]);
      } else {
        r = col[bidx<C, MY>(My - Ny + iy)];
      }
      v[f] = make_double2(sc * (double)r.x, sc * (double)r.y);
    }
    double cx, cy;
    rot_of(a, ix, iy, cx, cy);
    const size_t e = (size_t)z * a.Nk + (size_t)ix * Ny + iy;
    out[e] = F::mk<C>((T)v[0].x, (T)v[0].y);
    out[plane + e] = F::mk<C>((T)(cx * v[1].x + cy * v[2].x), (T)(cx * v[1].y + cy * v[2].y));
    out[2 * plane + e] = F::mk<C>((T)v[3].x, (T)v[3].y);
    out[3 * plane + e] = F::mk<C>((T)(-cy * v[1].x + cx * v[2].x), (T)(-cy * v[1].y + cx * v[2].y));
  }
}

// L delta for the Hermitian projection of the kx = 0 and kx = Nx/2 planes
// (the grid round trip of the stage fields, step_subproblem_rk.jl gathers
// through coeff_data!), subtracted from the stage L X:
//   delta = (X(m) - conj X(m'))/2 in Cartesian components, m' = (ix, -ky),
//   cont  i kx S d_ux + i ky S d_uy + SD d_uz
//   b     kappa (k^2 S - D2) d_b
//   mom   nu (k^2 S - D2) d_u  (- S d_b in z), rotated to (par, perp) rows.
// One thread per (row k, plane, iy): grid (ceil(2 Ny / 128), Nz).
// MASS: the same projection for M X of the multistep history (M delta: S d_b,
// S d_u rotated; continuity rows 0).
template <bool MASS>
__global__ void __launch_bounds__(128) k3_lx_project(R3Args a, double2* __restrict__ LX, const double2* __restrict__ X,
                                                     const double* __restrict__ s3, double s, double kappa, double nu,
                                                     double beta) {
  const int k = blockIdx.y, t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * a.Ny) return;
  const int Ny = a.Ny, Nz = a.Nz, Nk = a.Nk;
  const int ix = (t < Ny) ? 0 : a.Kx - 1, iy = t % Ny;
  const int iyp = (Ny - iy) % Ny;
  const int m = ix * Ny + iy, mp = ix * Ny + iyp;
  const size_t plane = (size_t)Nz * Nk;
  double cx, cy, px, py;
  rot_of(a, ix, iy, cx, cy);
  rot_of(a, ix, iyp, px, py);
  // Cartesian delta of field f (0 b, 1 u_x, 2 u_y, 3 u_z) at row kk
  auto delta = [&](int f, int kk) -> double2 {
    if (kk >= Nz) return make_double2(0.0, 0.0);
    const size_t i = (size_t)kk * Nk + m, ip = (size_t)kk * Nk + mp;
    double2 v, w;
    if (f == 0) {
      v = X[i];
      w = X[ip];
    } else if (f == 3) {
      v = X[2 * plane + i];
      w = X[2 * plane + ip];
    } else {
      const double2 up = X[plane + i], uq = X[4 * plane + i];
      const double2 wp = X[plane + ip], wq = X[4 * plane + ip];
      if (f == 1) {
        v = make_double2(cx * up.x - cy * uq.x, cx * up.y - cy * uq.y);
        w = make_double2(px * wp.x - py * wq.x, px * wp.y - py * wq.y);
      } else {
        v = make_double2(cy * up.x + cx * uq.x, cy * up.y + cx * uq.y);
        w = make_double2(py * wp.x + px * wq.x, py * wp.y + px * wq.y);
      }
    }
    return make_double2(0.5 * (v.x - w.x), 0.5 * (v.y + w.y));
  };
  const double s0 = s3[3 * k], s1 = s3[3 * k + 1], s2 = s3[3 * k + 2];
  auto Sd = [&](int f) -> double2 {
    const double2 d0 = delta(f, k), d2 = delta(f, k + 2), d4 = delta(f, k + 4);
    return make_double2(s0 * d0.x + s1 * d2.x + s2 * d4.x, s0 * d0.y + s1 * d2.y + s2 * d4.y);
  };
  const double kx = a.kx0 * ix, ky = a.ky0 * ky_index(iy, Ny), k2 = kx * kx + ky * ky;
  const double d2c = 2.0 * (k + 2) * s * s;
  const double2 Sb = Sd(0), Sux = Sd(1), Suy = Sd(2), Suz = Sd(3);
  const double2 Db = delta(0, k + 2), Dux = delta(1, k + 2), Duy = delta(2, k + 2), Duz = delta(3, k + 2);
  const double2 u1 = delta(3, k + 1), u3 = delta(3, k + 3);
  double2 L[5];
  double2 mx, my;
  if constexpr (MASS) {
    L[0] = make_double2(0.0, 0.0);
    L[1] = Sb;
    mx = Sux;
    my = Suy;
    L[3] = Suz;
  } else {
    // continuity: i kx S d_ux + i ky S d_uy + SD d_uz
    L[0] = make_double2(-kx * Sux.y - ky * Suy.y + s * (u1.x - u3.x), kx * Sux.x + ky * Suy.x + s * (u1.y - u3.y));
    L[1] = make_double2(kappa * (k2 * Sb.x - d2c * Db.x), kappa * (k2 * Sb.y - d2c * Db.y));
    mx = make_double2(nu * (k2 * Sux.x - d2c * Dux.x), nu * (k2 * Sux.y - d2c * Dux.y));
    my = make_double2(nu * (k2 * Suy.x - d2c * Duy.x), nu * (k2 * Suy.y - d2c * Duy.y));
    L[3] = make_double2(nu * (k2 * Suz.x - d2c * Duz.x) - Sb.x, nu * (k2 * Suz.y - d2c * Duz.y) - Sb.y);
  }
  L[2] = make_double2(cx * mx.x + cy * my.x, cx * mx.y + cy * my.y);
  L[4] = make_double2(-cy * mx.x + cx * my.x, -cy * mx.y + cx * my.y);
  (void)beta;
  const size_t i = (size_t)k * Nk + m;
#pragma unroll
  for (int e = 0; e < 5; ++e) {
    double2 r = LX[(size_t)e * plane + i];
    r.x -= L[e].x;
    r.y -= L[e].y;
    LX[(size_t)e * plane + i] = r;
  }
}

// FFT along y of the columns of a [z][y][kx] array (length Ny, in place),
// sign -1 forward (unnormalised) or +1 inverse (scaled by 1/Ny).  Grid (Kx, Nz).
__global__ void __launch_bounds__(256) k3_ycols(double2* __restrict__ a, int Ny, int Kx, FftPlan fp,
                                                const double2* __restrict__ ptw, int npt, int sign) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  double2* sm = reinterpret_cast<double2*>(sm_raw);
  const int kx = blockIdx.x, z = blockIdx.y;
  const int Ms = (Ny + 7) & ~7;
  double2* A = sm;
  double2* B = sm + Ms;
  double2* pt = sm + 2 * Ms;
  for (int t = threadIdx.x; t < npt; t += blockDim.x) pt[t] = ptw[t];
  double2* col = a + (size_t)z * Ny * Kx + kx;
  for (int y = threadIdx.x; y < Ny; y += blockDim.x) A[F::fidx<true>(y)] = col[(size_t)y * Kx];
  __syncthreads();
  const double2* R = F::fft<true>(A, B, fp, pt, sign);
  const double sc = sign > 0 ? 1.0 / Ny : 1.0;
  for (int y = threadIdx.x; y < Ny; y += blockDim.x) col[(size_t)y * Kx] = F::scale(R[F::fidx<true>(y)], sc);
}

// Public coefficient index of (z, mode m = ix Ny + iy): ix + Kx (iy + Ny z).
__device__ __forceinline__ size_t pub_of(const R3Args& a, int z, int m) {
  return (size_t)(m / a.Ny) + (size_t)a.Kx * ((size_t)(m % a.Ny) + (size_t)a.Ny * z);
}

// Field I/O: grid (ceil(Nk/256), Nz) over the plan's modes.
__global__ void __launch_bounds__(256) k3_state_get(R3Args a, const double2* __restrict__ X, int field,
                                                    double2* __restrict__ out) {
  const int z = blockIdx.y, m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.Nk) return;
  const size_t plane = (size_t)a.Nz * a.Nk, i = (size_t)z * a.Nk + m;
  double2 v;
  if (field == TB_FIELD_B) {
    v = X[i];
  } else if (field == TB_FIELD_UZ) {
    v = X[2 * plane + i];
  } else if (field == TB_FIELD_P) {
    v = X[3 * plane + i];
  } else {
    double cx, cy;
    rot_of(a, m / a.Ny, m % a.Ny, cx, cy);
    const double2 up = X[plane + i], uq = X[4 * plane + i];
    v = field == TB_FIELD_UX ? make_double2(cx * up.x - cy * uq.x, cx * up.y - cy * uq.y)
                             : make_double2(cy * up.x + cx * uq.x, cy * up.y + cx * uq.y);
  }
  out[pub_of(a, z, m)] = v;
}

__global__ void __launch_bounds__(256) k3_state_set(R3Args a, double2* __restrict__ X, int field,
                                                    const double2* __restrict__ in) {
  const int z = blockIdx.y, m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.Nk) return;
  const size_t plane = (size_t)a.Nz * a.Nk, i = (size_t)z * a.Nk + m;
  const double2 v = in[pub_of(a, z, m)];
  if (field == TB_FIELD_B) {
    X[i] = v;
  } else if (field == TB_FIELD_UZ) {
    X[2 * plane + i] = v;
  } else if (field == TB_FIELD_P) {
    X[3 * plane + i] = v;
  } else {
    double cx, cy;
    rot_of(a, m / a.Ny, m % a.Ny, cx, cy);
    const double2 up = X[plane + i], uq = X[4 * plane + i];
    double2 ux = make_double2(cx * up.x - cy * uq.x, cx * up.y - cy * uq.y);
    double2 uy = make_double2(cy * up.x + cx * uq.x, cy * up.y + cx * uq.y);
    if (field == TB_FIELD_UX)
      ux = v;
    else
      uy = v;
    X[plane + i] = make_double2(cx * ux.x + cy * uy.x, cx * ux.y + cy * uy.y);
    X[4 * plane + i] = make_double2(-cy * ux.x + cx * uy.x, -cy * ux.y + cx * uy.y);
  }
}

// Taus: public rows (tau_p, b1, b2, u1x, u1y, u1z, u2x, u2y, u2z) over (kx, ky)
// kx fastest; plan rows (tau_p, b1, b2, u1par, u1z, u2par, u2z, u1perp, u2perp)
// over modes.  Grid ceil(Nk/256).
__global__ void __launch_bounds__(256) k3_tau_io(R3Args a, double2* __restrict__ tau, double2* __restrict__ pub,
                                                 int set) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.Nk) return;
  const size_t Nk = a.Nk, pm = (size_t)(m / a.Ny) + (size_t)a.Kx * (m % a.Ny);
  double cx, cy;
  rot_of(a, m / a.Ny, m % a.Ny, cx, cy);
  const int direct_pub[5] = {0, 1, 2, 5, 8}, direct_int[5] = {0, 1, 2, 4, 6};
  for (int r = 0; r < 5; ++r) {
    double2* ti = tau + direct_int[r] * Nk + m;
    double2* tp = pub + direct_pub[r] * Nk + pm;
    if (set)
      *ti = *tp;
    else
      *tp = *ti;
  }
  for (int w = 0; w < 2; ++w) {
    double2* par = tau + (w ? 5 : 3) * Nk + m;
    double2* perp = tau + (w ? 8 : 7) * Nk + m;
    double2* px = pub + (w ? 6 : 3) * Nk + pm;
    double2* py = pub + (w ? 7 : 4) * Nk + pm;
    if (set) {
      const double2 ux = *px, uy = *py;
      *par = make_double2(cx * ux.x + cy * uy.x, cx * ux.y + cy * uy.y);
      *perp = make_double2(-cy * ux.x + cx * uy.x, -cy * ux.y + cx * uy.y);
    } else {
      const double2 up = *par, uq = *perp;
      *px = make_double2(cx * up.x - cy * uq.x, cx * up.y - cy * uq.y);
      *py = make_double2(cy * up.x + cx * uq.x, cy * up.y + cx * uq.y);
    }
  }
}

template <class C>
std::vector<C> pass_twiddles_t(const FftPlan& fp) {
  std::vector<C> t;
  const long double pi = 3.141592653589793238462643383279502884L;
  int Ns = 1;
  for (int s = 0; s < fp.nstages; ++s) {
    const int R = fp.radix[s];
    const int tstride = fp.n / (Ns * R);
    for (int j = 0; j < Ns; ++j) {
      const long double ang = -2.0L * pi * (long double)(j * tstride) / (long double)fp.n;
      C c;
      c.x = (decltype(c.x))cosl(ang);
      c.y = (decltype(c.y))sinl(ang);
      t.push_back(c);
    }
    Ns *= R;
  }
  return t;
}

R3Args args_of(const tb_plan* P) {
  R3Args a{};
  a.Nx = P->Nx;
  a.Ny = P->Ny;
  a.Nz = P->Nz;
  a.Kx = P->Kx;
  a.Mx = P->M;
  a.My = P->My;
  a.Nk = P->Nk;
  a.H = P->Nz / 2;
  a.kx0 = P->k0;
  a.ky0 = P->k0y;
  a.fpx = P->fpM;
  a.fpy = P->fpMy;
  // the FP32 384-point transform reads the full table exp(-2 pi i k/384)
  a.nptx = (P->mixed && P->M == 384) ? 384 : F::pass_twiddle_count(P->fpM);
  a.npty = (P->mixed && P->My == 384) ? 384 : F::pass_twiddle_count(P->fpMy);
  return a;
}

// Buffer length of the transform kernels for padded length m (see buf_len).
template <class C>
size_t buf_len_host(int m) {
  return (std::is_same<C, float2>::value && m == 384) ? (size_t)F::kLen384Buf : (size_t)F::pad_swz<C>(m);
}

template <class C>
size_t yinv_smem(const R3Args& a) {
  const size_t Ms = buf_len_host<C>(a.My);
  return (16 * (size_t)a.Ny + 24 * Ms + (size_t)a.npty) * sizeof(C);
}
template <class C, int RR>
size_t xpass_smem(const R3Args& a) {
  const size_t Ms = buf_len_host<C>(a.Mx);
  return (16 * RR * Ms + (size_t)a.nptx) * sizeof(C);
}
template <class C>
size_t yfwd_smem(const R3Args& a) {
  const size_t Ms = buf_len_host<C>(a.My);
  return (8 * Ms + (size_t)a.npty) * sizeof(C);
}

// Rows per x-pass CTA: 2 in FP32, 1 in FP64 (same shared memory).
template <class C>
struct XRows;
template <>
struct XRows<float2> {
  static constexpr int value = 2;
};
template <>
struct XRows<double2> {
  static constexpr int value = 1;
};

// Padded transform length with compiled plans (the 256-point grids of the 3D
// benchmark configuration); other lengths run the runtime plan.
constexpr int kFixedLen = 384;

template <class C>
void set_limits(int bytes) {
  const void* fns[] = {(const void*)k3_yinv<C, 0>,         (const void*)k3_yinv<C, kFixedLen>,
                       (const void*)k3_xpass<C, 1, 0>,    (const void*)k3_xpass<C, 1, kFixedLen>,
                       (const void*)k3_xpass<C, 2, 0>,    (const void*)k3_xpass<C, 2, kFixedLen>,
                       (const void*)k3_xpass<C, 4, 0>,    (const void*)k3_xpass<C, 4, kFixedLen>,
                       (const void*)k3_yfwd<C, 0>,         (const void*)k3_yfwd<C, kFixedLen>};
  for (const void* fn : fns) TB_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

// x-pass rows per CTA that fit (shared memory, padded Ny divisible).
template <class C>
bool xrows_ok(const tb_plan* P, const R3Args& a, int rr) {
  if (rr != 1 && rr != 2 && rr != 4) return false;
  if (P->My % rr) return false;
  const size_t Ms = buf_len_host<C>(a.Mx);
  return (16 * (size_t)rr * Ms + (size_t)a.nptx) * sizeof(C) <= 227 * 1024;
}

// Four rows per CTA run with 512 threads (one CTA per SM by shared memory):
// the staged loads then take whole 32-byte sectors (4 consecutive y of FP32
// complex) where one or two rows take a quarter or half of each.
template <class C, int RR>
void launch_xpass(tb_plan* P, const R3Args& a, cudaStream_t st) {
  auto kern = (P->M == kFixedLen) ? k3_xpass<C, RR, kFixedLen> : k3_xpass<C, RR, 0>;
  const int threads = RR == 4 ? 2 * kR3Threads : kR3Threads;
  kern<<<dim3(P->My / RR, P->Nz), threads, xpass_smem<C, RR>(a), st>>>(a, P->mix3.as<C>(), P->ptwX.as<C>(),
                                                                       P->pm3.as<C>());
}

inline int pad16(int k) { return (k + 15) / 16 * 16; }

template <class C>
void enqueue_rhs_t(tb_plan* P, const double2* Xin, double2* out4) {
  const R3Args a = args_of(P);
  const int N = P->Nz, H = N / 2;
  const size_t plane = P->plane, hplane = (size_t)H * P->Nk;
  const int ncol = 2 * P->Nk;
  C* Xc = P->Xc.as<C>();
  C* G = P->G3.as<C>();
  timed(P, "rhs3_prep", [&] {
    k3_prep<C><<<dim3((P->Nk + 255) / 256, N), 256, 0, P->st>>>(a, Xin, Xc);
  });
  constexpr bool f32 = sizeof(C) == sizeof(float2);
  if constexpr (f32) {
    GemmBatch32 bt{};
    const float* Am[4] = {P->bEv32.as<float>(), P->bOv32.as<float>(), P->bEd32.as<float>(), P->bOd32.as<float>()};
    for (int f = 0; f < 4; ++f)
      for (int w = 0; w < 4; ++w)
        bt.item[4 * f + w] = GemmItem32{Am[w], reinterpret_cast<const float*>(Xc + (size_t)f * plane),
                                        G + (size_t)(4 * f + w) * hplane, H, (w & 1) ? P->Ko : P->Ke,
                                        pad16((w & 1) ? P->Ko : P->Ke), GEMM_PARITY, w & 1};
    if (P->tc32 && P->tc3)
      timed(P, "z_backward_gemm", [&] {
        launch_tc32s(true, P->tc3Xc, P->tc3img.as<float>(), G, 4, N, ncol, P->st);
      });
    else
      timed(P, "z_backward_gemm", [&] { launch_gemm_f32(bt, 16, ncol, ncol, ncol, N, false, P->st); });
  } else {
    GemmBatch bt{};
    const double* Am[4] = {P->bEv.as<double>(), P->bOv.as<double>(), P->bEd.as<double>(), P->bOd.as<double>()};
    for (int f = 0; f < 4; ++f)
      for (int w = 0; w < 4; ++w)
        bt.item[4 * f + w] = GemmItem{Am[w], reinterpret_cast<const double*>(Xc + (size_t)f * plane),
                                      reinterpret_cast<double*>(G + (size_t)(4 * f + w) * hplane), H,
                                      (w & 1) ? P->Ko : P->Ke, pad16((w & 1) ? P->Ko : P->Ke), GEMM_PARITY, w & 1};
    timed(P, "z_backward_gemm", [&] { launch_gemm_f64(bt, 16, ncol, ncol, ncol, N, P->st); });
  }
  const bool fy = P->My == kFixedLen, fx = P->M == kFixedLen;
  timed(P, "rhs3_yinv", [&] {
    auto kern = fy ? k3_yinv<C, kFixedLen> : k3_yinv<C, 0>;
    kern<<<dim3(P->Kx, H), kR3Threads, yinv_smem<C>(a), P->st>>>(a, G, P->ptwY.as<C>(), P->mix3.as<C>());
  });
  (void)fx;
  timed(P, "rhs3_xpass", [&] {
    if (P->xrows == 4)
      launch_xpass<C, 4>(P, a, P->st);
    else if (P->xrows == 2)
      launch_xpass<C, 2>(P, a, P->st);
    else
      launch_xpass<C, 1>(P, a, P->st);
  });
  timed(P, "rhs3_yfwd", [&] {
    auto kern = fy ? k3_yfwd<C, kFixedLen> : k3_yfwd<C, 0>;
    kern<<<dim3(P->Kx, N), kR3Threads, yfwd_smem<C>(a), P->st>>>(a, P->pm3.as<C>(), P->ptwY.as<C>(), P->H3.as<C>());
  });
  const C* H3 = P->H3.as<C>();
  if constexpr (f32) {
    GemmBatch32 bf{};
    int nb = 0;
    for (int f = 0; f < 4; ++f) {
      const float* in = reinterpret_cast<const float*>(H3 + (size_t)f * plane);
      double* out = reinterpret_cast<double*>(out4 + (size_t)f * plane);
      bf.item[nb++] = GemmItem32{P->sfE32.as<float>(), in, out, P->Ke, H, pad16(H), GEMM_MIRROR, 0};
      bf.item[nb++] = GemmItem32{P->sfO32.as<float>(), in, out, P->Ko, H, pad16(H), GEMM_MIRROR, 1};
    }
    if (P->tc32 && P->tc3)
      timed(P, "z_forward_gemm", [&] {
        launch_tc32s(false, P->tc3H3, P->tc3img.as<float>(), out4, 4, N, ncol, P->st);
      });
    else
      timed(P, "z_forward_gemm", [&] { launch_gemm_f32(bf, nb, ncol, ncol, ncol, N, true, P->st); });
  } else {
    GemmBatch bf{};
    int nb = 0;
    for (int f = 0; f < 4; ++f) {
      const double* in = reinterpret_cast<const double*>(H3 + (size_t)f * plane);
      double* out = reinterpret_cast<double*>(out4 + (size_t)f * plane);
      bf.item[nb++] = GemmItem{P->sfE.as<double>(), in, out, P->Ke, H, pad16(H), GEMM_MIRROR, 0};
      bf.item[nb++] = GemmItem{P->sfO.as<double>(), in, out, P->Ko, H, pad16(H), GEMM_MIRROR, 1};
    }
    timed(P, "z_forward_gemm", [&] { launch_gemm_f64(bf, nb, ncol, ncol, ncol, N, P->st); });
  }
}

template <class C>
void setup_t(tb_plan* P) {
  constexpr int RR = XRows<C>::value;
  const R3Args a = args_of(P);
  TB_REQUIRE(P->My % RR == 0, TB_ENOTSUPPORTED, "padded Ny must be a multiple of the x-pass rows");
  const size_t lim = 227 * 1024;
  TB_REQUIRE(yinv_smem<C>(a) <= lim && xrows_ok<C>(P, a, RR) && yfwd_smem<C>(a) <= lim, TB_ENOTSUPPORTED,
             "Nx or Ny too large for the 3D transform kernels");
  P->xrows = RR;
  set_limits<C>((int)lim);
  const size_t plane = P->plane, H = (size_t)P->Nz / 2;
  P->Xc.alloc(4 * plane * sizeof(C));
  P->G3.alloc(16 * H * P->Nk * sizeof(C));
  const size_t slab = (size_t)P->Nz * P->Kx * P->My;
  P->mix3.alloc(12 * slab * sizeof(C));
  P->pm3.alloc(4 * slab * sizeof(C));
  P->H3.alloc(4 * plane * sizeof(C));
  if constexpr (std::is_same<C, float2>::value) {
    // the streaming tensor-core form of the z transforms
    const int N = P->Nz, ncol = 2 * P->Nk;
    P->tc3 = false;
    if (tc32s_supported(N, ncol)) {
      P->tc3img.alloc(tc32s_image_floats() * sizeof(float));
      make_tc32s_images(P->bEv32.as<float>(), P->bOv32.as<float>(), P->bEd32.as<float>(), P->bOd32.as<float>(),
                        pad16(P->Ke), pad16(P->Ko), P->sfE32.as<float>(), P->sfO32.as<float>(), pad16(N / 2), N,
                        P->tc3img.as<float>(), P->st);
      TB_CUDA_TRY(cudaGetLastError());
      TB_CUDA_TRY(cudaStreamSynchronize(P->st));
      P->tc3 = make_tc32s_tmap(&P->tc3Xc, reinterpret_cast<const float*>(P->Xc.p), 4, N, ncol) &&
               make_tc32s_tmap(&P->tc3H3, reinterpret_cast<const float*>(P->H3.p), 4, N, ncol);
    }
    P->tc32 = P->tc3;  // the default GEMM path of a 3D plan: faster than SIMT at every supported size measured
  }
  auto table = [&](const FftPlan& fp) {
    if (std::is_same<C, float2>::value && fp.n == 384) {
      std::vector<C> t(384);
      const long double pi = 3.141592653589793238462643383279502884L;
      for (int k = 0; k < 384; ++k) {
        t[k].x = (decltype(t[k].x))cosl(-2.0L * pi * k / 384.0L);
        t[k].y = (decltype(t[k].y))sinl(-2.0L * pi * k / 384.0L);
      }
      return t;
    }
    return pass_twiddles_t<C>(fp);
  };
  upload(P->ptwX, table(P->fpM));
  upload(P->ptwY, table(P->fpMy));
}

}  // namespace

void rbc3d_setup(tb_plan* P) {
  TB_REQUIRE(make_fft_plan(P->My, &P->fpMy) && make_fft_plan(P->Ny, &P->fpNy), TB_ENOTSUPPORTED,
             "Ny must be of the form 2^a 3^b with a padded length 3Ny/2 of the same form");
  upload(P->ptwNy, pass_twiddles_t<double2>(P->fpNy));
  P->tmp3.alloc(std::max(P->plane, (size_t)9 * P->Nk) * sizeof(double2));
  std::vector<double> km(P->Nk);
  for (int ix = 0; ix < P->Kx; ++ix)
    for (int iy = 0; iy < P->Ny; ++iy) {
      const double kx = P->k0 * ix, ky = P->k0y * (iy < P->Ny / 2 ? iy : iy - P->Ny);
      km[(size_t)ix * P->Ny + iy] = std::sqrt(kx * kx + ky * ky);
    }
  upload(P->kmag, km);
  if (P->mixed)
    setup_t<float2>(P);
  else
    setup_t<double2>(P);
}

bool rbc3d_xrows_ok(const tb_plan* P, int rows) {
  const R3Args a = args_of(P);
  return P->mixed ? xrows_ok<float2>(P, a, rows) : xrows_ok<double2>(P, a, rows);
}

void rbc3d_enqueue_rhs(tb_plan* P, const double2* Xin, double2* out4) {
  if (P->mixed)
    enqueue_rhs_t<float2>(P, Xin, out4);
  else
    enqueue_rhs_t<double2>(P, Xin, out4);
}

void rbc3d_lx_project(tb_plan* P, double2* LX, double beta, cudaStream_t st) {
  const R3Args a = args_of(P);
  timed(P, "lx_project", [&] {
    k3_lx_project<false><<<dim3((2 * P->Ny + 127) / 128, P->Nz), 128, 0, st ? st : P->st>>>(
        a, LX, P->X.as<double2>(), P->s3.as<double>(), P->s, P->d.kappa, P->d.nu, beta);
  });
}

void rbc3d_mx_project(tb_plan* P, double2* MX, cudaStream_t st) {
  const R3Args a = args_of(P);
  timed(P, "mx_project", [&] {
    k3_lx_project<true><<<dim3((2 * P->Ny + 127) / 128, P->Nz), 128, 0, st ? st : P->st>>>(
        a, MX, P->X.as<double2>(), P->s3.as<double>(), P->s, P->d.kappa, P->d.nu, 1.0);
  });
}

size_t rbc3d_device_bytes(const tb_plan* P) {
  return P->kmag.bytes + P->Xc.bytes + P->G3.bytes + P->mix3.bytes + P->pm3.bytes + P->H3.bytes + P->ptwX.bytes +
         P->ptwY.bytes + P->ptwNy.bytes + P->tmp3.bytes;
}

namespace {
void ycols(tb_plan* P, double2* a, int sign) {
  const int npt = F::pass_twiddle_count(P->fpNy);
  const size_t smem = (2 * (size_t)((P->Ny + 7) & ~7) + npt) * sizeof(double2);
  k3_ycols<<<dim3(P->Kx, P->Nz), 256, smem, P->st>>>(a, P->Ny, P->Kx, P->fpNy, P->ptwNy.as<double2>(), npt, sign);
}
}  // namespace

void periodic_ycols(double2* a, int Ny, int Kx, const FftPlan& fp, const double2* ptw, int sign, cudaStream_t st) {
  const int npt = F::pass_twiddle_count(fp);
  const size_t smem = (2 * (size_t)((Ny + 7) & ~7) + npt) * sizeof(double2);
  // the opt-in limit, never the launch's own size: the attribute is per
  // kernel and process-wide, and the 3D path launches k3_ycols too
  TB_CUDA_TRY(cudaFuncSetAttribute(k3_ycols, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  k3_ycols<<<dim3(Kx, 1), 256, smem, st>>>(a, Ny, Kx, fp, ptw, npt, sign);
}

void rbc3d_transform_forward(tb_plan* P, const double* grid, double2* coeff) {
  double2* t = P->tmp3.as<double2>();
  launch_x_rfft(grid, t, P->Nz * P->Ny, P->Nx, P->fpN, P->twN.as<double2>(), P->st);
  ycols(P, t, -1);
  const int H = P->Nz / 2, ncol = 2 * P->Nk;
  GemmBatch bt{};
  bt.item[0] = GemmItem{P->fE.as<double>(), reinterpret_cast<const double*>(t), reinterpret_cast<double*>(coeff),
                        P->Ke, H, pad16(H), GEMM_MIRROR, 0};
  bt.item[1] = GemmItem{P->fO.as<double>(), reinterpret_cast<const double*>(t), reinterpret_cast<double*>(coeff),
                        P->Ko, H, pad16(H), GEMM_MIRROR, 1};
  launch_gemm_f64(bt, 2, ncol, ncol, ncol, P->Nz, P->st);
}

void rbc3d_transform_backward(tb_plan* P, const double2* coeff, double* grid) {
  double2* t = P->tmp3.as<double2>();
  const int ncol = 2 * P->Nk;
  GemmBatch bt{};
  bt.item[0] = GemmItem{P->bwd.as<double>(), reinterpret_cast<const double*>(coeff), reinterpret_cast<double*>(t),
                        P->Nz, P->Nz, pad16(P->Nz), GEMM_PLAIN, 0};
  launch_gemm_f64(bt, 1, ncol, ncol, ncol, P->Nz, P->st);
  ycols(P, t, +1);
  launch_x_irfft(t, grid, P->Nz * P->Ny, P->Nx, P->fpN, P->twN.as<double2>(), P->st);
}

void rbc3d_state_get(tb_plan* P, int field, double2* dst) {
  const R3Args a = args_of(P);
  if (field == TB_FIELD_TAU)
    k3_tau_io<<<(P->Nk + 255) / 256, 256, 0, P->st>>>(a, P->tau.as<double2>(), dst, 0);
  else
    k3_state_get<<<dim3((P->Nk + 255) / 256, P->Nz), 256, 0, P->st>>>(a, P->X.as<double2>(), field, dst);
}

void rbc3d_state_set(tb_plan* P, int field, const double2* src) {
  const R3Args a = args_of(P);
  if (field == TB_FIELD_TAU)
    k3_tau_io<<<(P->Nk + 255) / 256, 256, 0, P->st>>>(a, P->tau.as<double2>(), const_cast<double2*>(src), 1);
  else
    k3_state_set<<<dim3((P->Nk + 255) / 256, P->Nz), 256, 0, P->st>>>(a, P->X.as<double2>(), field, src);
}

}  // namespace tb
