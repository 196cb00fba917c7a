// Stockham FFT building blocks in shared memory, generic over the complex
// type (float2 for the FP32 programs, double2).  Same formulation as the
// double-only transforms of the Chebyshev programs: radix 8/4/2/3 passes,
// natural-order output, XOR-swizzled buffers, per-pass twiddle tables
// pt[j] = exp(-2 pi i j n/(Ns R) / n) for j < Ns.
#pragma once

#include <cuda_runtime.h>

#include "tb_internal.h"

namespace tb {
namespace fftg {

template <class C>
struct Real;
template <>
struct Real<float2> {
  using type = float;
};
template <>
struct Real<double2> {
  using type = double;
};

template <class C>
__device__ __forceinline__ C mk(typename Real<C>::type x, typename Real<C>::type y) {
  C c;
  c.x = x;
  c.y = y;
  return c;
}
template <class C>
__device__ __forceinline__ C add(C a, C b) {
  return mk<C>(a.x + b.x, a.y + b.y);
}
template <class C>
__device__ __forceinline__ C sub(C a, C b) {
  return mk<C>(a.x - b.x, a.y - b.y);
}
template <class C>
__device__ __forceinline__ C mul(C a, C b) {
  return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class C>
__device__ __forceinline__ C scale(C a, typename Real<C>::type s) {
  return mk<C>(a.x * s, a.y * s);
}
template <class C>
__device__ __forceinline__ C conjg(C a) {
  return mk<C>(a.x, -a.y);
}
// multiply by exp(sign i pi/2)
template <class C>
__device__ __forceinline__ C rot4(C d, int sign) {
  return (sign < 0) ? mk<C>(d.y, -d.x) : mk<C>(-d.y, d.x);
}

template <bool SW>
__device__ __forceinline__ int fidx(int i) {
  return SW ? (i ^ ((i >> 3) & 7)) : i;
}

template <class C>
__device__ __forceinline__ void dft4(C& x0, C& x1, C& x2, C& x3, int sign) {
  const C t0 = add(x0, x2), t1 = sub(x0, x2), t2 = add(x1, x3), t3 = rot4(sub(x1, x3), sign);
  x0 = add(t0, t2);
  x1 = add(t1, t3);
  x2 = sub(t0, t2);
  x3 = sub(t1, t3);
}

template <int R, class C>
__device__ __forceinline__ void dft_small(C (&v)[R], int sign) {
  using T = typename Real<C>::type;
  if constexpr (R == 2) {
    const C a = v[0], b = v[1];
    v[0] = add(a, b);
    v[1] = sub(a, b);
  } else if constexpr (R == 3) {
    const T h = (T)0.86602540378443864676372317075294;  // sqrt(3)/2
    const C sm = add(v[1], v[2]), df = sub(v[1], v[2]);
    const C base = mk<C>(v[0].x - (T)0.5 * sm.x, v[0].y - (T)0.5 * sm.y);
    const C rot = mk<C>(-(T)sign * h * df.y, (T)sign * h * df.x);
    v[0] = add(v[0], sm);
    v[1] = add(base, rot);
    v[2] = sub(base, rot);
  } else if constexpr (R == 4) {
    dft4(v[0], v[1], v[2], v[3], sign);
  } else {
    const T r = (T)0.70710678118654752440084436210485;
    const T s = (T)sign;
    C a[4], b[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      a[n] = add(v[n], v[n + 4]);
      b[n] = sub(v[n], v[n + 4]);
    }
    b[1] = mk<C>(r * (b[1].x - s * b[1].y), r * (b[1].y + s * b[1].x));
    b[2] = rot4(b[2], sign);
    b[3] = mk<C>(r * (-b[3].x - s * b[3].y), r * (-b[3].y + s * b[3].x));
    dft4(a[0], a[1], a[2], a[3], sign);
    dft4(b[0], b[1], b[2], b[3], sign);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[2 * k] = a[k];
      v[2 * k + 1] = b[k];
    }
  }
}

template <int R, bool SW, class C>
__device__ __forceinline__ void pass(const C* __restrict__ in, C* __restrict__ out, int n, int Ns,
                                     const C* __restrict__ pt, int sign) {
  const int nR = n / R;
  for (int idx = threadIdx.x; idx < nR; idx += blockDim.x) {
    const int j = idx % Ns, k = idx / Ns;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = in[fidx<SW>(idx + r * nR)];
    if (Ns > 1) {
      C w1 = pt[j];
      if (sign > 0) w1.y = -w1.y;
      if constexpr (R == 8) {
        const C w2 = mul(w1, w1), w4 = mul(w2, w2), w3 = mul(w1, w2);
        v[1] = mul(v[1], w1);
        v[2] = mul(v[2], w2);
        v[3] = mul(v[3], w3);
        v[4] = mul(v[4], w4);
        v[5] = mul(v[5], mul(w1, w4));
        v[6] = mul(v[6], mul(w2, w4));
        v[7] = mul(v[7], mul(w3, w4));
      } else if constexpr (R == 4) {
        const C w2 = mul(w1, w1);
        v[1] = mul(v[1], w1);
        v[2] = mul(v[2], w2);
        v[3] = mul(v[3], mul(w1, w2));
      } else if constexpr (R == 3) {
        v[1] = mul(v[1], w1);
        v[2] = mul(v[2], mul(w1, w1));
      } else {
        v[1] = mul(v[1], w1);
      }
    }
    dft_small<R>(v, sign);
    const int ob = k * Ns * R + j;
#pragma unroll
    for (int r = 0; r < R; ++r) out[fidx<SW>(ob + r * Ns)] = v[r];
  }
}

// Whole-CTA FFT of length fp.n between buffers a and b; returns the buffer
// holding the result.  sign -1 forward, +1 inverse, both unnormalised.
template <bool SW, class C>
__device__ C* fft(C* a, C* b, const FftPlan& fp, const C* __restrict__ pt, int sign) {
  const int n = fp.n;
  int Ns = 1;
  C* in = a;
  C* out = b;
  for (int s = 0; s < fp.nstages; ++s) {
    const int R = fp.radix[s];
    if (R == 8)
      pass<8, SW>(in, out, n, Ns, pt, sign);
    else if (R == 4)
      pass<4, SW>(in, out, n, Ns, pt, sign);
    else if (R == 2)
      pass<2, SW>(in, out, n, Ns, pt, sign);
    else
      pass<3, SW>(in, out, n, Ns, pt, sign);
    __syncthreads();
    C* t = in;
    in = out;
    out = t;
    pt += Ns;
    Ns *= R;
  }
  return in;
}

// One Stockham pass over NA arrays stored Ms apart (the arrays share the
// pass's barrier); pass<R, SW> arithmetic for each array.
template <int R, bool SW, class C>
__device__ __forceinline__ void pass_multi(const C* __restrict__ in, C* __restrict__ out, int NA, int Ms, int n,
                                           int Ns, const C* __restrict__ pt, int sign) {
  const int nR = n / R, total = NA * nR;
  for (int item = threadIdx.x; item < total; item += blockDim.x) {
    const int arr = item / nR, idx = item - arr * nR;
    const C* ia = in + (size_t)arr * Ms;
    C* oa = out + (size_t)arr * Ms;
    const int j = idx % Ns, k = idx / Ns;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = ia[fidx<SW>(idx + r * nR)];
    if (Ns > 1) {
      C w1 = pt[j];
      if (sign > 0) w1.y = -w1.y;
      if constexpr (R == 8) {
        const C w2 = mul(w1, w1), w4 = mul(w2, w2), w3 = mul(w1, w2);
        v[1] = mul(v[1], w1);
        v[2] = mul(v[2], w2);
        v[3] = mul(v[3], w3);
        v[4] = mul(v[4], w4);
        v[5] = mul(v[5], mul(w1, w4));
        v[6] = mul(v[6], mul(w2, w4));
        v[7] = mul(v[7], mul(w3, w4));
      } else if constexpr (R == 4) {
        const C w2 = mul(w1, w1);
        v[1] = mul(v[1], w1);
        v[2] = mul(v[2], w2);
        v[3] = mul(v[3], mul(w1, w2));
      } else if constexpr (R == 3) {
        v[1] = mul(v[1], w1);
        v[2] = mul(v[2], mul(w1, w1));
      } else {
        v[1] = mul(v[1], w1);
      }
    }
    dft_small<R>(v, sign);
    const int ob = k * Ns * R + j;
#pragma unroll
    for (int r = 0; r < R; ++r) oa[fidx<SW>(ob + r * Ns)] = v[r];
  }
}

// NA whole-CTA FFTs of length fp.n at a + arr Ms, ping-ponging with b; returns
// the block holding the results.
template <bool SW, class C>
__device__ C* fft_multi(C* a, C* b, int NA, int Ms, const FftPlan& fp, const C* __restrict__ pt, int sign) {
  const int n = fp.n;
  int Ns = 1;
  C* in = a;
  C* out = b;
  for (int s = 0; s < fp.nstages; ++s) {
    const int R = fp.radix[s];
    if (R == 8)
      pass_multi<8, SW>(in, out, NA, Ms, n, Ns, pt, sign);
    else if (R == 4)
      pass_multi<4, SW>(in, out, NA, Ms, n, Ns, pt, sign);
    else if (R == 2)
      pass_multi<2, SW>(in, out, NA, Ms, n, Ns, pt, sign);
    else
      pass_multi<3, SW>(in, out, NA, Ms, n, Ns, pt, sign);
    __syncthreads();
    C* t = in;
    in = out;
    out = t;
    pt += Ns;
    Ns *= R;
  }
  return in;
}

// Swizzle keyed to the element size: the low bits of an index are XORed with
// the next ones over a group of 128 bytes (8 double2 or 16 float2), so that the
// stride-R stores of a pass and the unit-stride loads both spread over all
// banks.  Buffers are padded to whole groups (pad_swz).
template <class C>
struct SwzGroup;
template <>
struct SwzGroup<double2> {
  static constexpr int shift = 3;
};
template <>
struct SwzGroup<float2> {
  static constexpr int shift = 4;
};
template <class C>
__host__ __device__ constexpr int pad_swz(int n) {
  return (n + (1 << SwzGroup<C>::shift) - 1) & ~((1 << SwzGroup<C>::shift) - 1);
}
template <class C>
__device__ __forceinline__ int sidx(int i) {
  constexpr int s = SwzGroup<C>::shift;
  return i ^ ((i >> s) & ((1 << s) - 1));
}

// Radix of stage s of the Stockham plan of length n (radices 8, then 4, 2, 3:
// the order make_fft_plan uses), 0 past the last stage.
__host__ __device__ constexpr int ct_radix(int n, int s) {
  int k = 0;
  while (n % 8 == 0) {
    if (k == s) return 8;
    n /= 8;
    ++k;
  }
  while (n % 4 == 0) {
    if (k == s) return 4;
    n /= 4;
    ++k;
  }
  while (n % 2 == 0) {
    if (k == s) return 2;
    n /= 2;
    ++k;
  }
  while (n % 3 == 0) {
    if (k == s) return 3;
    n /= 3;
    ++k;
  }
  return 0;
}

template <int R, class C>
__device__ __forceinline__ void twiddle_apply(C (&v)[R], C w1) {
  if constexpr (R == 8) {
    const C w2 = mul(w1, w1), w4 = mul(w2, w2), w3 = mul(w1, w2);
    v[1] = mul(v[1], w1);
    v[2] = mul(v[2], w2);
    v[3] = mul(v[3], w3);
    v[4] = mul(v[4], w4);
    v[5] = mul(v[5], mul(w1, w4));
    v[6] = mul(v[6], mul(w2, w4));
    v[7] = mul(v[7], mul(w3, w4));
  } else if constexpr (R == 4) {
    const C w2 = mul(w1, w1);
    v[1] = mul(v[1], w1);
    v[2] = mul(v[2], w2);
    v[3] = mul(v[3], mul(w1, w2));
  } else if constexpr (R == 3) {
    v[1] = mul(v[1], w1);
    v[2] = mul(v[2], mul(w1, w1));
  } else {
    v[1] = mul(v[1], w1);
  }
}

// Compile-time form of pass_batch for a length-N plan (constant divisors and
// strides, typed swizzle).
template <int R, int NS, int N, class C>
__device__ __forceinline__ void pass_ct(const C* __restrict__ in, C* __restrict__ out, const C* __restrict__ pt,
                                        int sign, int nb, int stride) {
  constexpr int nR = N / R;
  for (int t = threadIdx.x; t < nb * nR; t += blockDim.x) {
    const int q = t / nR, idx = t - q * nR;
    const int j = idx % NS, k = idx / NS;
    const C* src = in + (size_t)q * stride;
    C* dst = out + (size_t)q * stride;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[sidx<C>(idx + r * nR)];
    if constexpr (NS > 1) {
      C w1 = pt[j];
      if (sign > 0) w1.y = -w1.y;
      twiddle_apply<R>(v, w1);
    }
    dft_small<R>(v, sign);
    const int ob = k * NS * R + j;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[sidx<C>(ob + r * NS)] = v[r];
  }
}

template <int N, int S, int NS, class C>
__device__ __forceinline__ C* stages_ct(C* in, C* out, const C* __restrict__ pt, int sign, int nb, int stride) {
  constexpr int R = ct_radix(N, S);
  if constexpr (R == 0) {
    return in;
  } else {
    pass_ct<R, NS, N>(in, out, pt, sign, nb, stride);
    __syncthreads();
    return stages_ct<N, S + 1, NS * R>(out, in, pt + NS, sign, nb, stride);
  }
}

// nb CTA-wide length-N transforms (N a compile-time constant) between buffer
// sets a and b; returns the set holding the results.  Same arithmetic and
// twiddle tables as fft_batch with the runtime plan of length N.
template <int N, class C>
__device__ C* fft_batch_ct(C* a, C* b, int nb, int stride, const C* __restrict__ pt, int sign) {
  return stages_ct<N, 0, 1>(a, b, pt, sign, nb, stride);
}

// ---------------------------------------------------------------------------
// Length-384 transforms in two register passes (384 = 16 x 24, four-step):
// pass 1 takes, per (transform, n2 < 24), the 16 inputs x[24 n1 + n2] into
// registers, a 16-point DFT (4 x 4 in registers), the twiddles w^(n2 k1), and
// stores row k1 of a [16][25] scratch; pass 2 takes, per (transform, k1 < 16),
// scratch row k1, a 24-point DFT (8 x 3 in registers) and stores X[k1 + 16 k2].
// Two shared-memory round trips per element instead of the four of the
// Stockham plan (8, 8, 2, 3).  Buffers in natural order (no swizzle), at least
// kLen384Buf elements apart.  w: exp(-2 pi i k / 384), k < 384.
// ---------------------------------------------------------------------------
constexpr int kLen384Buf = 400;  // 16 rows of 25 (padding spreads the row starts over the banks)

template <class C>
__device__ __forceinline__ C tw384(const C* __restrict__ w, int k, int sign) {
  C t = w[k];
  if (sign > 0) t.y = -t.y;
  return t;
}

// In-register DFT of length R1 R2 (natural order in and out); internal
// twiddles w_{R1 R2}^j = w_384^(j WS) with WS = 384 / (R1 R2).
template <int R1, int R2, int WS, class C>
__device__ __forceinline__ void dft_reg(C (&x)[R1 * R2], const C* __restrict__ w, int sign) {
  C y[R1 * R2];
#pragma unroll
  for (int n2 = 0; n2 < R2; ++n2) {
    C a[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) a[n1] = x[R2 * n1 + n2];
    dft_small<R1>(a, sign);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) y[k1 * R2 + n2] = (n2 * k1 == 0) ? a[k1] : mul(a[k1], tw384(w, n2 * k1 * WS, sign));
  }
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) {
    C b[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) b[n2] = y[k1 * R2 + n2];
    dft_small<R2>(b, sign);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) x[k1 + R1 * k2] = b[k2];
  }
}

// nb length-384 transforms, buffer q at a + q * stride (stride >= kLen384Buf),
// b the scratch set; results in a (returned).  sign -1 forward, +1 inverse,
// unnormalised.
template <class C>
__device__ C* fft384_batch(C* a, C* b, int nb, int stride, const C* __restrict__ w, int sign) {
  for (int t = threadIdx.x; t < nb * 24; t += blockDim.x) {
    const int q = t / 24, n2 = t - 24 * q;
    const C* src = a + (size_t)q * stride;
    C* dst = b + (size_t)q * stride;
    C v[16];
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) v[n1] = src[24 * n1 + n2];
    dft_reg<4, 4, 24>(v, w, sign);
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) dst[k1 * 25 + n2] = (k1 == 0 || n2 == 0) ? v[k1] : mul(v[k1], tw384(w, n2 * k1, sign));
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nb * 16; t += blockDim.x) {
    const int q = t / 16, k1 = t - 16 * q;
    const C* src = b + (size_t)q * stride + k1 * 25;
    C* dst = a + (size_t)q * stride;
    C v[24];
#pragma unroll
    for (int n2 = 0; n2 < 24; ++n2) v[n2] = src[n2];
    dft_reg<8, 3, 16>(v, w, sign);
#pragma unroll
    for (int k2 = 0; k2 < 24; ++k2) dst[k1 + 16 * k2] = v[k2];
  }
  __syncthreads();
  return a;
}

// Batched form: nb transforms of length fp.n, buffer q at a + q * stride (and
// b + q * stride), all butterflies of a pass spread over the CTA (typed swizzle).
template <int R, bool SW, class C>
__device__ __forceinline__ void pass_batch(const C* __restrict__ in, C* __restrict__ out, int n, int Ns,
                                           const C* __restrict__ pt, int sign, int nb, int stride) {
  const int nR = n / R;
  for (int t = threadIdx.x; t < nb * nR; t += blockDim.x) {
    const int q = t / nR, idx = t - q * nR;
    const int j = idx % Ns, k = idx / Ns;
    const C* src = in + (size_t)q * stride;
    C* dst = out + (size_t)q * stride;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[SW ? sidx<C>(idx + r * nR) : idx + r * nR];
    if (Ns > 1) {
      C w1 = pt[j];
      if (sign > 0) w1.y = -w1.y;
      twiddle_apply<R>(v, w1);
    }
    dft_small<R>(v, sign);
    const int ob = k * Ns * R + j;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[SW ? sidx<C>(ob + r * Ns) : ob + r * Ns] = v[r];
  }
}

// nb CTA-wide transforms between buffer sets a and b (buffer q at + q * stride);
// returns the set holding the results.
template <bool SW, class C>
__device__ C* fft_batch(C* a, C* b, int nb, int stride, const FftPlan& fp, const C* __restrict__ pt, int sign) {
  const int n = fp.n;
  int Ns = 1;
  C* in = a;
  C* out = b;
  for (int s = 0; s < fp.nstages; ++s) {
    const int R = fp.radix[s];
    if (R == 8)
      pass_batch<8, SW>(in, out, n, Ns, pt, sign, nb, stride);
    else if (R == 4)
      pass_batch<4, SW>(in, out, n, Ns, pt, sign, nb, stride);
    else if (R == 2)
      pass_batch<2, SW>(in, out, n, Ns, pt, sign, nb, stride);
    else
      pass_batch<3, SW>(in, out, n, Ns, pt, sign, nb, stride);
    __syncthreads();
    C* t = in;
    in = out;
    out = t;
    pt += Ns;
    Ns *= R;
  }
  return in;
}

// Number of per-pass twiddle entries of a plan (sum of the passes' Ns).
__host__ __device__ inline int pass_twiddle_count(const FftPlan& fp) {
  int c = 0, Ns = 1;
  for (int s = 0; s < fp.nstages; ++s) {
    c += Ns;
    Ns *= fp.radix[s];
  }
  return c;
}

// ---------------------------------------------------------------------------
// In-place mixed-radix passes over NA arrays (Ms apart), without a ping-pong
// buffer: decimation in frequency (natural order in, digit-reversed order
// out) and decimation in time (digit-reversed in, natural out) over the same
// radix sequence R_0 .. R_{S-1}.  Pass s works on blocks of L_s = n / (R_0 ...
// R_{s-1}) entries with butterfly stride m_s = L_s / R_s; each butterfly reads
// and writes the same R entries, so a pass needs one barrier.  A DIF inverse
// transform, a pointwise product and a DIT forward transform give the natural
// order result without any permutation pass (the digit reversal cancels).
// Twiddles: per pass s, exp(-2 pi i j / L_s) for j < m_s (ip_twiddle_count
// entries, the passes one after another); sign > 0 conjugates them.
// ---------------------------------------------------------------------------
// powers w^r (r = 1 .. R-1) of a pass twiddle, formed as twiddle_apply forms
// them (the same products, so the results are bitwise those of twiddle_apply)
template <int R, class C>
__device__ __forceinline__ void twiddle_powers(C (&w)[R], C w1) {
  w[1] = w1;
  if constexpr (R == 8) {
    w[2] = mul(w1, w1);
    w[4] = mul(w[2], w[2]);
    w[3] = mul(w1, w[2]);
    w[5] = mul(w1, w[4]);
    w[6] = mul(w[2], w[4]);
    w[7] = mul(w[3], w[4]);
  } else if constexpr (R == 4) {
    w[2] = mul(w1, w1);
    w[3] = mul(w1, w[2]);
  } else if constexpr (R == 3) {
    w[2] = mul(w1, w1);
  }
}

// G arrays per item (the same butterfly of G arrays: independent arithmetic
// chains that share one set of twiddle powers)
template <int R, bool SW, bool DIF, int G, class C>
__device__ __forceinline__ void pass_ip(C* __restrict__ buf, int NA, int Ms, int n, int L,
                                        const C* __restrict__ pt, int sign) {
  const int m = L / R, nb = n / R, total = (NA / G) * nb;
  for (int item = threadIdx.x; item < total; item += blockDim.x) {
    const int grp = item / nb, b = item - grp * nb;
    C* x = buf + (size_t)grp * G * Ms;
    const int block = b / m, j = b - block * m;
    const int base = block * L + j;
    C v[G][R];
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int r = 0; r < R; ++r) v[g][r] = x[(size_t)g * Ms + fidx<SW>(base + r * m)];
    if constexpr (G == 1) {
      // one array: the powers formed as they are applied (fewer live registers)
      C w1 = mk<C>(0, 0);
      if (m > 1) {
        w1 = pt[j];
        if (sign > 0) w1.y = -w1.y;
      }
      if constexpr (DIF) {
        dft_small<R>(v[0], sign);
        if (m > 1) twiddle_apply<R>(v[0], w1);
      } else {
        if (m > 1) twiddle_apply<R>(v[0], w1);
        dft_small<R>(v[0], sign);
      }
    } else {
      C w[R];
      if (m > 1) {
        C w1 = pt[j];
        if (sign > 0) w1.y = -w1.y;
        twiddle_powers<R>(w, w1);
      }
#pragma unroll
      for (int g = 0; g < G; ++g) {
        if constexpr (DIF) {
          dft_small<R>(v[g], sign);
          if (m > 1)
#pragma unroll
            for (int r = 1; r < R; ++r) v[g][r] = mul(v[g][r], w[r]);
        } else {
          if (m > 1)
#pragma unroll
            for (int r = 1; r < R; ++r) v[g][r] = mul(v[g][r], w[r]);
          dft_small<R>(v[g], sign);
        }
      }
    }
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int r = 0; r < R; ++r) x[(size_t)g * Ms + fidx<SW>(base + r * m)] = v[g][r];
  }
}

template <bool SW, bool DIF, class C>
__device__ __forceinline__ void pass_ip_r(int R, C* buf, int NA, int Ms, int n, int L, const C* pt, int sign) {
  // FP32: arrays in pairs when their count is even (FP64 pairs run out of
  // registers at two CTAs per SM and were no faster)
  if (sizeof(C) == sizeof(float2) && NA % 2 == 0) {
    if (R == 8)
      pass_ip<8, SW, DIF, 2>(buf, NA, Ms, n, L, pt, sign);
    else if (R == 4)
      pass_ip<4, SW, DIF, 2>(buf, NA, Ms, n, L, pt, sign);
    else if (R == 2)
      pass_ip<2, SW, DIF, 2>(buf, NA, Ms, n, L, pt, sign);
    else
      pass_ip<3, SW, DIF, 2>(buf, NA, Ms, n, L, pt, sign);
  } else {
    if (R == 8)
      pass_ip<8, SW, DIF, 1>(buf, NA, Ms, n, L, pt, sign);
    else if (R == 4)
      pass_ip<4, SW, DIF, 1>(buf, NA, Ms, n, L, pt, sign);
    else if (R == 2)
      pass_ip<2, SW, DIF, 1>(buf, NA, Ms, n, L, pt, sign);
    else
      pass_ip<3, SW, DIF, 1>(buf, NA, Ms, n, L, pt, sign);
  }
}

// DIF: natural order in, digit-reversed out (in place)
template <bool SW, class C>
__device__ void fft_ip_dif(C* buf, int NA, int Ms, const FftPlan& fp, const C* __restrict__ pt, int sign) {
  int L = fp.n;
  for (int s = 0; s < fp.nstages; ++s) {
    const int R = fp.radix[s];
    pass_ip_r<SW, true>(R, buf, NA, Ms, fp.n, L, pt, sign);
    __syncthreads();
    pt += L / R;
    L /= R;
  }
}

// DIT: digit-reversed order in (as fft_ip_dif leaves it), natural out (in place)
template <bool SW, class C>
__device__ void fft_ip_dit(C* buf, int NA, int Ms, const FftPlan& fp, const C* __restrict__ pt, int sign) {
  for (int s = fp.nstages - 1; s >= 0; --s) {
    int L = fp.n, off = 0;  // block length and twiddle offset of pass s
    for (int t = 0; t < s; ++t) {
      off += L / fp.radix[t];
      L /= fp.radix[t];
    }
    pass_ip_r<SW, false>(fp.radix[s], buf, NA, Ms, fp.n, L, pt + off, sign);
    __syncthreads();
  }
}

__host__ __device__ inline int ip_twiddle_count(const FftPlan& fp) {
  int L = fp.n, c = 0;
  for (int s = 0; s < fp.nstages; ++s) {
    c += L / fp.radix[s];
    L /= fp.radix[s];
  }
  return c;
}

// Row advection products with the transforms in place (k_xprod's arithmetic,
// batched): per grid row z (and stacked instance y) the velocity spectrum and
// the three gradient spectra are built from one read of the six half-plane
// inputs, transformed to the padded grid together by DIF passes (results in
// digit-reversed order), multiplied pointwise, and the two product spectra
// go back by DIT passes into natural order for the truncation.  Shared
// memory: four arrays of the padded length and the in-place twiddles, so two
// CTAs share an SM at the 1536-point length in FP64.  Args: XProdArgs-like
// (ev, ov, ed, od, out, iptw, fp, Nx, Nk, M, Nz, k0, ld, instances).
template <int NT, class C, class Args>
__global__ void __launch_bounds__(NT, NT == 256 ? 2 : 1) k_xprod_ip(Args a) {
  using Rt = typename Real<C>::type;
  extern __shared__ __align__(16) unsigned char xip_raw[];
  C* sm = reinterpret_cast<C*>(xip_raw);
  const int M = a.M, N = a.Nx, Nk = a.Nk;
  const int Ms = (M + 7) & ~7;
  C* A = sm;
  C* tw = sm + 4 * Ms;
  const int hN = N / 2;
  for (int t = threadIdx.x; t < a.niptw; t += blockDim.x) tw[t] = a.iptw[t];
  const int z = blockIdx.x;
  const int zm = a.Nz - 1 - z;
  const bool lower = z <= zm;
  const size_t ld = a.ld > 0 ? (size_t)a.ld : (size_t)Nk, col0 = (size_t)blockIdx.y * Nk;
  const size_t rr = (size_t)(lower ? z : zm) * ld + col0;
  auto hbin = [&](C v, int q) -> C {
    if (q == 0) return mk<C>(v.x, Rt(0));
    if (q == hN) return mk<C>(Rt(0.5) * v.x, Rt(0));
    return v;
  };
  auto put2 = [&](C* dst, int q, C P, C Q) {  // spectrum of P + i Q (half spectra) on M points
    dst[fidx<true>(q)] = mk<C>(P.x - Q.y, P.y + Q.x);
    if (q > 0) dst[fidx<true>(M - q)] = mk<C>(P.x + Q.y, -P.y + Q.x);
  };
  for (int q = threadIdx.x; q <= hN; q += blockDim.x) {
    C g[3], d[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const C e = a.ev[f][rr + q], o = a.ov[f][rr + q];
      const C ed = a.ed[f][rr + q], od = a.od[f][rr + q];
      g[f] = lower ? mk<C>(e.x + o.x, e.y + o.y) : mk<C>(e.x - o.x, e.y - o.y);
      d[f] = lower ? mk<C>(ed.x + od.x, ed.y + od.y) : mk<C>(od.x - ed.x, od.y - ed.y);
    }
    put2(A, q, hbin(g[1], q), hbin(g[2], q));
    const Rt kk = a.k0 * (Rt)q;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      C Ax = mk<C>(Rt(0), Rt(0));
      if (q > 0 && q < hN) Ax = mk<C>(-kk * g[f].y, kk * g[f].x);  // i k g
      put2(A + (size_t)(1 + f) * Ms, q, Ax, hbin(d[f], q));
    }
  }
  for (int k = hN + 1 + threadIdx.x; k < M - hN; k += blockDim.x)  // bins N/2 < k < M - N/2 are zero
#pragma unroll
    for (int arr = 0; arr < 4; ++arr) A[(size_t)arr * Ms + fidx<true>(k)] = mk<C>(Rt(0), Rt(0));
  __syncthreads();
  fft_ip_dif<true>(A, 4, Ms, a.fp, tw, +1);
  // products at every (permuted) grid point: (b + i ux) into array 0, uz into array 1
  for (int p = threadIdx.x; p < M; p += blockDim.x) {
    const int ps = fidx<true>(p);
    const C u = A[ps];
    Rt pr[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const C gg = A[(size_t)(1 + f) * Ms + ps];
      pr[f] = -(u.x * gg.x + u.y * gg.y);
    }
    A[ps] = mk<C>(pr[0], pr[1]);
    A[(size_t)Ms + ps] = mk<C>(pr[2], Rt(0));
  }
  __syncthreads();
  fft_ip_dit<true>(A, 2, Ms, a.fp, tw, -1);
  const C* C1 = A;
  const C* C2 = A + Ms;
  const Rt sc = Rt(1) / ((Rt)M * (Rt)N);
  const size_t ro = (size_t)z * ld + col0;
  for (int k = threadIdx.x; k < Nk; k += blockDim.x) {
    const C c = C1[fidx<true>(k)];
    const C cm = C1[fidx<true>((M - k) % M)];
    const C sb = mk<C>(Rt(0.5) * (c.x + cm.x), Rt(0.5) * (c.y - cm.y));
    const C su = mk<C>(Rt(0.5) * (c.y + cm.y), Rt(-0.5) * (c.x - cm.x));
    const C c2 = C2[fidx<true>(k)];
    C ob, ou, oz;
    if (k == 0) {
      ob = mk<C>(sb.x * sc, Rt(0));
      ou = mk<C>(su.x * sc, Rt(0));
      oz = mk<C>(c2.x * sc, Rt(0));
    } else if (k == hN) {
      ob = mk<C>(Rt(2) * sb.x * sc, Rt(0));
      ou = mk<C>(Rt(2) * su.x * sc, Rt(0));
      oz = mk<C>(Rt(2) * c2.x * sc, Rt(0));
    } else {
      ob = mk<C>(sb.x * sc, sb.y * sc);
      ou = mk<C>(su.x * sc, su.y * sc);
      oz = mk<C>(c2.x * sc, c2.y * sc);
    }
    a.out[0][ro + k] = ob;
    a.out[1][ro + k] = ou;
    a.out[2][ro + k] = oz;
  }
}

template <class C>
inline size_t xprod_ip_smem_bytes(int M, int niptw) {
  const size_t Ms = (size_t)((M + 7) & ~7);
  return (4 * Ms + (size_t)niptw) * sizeof(C);
}

}  // namespace fftg
}  // namespace tb
