// Chebyshev transform GEMMs of the mixed-precision RHS on the 5th-generation
// tensor cores: tcgen05.mma kind::tf32 with the operands in shared memory and
// the FP32 accumulator in tensor memory, FP32 accuracy from three TF32
// products per term (split a = a_hi + a_lo, b = b_hi + b_lo, sum
// a_hi b_hi + a_hi b_lo + a_lo b_hi; the a_lo b_lo term is below FP32
// rounding).  Same contract and row maps as k_gemm_f32 (tb_mixed.cu):
// C (M x ncol) = A (M x K) . B' (K x ncol), B' row k = B[k] (plain),
// B[2k + par] (parity), B[j] + sgn B[N-1-j] (mirror, output row 2r + par).
//
// One CTA of 4 warps owns one item and a strided set of 64-column tiles.
// Operands are split into TF32 hi/lo while they are staged: A rows as float4
// chunks, B as four K-consecutive values of one column per thread, each
// written as one 16-byte swizzled chunk (the eight lanes of a shared-memory
// phase hit eight distinct chunks: no bank conflicts).  The accumulator goes
// back through shared memory so the global stores are row-contiguous.
// Shared memory (1024-byte aligned, the 128-byte swizzle's period):
//   A_hi, A_lo: 128 x 128 TF32, K-major, 128-byte swizzle, loaded once;
//   B_hi, B_lo:  64 x 128 TF32, K-major, 128-byte swizzle, one tile at a time.
// A K-major tile is stored as [k / 32][row][128 B] with 8-row atoms of 1024 B
// (stride byte offset 1024) and the 16-byte chunk index of a row XORed with
// row % 8.  One thread issues the 3 x K/8 MMAs (M 128, N 64, K 8 each),
// commits them to an mbarrier, and every warp then reads its 32 accumulator
// lanes (rows) with tcgen05.ld and stores them.  M <= 128 and K <= 128
// (Chebyshev degrees up to 256); larger shapes use k_gemm_f32.
#include <cuda_runtime.h>

#include <cstdint>

#include "tb_kernels.cuh"

namespace tb {

namespace {

constexpr int kTcM = 128, kTcN = 64, kTcK = 128, kTcThreads = 128;
constexpr uint32_t kABytes = kTcM * kTcK * 4;  // one TF32 copy of the A tile
constexpr uint32_t kBBytes = kTcN * kTcK * 4;  // one TF32 copy of a B tile
constexpr uint32_t kOffAhi = 0, kOffAlo = kABytes, kOffBhi = 2 * kABytes, kOffBlo = 2 * kABytes + kBBytes;
constexpr uint32_t kOffBar = 2 * kABytes + 2 * kBBytes;  // mbarrier (8 B), then the TMEM address (4 B)
constexpr uint32_t kTcSmem = kOffBar + 64 + 1024;        // + alignment slack
constexpr uint32_t kTmemCols = 64;                       // N fp32 accumulator columns
// spin limit of the MMA-completion wait (about a second); past it the CTA
// flags the error and skips its stores
constexpr long long kTcSpinLimit = 1LL << 26;

__device__ int g_tc_timeout;  // set when a wait ran out (read by tc32_status)

// byte offset of element (row r, column k) in a K-major, 128-byte swizzled
// tile of `rows` rows (K-atoms of 32 TF32 elements stored one after another)
__device__ __forceinline__ uint32_t sw128_off(int r, int k, int rows) {
  return (uint32_t)((k >> 5) * rows * 128 + (r >> 3) * 1024 + (r & 7) * 128 + ((((k & 31) >> 2) ^ (r & 7)) << 4) +
                    ((k & 3) << 2));
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row atoms
// 1024 B apart (bits: start >> 4 [0,14), LBO >> 4 [16,30) = 1 (unused by the
// swizzled K-major form), SBO >> 4 [32,46), version 1 [46,48), layout 2 =
// SWIZZLE_128B [61,64))
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// instruction descriptor: D F32 [4,6) = 1, A TF32 [7,10) = 2, B TF32 [10,13) = 2,
// both K-major, N >> 3 [17,23), M >> 4 [24,29)
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcN >> 3) << 17) |
                              ((uint32_t)(kTcM >> 4) << 24);

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void split_store4(uint8_t* base_hi, uint8_t* base_lo, uint32_t off, float4 v) {
  const uint32_t h0 = to_tf32(v.x), h1 = to_tf32(v.y), h2 = to_tf32(v.z), h3 = to_tf32(v.w);
  *reinterpret_cast<uint4*>(base_hi + off) = make_uint4(h0, h1, h2, h3);
  *reinterpret_cast<uint4*>(base_lo + off) =
      make_uint4(to_tf32(v.x - __uint_as_float(h0)), to_tf32(v.y - __uint_as_float(h1)),
                 to_tf32(v.z - __uint_as_float(h2)), to_tf32(v.w - __uint_as_float(h3)));
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate));
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

template <class OutT>
__global__ void __launch_bounds__(kTcThreads, 1) k_gemm_tc32(GemmBatch32 bt, int ncol, int ldb, int ldc, int Nrows) {
  extern __shared__ uint8_t tc_smem_raw[];
  const uint32_t raw = (uint32_t)__cvta_generic_to_shared(tc_smem_raw);
  const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
  uint8_t* sm = tc_smem_raw + pad;
  const uint32_t sbase = raw + pad;
  const uint32_t bar = sbase + kOffBar;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kOffBar + 8);

  const GemmItem32& it = bt.item[blockIdx.z];
  const float* __restrict__ A = it.A;
  const float* __restrict__ B = it.B;
  const int Mo = it.M, K = it.K, Kp = it.Kpad, mode = it.mode, par = it.par;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int ntiles = (ncol + kTcN - 1) / kTcN;
  const bool mirror = mode == GEMM_MIRROR;
  const float sgn = par ? -1.f : 1.f;
  const int midk = (mirror && (Nrows & 1)) ? (Nrows - 1) / 2 : -1;
  const int nk8 = (K + 7) / 8;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sbase + kOffBar + 8),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  // A once, four K-consecutive values per thread and step (Kpad is a multiple
  // of 16 and the padding columns are zero); rows >= M are zero
  // (eight loads in flight per thread before any is split and stored)
  constexpr int AQ = kTcM * (kTcK / 4) / kTcThreads, AB = 8;  // float4 per thread, per batch
  static_assert(AQ % AB == 0, "A batches");
  for (int q0 = 0; q0 < AQ; q0 += AB) {
    float4 v[AB];
#pragma unroll
    for (int i = 0; i < AB; ++i) {
      const int idx = tid + (q0 + i) * kTcThreads;
      const int r = idx / (kTcK / 4), k = 4 * (idx % (kTcK / 4));
      v[i] = (r < Mo && k < Kp) ? *reinterpret_cast<const float4*>(A + (size_t)r * Kp + k)
                                : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int i = 0; i < AB; ++i) {
      const int idx = tid + (q0 + i) * kTcThreads;
      split_store4(sm + kOffAhi, sm + kOffAlo, sw128_off(idx / (kTcK / 4), 4 * (idx % (kTcK / 4)), kTcM), v[i]);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;

  uint32_t phase = 0;
  bool ok = true;
  for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
    const int n0 = t * kTcN;
    // B' tile: thread (column n, K-chunk kc) loads rows 4 kc .. 4 kc + 3 of
    // column n0 + n (the lanes of a warp read consecutive columns of one row)
    {
      const int n = tid % kTcN, gc = n0 + n;
      const bool colok = gc < ncol;
      constexpr int KCS = kTcThreads / kTcN;       // K-chunks started per step (2)
      constexpr int NKC = kTcK / 4 / KCS;          // K-chunks per thread (16)
      constexpr int CB = 4;                        // chunks per batch: 16 loads in flight
      static_assert(NKC % CB == 0, "B batches");
      for (int c0 = 0; c0 < NKC; c0 += CB) {
        float e[CB][4], w[CB][4];
#pragma unroll
        for (int c = 0; c < CB; ++c)
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int k = 4 * (tid / kTcN + (c0 + c) * KCS) + i;
            const bool ok = colok && k < K;
            const int srow = mode == GEMM_PARITY ? 2 * k + par : k;
            e[c][i] = ok ? B[(size_t)srow * ldb + gc] : 0.f;
            w[c][i] = (ok && mirror && k != midk) ? B[(size_t)(Nrows - 1 - k) * ldb + gc] : 0.f;
          }
#pragma unroll
        for (int c = 0; c < CB; ++c) {
          const int kc = tid / kTcN + (c0 + c) * KCS;
          float f[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int k = 4 * kc + i;
            f[i] = mirror ? ((k == midk) ? (par ? 0.f : e[c][i]) : fmaf(sgn, w[c][i], e[c][i])) : e[c][i];
          }
          split_store4(sm + kOffBhi, sm + kOffBlo, sw128_off(n, 4 * kc, kTcN), make_float4(f[0], f[1], f[2], f[3]));
        }
      }
    }
    // generic-proxy stores -> visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    if (tid == 0) {
      for (int j = 0; j < nk8; ++j) {
        const uint32_t ka = (uint32_t)(j >> 2) * (kTcM * 128) + (uint32_t)(j & 3) * 32;
        const uint32_t kb = (uint32_t)(j >> 2) * (kTcN * 128) + (uint32_t)(j & 3) * 32;
        const uint64_t ahi = sw128_desc(sbase + kOffAhi + ka), alo = sw128_desc(sbase + kOffAlo + ka);
        const uint64_t bhi = sw128_desc(sbase + kOffBhi + kb), blo = sw128_desc(sbase + kOffBlo + kb);
        mma_tf32(tmem, ahi, bhi, j > 0 ? 1u : 0u);
        mma_tf32(tmem, ahi, blo, 1u);
        mma_tf32(tmem, alo, bhi, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                   : "memory");
    }
    long long spins = 0;
    bool done = true;
    while (!mbar_try_wait(bar, phase)) {
      if (++spins > kTcSpinLimit) {
        done = false;
        break;
      }
    }
    phase ^= 1u;
    ok = __syncthreads_and(done) != 0;  // one decision for the whole CTA
    if (!ok) {
      if (tid == 0) atomicExch(&g_tc_timeout, 1);
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const int r = warp * 32 + lane;  // accumulator lane = output row of this thread
    OutT* stage = reinterpret_cast<OutT*>(sm + kOffBhi);  // [row][33]: the MMAs no longer read B
    constexpr int SLD = 33;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(half * 32);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
      for (int c = 0; c < 32; ++c) stage[r * SLD + c] = (OutT)__uint_as_float(v[c]);
      __syncthreads();
      // row-contiguous stores: a warp writes 32 consecutive columns of one row
      for (int idx = tid; idx < kTcM * 32; idx += kTcThreads) {
        const int rr = idx / 32, c = idx % 32;
        const int gc = n0 + half * 32 + c;
        if (rr < Mo && gc < ncol) {
          const int orow = mirror ? 2 * rr + par : rr;
          reinterpret_cast<OutT*>(it.C)[(size_t)orow * ldc + gc] = stage[rr * SLD + c];
        }
      }
      __syncthreads();
    }
    // every warp has read the accumulator and the MMAs have read B: the next
    // tile may overwrite both
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  }
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

bool gemm_tc32_supported(const GemmBatch32& bt, int nbatch) {
  for (int b = 0; b < nbatch; ++b)
    if (bt.item[b].M > kTcM || bt.item[b].K > kTcK) return false;
  return true;
}

cudaError_t set_tc32_smem_limits() {
  cudaError_t e = cudaFuncSetAttribute(k_gemm_tc32<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_gemm_tc32<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
}

namespace {
int tc32_ctas_per_item(int ncol, int nbatch) {
  const int ntiles = (ncol + kTcN - 1) / kTcN;
  int per = 148 / nbatch;  // one wave of CTAs (one per SM by shared memory)
  if (per < 1) per = 1;
  if (per > ntiles) per = ntiles;
  return per;
}
}  // namespace

int gemm_tc32_tiles_per_cta(int ncol, int nbatch) {
  const int ntiles = (ncol + kTcN - 1) / kTcN;
  const int per = tc32_ctas_per_item(ncol, nbatch);
  return (ntiles + per - 1) / per;
}

void launch_gemm_tc32(const GemmBatch32& bt, int nbatch, int ncol, int ldb, int ldc, int Nrows, bool out_f64,
                      cudaStream_t st) {
  const int per = tc32_ctas_per_item(ncol, nbatch);
  dim3 grid(per, 1, nbatch);
  if (out_f64)
    k_gemm_tc32<double><<<grid, kTcThreads, kTcSmem, st>>>(bt, ncol, ldb, ldc, Nrows);
  else
    k_gemm_tc32<float><<<grid, kTcThreads, kTcSmem, st>>>(bt, ncol, ldb, ldc, Nrows);
}

int tc32_status() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_tc_timeout, sizeof(int)) != cudaSuccess) return -1;
  return v;
}

}  // namespace tb
