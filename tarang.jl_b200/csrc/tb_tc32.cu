// Chebyshev transform GEMMs of the mixed-precision RHS on the 5th-generation
// tensor cores: tcgen05.mma kind::tf32 with the operands in shared memory and
// the FP32 accumulator in tensor memory, FP32 accuracy from three TF32
// products per term (split a = a_hi + a_lo, b = b_hi + b_lo, sum
// a_hi b_hi + a_hi b_lo + a_lo b_hi; the a_lo b_lo term is below FP32
// rounding).  Same contract and row maps as k_gemm_f32 (tb_mixed.cu):
// C (M x ncol) = A (M x K) . B' (K x ncol), B' row k = B[k] (plain),
// B[2k + par] (parity), B[j] + sgn B[N-1-j] (mirror, output row 2r + par).
//
// Operand images.  The tensor cores read K-major tiles with the 128-byte
// swizzle: a tile of `rows` rows is stored as [k / 32][row][128 B], 8-row atoms
// of 1024 B (stride byte offset 1024), the 16-byte chunk index of a row XORed
// with row % 8.  Both operands are prepared in global memory in exactly that
// form, TF32 hi part then lo part:
//   A (the constant transform matrix, M <= 128, K <= 128): once per plan,
//     128 KB (k_tc32_image_a);
//   B' (the data): per call, one 64 KB image per 64-column tile of every
//     distinct input (k_tc32_image_b; the value and derivative matrices of a
//     field share one input), the parity / mirror row maps applied while the
//     image is written.
// The GEMM kernel then moves operands with bulk copies (cp.async.bulk, one
// thread, completion on an mbarrier): A once per CTA, B one tile ahead - the
// next tile's copy is issued as soon as the MMAs of the current one have
// completed, so it overlaps the epilogue.  One CTA of 4 warps owns one item
// and a strided set of 64-column tiles; one thread issues the 3 x K/8 MMAs
// (M 128, N 64, K 8 each) and commits them to an mbarrier; every warp reads its
// 32 accumulator lanes (rows) with tcgen05.ld and the tile leaves through a
// shared-memory stage for row-contiguous stores.  Every wait is bounded.
//
// Streaming form for the 3D planes (k_tc32s, Nz <= 128): the raw FP32 input
// planes are read by TMA tile by tile (N <= 128 rows x 32 columns, no swizzle) and
// split into the TF32 hi / lo images in shared memory by the CTA's own
// threads; the row maps are folded into constant A operands instead:
//   backward (value and z-derivative on the half grid from the even and odd
//     coefficients): per parity p one A of 128 rows, [value rows; derivative
//     rows] of that parity's columns, times B_p = the tile's rows 2k + p;
//   forward (the C^(2) coefficients 2r + par from the grid): one A of 128
//     rows, [even outputs; odd outputs] over all N grid rows, the mirror sum
//     B[j] + sgn B[N-1-j] folded into the columns (A'[r][j] = A[r][j] for
//     j < N/2, sgn A[r][N-1-j] above), times the tile's N natural rows.
// One persistent CTA per SM runs (field, 32-column tile) tasks with its warps
// specialised: TMA loads, the split, the MMAs (into one of two accumulator
// buffers in tensor memory) and the epilogue of consecutive tiles overlap.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "tb_kernels.cuh"

namespace tb {

namespace {

constexpr int kTcM = 128, kTcN = 64, kTcK = 128, kTcThreads = 128;
constexpr uint32_t kABytes = kTcM * kTcK * 4;  // one TF32 copy of the A tile
constexpr uint32_t kBBytes = kTcN * kTcK * 4;  // one TF32 copy of a B tile
constexpr uint32_t kOffAhi = 0, kOffAlo = kABytes, kOffBhi = 2 * kABytes, kOffBlo = 2 * kABytes + kBBytes;
constexpr int kStageLd = 33;                                         // epilogue stage row stride (elements)
constexpr uint32_t kOffStage = 2 * kABytes + 2 * kBBytes;            // [row][33] of the output type
constexpr uint32_t kOffBar = kOffStage + kTcM * kStageLd * 8;        // mbarriers A, B, MMA (8 B each), TMEM address
constexpr uint32_t kTcSmem = kOffBar + 64 + 1024;                    // + alignment slack
static_assert(kTcSmem <= 232448, "one CTA per SM");
constexpr uint32_t kTmemCols = 64;                                   // N fp32 accumulator columns
constexpr uint32_t kImageChunk = 16384;                              // bytes per bulk copy
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

// bounded wait on an mbarrier phase: false after kTcSpinLimit polls
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  long long spins = 0;
  while (!mbar_try_wait(bar, parity))
    if (++spins > kTcSpinLimit) return false;
  return true;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

// bytes (a multiple of kImageChunk) from global src to shared dst, completing on bar
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  for (uint32_t o = 0; o < bytes; o += kImageChunk)
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst + o),
        "l"(static_cast<const char*>(src) + o), "r"(kImageChunk), "r"(bar)
        : "memory");
}

// A image: rows r < M of A (row stride Kpad, columns past K zero), four
// K-consecutive values per thread and step, split into TF32 hi / lo.
__global__ void __launch_bounds__(kTcThreads) k_tc32_image_a(const float* __restrict__ A, int M, int Kp,
                                                             float* __restrict__ image) {
  uint8_t* hi = reinterpret_cast<uint8_t*>(image);
  uint8_t* lo = hi + kABytes;
  for (int idx = threadIdx.x; idx < kTcM * (kTcK / 4); idx += kTcThreads) {
    const int r = idx / (kTcK / 4), k = 4 * (idx % (kTcK / 4));
    const float4 v = (r < M && k < Kp) ? *reinterpret_cast<const float4*>(A + (size_t)r * Kp + k)
                                       : make_float4(0.f, 0.f, 0.f, 0.f);
    split_store4(hi, lo, sw128_off(r, k, kTcM), v);
  }
}

// B' images: one CTA per (64-column tile, distinct input); thread (column n,
// K-chunk kc) gathers rows 4 kc .. 4 kc + 3 of column n0 + n through the row
// map (sixteen loads in flight, mirror partners included) and writes them as
// one swizzled 16-byte chunk of each of the hi and lo parts.
struct Tc32BInput {
  const float* B;
  float* image;  // ntiles images of 2 kBBytes
  int K, mode, par;
};
struct Tc32BInputs {
  Tc32BInput in[kGemmMaxBatch];
};
__global__ void __launch_bounds__(kTcThreads) k_tc32_image_b(Tc32BInputs bi, int ncol, int ldb, int Nrows) {
  const Tc32BInput& im = bi.in[blockIdx.y];
  const float* __restrict__ B = im.B;
  const int K = im.K, mode = im.mode, par = im.par;
  const bool mirror = mode == GEMM_MIRROR;
  const float sgn = par ? -1.f : 1.f;
  const int midk = (mirror && (Nrows & 1)) ? (Nrows - 1) / 2 : -1;
  const int tid = threadIdx.x, n0 = blockIdx.x * kTcN;
  uint8_t* hi = reinterpret_cast<uint8_t*>(im.image) + (size_t)blockIdx.x * 2 * kBBytes;
  uint8_t* lo = hi + kBBytes;
  const int n = tid % kTcN, gc = n0 + n;
  const bool colok = gc < ncol;
  constexpr int KCS = kTcThreads / kTcN;  // K-chunks started per step (2)
  constexpr int NKC = kTcK / 4 / KCS;     // K-chunks per thread (16)
  constexpr int CB = 4;                   // chunks per batch: 16 loads in flight
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
      split_store4(hi, lo, sw128_off(n, 4 * kc, kTcN), make_float4(f[0], f[1], f[2], f[3]));
    }
  }
}

template <class OutT>
__global__ void __launch_bounds__(kTcThreads, 1) k_gemm_tc32(GemmBatch32 bt, int ncol, int ldc) {
  extern __shared__ uint8_t tc_smem_raw[];
  const uint32_t raw = (uint32_t)__cvta_generic_to_shared(tc_smem_raw);
  const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
  uint8_t* sm = tc_smem_raw + pad;
  const uint32_t sbase = raw + pad;
  const uint32_t barA = sbase + kOffBar, barB = barA + 8, barM = barA + 16;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kOffBar + 24);

  const GemmItem32& it = bt.item[blockIdx.z];
  const int Mo = it.M, K = it.K, mode = it.mode, par = it.par;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int ntiles = (ncol + kTcN - 1) / kTcN;
  const bool mirror = mode == GEMM_MIRROR;
  const int nk8 = (K + 7) / 8;
  const int t0 = blockIdx.x;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sbase + kOffBar + 24),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  // copies in flight (issued by thread 0, waited by every thread)
  bool a_pending = false, b_pending = false;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(barA));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(barB));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(barM));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    mbar_expect_tx(barA, 2 * kABytes);
    bulk_copy(sbase + kOffAhi, it.Aimg, 2 * kABytes, barA);
    if (t0 < ntiles) {
      mbar_expect_tx(barB, 2 * kBBytes);
      bulk_copy(sbase + kOffBhi, it.Bimg + (size_t)t0 * (2 * kBBytes / 4), 2 * kBBytes, barB);
    }
  }
  a_pending = true;
  b_pending = t0 < ntiles;
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;

  uint32_t pb = 0, pm = 0;
  bool ok = __syncthreads_and(mbar_wait_bounded(barA, 0)) != 0;  // one decision for the whole CTA
  if (ok) a_pending = false;
  bool mma_pending = false;
  for (int t = t0; t < ntiles && ok; t += gridDim.x) {
    const int n0 = t * kTcN;
    ok = __syncthreads_and(mbar_wait_bounded(barB, pb)) != 0;
    if (!ok) break;
    b_pending = false;
    pb ^= 1u;
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
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(barM)
                   : "memory");
    }
    mma_pending = true;
    ok = __syncthreads_and(mbar_wait_bounded(barM, pm)) != 0;
    if (!ok) break;
    mma_pending = false;
    pm ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    // the MMAs have read B: the next tile's image streams in during the epilogue
    const int tn = t + gridDim.x;
    if (tn < ntiles) {
      if (tid == 0) {
        mbar_expect_tx(barB, 2 * kBBytes);
        bulk_copy(sbase + kOffBhi, it.Bimg + (size_t)tn * (2 * kBBytes / 4), 2 * kBBytes, barB);
      }
      b_pending = true;
    }
    const int r = warp * 32 + lane;  // accumulator lane = output row of this thread
    OutT* stage = reinterpret_cast<OutT*>(sm + kOffStage);
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
      for (int c = 0; c < 32; ++c) stage[r * kStageLd + c] = (OutT)__uint_as_float(v[c]);
      __syncthreads();
      // row-contiguous stores: a warp writes 32 consecutive columns of one row
      for (int idx = tid; idx < kTcM * 32; idx += kTcThreads) {
        const int rr = idx / 32, c = idx % 32;
        const int gc = n0 + half * 32 + c;
        if (rr < Mo && gc < ncol) {
          const int orow = mirror ? 2 * rr + par : rr;
          reinterpret_cast<OutT*>(it.C)[(size_t)orow * ldc + gc] = stage[rr * kStageLd + c];
        }
      }
      __syncthreads();
    }
    // every warp has read the accumulator: the next tile's MMAs may overwrite it
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  }
  if (!ok) {
    // a wait ran out: flag it, give the copies and MMAs still in flight a
    // bounded time to land (they write this CTA's shared and tensor memory)
    if (tid == 0) {
      atomicExch(&g_tc_timeout, 1);
      if (a_pending) mbar_wait_bounded(barA, 0);
      if (b_pending) mbar_wait_bounded(barB, pb);
      if (mma_pending) mbar_wait_bounded(barM, pm);
    }
  }
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols));
}


// ---- streaming form (3D planes) ----
constexpr int kSN = 64;                                  // columns per tile (the MMA's N)
constexpr int kSRows = 128;                              // input rows per tile (N <= 128)
constexpr int kSNR = 2;                                  // raw tile stages
constexpr int kSNH = 2;                                  // hi / lo image stages
constexpr uint32_t kSRawBytes = kSRows * kSN * 4;        // 32 KB raw tile
constexpr uint32_t kSHiloBytes = 2 * kSRows * kSN * 4;   // 64 KB of hi and lo images
constexpr uint32_t kSAtom = kSN * 128;                   // bytes of one 32-wide K atom of a B image
constexpr uint32_t kSOffRaw = 0;
constexpr uint32_t kSOffB = kSOffRaw + kSNR * kSRawBytes;
constexpr uint32_t kSOffBar = kSOffB + kSNH * kSHiloBytes;  // mbarriers, TMEM address, abort flag
constexpr uint32_t kSSmem = kSOffBar + 256 + 1024;          // + alignment slack
static_assert(kSSmem <= 232448, "one CTA per SM");
// Tensor memory: the A operands (hi and lo, 256 columns: backward parity p
// hi / lo at 64 (2p + h), forward hi at 0, lo at 128), then two accumulator
// buffers of 128 columns from column 256 (backward parity p at + 64 p).
constexpr uint32_t kSTmemCols = 512;
constexpr uint32_t kSTmemAcc = 256;
constexpr size_t kSImageFloats = 2 * 2 * 128 * 64 + 2 * 128 * 128;  // backward parts (K 64), forward (K 128)
// instruction descriptor: D F32, A and B TF32, both K-major, N 64, M 128
constexpr uint32_t kSIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kSN >> 3) << 17) |
                             ((uint32_t)(kTcM >> 4) << 24);

// D (tensor memory) += A (tensor memory, 128 lanes x 8 columns) . B (shared memory)
__device__ __forceinline__ void mma_tf32_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(bdesc), "r"(kSIdesc), "r"(accumulate));
}

// TF32 hi / lo parts of the streaming form's A operands, row-major (128 rows
// of K values each, the layout the epilogue warps copy into tensor memory):
// blockIdx.x 0 and 1 the backward parities (K 64: rows r < 64 value, r >= 64
// derivative, of the columns 2k + p), 2 the forward operand (K 128, the mirror
// folded in, rows r < 64 the even outputs 2r, r >= 64 the odd ones).
// Parts: backward parity p hi at 2p, lo at 2p + 1 (128 x 64 each), then the
// forward hi and lo (128 x 128 each).
__global__ void __launch_bounds__(kTcThreads) k_tc32s_image(const float* __restrict__ Ev, const float* __restrict__ Ov,
                                                            const float* __restrict__ Ed, const float* __restrict__ Od,
                                                            int kpe, int kpo, const float* __restrict__ sfE,
                                                            const float* __restrict__ sfO, int kph, int N,
                                                            float* __restrict__ images) {
  const int H = N / 2, Ke = (N + 1) / 2, Ko = N / 2;
  const int img = blockIdx.x;
  const int kt = img < 2 ? 64 : 128;  // K extent of this operand
  float* hi = images + (size_t)(img < 2 ? img : 2) * 2 * 128 * 64;
  float* lo = hi + (size_t)128 * kt;
  for (int idx = threadIdx.x; idx < 128 * kt; idx += kTcThreads) {
    const int r = idx / kt, k = idx % kt;
    float v = 0.f;
    if (img < 2) {
      const int p = img, K = p ? Ko : Ke, kp = p ? kpo : kpe, rr = r & 63;
      const float* src = r < 64 ? (p ? Ov : Ev) : (p ? Od : Ed);
      if (rr < H && k < K) v = src[(size_t)rr * kp + k];
    } else {
      const int par = r >= 64, rr = r & 63, M = par ? Ko : Ke;
      const float* src = par ? sfO : sfE;
      if (rr < M && k < N) v = k < H ? src[(size_t)rr * kph + k] : (par ? -1.f : 1.f) * src[(size_t)rr * kph + (N - 1 - k)];
    }
    const uint32_t h = to_tf32(v);
    hi[idx] = __uint_as_float(h);
    lo[idx] = __uint_as_float(to_tf32(v - __uint_as_float(h)));
  }
}

// 3D tile load: 64 columns x N rows of field z from the tensor map into dst
__device__ __forceinline__ void tma_load_tile(uint32_t dst, const CUtensorMap* map, int x, int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(0), "r"(z), "r"(bar)
      : "memory");
}

// Roles (10 warps): warps 0-3 the epilogue (warp w owns tensor-memory lanes
// 32w..32w+31; before the tiles they copy the A operands into tensor memory),
// warps 4-7 the split, warp 8 the TMA producer, warp 9 the MMA issuer.  Raw
// stage i % kSNR, hi / lo stage i % kSNH and accumulator buffer i % 2 of tile
// i; the hand-offs are mbarriers: aload (A in tensor memory -> MMA), full (TMA
// -> split), rawfree (split -> producer), splitfull (split -> MMA), hilofree
// and accfull (MMA completion, by tcgen05.commit), accfree (epilogue -> MMA).
// A in tensor memory leaves the MMAs only B to read from shared memory and
// the shared memory to tiles of 64 columns (N 64 per MMA: half the MMA
// instructions per column of N 32, whose fixed cost per instruction bounded
// the kernel).  The epilogue reads the accumulator in the 16 x 256-bit shape
// (four lanes per row, two columns each), so that every store of a warp
// writes whole 32-byte sectors straight from registers.
constexpr int kSSplitWarps = 4;  // warps of the split role
constexpr int kSSplitThreads = 32 * kSSplitWarps;
constexpr int kSEpi = 0, kSSplit = 4, kSProd = kSSplit + kSSplitWarps, kSMma = kSProd + 1;  // first warp of each role
constexpr int kSThreads = 32 * (kSMma + 2);  // two MMA issuer warps

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}

// bounded wait that also gives up once another role has aborted
__device__ __forceinline__ bool mbar_wait_or_abort(uint32_t bar, uint32_t parity, volatile int* abort) {
  long long spins = 0;
  while (!mbar_try_wait(bar, parity)) {
    ++spins;
    if ((spins & 255) == 0 && *abort) return false;
    if (spins > kTcSpinLimit) {
      *abort = 1;
      return false;
    }
  }
  return true;
}

// BWD: C_w (H x ncol, w = p + 2 d for parity p, derivative d) of each field
// f at out + (4 f + w) * H * ncol; forward: rows 2r + par of each field at
// out + f * N * ncol (FP64).
template <bool BWD>
__global__ void __launch_bounds__(kSThreads, 1) k_tc32s(const __grid_constant__ CUtensorMap map,
                                                        const float* __restrict__ images, void* out, int nfields,
                                                        int N, int ncol) {
  extern __shared__ uint8_t tc_smem_raw[];
  const uint32_t raw = (uint32_t)__cvta_generic_to_shared(tc_smem_raw);
  const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
  uint8_t* sm = tc_smem_raw + pad;
  const uint32_t sbase = raw + pad;
  // mbarriers: aload, full[kSNR], rawfree[kSNR], splitfull[kSNH], hilofree[kSNH], accfull[2], accfree[2]
  const uint32_t barL = sbase + kSOffBar;
  auto barFull = [&](int r) { return barL + 8u + 8u * (uint32_t)r; };
  auto barRawFree = [&](int r) { return barL + 8u + 8u * (uint32_t)(kSNR + r); };
  auto barSplitFull = [&](int h) { return barL + 8u + 8u * (uint32_t)(2 * kSNR + h); };
  auto barHiloFree = [&](int h) { return barL + 8u + 8u * (uint32_t)(2 * kSNR + kSNH + h); };
  auto barAccFull = [&](int a) { return barL + 8u + 8u * (uint32_t)(2 * kSNR + 2 * kSNH + a); };
  auto barAccFree = [&](int a) { return barL + 8u + 8u * (uint32_t)(2 * kSNR + 2 * kSNH + 2 + a); };
  constexpr uint32_t kBarBytes = 8u * (1 + 2 * kSNR + 2 * kSNH + 4);
  static_assert(kBarBytes + 16 <= 256, "barrier area");
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kSOffBar + kBarBytes);
  volatile int* abort = reinterpret_cast<volatile int*>(sm + kSOffBar + kBarBytes + 8);
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int H = N / 2, Ke = (N + 1) / 2, Ko = N / 2;
  const int ntiles = (ncol + kSN - 1) / kSN;
  const int ntask = nfields * ntiles;
  const uint32_t tile_bytes = (uint32_t)(kSN * N * 4);  // one TMA box: 64 columns x N rows
  // local tiles i = 0 .. n-1 are the tasks blockIdx.x + i gridDim.x
  const int n = blockIdx.x < ntask ? (ntask - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto task = [&](int i, int* f, int* n0) {
    const int t = blockIdx.x + i * gridDim.x;
    *f = t / ntiles;
    *n0 = (t % ntiles) * kSN;
  };
  // phase parity of tile i's use of a ring of depth D, and of tile i - D's
  auto ph = [](int i, int D) { return (uint32_t)(i / D) & 1u; };
  auto ph_prev = [](int i, int D) { return (uint32_t)(i / D - 1) & 1u; };

  if (warp == kSEpi) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sbase + kSOffBar +
                                                                                            kBarBytes),
                 "r"(kSTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    *abort = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;\n" ::"r"(barL));
    for (int r = 0; r < kSNR; ++r) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(barFull(r)));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(barRawFree(r)), "r"(kSSplitThreads));
    }
    // hilofree and accfull complete on the commits of both MMA issuers
    for (int h = 0; h < kSNH; ++h) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(barSplitFull(h)), "r"(kSSplitThreads));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;\n" ::"r"(barHiloFree(h)));
    }
    for (int a = 0; a < 2; ++a) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;\n" ::"r"(barAccFull(a)));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;\n" ::"r"(barAccFree(a)));
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;
  int last_load[kSNR], last_mma = -1;  // for the bounded drain after an abort
#pragma unroll
  for (int r = 0; r < kSNR; ++r) last_load[r] = -1;

  if (warp == kSProd) {
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&map)) : "memory");
      for (int i = 0; i < n; ++i) {
        const int r = i % kSNR;
        if (i >= kSNR && !mbar_wait_or_abort(barRawFree(r), ph_prev(i, kSNR), abort)) break;
        int f, n0;
        task(i, &f, &n0);
        mbar_expect_tx(barFull(r), tile_bytes);
        tma_load_tile(sbase + kSOffRaw + (uint32_t)r * kSRawBytes, &map, n0, f, barFull(r));
        last_load[r] = i;
      }
    }
  } else if (warp >= kSSplit && warp < kSSplit + kSSplitWarps) {
    const int t = tid - 32 * kSSplit;
    for (int i = 0; i < n; ++i) {
      const int r = i % kSNR, hs = i % kSNH;
      if (!mbar_wait_or_abort(barFull(r), ph(i, kSNR), abort)) break;
      if (i >= kSNH && !mbar_wait_or_abort(barHiloFree(hs), ph_prev(i, kSNH), abort)) break;
      // split the raw tile [row < N][64 columns] into the K-major hi / lo
      // images (rows past N are zero): backward, per parity a hi and a lo
      // image of K 64 (16 KB each); forward, hi and lo of K 128 (32 KB each)
      const float* rt = reinterpret_cast<const float*>(sm + kSOffRaw + (uint32_t)r * kSRawBytes);
      uint8_t* hb = sm + kSOffB + (uint32_t)hs * kSHiloBytes;
      auto row = [&](int j, int nn) { return j < N ? rt[(size_t)j * kSN + nn] : 0.f; };
      if constexpr (BWD) {
        for (int it = t; it < 2 * 16 * kSN; it += kSSplitThreads) {
          const int nn = it % kSN, kc = (it / kSN) % 16, p = it / (16 * kSN);
          const int j0 = 8 * kc + p;  // rows 2 (4 kc + i) + p
          const float4 v = make_float4(row(j0, nn), row(j0 + 2, nn), row(j0 + 4, nn), row(j0 + 6, nn));
          split_store4(hb + p * 32768, hb + p * 32768 + 16384, sw128_off(nn, 4 * kc, kSN), v);
        }
      } else {
        for (int it = t; it < 32 * kSN; it += kSSplitThreads) {
          const int nn = it % kSN, kc = it / kSN, j0 = 4 * kc;
          const float4 v = make_float4(row(j0, nn), row(j0 + 1, nn), row(j0 + 2, nn), row(j0 + 3, nn));
          split_store4(hb, hb + 32768, sw128_off(nn, 4 * kc, kSN), v);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      mbar_arrive(barRawFree(r));
      mbar_arrive(barSplitFull(hs));
    }
  } else if (warp == kSMma || warp == kSMma + 1) {
    // two issuers: backward, one parity each; forward, the first issues every
    // K step into one accumulator (splitting the steps over two accumulators
    // measured slower) and the second only commits
    const int jpar = warp - kSMma;
    if (lane == 0) {
      mbar_wait_or_abort(barL, 0, abort);  // A in tensor memory (sets the abort flag when it runs out)
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      for (int i = 0; i < n && !*abort; ++i) {
        const int hs = i % kSNH, a = i & 1;
        if (!mbar_wait_or_abort(barSplitFull(hs), ph(i, kSNH), abort)) break;
        if (i >= 2 && !mbar_wait_or_abort(barAccFree(a), ph_prev(i, 2), abort)) break;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        const uint32_t bb = sbase + kSOffB + (uint32_t)hs * kSHiloBytes;
        if constexpr (BWD) {
          {
            const int p = jpar;
            const uint32_t ahi = tmem + (uint32_t)(64 * (2 * p)), alo = tmem + (uint32_t)(64 * (2 * p + 1));
            const uint64_t bhi = sw128_desc(bb + (uint32_t)p * 32768u), blo = sw128_desc(bb + (uint32_t)p * 32768u + 16384u);
            const uint32_t d = tmem + kSTmemAcc + (uint32_t)(a * 128 + p * 64);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              // B: start-address field += byte offset / 16 (offsets stay below 256 KB); A: 8 columns per step
              const uint64_t kb = ((uint64_t)(j >> 2) * kSAtom + (uint64_t)(j & 3) * 32u) >> 4;
              mma_tf32_ts(d, ahi + 8u * j, bhi + kb, j > 0 ? 1u : 0u);
              mma_tf32_ts(d, ahi + 8u * j, blo + kb, 1u);
              mma_tf32_ts(d, alo + 8u * j, bhi + kb, 1u);
            }
          }
        } else {
          const uint32_t ahi = tmem, alo = tmem + 128u;
          const uint64_t bhi = sw128_desc(bb), blo = sw128_desc(bb + 32768u);
          const uint32_t d = tmem + kSTmemAcc + (uint32_t)(a * 128);
#pragma unroll
          for (int j = 0; j < (jpar == 0 ? 16 : 0); ++j) {
            const uint64_t kb = ((uint64_t)(j >> 2) * kSAtom + (uint64_t)(j & 3) * 32u) >> 4;
            mma_tf32_ts(d, ahi + 8u * j, bhi + kb, j > 0 ? 1u : 0u);
            mma_tf32_ts(d, ahi + 8u * j, blo + kb, 1u);
            mma_tf32_ts(d, alo + 8u * j, bhi + kb, 1u);
          }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         barHiloFree(hs))
                     : "memory");
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         barAccFull(a))
                     : "memory");
        last_mma = i;
      }
    }
  } else if (warp < kSEpi + 4) {
    // A operands into tensor memory: thread (warp w, lane l) owns row 32 w + l
    // and copies its K values of each part, 32 columns per store
    {
      const int r = warp * 32 + lane;
      constexpr int NPART = BWD ? 4 : 2, KP = BWD ? 64 : 128;
      const float* src = images + (BWD ? 0 : 2 * 2 * 128 * 64);
#pragma unroll 1
      for (int q = 0; q < NPART; ++q)
#pragma unroll 1
        for (int c = 0; c < KP / 32; ++c) {
          const float4* rowp = reinterpret_cast<const float4*>(src + ((size_t)q * 128 + r) * KP + 32 * c);
          uint32_t w[32];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const float4 x = rowp[k];
            w[4 * k] = __float_as_uint(x.x);
            w[4 * k + 1] = __float_as_uint(x.y);
            w[4 * k + 2] = __float_as_uint(x.z);
            w[4 * k + 3] = __float_as_uint(x.w);
          }
          const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(q * KP + 32 * c);
          asm volatile(
              "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
              "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};\n" ::"r"(taddr),
              "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]), "r"(w[8]),
              "r"(w[9]), "r"(w[10]), "r"(w[11]), "r"(w[12]), "r"(w[13]), "r"(w[14]), "r"(w[15]), "r"(w[16]),
              "r"(w[17]), "r"(w[18]), "r"(w[19]), "r"(w[20]), "r"(w[21]), "r"(w[22]), "r"(w[23]), "r"(w[24]),
              "r"(w[25]), "r"(w[26]), "r"(w[27]), "r"(w[28]), "r"(w[29]), "r"(w[30]), "r"(w[31])
              : "memory");
        }
      asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
      mbar_arrive(barL);
    }
    // 16 x 256-bit accumulator loads: lane l of the warp holds rows
    // l / 4 and l / 4 + 8 of a 16-row block, columns 8 k + 2 (l % 4) + {0, 1}
    // of repetition k (registers 4 k .. 4 k + 3: row l / 4, then row l / 4 + 8)
    for (int i = 0; i < n; ++i) {
      const int a = i & 1;
      // one decision per warp: the accumulator loads below are warp-wide
      if (!__all_sync(0xffffffffu, mbar_wait_or_abort(barAccFull(a), ph(i, 2), abort))) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      int f, n0;
      task(i, &f, &n0);
      const bool full = n0 + kSN <= ncol;
      constexpr int NACC = BWD ? 2 : 1;
#pragma unroll 1
      for (int acc = 0; acc < NACC; ++acc) {
        uint32_t v[2][2][16];  // [lane half][32-column half][registers]
        {
          constexpr int kh = 0;
          uint32_t u[2][2][16];
#pragma unroll
          for (int hb = 0; hb < 2; ++hb)
#pragma unroll
            for (int ch = 0; ch < 2; ++ch) {
              const uint32_t taddr = tmem + ((uint32_t)(warp * 32 + hb * 16) << 16) + kSTmemAcc +
                                     (uint32_t)(a * 128 + (acc + kh) * 64 + ch * 32);
              uint32_t* w = u[hb][ch];
              asm volatile(
                  "tcgen05.ld.sync.aligned.16x256b.x4.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                  "[%16];\n"
                  : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7]),
                    "=r"(w[8]), "=r"(w[9]), "=r"(w[10]), "=r"(w[11]), "=r"(w[12]), "=r"(w[13]), "=r"(w[14]),
                    "=r"(w[15])
                  : "r"(taddr));
            }
          asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
          for (int hb = 0; hb < 2; ++hb)
#pragma unroll
            for (int ch = 0; ch < 2; ++ch)
#pragma unroll
              for (int e = 0; e < 16; ++e)
                v[hb][ch][e] = kh ? __float_as_uint(__uint_as_float(v[hb][ch][e]) + __uint_as_float(u[hb][ch][e]))
                                  : u[hb][ch][e];
        }
        if (acc == NACC - 1) {
          // the accumulator buffer is read: the MMAs of tile i + 2 may overwrite it
          asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
          mbar_arrive(barAccFree(a));
        }
#pragma unroll
        for (int hb = 0; hb < 2; ++hb)
#pragma unroll
          for (int rh2 = 0; rh2 < 2; ++rh2) {
            const int rg = warp * 32 + hb * 16 + lane / 4 + 8 * rh2;  // accumulator row
            const int hh = rg >> 6, rh = rg & 63;
#pragma unroll
            for (int ch = 0; ch < 2; ++ch)
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                const int col = n0 + 32 * ch + 8 * k + 2 * (lane % 4);
                const float x0 = __uint_as_float(v[hb][ch][4 * k + 2 * rh2]);
                const float x1 = __uint_as_float(v[hb][ch][4 * k + 2 * rh2 + 1]);
                if constexpr (BWD) {
                  // parity acc, half hh (0 value, 1 derivative): item acc + 2 hh
                  if (rh < H) {
                    float* dst =
                        reinterpret_cast<float*>(out) + ((size_t)(4 * f + acc + 2 * hh) * H + rh) * ncol + col;
                    if (full) {
                      *reinterpret_cast<float2*>(dst) = make_float2(x0, x1);
                    } else {
                      if (col < ncol) dst[0] = x0;
                      if (col + 1 < ncol) dst[1] = x1;
                    }
                  }
                } else {
                  // half hh is the output parity: row 2 rh + hh
                  if (rh < (hh ? Ko : Ke)) {
                    double* dst = reinterpret_cast<double*>(out) + ((size_t)f * N + 2 * rh + hh) * ncol + col;
                    if (full) {
                      *reinterpret_cast<double2*>(dst) = make_double2((double)x0, (double)x1);
                    } else {
                      if (col < ncol) dst[0] = (double)x0;
                      if (col + 1 < ncol) dst[1] = (double)x1;
                    }
                  }
                }
              }
          }
      }
    }
  }
  __syncthreads();
  if (*abort) {
    // a wait ran out: flag it and give the copies and MMAs still in flight a
    // bounded time to land (they write this CTA's shared and tensor memory)
    if (warp == kSProd && lane == 0) {
      atomicExch(&g_tc_timeout, 1);
      for (int r = 0; r < kSNR; ++r)
        if (last_load[r] >= 0) mbar_wait_bounded(barFull(r), ph(last_load[r], kSNR));
    }
    if ((warp == kSMma || warp == kSMma + 1) && lane == 0 && last_mma >= 0)
      mbar_wait_bounded(barAccFull(last_mma & 1), ph(last_mma, 2));
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  if (warp == kSEpi) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kSTmemCols));
}


// ---- plane form (2D, N <= 256 rows, K <= 128 per operand) ----
// The 2D planes have an odd number of complex columns (Nx/2 + 1 per row), so
// their rows are 8-byte but not 16-byte aligned and no TMA tensor map can
// describe them; the split warps read the tile straight from global memory
// (8-byte loads, a warp covering 256 contiguous bytes of a row) and write the
// hi / lo images.  Each CTA serves one A operand (an M-tile role) held in
// tensor memory: backward, role q = p + 2 d is item w = q of a field (value
// or z-derivative of parity p, K = Ke or Ko over the rows 2k + p); forward,
// role par is the C^(2) rows 2r + par (K = N/2 over the mirror sums
// B[k] +- B[N-1-k]).  CTAs of one role share its (field, 64-column tile)
// tasks.
constexpr int kPN = 64;                                  // columns per tile
constexpr int kPK = 128;                                 // K extent of an operand
constexpr uint32_t kPHilo = 2 * kPK * kPN * 4;           // 64 KB of hi and lo images
constexpr int kPNH = 2;                                  // image stages
constexpr uint32_t kPOffBar = kPNH * kPHilo;
constexpr uint32_t kPSmem = kPOffBar + 256 + 1024;
constexpr uint32_t kPAtom = kPN * 128;
constexpr int kPThreads = 32 * 10;  // epilogue 0-3, split 4-7, MMA 8 (even K steps) and 9 (odd)
constexpr size_t kPImageFloats = (size_t)6 * 2 * 128 * kPK;  // 4 backward roles, 2 forward; hi and lo
constexpr uint32_t kPIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kPN >> 3) << 17) |
                             ((uint32_t)(kTcM >> 4) << 24);

__device__ __forceinline__ void mma_tf32_ts_n64(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "r"(tmem_a), "l"(bdesc), "r"(kPIdesc), "r"(acc));
}

// A parts of the plane form, 128 x 128 each, hi then lo per role: roles 0-3
// backward (Ev, Ov, Ed, Od: H x Kp row-major sources), 4-5 forward (sfE, sfO:
// Ke / Ko x Hp sources).  Layout [k / 4][row][k % 4]: the CTA stages a part
// in shared memory with bulk copies and thread `row` reads its 16-byte chunks
// of consecutive rows without bank conflicts.
__global__ void __launch_bounds__(kTcThreads) k_tc32p_image(const float* __restrict__ Ev, const float* __restrict__ Ov,
                                                            const float* __restrict__ Ed, const float* __restrict__ Od,
                                                            int kpe, int kpo, const float* __restrict__ sfE,
                                                            const float* __restrict__ sfO, int kph, int N,
                                                            float* __restrict__ images) {
  const int H = N / 2, Ke = (N + 1) / 2, Ko = N / 2;
  const int q = blockIdx.x;
  float* hi = images + (size_t)q * 2 * 128 * kPK;
  float* lo = hi + (size_t)128 * kPK;
  for (int idx = threadIdx.x; idx < 128 * kPK; idx += kTcThreads) {
    const int r = idx / kPK, k = idx % kPK;
    float v = 0.f;
    if (q < 4) {
      const int p = q & 1, K = p ? Ko : Ke, kp = p ? kpo : kpe;
      const float* src = q == 0 ? Ev : q == 1 ? Ov : q == 2 ? Ed : Od;
      if (r < H && k < K) v = src[(size_t)r * kp + k];
    } else {
      const int par = q - 4, M = par ? Ko : Ke;
      const float* src = par ? sfO : sfE;
      if (r < M && k < H) v = src[(size_t)r * kph + k];
    }
    const uint32_t h = to_tf32(v);
    const size_t o = ((size_t)(k / 4) * 128 + r) * 4 + (k % 4);
    hi[o] = __uint_as_float(h);
    lo[o] = __uint_as_float(to_tf32(v - __uint_as_float(h)));
  }
}

// in: nfields planes of N rows x ncol floats; BWD out: C_w (H x ncol) of
// field f at out + (4 f + w) H ncol; forward out: FP64 rows 2r + par at
// out + f N ncol.
template <bool BWD>
__global__ void __launch_bounds__(kPThreads, 1) k_tc32p(const float* __restrict__ in, const float* __restrict__ images,
                                                        void* out, int nfields, int N, int ncol) {
  extern __shared__ uint8_t tc_smem_raw[];
  const uint32_t raw = (uint32_t)__cvta_generic_to_shared(tc_smem_raw);
  const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
  uint8_t* sm = tc_smem_raw + pad;
  const uint32_t sbase = raw + pad;
  const uint32_t barL = sbase + kPOffBar;
  auto barSplitFull = [&](int h) { return barL + 8u + 8u * (uint32_t)h; };
  auto barHiloFree = [&](int h) { return barL + 8u + 8u * (uint32_t)(kPNH + h); };
  auto barAccFull = [&](int a) { return barL + 8u + 8u * (uint32_t)(2 * kPNH + a); };
  auto barAccFree = [&](int a) { return barL + 8u + 8u * (uint32_t)(2 * kPNH + 2 + a); };
  const uint32_t barA = barL + 8u + 8u * (uint32_t)(2 * kPNH + 4);  // A staged in shared memory
  constexpr uint32_t kBarBytes = 8u * (1 + 2 * kPNH + 4 + 1);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kPOffBar + kBarBytes);
  volatile int* abort = reinterpret_cast<volatile int*>(sm + kPOffBar + kBarBytes + 8);
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int H = N / 2, Ke = (N + 1) / 2, Ko = N / 2;
  constexpr int Q = BWD ? 4 : 2;  // roles
  const int q = blockIdx.x % Q, rank = blockIdx.x / Q, nq = ((int)gridDim.x - q + Q - 1) / Q;
  const int par = BWD ? (q & 1) : q;  // backward: parity of the rows read; forward: output parity
  const int K = BWD ? (par ? Ko : Ke) : H;
  const int nk8 = (K + 7) / 8;
  const int M = BWD ? H : (par ? Ko : Ke);  // valid output rows
  const int ntiles = (ncol + kPN - 1) / kPN;
  const int ntask = nfields * ntiles;
  const int n = rank < ntask ? (ntask - 1 - rank) / nq + 1 : 0;
  auto task = [&](int i, int* f, int* n0) {
    const int t = rank + i * nq;
    *f = t / ntiles;
    *n0 = (t % ntiles) * kPN;
  };
  auto ph = [](int i, int D) { return (uint32_t)(i / D) & 1u; };
  auto ph_prev = [](int i, int D) { return (uint32_t)(i / D - 1) & 1u; };

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sbase + kPOffBar +
                                                                                            kBarBytes),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    *abort = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;\n" ::"r"(barL));
    // hilofree and accfull complete on the commits of both MMA issuers
    for (int h = 0; h < kPNH; ++h) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;\n" ::"r"(barSplitFull(h)));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;\n" ::"r"(barHiloFree(h)));
    }
    for (int a = 0; a < 2; ++a) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 2;\n" ::"r"(barAccFull(a)));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;\n" ::"r"(barAccFree(a)));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(barA));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    // this role's A parts (hi, lo: 128 KB) into the image stages, which the
    // split fills only after they have gone on into tensor memory
    static_assert(2 * 128 * kPK * 4 <= kPNH * kPHilo, "A staging fits the image stages");
    mbar_expect_tx(barA, 2u * 128u * kPK * 4u);
    bulk_copy(sbase, images + (size_t)((BWD ? 0 : 4) + q) * 2 * 128 * kPK, 2u * 128u * kPK * 4u, barA);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;  // A hi at 0, lo at 128; accumulator pairs at 256 + 128 a
  int last_mma = -1;

  if (warp >= 4 && warp < 8) {
    // split: thread t loads rows 4 kc .. 4 kc + 3 of the operand (through the
    // row map) at columns 2 nn2, 2 nn2 + 1 of the tile and writes two K-major
    // chunks; the loads of all its items are issued before the first store
    const int t = tid - 128;
    bool need_a = true;  // the first stores wait until A has left the staging area
    for (int i = 0; i < n && !*abort; ++i) {
      const int hs = i % kPNH;
      if (i >= kPNH && !mbar_wait_or_abort(barHiloFree(hs), ph_prev(i, kPNH), abort)) break;
      int f, n0;
      task(i, &f, &n0);
      const float* src = in + (size_t)f * N * ncol;
      uint8_t* hb = sm + (uint32_t)hs * kPHilo;
      // items per load batch: all eight of the thread in the backward
      // transform; four in the forward one, whose values take two loads each
      // (the mirror rows), so that a batch's loads all stay in flight
      constexpr int UB = BWD ? 8 : 4;
      for (int it0 = t; it0 < (kPK / 4) * (kPN / 2); it0 += UB * 128) {
        float2 v[UB][4], w[UB][4];  // w: the mirror rows of the forward transform
        // every load of the batch first (no arithmetic between them, so that
        // they are all in flight), then the mirror sums
#pragma unroll
        for (int u = 0; u < UB; ++u) {
          const int it = it0 + u * 128;
          const int nn2 = it % (kPN / 2), kc = it / (kPN / 2);
          const int col = n0 + 2 * nn2;
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int k = 4 * kc + e;
            const bool ok = k < K && col < ncol;
            const int row = BWD ? 2 * k + par : k;
            v[u][e] = ok ? *reinterpret_cast<const float2*>(src + (size_t)row * ncol + col) : make_float2(0.f, 0.f);
            if constexpr (!BWD)
              w[u][e] = ok ? *reinterpret_cast<const float2*>(src + (size_t)(N - 1 - k) * ncol + col)
                           : make_float2(0.f, 0.f);
          }
        }
        if constexpr (!BWD) {
#pragma unroll
          for (int u = 0; u < UB; ++u)
#pragma unroll
            for (int e = 0; e < 4; ++e)
              v[u][e] = par ? make_float2(v[u][e].x - w[u][e].x, v[u][e].y - w[u][e].y)
                            : make_float2(v[u][e].x + w[u][e].x, v[u][e].y + w[u][e].y);
        }
        if (need_a) {
          // (the loads above overlap the A staging)
          if (!mbar_wait_or_abort(barL, 0, abort)) break;
          need_a = false;
        }
#pragma unroll
        for (int u = 0; u < UB; ++u) {
          const int it = it0 + u * 128;
          const int nn2 = it % (kPN / 2), kc = it / (kPN / 2);
          split_store4(hb, hb + kPHilo / 2, sw128_off(2 * nn2, 4 * kc, kPN),
                       make_float4(v[u][0].x, v[u][1].x, v[u][2].x, v[u][3].x));
          split_store4(hb, hb + kPHilo / 2, sw128_off(2 * nn2 + 1, 4 * kc, kPN),
                       make_float4(v[u][0].y, v[u][1].y, v[u][2].y, v[u][3].y));
        }
      }
      if (need_a) break;  // aborted while waiting for A
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      mbar_arrive(barSplitFull(hs));
    }
  } else if (warp == 8 || warp == 9) {
    const int jpar = warp - 8;  // this issuer's K steps: j % 2 == jpar, into accumulator jpar
    if (lane == 0) {
      mbar_wait_or_abort(barL, 0, abort);  // A in tensor memory
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      for (int i = 0; i < n && !*abort; ++i) {
        const int hs = i % kPNH, a = i & 1;
        if (!mbar_wait_or_abort(barSplitFull(hs), ph(i, kPNH), abort)) break;
        if (i >= 2 && !mbar_wait_or_abort(barAccFree(a), ph_prev(i, 2), abort)) break;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        const uint32_t bb = sbase + (uint32_t)hs * kPHilo;
        const uint64_t bhi = sw128_desc(bb), blo = sw128_desc(bb + kPHilo / 2);
        // two accumulators, the even and the odd K steps, issued by the two
        // issuers in parallel (the epilogue adds them)
        const uint32_t d = tmem + 256u + (uint32_t)(a * 128 + jpar * 64);
        for (int j = jpar; j < nk8; j += 2) {
          const uint64_t kb = ((uint64_t)(j >> 2) * kPAtom + (uint64_t)(j & 3) * 32u) >> 4;
          const uint32_t acc = j > 1 ? 1u : 0u;
          mma_tf32_ts_n64(d, tmem + 8u * j, bhi + kb, acc);
          mma_tf32_ts_n64(d, tmem + 8u * j, blo + kb, 1u);
          mma_tf32_ts_n64(d, tmem + 128u + 8u * j, bhi + kb, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         barHiloFree(hs))
                     : "memory");
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         barAccFull(a))
                     : "memory");
        last_mma = i;
      }
    }
  } else if (warp < 4) {
    {
      // this role's A (hi, lo) from its shared-memory staging into tensor
      // memory: thread row r = 32 w + l, 16-byte chunk c of part h at
      // [h][c][r] (consecutive rows in consecutive chunks)
      const int r = warp * 32 + lane;
      const bool staged = __all_sync(0xffffffffu, mbar_wait_or_abort(barA, 0, abort));
      const float4* stA = reinterpret_cast<const float4*>(sm);
#pragma unroll 1
      for (int h = 0; h < 2 && staged; ++h)
#pragma unroll 1
        for (int c = 0; c < kPK / 32; ++c) {
          uint32_t w[32];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const float4 x = stA[((size_t)h * (kPK / 4) + 8 * c + k) * 128 + r];
            w[4 * k] = __float_as_uint(x.x);
            w[4 * k + 1] = __float_as_uint(x.y);
            w[4 * k + 2] = __float_as_uint(x.z);
            w[4 * k + 3] = __float_as_uint(x.w);
          }
          const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(h * 128 + 32 * c);
          asm volatile(
              "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
              "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};\n" ::"r"(taddr),
              "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]), "r"(w[8]),
              "r"(w[9]), "r"(w[10]), "r"(w[11]), "r"(w[12]), "r"(w[13]), "r"(w[14]), "r"(w[15]), "r"(w[16]),
              "r"(w[17]), "r"(w[18]), "r"(w[19]), "r"(w[20]), "r"(w[21]), "r"(w[22]), "r"(w[23]), "r"(w[24]),
              "r"(w[25]), "r"(w[26]), "r"(w[27]), "r"(w[28]), "r"(w[29]), "r"(w[30]), "r"(w[31])
              : "memory");
        }
      asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
      mbar_arrive(barL);
    }
    // epilogue: 16 x 256-bit accumulator loads (lane l: rows l / 4, l / 4 + 8
    // of a 16-row block, columns 8 k + 2 (l % 4) + {0, 1})
    for (int i = 0; i < n; ++i) {
      const int a = i & 1;
      if (!__all_sync(0xffffffffu, mbar_wait_or_abort(barAccFull(a), ph(i, 2), abort))) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      int f, n0;
      task(i, &f, &n0);
      uint32_t v[2][2][16];  // [lane half][32-column half][registers]
      float vs[2][2][16];    // the sum of the two K-step accumulators
      const int nkh = nk8 > 1 ? 2 : 1;  // a single K step leaves the odd accumulator unused
#pragma unroll 1
      for (int kh = 0; kh < nkh; ++kh) {
#pragma unroll
        for (int hb = 0; hb < 2; ++hb)
#pragma unroll
          for (int ch = 0; ch < 2; ++ch) {
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32 + hb * 16) << 16) + 256u +
                                   (uint32_t)(a * 128 + kh * 64 + ch * 32);
            uint32_t* w = v[hb][ch];
            asm volatile(
                "tcgen05.ld.sync.aligned.16x256b.x4.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];\n"
                : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7]),
                  "=r"(w[8]), "=r"(w[9]), "=r"(w[10]), "=r"(w[11]), "=r"(w[12]), "=r"(w[13]), "=r"(w[14]),
                  "=r"(w[15])
                : "r"(taddr));
          }
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int hb = 0; hb < 2; ++hb)
#pragma unroll
          for (int ch = 0; ch < 2; ++ch)
#pragma unroll
            for (int e = 0; e < 16; ++e)
              vs[hb][ch][e] = kh ? vs[hb][ch][e] + __uint_as_float(v[hb][ch][e]) : __uint_as_float(v[hb][ch][e]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
      mbar_arrive(barAccFree(a));
#pragma unroll
      for (int hb = 0; hb < 2; ++hb)
#pragma unroll
        for (int rh2 = 0; rh2 < 2; ++rh2) {
          const int r = warp * 32 + hb * 16 + lane / 4 + 8 * rh2;  // output row of the role
          if (r >= M) continue;
#pragma unroll
          for (int ch = 0; ch < 2; ++ch)
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const int col = n0 + 32 * ch + 8 * k + 2 * (lane % 4);
              if (col >= ncol) continue;  // ncol is even: col + 1 < ncol too
              const float x0 = vs[hb][ch][4 * k + 2 * rh2];
              const float x1 = vs[hb][ch][4 * k + 2 * rh2 + 1];
              if constexpr (BWD) {
                float* dst = reinterpret_cast<float*>(out) + ((size_t)(4 * f + q) * H + r) * ncol + col;
                *reinterpret_cast<float2*>(dst) = make_float2(x0, x1);
              } else {
                double* dst = reinterpret_cast<double*>(out) + ((size_t)f * N + 2 * r + par) * ncol + col;
                *reinterpret_cast<double2*>(dst) = make_double2((double)x0, (double)x1);
              }
            }
        }
    }
  }
  __syncthreads();
  if (*abort) {
    if (tid == 0) {
      atomicExch(&g_tc_timeout, 1);
      mbar_wait_bounded(barA, 0);  // the A staging copy
    }
    if ((warp == 8 || warp == 9) && lane == 0 && last_mma >= 0)
      mbar_wait_bounded(barAccFull(last_mma & 1), ph(last_mma, 2));
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512));
}

}  // namespace

bool gemm_tc32_supported(const GemmBatch32& bt, int nbatch) {
  for (int b = 0; b < nbatch; ++b)
    if (bt.item[b].M > kTcM || bt.item[b].K > kTcK || bt.item[b].Kpad > kTcK) return false;
  return true;
}

size_t tc32_a_image_floats() { return 2 * kABytes / 4; }

size_t tc32_b_scratch_floats(int ncol, int nimages) {
  const size_t ntiles = (size_t)(ncol + kTcN - 1) / kTcN;
  return (size_t)nimages * ntiles * (2 * kBBytes / 4);
}

void make_tc32_a_image(const float* A, int M, int Kpad, float* image, cudaStream_t st) {
  k_tc32_image_a<<<1, kTcThreads, 0, st>>>(A, M, Kpad, image);
}

cudaError_t set_tc32_smem_limits() {
  cudaError_t e = cudaFuncSetAttribute(k_gemm_tc32<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_gemm_tc32<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_tc32s<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_tc32s<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_tc32p<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_tc32p<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPSmem);
}

bool launch_gemm_tc32(const GemmBatch32& bt_in, int nbatch, int ncol, int ldb, int ldc, int Nrows, bool out_f64,
                      cudaStream_t st, float* bscratch, size_t bscratch_floats) {
  if (!bscratch || nbatch < 1 || nbatch > kGemmMaxBatch) return false;
  GemmBatch32 bt = bt_in;
  Tc32BInputs bi{};
  int nimg = 0;
  const size_t per = tc32_b_scratch_floats(ncol, 1);
  for (int b = 0; b < nbatch; ++b) {
    GemmItem32& it = bt.item[b];
    if (!it.Aimg) return false;
    int j = 0;
    while (j < nimg && !(bi.in[j].B == it.B && bi.in[j].K == it.K && bi.in[j].mode == it.mode &&
                         (it.mode == GEMM_PLAIN || bi.in[j].par == it.par)))
      ++j;
    if (j == nimg) {
      if ((size_t)(nimg + 1) * per > bscratch_floats) return false;
      bi.in[nimg] = Tc32BInput{it.B, bscratch + (size_t)nimg * per, it.K, it.mode, it.par};
      ++nimg;
    }
    it.Bimg = bi.in[j].image;
  }
  const int ntiles = (ncol + kTcN - 1) / kTcN;
  k_tc32_image_b<<<dim3(ntiles, nimg), kTcThreads, 0, st>>>(bi, ncol, ldb, Nrows);
  int cpi = 148 / nbatch;  // CTAs per item: one wave, one CTA per SM by shared memory
  if (cpi < 1) cpi = 1;
  if (cpi > ntiles) cpi = ntiles;
  dim3 grid(cpi, 1, nbatch);
  if (out_f64)
    k_gemm_tc32<double><<<grid, kTcThreads, kTcSmem, st>>>(bt, ncol, ldc);
  else
    k_gemm_tc32<float><<<grid, kTcThreads, kTcSmem, st>>>(bt, ncol, ldc);
  return true;
}

bool tc32s_supported(int N, int ncol) { return N >= 2 && N <= kSRows && N % 2 == 0 && ncol > 0 && ncol % 4 == 0; }

size_t tc32s_image_floats() { return kSImageFloats; }

void make_tc32s_images(const float* Ev, const float* Ov, const float* Ed, const float* Od, int kpe, int kpo,
                       const float* sfE, const float* sfO, int kph, int N, float* images, cudaStream_t st) {
  k_tc32s_image<<<3, kTcThreads, 0, st>>>(Ev, Ov, Ed, Od, kpe, kpo, sfE, sfO, kph, N, images);
}

namespace {
// cuTensorMapEncodeTiled, reached through the runtime's driver entry point
// (no link-time dependency on the driver library)
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_tiled() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}
}  // namespace

bool make_tc32s_tmap(TmaDesc* d, const float* planes, int nfields, int N, int ncol) {
  static_assert(sizeof(TmaDesc) == sizeof(CUtensorMap) && alignof(TmaDesc) >= alignof(CUtensorMap), "tensor map");
  const EncodeTiled enc = encode_tiled();
  if (!enc || !tc32s_supported(N, ncol) || nfields < 1 || (reinterpret_cast<uintptr_t>(planes) & 15u)) return false;
  // fields of N rows of ncol floats; boxes of 32 columns x N rows of one
  // field (columns past ncol read as zero)
  const cuuint64_t dims[3] = {(cuuint64_t)ncol, (cuuint64_t)N, (cuuint64_t)nfields};
  const cuuint64_t strides[2] = {(cuuint64_t)ncol * 4, (cuuint64_t)N * ncol * 4};
  const cuuint32_t box[3] = {(cuuint32_t)kSN, (cuuint32_t)N, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(reinterpret_cast<CUtensorMap*>(d), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(planes), dims,
             strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void launch_tc32s(bool backward, const TmaDesc& d, const float* images, void* out, int nfields, int N, int ncol,
                  cudaStream_t st) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntask = nfields * ((ncol + kSN - 1) / kSN);
  const int grid = sms < ntask ? sms : ntask;
  CUtensorMap map;
  static_assert(sizeof(map) == sizeof(d.bytes), "tensor map");
  for (size_t i = 0; i < sizeof(map); ++i) reinterpret_cast<unsigned char*>(&map)[i] = d.bytes[i];
  if (backward)
    k_tc32s<true><<<grid, kSThreads, kSSmem, st>>>(map, images, out, nfields, N, ncol);
  else
    k_tc32s<false><<<grid, kSThreads, kSSmem, st>>>(map, images, out, nfields, N, ncol);
}

bool tc32p_supported(int N, int ncol) { return N >= 2 && N <= 2 * kPK && N % 2 == 0 && ncol > 0 && ncol % 2 == 0; }

size_t tc32p_image_floats() { return kPImageFloats; }

void make_tc32p_images(const float* Ev, const float* Ov, const float* Ed, const float* Od, int kpe, int kpo,
                       const float* sfE, const float* sfO, int kph, int N, float* images, cudaStream_t st) {
  k_tc32p_image<<<6, kTcThreads, 0, st>>>(Ev, Ov, Ed, Od, kpe, kpo, sfE, sfO, kph, N, images);
}

void launch_tc32p(bool backward, const float* in, const float* images, void* out, int nfields, int N, int ncol,
                  cudaStream_t st) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // every role gets at least one CTA and no CTA is left without a task
  const int Q = backward ? 4 : 2;
  const int ntask = nfields * ((ncol + kPN - 1) / kPN);
  const int grid = sms < Q * ntask ? sms : Q * ntask;
  if (backward)
    k_tc32p<true><<<grid, kPThreads, kPSmem, st>>>(in, images, out, nfields, N, ncol);
  else
    k_tc32p<false><<<grid, kPThreads, kPSmem, st>>>(in, images, out, nfields, N, ncol);
}

int tc32_status() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_tc_timeout, sizeof(int)) != cudaSuccess) return -1;
  return v;
}

}  // namespace tb
