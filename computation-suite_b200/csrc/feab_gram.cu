// POD of a snapshot panel: G = X^T X on the tensor cores, then an FP64 symmetric eigensolve.
//
// The reference computes the singular values of the snapshot matrix by an FP64 economy SVD
// (PodBasis._fit_standard, rom_engine/src/rom_engine/pod.py:140-147).  Here the snapshots X
// (n x 64, FP32, row major) are reduced to their 64 x 64 Gram matrix, whose eigenvalues are the
// squared singular values.
//
// Gram kernel (one CTA of 4 warps, several CTAs per SM, chunks of 64 rows, grid-stride):
//   1. one thread streams each 16 KB chunk of X into a shared-memory stage with
//      cp.async.bulk (mbarrier complete_tx), 4 stages deep;
//   2. all threads split the chunk into bf16 hi = bf16(x) and lo = bf16(x - hi) and write one
//      128 x 64 tile T = [hi^T ; lo^T] in the K-major no-swizzle core-matrix layout;
//   3. one thread issues 4 tcgen05.mma (M = N = 128, K = 16, bf16 -> fp32 in TMEM) with T as
//      both operands, so the 128 x 128 accumulator holds [hi^T hi, hi^T lo ; lo^T hi, lo^T lo];
//      tcgen05.commit signals an mbarrier when they are done;
//   4. every 16 chunks (and at the end) the accumulator is read with tcgen05.ld and added into
//      FP64 registers, hh + hl + lh (the split-bf16 "x3" product), bounding FP32 accumulation
//      to 1024 rows.
// Per-CTA FP64 partials are summed in a fixed order by a second kernel (deterministic).
// Every wait is bounded; a timeout sets an error flag, drains what is in flight with bounded
// waits, frees TMEM and returns.
#include <cuda_bf16.h>
#include <algorithm>
#include "feab_common.cuh"

namespace feab {
namespace {

constexpr int kCols = 64;            // snapshot columns (panel width)
constexpr int kChunk = 64;           // rows per chunk (MMA K per chunk)
constexpr int kStages = 4;           // FP32 staging buffers
constexpr int kThreadsG = 128;
constexpr int kDrain = 16;           // chunks accumulated in FP32 before an FP64 drain
constexpr uint32_t kLBO = 128;                      // next core matrix along K
constexpr uint32_t kSBO = (kChunk / 8) * 128;       // next 8-row group along M/N (1024 B)
constexpr long long kWaitCycles = 4000000000LL;     // ~2 s at 2 GHz

struct __align__(1024) GramSmem {
  float stage[kStages][kChunk * kCols];
  __nv_bfloat16 tile[2][128 * kChunk];
  unsigned long long full_bar[kStages];
  unsigned long long mma_bar[2];
  uint32_t tmem_base;
};

__device__ __forceinline__ int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(unsigned long long* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase; false (and *err set) on timeout.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t parity, int* err) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity)) {
    if (clock64() - t0 > kWaitCycles) {
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, unsigned long long* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// SM100 shared-memory matrix descriptor, K-major, no swizzle (start, LBO, SBO in 16 B units;
// version 1 at bits 46-47; layout type 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((kLBO >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((kSBO >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor, kind::f16: fp32 accumulate, bf16 A and B, both K-major, N = 128, M = 128.
__host__ __device__ constexpr uint32_t instr_desc() {
  return (1u << 4)                 // c_format = F32
         | (1u << 7)               // a_format = BF16
         | (1u << 10)              // b_format = BF16
         | ((128u >> 3) << 17)     // n_dim
         | ((128u >> 4) << 24);    // m_dim
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accum)
      : "memory");
}

__device__ __forceinline__ void mma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Convert staged FP32 rows [kChunk][kCols] into the bf16 tile T[m][k] (m < 64: hi of column m,
// m >= 64: lo of column m-64; k = row within the chunk), K-major core-matrix layout:
// byte (m/8)*SBO + (k/8)*LBO + (m%8)*16 + (k%8)*2.  Rows past `rows` are zero.
__device__ __forceinline__ void split_chunk(const float* st, __nv_bfloat16* tile, int rows) {
  for (int item = threadIdx.x; item < kCols * (kChunk / 8); item += kThreadsG) {
    const int m = item % kCols, kg = item / kCols;
    __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = kg * 8 + u;
      const float x = k < rows ? st[k * kCols + m] : 0.0f;
      const __nv_bfloat16 h = __float2bfloat16_rn(x);
      hi[u] = h;
      lo[u] = __float2bfloat16_rn(x - __bfloat162float(h));
    }
    char* base = reinterpret_cast<char*>(tile);
    *reinterpret_cast<uint4*>(base + (m / 8) * kSBO + kg * kLBO + (m % 8) * 16) = *reinterpret_cast<uint4*>(hi);
    const int ml = m + 64;
    *reinterpret_cast<uint4*>(base + (ml / 8) * kSBO + kg * kLBO + (ml % 8) * 16) = *reinterpret_cast<uint4*>(lo);
  }
}

__global__ void __launch_bounds__(kThreadsG) k_gram_bf16x3(const float* __restrict__ X, int64_t n,
                                                          double* __restrict__ part, int* err) {
  extern __shared__ unsigned char smem_raw[];
  GramSmem& S = *reinterpret_cast<GramSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5;
  const int64_t n_chunks = (n + kChunk - 1) / kChunk;
  // chunks of this CTA: blockIdx.x, blockIdx.x + gridDim.x, ...
  const int64_t my = n_chunks > blockIdx.x ? (n_chunks - 1 - blockIdx.x) / gridDim.x + 1 : 0;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&S.full_bar[s], 1);
    mbar_init(&S.mma_bar[0], 1);
    mbar_init(&S.mma_bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                 "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S.tmem_base;
  const uint32_t idesc = instr_desc();

  // prologue: fill the staging ring
  if (tid == 0) {
    for (int64_t i = 0; i < min64(my, kStages); ++i) {
      const int64_t c = blockIdx.x + i * gridDim.x;
      const int64_t r0 = c * kChunk;
      const int rows = (int)min64(kChunk, n - r0);
      bulk_load(S.stage[i], X + r0 * kCols, (uint32_t)rows * kCols * 4, &S.full_bar[i]);
    }
  }

  double acc[kCols];
#pragma unroll
  for (int j = 0; j < kCols; ++j) acc[j] = 0.0;
  bool ok = true;
  int since_drain = 0;
  int64_t issued = 0;  // chunks whose MMAs were issued

  auto drain = [&](int64_t last) {
    // wait for the MMAs of chunk `last` (commit tracks all earlier ones too), then read D
    const bool w = mbar_wait(&S.mma_bar[last & 1], (uint32_t)((last >> 1) & 1), err);
    if (!__syncthreads_and(w)) {  // block-uniform decision
      ok = false;
      return;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    float v[32];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      tmem_ld32(tmem + lane_base + (uint32_t)(q * 32), v);
      if (tid < 64 || q < 2) {
#pragma unroll
        for (int i = 0; i < 32; ++i) acc[(q & 1) * 32 + i] += (double)v[i];
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  };

  for (int64_t i = 0; i < my && ok; ++i) {
    const int s = (int)(i % kStages), t = (int)(i & 1);
    const int64_t c = blockIdx.x + i * gridDim.x;
    const int rows = (int)min64(kChunk, n - c * kChunk);
    // tile t was last read by the MMAs of chunk i-2
    bool w = true;
    if (i >= 2 && since_drain > 0) w = mbar_wait(&S.mma_bar[t], (uint32_t)(((i - 2) >> 1) & 1), err);
    if (w) w = mbar_wait(&S.full_bar[s], (uint32_t)((i / kStages) & 1), err);
    if (!__syncthreads_and(w)) {  // block-uniform decision
      ok = false;
      break;
    }
    split_chunk(S.stage[s], S.tile[t], rows);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    // stage s is free again: refill it with chunk i + kStages
    if (tid == 0 && i + kStages < my) {
      const int64_t c2 = blockIdx.x + (i + kStages) * gridDim.x;
      const int64_t r2 = c2 * kChunk;
      const int rows2 = (int)min64(kChunk, n - r2);
      bulk_load(S.stage[s], X + r2 * kCols, (uint32_t)rows2 * kCols * 4, &S.full_bar[s]);
    }
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = smem_u32(S.tile[t]);
#pragma unroll
      for (int ks = 0; ks < kChunk / 16; ++ks) {
        const uint64_t d = smem_desc(base + ks * 2 * kLBO);
        mma_bf16(tmem, d, d, idesc, (since_drain > 0 || ks > 0) ? 1u : 0u);
      }
      mma_commit(&S.mma_bar[t]);
    }
    ++issued;
    ++since_drain;
    if (since_drain == kDrain || i + 1 == my) {
      drain(i);
      since_drain = 0;
      __syncthreads();
      if (!ok) break;
    }
  }
  if (!ok) {
    // bounded wait for the MMAs and bulk copies already issued before leaving TMEM / smem
    if (issued > 0) {
      const int64_t last = issued - 1;
      const long long t0 = clock64();
      while (!mbar_try(&S.mma_bar[last & 1], (uint32_t)((last >> 1) & 1)) && clock64() - t0 < kWaitCycles) {
      }
    }
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128) : "memory");
  }
  // per-CTA partial: row tid of [hh + hl ; lh]
  double* out = part + ((int64_t)blockIdx.x * 128 + tid) * kCols;
#pragma unroll
  for (int j = 0; j < kCols; ++j) out[j] = acc[j];
}

// ---------------------------------------------------------------- exact-product int8 Gram
// G = X^T X with the products formed exactly on the tensor cores (tcgen05.mma kind::i8, s32
// accumulation), after the integer-slice method of Ozaki et al. for emulating high-precision
// products on integer matrix units (Ootomo, Ozaki & Yokota, "DGEMM on integer matrix
// multiplication unit", Int. J. High Perf. Comput. Appl. 2024).  Each CTA owns a contiguous range
// of rows.  Per column i it takes e_i with |x| < 2^e_i over its rows, and splits every value into
// kSlices signed 7-bit digits: x = 2^e_i sum_a s_a 2^(-7a), s_a = trunc of the scaled remainder
// (all steps exact in FP32).  Then
//   x_ri x_rj = 2^(e_i + e_j) sum_{a, c} s_a(r, i) s_c(r, j) 2^(-7(a + c)),
// and the digit products sum exactly in int32.  Pairs with a + c > kSlices + 1 are dropped
// (their weight is below 2^(-7(kSlices + 2)) of the scale).  With 7 digits a value keeps 49 bits
// below its CTA's column maximum, so the FP32 inputs are exact down to 2^-25 of that maximum and
// the dropped terms are below 1e-15 of it: G comes out with FP64-level accuracy.
//
// MMA arrangement (M = 128, N = 64, K = 64 per chunk of 64 rows): A = [S_a ; S_(a+1)] for odd a
// (S_8 = 0), B = S_c; the product adds S_a^T S_c (weight a + c) to the top 64 TMEM lanes and
// S_(a+1)^T S_c (weight a + c + 1) to the bottom 64 of region R_(a+c).  Seven regions
// R_2..R_8 of 64 columns each (448 of TMEM's 512) hold every needed pair with a fixed weight
// per half: weight v on top of R_v, v + 1 on the bottom.  16 MMAs (32 instructions) per chunk.
// The int32 regions are drained every kI8Drain chunks (and at the end) into an FP64 accumulator in
// shared memory, which bounds them below 2^31; per-CTA FP64 partials are summed by k_gram_reduce
// (fixed order).  512 threads: the digits are formed with integer operations from the FP32 bit
// pattern (a 49-bit fixed-point magnitude, then 7-bit fields), and the drain keeps 16 doubles per
// thread, so the kernel stays within 128 registers.
constexpr int kSlices = 7;
constexpr int kI8Threads = 512;
constexpr int kI8Drain = 192;                        // chunks between drains: < 2^31 / (4 * 64 * 127^2)
constexpr uint32_t kI8LBO = 128;                     // next core matrix (16 K-bytes) along K
constexpr uint32_t kI8SBO = 4 * 128;                 // next 8-row group along M / N
constexpr int kI8SliceBytes = 64 * kChunk;           // one 64-row x 64-K int8 slice tile
constexpr int kI8Regions = kSlices;                  // R_2 .. R_8

struct __align__(1024) Int8Smem {
  float stage[kStages][kChunk * kCols];              // 64 KB
  int8_t tile[2][(kSlices + 1) * kI8SliceBytes];     // 2 x 32 KB; slice 8 stays zero
  double acc[128 * kCols];                           // 64 KB: the drained sums, one row per TMEM lane
  unsigned long long full_bar[kStages];
  unsigned long long mma_bar[2];
  float colmax[kI8Threads / 16][kCols];
  int expo[kCols];
  uint32_t tmem_base;
};

__device__ __forceinline__ uint64_t smem_desc_i8(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((kI8LBO >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((kI8SBO >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// kind::i8 instruction descriptor: s32 accumulate (D format 2), signed 8-bit A and B, both
// K-major, N = 64, M = 128.
__host__ __device__ constexpr uint32_t instr_desc_i8() {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accum)
      : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int32_t (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = (int32_t)r[i];
}

// The 7-bit digit fields of |x| 2^(49 - e) (|x| < 2^e), from the FP32 bit pattern: mantissa with
// its hidden bit, shifted into a 49-bit fixed-point magnitude (bits below 2^(e - 49) drop, the
// truncation of x = 2^e sum_a s_a 2^(-7a)), then digit a = bits 49 - 7a .. 55 - 7a, with x's sign.
__device__ __forceinline__ void digits_i8(float x, int e, uint32_t (&d)[kSlices]) {
  const uint32_t u = __float_as_uint(x);
  const uint32_t ex = (u >> 23) & 0xffu;
  const uint64_t mant = (uint64_t)((u & 0x7fffffu) | (ex ? 0x800000u : 0u));
  const int sh = (ex ? (int)ex : 1) - 101 - e;   // x = mant 2^(ex - 150); 2^(49 - e) more
  const uint64_t mag = sh >= 0 ? (mant << sh) : (sh > -64 ? (mant >> -sh) : 0ull);
  const bool neg = (u >> 31) != 0;
#pragma unroll
  for (int a = 0; a < kSlices; ++a) {
    const uint32_t f = (uint32_t)(mag >> (49 - 7 * (a + 1))) & 0x7fu;
    d[a] = (neg ? (0u - f) : f) & 0xffu;
  }
}

// Split the staged FP32 rows of one chunk into the kSlices int8 digit tiles.  Thread t owns
// column m = t % 64 and rows 8 (t / 64) .. +7 (half of a 16-byte core-matrix row per digit).
__device__ __forceinline__ void split_chunk_i8(const float* st, int8_t* tiles, int rows, const int* expo) {
  const int m = threadIdx.x & 63, kg = threadIdx.x >> 6;
  const int e = expo[m];
  uint32_t packed[kSlices][2];
#pragma unroll
  for (int a = 0; a < kSlices; ++a) packed[a][0] = packed[a][1] = 0u;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int k = kg * 8 + u;
    uint32_t d[kSlices];
    digits_i8(k < rows ? st[k * kCols + m] : 0.0f, e, d);
#pragma unroll
    for (int a = 0; a < kSlices; ++a) packed[a][u >> 2] |= d[a] << (8 * (u & 3));
  }
  const uint32_t off = (m / 8) * kI8SBO + (kg >> 1) * kI8LBO + (m % 8) * 16 + (kg & 1) * 8;
#pragma unroll
  for (int a = 0; a < kSlices; ++a)
    *reinterpret_cast<uint2*>(tiles + a * kI8SliceBytes + off) = make_uint2(packed[a][0], packed[a][1]);
}

__global__ void __launch_bounds__(kI8Threads, 1) k_gram_int8(const float* __restrict__ X, int64_t n,
                                                            double* __restrict__ part, int* err) {
  extern __shared__ unsigned char smem_raw[];
  Int8Smem& S = *reinterpret_cast<Int8Smem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t n_chunks = (n + kChunk - 1) / kChunk;
  const int64_t per = (n_chunks + gridDim.x - 1) / gridDim.x;
  const int64_t c0 = min64(n_chunks, (int64_t)blockIdx.x * per), c1 = min64(n_chunks, c0 + per);
  const int64_t my = c1 - c0;
  const int64_t row0 = c0 * kChunk, row1 = min64(n, c1 * kChunk);

  // per-column exponents over this CTA's rows: thread t reads 4 columns (float4) of rows
  // row0 + t / 16, + 32, ..., kI8Ahead rows in flight per thread
  {
    constexpr int kI8Ahead = 8;
    constexpr int kRowStep = kI8Threads / 16;
    float mx[4] = {0.f, 0.f, 0.f, 0.f};
    const int cq = (tid & 15) * 4;
    for (int64_t r = row0 + (tid >> 4); r < row1; r += kRowStep * kI8Ahead) {
      float4 v[kI8Ahead];
#pragma unroll
      for (int u = 0; u < kI8Ahead; ++u) {
        const int64_t rr = r + (int64_t)kRowStep * u;
        v[u] = rr < row1 ? __ldg(reinterpret_cast<const float4*>(X + rr * kCols + cq)) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < kI8Ahead; ++u) {
        mx[0] = fmaxf(mx[0], fabsf(v[u].x));
        mx[1] = fmaxf(mx[1], fabsf(v[u].y));
        mx[2] = fmaxf(mx[2], fabsf(v[u].z));
        mx[3] = fmaxf(mx[3], fabsf(v[u].w));
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) S.colmax[tid >> 4][cq + j] = mx[j];
  }
  // zero both tile buffers (the eighth digit tile must stay zero) and the accumulator
  for (int i = tid; i < 2 * (kSlices + 1) * kI8SliceBytes / 16; i += kI8Threads)
    reinterpret_cast<int4*>(&S.tile[0][0])[i] = make_int4(0, 0, 0, 0);
  for (int i = tid; i < 128 * kCols; i += kI8Threads) S.acc[i] = 0.0;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&S.full_bar[s], 1);
    mbar_init(&S.mma_bar[0], 1);
    mbar_init(&S.mma_bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (tid < kCols) {
    float m = 0.f;
    for (int g = 0; g < kI8Threads / 16; ++g) m = fmaxf(m, S.colmax[g][tid]);
    int e = 0;
    if (m > 0.f) frexpf(m, &e);  // m = f 2^e, f in [0.5, 1): every |x| <= m < 2^e
    S.expo[tid] = e;
  }
  __syncthreads();
  const uint32_t tmem = S.tmem_base;
  const uint32_t idesc = instr_desc_i8();

  if (tid == 0) {
    for (int64_t i = 0; i < min64(my, kStages); ++i) {
      const int64_t r0 = (c0 + i) * kChunk;
      const int rows = (int)min64(kChunk, n - r0);
      bulk_load(S.stage[i], X + r0 * kCols, (uint32_t)rows * kCols * 4, &S.full_bar[i]);
    }
  }

  // the drain: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its lane quarter) and columns
  // 16 (w / 4) .. + 15 of every region, and adds them, weighted, into row lane_row of S.acc
  const int lane_row = 32 * (warp & 3) + lane;
  const int col0 = 16 * (warp >> 2);
  bool ok = true;
  int since_drain = 0;
  int64_t issued = 0;
  uint32_t seen = 0;  // regions written since the last drain (thread 0)

  auto drain = [&](int64_t last) {
    const bool w = mbar_wait(&S.mma_bar[last & 1], (uint32_t)((last >> 1) & 1), err);
    if (!__syncthreads_and(w)) {
      ok = false;
      return;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    // top lanes hold weight v of R_v, bottom lanes weight v + 1
    const int wshift = lane_row < 64 ? 0 : 1;
    double sum[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) sum[i] = 0.0;
    for (int r = 0; r < kI8Regions; ++r) {
      const double scale = ldexp(1.0, -7 * (r + 2 + wshift));
      int32_t v[16];
      tmem_ld16(tmem + lane_base + (uint32_t)(r * 64 + col0), v);
#pragma unroll
      for (int i = 0; i < 16; ++i) sum[i] += (double)v[i] * scale;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) S.acc[lane_row * kCols + col0 + i] += sum[i];
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  };

  for (int64_t i = 0; i < my && ok; ++i) {
    const int s = (int)(i % kStages), t = (int)(i & 1);
    const int rows = (int)min64(kChunk, n - (c0 + i) * kChunk);
    bool w = true;
    if (i >= 2 && since_drain > 0) w = mbar_wait(&S.mma_bar[t], (uint32_t)(((i - 2) >> 1) & 1), err);
    if (w) w = mbar_wait(&S.full_bar[s], (uint32_t)((i / kStages) & 1), err);
    if (!__syncthreads_and(w)) {
      ok = false;
      break;
    }
    split_chunk_i8(S.stage[s], S.tile[t], rows, S.expo);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0 && i + kStages < my) {
      const int64_t r2 = (c0 + i + kStages) * kChunk;
      const int rows2 = (int)min64(kChunk, n - r2);
      bulk_load(S.stage[s], X + r2 * kCols, (uint32_t)rows2 * kCols * 4, &S.full_bar[s]);
    }
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = smem_u32(S.tile[t]);
      for (int a = 1; a <= kSlices; a += 2) {
        for (int c = 1; c + a <= kSlices + 1; ++c) {
          const int v = a + c;  // region R_v, TMEM columns (v - 2) * 64
#pragma unroll
          for (int ks = 0; ks < kChunk / 32; ++ks) {
            const uint64_t da = smem_desc_i8(base + (a - 1) * kI8SliceBytes + ks * 2 * kI8LBO);
            const uint64_t db = smem_desc_i8(base + (c - 1) * kI8SliceBytes + ks * 2 * kI8LBO);
            mma_i8(tmem + (uint32_t)((v - 2) * 64), da, db, idesc, ((seen >> v) & 1u) || ks > 0 ? 1u : 0u);
          }
          seen |= 1u << v;
        }
      }
      mma_commit(&S.mma_bar[t]);
    }
    ++issued;
    ++since_drain;
    if (since_drain == kI8Drain || i + 1 == my) {
      drain(i);
      since_drain = 0;
      seen = 0;
      __syncthreads();
      if (!ok) break;
    }
  }
  if (!ok) {
    // bounded waits for what is still in flight before TMEM and shared memory are left: the
    // MMAs of the last issued chunk and the bulk copies of chunks issued .. loaded - 1
    const long long t0 = clock64();
    if (issued > 0) {
      const int64_t last = issued - 1;
      while (!mbar_try(&S.mma_bar[last & 1], (uint32_t)((last >> 1) & 1)) && clock64() - t0 < kWaitCycles) {
      }
    }
    const int64_t loaded = min64(my, issued + kStages);
    for (int64_t j = issued; j < loaded; ++j)
      while (!mbar_try(&S.full_bar[j % kStages], (uint32_t)((j / kStages) & 1)) && clock64() - t0 < 2 * kWaitCycles) {
      }
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
  // row r of the partial (top: column r of X, bottom: column r - 64), scaled by 2^(e_i + e_j)
  double* out = part + (int64_t)blockIdx.x * 128 * kCols;
  for (int e = tid; e < 128 * kCols; e += kI8Threads) {
    const int r = e / kCols, j = e % kCols;
    out[e] = ldexp(S.acc[e], S.expo[r & 63] + S.expo[j]);
  }
}

// G[m][n] = sum over CTAs of part[cta][m][n] + part[cta][64+m][n]; then symmetrised.  One warp
// per entry: lane l sums CTAs l, l+32, ... in order, then a fixed shuffle tree (deterministic).
constexpr int kReduceWarps = 8;

__global__ void __launch_bounds__(32 * kReduceWarps) k_gram_reduce(const double* __restrict__ part, int ctas,
                                                                   double* __restrict__ G) {
  const int idx = blockIdx.x * kReduceWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (idx >= kCols * kCols) return;
  const int m = idx / kCols, nn = idx % kCols;
  double s = 0.0, t = 0.0;
  for (int c = lane; c < ctas; c += 32) {
    s += __ldg(part + ((int64_t)c * 128 + m) * kCols + nn) + __ldg(part + ((int64_t)c * 128 + 64 + m) * kCols + nn);
    t += __ldg(part + ((int64_t)c * 128 + nn) * kCols + m) + __ldg(part + ((int64_t)c * 128 + 64 + nn) * kCols + m);
  }
  s = warp_sum(s);
  t = warp_sum(t);
  if (lane == 0) G[idx] = 0.5 * (s + t);
}

// One-block cyclic Jacobi eigensolver for a symmetric k x k FP64 matrix (k <= 64), round-robin
// ordering (k/2 disjoint rotations per round).  Eigenvalues sorted descending into w; A is
// overwritten.  Bounded by max_sweeps.
__global__ void k_symeig_jacobi(double* A, int k, double* w, double* V, int max_sweeps, int* sweeps_out) {
  extern __shared__ double jac_smem[];
  double (*a)[65] = reinterpret_cast<double (*)[65]>(jac_smem);
  double (*v)[65] = reinterpret_cast<double (*)[65]>(jac_smem + 64 * 65);
  __shared__ double cs[32], sn[32];
  __shared__ int pp[32], qq[32];
  __shared__ double off;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int kk = (k + 1) & ~1;  // even size (a zero row/col pads odd k)
  for (int i = tid; i < kk * kk; i += nt) {
    const int r = i / kk, c = i % kk;
    a[r][c] = (r < k && c < k) ? A[r * k + c] : 0.0;
    v[r][c] = r == c ? 1.0 : 0.0;
  }
  __syncthreads();
  double fro = 0.0;
  if (tid == 0) {
    for (int r = 0; r < kk; ++r)
      for (int c = 0; c < kk; ++c) fro += a[r][c] * a[r][c];
    off = fro;
  }
  __syncthreads();
  const double tol = 1e-30 * (off > 0 ? off : 1.0);
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    if (tid == 0) {
      double o = 0.0;
      for (int r = 0; r < kk; ++r)
        for (int c = 0; c < kk; ++c)
          if (r != c) o += a[r][c] * a[r][c];
      off = o;
    }
    __syncthreads();
    if (off <= tol) break;
    for (int round = 0; round < kk - 1; ++round) {
      if (tid < kk / 2) {
        // round-robin pairing: position 0 fixed, others rotate
        int i1 = tid == 0 ? 0 : ((tid - 1 + round) % (kk - 1)) + 1;
        int i2 = ((kk - 2 - tid + round) % (kk - 1)) + 1;
        const int p = min(i1, i2), q = max(i1, i2);
        const double apq = a[p][q], app = a[p][p], aqq = a[q][q];
        double c = 1.0, s = 0.0;
        if (apq != 0.0) {
          const double tau = (aqq - app) / (2.0 * apq);
          const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          c = 1.0 / sqrt(1.0 + t * t);
          s = t * c;
        }
        pp[tid] = p;
        qq[tid] = q;
        cs[tid] = c;
        sn[tid] = s;
      }
      __syncthreads();
      // rows: a <- J^T a
      for (int i = tid; i < (kk / 2) * kk; i += nt) {
        const int r = i / kk, col = i % kk;
        const int p = pp[r], q = qq[r];
        const double c = cs[r], s = sn[r];
        const double x = a[p][col], y = a[q][col];
        a[p][col] = c * x - s * y;
        a[q][col] = s * x + c * y;
      }
      __syncthreads();
      // columns: a <- a J ; v <- v J
      for (int i = tid; i < (kk / 2) * kk; i += nt) {
        const int r = i / kk, row = i % kk;
        const int p = pp[r], q = qq[r];
        const double c = cs[r], s = sn[r];
        const double x = a[row][p], y = a[row][q];
        a[row][p] = c * x - s * y;
        a[row][q] = s * x + c * y;
        const double vx = v[row][p], vy = v[row][q];
        v[row][p] = c * vx - s * vy;
        v[row][q] = s * vx + c * vy;
      }
      __syncthreads();
    }
  }
  if (tid == 0) {
    // selection sort of the diagonal, descending (k <= 64)
    int order[64];
    for (int i = 0; i < k; ++i) order[i] = i;
    for (int i = 0; i < k; ++i) {
      int best = i;
      for (int j = i + 1; j < k; ++j)
        if (a[order[j]][order[j]] > a[order[best]][order[best]]) best = j;
      const int t = order[i];
      order[i] = order[best];
      order[best] = t;
    }
    for (int i = 0; i < k; ++i) {
      w[i] = a[order[i]][order[i]];
      if (V)
        for (int r = 0; r < k; ++r) V[r * k + i] = v[r][order[i]];
    }
    if (sweeps_out) *sweeps_out = sweep;
  }
}

// FP64 Gram on the CUDA cores: G = X^T X accumulated in FP64 for X (n x 64, FP32 or FP64, row
// major).  The split-bf16 tensor-core Gram accumulates in FP32, which resolves eigenvalues down to
// about 1e-6 of the largest; snapshot sets of elastic solutions decay much faster (lambda_10 /
// lambda_1 ~ 1e-8), and their trailing singular values need FP64 accumulation.
// One CTA per SM; 256 threads = 4 row groups x 64 threads; thread (bi, bj) of a row group owns
// G[bi + 8u][bj + 8v] (u, v < 8, interleaved so that shared-memory reads are contiguous across
// the warp) and accumulates the rows r = rg (mod 4) of each 64-row tile.  The next tile is read
// into registers while the current one is consumed.  Row groups are summed in a fixed order
// through shared memory, CTAs by k_gram_reduce64, so G is deterministic.
constexpr int kGTile = 64;
constexpr int kGThreads = 256;

template <typename T>
__device__ __forceinline__ void gram_load_tile(const T* __restrict__ X, int64_t n, int64_t r0, double (&reg)[16]) {
  // 64 rows x 64 values: thread t loads values t, t + 256, ... (16 per thread), coalesced
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int e = threadIdx.x + kGThreads * i;
    const int r = e >> 6, c = e & 63;
    reg[i] = (r0 + r < n) ? (double)__ldcs(X + (r0 + r) * kCols + c) : 0.0;
  }
}

template <typename T>
__global__ void __launch_bounds__(kGThreads, 1) k_gram_fp64(const T* __restrict__ X, int64_t n,
                                                          double* __restrict__ part) {
  __shared__ double xs[kGTile * kCols];  // 32 KB: one tile, then the row-group reduction
  const int tid = threadIdx.x, rg = tid >> 6, t = tid & 63, bi = t >> 3, bj = t & 7;
  double acc[8][8];
#pragma unroll
  for (int u = 0; u < 8; ++u)
#pragma unroll
    for (int v = 0; v < 8; ++v) acc[u][v] = 0.0;
  const int64_t tiles = (n + kGTile - 1) / kGTile;
  double reg[16];
  int64_t tile = blockIdx.x;
  if (tile < tiles) gram_load_tile(X, n, tile * kGTile, reg);
  for (; tile < tiles; tile += gridDim.x) {
    __syncthreads();  // the previous tile is consumed
#pragma unroll
    for (int i = 0; i < 16; ++i) xs[threadIdx.x + kGThreads * i] = reg[i];
    __syncthreads();
    if (tile + gridDim.x < tiles) gram_load_tile(X, n, (tile + gridDim.x) * kGTile, reg);
    for (int r = rg; r < kGTile; r += 4) {  // rows past n were stored as zeros
      const double* row = xs + r * kCols;
      double a[8], b[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        a[u] = row[bi + 8 * u];
        b[u] = row[bj + 8 * u];
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
  }
  // row groups 0..3 summed in order
  for (int g = 0; g < 4; ++g) {
    __syncthreads();
    if (rg == g) {
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) {
          const int idx = (bi + 8 * u) * kCols + bj + 8 * v;
          xs[idx] = g == 0 ? acc[u][v] : xs[idx] + acc[u][v];
        }
    }
  }
  __syncthreads();
  for (int e = tid; e < kCols * kCols; e += kGThreads) part[(int64_t)blockIdx.x * kCols * kCols + e] = xs[e];
}

// G = sum over CTAs of part[cta], symmetrised; one warp per entry as k_gram_reduce (deterministic).
__global__ void __launch_bounds__(32 * kReduceWarps) k_gram_reduce64(const double* __restrict__ part, int ctas,
                                                                     double* __restrict__ G) {
  const int idx = blockIdx.x * kReduceWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (idx >= kCols * kCols) return;
  const int m = idx / kCols, nn = idx % kCols;
  double s = 0.0, t = 0.0;
  for (int c = lane; c < ctas; c += 32) {
    s += __ldg(part + (int64_t)c * kCols * kCols + m * kCols + nn);
    t += __ldg(part + (int64_t)c * kCols * kCols + nn * kCols + m);
  }
  s = warp_sum(s);
  t = warp_sum(t);
  if (lane == 0) G[idx] = 0.5 * (s + t);
}

int gram_fp64_grid(int64_t n) {
  const int64_t tiles = (n + kGTile - 1) / kGTile;
  return (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)sm_count()));
}

int gram_grid(int64_t n) {
  const int64_t chunks = (n + kChunk - 1) / kChunk;
  return (int)std::max<int64_t>(1, std::min<int64_t>(chunks, (int64_t)sm_count() * 2));
}

}  // namespace
}  // namespace feab

using namespace feab;

extern "C" size_t feab_gram_workspace_bytes(int64_t n, int32_t k) {
  if (n <= 0 || k != kCols) return 0;
  return sizeof(double) * (size_t)gram_grid(n) * 128 * kCols + 256;
}

extern "C" int32_t feab_gram_bf16x3(const float* X, int64_t n, int32_t k, double* G, void* workspace,
                                    size_t workspace_bytes, int32_t* error_flag, cudaStream_t s) {
  if (!X || !G || !workspace || !error_flag || n <= 0 || k != kCols) return FEAB_BAD_ARG;
  if ((reinterpret_cast<uintptr_t>(X) & 15) != 0) return FEAB_BAD_ARG;  // bulk copies need 16 B alignment
  if (feab_gram_workspace_bytes(n, k) > workspace_bytes) return FEAB_BAD_ARG;
  const int grid = gram_grid(n);
  const size_t smem = sizeof(GramSmem) + 1024;
  FEAB_CUDA(cudaFuncSetAttribute(k_gram_bf16x3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  double* part = static_cast<double*>(workspace);
  k_gram_bf16x3<<<grid, kThreadsG, smem, s>>>(X, n, part, error_flag);
  k_gram_reduce<<<(kCols * kCols + kReduceWarps - 1) / kReduceWarps, 32 * kReduceWarps, 0, s>>>(part, grid, G);
  count_launches(2);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}

extern "C" int32_t feab_gram_fp64(const void* X, int32_t x_bytes, int64_t n, int32_t k, double* G, void* workspace,
                                  size_t workspace_bytes, cudaStream_t s) {
  if (!X || !G || !workspace || n <= 0 || k != kCols || (x_bytes != 4 && x_bytes != 8)) return FEAB_BAD_ARG;
  if (feab_gram_workspace_bytes(n, k) > workspace_bytes) return FEAB_BAD_ARG;
  const int grid = gram_fp64_grid(n);
  double* part = static_cast<double*>(workspace);
  if (x_bytes == 4) k_gram_fp64<float><<<grid, kGThreads, 0, s>>>(static_cast<const float*>(X), n, part);
  else k_gram_fp64<double><<<grid, kGThreads, 0, s>>>(static_cast<const double*>(X), n, part);
  k_gram_reduce64<<<(kCols * kCols + kReduceWarps - 1) / kReduceWarps, 32 * kReduceWarps, 0, s>>>(part, grid, G);
  count_launches(2);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}

extern "C" int32_t feab_symeig_jacobi(double* A, int32_t k, double* evals, double* evecs, int32_t max_sweeps,
                                      int32_t* sweeps_out, cudaStream_t s) {
  if (!A || !evals || k <= 0 || k > 64) return FEAB_BAD_ARG;
  const size_t smem = sizeof(double) * 2 * 64 * 65;
  FEAB_CUDA(cudaFuncSetAttribute(k_symeig_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_symeig_jacobi<<<1, 256, smem, s>>>(A, k, evals, evecs, max_sweeps > 0 ? max_sweeps : 40, sweeps_out);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}

extern "C" int32_t feab_gram_int8(const float* X, int64_t n, int32_t k, double* G, void* workspace,
                                  size_t workspace_bytes, int32_t* error_flag, cudaStream_t s) {
  if (!X || !G || !workspace || !error_flag || n <= 0 || k != kCols) return FEAB_BAD_ARG;
  if ((reinterpret_cast<uintptr_t>(X) & 15) != 0) return FEAB_BAD_ARG;  // bulk copies and float4 reads
  if (feab_gram_workspace_bytes(n, k) > workspace_bytes) return FEAB_BAD_ARG;
  const int64_t chunks = (n + kChunk - 1) / kChunk;
  // contiguous row ranges, one CTA per SM; each CTA's chunk count bounds the int32 drains
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(chunks, (int64_t)sm_count()));
  const size_t smem = sizeof(Int8Smem) + 1024;
  FEAB_CUDA(cudaFuncSetAttribute(k_gram_int8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  double* part = static_cast<double*>(workspace);
  k_gram_int8<<<grid, kI8Threads, smem, s>>>(X, n, part, error_flag);
  k_gram_reduce<<<(kCols * kCols + kReduceWarps - 1) / kReduceWarps, 32 * kReduceWarps, 0, s>>>(part, grid, G);
  count_launches(2);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}
