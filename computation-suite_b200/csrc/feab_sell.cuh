// Sliced (SELL-32) node-group operator: device-side view and the per-lane row-group product.
//
// Node row groups (the 1-3 rows of one mesh node, which share one column list) are cut into
// slices of 32 consecutive groups; one warp takes a slice and lane l owns group 32 s + l.
// Slice s holds W_s column steps (a multiple of 4) from step soff[s]; steps come in blocks of 4,
// and within a block each lane's 4 entries are contiguous.  For the block starting at step b
// (b = soff[s] + 4i) and lane l:
//   columns    tcol[b * 32 + 4 l + u]                 u = 0..3, the 4 steps of the block
//   row k      value[(3 b + 4 k) * 32 + 4 l + u]      k = 0..2
// (or, when every column lies within 16 bits of the lane's first row, the 2-byte offsets
//   tcol16[b * 32 + 4 l + u] = column - r0, one 8-byte load per block),
// so per block a lane issues one 16-byte column load and, per row, one 16-byte (32-bit hi words)
// + one 8-byte (16-bit lo words) load, or two 16-byte FP64 loads; the warp's loads are 512 (or
// 256) contiguous bytes.  A lane accumulates its rows alone, in column order, with no cross-lane
// reduction.  Steps past a group's length point at the node's own first free DOF with value 0,
// so their contribution is exactly 0.
#pragma once
#include "feab_common.cuh"

// Blocks of 4 steps that a warp asks L2 to fetch ahead of its loads (0: none).
#ifndef FEAB_SELL_PREFETCH
#define FEAB_SELL_PREFETCH 0
#endif
// Blocks of 4 steps whose loads a lane issues before it consumes any, per operator kind.
#ifndef FEAB_SELL_BLOCKS_FP64
#define FEAB_SELL_BLOCKS_FP64 2
#endif
#ifndef FEAB_SELL_BLOCKS_MIXED
#define FEAB_SELL_BLOCKS_MIXED 1
#endif
// 1: load the operator with the streaming (evict-first) cache hint, so that the CG vectors
// (a few MB, re-read every iteration) stay in L2 while K streams through it.
#ifndef FEAB_SELL_STREAM
#define FEAB_SELL_STREAM 1
#endif
// 1: the PCG forms p = z + beta p inside the sliced SpMV's gathers (two gathers per column)
// instead of a separate pass.
#ifndef FEAB_SELL_FUSED_P
#define FEAB_SELL_FUSED_P 0
#endif
// Minimum resident 256-thread CTAs per SM for the sliced SpMV kernels (register budget), per
// operator kind.  Measured in the PCG at 128x32x32: the 48-bit kernel runs 54.4 us per iteration
// at 4 CTAs with one block in flight against 57.5 us at 2 CTAs with two; the FP64 kernel is
// fastest at 2 CTAs with two blocks.
#ifndef FEAB_SELL_MINB_FP64
#define FEAB_SELL_MINB_FP64 2
#endif
#ifndef FEAB_SELL_MINB_MIXED
#define FEAB_SELL_MINB_MIXED 4
#endif
// 1: software pipelining, one block of 4 steps: a lane issues the loads of block i + 1 before the
// gathers and products of block i, so the operator's DRAM latency overlaps the gathers' L2
// latency (per operator kind; replaces FEAB_SELL_BLOCKS_* and uses FEAB_SELL_PIPE_MINB_*).
// Measured in the PCG at 128x32x32 and left off: the second block's registers (80 for the 48-bit
// kernel, 3 CTAs per SM; 98 for FP64) cost more warps than the overlap gains, 63.9 against 51.8 us
// per iteration (mixed) and 62.4 against 59.4 us (FP64).
#ifndef FEAB_SELL_PIPE_FP64
#define FEAB_SELL_PIPE_FP64 0
#endif
#ifndef FEAB_SELL_PIPE_MIXED
#define FEAB_SELL_PIPE_MIXED 0
#endif
#ifndef FEAB_SELL_PIPE_MINB_FP64
#define FEAB_SELL_PIPE_MINB_FP64 2
#endif
#ifndef FEAB_SELL_PIPE_MINB_MIXED
#define FEAB_SELL_PIPE_MINB_MIXED 3
#endif

namespace feab {

template <typename T>
__device__ __forceinline__ T ld_op(const T* p) {
#if FEAB_SELL_STREAM
  return __ldcs(p);
#else
  return __ldg(p);
#endif
}

__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

struct SellView {
  int kind;                 // FEAB_PREC_FP64: plain y = K x; FEAB_PREC_MIXED: difference form
  int n_slices, n_groups;
  const int32_t* soff;
  const int32_t* tcol;
  const int16_t* tcol16;    // 2-byte column offsets from the lane's first row (or NULL)
  const double* v64;
  const uint32_t* vhi;
  const uint16_t* vlo;
  const uint8_t* gmask;
  const double* S;
  const int32_t* group_ptr;
};

// The lane's group: rows r0 .. r0+f-1 and (difference form) its free-DOF mask.
struct SellLane {
  int r0, f, mask;
  bool valid;
};

__device__ __forceinline__ SellLane sell_lane(const SellView& V, int slice, int lane) {
  SellLane L;
  const int g = slice * 32 + lane;
  L.valid = g < V.n_groups;
  L.r0 = L.valid ? __ldg(V.group_ptr + g) : 0;
  L.f = L.valid ? __ldg(V.group_ptr + g + 1) - L.r0 : 0;
  L.mask = (L.valid && V.gmask) ? __ldg(V.gmask + g) : 0;
  return L;
}

__device__ __forceinline__ double sell_dec48(uint32_t hi, uint16_t lo) {
  return __longlong_as_double((long long)(((unsigned long long)hi << 32) | ((unsigned long long)lo << 16)));
}

// Per-kind load depth and register budget of the sliced SpMV kernels.
template <int KIND>
struct SellTuning {
  static constexpr bool kPipe = KIND == FEAB_PREC_FP64 ? FEAB_SELL_PIPE_FP64 != 0 : FEAB_SELL_PIPE_MIXED != 0;
  static constexpr int kBlocks = KIND == FEAB_PREC_FP64 ? FEAB_SELL_BLOCKS_FP64 : FEAB_SELL_BLOCKS_MIXED;
  static constexpr int kMinBlocks =
      kPipe ? (KIND == FEAB_PREC_FP64 ? FEAB_SELL_PIPE_MINB_FP64 : FEAB_SELL_PIPE_MINB_MIXED)
            : (KIND == FEAB_PREC_FP64 ? FEAB_SELL_MINB_FP64 : FEAB_SELL_MINB_MIXED);
};

// One block of 4 steps of a lane: its columns and its rows' values as loaded.
template <int KIND>
struct SellBlock {
  unsigned t[4];
  double v[KIND == FEAB_PREC_FP64 ? 3 : 1][4];
  uint4 h[KIND == FEAB_PREC_FP64 ? 1 : 3];
  uint2 l[KIND == FEAB_PREC_FP64 ? 1 : 3];
};

// Issues the loads of the block starting at step b (columns decoded to absolute indices; the
// difference form's tag bits masked off).
template <int KIND, bool IDX16>
__device__ __forceinline__ void sell_load_block(const SellView& V, size_t b, int lane, int r0, SellBlock<KIND>& B) {
  if (IDX16) {
    const uint2 tq = ld_op(reinterpret_cast<const uint2*>(V.tcol16 + b * 32) + lane);
    B.t[0] = (unsigned)(r0 + (int)(int16_t)(tq.x & 0xffffu));
    B.t[1] = (unsigned)(r0 + (int)(int16_t)(tq.x >> 16));
    B.t[2] = (unsigned)(r0 + (int)(int16_t)(tq.y & 0xffffu));
    B.t[3] = (unsigned)(r0 + (int)(int16_t)(tq.y >> 16));
  } else {
    const uint4 tq = ld_op(reinterpret_cast<const uint4*>(V.tcol + b * 32) + lane);
    const unsigned m = KIND == FEAB_PREC_FP64 ? 0xffffffffu : 0x3fffffffu;
    B.t[0] = tq.x & m;
    B.t[1] = tq.y & m;
    B.t[2] = tq.z & m;
    B.t[3] = tq.w & m;
  }
  if (KIND == FEAB_PREC_FP64) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double2* vp = reinterpret_cast<const double2*>(V.v64 + (3 * b + 4 * k) * 32) + 2 * lane;
      const double2 p0 = ld_op(vp), p1 = ld_op(vp + 1);
      B.v[k][0] = p0.x;
      B.v[k][1] = p0.y;
      B.v[k][2] = p1.x;
      B.v[k][3] = p1.y;
    }
  } else {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const size_t o = (3 * b + 4 * k) * 32;
      B.h[k] = ld_op(reinterpret_cast<const uint4*>(V.vhi + o) + lane);
      B.l[k] = ld_op(reinterpret_cast<const uint2*>(V.vlo + o) + lane);
    }
  }
}

// a_k += sum_u value(k, u) d[u] over the block's 4 steps.
template <int KIND>
__device__ __forceinline__ void sell_use_block(const SellBlock<KIND>& B, const double (&d)[4], double& a0,
                                               double& a1, double& a2) {
  if (KIND == FEAB_PREC_FP64) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a0 = fma(B.v[0][u], d[u], a0);
      a1 = fma(B.v[1][u], d[u], a1);
      a2 = fma(B.v[2][u], d[u], a2);
    }
  } else {
    double* acc[3] = {&a0, &a1, &a2};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double a = *acc[k];
      a = fma(sell_dec48(B.h[k].x, (uint16_t)(B.l[k].x & 0xffffu)), d[0], a);
      a = fma(sell_dec48(B.h[k].y, (uint16_t)(B.l[k].x >> 16)), d[1], a);
      a = fma(sell_dec48(B.h[k].z, (uint16_t)(B.l[k].y & 0xffffu)), d[2], a);
      a = fma(sell_dec48(B.h[k].w, (uint16_t)(B.l[k].y >> 16)), d[3], a);
      *acc[k] = a;
    }
  }
}

// acc[k] = (K x)[r0 + k] for the lane's group, x read through xf(column).  Mixed kind: the
// difference form sum_{b != a} w (x_b - x_a) + S x_a, evaluated as sum_{b != a} w x_b + T x_a
// with T = S - sum_{b != a} w precomputed (the same value exactly, so the same rounding error of
// the 36-bit values); xs[j] = x of the node's own DOF component j (0 when that component is fixed).
template <int KIND, bool IDX16, typename XF>
__device__ __forceinline__ void sell_apply(const SellView& V, int slice, int lane, const SellLane& L, XF xf,
                                           double (&acc)[3], double (&xs)[3]) {
  constexpr int NB = SellTuning<KIND>::kBlocks;
  const int base = __ldg(V.soff + slice), W = __ldg(V.soff + slice + 1) - base;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll
  for (int j = 0; j < 3; ++j)
    xs[j] = (KIND == FEAB_PREC_MIXED && L.valid && ((L.mask >> j) & 1)) ? xf(L.r0 + __popc(L.mask & ((1 << j) - 1)))
                                                                       : 0.0;
  // one lane asks L2 for the blocks FEAB_SELL_PREFETCH ahead (16-byte aligned, sizes multiple of
  // 16, never past the slice's last block)
  auto prefetch_block = [&](int jj) {
    if (FEAB_SELL_PREFETCH > 0 && lane == 0 && jj < W) {
      const size_t b2 = (size_t)(base + jj);
      prefetch_l2(V.tcol + b2 * 32, 512u);
      if (KIND == FEAB_PREC_FP64) {
        prefetch_l2(V.v64 + 3 * b2 * 32, 3072u);
      } else {
        prefetch_l2(V.vhi + 3 * b2 * 32, 1536u);
        prefetch_l2(V.vlo + 3 * b2 * 32, 768u);
      }
    }
  };
#pragma unroll
  for (int i = 1; i < FEAB_SELL_PREFETCH; ++i) prefetch_block(4 * i);
  if constexpr (SellTuning<KIND>::kPipe) {
    // block i + 1's loads are in flight while block i's gathers and products run
    SellBlock<KIND> cur, nxt;
    if (W > 0) sell_load_block<KIND, IDX16>(V, (size_t)base, lane, L.r0, cur);
    for (int j = 0; j < W; j += 4) {
      if (j + 4 < W) sell_load_block<KIND, IDX16>(V, (size_t)(base + j + 4), lane, L.r0, nxt);
      double d[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) d[u] = xf((int)cur.t[u]);
      sell_use_block<KIND>(cur, d, a0, a1, a2);
      cur = nxt;
    }
  } else
  for (int j = 0; j < W; j += 4 * NB) {
    prefetch_block(j + 4 * FEAB_SELL_PREFETCH);
    // all loads of NB blocks first (a block past the slice end is skipped; W is
    // the same for the whole warp, so the test does not diverge)
    unsigned t[NB][4];
    double v[KIND == FEAB_PREC_FP64 ? NB : 1][3][4];
    uint4 h[KIND == FEAB_PREC_FP64 ? 1 : NB][3];
    uint2 l[KIND == FEAB_PREC_FP64 ? 1 : NB][3];
#pragma unroll
    for (int nb = 0; nb < NB; ++nb) {
      if (nb > 0 && j + 4 * nb >= W) break;
      const size_t b = (size_t)(base + j + 4 * nb);
      if (IDX16) {
        const uint2 tq = ld_op(reinterpret_cast<const uint2*>(V.tcol16 + b * 32) + lane);
        t[nb][0] = (unsigned)(L.r0 + (int)(int16_t)(tq.x & 0xffffu));
        t[nb][1] = (unsigned)(L.r0 + (int)(int16_t)(tq.x >> 16));
        t[nb][2] = (unsigned)(L.r0 + (int)(int16_t)(tq.y & 0xffffu));
        t[nb][3] = (unsigned)(L.r0 + (int)(int16_t)(tq.y >> 16));
      } else {
        const uint4 tq = ld_op(reinterpret_cast<const uint4*>(V.tcol + b * 32) + lane);
        t[nb][0] = tq.x;
        t[nb][1] = tq.y;
        t[nb][2] = tq.z;
        t[nb][3] = tq.w;
      }
      if (KIND == FEAB_PREC_FP64) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double2* vp = reinterpret_cast<const double2*>(V.v64 + (3 * b + 4 * k) * 32) + 2 * lane;
          const double2 p0 = ld_op(vp), p1 = ld_op(vp + 1);
          v[nb][k][0] = p0.x;
          v[nb][k][1] = p0.y;
          v[nb][k][2] = p1.x;
          v[nb][k][3] = p1.y;
        }
      } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const size_t o = (3 * b + 4 * k) * 32;
          h[nb][k] = ld_op(reinterpret_cast<const uint4*>(V.vhi + o) + lane);
          l[nb][k] = ld_op(reinterpret_cast<const uint2*>(V.vlo + o) + lane);
        }
      }
    }
#pragma unroll
    for (int nb = 0; nb < NB; ++nb) {
      if (nb > 0 && j + 4 * nb >= W) break;
      if (KIND == FEAB_PREC_FP64) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const double xv = xf((int)t[nb][u]);
          a0 = fma(v[nb][0][u], xv, a0);
          a1 = fma(v[nb][1][u], xv, a1);
          a2 = fma(v[nb][2][u], xv, a2);
        }
      } else {
        double d[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) d[u] = xf((int)(t[nb][u] & 0x3fffffffu));
        const uint4* hh = h[nb];
        const uint2* ll = l[nb];
        a0 = fma(sell_dec48(hh[0].x, (uint16_t)(ll[0].x & 0xffffu)), d[0], a0);
        a0 = fma(sell_dec48(hh[0].y, (uint16_t)(ll[0].x >> 16)), d[1], a0);
        a0 = fma(sell_dec48(hh[0].z, (uint16_t)(ll[0].y & 0xffffu)), d[2], a0);
        a0 = fma(sell_dec48(hh[0].w, (uint16_t)(ll[0].y >> 16)), d[3], a0);
        a1 = fma(sell_dec48(hh[1].x, (uint16_t)(ll[1].x & 0xffffu)), d[0], a1);
        a1 = fma(sell_dec48(hh[1].y, (uint16_t)(ll[1].x >> 16)), d[1], a1);
        a1 = fma(sell_dec48(hh[1].z, (uint16_t)(ll[1].y & 0xffffu)), d[2], a1);
        a1 = fma(sell_dec48(hh[1].w, (uint16_t)(ll[1].y >> 16)), d[3], a1);
        a2 = fma(sell_dec48(hh[2].x, (uint16_t)(ll[2].x & 0xffffu)), d[0], a2);
        a2 = fma(sell_dec48(hh[2].y, (uint16_t)(ll[2].x >> 16)), d[1], a2);
        a2 = fma(sell_dec48(hh[2].z, (uint16_t)(ll[2].y & 0xffffu)), d[2], a2);
        a2 = fma(sell_dec48(hh[2].w, (uint16_t)(ll[2].y >> 16)), d[3], a2);
      }
    }
  }
  if (KIND == FEAB_PREC_MIXED) {
    const double* __restrict__ Sp = V.S + (int64_t)L.r0 * 3;
    if (L.f > 0) a0 += __ldg(Sp) * xs[0] + __ldg(Sp + 1) * xs[1] + __ldg(Sp + 2) * xs[2];
    if (L.f > 1) a1 += __ldg(Sp + 3) * xs[0] + __ldg(Sp + 4) * xs[1] + __ldg(Sp + 5) * xs[2];
    if (L.f > 2) a2 += __ldg(Sp + 6) * xs[0] + __ldg(Sp + 7) * xs[1] + __ldg(Sp + 8) * xs[2];
  }
  acc[0] = a0;
  acc[1] = a1;
  acc[2] = a2;
}

SellView sell_view(const feab_csr* A, const feab_sell_operator* op);

// y = K x through the sliced operator (one warp per slice), on stream s.
void launch_sell_spmv(const SellView& V, const double* x, double* y, cudaStream_t s);

}  // namespace feab
