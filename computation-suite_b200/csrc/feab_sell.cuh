// Sliced (SELL-32) node-group operator: device-side view and the per-lane row-group product.
//
// Node row groups (the 1-3 rows of one mesh node, which share one column list) are cut into
// slices of 32 consecutive groups; one warp takes a slice and lane l owns group 32 s + l.
// Slice s holds W_s column steps (a multiple of 4) from step soff[s]; steps come in blocks of 4,
// and within a block each lane's 4 entries are contiguous.  For the block starting at step b
// (b = soff[s] + 4i) and lane l:
//   columns    tcol[b * 32 + 4 l + u]                 u = 0..3, the 4 steps of the block
//   row k      value[(3 b + 4 k) * 32 + 4 l + u]      k = 0..2
// so per block a lane issues one 16-byte column load and, per row, one 16-byte (32-bit hi words)
// + one 8-byte (16-bit lo words) load, or two 16-byte FP64 loads; the warp's loads are 512 (or
// 256) contiguous bytes.  A lane accumulates its rows alone, in column order, with no cross-lane
// reduction.  Steps past a group's length point at the node's own first free DOF with value 0,
// so their contribution is exactly 0.
#pragma once
#include "feab_common.cuh"

namespace feab {

struct SellView {
  int kind;                 // FEAB_PREC_FP64: plain y = K x; FEAB_PREC_MIXED: difference form
  int n_slices, n_groups;
  const int32_t* soff;
  const int32_t* tcol;
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

// acc[k] = (K x)[r0 + k] for the lane's group, x read through xf(column).  For the difference
// form xs[j] = x of the node's own DOF component j (0 when that component is fixed).
template <int KIND, typename XF>
__device__ __forceinline__ void sell_apply(const SellView& V, int slice, int lane, const SellLane& L, XF xf,
                                           double (&acc)[3], double (&xs)[3]) {
  const int base = __ldg(V.soff + slice), W = __ldg(V.soff + slice + 1) - base;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll
  for (int j = 0; j < 3; ++j)
    xs[j] = (KIND == FEAB_PREC_MIXED && L.valid && ((L.mask >> j) & 1)) ? xf(L.r0 + __popc(L.mask & ((1 << j) - 1)))
                                                                       : 0.0;
  for (int j = 0; j < W; j += 4) {
    const size_t b = (size_t)(base + j);
    const uint4 tq = __ldg(reinterpret_cast<const uint4*>(V.tcol + b * 32) + lane);
    const unsigned t[4] = {tq.x, tq.y, tq.z, tq.w};
    if (KIND == FEAB_PREC_FP64) {
      double v[3][4];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double2* vp = reinterpret_cast<const double2*>(V.v64 + (3 * b + 4 * k) * 32) + 2 * lane;
        const double2 p0 = __ldg(vp), p1 = __ldg(vp + 1);
        v[k][0] = p0.x;
        v[k][1] = p0.y;
        v[k][2] = p1.x;
        v[k][3] = p1.y;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double xv = xf((int)t[u]);
        a0 = fma(v[0][u], xv, a0);
        a1 = fma(v[1][u], xv, a1);
        a2 = fma(v[2][u], xv, a2);
      }
    } else {
      uint4 h[3];
      uint2 l[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const size_t o = (3 * b + 4 * k) * 32;
        h[k] = __ldg(reinterpret_cast<const uint4*>(V.vhi + o) + lane);
        l[k] = __ldg(reinterpret_cast<const uint2*>(V.vlo + o) + lane);
      }
      double d[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const unsigned jc = t[u] >> 30;
        d[u] = xf((int)(t[u] & 0x3fffffffu)) - (jc == 0u ? xs[0] : (jc == 1u ? xs[1] : xs[2]));
      }
      a0 = fma(sell_dec48(h[0].x, (uint16_t)(l[0].x & 0xffffu)), d[0], a0);
      a0 = fma(sell_dec48(h[0].y, (uint16_t)(l[0].x >> 16)), d[1], a0);
      a0 = fma(sell_dec48(h[0].z, (uint16_t)(l[0].y & 0xffffu)), d[2], a0);
      a0 = fma(sell_dec48(h[0].w, (uint16_t)(l[0].y >> 16)), d[3], a0);
      a1 = fma(sell_dec48(h[1].x, (uint16_t)(l[1].x & 0xffffu)), d[0], a1);
      a1 = fma(sell_dec48(h[1].y, (uint16_t)(l[1].x >> 16)), d[1], a1);
      a1 = fma(sell_dec48(h[1].z, (uint16_t)(l[1].y & 0xffffu)), d[2], a1);
      a1 = fma(sell_dec48(h[1].w, (uint16_t)(l[1].y >> 16)), d[3], a1);
      a2 = fma(sell_dec48(h[2].x, (uint16_t)(l[2].x & 0xffffu)), d[0], a2);
      a2 = fma(sell_dec48(h[2].y, (uint16_t)(l[2].x >> 16)), d[1], a2);
      a2 = fma(sell_dec48(h[2].z, (uint16_t)(l[2].y & 0xffffu)), d[2], a2);
      a2 = fma(sell_dec48(h[2].w, (uint16_t)(l[2].y >> 16)), d[3], a2);
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
