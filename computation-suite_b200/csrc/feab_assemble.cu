// Deterministic gather assembly of the reduced CSR values (c).
//
// One warp per mesh node a.  The warp keeps the three rows of a (3 x n_nbrs x 3 doubles) in
// shared memory, walks a's incident elements in ascending element order and adds the
// element blocks K_e(la, lb) into the slot of neighbour b.  Every slot is touched by one
// lane per element, so each CSR entry is summed over its elements in ascending element
// order with no atomics: the result is bit-reproducible run to run.  The rows are then
// streamed out in CSR order (FP64 values, FP32 copy, Jacobi inverse diagonal).
#include "feab_hex8.cuh"

namespace feab {
namespace {

constexpr int kWarps = 8;

__device__ __forceinline__ int lower_bound_i32(const int32_t* a, int n, int key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kWarps * 32) k_assemble(
    const double* __restrict__ ke, const int32_t* __restrict__ conn, const int32_t* __restrict__ inc_ptr,
    const int32_t* __restrict__ inc_elem, const int32_t* __restrict__ nbr_ptr, const int32_t* __restrict__ nbr_idx,
    int32_t n_nodes, int32_t max_nbrs, const int32_t* __restrict__ free_map, const int32_t* __restrict__ row_ptr,
    double* __restrict__ vals64, float* __restrict__ vals32, double* __restrict__ dinv64, float* __restrict__ dinv32,
    feab_device_status* st) {
  extern __shared__ unsigned char smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int a = blockIdx.x * kWarps + w;
  if (a >= n_nodes) return;
  // per-warp shared layout: acc[9*max_nbrs] doubles | nbr[max_nbrs] | off[max_nbrs]
  double* acc = reinterpret_cast<double*>(smem) + (size_t)w * 9 * max_nbrs;
  int32_t* nbr = reinterpret_cast<int32_t*>(reinterpret_cast<double*>(smem) + (size_t)kWarps * 9 * max_nbrs) +
                 (size_t)w * 2 * max_nbrs;
  int32_t* off = nbr + max_nbrs;

  int rows[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) rows[i] = free_map[3 * a + i];
  if (rows[0] < 0 && rows[1] < 0 && rows[2] < 0) return;  // no free row on this node

  const int s = nbr_ptr[a], nnb = nbr_ptr[a + 1] - s;
  if (nnb > max_nbrs) {
    if (lane == 0) set_status(reinterpret_cast<int*>(st), FEAB_CAPACITY, a);
    return;
  }
  int carry = 0;
  for (int k0 = 0; k0 < nnb; k0 += 32) {
    const int k = k0 + lane;
    int fb = 0;
    if (k < nnb) {
      const int b = nbr_idx[s + k];
      nbr[k] = b;
      fb = (free_map[3 * b] >= 0) + (free_map[3 * b + 1] >= 0) + (free_map[3 * b + 2] >= 0);
    }
    const int incl = warp_incl_scan(fb, lane);
    if (k < nnb) off[k] = carry + incl - fb;
    carry += __shfl_sync(FEAB_FULL_MASK, incl, 31);
  }
  for (int t = lane; t < 9 * nnb; t += 32) acc[t] = 0.0;
  __syncwarp();

  for (int k = inc_ptr[a]; k < inc_ptr[a + 1]; ++k) {
    const int64_t e = inc_elem[k];
    const int cl = conn[e * 8 + (lane & 7)];
    const unsigned m = __ballot_sync(FEAB_FULL_MASK, lane < 8 && cl == a);
    const int la = __ffs(m) - 1;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int t = lane + 32 * r;
      const int lb = min(t / 9, 7);
      const int b = __shfl_sync(FEAB_FULL_MASK, cl, lb);
      if (t < 72) {
        const int i = (t % 9) / 3, j = t % 3;
        const double val = la <= lb ? ke[(e * 36 + packed_block(la, lb)) * 9 + i * 3 + j]
                                    : ke[(e * 36 + packed_block(lb, la)) * 9 + j * 3 + i];
        const int pb = lower_bound_i32(nbr, nnb, b);
        acc[(i * nnb + pb) * 3 + j] += val;
      }
    }
    __syncwarp();
  }

#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int r = rows[i];
    if (r < 0) continue;
    const int64_t base = row_ptr[r];
    for (int t = lane; t < 3 * nnb; t += 32) {
      const int kk = t / 3, j = t % 3;
      const int b = nbr[kk];
      const int f0 = free_map[3 * b], f1 = free_map[3 * b + 1], f2 = free_map[3 * b + 2];
      const int c = j == 0 ? f0 : (j == 1 ? f1 : f2);
      if (c < 0) continue;
      const int jj = (j > 0 && f0 >= 0) + (j > 1 && f1 >= 0);
      const int64_t pos = base + off[kk] + jj;
      const double v = acc[(i * nnb + kk) * 3 + j];
      vals64[pos] = v;
      if (vals32) vals32[pos] = (float)v;
      if (b == a && j == i) {
        if (v == 0.0) set_status(reinterpret_cast<int*>(st), FEAB_ZERO_DIAGONAL, r);
        const double di = 1.0 / v;
        if (dinv64) dinv64[r] = di;
        if (dinv32) dinv32[r] = (float)di;
      }
    }
  }
}

}  // namespace
}  // namespace feab

using namespace feab;

extern "C" int32_t feab_assemble_csr(const double* ke_packed, const int32_t* conn, const int32_t* inc_ptr,
                                     const int32_t* inc_elem, const int32_t* nbr_ptr, const int32_t* nbr_idx,
                                     int32_t n_nodes, int32_t max_nbrs, const int32_t* free_map,
                                     const int32_t* row_ptr, double* vals64, float* vals32, double* dinv64,
                                     float* dinv32, feab_device_status* status, cudaStream_t s) {
  if (!ke_packed || !conn || !inc_ptr || !inc_elem || !nbr_ptr || !nbr_idx || !free_map || !row_ptr || !vals64 ||
      n_nodes <= 0 || max_nbrs <= 0 || max_nbrs > FEAB_MAX_NODE_NBRS || !status)
    return FEAB_BAD_ARG;
  const size_t smem = (size_t)kWarps * max_nbrs * (9 * sizeof(double) + 2 * sizeof(int32_t));
  static size_t configured = 0;
  if (smem > 48 * 1024 && smem > configured) {
    FEAB_CUDA(cudaFuncSetAttribute(k_assemble, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured = smem;
  }
  count_launches(1);
  k_assemble<<<(n_nodes + kWarps - 1) / kWarps, kWarps * 32, smem, s>>>(
      ke_packed, conn, inc_ptr, inc_elem, nbr_ptr, nbr_idx, n_nodes, max_nbrs, free_map, row_ptr, vals64, vals32,
      dinv64, dinv32, status);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}
