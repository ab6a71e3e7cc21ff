// Dense products of tall row-major panels with small matrices, in FP64 on the CUDA cores, for
// the Rayleigh-Ritz steps of the modal subspace iteration and for forming POD modes:
//   feab_panel_gram:   C = X^T Y  (X, Y: n x k panels, k <= 64; C: k x k)
//   feab_panel_small:  Z = Y V    (Y: n x k panel, V: k x m, m <= 64; Z: n x m panel)
// The reference forms these with dense NumPy/LAPACK products (solver.py:2047-2114 through
// scipy's eigsh, rom_engine/src/rom_engine/pod.py:140-160).  Both stream the panels once; the
// Gram reduces per-CTA partials in a fixed order, so its result is deterministic.
#include <algorithm>
#include "feab_common.cuh"

namespace feab {
namespace {

constexpr int kP = 64;         // largest panel width
constexpr int kPTile = 32;     // rows per staged tile
constexpr int kPThreads = 256;
constexpr int kPReduceWarps = 8;

// Stage rows [r0, r0 + kPTile) of an n x k panel (leading dimension ld) into a kPTile x 64
// shared tile, zero beyond n and beyond column k.
__device__ __forceinline__ void stage_tile(const double* __restrict__ A, int64_t n, int k, int ld, int64_t r0,
                                           double* __restrict__ t) {
  for (int e = threadIdx.x; e < kPTile * kP; e += kPThreads) {
    const int r = e >> 6, c = e & 63;
    t[e] = (r0 + r < n && c < k) ? __ldcs(A + (r0 + r) * (int64_t)ld + c) : 0.0;
  }
}

// One CTA per SM: thread (rg, bi, bj) owns C[bi + 8u][bj + 8v] (u, v < 8) over the rows
// r = rg (mod 4) of each tile; the 4 row groups are summed in a fixed order, CTAs by
// k_panel_gram_reduce.
__global__ void __launch_bounds__(kPThreads, 1) k_panel_gram(const double* __restrict__ X, int ldx,
                                                            const double* __restrict__ Y, int ldy, int64_t n, int k,
                                                            double* __restrict__ part) {
  __shared__ double xs[kPTile * kP];
  __shared__ double ys[kPTile * kP];
  const int tid = threadIdx.x, rg = tid >> 6, t = tid & 63, bi = t >> 3, bj = t & 7;
  double acc[8][8];
#pragma unroll
  for (int u = 0; u < 8; ++u)
#pragma unroll
    for (int v = 0; v < 8; ++v) acc[u][v] = 0.0;
  const int64_t tiles = (n + kPTile - 1) / kPTile;
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    __syncthreads();
    stage_tile(X, n, k, ldx, tile * kPTile, xs);
    stage_tile(Y, n, k, ldy, tile * kPTile, ys);
    __syncthreads();
    for (int r = rg; r < kPTile; r += 4) {
      double a[8], b[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        a[u] = xs[r * kP + bi + 8 * u];
        b[u] = ys[r * kP + bj + 8 * u];
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
  }
  // the 64 x 64 partial of this CTA, row groups summed in order; rows 0..31 go to xs and
  // rows 32..63 to ys (together 64 x 64 doubles)
  double* red = xs;
  for (int g = 0; g < 4; ++g) {
    __syncthreads();
    if (rg == g) {
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) {
          const int row = bi + 8 * u, col = bj + 8 * v;
          double* cell = (row < kPTile ? red + row * kP : ys + (row - kPTile) * kP) + col;
          *cell = g == 0 ? acc[u][v] : *cell + acc[u][v];
        }
    }
  }
  __syncthreads();
  for (int e = tid; e < kP * kP; e += kPThreads) {
    const int row = e >> 6, col = e & 63;
    part[(int64_t)blockIdx.x * kP * kP + e] = row < kPTile ? xs[row * kP + col] : ys[(row - kPTile) * kP + col];
  }
}

// C[i][j] = sum over CTAs of part[cta][i][j] (i, j < k), one warp per entry, fixed order.
__global__ void __launch_bounds__(32 * kPReduceWarps) k_panel_gram_reduce(const double* __restrict__ part, int ctas,
                                                                         int k, double* __restrict__ C) {
  const int idx = blockIdx.x * kPReduceWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (idx >= k * k) return;
  const int i = idx / k, j = idx % k;
  double s = 0.0;
  for (int c = lane; c < ctas; c += 32) s += __ldg(part + (int64_t)c * kP * kP + i * kP + j);
  s = warp_sum(s);
  if (lane == 0) C[idx] = s;
}

// Z = Y V: V (k x m) staged in shared memory; thread (row, col) of the n x m output.
__global__ void __launch_bounds__(kPThreads) k_panel_small(const double* __restrict__ Y, int ldy, int64_t n, int k,
                                                          const double* __restrict__ V, int m,
                                                          double* __restrict__ Z, int ldz) {
  __shared__ double vs[kP * kP];
  for (int e = threadIdx.x; e < k * m; e += kPThreads) vs[e] = V[e];
  __syncthreads();
  const int64_t total = n * (int64_t)m;
  for (int64_t e = (int64_t)blockIdx.x * kPThreads + threadIdx.x; e < total; e += (int64_t)gridDim.x * kPThreads) {
    const int64_t i = e / m;
    const int c = (int)(e - i * m);
    const double* y = Y + i * (int64_t)ldy;
    double s = 0.0;
    for (int j = 0; j < k; ++j) s = fma(__ldg(y + j), vs[j * m + c], s);
    Z[i * (int64_t)ldz + c] = s;
  }
}

int panel_grid(int64_t n) {
  const int64_t tiles = (n + kPTile - 1) / kPTile;
  return (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)sm_count()));
}

}  // namespace
}  // namespace feab

using namespace feab;

extern "C" size_t feab_panel_gram_workspace_bytes(int64_t n) {
  if (n <= 0) return 0;
  return sizeof(double) * (size_t)panel_grid(n) * kP * kP;
}

extern "C" int32_t feab_panel_gram(const double* X, int32_t ldx, const double* Y, int32_t ldy, int64_t n, int32_t k,
                                   double* C, void* workspace, size_t workspace_bytes, cudaStream_t s) {
  if (!X || !Y || !C || !workspace || n <= 0 || k < 1 || k > kP || ldx < k || ldy < k) return FEAB_BAD_ARG;
  if (feab_panel_gram_workspace_bytes(n) > workspace_bytes) return FEAB_BAD_ARG;
  const int grid = panel_grid(n);
  double* part = static_cast<double*>(workspace);
  k_panel_gram<<<grid, kPThreads, 0, s>>>(X, ldx, Y, ldy, n, k, part);
  k_panel_gram_reduce<<<(k * k + kPReduceWarps - 1) / kPReduceWarps, 32 * kPReduceWarps, 0, s>>>(part, grid, k, C);
  count_launches(2);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}

extern "C" int32_t feab_panel_small(const double* Y, int32_t ldy, int64_t n, int32_t k, const double* V, int32_t m,
                                    double* Z, int32_t ldz, cudaStream_t s) {
  if (!Y || !V || !Z || n <= 0 || k < 1 || k > kP || m < 1 || m > kP || ldy < k || ldz < m) return FEAB_BAD_ARG;
  if (Z == Y) return FEAB_BAD_ARG;  // every output row reads its whole input row
  const int64_t blocks = (n * (int64_t)m + kPThreads - 1) / kPThreads;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)sm_count() * 8));
  k_panel_small<<<grid, kPThreads, 0, s>>>(Y, ldy, n, k, V, m, Z, ldz);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}
