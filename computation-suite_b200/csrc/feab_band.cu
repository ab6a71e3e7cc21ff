// Direct solve of the reduced SPD system: banded tile Cholesky on the GPU.
//
// Replaces FESystem._sparse_lu_solve (fea_engine/src/fea_engine/solver.py:1681-1724), the SuperLU
// factorisation behind solve_static(method=None).  K_ff is SPD, so the factorisation without
// pivoting is its Cholesky factor L (U = D L^T with U_ii = L_ii^2), and the reference's
// singularity test on SuperLU's pivots (min |U_ii| < tol max |U_ii|) is made on the pivots L_ii^2.
//
// The caller renumbers the rows (a bandwidth-reducing order) so that every nonzero lies within
// `bandwidth` of the diagonal.  The lower band is kept as 64 x 64 tiles: block row I holds the
// tiles of block columns I - bands .. I, tile (I, d) being block column I - d.  The fill of a
// Cholesky factor stays inside the band, so the factorisation is a right-looking tile algorithm
// over block columns K = 0 .. n_tiles - 1:
//   1. factor the diagonal tile (K, K) in shared memory (k_band_potrf);
//   2. solve the tiles below it, L_IK = A_IK L_KK^{-T}, one CTA per tile (k_band_trsm);
//   3. update the trailing band, A_IJ -= L_IK L_JK^T for K < J <= I <= K + bands, one CTA per
//      tile (k_band_update, a 64 x 64 x 64 FP64 product with 4 x 4 outputs per thread).
// The solves walk the block rows forward (L y = b) and backward (L^T x = y), one kernel per block
// row: each CTA solves the block's 64 x 64 triangle with one warp and then applies one
// off-diagonal tile to a later (earlier) block of the right-hand side.
#include <algorithm>
#include <cmath>
#include <cstring>
#include "feab_common.cuh"

namespace feab {
namespace {

constexpr int kT = FEAB_BAND_TILE;       // tile edge
constexpr int kTile = kT * kT;           // doubles per tile
constexpr int kLd = kT + 1;              // shared-memory row stride of a staged triangle
constexpr int kGemmLd = kT + 2;          // row stride of the update's staged operands (16-byte rows)

__host__ __device__ inline size_t tile_index(int I, int d, int bands) {
  return ((size_t)I * (size_t)(bands + 1) + (size_t)d) * (size_t)kTile;
}

// ---------------------------------------------------------------- bandwidth and assembly
// One warp per CSR row: the largest |iperm[row] - iperm[col]|; an iperm entry outside [0, n)
// sets bad.
__global__ void k_band_width(const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ col_idx, int32_t n,
                             const int32_t* __restrict__ iperm, int32_t* width, int32_t* bad) {
  const int lane = threadIdx.x & 31;
  const int row = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  if (row >= n) return;
  const int i = __ldg(iperm + row);
  int w = 0;
  bool ok = i >= 0 && i < n;
  for (int e = __ldg(row_ptr + row) + lane; e < __ldg(row_ptr + row + 1); e += 32) {
    const int c = __ldg(col_idx + e);
    const int j = (c >= 0 && c < n) ? __ldg(iperm + c) : -1;
    if (j < 0 || j >= n) ok = false;
    else w = max(w, abs(i - j));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) w = max(w, __shfl_xor_sync(FEAB_FULL_MASK, w, o));
  const bool all_ok = __all_sync(FEAB_FULL_MASK, ok);
  if (lane == 0) {
    atomicMax(width, w);
    if (!all_ok) atomicExch(bad, 1);
  }
}

// One warp per CSR row: the row's lower entries (new row >= new column) into their tiles; an
// entry outside the band sets bad.
__global__ void k_band_scatter(const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ col_idx,
                               const double* __restrict__ vals, int32_t n, const int32_t* __restrict__ iperm,
                               int bands, double* __restrict__ tiles, int32_t* bad) {
  const int lane = threadIdx.x & 31;
  const int row = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  if (row >= n) return;
  const int i = __ldg(iperm + row), I = i / kT;
  for (int e = __ldg(row_ptr + row) + lane; e < __ldg(row_ptr + row + 1); e += 32) {
    const int c = __ldg(col_idx + e);
    const int j = (c >= 0 && c < n) ? __ldg(iperm + c) : -1;
    if (i < 0 || i >= n || j < 0 || j >= n) {  // not a permutation of the rows: skip, report
      atomicExch(bad, 1);
      continue;
    }
    if (j > i) continue;
    const int d = I - j / kT;
    if (d > bands) {
      atomicExch(bad, 1);
      continue;
    }
    tiles[tile_index(I, d, bands) + (size_t)(i % kT) * kT + (j % kT)] = __ldg(vals + e);
  }
}

// Rows n .. 64 n_tiles - 1 are identity rows.
__global__ void k_band_pad(int32_t n, int n_tiles, int bands, double* __restrict__ tiles) {
  const int r = n + blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_tiles * kT) return;
  tiles[tile_index(r / kT, 0, bands) + (size_t)(r % kT) * kT + (r % kT)] = 1.0;
}

// ---------------------------------------------------------------- factorisation
// The 256-byte header of the band storage.
struct BandState {
  unsigned long long piv_min, piv_max;  // bit patterns of positive doubles (order-preserving)
  int32_t status;
  int32_t bad;                          // assembly: an entry outside the band
};
static_assert(sizeof(BandState) <= FEAB_BAND_HEADER_BYTES, "band header");

// Cholesky of the diagonal tile (K, K) in shared memory; pivots of rows < n are recorded.
__global__ void __launch_bounds__(256) k_band_potrf(double* __restrict__ tiles, int bands, int K, int32_t n,
                                                   BandState* st) {
  __shared__ double A[kT][kLd];
  __shared__ double dk;
  double* T = tiles + tile_index(K, 0, bands);
  for (int q = threadIdx.x; q < kTile; q += blockDim.x) A[q / kT][q % kT] = T[q];
  __syncthreads();
  for (int k = 0; k < kT; ++k) {
    if (threadIdx.x == 0) {
      double p = A[k][k];
      if (K * kT + k < n) {
        if (p > 0.0) {
          const unsigned long long b = (unsigned long long)__double_as_longlong(p);
          atomicMin(&st->piv_min, b);
          atomicMax(&st->piv_max, b);
        } else {
          atomicCAS(&st->status, FEAB_OK, FEAB_NOT_SPD);
        }
      }
      if (!(p > 0.0)) p = 1.0;  // keep going with a harmless pivot; the status reports it
      dk = sqrt(p);
      A[k][k] = dk;
    }
    __syncthreads();
    for (int i = k + 1 + threadIdx.x; i < kT; i += blockDim.x) A[i][k] /= dk;
    __syncthreads();
    const int m = kT - 1 - k;
    for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
      const int i = k + 1 + q / m, j = k + 1 + q % m;
      if (j <= i) A[i][j] -= A[i][k] * A[j][k];
    }
    __syncthreads();
  }
  for (int q = threadIdx.x; q < kTile; q += blockDim.x) {
    const int i = q / kT, j = q % kT;
    if (j <= i) T[q] = A[i][j];
  }
}

// L_IK = A_IK L_KK^{-T} for the tiles I = K + 1 + blockIdx.x below the diagonal: each row r of
// the tile is a forward substitution x_c = (a_c - sum_{k<c} x_k L_ck) / L_cc, by 4 lanes that
// split the sum (k = q mod 4) and combine it with two shuffles.
__global__ void __launch_bounds__(256) k_band_trsm(double* __restrict__ tiles, int bands, int K) {
  extern __shared__ __align__(16) double tsm[];  // two staged tiles (dynamic: 66.5 KB)
  double (*L)[kLd] = reinterpret_cast<double (*)[kLd]>(tsm);
  double (*X)[kLd] = reinterpret_cast<double (*)[kLd]>(tsm + kT * kLd);
  const int I = K + 1 + blockIdx.x;
  const double* Ld = tiles + tile_index(K, 0, bands);
  double* T = tiles + tile_index(I, I - K, bands);
  for (int q = threadIdx.x; q < kTile; q += blockDim.x) {
    L[q / kT][q % kT] = Ld[q];
    X[q / kT][q % kT] = T[q];
  }
  __syncthreads();
  const int r = threadIdx.x >> 2, part = threadIdx.x & 3;
  for (int c = 0; c < kT; ++c) {
    double s = 0.0;
    for (int k = part; k < c; k += 4) s += X[r][k] * L[c][k];
    s += __shfl_xor_sync(FEAB_FULL_MASK, s, 1);
    s += __shfl_xor_sync(FEAB_FULL_MASK, s, 2);
    const double x = (X[r][c] - s) / L[c][c];
    __syncwarp();
    if (part == 0) X[r][c] = x;
    __syncwarp();
  }
  __syncthreads();
  for (int q = threadIdx.x; q < kTile; q += blockDim.x) T[q] = X[q / kT][q % kT];
}

// Trailing update of block column K: CTA a takes the pair (I, J) with K < J <= I, a = (I - K - 1)
// (I - K) / 2 + (J - K - 1): A_IJ -= L_IK L_JK^T.  Each thread owns a 4 x 4 block of the tile;
// the two factors are staged transposed (column k contiguous) so a thread reads its 4 rows and 4
// columns of step k as two 16-byte loads each.
__global__ void __launch_bounds__(256) k_band_update(double* __restrict__ tiles, int bands, int K) {
  extern __shared__ __align__(16) double gsm[];
  double* As = gsm;                  // As[k * kGemmLd + r] = L_IK[r][k]
  double* Bs = gsm + kT * kGemmLd;   // Bs[k * kGemmLd + c] = L_JK[c][k]
  const int a = blockIdx.x;
  int io = (int)((sqrt(8.0 * a + 1.0) - 1.0) * 0.5);
  while ((io + 1) * (io + 2) / 2 <= a) ++io;
  while (io * (io + 1) / 2 > a) --io;
  const int jo = a - io * (io + 1) / 2;
  const int I = K + 1 + io, J = K + 1 + jo;
  const double* Ap = tiles + tile_index(I, I - K, bands);
  const double* Bp = tiles + tile_index(J, J - K, bands);
  double* Cp = tiles + tile_index(I, I - J, bands);
  for (int q = threadIdx.x; q < kTile; q += blockDim.x) {
    const int row = q / kT, k = q % kT;
    As[k * kGemmLd + row] = Ap[q];
    Bs[k * kGemmLd + row] = Bp[q];
  }
  __syncthreads();
  const int tr = threadIdx.x >> 4, tc = threadIdx.x & 15;
  double acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
#pragma unroll 4
  for (int k = 0; k < kT; ++k) {
    const double2 a01 = *reinterpret_cast<const double2*>(As + k * kGemmLd + 4 * tr);
    const double2 a23 = *reinterpret_cast<const double2*>(As + k * kGemmLd + 4 * tr + 2);
    const double2 b01 = *reinterpret_cast<const double2*>(Bs + k * kGemmLd + 4 * tc);
    const double2 b23 = *reinterpret_cast<const double2*>(Bs + k * kGemmLd + 4 * tc + 2);
    const double av[4] = {a01.x, a01.y, a23.x, a23.y};
    const double bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = fma(av[u], bv[v], acc[u][v]);
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    double2* c = reinterpret_cast<double2*>(Cp + (size_t)(4 * tr + u) * kT + 4 * tc);
    double2 c01 = c[0], c23 = c[1];
    c01.x -= acc[u][0];
    c01.y -= acc[u][1];
    c23.x -= acc[u][2];
    c23.y -= acc[u][3];
    c[0] = c01;
    c[1] = c23;
  }
}
constexpr size_t kUpdateSmem = 2 * kT * kGemmLd * sizeof(double);
constexpr size_t kTrsmSmem = 2 * kT * kLd * sizeof(double);

// ---------------------------------------------------------------- solves
// Forward step K of L y = b: every CTA solves L_KK y_K = w_K with warp 0 (lane l owns rows l and
// l + 32; column c's value is broadcast by shuffle), CTA 0 writes y_K, and CTA i < n_below applies
// tile (K + 1 + i, i + 1): w_{K+1+i} -= L_{K+1+i,K} y_K (two threads per row).
__global__ void __launch_bounds__(128) k_band_fwd(const double* __restrict__ tiles, int bands, int K, int n_below,
                                                 double* __restrict__ w, double* __restrict__ y) {
  __shared__ double L[kT][kLd];
  __shared__ double ys[kT];
  const double* Ld = tiles + tile_index(K, 0, bands);
  for (int q = threadIdx.x; q < kTile; q += blockDim.x) L[q / kT][q % kT] = Ld[q];
  __syncthreads();
  if (threadIdx.x < 32) {
    const int l = threadIdx.x;
    double v0 = w[K * kT + l], v1 = w[K * kT + l + 32];
    for (int c = 0; c < kT; ++c) {
      const int owner = c & 31;
      double t = 0.0;
      if (l == owner) t = (c < 32 ? v0 : v1) / L[c][c];
      const double yc = __shfl_sync(FEAB_FULL_MASK, t, owner);
      if (l == owner) {
        if (c < 32) v0 = yc;
        else v1 = yc;
      }
      if (l > c) v0 -= L[l][c] * yc;
      if (l + 32 > c) v1 -= L[l + 32][c] * yc;
    }
    ys[l] = v0;
    ys[l + 32] = v1;
  }
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x < kT) y[K * kT + threadIdx.x] = ys[threadIdx.x];
  if ((int)blockIdx.x < n_below) {
    const int I = K + 1 + blockIdx.x;
    const double* T = tiles + tile_index(I, I - K, bands);
    const int r = threadIdx.x >> 1, h = threadIdx.x & 1;
    double s = 0.0;
#pragma unroll 8
    for (int c = 32 * h; c < 32 * h + 32; ++c) s += T[(size_t)r * kT + c] * ys[c];
    s += __shfl_xor_sync(FEAB_FULL_MASK, s, 1);
    if (h == 0) w[I * kT + r] -= s;
  }
}

// Backward step K of L^T x = y: every CTA solves L_KK^T x_K = w_K (rows descending), CTA 0 writes
// x_K, and CTA i < n_above applies tile (K, i + 1) transposed: w_{K-1-i} -= L_{K,K-1-i}^T x_K (two
// threads per column, each summing half of the rows).
__global__ void __launch_bounds__(128) k_band_bwd(const double* __restrict__ tiles, int bands, int K, int n_above,
                                                 double* __restrict__ w, double* __restrict__ x) {
  __shared__ double L[kT][kLd];
  __shared__ double xs[kT];
  const double* Ld = tiles + tile_index(K, 0, bands);
  for (int q = threadIdx.x; q < kTile; q += blockDim.x) L[q / kT][q % kT] = Ld[q];
  __syncthreads();
  if (threadIdx.x < 32) {
    const int l = threadIdx.x;
    double v0 = w[K * kT + l], v1 = w[K * kT + l + 32];
    for (int r = kT - 1; r >= 0; --r) {
      const int owner = r & 31;
      double t = 0.0;
      if (l == owner) t = (r < 32 ? v0 : v1) / L[r][r];
      const double xr = __shfl_sync(FEAB_FULL_MASK, t, owner);
      if (l == owner) {
        if (r < 32) v0 = xr;
        else v1 = xr;
      }
      if (l < r) v0 -= L[r][l] * xr;
      if (l + 32 < r) v1 -= L[r][l + 32] * xr;
    }
    xs[l] = v0;
    xs[l + 32] = v1;
  }
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x < kT) x[K * kT + threadIdx.x] = xs[threadIdx.x];
  if ((int)blockIdx.x < n_above) {
    const int J = K - 1 - blockIdx.x;
    const double* T = tiles + tile_index(K, K - J, bands);
    const int c = threadIdx.x >> 1, h = threadIdx.x & 1;
    double s = 0.0;
#pragma unroll 8
    for (int r = 32 * h; r < 32 * h + 32; ++r) s += T[(size_t)r * kT + c] * xs[r];
    s += __shfl_xor_sync(FEAB_FULL_MASK, s, 1);
    if (h == 0) w[J * kT + c] -= s;
  }
}

}  // namespace
}  // namespace feab


using namespace feab;

namespace {
BandState* band_state(const feab_band* B) { return reinterpret_cast<BandState*>(B->storage); }
double* band_tiles(const feab_band* B) {
  return reinterpret_cast<double*>(static_cast<char*>(B->storage) + FEAB_BAND_HEADER_BYTES);
}
bool band_ok(const feab_band* B) {
  return B && B->storage && B->n > 0 && B->bands >= 0 && B->n_tiles == (B->n + kT - 1) / kT &&
         (reinterpret_cast<uintptr_t>(B->storage) & 255) == 0;
}
}  // namespace

extern "C" size_t feab_band_bytes(int32_t n, int32_t bandwidth) {
  if (n <= 0 || bandwidth < 0) return 0;
  const size_t nt = (size_t)(n + kT - 1) / kT, bands = (size_t)(bandwidth + kT - 1) / kT;
  return FEAB_BAND_HEADER_BYTES + nt * (bands + 1) * (size_t)kTile * sizeof(double);
}

extern "C" int32_t feab_band_width(const feab_csr* A, const int32_t* iperm, int32_t* scratch, int32_t* bandwidth_out,
                                   cudaStream_t s) {
  if (!A || !iperm || !scratch || !bandwidth_out || A->n <= 0 || !A->row_ptr || !A->col_idx) return FEAB_BAD_ARG;
  FEAB_CUDA(cudaMemsetAsync(scratch, 0, 2 * sizeof(int32_t), s));
  const int threads = 256, rows = threads / 32;
  k_band_width<<<(A->n + rows - 1) / rows, threads, 0, s>>>(A->row_ptr, A->col_idx, A->n, iperm, scratch, scratch + 1);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  int32_t h[2] = {0, 0};
  FEAB_CUDA(cudaMemcpyAsync(h, scratch, sizeof(h), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaStreamSynchronize(s));
  if (h[1]) return FEAB_BAD_ARG;
  *bandwidth_out = h[0];
  return FEAB_OK;
}

extern "C" int32_t feab_band_assemble(const feab_csr* A, const int32_t* iperm, int32_t bandwidth, feab_band* B,
                                      cudaStream_t s) {
  if (!A || !iperm || !B || A->n <= 0 || !A->row_ptr || !A->col_idx || !A->vals64 || bandwidth < 0) return FEAB_BAD_ARG;
  B->n = A->n;
  B->n_tiles = (A->n + kT - 1) / kT;
  B->bands = (bandwidth + kT - 1) / kT;
  if (!band_ok(B)) return FEAB_BAD_ARG;
  FEAB_CUDA(cudaMemsetAsync(B->storage, 0, feab_band_bytes(A->n, bandwidth), s));
  BandState* st = band_state(B);
  const int threads = 256, rows = threads / 32;
  k_band_scatter<<<(A->n + rows - 1) / rows, threads, 0, s>>>(A->row_ptr, A->col_idx, A->vals64, A->n, iperm, B->bands,
                                                             band_tiles(B), &st->bad);
  const int pad = B->n_tiles * kT - A->n;
  if (pad > 0) k_band_pad<<<1, kT, 0, s>>>(A->n, B->n_tiles, B->bands, band_tiles(B));
  count_launches(pad > 0 ? 2 : 1);
  FEAB_CHECK_LAUNCH();
  int32_t bad = 0;
  FEAB_CUDA(cudaMemcpyAsync(&bad, &st->bad, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaStreamSynchronize(s));
  return bad ? FEAB_BAD_ARG : FEAB_OK;
}

extern "C" int32_t feab_band_cholesky(feab_band* B, double* pivots_out, cudaStream_t s) {
  if (!band_ok(B)) return FEAB_BAD_ARG;
  BandState init{};
  init.piv_min = 0x7ff0000000000000ull;  // +inf
  init.piv_max = 0ull;
  BandState* st = band_state(B);
  FEAB_CUDA(cudaMemcpyAsync(st, &init, sizeof(BandState), cudaMemcpyHostToDevice, s));
  FEAB_CUDA(cudaFuncSetAttribute(k_band_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUpdateSmem));
  FEAB_CUDA(cudaFuncSetAttribute(k_band_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem));
  double* tiles = band_tiles(B);
  const int NT = B->n_tiles, bands = B->bands;
  uint64_t launches = 0;
  for (int K = 0; K < NT; ++K) {
    k_band_potrf<<<1, 256, 0, s>>>(tiles, bands, K, B->n, st);
    const int below = std::min(bands, NT - 1 - K);
    if (below > 0) {
      k_band_trsm<<<below, 256, kTrsmSmem, s>>>(tiles, bands, K);
      k_band_update<<<below * (below + 1) / 2, 256, kUpdateSmem, s>>>(tiles, bands, K);
      launches += 2;
    }
    launches += 1;
  }
  count_launches(launches);
  FEAB_CHECK_LAUNCH();
  BandState h{};
  FEAB_CUDA(cudaMemcpyAsync(&h, st, sizeof(BandState), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaStreamSynchronize(s));
  if (pivots_out) {
    double lo, hi;
    std::memcpy(&lo, &h.piv_min, sizeof(double));
    std::memcpy(&hi, &h.piv_max, sizeof(double));
    pivots_out[0] = lo;
    pivots_out[1] = hi;
  }
  return h.status == FEAB_OK ? FEAB_OK : h.status;
}

extern "C" int32_t feab_band_solve(const feab_band* B, const double* b, double* x, double* work, cudaStream_t s) {
  if (!band_ok(B) || !b || !x || !work || x == b || x == work || b == work) return FEAB_BAD_ARG;
  const double* tiles = band_tiles(B);
  const int NT = B->n_tiles, bands = B->bands;
  const size_t bytes = (size_t)NT * kT * sizeof(double);
  // forward: work = b, updated in place; y into x
  FEAB_CUDA(cudaMemcpyAsync(work, b, bytes, cudaMemcpyDeviceToDevice, s));
  for (int K = 0; K < NT; ++K) {
    const int below = std::min(bands, NT - 1 - K);
    k_band_fwd<<<std::max(1, below), 128, 0, s>>>(tiles, bands, K, below, work, x);
  }
  // backward: x (= y) updated in place; the solution into work, then copied to x
  for (int K = NT - 1; K >= 0; --K) {
    const int above = std::min(bands, K);
    k_band_bwd<<<std::max(1, above), 128, 0, s>>>(tiles, bands, K, above, x, work);
  }
  count_launches(2 * (uint64_t)NT);
  FEAB_CHECK_LAUNCH();
  FEAB_CUDA(cudaMemcpyAsync(x, work, bytes, cudaMemcpyDeviceToDevice, s));
  // rows past n are identity rows with b = 0, so x is 0 there
  return FEAB_OK;
}
