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
//      and invert its factor, Linv_KK = L_KK^{-1} (kept beside the band);
//   2. form the tiles below it, L_IK = A_IK Linv_KK^T, one CTA per tile;
//   3. update the trailing band, A_IJ -= L_IK L_JK^T for K < J <= I <= K + bands, one CTA per
//      tile (k_band_tile_gemm: 64 x 64 x 64 FP64 products on the FP64 tensor path, mma.sync).
// Applying the inverted 64 x 64 diagonal factors (as blocked GPU triangular solvers do) turns the
// per-column triangular solves into tile products, so only step 1 is sequential within a column.
// The solves walk the block rows forward (L y = b) and backward (L^T x = y), one kernel per block
// row: each CTA forms the block's y_K = Linv_KK w_K (or x_K = Linv_KK^T w_K) and then applies one
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

// Cholesky of the diagonal tile (K, K), then the inverse of its factor.  The tile lives in
// registers, a 4 x 4 block per thread (16 x 16 threads).  The right-looking elimination keeps the
// columns unscaled (A_ij -= A_ik A_jk / p_k for j > k): the owners of column k + 1 copy it into a
// shared double buffer after their step-k update, and the owner of its diagonal entry stores
// 1 / p_{k+1}, so one barrier separates the steps.  The columns are scaled by 1 / sqrt(p_k) at the
// end.  Pivots of rows < n are recorded (a pivot <= 0 sets FEAB_NOT_SPD and is replaced by 1 so the
// kernel finishes).  Linv = L_KK^{-1} (lower triangular) is then formed the same way: X = I in
// registers, and for each row m, X_m = X_m / L_mm is published and X_i -= L_im X_m for i > m.
__global__ void __launch_bounds__(256) k_band_potrf(double* __restrict__ tiles, double* __restrict__ inv, int bands,
                                                   int K, int32_t n, BandState* st) {
  __shared__ double colbuf[2][kT];
  __shared__ double rpbuf[2];
  __shared__ double piv[kT];
  __shared__ double rowbuf[2][kT];
  extern __shared__ __align__(16) double psm[];  // the factor L (dynamic: 33 KB)
  double (*Ls)[kLd] = reinterpret_cast<double (*)[kLd]>(psm);
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  double* T = tiles + tile_index(K, 0, bands);
  double a[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const double2 p0 = *reinterpret_cast<const double2*>(T + (4 * ty + u) * kT + 4 * tx);
    const double2 p1 = *reinterpret_cast<const double2*>(T + (4 * ty + u) * kT + 4 * tx + 2);
    a[u][0] = p0.x;
    a[u][1] = p0.y;
    a[u][2] = p1.x;
    a[u][3] = p1.y;
  }
  // a[u][v] for run-time u, v, selected without indexing the register array
  auto row = [&](int u, int v) {
    return v == 0 ? a[u][0] : v == 1 ? a[u][1] : v == 2 ? a[u][2] : a[u][3];
  };
  auto sel = [&](int u, int v) {
    return u == 0 ? row(0, v) : u == 1 ? row(1, v) : u == 2 ? row(2, v) : row(3, v);
  };
  if (tx == 0) {
#pragma unroll
    for (int u = 0; u < 4; ++u) colbuf[0][4 * ty + u] = a[u][0];
    if (ty == 0) {
      const double p = a[0][0] > 0.0 ? a[0][0] : 1.0;
      rpbuf[0] = 1.0 / p;
    }
  }
  double pmin = INFINITY, pmax = 0.0;
  bool bad = false;
  for (int k = 0; k < kT; ++k) {
    __syncthreads();
    const double* col = colbuf[k & 1];
    const double rp = rpbuf[k & 1];
    if (tid == 0) {
      const double p0 = col[k];
      if (K * kT + k < n) {
        if (p0 > 0.0) {
          pmin = fmin(pmin, p0);
          pmax = fmax(pmax, p0);
        } else {
          bad = true;
        }
      }
      piv[k] = p0 > 0.0 ? p0 : 1.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = 4 * ty + u;
      const double ci = col[i] * rp;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int jj = 4 * tx + v;
        if (jj > k && i >= jj) a[u][v] -= ci * col[jj];
      }
    }
    const int k1 = k + 1;
    if (k1 < kT && tx == (k1 >> 2)) {
#pragma unroll
      for (int u = 0; u < 4; ++u) colbuf[k1 & 1][4 * ty + u] = sel(u, k1 & 3);
      if (ty == (k1 >> 2)) {
        const double p = sel(k1 & 3, k1 & 3);
        rpbuf[k1 & 1] = 1.0 / (p > 0.0 ? p : 1.0);
      }
    }
  }
  if (tid == 0) {
    if (pmax > 0.0) {
      atomicMin(&st->piv_min, (unsigned long long)__double_as_longlong(pmin));
      atomicMax(&st->piv_max, (unsigned long long)__double_as_longlong(pmax));
    }
    if (bad) atomicCAS(&st->status, FEAB_OK, FEAB_NOT_SPD);
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int i = 4 * ty + u;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int jj = 4 * tx + v;
      const double l = i > jj ? a[u][v] * rsqrt(piv[jj]) : (i == jj ? sqrt(piv[jj]) : 0.0);
      Ls[i][jj] = l;
      a[u][v] = l;
    }
    // the whole tile is written, with zeros above the diagonal
    *reinterpret_cast<double2*>(T + i * kT + 4 * tx) = make_double2(a[u][0], a[u][1]);
    *reinterpret_cast<double2*>(T + i * kT + 4 * tx + 2) = make_double2(a[u][2], a[u][3]);
  }
  // Linv: X = I; row m final after dividing by L_mm; rows below take X_i -= L_im X_m
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) a[u][v] = (4 * ty + u == 4 * tx + v) ? 1.0 : 0.0;
  __syncthreads();
  if (ty == 0) {
    const double rl = 1.0 / Ls[0][0];
#pragma unroll
    for (int v = 0; v < 4; ++v) rowbuf[0][4 * tx + v] = a[0][v] * rl;
  }
  for (int m = 0; m < kT; ++m) {
    __syncthreads();
    const double* xm = rowbuf[m & 1];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = 4 * ty + u;
      if (i == m) {
#pragma unroll
        for (int v = 0; v < 4; ++v) a[u][v] = xm[4 * tx + v];
      } else if (i > m) {
        const double lim = Ls[i][m];
#pragma unroll
        for (int v = 0; v < 4; ++v) a[u][v] -= lim * xm[4 * tx + v];
      }
    }
    const int m1 = m + 1;
    if (m1 < kT && ty == (m1 >> 2)) {
      const double rl = 1.0 / Ls[m1][m1];
      const int u = m1 & 3;
#pragma unroll
      for (int v = 0; v < 4; ++v) rowbuf[m1 & 1][4 * tx + v] = sel(u, v) * rl;
    }
  }
  double* Iv = inv + (size_t)K * kTile;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int i = 4 * ty + u;
    *reinterpret_cast<double2*>(Iv + i * kT + 4 * tx) = make_double2(a[u][0], a[u][1]);
    *reinterpret_cast<double2*>(Iv + i * kT + 4 * tx + 2) = make_double2(a[u][2], a[u][3]);
  }
}

// C (op)= A B^T for 64 x 64 tiles on the FP64 tensor path (mma.sync m8n8k4), one CTA per output
// tile: warp w owns rows 8 w .. 8 w + 7 and all 64 columns (eight 8 x 8 accumulators), and walks k
// in steps of 4.  Fragments (m8n8k4, .f64): A row-major 8 x 4, lane l holds (l / 4, l % 4); B
// column-major 4 x 8, lane l holds (l % 4, l / 4); C 8 x 8, lane l holds (l / 4, 2 (l % 4) + i).
// Both factors are staged row-major in shared memory with a padded row (kMmaLd doubles), so each
// fragment load of a half-warp touches 16 distinct banks.
//   UPDATE: the trailing update of block column K, CTA a -> (I, J) with K < J <= I, a = (I - K - 1)
//           (I - K) / 2 + (J - K - 1): A_IJ -= L_IK L_JK^T;
//   PANEL:  the panel below the diagonal tile, CTA b -> I = K + 1 + b: L_IK = A_IK Linv_KK^T.
constexpr int kMmaLd = kT + 4;

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

template <bool PANEL>
__global__ void __launch_bounds__(256) k_band_tile_gemm(double* __restrict__ tiles, const double* __restrict__ inv,
                                                       int bands, int K) {
  extern __shared__ __align__(16) double gsm[];
  double* As = gsm;                  // As[r * kMmaLd + k] = A[r][k]
  double* Bs = gsm + kT * kMmaLd;    // Bs[c * kMmaLd + k] = B[c][k]
  const double* Ap;
  const double* Bp;
  double* Cp;
  if (PANEL) {
    const int I = K + 1 + blockIdx.x;
    Ap = tiles + tile_index(I, I - K, bands);
    Bp = inv + (size_t)K * kTile;
    Cp = tiles + tile_index(I, I - K, bands);
  } else {
    const int a = blockIdx.x;
    int io = (int)((sqrt(8.0 * a + 1.0) - 1.0) * 0.5);
    while ((io + 1) * (io + 2) / 2 <= a) ++io;
    while (io * (io + 1) / 2 > a) --io;
    const int jo = a - io * (io + 1) / 2;
    const int I = K + 1 + io, J = K + 1 + jo;
    Ap = tiles + tile_index(I, I - K, bands);
    Bp = tiles + tile_index(J, J - K, bands);
    Cp = tiles + tile_index(I, I - J, bands);
  }
  for (int q = threadIdx.x; q < kTile / 2; q += blockDim.x) {
    const int row = q / (kT / 2), k2 = q % (kT / 2);
    *reinterpret_cast<double2*>(As + row * kMmaLd + 2 * k2) = reinterpret_cast<const double2*>(Ap)[q];
    *reinterpret_cast<double2*>(Bs + row * kMmaLd + 2 * k2) = reinterpret_cast<const double2*>(Bp)[q];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  double acc[8][2];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = 0.0;
  const double* Arow = As + (8 * warp + g) * kMmaLd + t;
  const double* Bcol = Bs + g * kMmaLd + t;
#pragma unroll 4
  for (int k0 = 0; k0 < kT; k0 += 4) {
    const double a = Arow[k0];
    double b[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) b[j] = Bcol[8 * j * kMmaLd + k0];
#pragma unroll
    for (int j = 0; j < 8; ++j) dmma884(acc[j], a, b[j]);
  }
  const int r = 8 * warp + g;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    double2* c = reinterpret_cast<double2*>(Cp + (size_t)r * kT + 8 * j + 2 * t);
    if (PANEL) {
      *c = make_double2(acc[j][0], acc[j][1]);
    } else {
      double2 cv = *c;
      cv.x -= acc[j][0];
      cv.y -= acc[j][1];
      *c = cv;
    }
  }
}
constexpr size_t kGemmSmem = 2 * kT * kMmaLd * sizeof(double);
constexpr size_t kPotrfSmem = kT * kLd * sizeof(double);

// ---------------------------------------------------------------- solves
// Forward step K of L y = b: every CTA forms y_K = Linv_KK w_K (two threads per row), CTA 0 writes
// it, and CTA i < n_below applies tile (K + 1 + i, i + 1): w_{K+1+i} -= L_{K+1+i,K} y_K.
__global__ void __launch_bounds__(128) k_band_fwd(const double* __restrict__ tiles, const double* __restrict__ inv,
                                                 int bands, int K, int n_below, double* __restrict__ w,
                                                 double* __restrict__ y) {
  __shared__ double wk[kT];
  __shared__ double ys[kT];
  if (threadIdx.x < kT) wk[threadIdx.x] = w[K * kT + threadIdx.x];
  __syncthreads();
  const int r = threadIdx.x >> 1, h = threadIdx.x & 1;
  const double* Iv = inv + (size_t)K * kTile;
  double s = 0.0;
#pragma unroll 8
  for (int c = 32 * h; c < 32 * h + 32; ++c) s += Iv[r * kT + c] * wk[c];
  s += __shfl_xor_sync(FEAB_FULL_MASK, s, 1);
  if (h == 0) ys[r] = s;
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x < kT) y[K * kT + threadIdx.x] = ys[threadIdx.x];
  if ((int)blockIdx.x < n_below) {
    const int I = K + 1 + blockIdx.x;
    const double* T = tiles + tile_index(I, I - K, bands);
    double t = 0.0;
#pragma unroll 8
    for (int c = 32 * h; c < 32 * h + 32; ++c) t += T[(size_t)r * kT + c] * ys[c];
    t += __shfl_xor_sync(FEAB_FULL_MASK, t, 1);
    if (h == 0) w[I * kT + r] -= t;
  }
}

// Backward step K of L^T x = y: every CTA forms x_K = Linv_KK^T w_K (two threads per column), CTA
// 0 writes it, and CTA i < n_above applies tile (K, i + 1) transposed: w_{K-1-i} -= L_{K,K-1-i}^T
// x_K.
__global__ void __launch_bounds__(128) k_band_bwd(const double* __restrict__ tiles, const double* __restrict__ inv,
                                                 int bands, int K, int n_above, double* __restrict__ w,
                                                 double* __restrict__ x) {
  __shared__ double wk[kT];
  __shared__ double xs[kT];
  if (threadIdx.x < kT) wk[threadIdx.x] = w[K * kT + threadIdx.x];
  __syncthreads();
  const int c = threadIdx.x >> 1, h = threadIdx.x & 1;
  const double* Iv = inv + (size_t)K * kTile;
  double s = 0.0;
#pragma unroll 8
  for (int r = 32 * h; r < 32 * h + 32; ++r) s += Iv[r * kT + c] * wk[r];
  s += __shfl_xor_sync(FEAB_FULL_MASK, s, 1);
  if (h == 0) xs[c] = s;
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x < kT) x[K * kT + threadIdx.x] = xs[threadIdx.x];
  if ((int)blockIdx.x < n_above) {
    const int J = K - 1 - blockIdx.x;
    const double* T = tiles + tile_index(K, K - J, bands);
    double t = 0.0;
#pragma unroll 8
    for (int r = 32 * h; r < 32 * h + 32; ++r) t += T[(size_t)r * kT + c] * xs[r];
    t += __shfl_xor_sync(FEAB_FULL_MASK, t, 1);
    if (h == 0) w[J * kT + c] -= t;
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
// The inverses of the diagonal factor tiles, one per block row, after the band.
double* band_inv(const feab_band* B) {
  return band_tiles(B) + (size_t)B->n_tiles * (size_t)(B->bands + 1) * kTile;
}
bool band_ok(const feab_band* B) {
  return B && B->storage && B->n > 0 && B->bands >= 0 && B->n_tiles == (B->n + kT - 1) / kT &&
         (reinterpret_cast<uintptr_t>(B->storage) & 255) == 0;
}
}  // namespace

extern "C" size_t feab_band_bytes(int32_t n, int32_t bandwidth) {
  if (n <= 0 || bandwidth < 0) return 0;
  const size_t nt = (size_t)(n + kT - 1) / kT, bands = (size_t)(bandwidth + kT - 1) / kT;
  return FEAB_BAND_HEADER_BYTES + nt * (bands + 2) * (size_t)kTile * sizeof(double);
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
  FEAB_CUDA(cudaFuncSetAttribute(k_band_potrf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPotrfSmem));
  FEAB_CUDA(cudaFuncSetAttribute(k_band_tile_gemm<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kGemmSmem));
  FEAB_CUDA(cudaFuncSetAttribute(k_band_tile_gemm<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kGemmSmem));
  double* tiles = band_tiles(B);
  double* inv = band_inv(B);
  const int NT = B->n_tiles, bands = B->bands;
  uint64_t launches = 0;
  for (int K = 0; K < NT; ++K) {
    k_band_potrf<<<1, 256, kPotrfSmem, s>>>(tiles, inv, bands, K, B->n, st);
    const int below = std::min(bands, NT - 1 - K);
    if (below > 0) {
      k_band_tile_gemm<true><<<below, 256, kGemmSmem, s>>>(tiles, inv, bands, K);
      k_band_tile_gemm<false><<<below * (below + 1) / 2, 256, kGemmSmem, s>>>(tiles, inv, bands, K);
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
  const double* inv = band_inv(B);
  const int NT = B->n_tiles, bands = B->bands;
  const size_t bytes = (size_t)NT * kT * sizeof(double);
  // forward: work = b, updated in place; y into x
  FEAB_CUDA(cudaMemcpyAsync(work, b, bytes, cudaMemcpyDeviceToDevice, s));
  for (int K = 0; K < NT; ++K) {
    const int below = std::min(bands, NT - 1 - K);
    k_band_fwd<<<std::max(1, below), 128, 0, s>>>(tiles, inv, bands, K, below, work, x);
  }
  // backward: x (= y) updated in place; the solution into work, then copied to x
  for (int K = NT - 1; K >= 0; --K) {
    const int above = std::min(bands, K);
    k_band_bwd<<<std::max(1, above), 128, 0, s>>>(tiles, inv, bands, K, above, x, work);
  }
  count_launches(2 * (uint64_t)NT);
  FEAB_CHECK_LAUNCH();
  FEAB_CUDA(cudaMemcpyAsync(x, work, bytes, cudaMemcpyDeviceToDevice, s));
  // rows past n are identity rows with b = 0, so x is 0 there
  return FEAB_OK;
}
