// SIMP optimality-criteria loop kernels (fea_engine/src/fea_engine/topopt.py:235-379):
//   - the sensitivity-filter weights H[e, j] = max(0, r - |c_e - c_j|) over element centroids
//     (build_filter_weights, :235-243), kept sparse (CSR over elements, columns ascending);
//   - the filter dc~_e = sum_j H_ej rho_j dc_j / max(max(rho_e, eps) sum_j H_ej, eps)
//     (apply_sensitivity_filter, :246-253);
//   - the OC update (oc_update, :259-295): the bracket expansion and the bisection on the
//     volume multiplier run on the device, one kernel per step, with the multiplier bracket in
//     device state; steps after convergence return at once, so no host synchronisation is needed.
//
// The filter build compares every pair of centroids, tiled through shared memory: O(E^2) work
// done once per mesh (E = 98,304 takes milliseconds).  Distances are formed as the reference forms
// them, ((dx^2 + dy^2) + dz^2) without fused multiply-adds, so the set of neighbours and the
// weights are the reference's bit for bit.
#include <algorithm>
#include "feab_common.cuh"
#include "feab_scan.cuh"

namespace feab {
namespace {

constexpr int kFiltThreads = 256;
constexpr int kOcThreads = 256;

size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

// centroid = mean of the 8 corner coordinates (mesh.nodes[conn].mean(axis=1)): summed in
// corner order, then divided by 8.
__global__ void k_centroids(const double* __restrict__ coords, const int32_t* __restrict__ conn, int64_t n_elem,
                            double* __restrict__ cent) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elem) return;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s = __dadd_rn(s, coords[(int64_t)conn[e * 8 + k] * 3 + j]);
    cent[e * 3 + j] = s / 8.0;
  }
}

// |c_e - c_j| as numpy forms it: diff, square, sum over the 3 axes in order, sqrt.
__device__ __forceinline__ double ref_dist(double ax, double ay, double az, double bx, double by, double bz) {
  const double dx = __dsub_rn(ax, bx), dy = __dsub_rn(ay, by), dz = __dsub_rn(az, bz);
  return sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

// Row e's neighbours j (ascending) with weight r - dist > 0.  FILL = false: counts only.
template <bool FILL>
__global__ void __launch_bounds__(kFiltThreads) k_filter_pairs(const double* __restrict__ cent, int64_t n_elem,
                                                               double radius, int32_t* __restrict__ counts,
                                                               const int32_t* __restrict__ ptr,
                                                               int32_t* __restrict__ idx, double* __restrict__ w,
                                                               double* __restrict__ rowsum) {
  __shared__ double tile[3][kFiltThreads];
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = e < n_elem;
  const double cx = live ? cent[e * 3] : 0.0, cy = live ? cent[e * 3 + 1] : 0.0, cz = live ? cent[e * 3 + 2] : 0.0;
  // cheap pre-test on the squared distance with a margin; the exact test is on r - dist
  const double r2 = radius * radius * (1.0 + 1e-9);
  int cnt = 0;
  int64_t out = FILL && live ? ptr[e] : 0;
  double rs = 0.0;
  for (int64_t j0 = 0; j0 < n_elem; j0 += kFiltThreads) {
    const int64_t j = j0 + threadIdx.x;
    __syncthreads();
    if (j < n_elem) {
      tile[0][threadIdx.x] = cent[j * 3];
      tile[1][threadIdx.x] = cent[j * 3 + 1];
      tile[2][threadIdx.x] = cent[j * 3 + 2];
    }
    __syncthreads();
    const int m = n_elem - j0 < kFiltThreads ? (int)(n_elem - j0) : kFiltThreads;
    if (!live) continue;
    for (int t = 0; t < m; ++t) {
      const double dx = cx - tile[0][t], dy = cy - tile[1][t], dz = cz - tile[2][t];
      if (dx * dx + dy * dy + dz * dz > r2) continue;
      const double h = radius - ref_dist(cx, cy, cz, tile[0][t], tile[1][t], tile[2][t]);
      if (!(h > 0.0)) continue;
      if (FILL) {
        idx[out] = (int32_t)(j0 + t);
        w[out] = h;
        ++out;
        rs += h;
      } else {
        ++cnt;
      }
    }
  }
  if (!live) return;
  if (FILL) rowsum[e] = rs;
  else counts[e] = cnt;
}

__global__ void k_filter_apply(const int32_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                               const double* __restrict__ w, const double* __restrict__ rowsum, int64_t n_elem,
                               const double* __restrict__ rho, const double* __restrict__ dc, double eps,
                               double* __restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elem) return;
  double s = 0.0;
  for (int k = ptr[e]; k < ptr[e + 1]; ++k) {
    const int j = idx[k];
    s += w[k] * (rho[j] * dc[j]);
  }
  const double denom = fmax(rho[e], eps) * rowsum[e];
  out[e] = s / fmax(denom, eps);
}

// ---- OC update ---------------------------------------------------------------------------
struct OcState {
  double l1, l2, lmid, max_change;
  int32_t phase;      // 0: expanding the bracket, 1: bisecting, 2: done
  int32_t steps;      // steps taken in the current phase
  uint32_t ticket;
  int32_t pad;
};

__global__ void k_oc_init(OcState* S) {
  S->l1 = 1e-12;
  S->l2 = 1.0;
  S->lmid = 0.0;
  S->max_change = 0.0;
  S->phase = 0;
  S->steps = 0;
  S->ticket = 0;
}

// One step of oc_update: the trial densities for the current multiplier, their sum (fixed order:
// per-block partials, reduced by the last block) and, in the bisection, the densities themselves
// and max |rho_new - rho|; the last block advances the bracket exactly as the reference does.
__global__ void __launch_bounds__(kOcThreads) k_oc_step(const double* __restrict__ rho, const double* __restrict__ dc,
                                                        int64_t n_elem, double vf, double move, double lo_bound,
                                                        double hi_bound, double tol, int max_expand, int max_bisect,
                                                        double* __restrict__ rho_new, double* __restrict__ partials,
                                                        OcState* S, double* __restrict__ max_change_out) {
  __shared__ double sh[2][kOcThreads / 32];
  __shared__ bool last;
  const int phase = S->phase;
  if (phase == 2) return;
  const double lam = phase == 0 ? S->l2 : 0.5 * (S->l1 + S->l2);
  double sum = 0.0, mx = 0.0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_elem; e += (int64_t)gridDim.x * blockDim.x) {
    const double d = fmin(dc[e], -1e-12);
    const double r = rho[e];
    double t = r * sqrt(-d / lam);
    t = fmin(fmax(t, r - move), r + move);
    t = fmin(fmax(t, lo_bound), hi_bound);
    sum += t;
    if (phase == 1) {
      rho_new[e] = t;
      mx = fmax(mx, fabs(t - r));
    }
  }
  sum = warp_sum(sum);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(FEAB_FULL_MASK, mx, o));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    sh[0][wid] = sum;
    sh[1][wid] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0, m = 0.0;
    for (int k = 0; k < kOcThreads / 32; ++k) {
      s += sh[0][k];
      m = fmax(m, sh[1][k]);
    }
    partials[2 * blockIdx.x] = s;
    partials[2 * blockIdx.x + 1] = m;
    __threadfence();
    last = atomicAdd(&S->ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  double s = 0.0, m = 0.0;
  for (unsigned b = 0; b < gridDim.x; ++b) {
    s += __ldcg(&partials[2 * b]);
    m = fmax(m, __ldcg(&partials[2 * b + 1]));
  }
  S->ticket = 0;
  const double mean = s / (double)n_elem;
  if (phase == 0) {
    // for _ in range(60): ...; if mean <= vf: break; l2 *= 2
    if (mean <= vf) {
      S->phase = 1;
      S->steps = 0;
    } else {
      S->l2 = S->l2 * 2.0;
      if (++S->steps >= max_expand) {
        S->phase = 1;
        S->steps = 0;
      }
    }
  } else {
    S->lmid = lam;
    if (mean > vf) S->l1 = lam;
    else S->l2 = lam;
    S->max_change = m;
    *max_change_out = m;
    if ((S->l2 - S->l1) < tol * fmax(S->l2, 1.0) || ++S->steps >= max_bisect) S->phase = 2;
  }
}

constexpr int kMaxExpand = 60;

int oc_grid(int64_t n_elem) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n_elem + kOcThreads - 1) / kOcThreads, 2 * (int64_t)sm_count()));
}

}  // namespace
}  // namespace feab

using namespace feab;

extern "C" int32_t feab_element_centroids(const double* coords, const int32_t* conn, int64_t n_elem,
                                          double* centroids, cudaStream_t s) {
  if (!coords || !conn || !centroids || n_elem <= 0) return FEAB_BAD_ARG;
  k_centroids<<<(unsigned)((n_elem + kFiltThreads - 1) / kFiltThreads), kFiltThreads, 0, s>>>(coords, conn, n_elem,
                                                                                             centroids);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}

extern "C" size_t feab_filter_scratch_bytes(int64_t n_elem) {
  if (n_elem <= 0) return 0;
  return a256(sizeof(int32_t) * ((size_t)n_elem + 1)) + a256(sizeof(int64_t) * ((size_t)scan_blocks(n_elem + 1) + 2)) +
         a256(sizeof(int64_t));
}

extern "C" int32_t feab_filter_build(const double* centroids, int64_t n_elem, double radius, int32_t* ptr,
                                     int32_t* idx, double* w, double* rowsum, int64_t* nnz_out, void* scratch,
                                     size_t scratch_bytes, cudaStream_t s) {
  if (!centroids || !ptr || n_elem <= 0 || n_elem >= INT32_MAX || !(radius > 0.0)) return FEAB_BAD_ARG;
  const bool fill = idx != nullptr;
  if (fill && (!w || !rowsum)) return FEAB_BAD_ARG;
  const unsigned grid = (unsigned)((n_elem + kFiltThreads - 1) / kFiltThreads);
  if (!fill) {
    if (!scratch || scratch_bytes < feab_filter_scratch_bytes(n_elem)) return FEAB_BAD_ARG;
    char* base = static_cast<char*>(scratch);
    int32_t* counts = reinterpret_cast<int32_t*>(base);
    int64_t* scan = reinterpret_cast<int64_t*>(base + a256(sizeof(int32_t) * ((size_t)n_elem + 1)));
    int64_t* total = reinterpret_cast<int64_t*>(reinterpret_cast<char*>(scan) +
                                                a256(sizeof(int64_t) * ((size_t)scan_blocks(n_elem + 1) + 2)));
    k_filter_pairs<false><<<grid, kFiltThreads, 0, s>>>(centroids, n_elem, radius, counts, nullptr, nullptr, nullptr,
                                                        nullptr);
    count_launches(1);
    FEAB_CHECK_LAUNCH();
    FEAB_CUDA(scan_exclusive_i32(counts, ptr, n_elem, scan, total, s));
    count_launches(3);
    int64_t nnz = 0;
    FEAB_CUDA(cudaMemcpyAsync(&nnz, total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    FEAB_CUDA(cudaStreamSynchronize(s));
    if (nnz >= INT32_MAX) return FEAB_CAPACITY;
    if (nnz_out) *nnz_out = nnz;
    return FEAB_OK;
  }
  k_filter_pairs<true><<<grid, kFiltThreads, 0, s>>>(centroids, n_elem, radius, nullptr, ptr, idx, w, rowsum);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}

extern "C" int32_t feab_filter_apply(const int32_t* ptr, const int32_t* idx, const double* w, const double* rowsum,
                                     int64_t n_elem, const double* rho, const double* dc, double eps, double* out,
                                     cudaStream_t s) {
  if (!ptr || !idx || !w || !rowsum || !rho || !dc || !out || n_elem <= 0) return FEAB_BAD_ARG;
  if (out == rho || out == dc) return FEAB_BAD_ARG;  // rows read other elements' inputs
  const int threads = 256;
  k_filter_apply<<<(unsigned)((n_elem + threads - 1) / threads), threads, 0, s>>>(ptr, idx, w, rowsum, n_elem, rho,
                                                                                  dc, eps, out);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}

extern "C" size_t feab_oc_workspace_bytes(int64_t n_elem) {
  return a256(sizeof(OcState)) + a256(sizeof(double) * 2 * (size_t)oc_grid(std::max<int64_t>(n_elem, 1)));
}

extern "C" int32_t feab_oc_update(const double* rho, const double* dc, int64_t n_elem, double volume_fraction,
                                  double move, double rho_min_bound, double rho_max_bound, double bisection_tol,
                                  int32_t max_bisection_iter, double* rho_new, double* max_change, void* workspace,
                                  size_t workspace_bytes, cudaStream_t s) {
  if (!rho || !dc || !rho_new || !max_change || n_elem <= 0 || max_bisection_iter < 1) return FEAB_BAD_ARG;
  if (rho_new == rho || rho_new == dc) return FEAB_BAD_ARG;
  if (!workspace || workspace_bytes < feab_oc_workspace_bytes(n_elem)) return FEAB_BAD_ARG;
  OcState* S = static_cast<OcState*>(workspace);
  double* partials = reinterpret_cast<double*>(static_cast<char*>(workspace) + a256(sizeof(OcState)));
  const int grid = oc_grid(n_elem);
  k_oc_init<<<1, 1, 0, s>>>(S);
  // every step returns at once after convergence, so the fixed number of launches needs no
  // host round trip
  for (int k = 0; k < kMaxExpand + max_bisection_iter; ++k)
    k_oc_step<<<grid, kOcThreads, 0, s>>>(rho, dc, n_elem, volume_fraction, move, rho_min_bound, rho_max_bound,
                                          bisection_tol, kMaxExpand, max_bisection_iter, rho_new, partials, S,
                                          max_change);
  count_launches(1 + (uint64_t)(kMaxExpand + max_bisection_iter));
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}
