// Jacobi-preconditioned conjugate gradients on the GPU (d).
//
// CSR path (FP64 or FP32 values): one CG iteration is one "step" of two kernels:
//   A  p_new = z + beta p_old (formed on the fly inside the SpMV gathers, written for the
//      warp's own rows into the other half of a p ping-pong buffer), Ap = K p_new, p_new.Ap
//   B  x += alpha p, r -= alpha Ap, z = M r, r.r and r.z, convergence test, beta
// Sliced path (feab_sell_operator, FP64 or mixed values): three kernels,
//   P  p = z + beta p in place (when a new direction is pending)
//   A  Ap = K p through the SELL-32 layout, p.Ap
//   B  as above
// so the SpMV gathers one vector instead of two.  Either way the arithmetic of the direction
// update is exactly the reference's p = z + beta p.  Scalars live in a device PcgState; each
// kernel's last block (ticket counter) reduces the per-block partials in a fixed order, so
// results are bit-reproducible.  A chunk of steps is captured once in a CUDA graph and replayed;
// kernels return at once when the state says done, and the host polls the done flag one chunk
// behind, so there is no host sync per iteration.
//
// Precisions (feab_pcg_params.precision):
//   FEAB_PREC_FP64   the reference recurrence (iterative_solvers.py:434-481) in FP64.
//   FEAB_PREC_MIXED  FP64 vectors and scalars; the SpMV reads 6-byte values (doubles rounded
//                    to 36 mantissa bits) and applies K in difference form,
//                    y_a = sum_{b != a} K_ab (x_b - x_a) + S_a x_a, S_a = sum_b K_ab exact in FP64,
//                    so value rounding multiplies x_b - x_a (small for the smooth low modes)
//                    instead of x.  The residual is replaced by the FP64 b - K x (FP64 SpMV)
//                    whenever it has dropped by reliable_delta, and convergence is declared on
//                    that FP64 residual only.
//   FEAB_PREC_FP32   FP32 values, FP32 p/r/Ap/x-correction, FP64 scalars, FP64 reliable updates
//                    folding the correction into an FP64 solution.
#include <algorithm>
#include <cmath>
#include "feab_common.cuh"
#include "feab_graph.cuh"
#include "feab_scan.cuh"
#include "feab_sell.cuh"

namespace feab {
namespace {

constexpr int kThreads = 256;
constexpr int kModeCG = 0;
constexpr int kModeReliable = 1;

struct PcgState {
  double bnorm, tol, delta;
  double rz_old, pAp, alpha, beta, rr, relres, rmax, rr64;
  int32_t iters, maxiter, done, status;
  int32_t mode, p_pending, psel, xsel, reliable_updates;
  uint32_t ticket[4];
};

struct PcgArgs {
  int32_t n, n_groups;
  const int32_t* row_ptr;
  const int32_t* col_idx;
  const int32_t* group_ptr;
  const double* vals64;
  const float* vals32;
  SellView sell;           // sliced operator (FP64 or mixed values), when use_sell
  int use_sell;
  int vec2;                // x and dinv64 16-byte aligned: the vector passes use double2
  const double* dinv64;
  const float* dinv32;
  const double* b;
  const double* x0;
  double* x;
  PcgState* S_;
  double* partials;
  double *r, *z, *p0, *p1, *Ap;      // FP64 vectors (fp64, mixed)
  double *x64a, *x64b, *r64;         // fp32 mode: FP64 solution ping-pong + FP64 residual
  float *r32, *z32, *q0, *q1, *Ap32, *x32;  // fp32 mode vectors (q = p)
  int use_dinv;
};

__device__ __forceinline__ bool last_block_of(uint32_t* ticket) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t t = atomicAdd(ticket, 1u);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  return is_last;
}

// Writes this block's NV partial sums; the last block reduces all blocks' partials in a fixed
// order into tot[] and returns true.
template <int NV>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], double* partials, uint32_t* ticket, double (&tot)[NV]) {
  __shared__ double sh[NV * 32];
  block_sum<NV>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[k * gridDim.x + blockIdx.x] = v[k];
  }
  if (!last_block_of(ticket)) return false;
  double s[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) s[k] = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
#pragma unroll
    for (int k = 0; k < NV; ++k) s[k] += __ldcg(&partials[k * gridDim.x + i]);
  }
  block_sum<NV>(s, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) tot[k] = s[k];
    *ticket = 0;
  }
  return true;
}

// A row group's rows (r0 .. r0+f-1), the first row's start in col_idx / vals, and its length
// (all rows of a group have the same length and sit back to back in vals).
struct Group {
  int g, r0, f, s0, len;
  bool valid;
};

// Visits every row group.  Each warp owns tiles of 32 consecutive groups; lane l loads the
// descriptor of the tile's l-th group (group_ptr -> row_ptr), so the two dependent pointer
// loads are paid once per 32 groups.  The warp is
// split into 32/LPG sub-warps of LPG lanes; sub-warp s takes groups s, s + 32/LPG, ... of the
// tile, so 32/LPG groups have their loads in flight at once.  Lanes of a sub-warp with no group
// left get len = 0 (they still join the sub-warp's shuffles) and `valid` false.
template <int LPG, typename F>
__device__ __forceinline__ void for_each_group(const PcgArgs& A, int lane, F fn) {
  constexpr int NSG = 32 / LPG;
  const int G = A.group_ptr ? A.n_groups : A.n;
  const int wg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const int ntiles = (G + 31) >> 5;
  const int sg = lane / LPG;
  for (int tile = wg; tile < ntiles; tile += nw) {
    const int g = (tile << 5) + lane;
    int r0 = 0, f = 0, s0 = 0, len = 0;
    if (g < G) {
      if (A.group_ptr) {
        r0 = __ldg(A.group_ptr + g);
        f = __ldg(A.group_ptr + g + 1) - r0;
      } else {
        r0 = g;
        f = 1;
      }
      s0 = __ldg(A.row_ptr + r0);
      len = __ldg(A.row_ptr + r0 + 1) - s0;
    }
    const int cnt = min(32, G - (tile << 5));
    for (int i = 0; i < cnt; i += NSG) {
      const int src = (i + sg) & 31;
      Group gr;
      gr.g = (tile << 5) + i + sg;
      gr.r0 = __shfl_sync(FEAB_FULL_MASK, r0, src);
      gr.f = __shfl_sync(FEAB_FULL_MASK, f, src);
      gr.s0 = __shfl_sync(FEAB_FULL_MASK, s0, src);
      gr.len = __shfl_sync(FEAB_FULL_MASK, len, src);
      gr.valid = i + sg < cnt;
      if (!gr.valid) {
        gr.f = 0;
        gr.len = 0;
      }
      fn(gr);
    }
  }
}

// Sum over the LPG lanes of a sub-warp (xor offsets below LPG stay inside the sub-warp).
template <int LPG, typename T>
__device__ __forceinline__ T seg_sum(T v) {
#pragma unroll
  for (int o = LPG / 2; o > 0; o >>= 1) v += __shfl_xor_sync(FEAB_FULL_MASK, v, o);
  return v;
}

// acc[k] = sum_c vals[row r0+k, c] * xf(col c) for the f (<= 3) rows of a group, over the
// group's LPG lanes (hl = lane within the sub-warp), 3 column passes issued together.
template <int LPG, typename AT, typename VT, typename XF>
__device__ __forceinline__ void group_spmv(const PcgArgs& A, const VT* __restrict__ vals, const Group& G, int hl,
                                           XF xf, AT (&acc)[3]) {
  const int len = G.len, f = G.f;
  const int32_t* __restrict__ col = A.col_idx + G.s0;
  const VT* __restrict__ v0 = vals + G.s0;
  AT a0 = 0, a1 = 0, a2 = 0;
  for (int c = hl; c < len; c += 3 * LPG) {
    const bool p1 = c + LPG < len, p2 = c + 2 * LPG < len;
    const int j0 = __ldg(col + c);
    const int j1 = p1 ? __ldg(col + c + LPG) : 0;
    const int j2 = p2 ? __ldg(col + c + 2 * LPG) : 0;
    const AT w00 = (AT)__ldg(v0 + c);
    const AT w01 = p1 ? (AT)__ldg(v0 + c + LPG) : AT(0);
    const AT w02 = p2 ? (AT)__ldg(v0 + c + 2 * LPG) : AT(0);
    AT w10 = 0, w11 = 0, w12 = 0, w20 = 0, w21 = 0, w22 = 0;
    if (f > 1) {
      w10 = (AT)__ldg(v0 + len + c);
      w11 = p1 ? (AT)__ldg(v0 + len + c + LPG) : AT(0);
      w12 = p2 ? (AT)__ldg(v0 + len + c + 2 * LPG) : AT(0);
    }
    if (f > 2) {
      w20 = (AT)__ldg(v0 + 2 * len + c);
      w21 = p1 ? (AT)__ldg(v0 + 2 * len + c + LPG) : AT(0);
      w22 = p2 ? (AT)__ldg(v0 + 2 * len + c + 2 * LPG) : AT(0);
    }
    const AT x0 = xf(j0);
    const AT x1 = p1 ? xf(j1) : AT(0);
    const AT x2 = p2 ? xf(j2) : AT(0);
    a0 += w00 * x0 + w01 * x1 + w02 * x2;
    a1 += w10 * x0 + w11 * x1 + w12 * x2;
    a2 += w20 * x0 + w21 * x1 + w22 * x2;
  }
  acc[0] = seg_sum<LPG>(a0);
  acc[1] = seg_sum<LPG>(a1);
  acc[2] = seg_sum<LPG>(a2);
}

__device__ __forceinline__ double pick3(const double (&a)[3], int k) { return k == 0 ? a[0] : (k == 1 ? a[1] : a[2]); }
__device__ __forceinline__ float pick3(const float (&a)[3], int k) { return k == 0 ? a[0] : (k == 1 ? a[1] : a[2]); }

__global__ void k_init_state(PcgState* S, double tol, double delta, int maxiter) {
  S->bnorm = 1.0;
  S->tol = tol;
  S->delta = delta;
  S->rz_old = S->pAp = S->alpha = S->beta = S->rr = S->relres = S->rmax = S->rr64 = 0.0;
  S->iters = 0;
  S->maxiter = maxiter;
  S->done = 0;
  S->status = FEAB_OK;
  S->mode = kModeCG;
  S->p_pending = 0;
  S->psel = 0;
  S->xsel = 0;
  S->reliable_updates = 0;
  for (int k = 0; k < 4; ++k) S->ticket[k] = 0;
}

// r = b - K64 x0 (plain form, FP64); ||b||, ||r||; early exit as iterative_solvers.py:437-443.
// fp32 mode writes the FP64 residual to r64, the others to r.
template <int PREC, int LPG>
__global__ void __launch_bounds__(kThreads) k_setup_a(PcgArgs A) {
  PcgState* S = A.S_;
  const int lane = threadIdx.x & 31;
  const int hl = lane % LPG;
  double* r = PREC == FEAB_PREC_FP32 ? A.r64 : A.r;
  double part[2] = {0.0, 0.0};
  for_each_group<LPG>(A, lane, [&](const Group& gr) {
    double acc[3] = {0.0, 0.0, 0.0};
    if (A.x0) group_spmv<LPG, double>(A, A.vals64, gr, hl, [&](int j) { return __ldg(A.x0 + j); }, acc);
    if (hl < gr.f) {
      const double bi = A.b[gr.r0 + hl];
      const double ri = bi - pick3(acc, hl);
      r[gr.r0 + hl] = ri;
      part[0] += bi * bi;
      part[1] += ri * ri;
    }
  });
  double tot[2];
  if (grid_reduce<2>(part, A.partials, &S->ticket[0], tot) && threadIdx.x == 0) {
    double bn = sqrt(tot[0]);
    if (bn == 0.0) bn = 1.0;
    S->bnorm = bn;
    S->rr = tot[1];
    S->rr64 = tot[1];
    S->relres = sqrt(tot[1]) / bn;
    if (S->relres < S->tol) {
      S->done = 1;
      S->status = FEAB_OK;
    }
  }
}

// z = M r, p = z, rz = r.z (fp32 mode: r32 = (float) r64 first, x32 = 0).
template <int PREC>
__global__ void __launch_bounds__(kThreads) k_setup_b(PcgArgs A) {
  PcgState* S = A.S_;
  if (S->done) return;
  double part[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
    if (PREC == FEAB_PREC_FP32) {
      const float ri = (float)A.r64[i];
      const float zi = A.use_dinv ? A.dinv32[i] * ri : ri;
      A.r32[i] = ri;
      A.z32[i] = zi;
      A.q0[i] = zi;
      A.x32[i] = 0.0f;
      part[0] += (double)ri * (double)zi;
    } else {
      const double ri = A.r[i];
      const double zi = A.use_dinv ? A.dinv64[i] * ri : ri;
      A.z[i] = zi;
      A.p0[i] = zi;
      part[0] += ri * zi;
    }
  }
  double tot[1];
  if (grid_reduce<1>(part, A.partials, &S->ticket[1], tot) && threadIdx.x == 0) {
    S->rz_old = tot[0];
    S->rmax = sqrt(S->rr);
    S->mode = kModeCG;
    S->p_pending = 0;
    S->psel = 0;
  }
}

// Step kernel A, CSR path (FP64 or FP32 values).
template <int PREC, int LPG>
__global__ void __launch_bounds__(kThreads, 4) k_step_a(PcgArgs A) {
  PcgState* S = A.S_;
  if (S->done) return;
  const int mode = S->mode;
  const int pend = S->p_pending;
  const int psel = S->psel;
  const int lane = threadIdx.x & 31;
  const int hl = lane % LPG;
  double part[1] = {0.0};
  if (PREC == FEAB_PREC_FP32 && mode == kModeReliable) {
    // r64 = b - K64 (x64 + x32); x64' = x64 + x32 (other half of the ping-pong)
    const double* xin = S->xsel ? A.x64b : A.x64a;
    double* xout = S->xsel ? A.x64a : A.x64b;
    for_each_group<LPG>(A, lane, [&](const Group& gr) {
      double acc[3];
      group_spmv<LPG, double>(A, A.vals64, gr, hl, [&](int j) { return __ldg(xin + j) + (double)__ldg(A.x32 + j); },
                         acc);
      if (hl < gr.f) {
        const int i = gr.r0 + hl;
        const double ri = A.b[i] - pick3(acc, hl);
        A.r64[i] = ri;
        xout[i] = xin[i] + (double)A.x32[i];
        part[0] += ri * ri;
      }
    });
  } else if (PREC == FEAB_PREC_FP32) {
    const float beta = (float)S->beta;
    const float* __restrict__ qo = psel ? A.q1 : A.q0;
    float* __restrict__ qn = psel ? A.q0 : A.q1;
    for_each_group<LPG>(A, lane, [&](const Group& gr) {
      float acc[3];
      if (pend) {
        group_spmv<LPG, float>(A, A.vals32, gr, hl, [&](int j) { return fmaf(beta, __ldg(qo + j), __ldg(A.z32 + j)); },
                          acc);
      } else {
        group_spmv<LPG, float>(A, A.vals32, gr, hl, [&](int j) { return __ldg(qo + j); }, acc);
      }
      if (hl < gr.f) {
        const int i = gr.r0 + hl;
        const float pi = pend ? fmaf(beta, qo[i], A.z32[i]) : qo[i];
        if (pend) qn[i] = pi;
        const float v = pick3(acc, hl);
        A.Ap32[i] = v;
        part[0] += (double)pi * (double)v;
      }
    });
  } else {
    const double beta = S->beta;
    const double* __restrict__ po = psel ? A.p1 : A.p0;
    double* __restrict__ pn = psel ? A.p0 : A.p1;
    for_each_group<LPG>(A, lane, [&](const Group& gr) {
      double acc[3];
      if (pend)
        group_spmv<LPG, double>(A, A.vals64, gr, hl, [&](int j) { return __ldg(A.z + j) + beta * __ldg(po + j); },
                                acc);
      else
        group_spmv<LPG, double>(A, A.vals64, gr, hl, [&](int j) { return __ldg(po + j); }, acc);
      if (hl < gr.f) {
        const int i = gr.r0 + hl;
        const double pi = pend ? A.z[i] + beta * po[i] : po[i];
        if (pend) pn[i] = pi;
        const double v = pick3(acc, hl);
        A.Ap[i] = v;
        part[0] += pi * v;
      }
    });
  }
  double tot[1];
  if (grid_reduce<1>(part, A.partials, &S->ticket[0], tot) && threadIdx.x == 0) {
    if (mode == kModeReliable && PREC != FEAB_PREC_FP64) {
      S->rr64 = tot[0];
    } else {
      if (pend) S->psel = psel ^ 1;
      S->p_pending = 0;
      S->pAp = tot[0];
      if (!(tot[0] > 0.0)) {  // p^T A p <= 0: A is not SPD (iterative_solvers.py:450-454)
        S->status = FEAB_NOT_SPD;
        S->done = 1;
      } else {
        S->alpha = S->rz_old / tot[0];
      }
    }
  }
}

// Sliced path, kernel P: p = z + beta p in place when a new direction is pending.
__global__ void __launch_bounds__(kThreads) k_step_p(PcgArgs A) {
  const PcgState* S = A.S_;
  if (S->done || !S->p_pending) return;
  const double beta = S->beta;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  if (!A.vec2) {
    for (int i = t0; i < A.n; i += stride) A.p0[i] = A.z[i] + beta * A.p0[i];
    return;
  }
  double2* __restrict__ p2 = reinterpret_cast<double2*>(A.p0);
  const double2* __restrict__ z2 = reinterpret_cast<const double2*>(A.z);
  for (int i = t0; i < (A.n >> 1); i += stride) {
    const double2 pv = p2[i], zv = z2[i];
    p2[i] = make_double2(zv.x + beta * pv.x, zv.y + beta * pv.y);
  }
  if ((A.n & 1) && t0 == 0) A.p0[A.n - 1] = A.z[A.n - 1] + beta * A.p0[A.n - 1];
}

// Sliced path, kernel A: Ap = K p and p.Ap through the SELL-32 operator (PREC = its kind); in a
// mixed reliable step, the FP64 residual r = b - K64 x through the CSR values instead.
template <int PREC, bool IDX16>
__global__ void __launch_bounds__(kThreads, SellTuning<PREC>::kMinBlocks) k_step_a_sell(PcgArgs A) {
  PcgState* S = A.S_;
  if (S->done) return;
  const int mode = S->mode;
  const int lane = threadIdx.x & 31;
  double part[1] = {0.0};
  if (PREC == FEAB_PREC_MIXED && mode == kModeReliable) {
    for_each_group<8>(A, lane, [&](const Group& gr) {
      double acc[3];
      const int hl = lane % 8;
      group_spmv<8, double>(A, A.vals64, gr, hl, [&](int j) { return __ldg(A.x + j); }, acc);
      if (hl < gr.f) {
        const int i = gr.r0 + hl;
        const double ri = A.b[i] - pick3(acc, hl);
        A.r[i] = ri;
        part[0] += ri * ri;
      }
    });
  } else if (FEAB_SELL_FUSED_P) {
    // p_new = z + beta p_old formed inside the gathers (two gathers per column) and written for
    // the lane's own rows into the other half of the p ping-pong; no separate P pass
    const int pend = S->p_pending, psel = S->psel;
    const double beta = S->beta;
    const double* __restrict__ po = psel ? A.p1 : A.p0;
    double* __restrict__ pn = psel ? A.p0 : A.p1;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int sl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; sl < A.sell.n_slices; sl += nw) {
      const SellLane L = sell_lane(A.sell, sl, lane);
      double acc[3], xs[3];
      if (pend)
        sell_apply<PREC, IDX16>(A.sell, sl, lane, L, [&](int j) { return __ldg(A.z + j) + beta * __ldg(po + j); }, acc, xs);
      else
        sell_apply<PREC, IDX16>(A.sell, sl, lane, L, [&](int j) { return __ldg(po + j); }, acc, xs);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (k < L.f) {
          const int i = L.r0 + k;
          const double pi = pend ? A.z[i] + beta * po[i] : po[i];
          if (pend) pn[i] = pi;
          A.Ap[i] = acc[k];
          part[0] += pi * acc[k];
        }
      }
    }
  } else {
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int sl = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; sl < A.sell.n_slices; sl += nw) {
      const SellLane L = sell_lane(A.sell, sl, lane);
      double acc[3], xs[3];
      sell_apply<PREC, IDX16>(A.sell, sl, lane, L, [&](int j) { return __ldg(A.p0 + j); }, acc, xs);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (k < L.f) {
          const int i = L.r0 + k;
          A.Ap[i] = acc[k];
          part[0] += A.p0[i] * acc[k];
        }
      }
    }
  }
  double tot[1];
  if (grid_reduce<1>(part, A.partials, &S->ticket[0], tot) && threadIdx.x == 0) {
    if (mode == kModeReliable && PREC != FEAB_PREC_FP64) {
      S->rr64 = tot[0];
    } else {
      if (FEAB_SELL_FUSED_P && S->p_pending) S->psel ^= 1;
      S->p_pending = 0;
      S->pAp = tot[0];
      if (!(tot[0] > 0.0)) {  // p^T A p <= 0: A is not SPD (iterative_solvers.py:450-454)
        S->status = FEAB_NOT_SPD;
        S->done = 1;
      } else {
        S->alpha = S->rz_old / tot[0];
      }
    }
  }
}

// Step kernel B.
template <int PREC>
__global__ void __launch_bounds__(kThreads) k_step_b(PcgArgs A) {
  PcgState* S = A.S_;
  if (S->done) return;
  const int mode = S->mode;
  const int psel = S->psel;
  const int stride = gridDim.x * blockDim.x;
  double part[2] = {0.0, 0.0};
  if (mode == kModeReliable && PREC == FEAB_PREC_FP32) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += stride) {
      const float ri = (float)A.r64[i];
      const float zi = A.use_dinv ? A.dinv32[i] * ri : ri;
      A.r32[i] = ri;
      A.z32[i] = zi;
      A.x32[i] = 0.0f;
      part[1] += (double)ri * (double)zi;
    }
  } else if (mode == kModeReliable && PREC == FEAB_PREC_MIXED) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += stride) {
      const double ri = A.r[i];
      const double zi = A.use_dinv ? A.dinv64[i] * ri : ri;
      A.z[i] = zi;
      part[1] += ri * zi;
    }
  } else if (PREC == FEAB_PREC_FP32) {
    const float alpha = (float)S->alpha;
    const float* __restrict__ q = psel ? A.q1 : A.q0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += stride) {
      A.x32[i] = fmaf(alpha, q[i], A.x32[i]);
      const float ri = fmaf(-alpha, A.Ap32[i], A.r32[i]);
      A.r32[i] = ri;
      const float zi = A.use_dinv ? A.dinv32[i] * ri : ri;
      A.z32[i] = zi;
      part[0] += (double)ri * (double)ri;
      part[1] += (double)ri * (double)zi;
    }
  } else {
    const double alpha = S->alpha;
    const double* __restrict__ p = psel ? A.p1 : A.p0;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    auto one = [&](int i) {
      A.x[i] += alpha * p[i];
      const double ri = A.r[i] - alpha * A.Ap[i];
      A.r[i] = ri;
      const double zi = A.use_dinv ? A.dinv64[i] * ri : ri;
      A.z[i] = zi;
      part[0] += ri * ri;
      part[1] += ri * zi;
    };
    if (A.vec2) {
      // two rows per thread with 16-byte loads, all loads of the pair issued together
      const double2* __restrict__ p2 = reinterpret_cast<const double2*>(p);
      double2* __restrict__ x2 = reinterpret_cast<double2*>(A.x);
      double2* __restrict__ r2 = reinterpret_cast<double2*>(A.r);
      double2* __restrict__ z2 = reinterpret_cast<double2*>(A.z);
      const double2* __restrict__ a2 = reinterpret_cast<const double2*>(A.Ap);
      const double2* __restrict__ d2 = reinterpret_cast<const double2*>(A.dinv64);
      for (int i = t0; i < (A.n >> 1); i += stride) {
        const double2 pv = p2[i], xv = x2[i], rv = r2[i], av = a2[i];
        const double2 dv = A.use_dinv ? d2[i] : make_double2(1.0, 1.0);
        const double r0 = rv.x - alpha * av.x, r1 = rv.y - alpha * av.y;
        const double z0 = A.use_dinv ? dv.x * r0 : r0, z1 = A.use_dinv ? dv.y * r1 : r1;
        x2[i] = make_double2(xv.x + alpha * pv.x, xv.y + alpha * pv.y);
        r2[i] = make_double2(r0, r1);
        z2[i] = make_double2(z0, z1);
        part[0] += r0 * r0;
        part[0] += r1 * r1;
        part[1] += r0 * z0;
        part[1] += r1 * z1;
      }
      if ((A.n & 1) && t0 == 0) one(A.n - 1);
    } else {
      for (int i = t0; i < A.n; i += stride) one(i);
    }
  }
  double tot[2];
  if (!grid_reduce<2>(part, A.partials, &S->ticket[1], tot) || threadIdx.x != 0) return;
  if (mode == kModeCG) {
    S->iters += 1;
    S->rr = tot[0];
    const double rel = sqrt(tot[0]) / S->bnorm;
    if (PREC == FEAB_PREC_FP64) {
      S->relres = rel;
      if (rel < S->tol) {
        S->done = 1;
        S->status = FEAB_OK;
        return;
      }
      if (S->iters >= S->maxiter || !(rel == rel)) {
        S->done = 1;
        S->status = FEAB_NOT_CONVERGED;
        return;
      }
    } else if (rel < S->tol || sqrt(tot[0]) < S->delta * S->rmax || S->iters >= S->maxiter || !(rel == rel)) {
      S->mode = kModeReliable;  // the next step replaces r by the FP64 residual; p waits for it
      return;
    }
    S->beta = tot[1] / S->rz_old;
    S->rz_old = tot[1];
    S->p_pending = 1;
  } else {
    S->reliable_updates += 1;
    if (PREC == FEAB_PREC_FP32) S->xsel ^= 1;
    const double rel = sqrt(S->rr64) / S->bnorm;
    S->relres = rel;
    if (rel < S->tol) {
      S->done = 1;
      S->status = FEAB_OK;
      return;
    }
    if (S->iters >= S->maxiter || !(rel == rel)) {
      S->done = 1;
      S->status = FEAB_NOT_CONVERGED;
      return;
    }
    S->rmax = sqrt(S->rr64);
    S->beta = tot[1] / S->rz_old;
    S->rz_old = tot[1];
    S->mode = kModeCG;
    S->p_pending = 1;
  }
}

// fp32 mode: x = x64 + x32 (the correction is zero after a final reliable step).
__global__ void k_finalize_fp32(PcgArgs A) {
  const double* x64 = A.S_->xsel ? A.x64b : A.x64a;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x)
    A.x[i] = x64[i] + (double)A.x32[i];
}

// Standalone y = A x with the step-A SpMV (same group_spmv code and launch shape).
template <typename T, int LPG>
__global__ void __launch_bounds__(kThreads, 4) k_spmv(PcgArgs A, const T* __restrict__ x, T* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int hl = lane % LPG;
  const T* vals;
  if constexpr (sizeof(T) == 8) vals = reinterpret_cast<const T*>(A.vals64);
  else vals = reinterpret_cast<const T*>(A.vals32);
  for_each_group<LPG>(A, lane, [&](const Group& gr) {
    T acc[3];
    group_spmv<LPG, T>(A, vals, gr, hl, [&](int j) { return __ldg(x + j); }, acc);
    if (hl < gr.f) y[gr.r0 + hl] = pick3(acc, hl);
  });
}

// Difference-form operator, pass 1: per group the padded off-node column count Lp (the f own
// columns leave the list) and the value count f * Lp, scanned afterwards into goff / voff.
__global__ void k_diff_counts(int32_t n_groups, const int32_t* __restrict__ group_ptr,
                              const int32_t* __restrict__ row_ptr, int32_t* __restrict__ ccount,
                              int32_t* __restrict__ vcount) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_groups) return;
  const int r0 = group_ptr[g], f = group_ptr[g + 1] - r0;
  const int len = row_ptr[r0 + 1] - row_ptr[r0];
  const int lp = (len - f + 3) & ~3;
  ccount[g] = lp;
  vcount[g] = f * lp;
}

// Pass 2, one warp per group: tagged columns, 48-bit values (rounded to nearest on the dropped
// 16 bits), group masks, and the row-block sums S[r][j] = sum over the row's columns of DOF
// component j, accumulated in a fixed order (lanes in order, chunks in order).  The node's own
// columns are the f consecutive entries r0 .. r0+f-1 of the sorted column list.
__global__ void __launch_bounds__(kThreads) k_build_diff(int32_t n_groups, const int32_t* __restrict__ group_ptr,
                                                         const int32_t* __restrict__ row_ptr,
                                                         const int32_t* __restrict__ col_idx,
                                                         const double* __restrict__ vals,
                                                         const int32_t* __restrict__ dof_of,
                                                         const int32_t* __restrict__ goff,
                                                         const int32_t* __restrict__ voff,
                                                         int32_t* __restrict__ tcol, uint32_t* __restrict__ vhi,
                                                         uint16_t* __restrict__ vlo, uint8_t* __restrict__ vlo2,
                                                         uint8_t* __restrict__ gmask,
                                                         double* __restrict__ Ssum, int32_t* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (g >= n_groups) return;
  const int r0 = group_ptr[g], f = group_ptr[g + 1] - r0;
  const int c0 = goff[g], lp = goff[g + 1] - c0, v0 = voff[g];
  const int s00 = row_ptr[r0], len = row_ptr[r0 + 1] - s00;
  // position of the own columns (the entry equal to r0) in the sorted list
  int own = -1;
  for (int cb = 0; cb < len && own < 0; cb += 32) {
    const int c = cb + lane;
    const unsigned bal = __ballot_sync(FEAB_FULL_MASK, c < len && col_idx[s00 + c] == r0);
    if (bal) own = cb + __ffs(bal) - 1;
  }
  if (own < 0 || own + f > len || lp < len - f || lp > len - f + 3) {
    if (lane == 0) atomicExch(err, 1);
    return;
  }
  const int j0 = dof_of[r0] % 3;
  if (lane == 0) {
    int m = 0;
    for (int k = 0; k < f; ++k) m |= 1 << (dof_of[r0 + k] % 3);
    gmask[g] = (uint8_t)m;
  }
  for (int k = 0; k < f; ++k) {
    const int s0 = row_ptr[r0 + k];
    double sj[3] = {0.0, 0.0, 0.0}, tj[3] = {0.0, 0.0, 0.0};
    for (int cb = 0; cb < len; cb += 32) {
      const int c = cb + lane;
      double v = 0.0;
      int j = 0;
      if (c < len) {
        const int col = col_idx[s0 + c];
        j = dof_of[col] % 3;
        v = vals[s0 + c];
        if (c < own || c >= own + f) {
          const int p = c < own ? c : c - f;
          if (k == 0) tcol[c0 + p] = (int32_t)((uint32_t)col | ((uint32_t)j << 30));
          const unsigned long long bits = (unsigned long long)__double_as_longlong(v) + 0x80ull;  // 44 bits
          vhi[v0 + k * lp + p] = (uint32_t)(bits >> 32);
          vlo[v0 + k * lp + p] = (uint16_t)((bits >> 16) & 0xffffull);
          vlo2[v0 + k * lp + p] = (uint8_t)((bits >> 8) & 0xffull);
        }
      }
      // rounded value of an off-node column (0 for own columns and past the end)
      double wv = 0.0;
      if (c < len && (c < own || c >= own + f)) {
        const unsigned long long bw = (unsigned long long)__double_as_longlong(v) + 0x80ull;
        wv = __longlong_as_double((long long)(bw & ~0xffull));
      }
      for (int u = 0; u < 32; ++u) {
        const double vu = __shfl_sync(FEAB_FULL_MASK, v, u);
        const double wu = __shfl_sync(FEAB_FULL_MASK, wv, u);
        const int ju = __shfl_sync(FEAB_FULL_MASK, j, u);
        if (cb + u < len) {
          sj[ju] += vu;
          tj[ju] += wu;
        }
      }
    }
    // padding: own first free DOF, value 0
    for (int p = len - f + lane; p < lp; p += 32) {
      if (k == 0) tcol[c0 + p] = (int32_t)((uint32_t)r0 | ((uint32_t)j0 << 30));
      vhi[v0 + k * lp + p] = 0u;
      vlo[v0 + k * lp + p] = 0;
      vlo2[v0 + k * lp + p] = 0;
    }
    // T = S - W (S: all exact values of component j, W: the rounded off-node ones), so that
    // sum_{b != a} w (x_b - x_a) + S x_a = sum_{b != a} w x_b + T x_a exactly
    if (lane < 3) {
      const double sv = lane == 0 ? sj[0] : (lane == 1 ? sj[1] : sj[2]);
      const double tv = lane == 0 ? tj[0] : (lane == 1 ? tj[1] : tj[2]);
      Ssum[(int64_t)(r0 + k) * 3 + lane] = sv - tv;
    }
  }
}

size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

int max_grid() { return sm_count() * 8; }

struct Grids {
  int a, b;
};

Grids grids_for(int n, int G) {
  Grids g;
  // A: one warp per tile of 32 groups, 8 warps per block
  g.a = std::max(1, (int)std::min<int64_t>(((int64_t)G + 255) / 256, (int64_t)max_grid()));
  g.b = std::max(1, (int)std::min<int64_t>(((int64_t)n + kThreads * 2 - 1) / (kThreads * 2), (int64_t)max_grid()));
  return g;
}

size_t layout(int32_t n, int32_t precision, char* base, PcgArgs* A) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += a256(bytes);
    return base ? base + o : nullptr;
  };
  const size_t nd = sizeof(double) * (size_t)n, nf = sizeof(float) * (size_t)n;
  char* s = take(sizeof(PcgState));
  char* part = take(sizeof(double) * 2 * (size_t)max_grid());
  if (A) {
    A->S_ = reinterpret_cast<PcgState*>(s);
    A->partials = reinterpret_cast<double*>(part);
  }
  if (precision == FEAB_PREC_FP32) {
    char* xa = take(nd);
    char* xb = take(nd);
    char* r64 = take(nd);
    char* r32 = take(nf);
    char* z32 = take(nf);
    char* q0 = take(nf);
    char* q1 = take(nf);
    char* ap32 = take(nf);
    char* x32 = take(nf);
    if (A) {
      A->x64a = reinterpret_cast<double*>(xa);
      A->x64b = reinterpret_cast<double*>(xb);
      A->r64 = reinterpret_cast<double*>(r64);
      A->r32 = reinterpret_cast<float*>(r32);
      A->z32 = reinterpret_cast<float*>(z32);
      A->q0 = reinterpret_cast<float*>(q0);
      A->q1 = reinterpret_cast<float*>(q1);
      A->Ap32 = reinterpret_cast<float*>(ap32);
      A->x32 = reinterpret_cast<float*>(x32);
    }
  } else {
    char* r = take(nd);
    char* z = take(nd);
    char* p0 = take(nd);
    char* p1 = take(nd);
    char* ap = take(nd);
    if (A) {
      A->r = reinterpret_cast<double*>(r);
      A->z = reinterpret_cast<double*>(z);
      A->p0 = reinterpret_cast<double*>(p0);
      A->p1 = reinterpret_cast<double*>(p1);
      A->Ap = reinterpret_cast<double*>(ap);
    }
  }
  return off;
}

template <int PREC>
void launch_setup(const PcgArgs& A, const Grids& gr, int lpg, cudaStream_t s) {
  if (lpg == 4) k_setup_a<PREC, 4><<<gr.a, kThreads, 0, s>>>(A);
  else if (lpg == 8) k_setup_a<PREC, 8><<<gr.a, kThreads, 0, s>>>(A);
  else if (lpg == 16) k_setup_a<PREC, 16><<<gr.a, kThreads, 0, s>>>(A);
  else k_setup_a<PREC, 32><<<gr.a, kThreads, 0, s>>>(A);
  k_setup_b<PREC><<<gr.b, kThreads, 0, s>>>(A);
  count_launches(2);
}

template <int PREC>
void launch_step(const PcgArgs& A, const Grids& gr, int lpg, cudaStream_t s) {
  if (lpg == 4) k_step_a<PREC, 4><<<gr.a, kThreads, 0, s>>>(A);
  else if (lpg == 8) k_step_a<PREC, 8><<<gr.a, kThreads, 0, s>>>(A);
  else if (lpg == 16) k_step_a<PREC, 16><<<gr.a, kThreads, 0, s>>>(A);
  else k_step_a<PREC, 32><<<gr.a, kThreads, 0, s>>>(A);
  k_step_b<PREC><<<gr.b, kThreads, 0, s>>>(A);
}

// Sliced path: P, A (one warp per slice of 32 node groups), B.
int sell_grid(const PcgArgs& A) {
  const int wpb = kThreads / 32;
  return std::max(1, std::min((A.sell.n_slices + wpb - 1) / wpb, max_grid()));
}

template <int PREC>
void launch_step_sell(const PcgArgs& A, const Grids& gr, cudaStream_t s) {
  if (!FEAB_SELL_FUSED_P) k_step_p<<<gr.b, kThreads, 0, s>>>(A);
  if (A.sell.tcol16) k_step_a_sell<PREC, true><<<sell_grid(A), kThreads, 0, s>>>(A);
  else k_step_a_sell<PREC, false><<<sell_grid(A), kThreads, 0, s>>>(A);
  k_step_b<PREC><<<gr.b, kThreads, 0, s>>>(A);
}

int normalize_lpg(int lpg) { return lpg == 4 || lpg == 8 || lpg == 16 || lpg == 32 ? lpg : 16; }

int32_t run_pcg(const PcgArgs& A, int prec, int chunk, int maxiter, int lpg, feab_pcg_result* result,
                cudaStream_t s) {
  const Grids gr = grids_for(A.n, A.group_ptr ? A.n_groups : A.n);
  SolverState& state = thread_solver_state<0>();
  HostFlag& flag = state.flag;
  if (!flag.ptr) return FEAB_CUDA_ERROR;
  if (prec == FEAB_PREC_FP32) launch_setup<FEAB_PREC_FP32>(A, gr, lpg, s);
  else if (prec == FEAB_PREC_MIXED) launch_setup<FEAB_PREC_MIXED>(A, gr, lpg, s);
  else launch_setup<FEAB_PREC_FP64>(A, gr, lpg, s);
  FEAB_CHECK_LAUNCH();

  GraphCache& graphs = state.graphs;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int32_t rc = FEAB_OK;
  int64_t launched = 0;
  auto fail = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == FEAB_OK) rc = FEAB_CUDA_ERROR;
    return e != cudaSuccess;
  };
  do {
    if (fail(graphs.events(ev))) break;
    // the chunk's launches bake in A, the launch shapes and the chunk length
    const uint64_t topo = topo_signature({prec, chunk, lpg, A.use_sell, gr.a, gr.b, A.use_sell ? sell_grid(A) : 0,
                                          FEAB_SELL_FUSED_P});
    auto record = [&](cudaStream_t cs) {
      for (int c = 0; c < chunk; ++c) {
        if (prec == FEAB_PREC_FP32) launch_step<FEAB_PREC_FP32>(A, gr, lpg, cs);
        else if (prec == FEAB_PREC_MIXED) launch_step_sell<FEAB_PREC_MIXED>(A, gr, cs);
        else if (A.use_sell) launch_step_sell<FEAB_PREC_FP64>(A, gr, cs);
        else launch_step<FEAB_PREC_FP64>(A, gr, lpg, cs);
      }
      cudaMemcpyAsync((void*)flag.ptr, &A.S_->done, sizeof(int32_t), cudaMemcpyDeviceToHost, cs);
    };
    if (fail(graphs.acquire(&A, sizeof(A), topo, record, &exec))) break;

    // Every CG iteration is one step and a reliable step follows at most every iteration, so
    // 2*maxiter + 2 steps always suffice: the host loop is bounded.
    const int64_t max_launch = (2 * (int64_t)maxiter + 2 + chunk - 1) / chunk + 1;
    flag.ptr[0] = 0;
    if (fail(cudaGraphLaunch(exec, s))) break;
    if (fail(cudaEventRecord(ev[0], s))) break;
    launched = 1;
    const uint64_t per_step = A.use_sell ? (FEAB_SELL_FUSED_P ? 2 : 3) : 2;
    count_launches(per_step * (uint64_t)chunk);
    while (true) {
      const bool more = launched < max_launch;
      if (more) {
        if (fail(cudaGraphLaunch(exec, s))) break;
        if (fail(cudaEventRecord(ev[launched & 1], s))) break;
        ++launched;
        count_launches(per_step * (uint64_t)chunk);
      }
      if (fail(cudaEventSynchronize(ev[more ? ((launched - 2) & 1) : ((launched - 1) & 1)]))) break;
      if (flag.ptr[0] != 0 || !more) break;
    }
  } while (false);

  if (rc == FEAB_OK && prec == FEAB_PREC_FP32) {
    k_finalize_fp32<<<gr.b, kThreads, 0, s>>>(A);
    count_launches(1);
    fail(cudaGetLastError());
  }
  PcgState hs;
  if (rc == FEAB_OK) {
    if (!fail(cudaMemcpyAsync(&hs, A.S_, sizeof(PcgState), cudaMemcpyDeviceToHost, s))) fail(cudaStreamSynchronize(s));
  }
  if (rc != FEAB_OK) {
    if (result) result->status = rc;
    return rc;
  }
  int32_t st = hs.status;
  if (hs.done == 0) st = FEAB_NOT_CONVERGED;
  if (result) {
    result->status = st;
    result->iters = hs.iters;
    result->reliable_updates = hs.reliable_updates;
    result->graph_launches = (int32_t)launched;
    result->relres = hs.relres;
    result->bnorm = hs.bnorm;
  }
  return st;
}

// The FP64 vector passes read two rows per 16-byte load when every vector they touch is 16-byte
// aligned (workspace vectors sit at 256-byte offsets of the caller's buffer).
void set_vec2(PcgArgs* A) {
  auto al = [](const void* p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  A->vec2 = al(A->x) && (!A->use_dinv || al(A->dinv64)) && al(A->r) && al(A->z) && al(A->p0) && al(A->p1) &&
            al(A->Ap);
}

void fill_matrix(const feab_csr* M, PcgArgs* A) {
  A->n = M->n;
  A->n_groups = M->n_groups;
  A->row_ptr = M->row_ptr;
  A->col_idx = M->col_idx;
  A->group_ptr = M->group_ptr;
  A->vals64 = M->vals64;
  A->vals32 = M->vals32;
}

void fill_sell(const feab_csr* M, const feab_sell_operator* D, PcgArgs* A) {
  A->sell = sell_view(M, D);
  A->use_sell = 1;
}

// A sliced operator fits A, is of the kind the precision needs, and its arrays have the alignment
// of the SpMV's vector loads (16 bytes; 8 for the 16-bit lo words).
bool sell_fits(const feab_csr* M, const feab_sell_operator* D, int kind) {
  auto al = [](const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; };
  return D && M->group_ptr && M->n_groups > 0 && D->kind == kind && D->n_slices == (M->n_groups + 31) / 32 &&
         D->soff && D->tcol && al(D->tcol, 16) && (!D->tcol16 || al(D->tcol16, 8)) &&
         (kind == FEAB_PREC_FP64 ? (D->v64 != nullptr && al(D->v64, 16))
                                 : (D->vhi && D->vlo && D->gmask && D->S && al(D->vhi, 16) && al(D->vlo, 8)));
}

// Upper bounds from the sizes: sum_g Lp_g <= sum_g (len_g - f_g + 3) <= nnz + 3 G (f_g >= 1) and
// sum_g f_g Lp_g <= sum_g (f_g len_g - f_g^2 + 3 f_g) <= nnz + 2 G.
struct DiffScratch {
  int64_t* scan;
  int64_t* total;
  int32_t* err;
};

void diff_layout(int32_t n, int64_t nnz, int32_t n_groups, char* base, feab_diff_operator* D, size_t* total,
                 DiffScratch* X = nullptr) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + off : nullptr;
    off += a256(bytes);
    return p;
  };
  const size_t ncol = (size_t)nnz + 3 * (size_t)n_groups, nval = (size_t)nnz + 2 * (size_t)n_groups;
  char* tc = take(sizeof(int32_t) * ncol);
  char* hi = take(sizeof(uint32_t) * nval);
  char* lo = take(sizeof(uint16_t) * nval);
  char* lo2 = take(sizeof(uint8_t) * nval);
  char* gm = take((size_t)n_groups);
  char* ss = take(sizeof(double) * 3 * (size_t)n);
  char* go = take(sizeof(int32_t) * ((size_t)n_groups + 1));
  char* vo = take(sizeof(int32_t) * ((size_t)n_groups + 1));
  char* sc = take(sizeof(int64_t) * ((size_t)scan_blocks((int64_t)n_groups + 1) + 2));
  char* tt = take(sizeof(int64_t) + sizeof(int32_t));
  if (D) {
    D->tcol = reinterpret_cast<int32_t*>(tc);
    D->vhi = reinterpret_cast<uint32_t*>(hi);
    D->vlo = reinterpret_cast<uint16_t*>(lo);
    D->vlo2 = reinterpret_cast<uint8_t*>(lo2);
    D->gmask = reinterpret_cast<uint8_t*>(gm);
    D->S = reinterpret_cast<double*>(ss);
    D->goff = reinterpret_cast<int32_t*>(go);
    D->voff = reinterpret_cast<int32_t*>(vo);
  }
  if (X) {
    X->scan = reinterpret_cast<int64_t*>(sc);
    X->total = reinterpret_cast<int64_t*>(tt);
    X->err = reinterpret_cast<int32_t*>(tt + sizeof(int64_t));
  }
  if (total) *total = off;
}

}  // namespace
}  // namespace feab

using namespace feab;

extern "C" size_t feab_pcg_workspace_bytes(int32_t n, int32_t precision) {
  if (n < 0 || precision < FEAB_PREC_FP64 || precision > FEAB_PREC_FP32) return 0;
  return layout(n, precision, nullptr, nullptr);
}

extern "C" size_t feab_diff_operator_bytes(int32_t n, int64_t nnz, int32_t n_groups) {
  if (n < 0 || nnz < 0 || n_groups < 0) return 0;
  size_t total = 0;
  diff_layout(n, nnz, n_groups, nullptr, nullptr, &total);
  return total;
}

extern "C" int32_t feab_diff_operator_build(const feab_csr* M, const int32_t* dof_of, void* storage,
                                            size_t storage_bytes, feab_diff_operator* out, cudaStream_t s) {
  if (!M || !dof_of || !storage || !out || !M->group_ptr || M->n_groups <= 0 || !M->vals64 || M->n <= 0)
    return FEAB_BAD_ARG;
  if (reinterpret_cast<uintptr_t>(storage) & 15u) return FEAB_BAD_ARG;  // 16-byte quad loads of the operator
  if (M->n >= (1 << 30) || M->nnz + 3 * (int64_t)M->n_groups >= (int64_t)INT32_MAX) return FEAB_CAPACITY;
  if (feab_diff_operator_bytes(M->n, M->nnz, M->n_groups) > storage_bytes) return FEAB_BAD_ARG;
  DiffScratch X;
  diff_layout(M->n, M->nnz, M->n_groups, static_cast<char*>(storage), out, nullptr, &X);
  FEAB_CUDA(cudaMemsetAsync(X.err, 0, sizeof(int32_t), s));
  const int G = M->n_groups;
  k_diff_counts<<<(G + kThreads - 1) / kThreads, kThreads, 0, s>>>(G, M->group_ptr, M->row_ptr, out->goff, out->voff);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  FEAB_CUDA(scan_exclusive_i32(out->goff, out->goff, G, X.scan, X.total, s));
  FEAB_CUDA(scan_exclusive_i32(out->voff, out->voff, G, X.scan, X.total, s));
  const int wpb = kThreads / 32;
  k_build_diff<<<(G + wpb - 1) / wpb, kThreads, 0, s>>>(G, M->group_ptr, M->row_ptr, M->col_idx, M->vals64, dof_of,
                                                         out->goff, out->voff, out->tcol, out->vhi, out->vlo, out->vlo2,
                                                         out->gmask, out->S, X.err);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  int32_t err = 0;
  FEAB_CUDA(cudaMemcpyAsync(&err, X.err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaStreamSynchronize(s));
  return err ? FEAB_BAD_ARG : FEAB_OK;
}

extern "C" int32_t feab_pcg_solve(const feab_csr* M, const feab_sell_operator* sell, const double* dinv64,
                                  const float* dinv32, const double* b, const double* x0, double* x,
                                  const feab_pcg_params* prm, void* workspace, size_t workspace_bytes,
                                  feab_pcg_result* result, cudaStream_t s) {
  if (!M || !prm || !b || !x || !workspace || M->n <= 0 || !M->row_ptr || !M->col_idx || !M->vals64)
    return FEAB_BAD_ARG;
  const int prec = prm->precision;
  if (prec < FEAB_PREC_FP64 || prec > FEAB_PREC_FP32) return FEAB_BAD_ARG;
  if (prec == FEAB_PREC_FP32 && !M->vals32) return FEAB_BAD_ARG;
  if (prec == FEAB_PREC_MIXED && !sell_fits(M, sell, FEAB_PREC_MIXED)) return FEAB_BAD_ARG;
  if (prec == FEAB_PREC_FP64 && sell && !sell_fits(M, sell, FEAB_PREC_FP64)) return FEAB_BAD_ARG;
  if (prm->use_dinv && (prec == FEAB_PREC_FP32 ? !dinv32 : !dinv64)) return FEAB_BAD_ARG;
  if (M->group_ptr && M->n_groups <= 0) return FEAB_BAD_ARG;
  if (!(prm->tol >= 0.0)) return FEAB_BAD_ARG;
  PcgArgs A{};
  if (layout(M->n, prec, static_cast<char*>(workspace), &A) > workspace_bytes) return FEAB_BAD_ARG;
  fill_matrix(M, &A);
  if (sell && prec != FEAB_PREC_FP32) fill_sell(M, sell, &A);
  A.dinv64 = dinv64;
  A.dinv32 = dinv32;
  A.b = b;
  A.x0 = x0;
  A.x = x;
  A.use_dinv = prm->use_dinv ? 1 : 0;
  set_vec2(&A);
  const int maxiter = prm->maxiter > 0 ? prm->maxiter : (int)std::min<int64_t>(10 * (int64_t)M->n, INT32_MAX / 4);
  const double delta = prm->reliable_delta > 0.0 && prm->reliable_delta < 1.0 ? prm->reliable_delta : 0.1;
  const int chunk = prm->chunk > 0 ? std::min(prm->chunk, 256) : 16;
  k_init_state<<<1, 1, 0, s>>>(A.S_, prm->tol, delta, maxiter);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  if (prec == FEAB_PREC_FP32) {
    if (x0) FEAB_CUDA(cudaMemcpyAsync(A.x64a, x0, sizeof(double) * M->n, cudaMemcpyDeviceToDevice, s));
    else FEAB_CUDA(cudaMemsetAsync(A.x64a, 0, sizeof(double) * M->n, s));
    FEAB_CUDA(cudaMemsetAsync(A.x32, 0, sizeof(float) * M->n, s));
  } else if (x0) {
    if (x0 != x) FEAB_CUDA(cudaMemcpyAsync(x, x0, sizeof(double) * M->n, cudaMemcpyDeviceToDevice, s));
  } else {
    FEAB_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * M->n, s));
  }
  return run_pcg(A, prec, chunk, maxiter, normalize_lpg(prm->lanes_per_group), result, s);
}

extern "C" int32_t feab_csr_spmv(const feab_csr* M, const feab_sell_operator* sell, int32_t precision,
                                 int32_t lanes_per_group, const void* x, void* y, cudaStream_t s) {
  if (!M || !x || !y || M->n <= 0 || !M->row_ptr || !M->col_idx) return FEAB_BAD_ARG;
  if (precision < FEAB_PREC_FP64 || precision > FEAB_PREC_FP32) return FEAB_BAD_ARG;
  if (precision == FEAB_PREC_FP32 ? !M->vals32 : !M->vals64) return FEAB_BAD_ARG;
  if (precision == FEAB_PREC_MIXED && !sell_fits(M, sell, FEAB_PREC_MIXED)) return FEAB_BAD_ARG;
  if (precision == FEAB_PREC_FP64 && sell && !sell_fits(M, sell, FEAB_PREC_FP64)) return FEAB_BAD_ARG;
  if (M->group_ptr && M->n_groups <= 0) return FEAB_BAD_ARG;
  if (sell && precision != FEAB_PREC_FP32) {
    launch_sell_spmv(sell_view(M, sell), static_cast<const double*>(x), static_cast<double*>(y), s);
    FEAB_CHECK_LAUNCH();
    return FEAB_OK;
  }
  PcgArgs A{};
  fill_matrix(M, &A);
  const Grids gr = grids_for(A.n, A.group_ptr ? A.n_groups : A.n);
  const int lpg = normalize_lpg(lanes_per_group);
  const double* xd = static_cast<const double*>(x);
  double* yd = static_cast<double*>(y);
  const float* xf = static_cast<const float*>(x);
  float* yf = static_cast<float*>(y);
  if (precision != FEAB_PREC_FP32) {
    if (lpg == 4) k_spmv<double, 4><<<gr.a, kThreads, 0, s>>>(A, xd, yd);
    else if (lpg == 8) k_spmv<double, 8><<<gr.a, kThreads, 0, s>>>(A, xd, yd);
    else if (lpg == 16) k_spmv<double, 16><<<gr.a, kThreads, 0, s>>>(A, xd, yd);
    else k_spmv<double, 32><<<gr.a, kThreads, 0, s>>>(A, xd, yd);
  } else if (precision == FEAB_PREC_FP32) {
    if (lpg == 4) k_spmv<float, 4><<<gr.a, kThreads, 0, s>>>(A, xf, yf);
    else if (lpg == 8) k_spmv<float, 8><<<gr.a, kThreads, 0, s>>>(A, xf, yf);
    else if (lpg == 16) k_spmv<float, 16><<<gr.a, kThreads, 0, s>>>(A, xf, yf);
    else k_spmv<float, 32><<<gr.a, kThreads, 0, s>>>(A, xf, yf);
  }
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}

// ---------------------------------------------------------------- allocation-free FP64 PCG
// Fixed device scratch for feab_pcg_solve_noalloc: the PCG state, the block partials and the
// five FP64 work vectors live here instead of in caller-provided memory.  Every GPU that loads
// this library holds the array until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

extern "C" size_t feab_pcg_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

extern "C" int32_t feab_pcg_noalloc_max_n(void) {
  // largest n whose FP64 workspace layout fits the fixed scratch (layout grows by 40 B per row)
  int32_t lo = 0, hi = (int32_t)(kNoAllocScratchBytes / (5 * sizeof(double))) + 1;
  while (lo < hi) {
    const int32_t mid = lo + (hi - lo + 1) / 2;
    if (layout(mid, FEAB_PREC_FP64, nullptr, nullptr) <= kNoAllocScratchBytes) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

extern "C" int32_t feab_pcg_solve_noalloc(const feab_csr* M, const double* dinv64, const double* b, const double* x0,
                                          double* x, const feab_pcg_params* prm, feab_pcg_result* result,
                                          cudaStream_t s) {
  if (!M || !prm || !b || !x || M->n <= 0 || !M->row_ptr || !M->col_idx || !M->vals64) return FEAB_BAD_ARG;
  if (prm->precision != FEAB_PREC_FP64) return FEAB_BAD_ARG;
  if (prm->use_dinv && !dinv64) return FEAB_BAD_ARG;
  if (M->group_ptr && M->n_groups <= 0) return FEAB_BAD_ARG;
  if (!(prm->tol >= 0.0)) return FEAB_BAD_ARG;
  if (layout(M->n, FEAB_PREC_FP64, nullptr, nullptr) > kNoAllocScratchBytes) return FEAB_SCRATCH_LIMIT;
  // The array's device address on the current device, looked up on every call: the lookup
  // allocates nothing, and a cached address could go stale once the device's context is torn
  // down and created again (cudaDeviceReset), which moves the array.  The first call on a device
  // also loads this library's device code there, so it should come before any stream capture.
  void* scratch = nullptr;
  if (cudaGetSymbolAddress(&scratch, g_noalloc_scratch) != cudaSuccess || !scratch) return FEAB_CUDA_ERROR;
  PcgArgs A{};
  layout(M->n, FEAB_PREC_FP64, static_cast<char*>(scratch), &A);
  fill_matrix(M, &A);
  A.dinv64 = dinv64;
  A.b = b;
  A.x0 = x0;
  A.x = x;
  A.use_dinv = prm->use_dinv ? 1 : 0;
  set_vec2(&A);
  const int maxiter = prm->maxiter > 0 ? prm->maxiter : (int)std::min<int64_t>(10 * (int64_t)M->n, INT32_MAX / 4);
  const int chunk = prm->chunk > 0 ? std::min(prm->chunk, 256) : 16;
  const int lpg = normalize_lpg(prm->lanes_per_group);
  const Grids gr = grids_for(A.n, A.group_ptr ? A.n_groups : A.n);
  // the state (including the ticket counters) is rebuilt by every call
  k_init_state<<<1, 1, 0, s>>>(A.S_, prm->tol, 0.1, maxiter);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  if (x0) {
    if (x0 != x) FEAB_CUDA(cudaMemcpyAsync(x, x0, sizeof(double) * M->n, cudaMemcpyDeviceToDevice, s));
  } else {
    FEAB_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * M->n, s));
  }
  launch_setup<FEAB_PREC_FP64>(A, gr, lpg, s);
  FEAB_CHECK_LAUNCH();
  // plain launches in chunks, done flag read into a stack variable after each chunk
  const int64_t max_chunks = ((int64_t)maxiter + chunk - 1) / chunk + 1;
  int32_t done = 0;
  for (int64_t c = 0; c < max_chunks && !done; ++c) {
    for (int k = 0; k < chunk; ++k) launch_step<FEAB_PREC_FP64>(A, gr, lpg, s);
    count_launches(2 * (uint64_t)chunk);
    FEAB_CHECK_LAUNCH();
    FEAB_CUDA(cudaMemcpyAsync(&done, &A.S_->done, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    FEAB_CUDA(cudaStreamSynchronize(s));
  }
  PcgState hs;
  FEAB_CUDA(cudaMemcpyAsync(&hs, A.S_, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaStreamSynchronize(s));
  int32_t st = hs.done ? hs.status : FEAB_NOT_CONVERGED;
  if (result) {
    result->status = st;
    result->iters = hs.iters;
    result->reliable_updates = 0;
    result->graph_launches = 0;
    result->relres = hs.relres;
    result->bnorm = hs.bnorm;
  }
  return st;
}
