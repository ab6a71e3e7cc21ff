// Batched multi-RHS Jacobi-PCG: many independent problems (a block-diagonal K), each with a
// panel of K right-hand sides, solved together.  Every RHS column runs its own CG recurrence
// (its own alpha, beta, convergence test) -- the reference's preconditioned_cg
// (iterative_solvers.py:434-481) applied column by column, as solve_static_batched
// (batched_solve.py:105-164) applies one factorisation to many columns -- while the matrix is
// read once per step for all columns of a problem (SpMM over the panel).
//
// One step is three kernels: P (P = M R + beta P for problems with a pending direction), A
// (SpMM AP = K P and the per-column p.Ap, or the FP64 residual in a reliable step) and B (X, R,
// per-column r.r and r.z, convergence, beta).  The preconditioned residual Z = M R (Jacobi) is
// never stored: P and B form it from R and the inverse diagonal where they need it.
//
// Layout: vectors are row-major panels n x K (K = panel width, a power of two <= 64);
// problem p owns a contiguous row range and a contiguous range of node row groups.  Work is
// cut into items of <= 64 groups of one problem; a block processes items (grid-stride), and
// reductions are per item then per problem: the last block to finish an item of problem p
// (a per-problem ticket) reduces p's item partials in a fixed order, so results are
// deterministic.  Converged problems are skipped; the host polls a "problems remaining"
// counter one CUDA-graph chunk behind.
//
// Precisions: FEAB_PREC_FP64 (reference recurrence) and FEAB_PREC_MIXED (SpMM on 7-byte values,
// 44-bit mantissas, in difference form with FP64 vectors; per problem, an FP64 residual replacement with the
// FP64 values whenever a column's residual dropped by reliable_delta; convergence on the FP64
// residual).
#include <algorithm>
#include <cmath>
#include "feab_common.cuh"
#include "feab_graph.cuh"

namespace feab {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kModeCG = 0;
constexpr int kModeReliable = 1;

struct ProbState {  // per problem
  int32_t mode, pending, psel, done, status, iters, reliable, last_reliable;
  uint32_t ticket_a, ticket_b;
};

// Mixed: fewest CG steps between two FP64 residual replacements of a problem, unless every
// unconverged column is ready for one (a replacement is an FP64 SpMM over the whole panel).
constexpr int kMinReliableGap = 32;

struct ColState {  // per (problem, column)
  double bnorm, rz_old, rz_prev, alpha, beta, rr, relres, rmax;
  int32_t active, iters, converged, pad;
};

struct BArgs {
  int32_t n, n_groups, n_problems, n_items, k;
  const int32_t* row_ptr;
  const int32_t* col_idx;
  const int32_t* group_ptr;
  const double* vals64;
  const uint32_t* vhi;
  const uint16_t* vlo;
  const uint8_t* vlo2;
  const int32_t* tcol;
  const uint8_t* gmask;
  const double* S;
  const int32_t* goff;
  const int32_t* voff;
  const double* dinv;
  const int32_t* item_problem;
  const int32_t* item_g0;
  const int32_t* item_g1;
  const int32_t* prob_items;
  const int32_t* prob_cols;
  const double* B;   // n x k
  double* X;         // n x k
  double *R, *P0, *AP;
  double* part;      // n_items x 2k
  ProbState* ps;
  ColState* cs;
  int32_t* remaining;
  double tol, delta;
  int32_t maxiter;
};

// True in the block that completes the last of problem p's n_items_p work items; `count` items
// are completed by this call.
__device__ __forceinline__ bool last_of_problem(uint32_t* ticket, int n_items_p, int count = 1) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(ticket, (uint32_t)count) == (uint32_t)(n_items_p - count));
  __syncthreads();
  return last;
}

// The vector passes P and B take runs of up to kBRun consecutive work items of one problem as
// one contiguous row range (the items of a problem cover consecutive row groups), which cuts
// their per-item block reductions and tickets; the SpMM keeps the finer items for its balance.
#ifndef FEAB_BLOCK_BRUN
#define FEAB_BLOCK_BRUN 4
#endif
constexpr int kBRun = FEAB_BLOCK_BRUN;

// Block-wide per-column sums: thread t contributes v to column t % K (blockDim multiple of K).
template <int K>
__device__ __forceinline__ void block_col_sums(double v, double* sm) {
  sm[threadIdx.x] = v;
  __syncthreads();
  for (int s = kThreads / 2; s >= K; s >>= 1) {
    if (threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
    __syncthreads();
  }
}

// A difference-form value from its three stored parts (44 mantissa bits).
__device__ __forceinline__ double dec56(uint32_t hi, uint32_t lo, uint32_t lo2) {
  return __longlong_as_double((long long)(((unsigned long long)hi << 32) | ((unsigned long long)(lo & 0xffffu) << 16) |
                                          ((unsigned long long)(lo2 & 0xffu) << 8)));
}

// A warp's staging area for one row group's columns and values (FP64, decoded from the 56-bit
// form for the difference operator), filled with coalesced loads before the SpMM reads them as
// broadcasts; groups longer than kStageCols are staged in pieces.
constexpr int kStageCols = 128;
// matrix columns whose panel rows a lane gathers before using any
#ifndef FEAB_BLOCK_UNROLL
#define FEAB_BLOCK_UNROLL 8
#endif
constexpr int kUnroll = FEAB_BLOCK_UNROLL;
// 1: the vector pass moves two adjacent panel columns per 16-byte access
#ifndef FEAB_BLOCK_VECB
#define FEAB_BLOCK_VECB 1
#endif
// column pairs per thread and trip of the vector pass (loads in flight before any store)
#ifndef FEAB_BLOCK_VECU
#define FEAB_BLOCK_VECU 4
#endif
constexpr int kVecU = FEAB_BLOCK_VECU;
// minimum resident CTAs per SM of the SpMM kernel (register budget)
#ifndef FEAB_BLOCK_MINB
#define FEAB_BLOCK_MINB 2
#endif
// gathers in flight per lane in the FP64 SpMM (the mixed one keeps kUnroll: at 16 its decode and
// own-node term push it past the 128 registers of two CTAs per SM); measured at 128x32x32 with
// 64 columns: 1078 -> 1003 us per FP64 step
constexpr int kUnrollFp64 = 16;
static_assert(kStageCols % kUnrollFp64 == 0 && kStageCols % kUnroll == 0, "vector reads stay inside the stage");

struct __align__(16) GroupStage {
  int col[kStageCols];
  double val[3][kStageCols];
};
// 1: with one sub-warp per warp (panels of 32 or more columns) the SpMM reads the staged
// columns and values as 16-byte broadcasts (4 columns / 2 values per shared-memory load)
#ifndef FEAB_BLOCK_VLDS
#define FEAB_BLOCK_VLDS 1
#endif

// Panel column of accumulator q of lane-in-sub-warp cl: a 64-wide panel gives each lane two
// adjacent columns (one 16-byte gather per panel row), narrower panels one column per lane.
template <int K>
__device__ __forceinline__ int panel_col(int cl, int q) {
  return K >= 64 ? 2 * cl + q : cl + 32 * q;
}

// The lane's CPL values of panel row j of src (n x K, row major; 16-byte aligned when K = 64).
template <int K>
__device__ __forceinline__ void gather_row(const double* __restrict__ src, int j, int cl,
                                           double (&v)[K >= 32 ? K / 32 : 1]) {
  if constexpr (K >= 64) {
    const double2 t = __ldg(reinterpret_cast<const double2*>(src + (int64_t)j * K) + cl);
    v[0] = t.x;
    v[1] = t.y;
  } else {
    v[0] = __ldg(src + (int64_t)j * K + cl);
  }
}

// SpMM for one row group: acc[row][q] = (K src)[row][panel_col(cl, q)].
// Lanes are split into MPW = max(1, 32/K) sub-warps, each walking every MPW-th matrix column;
// a lane covers CPL = max(1, K/32) panel columns.
template <int K, bool DIFF, int U = kUnroll>
__device__ __forceinline__ void group_spmm(const BArgs& A, int g, int lane, GroupStage& st,
                                           const double* __restrict__ src,
                                           double (&acc)[3][K >= 32 ? K / 32 : 1]) {
  constexpr int CPL = K >= 32 ? K / 32 : 1;
  constexpr int MPW = K >= 32 ? 1 : 32 / K;
  constexpr int LW = K >= 32 ? 32 : K;  // lanes per sub-warp
  const int sub = lane / LW, cl = lane % LW;
  const int r0 = A.group_ptr[g], f = A.group_ptr[g + 1] - r0;
  // plain: the CSR rows; difference form: the group's padded off-node columns and values
  const int s0 = DIFF ? A.voff[g] : A.row_ptr[r0];
  const int c0 = DIFF ? A.goff[g] : 0;
  const int len = DIFF ? A.goff[g + 1] - c0 : A.row_ptr[r0 + 1] - s0;
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int q = 0; q < CPL; ++q) acc[k][q] = 0.0;
  double xs[3][CPL];
  if (DIFF) {
    const int mask = A.gmask[g];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      if ((mask >> j) & 1) {
        gather_row<K>(src, r0 + __popc(mask & ((1 << j) - 1)), cl, xs[j]);
      } else {
#pragma unroll
        for (int q = 0; q < CPL; ++q) xs[j][q] = 0.0;
      }
    }
  }
  for (int cb = 0; cb < len; cb += kStageCols) {
    const int nc = min(kStageCols, len - cb);
    if (!DIFF) {
      for (int m = lane; m < nc; m += 32) {
        st.col[m] = __ldg(A.col_idx + s0 + cb + m);
#pragma unroll
        for (int k = 0; k < 3; ++k) st.val[k][m] = k < f ? __ldg(A.vals64 + s0 + k * len + cb + m) : 0.0;
      }
    } else {
      // the difference-form operator is packed in 4-column quads (group offsets and lengths are
      // multiples of 4): one 16-byte column load and, per row, a 16 + 8-byte value load per quad
      for (int mq = lane; mq < (nc >> 2); mq += 32) {
        const int m = 4 * mq;
        const uint4 tq = __ldg(reinterpret_cast<const uint4*>(A.tcol + c0 + cb + m));
        st.col[m] = (int)tq.x;
        st.col[m + 1] = (int)tq.y;
        st.col[m + 2] = (int)tq.z;
        st.col[m + 3] = (int)tq.w;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          if (k < f) {
            const uint4 h = __ldg(reinterpret_cast<const uint4*>(A.vhi + s0 + k * len + cb + m));
            const uint2 l = __ldg(reinterpret_cast<const uint2*>(A.vlo + s0 + k * len + cb + m));
            const uint32_t l2 = __ldg(reinterpret_cast<const uint32_t*>(A.vlo2 + s0 + k * len + cb + m));
            st.val[k][m] = dec56(h.x, l.x, l2);
            st.val[k][m + 1] = dec56(h.y, l.x >> 16, l2 >> 8);
            st.val[k][m + 2] = dec56(h.z, l.y, l2 >> 16);
            st.val[k][m + 3] = dec56(h.w, l.y >> 16, l2 >> 24);
          } else {
            st.val[k][m] = st.val[k][m + 1] = st.val[k][m + 2] = st.val[k][m + 3] = 0.0;
          }
        }
      }
    }
    __syncwarp();
    if constexpr (MPW == 1 && FEAB_BLOCK_VLDS && U % 4 == 0) {
      // m0 is a multiple of U, so the vector reads stay inside the kStageCols-entry stage
      // (entries past nc are read but not used)
      for (int m0 = 0; m0 < nc; m0 += U) {
        unsigned t[U];
        double xv[U][CPL];
#pragma unroll
        for (int u4 = 0; u4 < U / 4; ++u4) {
          const int4 tq = *reinterpret_cast<const int4*>(&st.col[m0 + 4 * u4]);
          t[4 * u4] = (unsigned)tq.x;
          t[4 * u4 + 1] = (unsigned)tq.y;
          t[4 * u4 + 2] = (unsigned)tq.z;
          t[4 * u4 + 3] = (unsigned)tq.w;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (m0 + u < nc) {
            gather_row<K>(src, (int)(DIFF ? (t[u] & 0x3fffffffu) : t[u]), cl, xv[u]);
          } else {
#pragma unroll
            for (int q = 0; q < CPL; ++q) xv[u][q] = 0.0;
          }
        }
#pragma unroll
        for (int u2 = 0; u2 < U / 2; ++u2) {
          if (m0 + 2 * u2 >= nc) break;
          const double2 w0 = *reinterpret_cast<const double2*>(&st.val[0][m0 + 2 * u2]);
          const double2 w1 = *reinterpret_cast<const double2*>(&st.val[1][m0 + 2 * u2]);
          const double2 w2 = *reinterpret_cast<const double2*>(&st.val[2][m0 + 2 * u2]);
          // a column past nc has xv = 0 but a stale value: skip it rather than form 0 * stale
          const bool two = m0 + 2 * u2 + 1 < nc;
#pragma unroll
          for (int q = 0; q < CPL; ++q) {
            const double d = xv[2 * u2][q];
            acc[0][q] = fma(w0.x, d, acc[0][q]);
            acc[1][q] = fma(w1.x, d, acc[1][q]);
            acc[2][q] = fma(w2.x, d, acc[2][q]);
          }
          if (two) {
#pragma unroll
            for (int q = 0; q < CPL; ++q) {
              const double d = xv[2 * u2 + 1][q];
              acc[0][q] = fma(w0.y, d, acc[0][q]);
              acc[1][q] = fma(w1.y, d, acc[1][q]);
              acc[2][q] = fma(w2.y, d, acc[2][q]);
            }
          }
        }
      }
    } else
    for (int m0 = sub; m0 < nc; m0 += MPW * U) {
      unsigned t[U];
      double xv[U][CPL];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int m = m0 + u * MPW;
        t[u] = m < nc ? (unsigned)st.col[m] : 0u;
        if (m < nc) {
          gather_row<K>(src, (int)(DIFF ? (t[u] & 0x3fffffffu) : t[u]), cl, xv[u]);
        } else {
#pragma unroll
          for (int q = 0; q < CPL; ++q) xv[u][q] = 0.0;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int m = m0 + u * MPW;
        if (m >= nc) break;
        const double w0 = st.val[0][m], w1 = st.val[1][m], w2 = st.val[2][m];
#pragma unroll
        for (int q = 0; q < CPL; ++q) {
          // difference form as sum w x_b + T x_a (T folded into S at build time); padding
          // columns carry value 0
          const double d = xv[u][q];
          acc[0][q] = fma(w0, d, acc[0][q]);
          acc[1][q] = fma(w1, d, acc[1][q]);
          acc[2][q] = fma(w2, d, acc[2][q]);
        }
      }
    }
    __syncwarp();
  }
  // combine the sub-warps (lanes with equal cl)
#pragma unroll
  for (int o = LW; o < 32; o <<= 1)
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int q = 0; q < CPL; ++q) acc[k][q] += __shfl_xor_sync(FEAB_FULL_MASK, acc[k][q], o);
  if (DIFF) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (k < f) {
        const double s0v = A.S[(int64_t)(r0 + k) * 3 + 0], s1v = A.S[(int64_t)(r0 + k) * 3 + 1],
                     s2v = A.S[(int64_t)(r0 + k) * 3 + 2];
#pragma unroll
        for (int q = 0; q < CPL; ++q) acc[k][q] += s0v * xs[0][q] + s1v * xs[1][q] + s2v * xs[2][q];
      }
    }
  }
}

// ---------------------------------------------------------------- pipelined group staging
// 1: in the SpMM of step A (panels of 32 or 64 columns), a warp copies the next row group's
// columns and values into shared memory with cp.async while it gathers and multiplies the current
// one (two raw stages per warp, dynamic shared memory), so the staging latency is off the
// critical path.  The difference form's 56-bit values are copied as stored and decoded when read.
#ifndef FEAB_BLOCK_PIPE
#define FEAB_BLOCK_PIPE 0
#endif

struct __align__(16) RawStage {  // the same size as GroupStage, which it stands in for
  int col[kStageCols];
  union {
    double v64[3][kStageCols];
    struct {
      uint32_t hi[3][kStageCols];
      uint16_t lo[3][kStageCols];
      uint8_t lo2[3][kStageCols];
    } d;
  };
};
static_assert(sizeof(RawStage) == sizeof(GroupStage), "a raw stage doubles as a synchronous stage");

__device__ __forceinline__ uint32_t shared_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(shared_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(shared_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(shared_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Start the copies of group g's columns and values into st; false (nothing issued) when the
// group does not fit one stage.  Rows the group does not have are zero-filled.
template <bool DIFF>
__device__ __forceinline__ bool stage_issue(const BArgs& A, int g, int lane, RawStage& st) {
  const int r0 = A.group_ptr[g], f = A.group_ptr[g + 1] - r0;
  if (DIFF) {
    const int c0 = A.goff[g], s0 = A.voff[g], len = A.goff[g + 1] - c0;
    if (len > kStageCols) return false;
    for (int mq = lane; mq < (len >> 2); mq += 32) {
      const int m = 4 * mq;
      cp_async16(&st.col[m], A.tcol + c0 + m);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (k < f) {
          cp_async16(&st.d.hi[k][m], A.vhi + s0 + k * len + m);
          cp_async8(&st.d.lo[k][m], A.vlo + s0 + k * len + m);
          cp_async4(&st.d.lo2[k][m], A.vlo2 + s0 + k * len + m);
        } else {
          *reinterpret_cast<uint4*>(&st.d.hi[k][m]) = make_uint4(0u, 0u, 0u, 0u);
          *reinterpret_cast<uint2*>(&st.d.lo[k][m]) = make_uint2(0u, 0u);
          *reinterpret_cast<uint32_t*>(&st.d.lo2[k][m]) = 0u;
        }
      }
    }
  } else {
    const int s0 = A.row_ptr[r0], len = A.row_ptr[r0 + 1] - s0;
    if (len > kStageCols) return false;
    for (int m = lane; m < len; m += 32) {
      cp_async4(&st.col[m], A.col_idx + s0 + m);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (k < f) cp_async8(&st.v64[k][m], A.vals64 + s0 + k * len + m);
        else st.v64[k][m] = 0.0;
      }
    }
  }
  cp_async_commit();
  return true;
}

// The SpMM of group g from a stage filled by stage_issue (one sub-warp, K >= 32).
template <int K, bool DIFF>
__device__ __forceinline__ void group_spmm_staged(const BArgs& A, int g, int lane, const RawStage& st,
                                                  const double* __restrict__ src, double (&acc)[3][K / 32]) {
  constexpr int CPL = K / 32;
  const int r0 = A.group_ptr[g], f = A.group_ptr[g + 1] - r0;
  const int nc = DIFF ? A.goff[g + 1] - A.goff[g] : A.row_ptr[r0 + 1] - A.row_ptr[r0];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int q = 0; q < CPL; ++q) acc[k][q] = 0.0;
  double xs[3][CPL];
  if (DIFF) {
    const int mask = A.gmask[g];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      if ((mask >> j) & 1) {
        gather_row<K>(src, r0 + __popc(mask & ((1 << j) - 1)), lane, xs[j]);
      } else {
#pragma unroll
        for (int q = 0; q < CPL; ++q) xs[j][q] = 0.0;
      }
    }
  }
  for (int m0 = 0; m0 < nc; m0 += kUnroll) {
    unsigned t[kUnroll];
    double xv[kUnroll][CPL];
#pragma unroll
    for (int u4 = 0; u4 < kUnroll / 4; ++u4) {
      const int4 tq = *reinterpret_cast<const int4*>(&st.col[m0 + 4 * u4]);
      t[4 * u4] = (unsigned)tq.x;
      t[4 * u4 + 1] = (unsigned)tq.y;
      t[4 * u4 + 2] = (unsigned)tq.z;
      t[4 * u4 + 3] = (unsigned)tq.w;
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      if (m0 + u < nc) {
        gather_row<K>(src, (int)(DIFF ? (t[u] & 0x3fffffffu) : t[u]), lane, xv[u]);
      } else {
#pragma unroll
        for (int q = 0; q < CPL; ++q) xv[u][q] = 0.0;
      }
    }
#pragma unroll
    for (int u2 = 0; u2 < kUnroll / 2; ++u2) {
      const int m = m0 + 2 * u2;
      if (m >= nc) break;
      double2 w[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (DIFF) {
          const uint2 h = *reinterpret_cast<const uint2*>(&st.d.hi[k][m]);
          const uint32_t l = *reinterpret_cast<const uint32_t*>(&st.d.lo[k][m]);
          const uint32_t l2 = *reinterpret_cast<const uint16_t*>(&st.d.lo2[k][m]);
          w[k] = make_double2(dec56(h.x, l, l2), dec56(h.y, l >> 16, l2 >> 8));
        } else {
          w[k] = *reinterpret_cast<const double2*>(&st.v64[k][m]);
        }
      }
      const bool two = m + 1 < nc;  // a column past nc has xv = 0 but a stale value
#pragma unroll
      for (int q = 0; q < CPL; ++q) {
        const double d = xv[2 * u2][q];
        acc[0][q] = fma(w[0].x, d, acc[0][q]);
        acc[1][q] = fma(w[1].x, d, acc[1][q]);
        acc[2][q] = fma(w[2].x, d, acc[2][q]);
      }
      if (two) {
#pragma unroll
        for (int q = 0; q < CPL; ++q) {
          const double d = xv[2 * u2 + 1][q];
          acc[0][q] = fma(w[0].y, d, acc[0][q]);
          acc[1][q] = fma(w[1].y, d, acc[1][q]);
          acc[2][q] = fma(w[2].y, d, acc[2][q]);
        }
      }
    }
  }
  if (DIFF) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (k < f) {
        const double s0v = A.S[(int64_t)(r0 + k) * 3 + 0], s1v = A.S[(int64_t)(r0 + k) * 3 + 1],
                     s2v = A.S[(int64_t)(r0 + k) * 3 + 2];
#pragma unroll
        for (int q = 0; q < CPL; ++q) acc[k][q] += s0v * xs[0][q] + s1v * xs[1][q] + s2v * xs[2][q];
      }
    }
  }
}

// setup: R = B - 0 (x0 = 0), P = M R, per column ||b||, r.z; columns beyond the problem's
// RHS count are inactive from the start.
template <int K>
__global__ void __launch_bounds__(kThreads) k_bsetup(BArgs A) {
  __shared__ double sm[2][kThreads];
  const int c = threadIdx.x % K;
  for (int it = blockIdx.x; it < A.n_items; it += gridDim.x) {
    const int p = A.item_problem[it];
    const int r0 = A.group_ptr[A.item_g0[it]], r1 = A.group_ptr[A.item_g1[it]];
    double bb = 0.0, rz = 0.0;
    for (int64_t idx = (int64_t)r0 * K + threadIdx.x; idx < (int64_t)r1 * K; idx += kThreads) {
      const int i = (int)(idx / K);
      const double bi = A.B[idx];
      const double zi = A.dinv[i] * bi;
      A.R[idx] = bi;
      A.P0[idx] = zi;
      A.X[idx] = 0.0;
      bb += bi * bi;
      rz += bi * zi;
    }
    block_col_sums<K>(bb, sm[0]);
    block_col_sums<K>(rz, sm[1]);
    if (threadIdx.x < K) {
      A.part[(int64_t)it * 2 * K + c] = sm[0][c];
      A.part[(int64_t)it * 2 * K + K + c] = sm[1][c];
    }
    const int i0 = A.prob_items[p], n_it = A.prob_items[p + 1] - i0;
    if (last_of_problem(&A.ps[p].ticket_a, n_it)) {
      if (threadIdx.x < K) {
        double s0 = 0.0, s1 = 0.0;
        for (int q = 0; q < n_it; ++q) {
          s0 += __ldcg(&A.part[(int64_t)(i0 + q) * 2 * K + c]);
          s1 += __ldcg(&A.part[(int64_t)(i0 + q) * 2 * K + K + c]);
        }
        ColState& C = A.cs[(int64_t)p * K + c];
        double bn = sqrt(s0);
        if (bn == 0.0) bn = 1.0;
        C.bnorm = bn;
        C.rz_old = s1;
        C.rz_prev = s1;
        C.rr = s0;
        C.rmax = sqrt(s0);
        C.relres = sqrt(s0) / bn;
        C.alpha = C.beta = 0.0;
        C.iters = 0;
        C.active = c < A.prob_cols[p] ? 1 : 0;
        C.converged = (!C.active || C.relres < A.tol) ? 1 : 0;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        ProbState& P = A.ps[p];
        int all = 1;
        for (int q = 0; q < K; ++q) all &= A.cs[(int64_t)p * K + q].converged;
        P.ticket_a = 0;
        P.mode = kModeCG;
        P.pending = 0;
        P.psel = 0;
        P.iters = 0;
        P.reliable = 0;
        P.last_reliable = 0;
        P.status = FEAB_OK;
        P.done = all;
        if (all) atomicSub(A.remaining, 1);
      }
    }
    __syncthreads();
  }
}

// Step A: AP = K P (P updated by k_bstep_p; or, in a reliable step, R = B - K64 X);
// per-column partial p.Ap (or r.r).
template <int K, bool MIXED>
__global__ void __launch_bounds__(kThreads, FEAB_BLOCK_MINB) k_bstep_a(BArgs A) {
  constexpr int CPL = K >= 32 ? K / 32 : 1;
  constexpr int LW = K >= 32 ? 32 : K;
  constexpr bool PIPE = FEAB_BLOCK_PIPE && K >= 32;
  __shared__ double sm[kWarps][K];
  __shared__ GroupStage stage[PIPE ? 1 : kWarps];
  extern __shared__ __align__(16) unsigned char dyn_stage[];  // PIPE: two raw stages per warp
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  RawStage* rs = reinterpret_cast<RawStage*>(dyn_stage) + 2 * w;
  for (int it = blockIdx.x; it < A.n_items; it += gridDim.x) {
    const int p = A.item_problem[it];
    const ProbState P = A.ps[p];
    if (P.done) continue;
    const bool reliable = MIXED && P.mode == kModeReliable;
    const bool diff = MIXED && !reliable;
    const double* __restrict__ po = A.P0;  // the direction, already updated by k_bstep_p
    const double* __restrict__ src = reliable ? A.X : po;
    double part[CPL];
#pragma unroll
    for (int q = 0; q < CPL; ++q) part[q] = 0.0;
    const int g1 = A.item_g1[it];
    int buf = 0;
    bool staged = false;
    if constexpr (PIPE) {
      const int g = A.item_g0[it] + w;
      if (g < g1) staged = diff ? stage_issue<true>(A, g, lane, rs[0]) : stage_issue<false>(A, g, lane, rs[0]);
    }
    for (int g = A.item_g0[it] + w; g < g1; g += kWarps) {
      double acc[3][CPL];
      if constexpr (PIPE) {
        // group g's copies have landed; start group g + kWarps's into the other stage
        cp_async_wait_all();
        __syncwarp();
        bool staged_next = false;
        const int gn = g + kWarps;
        if (gn < g1)
          staged_next = diff ? stage_issue<true>(A, gn, lane, rs[buf ^ 1]) : stage_issue<false>(A, gn, lane, rs[buf ^ 1]);
        if (staged) {
          if (diff) group_spmm_staged<K, true>(A, g, lane, rs[buf], src, acc);
          else group_spmm_staged<K, false>(A, g, lane, rs[buf], src, acc);
        } else {
          GroupStage& gs = *reinterpret_cast<GroupStage*>(&rs[buf]);
          if (diff) group_spmm<K, MIXED>(A, g, lane, gs, src, acc);
          else group_spmm<K, false>(A, g, lane, gs, src, acc);
        }
        __syncwarp();  // every lane is done with rs[buf] before it is refilled
        staged = staged_next;
        buf ^= 1;
      } else if constexpr (MIXED) {
        if (!diff) group_spmm<K, false>(A, g, lane, stage[w], src, acc);
        else group_spmm<K, true>(A, g, lane, stage[w], po, acc);
      } else {
        group_spmm<K, false, kUnrollFp64>(A, g, lane, stage[w], po, acc);
      }
      if (lane < LW) {
        const int r0 = A.group_ptr[g], f = A.group_ptr[g + 1] - r0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          if (k >= f) break;
#pragma unroll
          for (int q = 0; q < CPL; ++q) {
            const int64_t idx = (int64_t)(r0 + k) * K + panel_col<K>(lane, q);
            if (reliable) {
              const double ri = A.B[idx] - acc[k][q];
              A.R[idx] = ri;
              part[q] += ri * ri;
            } else {
              const double pv = po[idx];
              A.AP[idx] = acc[k][q];
              part[q] += pv * acc[k][q];
            }
          }
        }
      }
    }
    if (lane < LW) {
#pragma unroll
      for (int q = 0; q < CPL; ++q) sm[w][panel_col<K>(lane, q)] = part[q];
    }
    __syncthreads();
    if (threadIdx.x < K) {
      double s = 0.0;
      for (int q = 0; q < kWarps; ++q) s += sm[q][threadIdx.x];
      A.part[(int64_t)it * 2 * K + threadIdx.x] = s;
    }
    const int i0 = A.prob_items[p], n_it = A.prob_items[p + 1] - i0;
    if (last_of_problem(&A.ps[p].ticket_a, n_it)) {
      if (threadIdx.x < K) {
        const int c = threadIdx.x;
        double s = 0.0;
        for (int q = 0; q < n_it; ++q) s += __ldcg(&A.part[(int64_t)(i0 + q) * 2 * K + c]);
        ColState& C = A.cs[(int64_t)p * K + c];
        if (reliable) {
          C.rr = s;
        } else {
          C.alpha = 0.0;
          if (C.active && !C.converged) {
            if (!(s > 0.0)) atomicCAS(&A.ps[p].status, FEAB_OK, FEAB_NOT_SPD);
            else C.alpha = C.rz_old / s;
          }
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        ProbState& Pm = A.ps[p];
        Pm.ticket_a = 0;
        if (!reliable) {
          Pm.pending = 0;
          if (Pm.status != FEAB_OK) {
            Pm.done = 1;
            atomicSub(A.remaining, 1);
          }
        }
      }
    }
    __syncthreads();
  }
}

// Direction update P = M R + beta P (in place, per column beta; frozen columns have beta = 0,
// so P = M R) for the problems whose new direction is pending.
template <int K>
__global__ void __launch_bounds__(kThreads) k_bstep_p(BArgs A) {
  double* __restrict__ P0 = A.P0;
  const double* __restrict__ R = A.R;
  for (int ru = blockIdx.x; ru * kBRun < A.n_items; ru += gridDim.x) {
   const int it_end = min(A.n_items, (ru + 1) * kBRun);
   for (int it = ru * kBRun, it2 = it; it < it_end; it = it2) {
    const int p = A.item_problem[it];
    for (it2 = it + 1; it2 < it_end && A.item_problem[it2] == p; ++it2) {
    }
    const ProbState P = A.ps[p];
    if (P.done || !P.pending) continue;
    const int r0 = A.group_ptr[A.item_g0[it]], r1 = A.group_ptr[A.item_g1[it2 - 1]];
    if constexpr (K >= 2) {
      // two adjacent columns per thread with 16-byte accesses, four pairs per trip
      const int c2 = 2 * (threadIdx.x % (K / 2));
      const double b0 = A.cs[(int64_t)p * K + c2].beta, b1 = A.cs[(int64_t)p * K + c2 + 1].beta;
      const int64_t q0 = (int64_t)r0 * (K / 2) + threadIdx.x, q1 = (int64_t)r1 * (K / 2);
      double2* __restrict__ P2 = reinterpret_cast<double2*>(P0);
      const double2* __restrict__ R2 = reinterpret_cast<const double2*>(R);
      for (int64_t q = q0; q < q1; q += 4 * kThreads) {
        double2 rv[4], pv[4];
        double dv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int64_t e = q + (int64_t)u * kThreads;
          const bool ok = e < q1;
          rv[u] = ok ? R2[e] : make_double2(0.0, 0.0);
          pv[u] = ok ? P2[e] : make_double2(0.0, 0.0);
          dv[u] = ok ? __ldg(A.dinv + e / (K / 2)) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int64_t e = q + (int64_t)u * kThreads;
          if (e < q1) P2[e] = make_double2(dv[u] * rv[u].x + b0 * pv[u].x, dv[u] * rv[u].y + b1 * pv[u].y);
        }
      }
    } else {
      const double beta = A.cs[(int64_t)p].beta;
      const int64_t e0 = (int64_t)r0 + threadIdx.x, e1 = (int64_t)r1;
      for (int64_t idx = e0; idx < e1; idx += 4 * kThreads) {
        double rv[4], pv[4], dv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int64_t e = idx + (int64_t)u * kThreads;
          rv[u] = e < e1 ? R[e] : 0.0;
          pv[u] = e < e1 ? P0[e] : 0.0;
          dv[u] = e < e1 ? __ldg(A.dinv + e) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int64_t e = idx + (int64_t)u * kThreads;
          if (e < e1) P0[e] = dv[u] * rv[u] + beta * pv[u];
        }
      }
    }
   }
  }
}

// Step B: X += alpha P, R -= alpha AP (CG step; a reliable step leaves both); per column r.r
// and r.z with z = M r formed on the fly; per-column convergence, beta, problem bookkeeping.
#ifndef FEAB_BLOCK_B_MINB
#define FEAB_BLOCK_B_MINB 2
#endif
template <int K, bool MIXED>
__global__ void __launch_bounds__(kThreads, FEAB_BLOCK_B_MINB) k_bstep_b(BArgs A) {
  __shared__ double sm[2][kThreads];
  __shared__ double smv[2][2 * kThreads];
  __shared__ int flag_any, flag_all;
  const int c = threadIdx.x % K;
  for (int ru = blockIdx.x; ru * kBRun < A.n_items; ru += gridDim.x) {
   const int it_end = min(A.n_items, (ru + 1) * kBRun);
   for (int it = ru * kBRun, it2 = it; it < it_end; it = it2) {
    const int p = A.item_problem[it];
    for (it2 = it + 1; it2 < it_end && A.item_problem[it2] == p; ++it2) {
    }
    const ProbState P = A.ps[p];
    if (P.done) continue;
    const bool reliable = MIXED && P.mode == kModeReliable;
    const double* __restrict__ pc = A.P0;
    double* __restrict__ X = A.X;
    double* __restrict__ R = A.R;
    const double* __restrict__ AP = A.AP;
    const int r0 = A.group_ptr[A.item_g0[it]], r1 = A.group_ptr[A.item_g1[it2 - 1]];
    if constexpr (K >= 2 && FEAB_BLOCK_VECB) {
      // two adjacent columns c2, c2 + 1 per thread with 16-byte accesses, kVecU pairs per trip,
      // every load of the trip issued before any store
      const int c2 = 2 * (threadIdx.x % (K / 2));
      const double al0 = A.cs[(int64_t)p * K + c2].alpha, al1 = A.cs[(int64_t)p * K + c2 + 1].alpha;
      double rr0 = 0.0, rr1 = 0.0, rz0 = 0.0, rz1 = 0.0;
      const int64_t q0 = (int64_t)r0 * (K / 2) + threadIdx.x, q1 = (int64_t)r1 * (K / 2);
      const double2* __restrict__ P2 = reinterpret_cast<const double2*>(pc);
      const double2* __restrict__ AP2 = reinterpret_cast<const double2*>(AP);
      double2* __restrict__ X2 = reinterpret_cast<double2*>(X);
      double2* __restrict__ R2 = reinterpret_cast<double2*>(R);
      for (int64_t q = q0; q < q1; q += kVecU * kThreads) {
        double2 xv[kVecU], pv[kVecU], rv[kVecU], av[kVecU];
        double dv[kVecU];
#pragma unroll
        for (int u = 0; u < kVecU; ++u) {
          const int64_t e = q + (int64_t)u * kThreads;
          const bool ok = e < q1;
          rv[u] = ok ? R2[e] : make_double2(0.0, 0.0);
          dv[u] = ok ? __ldg(A.dinv + e / (K / 2)) : 0.0;
          if (!reliable) {
            xv[u] = ok ? X2[e] : make_double2(0.0, 0.0);
            pv[u] = ok ? P2[e] : make_double2(0.0, 0.0);
            av[u] = ok ? AP2[e] : make_double2(0.0, 0.0);
          }
        }
#pragma unroll
        for (int u = 0; u < kVecU; ++u) {
          const int64_t e = q + (int64_t)u * kThreads;
          if (e >= q1) break;
          double ri0 = rv[u].x, ri1 = rv[u].y;
          if (!reliable) {
            X2[e] = make_double2(xv[u].x + al0 * pv[u].x, xv[u].y + al1 * pv[u].y);
            ri0 = rv[u].x - al0 * av[u].x;
            ri1 = rv[u].y - al1 * av[u].y;
            R2[e] = make_double2(ri0, ri1);
          }
          const double zi0 = dv[u] * ri0, zi1 = dv[u] * ri1;
          rr0 += ri0 * ri0;
          rr1 += ri1 * ri1;
          rz0 += ri0 * zi0;
          rz1 += ri1 * zi1;
        }
      }
      // per-column sums: entry 2t + h holds column (2t + h) % K; fold entries s apart (s >= K)
      smv[0][2 * threadIdx.x] = rr0;
      smv[0][2 * threadIdx.x + 1] = rr1;
      smv[1][2 * threadIdx.x] = rz0;
      smv[1][2 * threadIdx.x + 1] = rz1;
      for (int sh = kThreads; sh >= K; sh >>= 1) {
        __syncthreads();
        if (threadIdx.x < sh) {
          smv[0][threadIdx.x] += smv[0][threadIdx.x + sh];
          smv[1][threadIdx.x] += smv[1][threadIdx.x + sh];
        }
      }
      __syncthreads();
      if (threadIdx.x < K) {
        A.part[(int64_t)it * 2 * K + c] = smv[0][c];
        A.part[(int64_t)it * 2 * K + K + c] = smv[1][c];
        for (int z = it + 1; z < it2; ++z) A.part[(int64_t)z * 2 * K + c] = A.part[(int64_t)z * 2 * K + K + c] = 0.0;
      }
    } else {
      const double alpha = A.cs[(int64_t)p * K + c].alpha;
      double rr = 0.0, rz = 0.0;
      // 4 elements of this thread's column per trip (kThreads is a multiple of K), every load of
      // the trip issued before any store
      const int64_t e0 = (int64_t)r0 * K + threadIdx.x, e1 = (int64_t)r1 * K;
      for (int64_t idx = e0; idx < e1; idx += 4 * kThreads) {
        double xv[4], pv[4], rv[4], av[4], dv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int64_t e = idx + (int64_t)u * kThreads;
          const bool ok = e < e1;
          rv[u] = ok ? R[e] : 0.0;
          dv[u] = ok ? __ldg(A.dinv + e / K) : 0.0;
          if (!reliable) {
            xv[u] = ok ? X[e] : 0.0;
            pv[u] = ok ? pc[e] : 0.0;
            av[u] = ok ? AP[e] : 0.0;
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int64_t e = idx + (int64_t)u * kThreads;
          if (e >= e1) break;
          double ri = rv[u];
          if (!reliable) {
            X[e] = xv[u] + alpha * pv[u];
            ri = rv[u] - alpha * av[u];
            R[e] = ri;
          }
          const double zi = dv[u] * ri;
          rr += ri * ri;
          rz += ri * zi;
        }
      }
      block_col_sums<K>(rr, sm[0]);
      block_col_sums<K>(rz, sm[1]);
      if (threadIdx.x < K) {
        A.part[(int64_t)it * 2 * K + c] = sm[0][c];
        A.part[(int64_t)it * 2 * K + K + c] = sm[1][c];
        for (int z = it + 1; z < it2; ++z) A.part[(int64_t)z * 2 * K + c] = A.part[(int64_t)z * 2 * K + K + c] = 0.0;
      }
    }
    const int i0 = A.prob_items[p], n_it = A.prob_items[p + 1] - i0;
    if (last_of_problem(&A.ps[p].ticket_b, n_it, it2 - it)) {
      // mixed: a column is ready for an FP64 residual replacement once its recursive residual
      // dropped by delta since the last one or reached tol; the problem replaces when a column
      // is ready and kMinReliableGap steps have passed, or when every unconverged column is ready
      if (threadIdx.x == 0) {
        flag_any = 0;
        flag_all = 1;
      }
      __syncthreads();
      if (threadIdx.x < K) {
        double s0 = 0.0, s1 = 0.0;
        for (int q = 0; q < n_it; ++q) {
          s0 += __ldcg(&A.part[(int64_t)(i0 + q) * 2 * K + c]);
          s1 += __ldcg(&A.part[(int64_t)(i0 + q) * 2 * K + K + c]);
        }
        ColState& C = A.cs[(int64_t)p * K + c];
        if (C.active && !C.converged) {
          if (!reliable) C.iters += 1;
          const double rrv = reliable ? C.rr : s0;
          const double rel = sqrt(rrv) / C.bnorm;
          C.relres = rel;
          const bool conv = rel < A.tol;
          if (!MIXED || reliable) {
            if (conv) C.converged = 1;
            if (reliable) C.rmax = sqrt(rrv);
          } else if (conv || sqrt(rrv) < A.delta * C.rmax) {
            atomicOr(&flag_any, 1);
          } else {
            atomicAnd(&flag_all, 0);
          }
          if (reliable) {
            C.beta = s1 / C.rz_prev;  // r replaced the recurrence residual of the previous step
          } else {
            C.rz_prev = C.rz_old;
            C.beta = s1 / C.rz_old;
          }
          C.rz_old = s1;
        }
        if (!C.active || C.converged) C.beta = 0.0;  // frozen columns: p = z, alpha = 0
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        ProbState& Pm = A.ps[p];
        Pm.ticket_b = 0;
        if (!reliable) Pm.iters += 1;
        else Pm.reliable += 1;
        int all = 1;
        for (int q = 0; q < K; ++q) all &= A.cs[(int64_t)p * K + q].converged;
        const bool replace = flag_any && (flag_all || Pm.iters - Pm.last_reliable >= kMinReliableGap);
        if (MIXED && !reliable && replace) {
          Pm.last_reliable = Pm.iters;
          // FP64 residual replacement next; the search directions wait for it.  rz_old of the
          // columns was advanced above; it is recomputed from the replaced residual.
          Pm.mode = kModeReliable;
          Pm.pending = 0;
        } else {
          Pm.mode = kModeCG;
          Pm.pending = 1;
        }
        if (all) {
          Pm.done = 1;
          atomicSub(A.remaining, 1);
        } else if (Pm.iters >= A.maxiter) {
          Pm.done = 1;
          Pm.status = FEAB_NOT_CONVERGED;
          atomicSub(A.remaining, 1);
        }
      }
    }
    __syncthreads();
   }
  }
}

// Y = K X for a whole n x K panel (the plain CSR, FP64 values): the SpMM of step A on its own,
// one warp per node row group, grid-stride over the groups.
template <int K>
__global__ void __launch_bounds__(kThreads, FEAB_BLOCK_MINB) k_block_spmm(BArgs A, const double* __restrict__ src,
                                                                         double* __restrict__ dst) {
  constexpr int CPL = K >= 32 ? K / 32 : 1;
  constexpr int LW = K >= 32 ? 32 : K;
  __shared__ GroupStage stage[kWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int g = blockIdx.x * kWarps + w; g < A.n_groups; g += gridDim.x * kWarps) {
    double acc[3][CPL];
    group_spmm<K, false, kUnrollFp64>(A, g, lane, stage[w], src, acc);
    if (lane < LW) {
      const int r0 = A.group_ptr[g], f = A.group_ptr[g + 1] - r0;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (k >= f) break;
#pragma unroll
        for (int q = 0; q < CPL; ++q) dst[(int64_t)(r0 + k) * K + panel_col<K>(lane, q)] = acc[k][q];
      }
    }
  }
}

template <int K>
void launch_block_spmm(const BArgs& A, const double* X, double* Y, cudaStream_t s) {
  const int grid = std::max(1, std::min((A.n_groups + kWarps - 1) / kWarps, sm_count() * 8));
  k_block_spmm<K><<<grid, kThreads, 0, s>>>(A, X, Y);
}

size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

struct BLayout {
  size_t total;
  size_t o_R, o_P0, o_AP, o_part, o_ps, o_cs, o_rem;
};

BLayout blayout(int32_t n, int32_t k, int32_t n_problems, int32_t n_items) {
  BLayout L{};
  size_t off = 0;
  auto take = [&](size_t b) {
    size_t o = off;
    off += a256(b);
    return o;
  };
  const size_t panel = sizeof(double) * (size_t)n * (size_t)k;
  L.o_R = take(panel);
  L.o_P0 = take(panel);
  L.o_AP = take(panel);
  L.o_part = take(sizeof(double) * 2 * (size_t)k * (size_t)n_items);
  L.o_ps = take(sizeof(ProbState) * (size_t)n_problems);
  L.o_cs = take(sizeof(ColState) * (size_t)n_problems * (size_t)k);
  L.o_rem = take(sizeof(int32_t));
  L.total = off;
  return L;
}

template <int K>
int32_t run_block(BArgs A, int prec, int chunk, int maxiter, cudaStream_t s, int32_t* host_iters, double* host_relres,
                  int32_t* host_status) {
  const int grid = std::max(1, std::min(A.n_items, sm_count() * 4));
  const int grid_pb = std::max(1, std::min((A.n_items + kBRun - 1) / kBRun, sm_count() * 4));  // P and B runs
  cudaMemsetAsync(A.ps, 0, sizeof(ProbState) * A.n_problems, s);
  int32_t np = A.n_problems;
  cudaMemcpyAsync(A.remaining, &np, sizeof(int32_t), cudaMemcpyHostToDevice, s);
  k_bsetup<K><<<grid, kThreads, 0, s>>>(A);
  count_launches(1);
  if (cudaGetLastError() != cudaSuccess) return FEAB_CUDA_ERROR;
  static thread_local HostFlag flag;
  static thread_local GraphCache graphs;
  if (!flag.ptr) return FEAB_CUDA_ERROR;
  volatile int32_t* hflag = flag.ptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int32_t rc = FEAB_OK;
  auto fail = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == FEAB_OK) rc = FEAB_CUDA_ERROR;
    return e != cudaSuccess;
  };
  do {
    if (fail(graphs.events(ev))) break;
    const size_t smem_a = (FEAB_BLOCK_PIPE && K >= 32) ? 2 * kWarps * sizeof(RawStage) : 0;
    if (smem_a) {
      if (fail(cudaFuncSetAttribute(k_bstep_a<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_a))) break;
      if (fail(cudaFuncSetAttribute(k_bstep_a<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_a))) break;
    }
    auto record = [&](cudaStream_t cs) {
      for (int q = 0; q < chunk; ++q) {
        if (prec == FEAB_PREC_MIXED) {
          k_bstep_p<K><<<grid_pb, kThreads, 0, cs>>>(A);
          k_bstep_a<K, true><<<grid, kThreads, smem_a, cs>>>(A);
          k_bstep_b<K, true><<<grid_pb, kThreads, 0, cs>>>(A);
        } else {
          k_bstep_p<K><<<grid_pb, kThreads, 0, cs>>>(A);
          k_bstep_a<K, false><<<grid, kThreads, smem_a, cs>>>(A);
          k_bstep_b<K, false><<<grid_pb, kThreads, 0, cs>>>(A);
        }
      }
      cudaMemcpyAsync((void*)hflag, A.remaining, sizeof(int32_t), cudaMemcpyDeviceToHost, cs);
    };
    if (fail(graphs.acquire(&A, sizeof(A), topo_signature({K, prec, chunk, grid, grid_pb}), record, &exec))) break;
    // iterations and reliable steps per problem are bounded by maxiter each
    const int64_t max_launch = (2 * (int64_t)maxiter + 2 + chunk - 1) / chunk + 1;
    hflag[0] = np;
    int64_t launched = 0;
    if (fail(cudaGraphLaunch(exec, s))) break;
    if (fail(cudaEventRecord(ev[0], s))) break;
    launched = 1;
    count_launches(3 * (uint64_t)chunk);
    while (true) {
      const bool more = launched < max_launch;
      if (more) {
        if (fail(cudaGraphLaunch(exec, s))) break;
        if (fail(cudaEventRecord(ev[launched & 1], s))) break;
        ++launched;
        count_launches(3 * (uint64_t)chunk);
      }
      if (fail(cudaEventSynchronize(ev[more ? ((launched - 2) & 1) : ((launched - 1) & 1)]))) break;
      if (((volatile int32_t*)hflag)[0] <= 0 || !more) break;
    }
  } while (false);
  if (rc == FEAB_OK) fail(cudaStreamSynchronize(s));
  int32_t worst = rc;
  if (rc == FEAB_OK) {
    // per-problem / per-column results
    const int P = A.n_problems;
    ProbState* hp = (ProbState*)malloc(sizeof(ProbState) * P);
    ColState* hc = (ColState*)malloc(sizeof(ColState) * (size_t)P * K);
    if (hp && hc && cudaMemcpy(hp, A.ps, sizeof(ProbState) * P, cudaMemcpyDeviceToHost) == cudaSuccess &&
        cudaMemcpy(hc, A.cs, sizeof(ColState) * (size_t)P * K, cudaMemcpyDeviceToHost) == cudaSuccess) {
      for (int p = 0; p < P; ++p) {
        int st = hp[p].status;
        if (!hp[p].done) st = FEAB_NOT_CONVERGED;
        if (host_status) host_status[p] = st;
        if (st != FEAB_OK && worst == FEAB_OK) worst = st;
        for (int c = 0; c < K; ++c) {
          if (host_iters) host_iters[(size_t)p * K + c] = hc[(size_t)p * K + c].iters;
          if (host_relres) host_relres[(size_t)p * K + c] = hc[(size_t)p * K + c].relres;
        }
      }
    } else {
      worst = FEAB_CUDA_ERROR;
    }
    free(hp);
    free(hc);
  }
  return worst;
}

}  // namespace
}  // namespace feab

using namespace feab;

extern "C" size_t feab_block_pcg_workspace_bytes(int32_t n, int32_t k, int32_t n_problems, int32_t n_items) {
  if (n <= 0 || k <= 0 || n_problems <= 0 || n_items <= 0) return 0;
  return blayout(n, k, n_problems, n_items).total;
}

extern "C" int32_t feab_block_pcg_solve(const feab_csr* M, const feab_diff_operator* D, const feab_batch* bt,
                                        const double* dinv64, const double* B, double* X, const feab_pcg_params* prm,
                                        void* workspace, size_t workspace_bytes, int32_t* iters_out,
                                        double* relres_out, int32_t* status_out, cudaStream_t s) {
  if (!M || !bt || !dinv64 || !B || !X || !prm || !workspace || !M->group_ptr || !M->vals64) return FEAB_BAD_ARG;
  const int k = bt->k;
  if (k != 1 && k != 2 && k != 4 && k != 8 && k != 16 && k != 32 && k != 64) return FEAB_BAD_ARG;
  if (bt->n_problems <= 0 || bt->n_items <= 0 || !bt->item_problem || !bt->item_group0 || !bt->item_group1 ||
      !bt->problem_items || !bt->problem_cols)
    return FEAB_BAD_ARG;
  const int prec = prm->precision;
  if (prec != FEAB_PREC_FP64 && prec != FEAB_PREC_MIXED) return FEAB_BAD_ARG;
  if (prec == FEAB_PREC_MIXED && !D) return FEAB_BAD_ARG;
  if ((reinterpret_cast<uintptr_t>(X) & 15) != 0) return FEAB_BAD_ARG;  // 16-byte panel gathers
  // the R / P / AP panels are carved from the workspace at 256-byte offsets and are read and
  // written with 16-byte accesses by the vector passes
  if ((reinterpret_cast<uintptr_t>(workspace) & 15) != 0) return FEAB_BAD_ARG;
  if (D && (!D->tcol || !D->vhi || !D->vlo || !D->vlo2 || (reinterpret_cast<uintptr_t>(D->tcol) & 15) ||
            (reinterpret_cast<uintptr_t>(D->vhi) & 15) || (reinterpret_cast<uintptr_t>(D->vlo) & 7) ||
            (reinterpret_cast<uintptr_t>(D->vlo2) & 3)))
    return FEAB_BAD_ARG;  // 16-byte column / hi-word quads, 8-byte lo and 4-byte lo2 words
  const BLayout L = blayout(M->n, k, bt->n_problems, bt->n_items);
  if (L.total > workspace_bytes) return FEAB_BAD_ARG;
  char* w = static_cast<char*>(workspace);
  BArgs A{};
  A.n = M->n;
  A.n_groups = M->n_groups;
  A.n_problems = bt->n_problems;
  A.n_items = bt->n_items;
  A.k = k;
  A.row_ptr = M->row_ptr;
  A.col_idx = M->col_idx;
  A.group_ptr = M->group_ptr;
  A.vals64 = M->vals64;
  if (D) {
    A.vhi = D->vhi;
    A.vlo = D->vlo;
    A.vlo2 = D->vlo2;
    A.tcol = D->tcol;
    A.gmask = D->gmask;
    A.goff = D->goff;
    A.voff = D->voff;
    A.S = D->S;
  }
  A.dinv = dinv64;
  A.item_problem = bt->item_problem;
  A.item_g0 = bt->item_group0;
  A.item_g1 = bt->item_group1;
  A.prob_items = bt->problem_items;
  A.prob_cols = bt->problem_cols;
  A.B = B;
  A.X = X;
  A.R = reinterpret_cast<double*>(w + L.o_R);
  A.P0 = reinterpret_cast<double*>(w + L.o_P0);
  A.AP = reinterpret_cast<double*>(w + L.o_AP);
  A.part = reinterpret_cast<double*>(w + L.o_part);
  A.ps = reinterpret_cast<ProbState*>(w + L.o_ps);
  A.cs = reinterpret_cast<ColState*>(w + L.o_cs);
  A.remaining = reinterpret_cast<int32_t*>(w + L.o_rem);
  A.tol = prm->tol;
  A.delta = prm->reliable_delta > 0.0 && prm->reliable_delta < 1.0 ? prm->reliable_delta : 0.1;
  A.maxiter = prm->maxiter > 0 ? prm->maxiter : (int)std::min<int64_t>(10 * (int64_t)M->n, INT32_MAX / 4);
  const int chunk = prm->chunk > 0 ? std::min(prm->chunk, 256) : 16;
  switch (k) {
    case 1: return run_block<1>(A, prec, chunk, A.maxiter, s, iters_out, relres_out, status_out);
    case 2: return run_block<2>(A, prec, chunk, A.maxiter, s, iters_out, relres_out, status_out);
    case 4: return run_block<4>(A, prec, chunk, A.maxiter, s, iters_out, relres_out, status_out);
    case 8: return run_block<8>(A, prec, chunk, A.maxiter, s, iters_out, relres_out, status_out);
    case 16: return run_block<16>(A, prec, chunk, A.maxiter, s, iters_out, relres_out, status_out);
    case 32: return run_block<32>(A, prec, chunk, A.maxiter, s, iters_out, relres_out, status_out);
    default: return run_block<64>(A, prec, chunk, A.maxiter, s, iters_out, relres_out, status_out);
  }
}

extern "C" int32_t feab_block_spmm(const feab_csr* M, const double* X, double* Y, int32_t k, cudaStream_t s) {
  if (!M || !X || !Y || M->n <= 0 || !M->row_ptr || !M->col_idx || !M->vals64 || !M->group_ptr || M->n_groups <= 0)
    return FEAB_BAD_ARG;
  if (k != 1 && k != 2 && k != 4 && k != 8 && k != 16 && k != 32 && k != 64) return FEAB_BAD_ARG;
  if (X == Y) return FEAB_BAD_ARG;
  if (k == 64 && ((reinterpret_cast<uintptr_t>(X) & 15) != 0)) return FEAB_BAD_ARG;  // 16-byte panel-row gathers
  BArgs A{};
  A.n = M->n;
  A.n_groups = M->n_groups;
  A.k = k;
  A.row_ptr = M->row_ptr;
  A.col_idx = M->col_idx;
  A.group_ptr = M->group_ptr;
  A.vals64 = M->vals64;
  switch (k) {
    case 1: launch_block_spmm<1>(A, X, Y, s); break;
    case 2: launch_block_spmm<2>(A, X, Y, s); break;
    case 4: launch_block_spmm<4>(A, X, Y, s); break;
    case 8: launch_block_spmm<8>(A, X, Y, s); break;
    case 16: launch_block_spmm<16>(A, X, Y, s); break;
    case 32: launch_block_spmm<32>(A, X, Y, s); break;
    default: launch_block_spmm<64>(A, X, Y, s); break;
  }
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}
