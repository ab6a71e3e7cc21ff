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
  // node tiles (feab_tile_operator; t_g0 == null: the SpMM walks single row groups)
  const int32_t* t_g0;
  const int32_t* t_gt;
  const int32_t* t_uoff;
  const int32_t* t_poff;
  const int32_t* t_ucol;
  const uint8_t* t_umask;
  const double* t_v64;
  const uint32_t* t_vhi;
  const uint16_t* t_vlo;
  const uint8_t* t_vlo2;
  const int32_t* t_cptr;
  const int32_t* t_chunk;
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
// The group-path SpMM (kernel A when the operator has no node tiles, and the stand-alone block
// SpMM) is bound by the L1 data path (each 512-byte panel-row gather is four wavefronts, each
// value broadcast one); it runs at FEAB_BLOCK_GROUP_MINB resident CTAs per SM with
// FEAB_BLOCK_GROUP_UNROLL gathers in flight per lane, so that more warps hide the gathers'
// latency.  Measured at 128x32x32 with 64 columns (FP64 SpMM, L2 flushed): 4 CTAs and 8 gathers
// 386 us, 4 and 4 401 us, 3 and 8 434 us, 2 and 16 475 us (a few spilled registers at 4 CTAs and
// 8 gathers cost less than the occupancy gains).
#ifndef FEAB_BLOCK_GROUP_MINB
#define FEAB_BLOCK_GROUP_MINB 4
#endif
#ifndef FEAB_BLOCK_GROUP_UNROLL
#define FEAB_BLOCK_GROUP_UNROLL 8
#endif
constexpr int kGroupU = FEAB_BLOCK_GROUP_UNROLL;
static_assert(kStageCols % kUnrollFp64 == 0 && kStageCols % kUnroll == 0 && kStageCols % kGroupU == 0,
              "vector reads stay inside the stage");

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
      // multiples of 4): one 16-byte column load per quad, stored with the tag bits cleared so
      // the gathers below index with it directly, and a 16 + 8 + 4-byte value load per (row,
      // quad) pair, the pairs spread over all lanes
      const int nq = nc >> 2;
      for (int mq = lane; mq < nq; mq += 32) {
        const uint4 tq = __ldg(reinterpret_cast<const uint4*>(A.tcol + c0 + cb + 4 * mq));
        *reinterpret_cast<int4*>(&st.col[4 * mq]) =
            make_int4((int)(tq.x & 0x3fffffffu), (int)(tq.y & 0x3fffffffu), (int)(tq.z & 0x3fffffffu),
                      (int)(tq.w & 0x3fffffffu));
      }
      for (int pq = lane; pq < 3 * nq; pq += 32) {
        const int k = pq >= nq ? (pq >= 2 * nq ? 2 : 1) : 0;
        const int m = 4 * (pq - k * nq);
        double2* dst = reinterpret_cast<double2*>(&st.val[k][m]);
        if (k < f) {
          const int64_t e = s0 + (int64_t)k * len + cb + m;
          const uint4 h = __ldg(reinterpret_cast<const uint4*>(A.vhi + e));
          const uint2 l = __ldg(reinterpret_cast<const uint2*>(A.vlo + e));
          const uint32_t l2 = __ldg(reinterpret_cast<const uint32_t*>(A.vlo2 + e));
          dst[0] = make_double2(dec56(h.x, l.x, l2), dec56(h.y, l.x >> 16, l2 >> 8));
          dst[1] = make_double2(dec56(h.z, l.y, l2 >> 16), dec56(h.w, l.y >> 16, l2 >> 24));
        } else {
          dst[0] = dst[1] = make_double2(0.0, 0.0);
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
            gather_row<K>(src, (int)t[u], cl, xv[u]);
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
          gather_row<K>(src, (int)t[u], cl, xv[u]);
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

// ---------------------------------------------------------------- node tiles
// A warp applies a tile of up to kTG consecutive row groups (feab_tile_operator): it walks the
// union of their column lists, gathers each union column's panel row once and adds it, with the
// column's value triple of each group that has the column, to that group's rows.  The union is
// staged in chunks of kTileChunk columns: the columns, the group masks, each column's first
// value triple within the chunk (a warp scan of the mask popcounts) and the chunk's values
// (decoded to FP64 for the difference form).  The tile's columns are grouped by mask, so a chunk
// is a few runs of one mask each, and each run goes through a loop specialised for its mask.
constexpr int kTG = FEAB_TILE_GROUPS;
constexpr int kTileChunk = FEAB_TILE_CHUNK;
// union columns whose panel rows a lane gathers before using any
#ifndef FEAB_TILE_UNROLL
#define FEAB_TILE_UNROLL 8
#endif
constexpr int kTileU = FEAB_TILE_UNROLL;

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

struct __align__(16) TileStage {
  int col[kTileChunk];
  uint16_t pair[kTileChunk];
  uint32_t mask4[kTileChunk / 4];
  double val[3 * kTG * kTileChunk];
};

// A warp's shared-memory stage: one row group's columns and values, or one tile chunk.
union __align__(16) WarpStage {
  GroupStage g;
  TileStage t;
};

constexpr int popc4(int m) { return (m & 1) + ((m >> 1) & 1) + ((m >> 2) & 1) + ((m >> 3) & 1); }
static_assert(kTG >= 1 && kTG <= 4, "tiles of 1 to 4 row groups (4-bit group masks)");

// Staged columns [mb, me) of one mask M: each column's value triples (one per set bit of M, in
// bit order) are contiguous from value vb, so the loop is free of per-group branches.
template <int M, int K>
__device__ __forceinline__ void tile_run(const int* __restrict__ col, const double* __restrict__ val, int mb, int me,
                                         int vb, int sub, int cl, const double* __restrict__ src,
                                         double (&acc)[kTG][3][K >= 32 ? K / 32 : 1]) {
  constexpr int CPL = K >= 32 ? K / 32 : 1;
  constexpr int MPW = K >= 32 ? 1 : 32 / K;
  constexpr int U = kTileU;
  constexpr int NB = popc4(M);
  for (int m0 = mb + sub; m0 < me; m0 += MPW * U) {
    double xv[U][CPL];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int m = m0 + u * MPW;
      if (m < me) {
        gather_row<K>(src, col[m], cl, xv[u]);
      } else {
#pragma unroll
        for (int q = 0; q < CPL; ++q) xv[u][q] = 0.0;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int m = m0 + u * MPW;
      if (m >= me) break;
      const double* w = &val[vb + 3 * NB * (m - mb)];
      int b = 0;
#pragma unroll
      for (int j = 0; j < kTG; ++j) {
        if ((M >> j) & 1) {
          const double w0 = w[3 * b], w1 = w[3 * b + 1], w2 = w[3 * b + 2];
#pragma unroll
          for (int q = 0; q < CPL; ++q) {
            acc[j][0][q] = fma(w0, xv[u][q], acc[j][0][q]);
            acc[j][1][q] = fma(w1, xv[u][q], acc[j][1][q]);
            acc[j][2][q] = fma(w2, xv[u][q], acc[j][2][q]);
          }
          ++b;
        }
      }
    }
  }
}

// tile_run for the run's mask mk (1 .. 2^kTG - 1): a chain of uniform branches.
template <int M, int K>
__device__ __forceinline__ void dispatch_run(unsigned mk, const int* __restrict__ col, const double* __restrict__ val,
                                             int mb, int me, int vb, int sub, int cl, const double* __restrict__ src,
                                             double (&acc)[kTG][3][K >= 32 ? K / 32 : 1]) {
  if (mk == (unsigned)M) {
    tile_run<M, K>(col, val, mb, me, vb, sub, cl, src, acc);
  } else if constexpr (M + 1 < (1 << kTG)) {
    dispatch_run<M + 1, K>(mk, col, val, mb, me, vb, sub, cl, src, acc);
  }
}

// acc[j][row][q] = (K src) for row `row` of group j of tile t, panel column panel_col(cl, q).
// Each chunk is staged in one round trip (columns and masks through registers, FP64 values by
// cp.async straight to shared memory); the next chunk's descriptor is loaded meanwhile.  (A
// variant that copied the next chunk in while applying this one, two buffers per warp, measured
// 507 against 436 us per 128x32x32 SpMM with 64 columns: the gathers set the pace, and its larger
// code missed in the instruction cache.)
template <int K, bool DIFF>
__device__ __forceinline__ void tile_spmm(const BArgs& A, int t, int lane, TileStage& st,
                                          const double* __restrict__ src,
                                          double (&acc)[kTG][3][K >= 32 ? K / 32 : 1]) {
  constexpr int CPL = K >= 32 ? K / 32 : 1;
  constexpr int LW = K >= 32 ? 32 : K;
  const int sub = lane / LW, cl = lane % LW;
  const int4* __restrict__ chunks = reinterpret_cast<const int4*>(A.t_chunk);
  const int c1 = A.t_cptr[t + 1];
  int c = A.t_cptr[t];
#pragma unroll
  for (int j = 0; j < kTG; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int q = 0; q < CPL; ++q) acc[j][k][q] = 0.0;
  // chunk descriptor {first union column, columns, first value, values}
  int4 d = c < c1 ? __ldg(chunks + c) : make_int4(0, 0, 0, 0);
  for (; c < c1; ++c) {
    const int4 dn = c + 1 < c1 ? __ldg(chunks + c + 1) : d;
    const int nc = d.y, nv = d.w;  // nc a multiple of 4
    if (!DIFF) {
      for (int i = lane; i < nv; i += 32) cp_async8(&st.val[i], A.t_v64 + (int64_t)d.z + i);
      cp_async_commit();
    } else {
      for (int i = lane; i < nv; i += 32) {
        const int64_t q = (int64_t)d.z + i;
        st.val[i] = dec56(__ldg(A.t_vhi + q), __ldg(A.t_vlo + q), __ldg(A.t_vlo2 + q));
      }
    }
    int np = 0, p4[4] = {0, 0, 0, 0};
    if (4 * lane < nc) {
      const int4 c4 = __ldg(reinterpret_cast<const int4*>(A.t_ucol + d.x) + lane);
      const uint32_t m4 = __ldg(reinterpret_cast<const uint32_t*>(A.t_umask + d.x) + lane);
      *reinterpret_cast<int4*>(&st.col[4 * lane]) = c4;
      st.mask4[lane] = m4;
#pragma unroll
      for (int e = 0; e < 4; ++e) p4[e] = __popc((m4 >> (8 * e)) & 0xffu);
      np = p4[0] + p4[1] + p4[2] + p4[3];
    }
    // the first value triple of every column within the chunk: a warp scan of mask popcounts
    const int incl = warp_incl_scan(np, lane);
    if (4 * lane < nc) {
      int e = incl - np;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        st.pair[4 * lane + q] = (uint16_t)e;
        e += p4[q];
      }
    }
    if (!DIFF) cp_async_wait_all();
    __syncwarp();
    // runs of columns with the same mask (a tile's columns are grouped by mask; padding, mask
    // 0, comes last)
    int m = 0;
    while (m < nc) {
      const unsigned mk = (st.mask4[m >> 2] >> (8 * (m & 3))) & 0xffu;
      if (mk == 0u) break;
      int e = m;
      while (true) {
        const int q = e + lane;
        const bool other = q >= nc || ((st.mask4[q >> 2] >> (8 * (q & 3))) & 0xffu) != mk;
        const unsigned bal = __ballot_sync(FEAB_FULL_MASK, other);
        if (bal) {
          e += __ffs(bal) - 1;
          break;
        }
        e += 32;
      }
      dispatch_run<1, K>(mk, st.col, st.val, m, e, 3 * st.pair[m], sub, cl, src, acc);
      m = e;
    }
    __syncwarp();  // every lane is done with the stage before it is refilled
    d = dn;
  }
  // combine the sub-warps (lanes with equal cl)
#pragma unroll
  for (int o = LW; o < 32; o <<= 1)
#pragma unroll
    for (int j = 0; j < kTG; ++j)
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int q = 0; q < CPL; ++q) acc[j][k][q] += __shfl_xor_sync(FEAB_FULL_MASK, acc[j][k][q], o);
  if constexpr (DIFF) {
    // the own-node term T_a x_a of every group (the difference form leaves own columns out)
    const int g0 = A.t_g0[t], nt = A.t_g0[t + 1] - g0;
#pragma unroll
    for (int j = 0; j < kTG; ++j) {
      if (j >= nt) break;
      const int g = g0 + j;
      const int r0 = A.group_ptr[g], f = A.group_ptr[g + 1] - r0;
      const int mask = A.gmask[g];
      double xs[3][CPL];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        if ((mask >> cc) & 1) {
          gather_row<K>(src, r0 + __popc(mask & ((1 << cc) - 1)), cl, xs[cc]);
        } else {
#pragma unroll
          for (int q = 0; q < CPL; ++q) xs[cc][q] = 0.0;
        }
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (k < f) {
          const double s0v = A.S[(int64_t)(r0 + k) * 3 + 0], s1v = A.S[(int64_t)(r0 + k) * 3 + 1],
                       s2v = A.S[(int64_t)(r0 + k) * 3 + 2];
#pragma unroll
          for (int q = 0; q < CPL; ++q) acc[j][k][q] += s0v * xs[0][q] + s1v * xs[1][q] + s2v * xs[2][q];
        }
      }
    }
  }
}

// The item's tiles [t0, t1): its groups are whole tiles (checked before the solve starts).
__device__ __forceinline__ void item_tiles(const BArgs& A, int it, int& t0, int& t1) {
  t0 = A.t_gt[A.item_g0[it]];
  t1 = A.t_gt[A.item_g1[it] - 1] + 1;
}

// Every work item starts and ends on a tile boundary; flag[0] = 1 otherwise.
__global__ void k_tile_items_check(BArgs A, int32_t* flag) {
  const int it = blockIdx.x * blockDim.x + threadIdx.x;
  if (it >= A.n_items) return;
  const int g0 = A.item_g0[it], g1 = A.item_g1[it];
  if (g0 < 0 || g1 <= g0 || g1 > A.n_groups || A.t_g0[A.t_gt[g0]] != g0 || A.t_g0[A.t_gt[g1 - 1] + 1] != g1)
    atomicExch(flag, 1);
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
// per-column partial p.Ap (or r.r).  TILES: the operator has node tiles (the CG steps walk them;
// a reliable step walks the row groups); otherwise every step walks the row groups, at the
// group path's occupancy and with a group-sized stage.
template <int K, bool MIXED, bool TILES>
__global__ void __launch_bounds__(kThreads, TILES ? FEAB_BLOCK_MINB : FEAB_BLOCK_GROUP_MINB) k_bstep_a(BArgs A) {
  constexpr int CPL = K >= 32 ? K / 32 : 1;
  constexpr int LW = K >= 32 ? 32 : K;
  __shared__ double sm[kWarps][K];
  // one stage per warp: a WarpStage with tiles, a GroupStage without
  extern __shared__ __align__(16) unsigned char dyn_stage[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  GroupStage& gstage =
      TILES ? reinterpret_cast<WarpStage*>(dyn_stage)[w].g : reinterpret_cast<GroupStage*>(dyn_stage)[w];
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
    // one output row: AP and p.Ap, or (reliable step) R = B - K X and r.r
    auto emit = [&](int row, const double (&v)[CPL]) {
#pragma unroll
      for (int q = 0; q < CPL; ++q) {
        const int64_t idx = (int64_t)row * K + panel_col<K>(lane, q);
        if (reliable) {
          const double ri = A.B[idx] - v[q];
          A.R[idx] = ri;
          part[q] += ri * ri;
        } else {
          const double pv = po[idx];
          A.AP[idx] = v[q];
          part[q] += pv * v[q];
        }
      }
    };
    if (TILES && !reliable) {
      int t0, t1;
      item_tiles(A, it, t0, t1);
      for (int t = t0 + w; t < t1; t += kWarps) {
        double acc[kTG][3][CPL];
        tile_spmm<K, MIXED>(A, t, lane, reinterpret_cast<WarpStage*>(dyn_stage)[w].t, po, acc);
        if (lane < LW) {
          const int tg0 = A.t_g0[t], nt = A.t_g0[t + 1] - tg0;
#pragma unroll
          for (int j = 0; j < kTG; ++j) {
            if (j >= nt) break;
            const int r0 = A.group_ptr[tg0 + j], f = A.group_ptr[tg0 + j + 1] - r0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              if (k >= f) break;
              emit(r0 + k, acc[j][k]);
            }
          }
        }
      }
    } else {
      const int g1 = A.item_g1[it];
      for (int g = A.item_g0[it] + w; g < g1; g += kWarps) {
        double acc[3][CPL];
        if constexpr (MIXED) {
          if (!diff) group_spmm<K, false, TILES ? kUnroll : kGroupU>(A, g, lane, gstage, src, acc);
          else group_spmm<K, true, TILES ? kUnroll : kGroupU>(A, g, lane, gstage, po, acc);
        } else {
          group_spmm<K, false, TILES ? kUnrollFp64 : kGroupU>(A, g, lane, gstage, po, acc);
        }
        if (lane < LW) {
          const int r0 = A.group_ptr[g], f = A.group_ptr[g + 1] - r0;
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            if (k >= f) break;
            emit(r0 + k, acc[k]);
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
__global__ void __launch_bounds__(kThreads, FEAB_BLOCK_GROUP_MINB) k_block_spmm(BArgs A, const double* __restrict__ src,
                                                                               double* __restrict__ dst) {
  constexpr int CPL = K >= 32 ? K / 32 : 1;
  constexpr int LW = K >= 32 ? 32 : K;
  __shared__ GroupStage stage[kWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int g = blockIdx.x * kWarps + w; g < A.n_groups; g += gridDim.x * kWarps) {
    double acc[3][CPL];
    group_spmm<K, false, kGroupU>(A, g, lane, stage[w], src, acc);
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

// The same through the node tiles (FP64 tile values), one warp per tile.
template <int K>
__global__ void __launch_bounds__(kThreads, FEAB_BLOCK_MINB) k_block_spmm_tiles(BArgs A, int32_t n_tiles,
                                                                               const double* __restrict__ src,
                                                                               double* __restrict__ dst) {
  constexpr int CPL = K >= 32 ? K / 32 : 1;
  constexpr int LW = K >= 32 ? 32 : K;
  extern __shared__ __align__(16) unsigned char dyn_stage[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  WarpStage& stage = reinterpret_cast<WarpStage*>(dyn_stage)[w];
  for (int t = blockIdx.x * kWarps + w; t < n_tiles; t += gridDim.x * kWarps) {
    double acc[kTG][3][CPL];
    tile_spmm<K, false>(A, t, lane, stage.t, src, acc);
    if (lane < LW) {
      const int tg0 = A.t_g0[t], nt = A.t_g0[t + 1] - tg0;
#pragma unroll
      for (int j = 0; j < kTG; ++j) {
        if (j >= nt) break;
        const int r0 = A.group_ptr[tg0 + j], f = A.group_ptr[tg0 + j + 1] - r0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          if (k >= f) break;
#pragma unroll
          for (int q = 0; q < CPL; ++q) dst[(int64_t)(r0 + k) * K + panel_col<K>(lane, q)] = acc[j][k][q];
        }
      }
    }
  }
}

constexpr size_t kStageBytes = kWarps * sizeof(WarpStage);

template <int K>
cudaError_t launch_block_spmm(const BArgs& A, int32_t n_tiles, const double* X, double* Y, cudaStream_t s) {
  if (A.t_g0) {
    cudaError_t e = cudaFuncSetAttribute(k_block_spmm_tiles<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kStageBytes);
    if (e != cudaSuccess) return e;
    const int grid = std::max(1, std::min((n_tiles + kWarps - 1) / kWarps, sm_count() * 8));
    k_block_spmm_tiles<K><<<grid, kThreads, kStageBytes, s>>>(A, n_tiles, X, Y);
  } else {
    const int grid = std::max(1, std::min((A.n_groups + kWarps - 1) / kWarps, sm_count() * 8));
    k_block_spmm<K><<<grid, kThreads, 0, s>>>(A, X, Y);
  }
  return cudaGetLastError();
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
  L.o_rem = take(2 * sizeof(int32_t));  // problems remaining, tile-alignment flag
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
  SolverState& state = thread_solver_state<1>();
  HostFlag& flag = state.flag;
  GraphCache& graphs = state.graphs;
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
    const bool tiles = A.t_g0 != nullptr;
    const size_t smem_a = tiles ? kStageBytes : kWarps * sizeof(GroupStage);
    if (fail(cudaFuncSetAttribute(k_bstep_a<K, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kStageBytes)))
      break;
    if (fail(cudaFuncSetAttribute(k_bstep_a<K, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kStageBytes)))
      break;
    auto record = [&](cudaStream_t cs) {
      for (int q = 0; q < chunk; ++q) {
        k_bstep_p<K><<<grid_pb, kThreads, 0, cs>>>(A);
        if (prec == FEAB_PREC_MIXED) {
          if (tiles) k_bstep_a<K, true, true><<<grid, kThreads, smem_a, cs>>>(A);
          else k_bstep_a<K, true, false><<<grid, kThreads, smem_a, cs>>>(A);
          k_bstep_b<K, true><<<grid_pb, kThreads, 0, cs>>>(A);
        } else {
          if (tiles) k_bstep_a<K, false, true><<<grid, kThreads, smem_a, cs>>>(A);
          else k_bstep_a<K, false, false><<<grid, kThreads, smem_a, cs>>>(A);
          k_bstep_b<K, false><<<grid_pb, kThreads, 0, cs>>>(A);
        }
      }
      cudaMemcpyAsync((void*)hflag, A.remaining, sizeof(int32_t), cudaMemcpyDeviceToHost, cs);
    };
    if (fail(graphs.acquire(&A, sizeof(A), topo_signature({K, prec, chunk, grid, grid_pb, tiles ? 1 : 0}), record, &exec))) break;
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

// Fills the tile fields of A from T; false if T does not fit A's groups or the precision.
bool set_tiles(BArgs& A, const feab_tile_operator* T, int prec) {
  if (!T) return true;
  if (T->n_groups != A.n_groups || T->precision != prec || T->n_tiles <= 0 || !T->tile_g0 || !T->group_tile ||
      !T->uoff || !T->poff || !T->ucol || !T->umask || !T->cptr || !T->chunk)
    return false;
  if ((reinterpret_cast<uintptr_t>(T->ucol) & 15) || (reinterpret_cast<uintptr_t>(T->umask) & 3) ||
      (reinterpret_cast<uintptr_t>(T->chunk) & 15) || (T->v64 && (reinterpret_cast<uintptr_t>(T->v64) & 7)))
    return false;
  if (prec == FEAB_PREC_FP64 ? !T->v64 : (!T->vhi || !T->vlo || !T->vlo2)) return false;
  A.t_g0 = T->tile_g0;
  A.t_gt = T->group_tile;
  A.t_uoff = T->uoff;
  A.t_poff = T->poff;
  A.t_ucol = T->ucol;
  A.t_umask = T->umask;
  A.t_v64 = T->v64;
  A.t_vhi = T->vhi;
  A.t_vlo = T->vlo;
  A.t_vlo2 = T->vlo2;
  A.t_cptr = T->cptr;
  A.t_chunk = T->chunk;
  return true;
}

}  // namespace
}  // namespace feab

using namespace feab;

extern "C" size_t feab_block_pcg_workspace_bytes(int32_t n, int32_t k, int32_t n_problems, int32_t n_items) {
  if (n <= 0 || k <= 0 || n_problems <= 0 || n_items <= 0) return 0;
  return blayout(n, k, n_problems, n_items).total;
}

extern "C" int32_t feab_block_pcg_solve(const feab_csr* M, const feab_diff_operator* D, const feab_tile_operator* T,
                                        const feab_batch* bt, const double* dinv64, const double* B, double* X,
                                        const feab_pcg_params* prm, void* workspace, size_t workspace_bytes,
                                        int32_t* iters_out, double* relres_out, int32_t* status_out, cudaStream_t s) {
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
  if (!set_tiles(A, T, prec)) return FEAB_BAD_ARG;
  if (T) {  // every work item must be whole tiles
    FEAB_CUDA(cudaMemsetAsync(A.remaining + 1, 0, sizeof(int32_t), s));
    k_tile_items_check<<<(A.n_items + kThreads - 1) / kThreads, kThreads, 0, s>>>(A, A.remaining + 1);
    count_launches(1);
    FEAB_CHECK_LAUNCH();
    int32_t bad = 0;
    FEAB_CUDA(cudaMemcpyAsync(&bad, A.remaining + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    FEAB_CUDA(cudaStreamSynchronize(s));
    if (bad) return FEAB_BAD_ARG;
  }
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

extern "C" int32_t feab_block_spmm(const feab_csr* M, const feab_tile_operator* T, const double* X, double* Y,
                                   int32_t k, cudaStream_t s) {
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
  if (!set_tiles(A, T, FEAB_PREC_FP64)) return FEAB_BAD_ARG;
  const int32_t nt = T ? T->n_tiles : 0;
  cudaError_t e;
  switch (k) {
    case 1: e = launch_block_spmm<1>(A, nt, X, Y, s); break;
    case 2: e = launch_block_spmm<2>(A, nt, X, Y, s); break;
    case 4: e = launch_block_spmm<4>(A, nt, X, Y, s); break;
    case 8: e = launch_block_spmm<8>(A, nt, X, Y, s); break;
    case 16: e = launch_block_spmm<16>(A, nt, X, Y, s); break;
    case 32: e = launch_block_spmm<32>(A, nt, X, Y, s); break;
    default: e = launch_block_spmm<64>(A, nt, X, Y, s); break;
  }
  count_launches(1);
  return e == cudaSuccess ? FEAB_OK : FEAB_CUDA_ERROR;
}
