// Sliced (SELL-32) node-group operator: build from the CSR, and the standalone SpMV.
#include <algorithm>
#include "feab_scan.cuh"
#include "feab_sell.cuh"

namespace feab {

namespace {

constexpr int kThreads = 256;

size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

int round4(int v) { return (v + 3) & ~3; }

struct SellScratch {
  int64_t* scan;
  int64_t* total;
  int32_t* err;
  int32_t* wide;   // set when a column lies more than 16 bits from its lane's first row
};

// Storage: soff, scan scratch, flags, then columns and values for n_slices slices of at most
// round4(max_row_len) steps each (the scan packs the slices, so only the front is used).
void sell_layout(int32_t n, int32_t n_groups, int32_t max_row_len, int32_t kind, char* base, feab_sell_operator* D,
                 SellScratch* X, size_t* total) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base ? base + off : nullptr;
    off += a256(bytes);
    return p;
  };
  const int32_t ns = (n_groups + 31) / 32;
  const size_t steps = (size_t)ns * (size_t)round4(max_row_len);
  char* so = take(sizeof(int32_t) * ((size_t)ns + 1));
  char* sc = take(sizeof(int64_t) * ((size_t)scan_blocks((int64_t)ns + 1) + 2));
  char* tt = take(sizeof(int64_t) + 2 * sizeof(int32_t));
  char* tc = take(sizeof(int32_t) * 32 * steps);
  char* t16 = take(sizeof(int16_t) * 32 * steps);
  char *v64 = nullptr, *hi = nullptr, *lo = nullptr, *gm = nullptr, *ss = nullptr;
  if (kind == FEAB_PREC_FP64) {
    v64 = take(sizeof(double) * 96 * steps);
  } else {
    hi = take(sizeof(uint32_t) * 96 * steps);
    lo = take(sizeof(uint16_t) * 96 * steps);
    gm = take((size_t)n_groups);
    ss = take(sizeof(double) * 3 * (size_t)n);
  }
  if (D) {
    D->kind = kind;
    D->n_slices = ns;
    D->soff = reinterpret_cast<int32_t*>(so);
    D->tcol = reinterpret_cast<int32_t*>(tc);
    D->tcol16 = reinterpret_cast<int16_t*>(t16);
    D->v64 = reinterpret_cast<double*>(v64);
    D->vhi = reinterpret_cast<uint32_t*>(hi);
    D->vlo = reinterpret_cast<uint16_t*>(lo);
    D->gmask = reinterpret_cast<uint8_t*>(gm);
    D->S = reinterpret_cast<double*>(ss);
  }
  if (X) {
    X->scan = reinterpret_cast<int64_t*>(sc);
    X->total = reinterpret_cast<int64_t*>(tt);
    X->err = reinterpret_cast<int32_t*>(tt + sizeof(int64_t));
    X->wide = reinterpret_cast<int32_t*>(tt + sizeof(int64_t) + sizeof(int32_t));
  }
  if (total) *total = off;
}

// Pass 1, one thread per slice: W_s = the longest group's column count (all columns for FP64,
// off-node columns for the difference form), rounded up to 4.
__global__ void k_sell_widths(int32_t n_groups, int32_t n_slices, int kind, int32_t wmax,
                              const int32_t* __restrict__ group_ptr, const int32_t* __restrict__ row_ptr,
                              int32_t* __restrict__ width, int32_t* __restrict__ err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slices) return;
  int w = 0;
  const int g1 = min(n_groups, 32 * s + 32);
  for (int g = 32 * s; g < g1; ++g) {
    const int r0 = group_ptr[g], f = group_ptr[g + 1] - r0;
    const int len = row_ptr[r0 + 1] - row_ptr[r0];
    w = max(w, kind == FEAB_PREC_FP64 ? len : len - f);
  }
  w = (w + 3) & ~3;
  if (w > wmax) atomicExch(err, 1);
  width[s] = min(w, wmax);
}

// Pass 2, one warp per slice, lane l writing group 32 s + l: columns, values (FP64 or rounded to
// 36 mantissa bits), and for the mixed kind the free-DOF mask and the own-node terms T (below).
__global__ void __launch_bounds__(kThreads) k_sell_fill(int32_t n_groups, int32_t n_slices, int kind,
                                                        const int32_t* __restrict__ group_ptr,
                                                        const int32_t* __restrict__ row_ptr,
                                                        const int32_t* __restrict__ col_idx,
                                                        const double* __restrict__ vals,
                                                        const int32_t* __restrict__ dof_of,
                                                        const int32_t* __restrict__ soff, int32_t* __restrict__ tcol,
                                                        int16_t* __restrict__ tcol16, int32_t* __restrict__ wide,
                                                        double* __restrict__ v64, uint32_t* __restrict__ vhi,
                                                        uint16_t* __restrict__ vlo, uint8_t* __restrict__ gmask,
                                                        double* __restrict__ Ssum, int32_t* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (s >= n_slices) return;
  const int g = 32 * s + lane;
  const bool valid = g < n_groups;
  const bool diff = kind != FEAB_PREC_FP64;
  int r0 = 0, f = 0, s0 = 0, len = 0, own = 0, j0 = 0;
  if (valid) {
    r0 = group_ptr[g];
    f = group_ptr[g + 1] - r0;
    s0 = row_ptr[r0];
    len = row_ptr[r0 + 1] - s0;
    if (diff) {
      own = -1;
      for (int c = 0; c < len; ++c)
        if (col_idx[s0 + c] == r0) {
          own = c;
          break;
        }
      if (own < 0 || own + f > len) {
        atomicExch(err, 2);
        own = 0;
        f = 0;
        len = 0;
      }
      j0 = dof_of[r0] % 3;
      int m = 0;
      for (int k = 0; k < f; ++k) m |= 1 << (dof_of[r0 + k] % 3);
      gmask[g] = (uint8_t)m;
    }
  }
  const int base = soff[s], W = soff[s + 1] - base;
  const int ncols = diff ? len - f : len;
  const int32_t pad = valid ? (diff ? (int32_t)((uint32_t)r0 | ((uint32_t)j0 << 30)) : r0) : 0;
  for (int j = 0; j < W; ++j) {
    const size_t b = (size_t)(base + (j & ~3)), u = (size_t)(j & 3);
    const size_t e = b * 32 + 4 * lane + u;
    const bool real = j < ncols;
    const int c = diff ? (j < own ? j : j + f) : j;
    int32_t tag = pad;
    if (real) {
      const int col = col_idx[s0 + c];
      tag = diff ? (int32_t)((uint32_t)col | ((uint32_t)(dof_of[col] % 3) << 30)) : col;
    }
    tcol[e] = tag;
    const int delta = (int)((uint32_t)tag & 0x3fffffffu) - r0;
    if (delta < -32768 || delta > 32767) atomicExch(wide, 1);
    tcol16[e] = (int16_t)delta;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double v = (real && k < f) ? vals[row_ptr[r0 + k] + c] : 0.0;
      const size_t ev = (3 * b + 4 * k) * 32 + 4 * lane + u;
      if (!diff) {
        v64[ev] = v;
      } else {
        const unsigned long long bits = (unsigned long long)__double_as_longlong(v) + 0x8000ull;
        vhi[ev] = (uint32_t)(bits >> 32);
        vlo[ev] = (uint16_t)((bits >> 16) & 0xffffull);
      }
    }
  }
  if (diff && valid) {
    // T[r][j] = S[r][j] - W[r][j]: S sums all of row r's exact values of DOF component j, W its
    // rounded off-node values of component j (both in column order).  Then
    //   sum_{b != a} w (x_b - x_a) + S x_a  =  sum_{b != a} w x_b + T x_a
    // exactly, so the kernel applies the plain form to the rounded values plus T on the own node,
    // with the same value-rounding error as the difference form.
    for (int k = 0; k < f; ++k) {
      const int sk = row_ptr[r0 + k];
      double sj[3] = {0.0, 0.0, 0.0}, wj[3] = {0.0, 0.0, 0.0};
      for (int c = 0; c < len; ++c) {
        const int jc = dof_of[col_idx[sk + c]] % 3;
        const double v = vals[sk + c];
        sj[jc] += v;
        if (c < own || c >= own + f) {
          const unsigned long long bits = (unsigned long long)__double_as_longlong(v) + 0x8000ull;
          wj[jc] += __longlong_as_double((long long)(bits & ~0xffffull));
        }
      }
      for (int j = 0; j < 3; ++j) Ssum[(int64_t)(r0 + k) * 3 + j] = sj[j] - wj[j];
    }
  }
}

template <int KIND, bool IDX16>
__global__ void __launch_bounds__(kThreads, SellTuning<KIND>::kMinBlocks) k_sell_spmv(SellView V, const double* __restrict__ x,
                                                           double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < V.n_slices; s += nw) {
    const SellLane L = sell_lane(V, s, lane);
    double acc[3], xs[3];
    sell_apply<KIND, IDX16>(V, s, lane, L, [&](int j) { return __ldg(x + j); }, acc, xs);
    if (L.f > 0) y[L.r0] = acc[0];
    if (L.f > 1) y[L.r0 + 1] = acc[1];
    if (L.f > 2) y[L.r0 + 2] = acc[2];
  }
}

}  // namespace

SellView sell_view(const feab_csr* A, const feab_sell_operator* op) {
  SellView V;
  V.kind = op->kind;
  V.n_slices = op->n_slices;
  V.n_groups = A->n_groups;
  V.soff = op->soff;
  V.tcol = op->tcol;
  V.tcol16 = op->tcol16;
  V.v64 = op->v64;
  V.vhi = op->vhi;
  V.vlo = op->vlo;
  V.gmask = op->gmask;
  V.S = op->S;
  V.group_ptr = A->group_ptr;
  return V;
}

void launch_sell_spmv(const SellView& V, const double* x, double* y, cudaStream_t s) {
  const int wpb = kThreads / 32;
  const int grid = std::max(1, std::min((V.n_slices + wpb - 1) / wpb, sm_count() * 8));
  if (V.kind == FEAB_PREC_FP64) {
    if (V.tcol16) k_sell_spmv<FEAB_PREC_FP64, true><<<grid, kThreads, 0, s>>>(V, x, y);
    else k_sell_spmv<FEAB_PREC_FP64, false><<<grid, kThreads, 0, s>>>(V, x, y);
  } else {
    if (V.tcol16) k_sell_spmv<FEAB_PREC_MIXED, true><<<grid, kThreads, 0, s>>>(V, x, y);
    else k_sell_spmv<FEAB_PREC_MIXED, false><<<grid, kThreads, 0, s>>>(V, x, y);
  }
  count_launches(1);
}

}  // namespace feab

using namespace feab;

extern "C" size_t feab_sell_operator_bytes(int32_t n, int32_t n_groups, int32_t max_row_len, int32_t kind) {
  if (n <= 0 || n_groups <= 0 || max_row_len <= 0) return 0;
  if (kind != FEAB_PREC_FP64 && kind != FEAB_PREC_MIXED) return 0;
  size_t total = 0;
  sell_layout(n, n_groups, max_row_len, kind, nullptr, nullptr, nullptr, &total);
  return total;
}

extern "C" int32_t feab_sell_operator_build(const feab_csr* A, const int32_t* dof_of, int32_t kind,
                                            int32_t max_row_len, void* storage, size_t storage_bytes,
                                            feab_sell_operator* out, cudaStream_t s) {
  if (!A || !storage || !out || !A->group_ptr || A->n_groups <= 0 || !A->vals64 || A->n <= 0 || max_row_len <= 0)
    return FEAB_BAD_ARG;
  if (kind != FEAB_PREC_FP64 && kind != FEAB_PREC_MIXED) return FEAB_BAD_ARG;
  if (kind == FEAB_PREC_MIXED && !dof_of) return FEAB_BAD_ARG;
  if (reinterpret_cast<uintptr_t>(storage) & 15u) return FEAB_BAD_ARG;  // the SpMV's 16-byte loads
  if (A->n >= (1 << 30)) return FEAB_CAPACITY;
  const int32_t ns = (A->n_groups + 31) / 32;
  if ((int64_t)ns * round4(max_row_len) * 96 >= ((int64_t)1 << 40)) return FEAB_CAPACITY;
  if ((int64_t)ns * round4(max_row_len) >= (int64_t)INT32_MAX) return FEAB_CAPACITY;
  const size_t need = feab_sell_operator_bytes(A->n, A->n_groups, max_row_len, kind);
  if (need == 0 || need > storage_bytes) return FEAB_BAD_ARG;
  SellScratch X;
  sell_layout(A->n, A->n_groups, max_row_len, kind, static_cast<char*>(storage), out, &X, nullptr);
  FEAB_CUDA(cudaMemsetAsync(X.err, 0, 2 * sizeof(int32_t), s));  // err and wide
  k_sell_widths<<<(ns + kThreads - 1) / kThreads, kThreads, 0, s>>>(A->n_groups, ns, kind, round4(max_row_len),
                                                                     A->group_ptr, A->row_ptr, out->soff, X.err);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  FEAB_CUDA(scan_exclusive_i32(out->soff, out->soff, ns, X.scan, X.total, s));
  const int wpb = kThreads / 32;
  k_sell_fill<<<(ns + wpb - 1) / wpb, kThreads, 0, s>>>(A->n_groups, ns, kind, A->group_ptr, A->row_ptr, A->col_idx,
                                                        A->vals64, dof_of, out->soff, out->tcol, out->tcol16, X.wide,
                                                        out->v64, out->vhi,
                                                        out->vlo, out->gmask, out->S, X.err);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  int32_t flags[2] = {0, 0};
  FEAB_CUDA(cudaMemcpyAsync(flags, X.err, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaStreamSynchronize(s));
  if (flags[1]) out->tcol16 = nullptr;  // some offset needs more than 16 bits: the SpMV reads tcol
  return flags[0] ? FEAB_BAD_ARG : FEAB_OK;
}


extern "C" int32_t feab_sell_spmv(const feab_csr* A, const feab_sell_operator* op, const double* x, double* y,
                                  cudaStream_t s) {
  if (!A || !op || !x || !y || !A->group_ptr || A->n_groups <= 0 || op->n_slices != (A->n_groups + 31) / 32)
    return FEAB_BAD_ARG;
  if (op->kind != FEAB_PREC_FP64 && op->kind != FEAB_PREC_MIXED) return FEAB_BAD_ARG;
  auto al = [](const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; };
  if (!op->soff || !op->tcol || !al(op->tcol, 16) || (op->tcol16 && !al(op->tcol16, 8))) return FEAB_BAD_ARG;
  if (op->kind == FEAB_PREC_FP64 ? (!op->v64 || !al(op->v64, 16))
                                 : (!op->vhi || !op->vlo || !op->gmask || !op->S || !al(op->vhi, 16) || !al(op->vlo, 8)))
    return FEAB_BAD_ARG;
  launch_sell_spmv(sell_view(A, op), x, y, s);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}
