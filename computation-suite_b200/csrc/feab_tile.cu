// Node tiles of the block SpMM (feab_tile_operator): FEAB_TILE_GROUPS consecutive node row
// groups of one problem, their column lists merged into one sorted union with a per-column mask
// of the groups that have it, and the values re-ordered to (union column, group, row).
//
// Build steps (all on the device):
//   1. tiles per problem = ceil(groups / T), exclusive scan -> first tile of each problem;
//   2. one thread per tile: its first group, the tile of each of its groups;
//   3. one thread per tile: T-way merge of the sorted column lists, counting the union (padded to
//      a multiple of 4) and the (column, group) pairs; exclusive scans -> uoff, poff;
//   4. (build) one thread per tile: the same merge twice, counting then writing ucol / umask /
//      upair grouped by mask (all columns of mask 1, then of mask 2, ..., ascending columns within
//      a mask), so that the SpMM walks runs of columns shared by the same groups;
//   5. (build) one warp per group: each list entry finds its mask (binary searches in the tile's
//      lists), its mask's run and its column there, and writes its rows' values at
//      3 * (poff + upair + rank of the group among the mask's set bits) + row.
#include <algorithm>
#include <climits>
#include "feab_common.cuh"
#include "feab_scan.cuh"

namespace feab {
namespace {

constexpr int kT = FEAB_TILE_GROUPS;
constexpr int kChunk = FEAB_TILE_CHUNK;
constexpr int kThreads = 256;
constexpr int32_t kColMask = 0x3fffffff;  // the difference form tags columns with the DOF component

size_t a256(size_t b) { return (b + 255) & ~size_t(255); }

// The column list of row group g: the CSR row of its first row (FP64), or the difference form's
// off-node columns without the padding (MIXED).
struct Lists {
  const int32_t* group_ptr;
  const int32_t* row_ptr;
  const int32_t* col_idx;
  const int32_t* goff;   // MIXED: the difference form's tagged columns
  const int32_t* tcol;
  bool diff;
  __device__ __forceinline__ void get(int g, const int32_t*& cols, int& len) const {
    const int r0 = group_ptr[g], f = group_ptr[g + 1] - r0;
    const int s0 = row_ptr[r0], rl = row_ptr[r0 + 1] - s0;
    if (diff) {
      cols = tcol + goff[g];
      len = rl - f;
    } else {
      cols = col_idx + s0;
      len = rl;
    }
  }
};

__global__ void k_tiles_per_problem(int32_t P, int32_t G, const int32_t* __restrict__ pg, int32_t* __restrict__ pt,
                                    int32_t* __restrict__ err) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const int a = pg[p], b = pg[p + 1];
  if (a < 0 || b <= a || b > G || (p == 0 && a != 0) || (p == P - 1 && b != G)) atomicExch(err, 1);
  pt[p] = b > a ? (b - a + kT - 1) / kT : 0;
}

// tile_g0[t] for t < n_tiles and tile_g0[n_tiles] = G; group_tile (may be null)
__global__ void k_tile_map(int32_t n_tiles, int32_t P, int32_t G, const int32_t* __restrict__ pg,
                           const int32_t* __restrict__ pt, int32_t* __restrict__ tile_g0,
                           int32_t* __restrict__ group_tile) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t > n_tiles) return;
  if (t == n_tiles) {
    tile_g0[t] = G;
    return;
  }
  int lo = 0, hi = P;  // the problem p with pt[p] <= t < pt[p + 1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pt[mid] <= t) lo = mid;
    else hi = mid;
  }
  const int g0 = pg[lo] + (t - pt[lo]) * kT, g1 = min(g0 + kT, pg[lo + 1]);
  tile_g0[t] = g0;
  if (group_tile)
    for (int g = g0; g < g1; ++g) group_tile[g] = t;
}

// The order of masks within a tile: 1, 2, ..., 2^T - 1, then the padding (mask 0).
__device__ __forceinline__ int mask_key(int m) { return m == 0 ? 1 << kT : m; }

// The merged union of tile t's lists, in ascending column order: calls emit(column, mask).
template <typename F>
__device__ __forceinline__ void merge_tile(const Lists& Ls, int g0, int nt, F&& emit) {
  const int32_t* L[kT];
  int len[kT], h[kT];
#pragma unroll
  for (int j = 0; j < kT; ++j) {
    L[j] = nullptr;
    len[j] = 0;
    h[j] = 0;
    if (j < nt) Ls.get(g0 + j, L[j], len[j]);
  }
  while (true) {
    int c = INT_MAX;
#pragma unroll
    for (int j = 0; j < kT; ++j)
      if (h[j] < len[j]) c = min(c, L[j][h[j]] & kColMask);
    if (c == INT_MAX) break;
    int m = 0;
#pragma unroll
    for (int j = 0; j < kT; ++j)
      if (h[j] < len[j] && (L[j][h[j]] & kColMask) == c) {
        m |= 1 << j;
        ++h[j];
      }
    emit(c, m);
  }
}

// count mode (ucol == null): ucnt[t] = union padded to 4, pcnt[t] = pairs.  write mode: the
// union from uoff[t], grouped by mask (mask_key order, ascending columns within a mask), each
// column with its first pair within the tile; padding columns (the tile's last column, mask 0)
// at the end.
__global__ void k_tile_merge(int32_t n_tiles, Lists Ls, const int32_t* __restrict__ tile_g0,
                             int32_t* __restrict__ ucnt, int32_t* __restrict__ pcnt, int32_t* __restrict__ ccnt,
                             const int32_t* __restrict__ uoff, const int32_t* __restrict__ poff,
                             const int32_t* __restrict__ cptr, int32_t* __restrict__ ucol,
                             uint8_t* __restrict__ umask, int32_t* __restrict__ upair, int4* __restrict__ chunk) {
  constexpr int NM = 1 << kT;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tiles) return;
  const int g0 = tile_g0[t], nt = tile_g0[t + 1] - g0;
  int cnt[NM];
#pragma unroll
  for (int m = 0; m < NM; ++m) cnt[m] = 0;
  int nu = 0, np = 0, last = 0;
  merge_tile(Ls, g0, nt, [&](int c, int m) {
    ++cnt[m];
    np += __popc(m);
    last = c;
    ++nu;
  });
  const int padded = (nu + 3) & ~3;
  if (!ucol) {
    ucnt[t] = padded;
    pcnt[t] = np;
    ccnt[t] = (padded + kChunk - 1) / kChunk;
    return;
  }
  // bucket starts (columns and pairs) in mask_key order
  int pos[NM], pair[NM];
  int cu = 0, cp = 0;
#pragma unroll
  for (int m = 1; m < NM; ++m) {
    pos[m] = cu;
    pair[m] = cp;
    cu += cnt[m];
    cp += cnt[m] * __popc(m);
  }
  const int base = uoff[t];
  merge_tile(Ls, g0, nt, [&](int c, int m) {
    const int i = base + pos[m]++;
    ucol[i] = c;
    umask[i] = (uint8_t)m;
    upair[i] = pair[m];
    pair[m] += __popc(m);
  });
  for (int u = nu; u < padded; ++u) {
    ucol[base + u] = last;
    umask[base + u] = 0;
    upair[base + u] = np;
  }
  // chunk descriptors: first union column, columns, first value, values
  const int64_t v0 = 3 * (int64_t)poff[t];
  for (int c = 0, q = cptr[t]; c < padded; c += kChunk, ++q) {
    const int nc = min(kChunk, padded - c);
    const int pa = upair[base + c], pe = c + kChunk < padded ? upair[base + c + kChunk] : np;
    chunk[q] = make_int4(base + c, nc, (int)(v0 + 3 * pa), 3 * (pe - pa));
  }
}

// One warp per row group: every list entry's rows go to their (union column, group) pair.
__global__ void __launch_bounds__(kThreads) k_tile_values(int32_t G, Lists Ls, const double* __restrict__ vals64,
                                                         const uint32_t* __restrict__ dvhi,
                                                         const uint16_t* __restrict__ dvlo,
                                                         const uint8_t* __restrict__ dvlo2,
                                                         const int32_t* __restrict__ dvoff,
                                                         const int32_t* __restrict__ tile_g0,
                                                         const int32_t* __restrict__ group_tile,
                                                         const int32_t* __restrict__ uoff,
                                                         const int32_t* __restrict__ poff,
                                                         const int32_t* __restrict__ ucol,
                                                         const uint8_t* __restrict__ umask,
                                                         const int32_t* __restrict__ upair, double* __restrict__ v64,
                                                         uint32_t* __restrict__ vhi, uint16_t* __restrict__ vlo,
                                                         uint8_t* __restrict__ vlo2, int32_t* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (g >= G) return;
  const int t = group_tile[g], j = g - tile_g0[t];
  const int u0 = uoff[t], nu = uoff[t + 1] - u0;
  const int64_t p0 = poff[t];
  const int r0 = Ls.group_ptr[g], f = Ls.group_ptr[g + 1] - r0;
  const int32_t* cols;
  int len;
  Ls.get(g, cols, len);
  // difference form: the group's values are f rows of lp (padded) entries from dvoff[g]
  const int lp = Ls.diff ? Ls.goff[g + 1] - Ls.goff[g] : 0;
  // the tile's lists, to find which groups share a column
  const int g0 = tile_g0[t], nt = tile_g0[t + 1] - g0;
  const int32_t* TL[kT];
  int tlen[kT];
#pragma unroll
  for (int q = 0; q < kT; ++q) {
    TL[q] = nullptr;
    tlen[q] = 0;
    if (q < nt) Ls.get(g0 + q, TL[q], tlen[q]);
  }
  for (int i = lane; i < len; i += 32) {
    const int c = cols[i] & kColMask;
    int mc = 0;
#pragma unroll
    for (int q = 0; q < kT; ++q) {
      int lo = 0, hi = tlen[q];
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((TL[q][mid] & kColMask) < c) lo = mid + 1;
        else hi = mid;
      }
      if (lo < tlen[q] && (TL[q][lo] & kColMask) == c) mc |= 1 << q;
    }
    // the bucket of mask mc: umask is ordered by mask_key within the tile
    int blo = 0, bhi = nu;
    while (blo < bhi) {
      const int mid = (blo + bhi) >> 1;
      if (mask_key(umask[u0 + mid]) < mask_key(mc)) blo = mid + 1;
      else bhi = mid;
    }
    int lo = blo, hi = nu;  // the bucket ends where the key grows
    {
      int e0 = blo, e1 = nu;
      while (e0 < e1) {
        const int mid = (e0 + e1) >> 1;
        if (mask_key(umask[u0 + mid]) <= mask_key(mc)) e0 = mid + 1;
        else e1 = mid;
      }
      hi = e0;
    }
    while (lo < hi) {  // first column >= c within the bucket
      const int mid = (lo + hi) >> 1;
      if (ucol[u0 + mid] < c) lo = mid + 1;
      else hi = mid;
    }
    if (!((mc >> j) & 1) || lo >= nu || ucol[u0 + lo] != c || umask[u0 + lo] != mc) {
      atomicExch(err, 1);
      continue;
    }
    const int m = umask[u0 + lo];
    const int64_t v = 3 * (p0 + upair[u0 + lo] + __popc(m & ((1 << j) - 1)));
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (Ls.diff) {
        uint32_t hv = 0u;
        uint16_t lv = 0;
        uint8_t l2 = 0;
        if (k < f) {
          const int64_t q = (int64_t)dvoff[g] + (int64_t)k * lp + i;
          hv = dvhi[q];
          lv = dvlo[q];
          l2 = dvlo2[q];
        }
        vhi[v + k] = hv;
        vlo[v + k] = lv;
        vlo2[v + k] = l2;
      } else {
        v64[v + k] = k < f ? vals64[Ls.row_ptr[r0 + k] + i] : 0.0;
      }
    }
  }
}

struct TileScratch {
  int32_t* pt;      // n_problems + 1
  int32_t* tg0;     // count mode: tile_g0 (n_groups + 1)
  int32_t* ucnt;    // n_groups + 1
  int32_t* pcnt;    // n_groups + 1
  int32_t* ccnt;    // n_groups + 1
  int64_t* scan;
  int64_t* total;   // 1
  int32_t* err;     // 1
  size_t bytes;
};

TileScratch scratch_layout(int32_t G, int32_t P, char* base) {
  TileScratch X{};
  size_t off = 0;
  auto take = [&](size_t b) {
    char* p = base ? base + off : nullptr;
    off += a256(b);
    return p;
  };
  X.pt = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * ((size_t)P + 1)));
  X.tg0 = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * ((size_t)G + 1)));
  X.ucnt = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * ((size_t)G + 1)));
  X.pcnt = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * ((size_t)G + 1)));
  X.ccnt = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * ((size_t)G + 1)));
  const int64_t m = std::max<int64_t>((int64_t)G + 1, (int64_t)P + 1);
  X.scan = reinterpret_cast<int64_t*>(take(sizeof(int64_t) * ((size_t)scan_blocks(m) + 2)));
  X.total = reinterpret_cast<int64_t*>(take(sizeof(int64_t)));
  X.err = reinterpret_cast<int32_t*>(take(sizeof(int32_t)));
  X.bytes = off;
  return X;
}

// Storage layout of the operator for n_tiles tiles, nu union columns and np pairs.
size_t storage_layout(int32_t n_tiles, int32_t G, int64_t nu, int64_t np, int64_t nch, int prec, char* base,
                      feab_tile_operator* T) {
  size_t off = 0;
  auto take = [&](size_t b) {
    char* p = base ? base + off : nullptr;
    off += a256(b);
    return p;
  };
  char* tg = take(sizeof(int32_t) * ((size_t)n_tiles + 1));
  char* gt = take(sizeof(int32_t) * (size_t)G);
  char* uo = take(sizeof(int32_t) * ((size_t)n_tiles + 1));
  char* po = take(sizeof(int32_t) * ((size_t)n_tiles + 1));
  char* uc = take(sizeof(int32_t) * (size_t)nu);
  char* up = take(sizeof(int32_t) * (size_t)nu);
  char* um = take((size_t)nu);
  char* cp = take(sizeof(int32_t) * ((size_t)n_tiles + 1));
  char* ch = take(sizeof(int4) * (size_t)nch);
  char *v64 = nullptr, *hi = nullptr, *lo = nullptr, *lo2 = nullptr;
  const size_t nv = 3 * (size_t)np;
  if (prec == FEAB_PREC_FP64) {
    v64 = take(sizeof(double) * nv);
  } else {
    hi = take(sizeof(uint32_t) * nv);
    lo = take(sizeof(uint16_t) * nv);
    lo2 = take(nv);
  }
  if (T) {
    T->tile_g0 = reinterpret_cast<int32_t*>(tg);
    T->group_tile = reinterpret_cast<int32_t*>(gt);
    T->uoff = reinterpret_cast<int32_t*>(uo);
    T->poff = reinterpret_cast<int32_t*>(po);
    T->ucol = reinterpret_cast<int32_t*>(uc);
    T->upair = reinterpret_cast<int32_t*>(up);
    T->umask = reinterpret_cast<uint8_t*>(um);
    T->v64 = reinterpret_cast<double*>(v64);
    T->vhi = reinterpret_cast<uint32_t*>(hi);
    T->vlo = reinterpret_cast<uint16_t*>(lo);
    T->vlo2 = reinterpret_cast<uint8_t*>(lo2);
    T->cptr = reinterpret_cast<int32_t*>(cp);
    T->chunk = reinterpret_cast<int32_t*>(ch);
  }
  return off;
}

}  // namespace
}  // namespace feab

using namespace feab;

extern "C" size_t feab_tile_scratch_bytes(int32_t n_groups, int32_t n_problems) {
  if (n_groups <= 0 || n_problems <= 0) return 0;
  return scratch_layout(n_groups, n_problems, nullptr).bytes;
}

extern "C" int32_t feab_tile_operator_build(const feab_csr* M, const feab_diff_operator* D,
                                            const int32_t* problem_groups, int32_t P, int32_t prec, void* scratch,
                                            size_t scratch_bytes, void* storage, size_t storage_bytes,
                                            size_t* bytes_out, feab_tile_operator* out, cudaStream_t s) {
  if (!M || !problem_groups || P <= 0 || !scratch || !M->group_ptr || M->n_groups <= 0 || !M->row_ptr ||
      !M->col_idx || !M->vals64)
    return FEAB_BAD_ARG;
  if (prec != FEAB_PREC_FP64 && prec != FEAB_PREC_MIXED) return FEAB_BAD_ARG;
  if (prec == FEAB_PREC_MIXED && (!D || !D->tcol || !D->goff || !D->voff || !D->vhi || !D->vlo || !D->vlo2))
    return FEAB_BAD_ARG;
  if (storage && (!out || (reinterpret_cast<uintptr_t>(storage) & 15u))) return FEAB_BAD_ARG;
  if (!storage && !bytes_out) return FEAB_BAD_ARG;
  const int32_t G = M->n_groups;
  if (P > G) return FEAB_BAD_ARG;
  if (scratch_layout(G, P, nullptr).bytes > scratch_bytes) return FEAB_BAD_ARG;
  const TileScratch X = scratch_layout(G, P, static_cast<char*>(scratch));
  FEAB_CUDA(cudaMemsetAsync(X.err, 0, sizeof(int32_t), s));
  k_tiles_per_problem<<<(P + kThreads - 1) / kThreads, kThreads, 0, s>>>(P, G, problem_groups, X.pt, X.err);
  count_launches(1);
  FEAB_CHECK_LAUNCH();
  FEAB_CUDA(scan_exclusive_i32(X.pt, X.pt, P, X.scan, X.total, s));
  int64_t n_tiles64 = 0;
  int32_t err = 0;
  FEAB_CUDA(cudaMemcpyAsync(&n_tiles64, X.total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaMemcpyAsync(&err, X.err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaStreamSynchronize(s));
  if (err || n_tiles64 <= 0 || n_tiles64 > G) return FEAB_BAD_ARG;
  const int32_t n_tiles = (int32_t)n_tiles64;
  Lists Ls{M->group_ptr, M->row_ptr, M->col_idx, D ? D->goff : nullptr, D ? D->tcol : nullptr,
           prec == FEAB_PREC_MIXED};
  const int tb = (n_tiles + 1 + kThreads - 1) / kThreads;
  // counts: tile map into scratch, merge counts, totals
  k_tile_map<<<tb, kThreads, 0, s>>>(n_tiles, P, G, problem_groups, X.pt, X.tg0, nullptr);
  k_tile_merge<<<tb, kThreads, 0, s>>>(n_tiles, Ls, X.tg0, X.ucnt, X.pcnt, X.ccnt, nullptr, nullptr, nullptr, nullptr,
                                       nullptr, nullptr, nullptr);
  count_launches(2);
  FEAB_CHECK_LAUNCH();
  int64_t nu = 0, np = 0;
  FEAB_CUDA(scan_exclusive_i32(X.ucnt, X.ucnt, n_tiles, X.scan, X.total, s));
  FEAB_CUDA(cudaMemcpyAsync(&nu, X.total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaStreamSynchronize(s));
  FEAB_CUDA(scan_exclusive_i32(X.pcnt, X.pcnt, n_tiles, X.scan, X.total, s));
  FEAB_CUDA(cudaMemcpyAsync(&np, X.total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaStreamSynchronize(s));
  int64_t nch = 0;
  FEAB_CUDA(scan_exclusive_i32(X.ccnt, X.ccnt, n_tiles, X.scan, X.total, s));
  FEAB_CUDA(cudaMemcpyAsync(&nch, X.total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaStreamSynchronize(s));
  if (nu >= (int64_t)INT32_MAX || 3 * np >= (int64_t)INT32_MAX) return FEAB_CAPACITY;
  const size_t need = storage_layout(n_tiles, G, nu, np, nch, prec, nullptr, nullptr);
  if (bytes_out) *bytes_out = need;
  if (!storage) return FEAB_OK;
  if (need > storage_bytes) return FEAB_BAD_ARG;
  feab_tile_operator T{};
  storage_layout(n_tiles, G, nu, np, nch, prec, static_cast<char*>(storage), &T);
  T.n_tiles = n_tiles;
  T.precision = prec;
  T.n_groups = G;
  // the scanned counts are the offsets
  FEAB_CUDA(cudaMemcpyAsync(T.uoff, X.ucnt, sizeof(int32_t) * ((size_t)n_tiles + 1), cudaMemcpyDeviceToDevice, s));
  FEAB_CUDA(cudaMemcpyAsync(T.poff, X.pcnt, sizeof(int32_t) * ((size_t)n_tiles + 1), cudaMemcpyDeviceToDevice, s));
  FEAB_CUDA(cudaMemcpyAsync(T.cptr, X.ccnt, sizeof(int32_t) * ((size_t)n_tiles + 1), cudaMemcpyDeviceToDevice, s));
  k_tile_map<<<tb, kThreads, 0, s>>>(n_tiles, P, G, problem_groups, X.pt, T.tile_g0, T.group_tile);
  k_tile_merge<<<tb, kThreads, 0, s>>>(n_tiles, Ls, T.tile_g0, nullptr, nullptr, nullptr, T.uoff, T.poff, T.cptr,
                                       T.ucol, T.umask, T.upair, reinterpret_cast<int4*>(T.chunk));
  const int wpb = kThreads / 32;
  k_tile_values<<<(G + wpb - 1) / wpb, kThreads, 0, s>>>(
      G, Ls, M->vals64, D ? D->vhi : nullptr, D ? D->vlo : nullptr, D ? D->vlo2 : nullptr, D ? D->voff : nullptr,
      T.tile_g0, T.group_tile, T.uoff, T.poff, T.ucol, T.umask, T.upair, T.v64, T.vhi, T.vlo, T.vlo2, X.err);
  count_launches(3);
  FEAB_CHECK_LAUNCH();
  FEAB_CUDA(cudaMemcpyAsync(&err, X.err, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaStreamSynchronize(s));
  if (err) return FEAB_BAD_ARG;
  *out = T;
  return FEAB_OK;
}
