// Mesh topology and the CSR pattern of the reduced (free x free) stiffness.
//
// The reference builds the pattern implicitly: COO triples (row = repeat(g), col = tile(g))
// -> scipy CSR with duplicates summed -> K[np.ix_(free, free)]
// (fea_engine/src/fea_engine/vectorized_assembly.py:217-262, solver.py:1977-1978).  The
// structural pattern that produces is: row (a, i) holds every DOF (b, j) of every node b
// sharing an element with a, columns sorted.  Here it is built node-centrically:
//   node -> incident elements (sorted)  ->  node -> sorted distinct neighbour nodes
//   -> row lengths -> exclusive scan -> column fill through free_map.
// All integer work; the result is bit-identical to SciPy's int32 CSR.
#include "feab_common.cuh"
#include "feab_scan.cuh"

namespace feab {

int sm_count() {
  static int cached = 0;
  if (cached == 0) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    cached = v > 0 ? v : 148;
  }
  return cached;
}

namespace {

constexpr int kThreads = 256;
constexpr int kWarpsPerBlock = kThreads / 32;
constexpr int kMaxCand = 8 * FEAB_MAX_NODE_ELEMS;  // candidate neighbour slots per node

inline unsigned grid_for(int64_t work, int per_block) {
  int64_t g = (work + per_block - 1) / per_block;
  return (unsigned)(g < 1 ? 1 : g);
}

// Scratch layout shared by the topology calls.
struct TopoScratch {
  int32_t* counts;   // n_nodes + 1   (degrees, cursors, group flags)
  int32_t* counts2;  // 3*n_nodes + 1 (row lengths are scanned in place in row_ptr instead)
  int64_t* scan;     // scan tile sums
  int64_t* total;    // 1
  int32_t* maxv;     // 1
};

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

size_t scratch_layout(int32_t n_nodes, TopoScratch* out, void* base) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += align256(bytes);
    return o;
  };
  size_t o_counts = take(sizeof(int32_t) * ((size_t)n_nodes + 1));
  size_t o_counts2 = take(sizeof(int32_t) * (3 * (size_t)n_nodes + 1));
  int64_t nb = scan_blocks(3 * (int64_t)n_nodes + 1) + 2;
  size_t o_scan = take(sizeof(int64_t) * (size_t)nb);
  size_t o_total = take(sizeof(int64_t));
  size_t o_max = take(sizeof(int32_t));
  if (out && base) {
    char* b = static_cast<char*>(base);
    out->counts = reinterpret_cast<int32_t*>(b + o_counts);
    out->counts2 = reinterpret_cast<int32_t*>(b + o_counts2);
    out->scan = reinterpret_cast<int64_t*>(b + o_scan);
    out->total = reinterpret_cast<int64_t*>(b + o_total);
    out->maxv = reinterpret_cast<int32_t*>(b + o_max);
  }
  return off;
}

// ---------------------------------------------------------------- incidence
__global__ void k_incidence_count(const int32_t* __restrict__ conn, int64_t n_elem, int32_t n_nodes,
                                  int32_t* __restrict__ deg, feab_device_status* st) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elem) return;
  int v[8];
#pragma unroll
  for (int l = 0; l < 8; ++l) v[l] = conn[e * 8 + l];
  bool ok = true;
#pragma unroll
  for (int l = 0; l < 8; ++l) {
    if (v[l] < 0 || v[l] >= n_nodes) ok = false;
#pragma unroll
    for (int m = 0; m < l; ++m)
      if (v[m] == v[l]) ok = false;
  }
  if (!ok) {  // out-of-range or repeated node: reject the element, count nothing
    set_status(reinterpret_cast<int*>(st), FEAB_BAD_ARG, e);
    return;
  }
#pragma unroll
  for (int l = 0; l < 8; ++l) atomicAdd(&deg[v[l]], 1);
}

__global__ void k_max_i32(const int32_t* __restrict__ a, int64_t m, int32_t* __restrict__ out) {
  int best = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    best = max(best, a[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(FEAB_FULL_MASK, best, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

__global__ void k_incidence_fill(const int32_t* __restrict__ conn, int64_t n_elem, int32_t n_nodes,
                                 const int32_t* __restrict__ inc_ptr, int32_t* __restrict__ cursor,
                                 int32_t* __restrict__ inc_elem) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elem) return;
  int v[8];
  bool ok = true;
#pragma unroll
  for (int l = 0; l < 8; ++l) {
    v[l] = conn[e * 8 + l];
    if (v[l] < 0 || v[l] >= n_nodes) ok = false;
  }
#pragma unroll
  for (int l = 0; l < 8; ++l)
#pragma unroll
    for (int m = 0; m < l; ++m)
      if (v[m] == v[l]) ok = false;
  if (!ok) return;
#pragma unroll
  for (int l = 0; l < 8; ++l) {
    int slot = atomicAdd(&cursor[v[l]], 1);
    inc_elem[inc_ptr[v[l]] + slot] = (int32_t)e;
  }
}

// Per-node insertion sort: the fill order above depends on atomics; sorting makes the
// element lists (and so every later summation order) deterministic.
__global__ void k_incidence_sort(const int32_t* __restrict__ inc_ptr, int32_t* __restrict__ inc_elem,
                                 int32_t n_nodes) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n_nodes) return;
  int s = inc_ptr[a], t = inc_ptr[a + 1];
  for (int i = s + 1; i < t; ++i) {
    int key = inc_elem[i];
    int j = i - 1;
    while (j >= s && inc_elem[j] > key) {
      inc_elem[j + 1] = inc_elem[j];
      --j;
    }
    inc_elem[j + 1] = key;
  }
}

// ---------------------------------------------------------------- adjacency
// One warp per node: candidates = nodes of the incident elements (<= 8*64); the distinct
// ones, ranked, are the sorted neighbour list.  Quadratic in the candidate count, which
// is 64 on a structured hex mesh.
template <bool FILL>
__global__ void k_adjacency(const int32_t* __restrict__ conn, const int32_t* __restrict__ inc_ptr,
                            const int32_t* __restrict__ inc_elem, int32_t n_nodes,
                            int32_t* __restrict__ cnt, const int32_t* __restrict__ nbr_ptr,
                            int32_t* __restrict__ nbr_idx, feab_device_status* st) {
  __shared__ int32_t cand[kWarpsPerBlock][kMaxCand];
  __shared__ unsigned char first[kWarpsPerBlock][kMaxCand];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int a = blockIdx.x * kWarpsPerBlock + w;
  if (a >= n_nodes) return;
  const int s = inc_ptr[a], deg = inc_ptr[a + 1] - s;
  if (deg > FEAB_MAX_NODE_ELEMS) {
    if (lane == 0) set_status(reinterpret_cast<int*>(st), FEAB_CAPACITY, a);
    if (!FILL && lane == 0) cnt[a] = 0;
    return;
  }
  const int m = deg * 8;
  for (int t = lane; t < m; t += 32) cand[w][t] = conn[(int64_t)inc_elem[s + (t >> 3)] * 8 + (t & 7)];
  __syncwarp();
  int distinct = 0;
  for (int t = lane; t < m; t += 32) {
    int c = cand[w][t];
    bool f = true;
    for (int u = 0; u < t; ++u)
      if (cand[w][u] == c) {
        f = false;
        break;
      }
    first[w][t] = f;
    distinct += f;
  }
  distinct = warp_sum(distinct);
  if (!FILL) {
    if (lane == 0) {
      cnt[a] = distinct;
      if (distinct > FEAB_MAX_NODE_NBRS) set_status(reinterpret_cast<int*>(st), FEAB_CAPACITY, a);
    }
    return;
  }
  __syncwarp();
  const int base = nbr_ptr[a];
  for (int t = lane; t < m; t += 32) {
    if (!first[w][t]) continue;
    int c = cand[w][t], rank = 0;
    for (int u = 0; u < m; ++u) rank += (first[w][u] && cand[w][u] < c);
    nbr_idx[base + rank] = c;
  }
}

// ---------------------------------------------------------------- CSR pattern
__device__ __forceinline__ int nfree3(const int32_t* free_map, int b) {
  return (free_map[3 * b] >= 0) + (free_map[3 * b + 1] >= 0) + (free_map[3 * b + 2] >= 0);
}

// Row lengths written in place into row_ptr[r]; group flag per node into gflag[a].
__global__ void k_row_lengths(const int32_t* __restrict__ nbr_ptr, const int32_t* __restrict__ nbr_idx,
                              int32_t n_nodes, const int32_t* __restrict__ free_map, int32_t* __restrict__ row_len,
                              int32_t* __restrict__ gflag) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n_nodes) return;
  int fa = nfree3(free_map, a);
  if (gflag) gflag[a] = fa > 0 ? 1 : 0;
  if (fa == 0) return;
  int len = 0;
  for (int k = nbr_ptr[a]; k < nbr_ptr[a + 1]; ++k) len += nfree3(free_map, nbr_idx[k]);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    int r = free_map[3 * a + i];
    if (r >= 0) row_len[r] = len;
  }
}

__global__ void k_group_ptr(const int32_t* __restrict__ gidx, int32_t n_nodes, const int32_t* __restrict__ free_map,
                            int32_t n_free, int32_t* __restrict__ group_ptr) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a > n_nodes) return;
  if (a == n_nodes) {
    group_ptr[gidx[n_nodes]] = n_free;
    return;
  }
  if (gidx[a + 1] == gidx[a]) return;  // node without free DOFs
  int r = -1;
#pragma unroll
  for (int i = 2; i >= 0; --i)
    if (free_map[3 * a + i] >= 0) r = free_map[3 * a + i];
  group_ptr[gidx[a]] = r;
}

__global__ void k_col_fill(const int32_t* __restrict__ nbr_ptr, const int32_t* __restrict__ nbr_idx, int32_t n_nodes,
                           const int32_t* __restrict__ free_map, const int32_t* __restrict__ row_ptr,
                           int32_t* __restrict__ col_idx) {
  const int lane = threadIdx.x & 31;
  const int a = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  if (a >= n_nodes) return;
  int rows[3], nr = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    int r = free_map[3 * a + i];
    if (r >= 0) rows[nr++] = r;
  }
  if (nr == 0) return;
  const int s = nbr_ptr[a], nnb = nbr_ptr[a + 1] - s;
  int carry = 0;
  for (int k0 = 0; k0 < nnb; k0 += 32) {
    int k = k0 + lane;
    int b = k < nnb ? nbr_idx[s + k] : 0;
    int c0 = -1, c1 = -1, c2 = -1, fb = 0;
    if (k < nnb) {
      c0 = free_map[3 * b];
      c1 = free_map[3 * b + 1];
      c2 = free_map[3 * b + 2];
      fb = (c0 >= 0) + (c1 >= 0) + (c2 >= 0);
    }
    int incl = warp_incl_scan(fb, lane);
    int off = carry + incl - fb;
    if (k < nnb) {
      for (int q = 0; q < nr; ++q) {
        int p = row_ptr[rows[q]] + off;
        if (c0 >= 0) col_idx[p++] = c0;
        if (c1 >= 0) col_idx[p++] = c1;
        if (c2 >= 0) col_idx[p++] = c2;
      }
    }
    carry += __shfl_sync(FEAB_FULL_MASK, incl, 31);
  }
}

}  // namespace
}  // namespace feab

using namespace feab;

extern "C" size_t feab_topology_scratch_bytes(int32_t n_nodes, int64_t n_elem) {
  (void)n_elem;
  return scratch_layout(n_nodes, nullptr, nullptr);
}

extern "C" int32_t feab_node_incidence(const int32_t* conn, int64_t n_elem, int32_t n_nodes, int32_t* inc_ptr,
                                       int32_t* inc_elem, void* scratch, size_t scratch_bytes,
                                       feab_device_status* status, int32_t* max_elems_out, cudaStream_t s) {
  if (!conn || !inc_ptr || !inc_elem || !scratch || n_elem < 0 || n_nodes <= 0 || !status) return FEAB_BAD_ARG;
  if (8 * n_elem > INT32_MAX) return FEAB_BAD_ARG;
  TopoScratch sc;
  if (scratch_layout(n_nodes, &sc, scratch) > scratch_bytes) return FEAB_BAD_ARG;
  FEAB_CUDA(cudaMemsetAsync(sc.counts, 0, sizeof(int32_t) * ((size_t)n_nodes + 1), s));
  FEAB_CUDA(cudaMemsetAsync(sc.maxv, 0, sizeof(int32_t), s));
  if (n_elem > 0) count_launches(1);
  if (n_elem > 0) k_incidence_count<<<grid_for(n_elem, kThreads), kThreads, 0, s>>>(conn, n_elem, n_nodes, sc.counts, status);
  FEAB_CHECK_LAUNCH();
  k_max_i32<<<std::min<unsigned>(grid_for(n_nodes, kThreads), 1024), kThreads, 0, s>>>(sc.counts, n_nodes, sc.maxv);
  count_launches(1);
  FEAB_CUDA(scan_exclusive_i32(sc.counts, inc_ptr, n_nodes, sc.scan, sc.total, s));
  FEAB_CUDA(cudaMemsetAsync(sc.counts, 0, sizeof(int32_t) * ((size_t)n_nodes + 1), s));
  count_launches(n_elem > 0 ? 2 : 1);
  if (n_elem > 0)
    k_incidence_fill<<<grid_for(n_elem, kThreads), kThreads, 0, s>>>(conn, n_elem, n_nodes, inc_ptr, sc.counts, inc_elem);
  k_incidence_sort<<<grid_for(n_nodes, kThreads), kThreads, 0, s>>>(inc_ptr, inc_elem, n_nodes);
  FEAB_CHECK_LAUNCH();
  int32_t mx = 0;
  FEAB_CUDA(cudaMemcpyAsync(&mx, sc.maxv, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  FEAB_CUDA(cudaStreamSynchronize(s));
  if (max_elems_out) *max_elems_out = mx;
  return mx > FEAB_MAX_NODE_ELEMS ? FEAB_CAPACITY : FEAB_OK;
}

extern "C" int32_t feab_node_adjacency(const int32_t* conn, const int32_t* inc_ptr, const int32_t* inc_elem,
                                       int32_t n_nodes, int32_t* nbr_ptr, int32_t* nbr_idx, void* scratch,
                                       size_t scratch_bytes, feab_device_status* status, int64_t* total_out,
                                       int32_t* max_nbrs_out, cudaStream_t s) {
  if (!conn || !inc_ptr || !inc_elem || !nbr_ptr || !scratch || n_nodes <= 0 || !status) return FEAB_BAD_ARG;
  TopoScratch sc;
  if (scratch_layout(n_nodes, &sc, scratch) > scratch_bytes) return FEAB_BAD_ARG;
  const unsigned grid = grid_for(n_nodes, kWarpsPerBlock);
  if (nbr_idx == nullptr) {
    count_launches(2);
    k_adjacency<false><<<grid, kThreads, 0, s>>>(conn, inc_ptr, inc_elem, n_nodes, sc.counts, nullptr, nullptr, status);
    FEAB_CHECK_LAUNCH();
    FEAB_CUDA(cudaMemsetAsync(sc.maxv, 0, sizeof(int32_t), s));
    k_max_i32<<<std::min<unsigned>(grid_for(n_nodes, kThreads), 1024), kThreads, 0, s>>>(sc.counts, n_nodes, sc.maxv);
    FEAB_CUDA(scan_exclusive_i32(sc.counts, nbr_ptr, n_nodes, sc.scan, sc.total, s));
    int64_t tot = 0;
    int32_t mx = 0;
    FEAB_CUDA(cudaMemcpyAsync(&tot, sc.total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    FEAB_CUDA(cudaMemcpyAsync(&mx, sc.maxv, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    FEAB_CUDA(cudaStreamSynchronize(s));
    if (total_out) *total_out = tot;
    if (max_nbrs_out) *max_nbrs_out = mx;
    if (tot > INT32_MAX) return FEAB_CAPACITY;
    return mx > FEAB_MAX_NODE_NBRS ? FEAB_CAPACITY : FEAB_OK;
  }
  count_launches(1);
  k_adjacency<true><<<grid, kThreads, 0, s>>>(conn, inc_ptr, inc_elem, n_nodes, nullptr, nbr_ptr, nbr_idx, status);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}

extern "C" int32_t feab_csr_pattern(const int32_t* nbr_ptr, const int32_t* nbr_idx, int32_t n_nodes,
                                    const int32_t* free_map, int32_t n_free, int32_t* row_ptr, int32_t* group_ptr,
                                    int32_t* col_idx, void* scratch, size_t scratch_bytes, int64_t* nnz_out,
                                    int32_t* n_groups_out, cudaStream_t s) {
  if (!nbr_ptr || !nbr_idx || !free_map || !row_ptr || n_nodes <= 0 || n_free < 0 || !scratch) return FEAB_BAD_ARG;
  TopoScratch sc;
  if (scratch_layout(n_nodes, &sc, scratch) > scratch_bytes) return FEAB_BAD_ARG;
  if (col_idx == nullptr) {
    count_launches(1);
    k_row_lengths<<<grid_for(n_nodes, kThreads), kThreads, 0, s>>>(nbr_ptr, nbr_idx, n_nodes, free_map, row_ptr,
                                                                    sc.counts);
    FEAB_CHECK_LAUNCH();
    FEAB_CUDA(scan_exclusive_i32(row_ptr, row_ptr, n_free, sc.scan, sc.total, s));
    int64_t nnz = 0;
    FEAB_CUDA(cudaMemcpyAsync(&nnz, sc.total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    int64_t ng = 0;
    if (group_ptr) {
      // group index per node = exclusive scan of "node has a free DOF"
      FEAB_CUDA(scan_exclusive_i32(sc.counts, sc.counts2, n_nodes, sc.scan, sc.total, s));
      count_launches(1);
      k_group_ptr<<<grid_for((int64_t)n_nodes + 1, kThreads), kThreads, 0, s>>>(sc.counts2, n_nodes, free_map, n_free,
                                                                                 group_ptr);
      FEAB_CHECK_LAUNCH();
      FEAB_CUDA(cudaMemcpyAsync(&ng, sc.total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    }
    FEAB_CUDA(cudaStreamSynchronize(s));
    if (nnz_out) *nnz_out = nnz;
    if (n_groups_out) *n_groups_out = (int32_t)ng;
    return nnz > INT32_MAX ? FEAB_CAPACITY : FEAB_OK;
  }
  count_launches(1);
  k_col_fill<<<grid_for(n_nodes, kWarpsPerBlock), kThreads, 0, s>>>(nbr_ptr, nbr_idx, n_nodes, free_map, row_ptr,
                                                                     col_idx);
  FEAB_CHECK_LAUNCH();
  return FEAB_OK;
}
