// Three-pass exclusive scan: tile sums -> single-block scan of tile sums -> tile scan + offset.
#include "feab_scan.cuh"

namespace feab {

namespace {

__device__ __forceinline__ long long block_excl_scan_ll(long long v, long long* sh, long long* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long t = __shfl_up_sync(FEAB_FULL_MASK, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) sh[wid] = x;
  __syncthreads();
  if (wid == 0) {
    long long w = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
    long long y = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      long long t = __shfl_up_sync(FEAB_FULL_MASK, y, o);
      if (lane >= o) y += t;
    }
    sh[32 + lane] = y - w;  // exclusive warp offsets
    if (lane == 31) sh[64] = y;
  }
  __syncthreads();
  long long r = sh[32 + wid] + x - v;
  *total = sh[64];
  __syncthreads();
  return r;
}

__global__ void k_tile_sums(const int32_t* __restrict__ in, int64_t m, int64_t* __restrict__ sums) {
  __shared__ long long sh[65];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < m) s += in[base + k];
  long long tot;
  block_excl_scan_ll(s, sh, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// One block scans all tile sums sequentially in chunks of blockDim.x.
__global__ void k_scan_sums(int64_t* __restrict__ sums, int64_t nb, int64_t* __restrict__ d_total) {
  __shared__ long long sh[65];
  long long carry = 0;
  for (int64_t c = 0; c < nb; c += blockDim.x) {
    int64_t i = c + threadIdx.x;
    long long v = i < nb ? sums[i] : 0;
    long long tot;
    long long e = block_excl_scan_ll(v, sh, &tot);
    if (i < nb) sums[i] = carry + e;
    carry += tot;
  }
  if (threadIdx.x == 0) *d_total = carry;
}

__global__ void k_tile_scan(const int32_t* in, int32_t* out, int64_t m, const int64_t* __restrict__ offs,
                            const int64_t* __restrict__ d_total) {
  __shared__ long long sh[65];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int32_t v[kScanItems];
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < m) ? in[base + k] : 0;
    s += v[k];
  }
  long long tot;
  long long e = block_excl_scan_ll(s, sh, &tot) + offs[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < m) out[base + k] = (int32_t)e;
    e += v[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[m] = (int32_t)(*d_total);
}

}  // namespace

cudaError_t scan_exclusive_i32(const int32_t* in, int32_t* out, int64_t m, int64_t* scratch,
                               int64_t* d_total, cudaStream_t s) {
  const int64_t nb = scan_blocks(m);
  if (nb == 0) {
    cudaMemsetAsync(d_total, 0, sizeof(int64_t), s);
    return cudaMemsetAsync(out, 0, sizeof(int32_t), s);
  }
  k_tile_sums<<<(unsigned)nb, kScanThreads, 0, s>>>(in, m, scratch);
  k_scan_sums<<<1, 1024, 0, s>>>(scratch, nb, d_total);
  k_tile_scan<<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, m, scratch, d_total);
  count_launches(3);
  return cudaGetLastError();
}

}  // namespace feab
