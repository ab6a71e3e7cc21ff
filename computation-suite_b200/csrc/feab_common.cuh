// Shared helpers for the feab200 CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "feab200.h"

#define FEAB_WARP 32
#define FEAB_FULL_MASK 0xffffffffu

// Launch-time error check: maps any pending CUDA error to FEAB_CUDA_ERROR.
#define FEAB_CHECK_LAUNCH()                                  \
  do {                                                       \
    cudaError_t _e = cudaGetLastError();                     \
    if (_e != cudaSuccess) return FEAB_CUDA_ERROR;           \
  } while (0)

#define FEAB_CUDA(call)                                      \
  do {                                                       \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return FEAB_CUDA_ERROR;           \
  } while (0)

namespace feab {

// Records the first device-side error: status word 0 -> code, plus the offending index.
__device__ __forceinline__ void set_status(int* status, int code, long long where) {
  if (status == nullptr) return;
  if (atomicCAS(status, 0, code) == 0) {
    // index slot lives right after the code word
    reinterpret_cast<volatile long long*>(status + 2)[0] = where;
  }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FEAB_FULL_MASK, v, o);
  return v;
}

__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(FEAB_FULL_MASK, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide sum of NV doubles; result valid in thread 0.  `sh` needs NV*32 doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[k * 32 + wid] = v[k];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = lane < nw ? sh[k * 32 + lane] : 0.0;
      v[k] = warp_sum(t);
    }
  }
  __syncthreads();
}

// Number of SMs of the current device, cached per process.
int sm_count();

// Library-wide count of kernel launches (feab_launch_count).
void count_launches(uint64_t n);

}  // namespace feab
