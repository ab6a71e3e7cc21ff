// Exclusive prefix sum of int32 counts (in place allowed) with a 64-bit total.
#pragma once
#include "feab_common.cuh"

namespace feab {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

inline int64_t scan_blocks(int64_t m) { return (m + kScanTile - 1) / kScanTile; }

// Scratch: (scan_blocks(m) + 2) int64.
// out[0..m] = exclusive scan of in[0..m-1]; out[m] = total (narrowed to int32).
// *d_total (device, int64) receives the exact total.  in == out is allowed.
cudaError_t scan_exclusive_i32(const int32_t* in, int32_t* out, int64_t m, int64_t* scratch,
                               int64_t* d_total, cudaStream_t s);

}  // namespace feab
