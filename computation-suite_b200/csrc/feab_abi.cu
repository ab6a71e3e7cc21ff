// Library-level entry points: ABI version and status strings.
#include <atomic>
#include "feab_common.cuh"

namespace feab {
namespace {
std::atomic<uint64_t> g_launches{0};
}
void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace feab

extern "C" uint64_t feab_launch_count(void) { return feab::g_launches.load(); }

extern "C" int32_t feab_abi_version(void) { return 2; }

extern "C" const char* feab_status_string(int32_t code) {
  switch (code) {
    case FEAB_OK: return "ok";
    case FEAB_BAD_ARG: return "bad argument";
    case FEAB_DEGENERATE_ELEMENT: return "degenerate element(s) found (near-zero detJ)";
    case FEAB_ZERO_DIAGONAL: return "A has a zero diagonal entry";
    case FEAB_NOT_SPD: return "p^T A p <= 0: A is not SPD";
    case FEAB_NOT_CONVERGED: return "did not converge";
    case FEAB_CUDA_ERROR: return "CUDA error";
    case FEAB_CAPACITY: return "node valence beyond the kernels' limit";
    case FEAB_SCRATCH_LIMIT: return "problem too large for the fixed scratch of feab_pcg_solve_noalloc";
    default: return "unknown status";
  }
}

// The library carries its own (static) CUDA runtime, whose current device is per host thread;
// callers that drive a GPU other than device 0 select it here first (the Python layer does).
extern "C" int32_t feab_set_device(int32_t device) {
  return cudaSetDevice(device) == cudaSuccess ? FEAB_OK : FEAB_CUDA_ERROR;
}
