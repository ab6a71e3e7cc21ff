// Per-thread reuse of the solvers' CUDA graphs, events and pinned done flag.
//
// The PCG and block-PCG drivers replay a captured chunk of step kernels until the device says
// done.  Capturing a chunk is cheap; instantiating it is not, and a solver called in a loop
// (the SIMP optimality-criteria iterations, the modal subspace iteration's inner solves, the
// benchmark's repeated steps) would otherwise instantiate and destroy a graph on every call.
//
// GraphCache keeps a few instantiated graphs per thread.  A graph is keyed by the exact bytes of
// what its launches bake in (the kernel arguments struct, launch shapes, chunk length) and by the
// device.  A call with the same key replays the cached executable without capturing.  A call
// with a new key captures the chunk again and, when a cached graph has the same topology
// signature (same kernels and launch shapes, other arguments), updates that executable in place
// with cudaGraphExecUpdate; only otherwise does it instantiate a new one, evicting the least
// recently used.  Nothing here allocates device memory.
#pragma once
#include <cstring>
#include <vector>

#include "feab_common.cuh"

namespace feab {

// A 64-byte pinned host word the captured chunk copies the device's "done" state into.
struct HostFlag {
  volatile int32_t* ptr = nullptr;
  HostFlag() {
    void* p = nullptr;
    if (cudaHostAlloc(&p, 64, cudaHostAllocDefault) == cudaSuccess) ptr = static_cast<volatile int32_t*>(p);
  }
  ~HostFlag() {
    if (ptr) cudaFreeHost((void*)ptr);
  }
  HostFlag(const HostFlag&) = delete;
  HostFlag& operator=(const HostFlag&) = delete;
};

class GraphCache {
 public:
  static constexpr int kSlots = 4;
  static constexpr int kMaxDevices = 64;

  GraphCache() = default;
  GraphCache(const GraphCache&) = delete;
  GraphCache& operator=(const GraphCache&) = delete;

  ~GraphCache() {
    for (auto& s : slots_)
      if (s.exec) cudaGraphExecDestroy(s.exec);
    for (int d = 0; d < kMaxDevices; ++d) {
      if (capture_[d]) cudaStreamDestroy(capture_[d]);
      for (auto& e : events_[d])
        if (e) cudaEventDestroy(e);
    }
  }

  // Two timing-free events of the current device, created once per thread.
  cudaError_t events(cudaEvent_t (&ev)[2]) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    for (int i = 0; i < 2; ++i) {
      if (!events_[dev][i]) {
        e = cudaEventCreateWithFlags(&events_[dev][i], cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
      }
      ev[i] = events_[dev][i];
    }
    return cudaSuccess;
  }

  // The executable graph of the launches `record(stream)` issues, for `key` (exact contents)
  // and `topo` (topology signature).  *reused tells whether a cached executable was replayed
  // or updated in place rather than instantiated.
  template <class Record>
  cudaError_t acquire(const void* key, size_t key_bytes, uint64_t topo, Record&& record, cudaGraphExec_t* exec,
                      bool* reused = nullptr) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    ++clock_;
    const unsigned char* kb = static_cast<const unsigned char*>(key);
    for (auto& s : slots_) {
      if (s.exec && s.device == dev && s.topo == topo && s.key.size() == key_bytes &&
          std::memcmp(s.key.data(), kb, key_bytes) == 0) {
        s.stamp = clock_;
        *exec = s.exec;
        if (reused) *reused = true;
        return cudaSuccess;
      }
    }
    if (!capture_[dev]) {
      e = cudaStreamCreateWithFlags(&capture_[dev], cudaStreamNonBlocking);
      if (e != cudaSuccess) return e;
    }
    cudaGraph_t graph = nullptr;
    e = cudaStreamBeginCapture(capture_[dev], cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    record(capture_[dev]);
    e = cudaStreamEndCapture(capture_[dev], &graph);
    if (e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return e;
    }
    Slot* target = nullptr;
    for (auto& s : slots_)
      if (s.exec && s.device == dev && s.topo == topo) target = &s;
    bool updated = false;
    if (target) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(target->exec, graph, &info) == cudaSuccess) {
        updated = true;
      } else {
        cudaGetLastError();  // a refused update is not an error: instantiate instead
        cudaGraphExecDestroy(target->exec);
        target->exec = nullptr;
      }
    } else {
      target = &slots_[0];
      for (auto& s : slots_) {
        if (!s.exec) {
          target = &s;
          break;
        }
        if (s.stamp < target->stamp) target = &s;
      }
      if (target->exec) cudaGraphExecDestroy(target->exec);
      target->exec = nullptr;
    }
    if (!updated) {
      e = cudaGraphInstantiate(&target->exec, graph, 0);
      if (e != cudaSuccess) {
        target->exec = nullptr;
        cudaGraphDestroy(graph);
        return e;
      }
    }
    cudaGraphDestroy(graph);
    target->key.assign(kb, kb + key_bytes);
    target->topo = topo;
    target->device = dev;
    target->stamp = clock_;
    *exec = target->exec;
    if (reused) *reused = updated;
    return cudaSuccess;
  }

 private:
  struct Slot {
    std::vector<unsigned char> key;
    uint64_t topo = 0;
    int device = -1;
    cudaGraphExec_t exec = nullptr;
    uint64_t stamp = 0;
  };
  Slot slots_[kSlots];
  cudaStream_t capture_[kMaxDevices] = {};
  cudaEvent_t events_[kMaxDevices][2] = {};
  uint64_t clock_ = 0;
};

// Per-thread solver state: the pinned done flag and the graph cache.  It is created on a thread's
// first solve and deliberately never destroyed.  Destructors that run at thread or process exit
// would make CUDA calls while the CUDA runtime may already be shutting down (process exit), which
// can crash the exiting process after all its work is done.  So a thread that has solved keeps a
// 64-byte pinned word, at most kSlots graph executables, two events and one capture stream per
// device until the process ends.  ID separates the single- and multi-right-hand-side solvers.
struct SolverState {
  HostFlag flag;
  GraphCache graphs;
};

template <int ID>
inline SolverState& thread_solver_state() {
  static thread_local SolverState* state = nullptr;  // trivially destructible: no exit-time work
  if (!state) state = new SolverState();
  return *state;
}

// FNV-1a over a few integers: the topology signature of a captured chunk.
inline uint64_t topo_signature(std::initializer_list<int64_t> v) {
  uint64_t h = 1469598103934665603ull;
  for (int64_t x : v) {
    for (int b = 0; b < 8; ++b) {
      h ^= (uint64_t)((x >> (8 * b)) & 0xff);
      h *= 1099511628211ull;
    }
  }
  return h;
}

}  // namespace feab
