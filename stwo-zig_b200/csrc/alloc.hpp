// Device and pinned allocations of the provers and the op-level calls, with a
// test hook that makes the n-th allocation from now on fail as if the device
// were out of memory. The reference tests its failure paths the same way, with
// armed failures on the host (armOwnershipTransferFailureForTesting,
// src/backends/metal/runtime/ownership_testing.zig; fail-closed admission,
// src/prover/native/resource_admission.zig:73-89); nothing here touches the GPU.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

namespace sb {

// 0: disarmed; k > 0: the k-th allocation from now on fails (once).
inline std::atomic<int64_t>& alloc_fail_countdown() {
  static std::atomic<int64_t> n{0};
  return n;
}

inline bool alloc_fails_now() {
  std::atomic<int64_t>& n = alloc_fail_countdown();
  int64_t cur = n.load(std::memory_order_relaxed);
  while (cur > 0) {
    if (n.compare_exchange_weak(cur, cur - 1, std::memory_order_relaxed)) return cur == 1;
  }
  return false;
}

inline cudaError_t dev_malloc(void** p, size_t bytes) {
  if (alloc_fails_now()) { *p = nullptr; return cudaErrorMemoryAllocation; }
  return cudaMalloc(p, bytes);
}

inline cudaError_t dev_malloc_async(void** p, size_t bytes, cudaStream_t s) {
  if (alloc_fails_now()) { *p = nullptr; return cudaErrorMemoryAllocation; }
  return cudaMallocAsync(p, bytes, s);
}

inline cudaError_t host_malloc_pinned(void** p, size_t bytes) {
  if (alloc_fails_now()) { *p = nullptr; return cudaErrorMemoryAllocation; }
  return cudaMallocHost(p, bytes);
}

}  // namespace sb
