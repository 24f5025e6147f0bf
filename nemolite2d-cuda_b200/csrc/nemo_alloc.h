// Every device and page-locked allocation of the library goes through these
// two wrappers, so that a test can make the n-th of them report
// cudaErrorMemoryAllocation without allocating (nemo_debug_fail_alloc) and
// check each error path: the status, that nothing leaks, that the library
// stays usable.  The reference stops the program on a failed ALLOCATE
// (original/nemolite2d.f90:308); this library returns NEMO_ERR_ALLOC instead.
#pragma once

#include <cuda_runtime.h>

namespace nemo {

// Consumes one step of the countdown set by nemo_debug_fail_alloc; true for
// the allocation it designates.
bool alloc_should_fail();

template <class T>
inline cudaError_t dev_alloc(T** p, size_t bytes) {
  if (alloc_should_fail()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}

template <class T>
inline cudaError_t host_alloc(T** p, size_t bytes) {
  if (alloc_should_fail()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocHost(reinterpret_cast<void**>(p), bytes);
}

}  // namespace nemo
