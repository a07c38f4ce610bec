// Stream-ordered device memory for solver and batch state: a per-device pool
// owned by the library that keeps released blocks for reuse, so creating and
// destroying solves while others run causes no device-wide synchronisation
// (cudaMalloc / cudaFree do) and no repeated trips to the driver.  Memory is
// valid for work on the allocating stream from the allocation on, and is
// released in that stream's order.
#pragma once

#include <cuda_runtime.h>

namespace cfd {

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t stream);
cudaError_t pool_free(void* p, cudaStream_t stream);

}  // namespace cfd
