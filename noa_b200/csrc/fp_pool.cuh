// Stream-ordered scratch allocations for the kernels that stage data (volume pair copy for extraction,
// interleaved accumulator for rasterization): one CUDA memory pool per device, created on first use
// with a release threshold that keeps freed blocks for reuse, so steady-state calls do not go back to
// the driver.
#pragma once

#include <cuda_runtime.h>

namespace nb {

// Allocates `bytes` on `stream` from this library's pool of the current device; nullptr on failure
// (the CUDA error is cleared: callers fall back to a path without scratch).
void* scratch_alloc(size_t bytes, cudaStream_t stream);
void scratch_free(void* ptr, cudaStream_t stream);

} // namespace nb
