// Device memory this library allocates on its own behalf:
//  * stream-ordered scratch for the kernels that stage data (volume pair copy for extraction,
//    interleaved accumulator for rasterization and the scatter insertion, batch descriptors of one-shot
//    launches): one CUDA memory pool per device, created on first use with a release threshold that
//    keeps freed blocks for reuse, so steady-state calls do not go back to the driver;
//  * the long-lived buffers of a captured batch (descriptors, pair copies), from cudaMalloc.
// Both go through a per-device cap on the size of one allocation (nb_set_scratch_limit): a request
// above it fails as if the device were out of memory, and the caller takes its path without it.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace nb {

// Allocates `bytes` on `stream` from this library's pool of the current device; nullptr on failure
// or above the device's cap (the CUDA error is cleared: callers fall back to a path without scratch).
void* scratch_alloc(size_t bytes, cudaStream_t stream);
void scratch_free(void* ptr, cudaStream_t stream);

// cudaMalloc on the current device under the same cap; nullptr on failure (error cleared).
void* device_alloc(size_t bytes);

// The cap of `device` in bytes (-1: none). Setting a negative value removes it.
bool set_scratch_limit(int device, int64_t bytes);
int64_t scratch_limit(int device);

// How many allocations scratch_alloc and device_alloc refused on `device` since the library loaded
// (-1 for a bad device index).
int64_t refused_allocations(int device);

// Copies `bytes` (a multiple of 4) of host memory to device memory in stream order, in a form a
// stream capture records safely: while `stream` is capturing, the bytes travel as the parameters of
// small copy kernels (a graph keeps its own copy of every launch's parameters), so replays never read
// the host buffer; otherwise by cudaMemcpyAsync (the runtime stages pageable memory before
// returning). Either way the host buffer may be released as soon as this returns.
cudaError_t upload_async(void* dst, const void* src, size_t bytes, cudaStream_t stream);

// Whether `stream` is being captured into a graph (false if the query fails).
bool stream_capturing(cudaStream_t stream);

} // namespace nb
