// Device and pinned-host allocations of the library's handles and batches.
//
// A server that admits and retires simulations every few steps creates and
// destroys handles continuously.  cudaFree and cudaFreeHost wait for the whole
// device, so each retirement would stall every other simulation's work in
// flight.  With the allocation cache enabled for a device (see
// fluid_pp_set_allocation_cache), a released block waits only for the stream
// that last used it and then goes to a per-device free list, from which a
// later allocation of a similar size takes it without any CUDA call.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace fpp {

// Device memory on the current device: a cached block of at least `bytes`
// (at most a quarter larger) or a new cudaMalloc.
cudaError_t dev_alloc(void** p, size_t bytes);
// Returns p to its device's cache once `last_use` has drained, or frees it
// when the cache is off or full.  p may be null.
void dev_release(void* p, cudaStream_t last_use);

// Pinned host memory, cached like device memory under device key -1.
cudaError_t host_alloc(void** p, size_t bytes);
void host_release(void* p, cudaStream_t last_use);

// Orders `next` after the work already issued to `prev` (an event recorded on
// prev that next waits for), so a handle moved to another stream never runs
// beside its own earlier work.  No-op when the two are the same stream.
cudaError_t order_streams(cudaStream_t prev, cudaStream_t next);

}  // namespace fpp
