// Per-device, stream-ordered memory pool for the temporary buffers of single
// calls (voxelizer scratch, Q-criterion staging): scratch_pool.cu.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace cfdx {

// Bytes the pool keeps mapped between calls (memory above it is returned to the
// driver when a stream synchronises).
constexpr std::uint64_t kScratchKeep = 8ULL << 30;

// The current device's pool (created on first use).
cudaError_t scratch_pool(cudaMemPool_t* pool);
// Stream-ordered allocation / release from the current device's pool.
cudaError_t scratch_alloc(void** p, std::size_t bytes, cudaStream_t s);
void scratch_free(void* p, cudaStream_t s);
// Returns the pool's unused memory on `device` to the driver.
cudaError_t scratch_release(int device);

} // namespace cfdx
