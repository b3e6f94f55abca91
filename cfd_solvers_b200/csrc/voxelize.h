// Device triangle-surface voxelizer (voxelize.cu), used by the C ABI.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace cfdx {

// Planes z_first .. z_first + z_count - 1 (taken mod nz) of an nx x ny x nz
// voxel grid over [lo, hi]; solid cells get `value`, the others base[n] (a
// device array of the same nx*ny*z_count cells) or 0 without one.
struct VoxelRequest {
    std::size_t nx, ny, nz;
    double lo[3], hi[3];
    std::uint32_t z_first, z_count;
    std::uint8_t value;
    const std::uint8_t* base;
};

// Writes nx*ny*z_count bytes to out_device (on the current device, ordered
// on stream s; returns after the stream has finished).  Returns the first CUDA
// error (cudaErrorMemoryAllocation when a scratch buffer cannot be had) and
// names the failing step in *what.
cudaError_t voxelize_device(const double* host_tris, std::size_t count, const VoxelRequest& q,
                            std::uint8_t* out_device, cudaStream_t s, const char** what);

} // namespace cfdx
