// Field export of the engine (export.cu): the reference's legacy-VTK and JSON
// live-state writers, and the Q-criterion on the device.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace cfdx {

// Writers throw std::invalid_argument on size errors and std::runtime_error
// on I/O errors.  velocity: 3 doubles per cell (x, y, z) or nullptr; solid:
// one byte per cell or nullptr.
void write_vtk_3d(const char* path, std::size_t nx, std::size_t ny, std::size_t nz, const double* scalar,
                  const double* velocity, const std::uint8_t* solid, const char* name, bool binary);
void write_json_state_3d(const char* path, std::size_t nx, std::size_t ny, std::size_t nz, std::uint64_t step,
                         const double* scalar, const std::uint8_t* solid, const char* name);

// Q-criterion of a velocity field on the device, components at ux[n*stride],
// uy[n*stride], uz[n*stride] (float or double), into q (nx*ny*nz doubles).
cudaError_t launch_q_criterion(const void* ux, const void* uy, const void* uz, bool f64, std::size_t stride,
                               std::size_t nx, std::size_t ny, std::size_t nz, double dx, double dy, double dz,
                               double* q, cudaStream_t s);

} // namespace cfdx
