// Resident solvers coupled to the flow through its device views (resident.cu):
// the reference's ResidentFreeSurfaceSycl3D, ResidentParticlesSycl3D and
// ResidentFlowDiagnosticsSycl3D (resident_multiphysics_sycl.hpp:202-411).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "thermal.h"

namespace cfdx {

cudaError_t launch_fill_uniform(float* fill, ThermalGrid t, float value, cudaStream_t s);
cudaError_t launch_fill_half_space_x(float* fill, ThermalGrid t, float interface_x, cudaStream_t s);
// upwind advection of the fill by the face velocities, clamped to [0, 1]
cudaError_t launch_fill_advect(const float* fill, float* out, ThermalGrid t, const float* ux, const float* uy,
                               const float* uz, float dt, cudaStream_t s);
// geometry = normals x | y | z | curvature (4 * cells)
cudaError_t launch_fill_geometry(const float* fill, float* geometry, ThermalGrid t, cudaStream_t s);
cudaError_t launch_surface_tension(const float* fill, const float* curvature, ThermalGrid t, float* ax, float* ay,
                                   float* az, float sigma, float density, cudaStream_t s);
// FP64 sum of `count` floats into out[0] (partials: `blocks` doubles)
cudaError_t launch_sum_floats(const float* v, std::size_t count, double* partials, int blocks, double* out,
                              cudaStream_t s);
// particles: state = x | y | z | vx | vy | vz | mass | response (8 * count floats)
cudaError_t launch_particles_advance(float* state, std::uint32_t count, ThermalGrid t, const float* ux,
                                     const float* uy, const float* uz, float* ax, float* ay, float* az, float dt,
                                     bool two_way, float gx, float gy, float gz, cudaStream_t s);
// periodic FP32 Q-criterion
cudaError_t launch_resident_q(const float* ux, const float* uy, const float* uz, ThermalGrid t, float* q,
                              cudaStream_t s);

} // namespace cfdx
