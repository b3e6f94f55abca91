// Device-resident D3Q7 temperature lattice coupled to the flow (thermal.cu):
// the reference's ResidentThermalD3Q7Sycl (resident_multiphysics_sycl.hpp:51-200).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace cfdx {

struct ThermalGrid {
    std::uint32_t nx, ny, nz;
    std::uint32_t cells;
};

// g[d][n] = w_d * temperature (every cell).
cudaError_t launch_thermal_uniform(float* g, ThermalGrid t, float temperature, cudaStream_t s);
// g[d][n] = w_d * temperature[n].
cudaError_t launch_thermal_field(float* g, ThermalGrid t, const float* temperature, cudaStream_t s);
// One two-grid advection-diffusion step in -> out with the velocity ux/uy/uz.
cudaError_t launch_thermal_step(const float* in, float* out, ThermalGrid t, const float* ux, const float* uy,
                                const float* uz, float omega, cudaStream_t s);
// temperature[n] = sum_d g[d][n].
cudaError_t launch_thermal_scalar(const float* g, ThermalGrid t, float* temperature, cudaStream_t s);
// temperature = sum_d g[d] (written), then a += -beta (T - t_ref) * gravity, in one pass.
cudaError_t launch_thermal_boussinesq(const float* g, ThermalGrid t, float* temperature, float* ax, float* ay,
                                     float* az, float t_ref, float beta, float gx, float gy, float gz,
                                     cudaStream_t s);
// FP64 sum of the 7 * cells populations into out[0] (partials: `blocks` doubles of scratch).
cudaError_t launch_thermal_total(const float* g, ThermalGrid t, double* partials, int blocks, double* out,
                                 cudaStream_t s);

} // namespace cfdx
