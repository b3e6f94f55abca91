// Device-resident D3Q7 temperature lattice (reference ResidentThermalD3Q7Sycl,
// resident_multiphysics_sycl.hpp:51-200): a two-grid BGK advection-diffusion
// lattice (c_s^2 = 1/4, w_0 = 1/4, w_1..6 = 1/8, tau = 1/2 + 4 D) driven by the
// flow's device velocity, and the Boussinesq acceleration it adds into the
// flow's device acceleration field.  Every expression keeps the reference's
// operand order with explicitly rounded FP32 operations, so the oracle
// restatement reproduces the populations bit for bit.  HBM-bound: 56 B of
// populations and 12 B of velocity per cell and step.
#include "thermal.h"

namespace cfdx {
namespace {

__device__ __forceinline__ int tcx(int d) { return d == 1 ? 1 : (d == 2 ? -1 : 0); }
__device__ __forceinline__ int tcy(int d) { return d == 3 ? 1 : (d == 4 ? -1 : 0); }
__device__ __forceinline__ int tcz(int d) { return d == 5 ? 1 : (d == 6 ? -1 : 0); }
__device__ __forceinline__ float tw(int d) { return d == 0 ? 0.25F : 0.125F; }

__device__ __forceinline__ std::uint32_t wrap_shift(std::uint32_t v, int delta, std::uint32_t n) {
    if (delta > 0) return v + 1U == n ? 0U : v + 1U;
    if (delta < 0) return v == 0U ? n - 1U : v - 1U;
    return v;
}

__global__ void __launch_bounds__(256) k_thermal_uniform(float* g, ThermalGrid t, float temperature) {
    const std::uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= t.cells) return;
#pragma unroll
    for (int d = 0; d < 7; ++d) g[std::size_t(d) * t.cells + n] = __fmul_rn(tw(d), temperature);
}

__global__ void __launch_bounds__(256) k_thermal_field(float* g, ThermalGrid t, const float* temperature) {
    const std::uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= t.cells) return;
    const float v = temperature[n];
#pragma unroll
    for (int d = 0; d < 7; ++d) g[std::size_t(d) * t.cells + n] = __fmul_rn(tw(d), v);
}

__global__ void __launch_bounds__(256) k_thermal_step(const float* in, float* out, ThermalGrid t, const float* ux,
                                                      const float* uy, const float* uz, float omega) {
    const std::uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    if (x >= t.nx) return;
    const std::uint32_t n = (z * t.ny + y) * t.nx + x;
    float local[7];
    float temperature = 0.0F;
#pragma unroll
    for (int d = 0; d < 7; ++d) {
        const std::uint32_t xs = wrap_shift(x, -tcx(d), t.nx), ys = wrap_shift(y, -tcy(d), t.ny),
                            zs = wrap_shift(z, -tcz(d), t.nz);
        local[d] = in[std::size_t(d) * t.cells + (zs * t.ny + ys) * t.nx + xs];
        temperature = __fadd_rn(temperature, local[d]);
    }
    const float u = ux[n], v = uy[n], w = uz[n];
#pragma unroll
    for (int d = 0; d < 7; ++d) {
        const float cu = __fadd_rn(__fadd_rn(__fmul_rn(float(tcx(d)), u), __fmul_rn(float(tcy(d)), v)),
                                   __fmul_rn(float(tcz(d)), w));
        const float geq = __fmul_rn(__fmul_rn(tw(d), temperature), __fadd_rn(1.0F, __fmul_rn(4.0F, cu)));
        out[std::size_t(d) * t.cells + n] = __fsub_rn(local[d], __fmul_rn(omega, __fsub_rn(local[d], geq)));
    }
}

__global__ void __launch_bounds__(256) k_thermal_scalar(const float* g, ThermalGrid t, float* temperature) {
    const std::uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= t.cells) return;
    float v = 0.0F;
#pragma unroll
    for (int d = 0; d < 7; ++d) v = __fadd_rn(v, g[std::size_t(d) * t.cells + n]);
    temperature[n] = v;
}

// The temperature (as k_thermal_scalar) and the Boussinesq term in one pass:
// the temperature is written (the device scalar field) and used without
// being read back.
__global__ void __launch_bounds__(256) k_thermal_boussinesq(const float* g, ThermalGrid t, float* temperature,
                                                            float* ax, float* ay, float* az, float t_ref, float beta,
                                                            float gx, float gy, float gz) {
    const std::uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= t.cells) return;
    float v = 0.0F;
#pragma unroll
    for (int d = 0; d < 7; ++d) v = __fadd_rn(v, g[std::size_t(d) * t.cells + n]);
    temperature[n] = v;
    const float scale = __fmul_rn(-beta, __fsub_rn(v, t_ref));
    ax[n] = __fadd_rn(ax[n], __fmul_rn(scale, gx));
    ay[n] = __fadd_rn(ay[n], __fmul_rn(scale, gy));
    az[n] = __fadd_rn(az[n], __fmul_rn(scale, gz));
}

__global__ void __launch_bounds__(256) k_thermal_partials(const float* g, std::size_t count, double* partials) {
    __shared__ double part[256];
    double s = 0.0;
    for (std::size_t i = blockIdx.x * std::size_t(blockDim.x) + threadIdx.x; i < count;
         i += std::size_t(gridDim.x) * blockDim.x)
        s += double(g[i]);
    part[threadIdx.x] = s;
    __syncthreads();
    for (unsigned w = blockDim.x / 2U; w > 0U; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0U) partials[blockIdx.x] = part[0];
}

__global__ void __launch_bounds__(256) k_thermal_final(const double* partials, int count, double* out) {
    __shared__ double part[256];
    double s = 0.0;
    for (int i = static_cast<int>(threadIdx.x); i < count; i += blockDim.x) s += partials[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (unsigned w = blockDim.x / 2U; w > 0U; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0U) out[0] = part[0];
}

unsigned blocks_for(std::uint32_t cells) { return (cells + 255U) / 256U; }

} // namespace

cudaError_t launch_thermal_uniform(float* g, ThermalGrid t, float temperature, cudaStream_t s) {
    k_thermal_uniform<<<blocks_for(t.cells), 256, 0, s>>>(g, t, temperature);
    return cudaGetLastError();
}

cudaError_t launch_thermal_field(float* g, ThermalGrid t, const float* temperature, cudaStream_t s) {
    k_thermal_field<<<blocks_for(t.cells), 256, 0, s>>>(g, t, temperature);
    return cudaGetLastError();
}

cudaError_t launch_thermal_step(const float* in, float* out, ThermalGrid t, const float* ux, const float* uy,
                                const float* uz, float omega, cudaStream_t s) {
    const dim3 grid((t.nx + 127U) / 128U, t.ny, t.nz);
    k_thermal_step<<<grid, 128, 0, s>>>(in, out, t, ux, uy, uz, omega);
    return cudaGetLastError();
}

cudaError_t launch_thermal_scalar(const float* g, ThermalGrid t, float* temperature, cudaStream_t s) {
    k_thermal_scalar<<<blocks_for(t.cells), 256, 0, s>>>(g, t, temperature);
    return cudaGetLastError();
}

cudaError_t launch_thermal_boussinesq(const float* g, ThermalGrid t, float* temperature, float* ax, float* ay,
                                     float* az, float t_ref, float beta, float gx, float gy, float gz,
                                     cudaStream_t s) {
    k_thermal_boussinesq<<<blocks_for(t.cells), 256, 0, s>>>(g, t, temperature, ax, ay, az, t_ref, beta, gx, gy, gz);
    return cudaGetLastError();
}

cudaError_t launch_thermal_total(const float* g, ThermalGrid t, double* partials, int blocks, double* out,
                                 cudaStream_t s) {
    k_thermal_partials<<<blocks, 256, 0, s>>>(g, std::size_t(7) * t.cells, partials);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_thermal_final<<<1, 256, 0, s>>>(partials, blocks, out);
    return cudaGetLastError();
}

} // namespace cfdx
