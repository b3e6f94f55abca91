// Resident solvers coupled to the flow through its device velocity and
// acceleration views (reference resident_multiphysics_sycl.hpp:202-411):
//   * a fill field advected with first-order upwind face fluxes and clamped to
//     [0, 1] (VOF-like free surface), its normals and curvature, and the
//     surface-tension acceleration sigma * kappa * grad(phi) / rho;
//   * point particles: trilinear velocity interpolation, Stokes drag with a
//     response time, explicit Euler push, periodic positions, and (two-way)
//     the drag spread back onto the eight cells as acceleration with atomics;
//   * the periodic FP32 Q-criterion of the velocity.
// Every expression keeps the reference's operand order with explicitly
// rounded FP32 operations, so the restatements match bit for bit, except the
// atomically summed particle force, whose order of additions is not fixed.
#include "resident.h"

namespace cfdx {
namespace {

using u32 = std::uint32_t;

__device__ __forceinline__ u32 shp(u32 v, u32 n) { return v + 1U == n ? 0U : v + 1U; }
__device__ __forceinline__ u32 shm(u32 v, u32 n) { return v == 0U ? n - 1U : v - 1U; }
__device__ __forceinline__ u32 at(u32 x, u32 y, u32 z, const ThermalGrid& t) { return (z * t.ny + y) * t.nx + x; }

struct Stencil {
    u32 n, xp, xm, yp, ym, zp, zm;
};

__device__ __forceinline__ bool stencil(const ThermalGrid& t, Stencil& s) {
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    if (x >= t.nx) return false;
    s.n = at(x, y, z, t);
    s.xp = at(shp(x, t.nx), y, z, t);
    s.xm = at(shm(x, t.nx), y, z, t);
    s.yp = at(x, shp(y, t.ny), z, t);
    s.ym = at(x, shm(y, t.ny), z, t);
    s.zp = at(x, y, shp(z, t.nz), t);
    s.zm = at(x, y, shm(z, t.nz), t);
    return true;
}

__device__ __forceinline__ float half_sum(float a, float b) { return __fmul_rn(0.5F, __fadd_rn(a, b)); }
__device__ __forceinline__ float half_diff(float a, float b) { return __fmul_rn(0.5F, __fsub_rn(a, b)); }
__device__ __forceinline__ float upwind(float u, float here, float there) { return __fmul_rn(u, u >= 0.0F ? here : there); }

__global__ void __launch_bounds__(256) k_fill_uniform(float* fill, u32 cells, float value) {
    const u32 n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < cells) fill[n] = value;
}

__global__ void __launch_bounds__(256) k_fill_half_space_x(float* fill, ThermalGrid t, float interface_x) {
    const u32 n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= t.cells) return;
    const float left = float(n % t.nx), right = __fadd_rn(left, 1.0F);
    fill[n] = interface_x <= left ? 0.0F : (interface_x >= right ? 1.0F : __fsub_rn(interface_x, left));
}

__global__ void __launch_bounds__(128) k_fill_advect(const float* phi, float* out, ThermalGrid t, const float* ux,
                                                     const float* uy, const float* uz, float dt) {
    Stencil s;
    if (!stencil(t, s)) return;
    const u32 n = s.n;
    const float uxp = half_sum(ux[n], ux[s.xp]), uxm = half_sum(ux[s.xm], ux[n]);
    const float uyp = half_sum(uy[n], uy[s.yp]), uym = half_sum(uy[s.ym], uy[n]);
    const float uzp = half_sum(uz[n], uz[s.zp]), uzm = half_sum(uz[s.zm], uz[n]);
    const float fxp = upwind(uxp, phi[n], phi[s.xp]), fxm = upwind(uxm, phi[s.xm], phi[n]);
    const float fyp = upwind(uyp, phi[n], phi[s.yp]), fym = upwind(uym, phi[s.ym], phi[n]);
    const float fzp = upwind(uzp, phi[n], phi[s.zp]), fzm = upwind(uzm, phi[s.zm], phi[n]);
    const float div = __fadd_rn(__fadd_rn(__fsub_rn(fxp, fxm), __fsub_rn(fyp, fym)), __fsub_rn(fzp, fzm));
    float value = __fsub_rn(phi[n], __fmul_rn(dt, div));
    value = value < 0.0F ? 0.0F : (value > 1.0F ? 1.0F : value);
    out[n] = value;
}

__global__ void __launch_bounds__(128) k_fill_normals(const float* phi, float* g, ThermalGrid t) {
    Stencil s;
    if (!stencil(t, s)) return;
    const float gx = half_diff(phi[s.xp], phi[s.xm]), gy = half_diff(phi[s.yp], phi[s.ym]),
                gz = half_diff(phi[s.zp], phi[s.zm]);
    const float mag = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)), __fmul_rn(gz, gz)));
    const bool ok = mag > 1.0e-12F;
    const std::size_t cells = t.cells;
    g[s.n] = ok ? __fdiv_rn(gx, mag) : 0.0F;
    g[cells + s.n] = ok ? __fdiv_rn(gy, mag) : 0.0F;
    g[2U * cells + s.n] = ok ? __fdiv_rn(gz, mag) : 0.0F;
}

__global__ void __launch_bounds__(128) k_fill_curvature(float* g, ThermalGrid t) {
    Stencil s;
    if (!stencil(t, s)) return;
    const std::size_t cells = t.cells;
    const float* nx = g;
    const float* ny = g + cells;
    const float* nz = g + 2U * cells;
    const float d = __fadd_rn(__fadd_rn(__fsub_rn(nx[s.xp], nx[s.xm]), __fsub_rn(ny[s.yp], ny[s.ym])),
                              __fsub_rn(nz[s.zp], nz[s.zm]));
    g[3U * cells + s.n] = __fmul_rn(-0.5F, d);
}

__global__ void __launch_bounds__(128) k_surface_tension(const float* phi, const float* curvature, ThermalGrid t,
                                                         float* ax, float* ay, float* az, float sigma,
                                                         float density) {
    Stencil s;
    if (!stencil(t, s)) return;
    const float gx = half_diff(phi[s.xp], phi[s.xm]), gy = half_diff(phi[s.yp], phi[s.ym]),
                gz = half_diff(phi[s.zp], phi[s.zm]);
    const float c = __fdiv_rn(__fmul_rn(sigma, curvature[s.n]), density);
    ax[s.n] = __fadd_rn(ax[s.n], __fmul_rn(c, gx));
    ay[s.n] = __fadd_rn(ay[s.n], __fmul_rn(c, gy));
    az[s.n] = __fadd_rn(az[s.n], __fmul_rn(c, gz));
}

__global__ void __launch_bounds__(256) k_sum_floats(const float* v, std::size_t count, double* partials) {
    __shared__ double part[256];
    double s = 0.0;
    for (std::size_t i = blockIdx.x * std::size_t(blockDim.x) + threadIdx.x; i < count;
         i += std::size_t(gridDim.x) * blockDim.x)
        s += double(v[i]);
    part[threadIdx.x] = s;
    __syncthreads();
    for (unsigned w = blockDim.x / 2U; w > 0U; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0U) partials[blockIdx.x] = part[0];
}

__global__ void __launch_bounds__(256) k_sum_final(const double* partials, int count, double* out) {
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

// floor of a float as an integer, and a coordinate wrapped into [0, extent)
__device__ __forceinline__ long long floor_ll(float v) {
    long long i = static_cast<long long>(v);
    if (float(i) > v) --i;
    return i;
}
__device__ __forceinline__ float periodic(float v, u32 extent) {
    const float e = float(extent);
    const long long turns = floor_ll(__fdiv_rn(v, e));
    v = __fsub_rn(v, __fmul_rn(float(turns), e));
    if (v >= e) v = __fsub_rn(v, e);
    if (v < 0.0F) v = __fadd_rn(v, e);
    return v;
}
__device__ __forceinline__ u32 wrap(long long v, u32 extent) {
    const long long e = extent;
    v %= e;
    if (v < 0) v += e;
    return static_cast<u32>(v);
}

__global__ void __launch_bounds__(128) k_particles(float* st, u32 count, ThermalGrid t, const float* ux,
                                                   const float* uy, const float* uz, float* ax, float* ay, float* az,
                                                   float dt, int two_way, float gx, float gy, float gz) {
    const u32 p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    float px = periodic(st[p], t.nx), py = periodic(st[count + p], t.ny), pz = periodic(st[2U * count + p], t.nz);
    float vx = st[3U * count + p], vy = st[4U * count + p], vz = st[5U * count + p];
    const float mass = st[6U * count + p], response = st[7U * count + p];
    // a position that is not finite (an overflowed velocity) samples cell 0 instead of
    // converting inf/NaN to an integer
    const long long x0 = isfinite(px) ? floor_ll(px) : 0, y0 = isfinite(py) ? floor_ll(py) : 0,
                    z0 = isfinite(pz) ? floor_ll(pz) : 0;
    const float tx = __fsub_rn(px, float(x0)), ty = __fsub_rn(py, float(y0)), tz = __fsub_rn(pz, float(z0));
    float fu = 0.0F, fv = 0.0F, fw = 0.0F;
    u32 ids[8];
    float weights[8];
    int k = 0;
#pragma unroll
    for (int dz = 0; dz <= 1; ++dz)
#pragma unroll
        for (int dy = 0; dy <= 1; ++dy)
#pragma unroll
            for (int dx = 0; dx <= 1; ++dx) {
                const float wx = dx ? tx : __fsub_rn(1.0F, tx), wy = dy ? ty : __fsub_rn(1.0F, ty),
                            wz = dz ? tz : __fsub_rn(1.0F, tz);
                const u32 n = at(wrap(x0 + dx, t.nx), wrap(y0 + dy, t.ny), wrap(z0 + dz, t.nz), t);
                const float w = __fmul_rn(__fmul_rn(wx, wy), wz);
                ids[k] = n;
                weights[k] = w;
                ++k;
                fu = __fadd_rn(fu, __fmul_rn(w, ux[n]));
                fv = __fadd_rn(fv, __fmul_rn(w, uy[n]));
                fw = __fadd_rn(fw, __fmul_rn(w, uz[n]));
            }
    const float dragx = __fdiv_rn(__fmul_rn(mass, __fsub_rn(fu, vx)), response);
    const float dragy = __fdiv_rn(__fmul_rn(mass, __fsub_rn(fv, vy)), response);
    const float dragz = __fdiv_rn(__fmul_rn(mass, __fsub_rn(fw, vz)), response);
    if (two_way) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            atomicAdd(ax + ids[j], __fmul_rn(-dragx, weights[j]));
            atomicAdd(ay + ids[j], __fmul_rn(-dragy, weights[j]));
            atomicAdd(az + ids[j], __fmul_rn(-dragz, weights[j]));
        }
    }
    vx = __fadd_rn(vx, __fmul_rn(dt, __fadd_rn(__fdiv_rn(dragx, mass), gx)));
    vy = __fadd_rn(vy, __fmul_rn(dt, __fadd_rn(__fdiv_rn(dragy, mass), gy)));
    vz = __fadd_rn(vz, __fmul_rn(dt, __fadd_rn(__fdiv_rn(dragz, mass), gz)));
    px = periodic(__fadd_rn(px, __fmul_rn(dt, vx)), t.nx);
    py = periodic(__fadd_rn(py, __fmul_rn(dt, vy)), t.ny);
    pz = periodic(__fadd_rn(pz, __fmul_rn(dt, vz)), t.nz);
    st[p] = px;
    st[count + p] = py;
    st[2U * count + p] = pz;
    st[3U * count + p] = vx;
    st[4U * count + p] = vy;
    st[5U * count + p] = vz;
}

__global__ void __launch_bounds__(128) k_resident_q(const float* ux, const float* uy, const float* uz, ThermalGrid t,
                                                    float* q) {
    Stencil s;
    if (!stencil(t, s)) return;
    const u32 P[3] = {s.xp, s.yp, s.zp}, M[3] = {s.xm, s.ym, s.zm};
    float g[3][3];
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        g[0][axis] = half_diff(ux[P[axis]], ux[M[axis]]);
        g[1][axis] = half_diff(uy[P[axis]], uy[M[axis]]);
        g[2][axis] = half_diff(uz[P[axis]], uz[M[axis]]);
    }
    float s2 = 0.0F, o2 = 0.0F;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float sij = half_sum(g[i][j], g[j][i]), oij = half_diff(g[i][j], g[j][i]);
            s2 = __fadd_rn(s2, __fmul_rn(sij, sij));
            o2 = __fadd_rn(o2, __fmul_rn(oij, oij));
        }
    q[s.n] = __fmul_rn(0.5F, __fsub_rn(o2, s2));
}

dim3 cell_grid3(const ThermalGrid& t) { return dim3((t.nx + 127U) / 128U, t.ny, t.nz); }

} // namespace

cudaError_t launch_fill_uniform(float* fill, ThermalGrid t, float value, cudaStream_t s) {
    k_fill_uniform<<<(t.cells + 255U) / 256U, 256, 0, s>>>(fill, t.cells, value);
    return cudaGetLastError();
}

cudaError_t launch_fill_half_space_x(float* fill, ThermalGrid t, float interface_x, cudaStream_t s) {
    k_fill_half_space_x<<<(t.cells + 255U) / 256U, 256, 0, s>>>(fill, t, interface_x);
    return cudaGetLastError();
}

cudaError_t launch_fill_advect(const float* fill, float* out, ThermalGrid t, const float* ux, const float* uy,
                               const float* uz, float dt, cudaStream_t s) {
    k_fill_advect<<<cell_grid3(t), 128, 0, s>>>(fill, out, t, ux, uy, uz, dt);
    return cudaGetLastError();
}

cudaError_t launch_fill_geometry(const float* fill, float* geometry, ThermalGrid t, cudaStream_t s) {
    k_fill_normals<<<cell_grid3(t), 128, 0, s>>>(fill, geometry, t);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_fill_curvature<<<cell_grid3(t), 128, 0, s>>>(geometry, t);
    return cudaGetLastError();
}

cudaError_t launch_surface_tension(const float* fill, const float* curvature, ThermalGrid t, float* ax, float* ay,
                                   float* az, float sigma, float density, cudaStream_t s) {
    k_surface_tension<<<cell_grid3(t), 128, 0, s>>>(fill, curvature, t, ax, ay, az, sigma, density);
    return cudaGetLastError();
}

cudaError_t launch_sum_floats(const float* v, std::size_t count, double* partials, int blocks, double* out,
                              cudaStream_t s) {
    k_sum_floats<<<blocks, 256, 0, s>>>(v, count, partials);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_sum_final<<<1, 256, 0, s>>>(partials, blocks, out);
    return cudaGetLastError();
}

cudaError_t launch_particles_advance(float* state, std::uint32_t count, ThermalGrid t, const float* ux,
                                     const float* uy, const float* uz, float* ax, float* ay, float* az, float dt,
                                     bool two_way, float gx, float gy, float gz, cudaStream_t s) {
    if (count == 0U) return cudaSuccess;
    k_particles<<<(count + 127U) / 128U, 128, 0, s>>>(state, count, t, ux, uy, uz, ax, ay, az, dt, two_way ? 1 : 0,
                                                      gx, gy, gz);
    return cudaGetLastError();
}

cudaError_t launch_resident_q(const float* ux, const float* uy, const float* uz, ThermalGrid t, float* q,
                              cudaStream_t s) {
    k_resident_q<<<cell_grid3(t), 128, 0, s>>>(ux, uy, uz, t, q);
    return cudaGetLastError();
}

} // namespace cfdx
