// Triangle-surface voxelizer (reference cfd::lbm::voxelize_surface,
// src/lbm/voxelize.cpp:4-5, and its SYCL twin src/sycl/voxelize_sycl.cpp:13-68).
//
// Cell (i, j, k) is solid when the ray from its centre
//     o = (lo.x + (i+0.5) dx, lo.y + (j+0.5) dy + 1e-10 dx, lo.z + (k+0.5) dz + 2e-10 dx)
// in direction +x hits an odd number of triangles (Moller-Trumbore: |det| >=
// 1e-12, u in [0,1], v >= 0, u+v <= 1, distance > 1e-10).  The reference tests
// every cell against every triangle.  Here the test is split the way the
// arithmetic allows: with d = +x, h = d x e2 has h.x = +-0, so u = inv (s.h)
// and v = inv q.x do not depend on the cell's x (s.x only ever multiplies a
// zero); only the distance does.  So
//   1. one warp per triangle tests the (j, k) rows under the triangle's
//      bounding box and appends the triangle to the rows it passes (count,
//      scan, fill);
//   2. one thread per cell evaluates the distance against its row's few
//      candidates and writes the parity.
// Every expression is the reference's, in its operand order, with explicitly
// rounded FP64 operations (no contraction), so the mask equals the reference
// CPU voxelizer's bit for bit.  Hits are counted, so the order of a row's
// candidates does not matter.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "scratch_pool.h"
#include "voxelize.h"

namespace cfdx {
namespace {

struct Tri {
    double ax, ay, az;
    double e1x, e1y, e1z;
    double e2x, e2y, e2z;
    double hx, hy, hz;
    double inv;
    int valid; // |det| >= 1e-12
};

struct Grid {
    double lox, loy, loz, dx, dy, dz;
    std::uint32_t nx, ny, nz, z_first, z_count;
};

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
// a.x*b.x + a.y*b.y + a.z*b.z, left to right
__device__ __forceinline__ double dot3(double ax, double ay, double az, double bx, double by, double bz) {
    return add(add(mul(ax, bx), mul(ay, by)), mul(az, bz));
}

// Row origins: y of row j, z of global plane k (the reference's expressions).
__device__ __forceinline__ double origin_x(const Grid& g, std::uint32_t i) {
    return add(g.lox, mul(add(double(i), 0.5), g.dx));
}
__device__ __forceinline__ double origin_y(const Grid& g, std::uint32_t j) {
    return add(add(g.loy, mul(add(double(j), 0.5), g.dy)), mul(1e-10, g.dx));
}
__device__ __forceinline__ double origin_z(const Grid& g, std::uint32_t k) {
    return add(add(g.loz, mul(add(double(k), 0.5), g.dz)), mul(2e-10, g.dx));
}

__global__ void __launch_bounds__(256) k_vox_prepare(const double* v, std::size_t count, Tri* out) {
    const std::size_t t = blockIdx.x * std::size_t(blockDim.x) + threadIdx.x;
    if (t >= count) return;
    const double* p = v + 9 * t;
    Tri r;
    r.ax = p[0];
    r.ay = p[1];
    r.az = p[2];
    r.e1x = sub(p[3], p[0]);
    r.e1y = sub(p[4], p[1]);
    r.e1z = sub(p[5], p[2]);
    r.e2x = sub(p[6], p[0]);
    r.e2y = sub(p[7], p[1]);
    r.e2z = sub(p[8], p[2]);
    // h = d x e2 with d = (1, 0, 0)
    r.hx = sub(mul(0.0, r.e2z), mul(0.0, r.e2y));
    r.hy = sub(mul(0.0, r.e2x), mul(1.0, r.e2z));
    r.hz = sub(mul(1.0, r.e2y), mul(0.0, r.e2x));
    const double det = dot3(r.e1x, r.e1y, r.e1z, r.hx, r.hy, r.hz);
    r.valid = fabs(det) < 1e-12 ? 0 : 1;
    r.inv = r.valid ? 1.0 / det : 0.0;
    out[t] = r;
}

// Does the +x ray of row (oy, oz) pass triangle r's u/v test?  (ox is any
// finite x: it only multiplies h.x = +-0 and the zero components of d.)
__device__ __forceinline__ bool row_passes(const Tri& r, double ox, double oy, double oz) {
    const double sx = sub(ox, r.ax), sy = sub(oy, r.ay), sz = sub(oz, r.az);
    const double u = mul(r.inv, dot3(sx, sy, sz, r.hx, r.hy, r.hz));
    if (u < 0.0 || u > 1.0) return false;
    const double qx = sub(mul(sy, r.e1z), mul(sz, r.e1y));
    const double qy = sub(mul(sz, r.e1x), mul(sx, r.e1z));
    const double qz = sub(mul(sx, r.e1y), mul(sy, r.e1x));
    const double v = mul(r.inv, dot3(1.0, 0.0, 0.0, qx, qy, qz));
    return !(v < 0.0 || add(u, v) > 1.0);
}

// Inclusive index range of rows whose origin coordinate lies within [lo_v, hi_v]
// of a bounding box, widened by two rows for the rounding of the origins.
__device__ __forceinline__ bool row_range(double lo_v, double hi_v, double base, double step, std::uint32_t n,
                                          std::uint32_t& first, std::uint32_t& last) {
    const double a = floor((lo_v - base) / step - 0.5) - 2.0;
    const double b = ceil((hi_v - base) / step - 0.5) + 2.0;
    if (!(b >= 0.0) || !(a <= double(n) - 1.0)) return false;
    first = a < 0.0 ? 0U : std::uint32_t(a);
    last = b > double(n) - 1.0 ? n - 1U : std::uint32_t(b);
    return first <= last;
}

// FILL = false: counts[row] += 1 for every row triangle t passes;
// FILL = true:  list[offsets[row] + cursor[row]++] = t.
template <bool FILL>
__global__ void __launch_bounds__(256) k_vox_rows(const double* v, const Tri* tris, std::size_t count, Grid g,
                                                  std::uint32_t* counts, const std::uint32_t* offsets,
                                                  std::uint32_t* list) {
    const std::size_t t = (blockIdx.x * std::size_t(blockDim.x) + threadIdx.x) / 32U;
    const unsigned lane = threadIdx.x & 31U;
    if (t >= count) return;
    const Tri r = tris[t];
    if (!r.valid) return;
    const double* p = v + 9 * t;
    const double ylo = fmin(fmin(p[1], p[4]), p[7]), yhi = fmax(fmax(p[1], p[4]), p[7]);
    const double zlo = fmin(fmin(p[2], p[5]), p[8]), zhi = fmax(fmax(p[2], p[5]), p[8]);
    std::uint32_t j0, j1, k0, k1;
    if (!row_range(ylo, yhi, g.loy, g.dy, g.ny, j0, j1) || !row_range(zlo, zhi, g.loz, g.dz, g.nz, k0, k1)) return;
    const std::uint32_t nj = j1 - j0 + 1U;
    const std::uint64_t rows = std::uint64_t(nj) * (k1 - k0 + 1U);
    const double ox = origin_x(g, 0U);
    for (std::uint64_t e = lane; e < rows; e += 32U) {
        const std::uint32_t j = j0 + std::uint32_t(e % nj);
        const std::uint32_t k = k0 + std::uint32_t(e / nj);
        // local plane of global plane k (the requested planes may wrap past nz)
        if (!row_passes(r, ox, origin_y(g, j), origin_z(g, k))) continue;
        for (std::uint32_t kl = (k + g.nz - g.z_first % g.nz) % g.nz; kl < g.z_count; kl += g.nz) {
            const std::uint32_t row = kl * g.ny + j;
            if constexpr (FILL) {
                list[offsets[row] + atomicAdd(counts + row, 1U)] = std::uint32_t(t);
            } else {
                atomicAdd(counts + row, 1U);
            }
        }
    }
}

__global__ void __launch_bounds__(128) k_vox_cells(const Tri* tris, Grid g, const std::uint32_t* offsets,
                                                   const std::uint32_t* list, std::uint8_t value,
                                                   const std::uint8_t* base, std::uint8_t* out) {
    const std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const std::uint32_t j = blockIdx.y, kl = blockIdx.z;
    if (i >= g.nx) return;
    const std::uint32_t row = kl * g.ny + j;
    const std::uint32_t k = (g.z_first + kl) % g.nz;
    const double ox = origin_x(g, i), oy = origin_y(g, j), oz = origin_z(g, k);
    unsigned hits = 0U;
    for (std::uint32_t e = offsets[row]; e < offsets[row + 1]; ++e) {
        const Tri r = tris[list[e]];
        const double sx = sub(ox, r.ax), sy = sub(oy, r.ay), sz = sub(oz, r.az);
        const double qx = sub(mul(sy, r.e1z), mul(sz, r.e1y));
        const double qy = sub(mul(sz, r.e1x), mul(sx, r.e1z));
        const double qz = sub(mul(sx, r.e1y), mul(sy, r.e1x));
        const double dist = mul(r.inv, dot3(r.e2x, r.e2y, r.e2z, qx, qy, qz));
        hits += dist > 1e-10 ? 1U : 0U;
    }
    const std::size_t n = (std::size_t(kl) * g.ny + j) * g.nx + i;
    out[n] = (hits & 1U) ? value : (base ? base[n] : std::uint8_t(0));
}

// Scratch from the library's per-device pool (scratch_pool.cu), released on
// the call's stream when the buffer goes out of scope.
struct DeviceBuffer {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    explicit DeviceBuffer(cudaStream_t stream) : s(stream) {}
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() {
        scratch_free(p, s);
    }
    cudaError_t alloc(std::size_t bytes) { return scratch_alloc(&p, bytes, s); }
};

} // namespace

cudaError_t voxelize_device(const double* host_tris, std::size_t count, const VoxelRequest& q,
                            std::uint8_t* out_device, cudaStream_t s, const char** what) {
    cudaError_t e = cudaSuccess;
    auto step = [&](cudaError_t r, const char* name) {
        if (r != cudaSuccess && e == cudaSuccess) {
            e = r;
            *what = name;
        }
        return e == cudaSuccess;
    };
    const std::uint32_t nx = std::uint32_t(q.nx), ny = std::uint32_t(q.ny), nz = std::uint32_t(q.nz);
    const Grid g{q.lo[0], q.lo[1], q.lo[2], (q.hi[0] - q.lo[0]) / double(q.nx), (q.hi[1] - q.lo[1]) / double(q.ny),
                 (q.hi[2] - q.lo[2]) / double(q.nz), nx, ny, nz, q.z_first, q.z_count};
    const std::size_t rows = std::size_t(ny) * q.z_count;
    DeviceBuffer dv(s), dt(s), dc(s), doff(s), dlist(s), dtmp(s);
    if (!step(dv.alloc(9 * count * sizeof(double)), "triangle buffer") ||
        !step(dt.alloc(count * sizeof(Tri)), "triangle data") ||
        !step(dc.alloc((rows + 1) * sizeof(std::uint32_t)), "row counts") ||
        !step(doff.alloc((rows + 1) * sizeof(std::uint32_t)), "row offsets"))
        return e;
    double* v = static_cast<double*>(dv.p);
    Tri* tris = static_cast<Tri*>(dt.p);
    std::uint32_t* counts = static_cast<std::uint32_t*>(dc.p);
    std::uint32_t* offsets = static_cast<std::uint32_t*>(doff.p);
    if (!step(cudaMemcpyAsync(v, host_tris, 9 * count * sizeof(double), cudaMemcpyHostToDevice, s), "triangle upload"))
        return e;
    k_vox_prepare<<<unsigned((count + 255) / 256), 256, 0, s>>>(v, count, tris);
    if (!step(cudaGetLastError(), "voxelizer prepare kernel") ||
        !step(cudaMemsetAsync(counts, 0, (rows + 1) * sizeof(std::uint32_t), s), "cudaMemsetAsync"))
        return e;
    const unsigned warp_blocks = unsigned((count * 32 + 255) / 256);
    k_vox_rows<false><<<warp_blocks, 256, 0, s>>>(v, tris, count, g, counts, nullptr, nullptr);
    if (!step(cudaGetLastError(), "voxelizer row count kernel")) return e;
    // offsets = exclusive prefix sum of counts (rows + 1 entries: the last is the total)
    std::size_t tmp_bytes = 0;
    if (!step(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, counts, offsets, int(rows + 1), s), "scan size") ||
        !step(dtmp.alloc(tmp_bytes), "scan scratch") ||
        !step(cub::DeviceScan::ExclusiveSum(dtmp.p, tmp_bytes, counts, offsets, int(rows + 1), s), "row scan"))
        return e;
    std::uint32_t total = 0;
    if (!step(cudaMemcpyAsync(&total, offsets + rows, sizeof total, cudaMemcpyDeviceToHost, s), "candidate count") ||
        !step(cudaStreamSynchronize(s), "cudaStreamSynchronize") ||
        !step(dlist.alloc(std::size_t(total) * sizeof(std::uint32_t)), "row candidate lists") ||
        !step(cudaMemsetAsync(counts, 0, (rows + 1) * sizeof(std::uint32_t), s), "cudaMemsetAsync"))
        return e;
    std::uint32_t* list = static_cast<std::uint32_t*>(dlist.p);
    k_vox_rows<true><<<warp_blocks, 256, 0, s>>>(v, tris, count, g, counts, offsets, list);
    if (!step(cudaGetLastError(), "voxelizer row fill kernel")) return e;
    const dim3 grid((nx + 127) / 128, ny, q.z_count);
    k_vox_cells<<<grid, 128, 0, s>>>(tris, g, offsets, list, q.value, q.base, out_device);
    step(cudaGetLastError(), "voxelizer cell kernel");
    step(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    return e;
}

} // namespace cfdx
