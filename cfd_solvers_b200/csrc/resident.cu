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

#include <cstdint>

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

// A field at a cell and its six periodic neighbours.
struct Nb {
    float c, xp, xm, yp, ym, zp, zm;
};

__device__ __forceinline__ Nb nb_of(const float* f, const Stencil& s) {
    return Nb{f[s.n], f[s.xp], f[s.xm], f[s.yp], f[s.ym], f[s.zp], f[s.zm]};
}

// ---- the per-cell arithmetic, shared by the one-cell and four-cell kernels
__device__ __forceinline__ float advect_cell(const Nb& p, const Nb& ux, const Nb& uy, const Nb& uz, float dt) {
    const float uxp = half_sum(ux.c, ux.xp), uxm = half_sum(ux.xm, ux.c);
    const float uyp = half_sum(uy.c, uy.yp), uym = half_sum(uy.ym, uy.c);
    const float uzp = half_sum(uz.c, uz.zp), uzm = half_sum(uz.zm, uz.c);
    const float fxp = upwind(uxp, p.c, p.xp), fxm = upwind(uxm, p.xm, p.c);
    const float fyp = upwind(uyp, p.c, p.yp), fym = upwind(uym, p.ym, p.c);
    const float fzp = upwind(uzp, p.c, p.zp), fzm = upwind(uzm, p.zm, p.c);
    const float div = __fadd_rn(__fadd_rn(__fsub_rn(fxp, fxm), __fsub_rn(fyp, fym)), __fsub_rn(fzp, fzm));
    const float value = __fsub_rn(p.c, __fmul_rn(dt, div));
    return value < 0.0F ? 0.0F : (value > 1.0F ? 1.0F : value);
}

__device__ __forceinline__ float3 normal_cell(const Nb& p) {
    const float gx = half_diff(p.xp, p.xm), gy = half_diff(p.yp, p.ym), gz = half_diff(p.zp, p.zm);
    const float mag = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)), __fmul_rn(gz, gz)));
    if (!(mag > 1.0e-12F)) return make_float3(0.0F, 0.0F, 0.0F);
    return make_float3(__fdiv_rn(gx, mag), __fdiv_rn(gy, mag), __fdiv_rn(gz, mag));
}

__device__ __forceinline__ float curvature_cell(const Nb& nx, const Nb& ny, const Nb& nz) {
    const float d =
        __fadd_rn(__fadd_rn(__fsub_rn(nx.xp, nx.xm), __fsub_rn(ny.yp, ny.ym)), __fsub_rn(nz.zp, nz.zm));
    return __fmul_rn(-0.5F, d);
}

// sigma * kappa / rho * grad(phi), to be added to the acceleration
__device__ __forceinline__ float3 tension_cell(const Nb& p, float kappa, float sigma, float density) {
    const float gx = half_diff(p.xp, p.xm), gy = half_diff(p.yp, p.ym), gz = half_diff(p.zp, p.zm);
    const float c = __fdiv_rn(__fmul_rn(sigma, kappa), density);
    return make_float3(__fmul_rn(c, gx), __fmul_rn(c, gy), __fmul_rn(c, gz));
}

// Q = (|Omega|^2 - |S|^2) / 2 with the sums over (i, j) in row order, as the
// reference adds them.  Terms that are equal in IEEE arithmetic are computed
// once: s_ji = s_ij (addition commutes), o_ji = -o_ij (so o_ji^2 = o_ij^2),
// s_ii = g_ii (0.5 (a + a) = a) and o_ii = +0, whose square adds nothing to the
// non-negative o2.  The result is bit for bit the nine-term loop's.
__device__ __forceinline__ float q_cell(const Nb& ux, const Nb& uy, const Nb& uz) {
    const Nb* u[3] = {&ux, &uy, &uz};
    float g[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        g[i][0] = half_diff(u[i]->xp, u[i]->xm);
        g[i][1] = half_diff(u[i]->yp, u[i]->ym);
        g[i][2] = half_diff(u[i]->zp, u[i]->zm);
    }
    float ss[3][3], oo[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        ss[i][i] = __fmul_rn(g[i][i], g[i][i]);
#pragma unroll
        for (int j = i + 1; j < 3; ++j) {
            const float sij = half_sum(g[i][j], g[j][i]), oij = half_diff(g[i][j], g[j][i]);
            ss[i][j] = ss[j][i] = __fmul_rn(sij, sij);
            oo[i][j] = oo[j][i] = __fmul_rn(oij, oij);
        }
    }
    float s2 = 0.0F, o2 = 0.0F;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            s2 = __fadd_rn(s2, ss[i][j]);
            if (i != j) o2 = __fadd_rn(o2, oo[i][j]);
        }
    return __fmul_rn(0.5F, __fsub_rn(o2, s2));
}

// ---- one cell per thread (any nx)
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
    out[s.n] = advect_cell(nb_of(phi, s), nb_of(ux, s), nb_of(uy, s), nb_of(uz, s), dt);
}

__global__ void __launch_bounds__(128) k_fill_normals(const float* phi, float* g, ThermalGrid t) {
    Stencil s;
    if (!stencil(t, s)) return;
    const float3 v = normal_cell(nb_of(phi, s));
    const std::size_t cells = t.cells;
    g[s.n] = v.x;
    g[cells + s.n] = v.y;
    g[2U * cells + s.n] = v.z;
}

__global__ void __launch_bounds__(128) k_fill_curvature(float* g, ThermalGrid t) {
    Stencil s;
    if (!stencil(t, s)) return;
    const std::size_t cells = t.cells;
    g[3U * cells + s.n] = curvature_cell(nb_of(g, s), nb_of(g + cells, s), nb_of(g + 2U * cells, s));
}

__global__ void __launch_bounds__(128) k_surface_tension(const float* phi, const float* curvature, ThermalGrid t,
                                                         float* ax, float* ay, float* az, float sigma,
                                                         float density) {
    Stencil s;
    if (!stencil(t, s)) return;
    const float3 d = tension_cell(nb_of(phi, s), curvature[s.n], sigma, density);
    ax[s.n] = __fadd_rn(ax[s.n], d.x);
    ay[s.n] = __fadd_rn(ay[s.n], d.y);
    az[s.n] = __fadd_rn(az[s.n], d.z);
}

__global__ void __launch_bounds__(128) k_resident_q(const float* ux, const float* uy, const float* uz, ThermalGrid t,
                                                    float* q) {
    Stencil s;
    if (!stencil(t, s)) return;
    q[s.n] = q_cell(nb_of(ux, s), nb_of(uy, s), nb_of(uz, s));
}

// ---- four x-adjacent cells per thread (nx % 4 == 0, 16-byte aligned fields):
// each row segment is one float4 load; the x neighbours of the segment's ends
// are two scalar loads.  Same arithmetic as the one-cell kernels.
struct Rows {
    u32 c, yp, ym, zp, zm; // element offsets of the x0 of the five rows
    u32 x0, xl, xr;        // x0, x0 - 1 and x0 + 4 (periodic)
};

__device__ __forceinline__ bool rows_of(const ThermalGrid& t, Rows& r) {
    r.x0 = 4U * (blockIdx.x * blockDim.x + threadIdx.x);
    if (r.x0 >= t.nx) return false;
    const u32 y = blockIdx.y, z = blockIdx.z;
    r.c = at(r.x0, y, z, t);
    r.yp = at(r.x0, shp(y, t.ny), z, t);
    r.ym = at(r.x0, shm(y, t.ny), z, t);
    r.zp = at(r.x0, y, shp(z, t.nz), t);
    r.zm = at(r.x0, y, shm(z, t.nz), t);
    r.xl = r.x0 == 0U ? t.nx - 1U : r.x0 - 1U;
    r.xr = r.x0 + 4U == t.nx ? 0U : r.x0 + 4U;
    return true;
}

__device__ __forceinline__ float4 ld4(const float* f, u32 off) { return *reinterpret_cast<const float4*>(f + off); }
__device__ __forceinline__ void st4(float* f, u32 off, float4 v) { *reinterpret_cast<float4*>(f + off) = v; }
__device__ __forceinline__ float lane(const float4& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); }

// The four cells' neighbourhoods of one field; X / YZ select which neighbours are loaded.
template <bool X, bool YZ> struct Quad {
    float4 c, yp, ym, zp, zm;
    float xl, xr;
    __device__ __forceinline__ Quad(const float* f, const Rows& r) {
        c = ld4(f, r.c);
        if constexpr (X) {
            xl = f[r.c - r.x0 + r.xl];
            xr = f[r.c - r.x0 + r.xr];
        }
        if constexpr (YZ) {
            yp = ld4(f, r.yp);
            ym = ld4(f, r.ym);
            zp = ld4(f, r.zp);
            zm = ld4(f, r.zm);
        }
    }
    __device__ __forceinline__ Nb at(int k) const {
        Nb n{};
        n.c = lane(c, k);
        if constexpr (X) {
            n.xm = k == 0 ? xl : lane(c, k - 1);
            n.xp = k == 3 ? xr : lane(c, k + 1);
        }
        if constexpr (YZ) {
            n.yp = lane(yp, k);
            n.ym = lane(ym, k);
            n.zp = lane(zp, k);
            n.zm = lane(zm, k);
        }
        return n;
    }
};

__global__ void __launch_bounds__(128) k_fill_advect4(const float* phi, float* out, ThermalGrid t, const float* ux,
                                                      const float* uy, const float* uz, float dt) {
    Rows r;
    if (!rows_of(t, r)) return;
    const Quad<true, true> p(phi, r);
    const Quad<true, false> u(ux, r);
    const Nb v0{}; // uy / uz: only their y / z neighbours enter
    const float4 vc = ld4(uy, r.c), vp = ld4(uy, r.yp), vm = ld4(uy, r.ym);
    const float4 wc = ld4(uz, r.c), wp = ld4(uz, r.zp), wm = ld4(uz, r.zm);
    float o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        Nb v = v0, w = v0;
        v.c = lane(vc, k);
        v.yp = lane(vp, k);
        v.ym = lane(vm, k);
        w.c = lane(wc, k);
        w.zp = lane(wp, k);
        w.zm = lane(wm, k);
        o[k] = advect_cell(p.at(k), u.at(k), v, w, dt);
    }
    st4(out, r.c, make_float4(o[0], o[1], o[2], o[3]));
}

__global__ void __launch_bounds__(128) k_fill_normals4(const float* phi, float* g, ThermalGrid t) {
    Rows r;
    if (!rows_of(t, r)) return;
    const Quad<true, true> p(phi, r);
    float3 v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = normal_cell(p.at(k));
    const std::size_t cells = t.cells;
    st4(g, r.c, make_float4(v[0].x, v[1].x, v[2].x, v[3].x));
    st4(g + cells, r.c, make_float4(v[0].y, v[1].y, v[2].y, v[3].y));
    st4(g + 2U * cells, r.c, make_float4(v[0].z, v[1].z, v[2].z, v[3].z));
}

__global__ void __launch_bounds__(128) k_fill_curvature4(float* g, ThermalGrid t) {
    Rows r;
    if (!rows_of(t, r)) return;
    const std::size_t cells = t.cells;
    const Quad<true, false> nx(g, r);
    const float4 yp = ld4(g + cells, r.yp), ym = ld4(g + cells, r.ym);
    const float4 zp = ld4(g + 2U * cells, r.zp), zm = ld4(g + 2U * cells, r.zm);
    float o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        Nb ny{}, nz{};
        ny.yp = lane(yp, k);
        ny.ym = lane(ym, k);
        nz.zp = lane(zp, k);
        nz.zm = lane(zm, k);
        o[k] = curvature_cell(nx.at(k), ny, nz);
    }
    st4(g + 3U * cells, r.c, make_float4(o[0], o[1], o[2], o[3]));
}

__global__ void __launch_bounds__(128) k_surface_tension4(const float* phi, const float* curvature, ThermalGrid t,
                                                          float* ax, float* ay, float* az, float sigma,
                                                          float density) {
    Rows r;
    if (!rows_of(t, r)) return;
    const Quad<true, true> p(phi, r);
    const float4 kappa = ld4(curvature, r.c);
    float4 a = ld4(ax, r.c), b = ld4(ay, r.c), c = ld4(az, r.c);
    float3 d[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) d[k] = tension_cell(p.at(k), lane(kappa, k), sigma, density);
    a = make_float4(__fadd_rn(a.x, d[0].x), __fadd_rn(a.y, d[1].x), __fadd_rn(a.z, d[2].x), __fadd_rn(a.w, d[3].x));
    b = make_float4(__fadd_rn(b.x, d[0].y), __fadd_rn(b.y, d[1].y), __fadd_rn(b.z, d[2].y), __fadd_rn(b.w, d[3].y));
    c = make_float4(__fadd_rn(c.x, d[0].z), __fadd_rn(c.y, d[1].z), __fadd_rn(c.z, d[2].z), __fadd_rn(c.w, d[3].z));
    st4(ax, r.c, a);
    st4(ay, r.c, b);
    st4(az, r.c, c);
}

// The Q-criterion needs all six neighbours of three fields.  A thread takes
// four x-adjacent cells through kQPlanes z-planes, carrying each field's rows
// z-1, z and z+1 in registers: per plane it loads the z+1 row, the two y
// neighbour rows and the segment's two x-edge values instead of the five rows
// of the one-plane form.
constexpr u32 kQPlanes = 8U;

struct QColumn {
    float4 below, cur, above; // rows z-1, z, z+1 of the segment
    float xl, xr;             // row z at x0 - 1 and x0 + 4
};

__device__ __forceinline__ Nb q_nb(const QColumn& col, float4 yp, float4 ym, int k) {
    Nb n;
    n.c = lane(col.cur, k);
    n.xm = k == 0 ? col.xl : lane(col.cur, k - 1);
    n.xp = k == 3 ? col.xr : lane(col.cur, k + 1);
    n.yp = lane(yp, k);
    n.ym = lane(ym, k);
    n.zp = lane(col.above, k);
    n.zm = lane(col.below, k);
    return n;
}

__global__ void __launch_bounds__(128) k_resident_q4z(const float* ux, const float* uy, const float* uz, ThermalGrid t,
                                                      float* q) {
    const u32 x0 = 4U * (blockIdx.x * blockDim.x + threadIdx.x);
    if (x0 >= t.nx) return;
    const u32 y = blockIdx.y, z0 = blockIdx.z * kQPlanes;
    const u32 z_end = min(z0 + kQPlanes, t.nz);
    const u32 yp = shp(y, t.ny), ym = shm(y, t.ny);
    const u32 xl = x0 == 0U ? t.nx - 1U : x0 - 1U, xr = x0 + 4U == t.nx ? 0U : x0 + 4U;
    const float* f[3] = {ux, uy, uz};
    QColumn col[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        col[c].below = ld4(f[c], at(x0, y, shm(z0, t.nz), t));
        col[c].cur = ld4(f[c], at(x0, y, z0, t));
        col[c].above = ld4(f[c], at(x0, y, shp(z0, t.nz), t));
        col[c].xl = f[c][at(xl, y, z0, t)];
        col[c].xr = f[c][at(xr, y, z0, t)];
    }
    for (u32 z = z0; z < z_end; ++z) {
        float4 yps[3], yms[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            yps[c] = ld4(f[c], at(x0, yp, z, t));
            yms[c] = ld4(f[c], at(x0, ym, z, t));
        }
        float o[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            o[k] = q_cell(q_nb(col[0], yps[0], yms[0], k), q_nb(col[1], yps[1], yms[1], k),
                          q_nb(col[2], yps[2], yms[2], k));
        st4(q, at(x0, y, z, t), make_float4(o[0], o[1], o[2], o[3]));
        if (z + 1U < z_end) {
            const u32 zn = z + 1U, znp = shp(zn, t.nz);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                col[c].below = col[c].cur;
                col[c].cur = col[c].above;
                col[c].above = ld4(f[c], at(x0, y, znp, t));
                col[c].xl = f[c][at(xl, y, zn, t)];
                col[c].xr = f[c][at(xr, y, zn, t)];
            }
        }
    }
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

dim3 cell_grid3(const ThermalGrid& t) { return dim3((t.nx + 127U) / 128U, t.ny, t.nz); }
dim3 quad_grid(const ThermalGrid& t) { return dim3((t.nx / 4U + 127U) / 128U, t.ny, t.nz); }

bool aligned16(const void* p) { return (reinterpret_cast<std::uintptr_t>(p) & 15U) == 0U; }
// The four-cell kernels need whole float4 rows: nx % 4 == 0 and 16-byte aligned fields.
template <class... P> bool quads(const ThermalGrid& t, P... fields) {
    return t.nx % 4U == 0U && (aligned16(fields) && ...);
}

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
    if (quads(t, fill, out, ux, uy, uz))
        k_fill_advect4<<<quad_grid(t), 128, 0, s>>>(fill, out, t, ux, uy, uz, dt);
    else
        k_fill_advect<<<cell_grid3(t), 128, 0, s>>>(fill, out, t, ux, uy, uz, dt);
    return cudaGetLastError();
}

cudaError_t launch_fill_geometry(const float* fill, float* geometry, ThermalGrid t, cudaStream_t s) {
    const bool q4 = quads(t, fill, geometry);
    if (q4)
        k_fill_normals4<<<quad_grid(t), 128, 0, s>>>(fill, geometry, t);
    else
        k_fill_normals<<<cell_grid3(t), 128, 0, s>>>(fill, geometry, t);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (q4)
        k_fill_curvature4<<<quad_grid(t), 128, 0, s>>>(geometry, t);
    else
        k_fill_curvature<<<cell_grid3(t), 128, 0, s>>>(geometry, t);
    return cudaGetLastError();
}

cudaError_t launch_surface_tension(const float* fill, const float* curvature, ThermalGrid t, float* ax, float* ay,
                                   float* az, float sigma, float density, cudaStream_t s) {
    if (quads(t, fill, curvature, ax, ay, az))
        k_surface_tension4<<<quad_grid(t), 128, 0, s>>>(fill, curvature, t, ax, ay, az, sigma, density);
    else
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
    if (quads(t, ux, uy, uz, q))
        k_resident_q4z<<<dim3((t.nx / 4U + 127U) / 128U, t.ny, (t.nz + kQPlanes - 1U) / kQPlanes), 128, 0, s>>>(
            ux, uy, uz, t, q);
    else
        k_resident_q<<<cell_grid3(t), 128, 0, s>>>(ux, uy, uz, t, q);
    return cudaGetLastError();
}

} // namespace cfdx
