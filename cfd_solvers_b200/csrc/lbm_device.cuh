// Device side of the in-place Esoteric-Pull lattice-Boltzmann step (sm_100a).
//
// One thread owns one cell.  Every launch reads and writes each population
// slot exactly once: a cell reads the q slots its pairs own at this parity and
// writes the post-collision values back into the same q slots, so the update
// is race-free with a single lattice in HBM (access pattern: Lehmann,
// Computation 10(6) 92, 2022; reference esoteric_pull.hpp:349-382).
//
// Layout in HBM: populations are a structure of arrays f[d*N + n] with
// n = (z*ny + y)*nx + x (reference esoteric_pull.hpp:304-310), so a warp
// reads 32 consecutive x cells of one direction: c_x = 0 directions are
// aligned 128-byte (FP32) rows, c_x = +-1 directions are shifted by one
// element and share their edge sector with the neighbouring warp, which L1/L2
// absorb.
#pragma once

#include <cuda_fp16.h>

#include <cstdint>

#include "lattice.cuh"
#include "lbm_args.h"

namespace cfdx {

// ------------------------------------------------------------- storage traits
struct StF32 {
    using T = float;
    using R = float;
};
struct StF64 {
    using T = double;
    using R = double;
};
// FP16 shifted storage: h = half((f - w_d) * s_d), f = w_d + float(h) / s_d.
// Scales are equal within an opposite pair, so a bounced load that reads the
// partner direction's slot decodes with the same constants.
struct StF16 {
    using T = __half;
    using R = float;
};

template <class S, class L, int D>
__device__ __forceinline__ typename S::R ld(const typename S::T* p, const LbmArgs& a) {
    if constexpr (sizeof(typename S::T) == 2) {
        return fmaf(__half2float(*p), a.inv_scale[D], static_cast<float>(L::w(D)));
    } else {
        return *p;
    }
}

template <class S, class L, int D>
__device__ __forceinline__ void st(typename S::T* p, typename S::R v, const LbmArgs& a) {
    if constexpr (sizeof(typename S::T) == 2) {
        *p = __float2half_rn((v - static_cast<float>(L::w(D))) * a.scale[D]);
    } else {
        *p = v;
    }
}

// ------------------------------------------------------- periodic neighbours
// Offsets of the x-1/x/x+1, y-1/y/y+1, z-1/z/z+1 neighbours, periodic wrap
// (reference esoteric_pull.hpp:40-46).  Indexed by c + 1.
struct Nbr {
    long long ox[3], oy[3], oz[3];
};

__device__ __forceinline__ Nbr make_nbr(const LbmArgs& a, long long x, long long y, long long z) {
    Nbr o;
    const long long plane = a.nx * a.ny;
    o.ox[0] = x == 0 ? a.nx - 1 : -1;
    o.ox[1] = 0;
    o.ox[2] = x == a.nx - 1 ? -(a.nx - 1) : 1;
    o.oy[0] = (y == 0 ? a.ny - 1 : -1) * a.nx;
    o.oy[1] = 0;
    o.oy[2] = (y == a.ny - 1 ? -(a.ny - 1) : 1) * a.nx;
    o.oz[0] = (z == 0 ? a.nz - 1 : -1) * plane;
    o.oz[1] = 0;
    o.oz[2] = (z == a.nz - 1 ? -(a.nz - 1) : 1) * plane;
    return o;
}

template <class L, int D>
__device__ __forceinline__ long long nbr_off(const Nbr& o) {
    return o.ox[L::cx(D) + 1] + o.oy[L::cy(D) + 1] + o.oz[L::cz(D) + 1];
}

// ------------------------------------------------------------------- gather
// Incoming (post-streaming, pre-collision) populations of fluid cell n.
// Pair p = (i, j = i+1), nb = n + c_j is the source of direction i,
// nf = n + c_i the source of direction j.
//   even step: fin_i = f[i][nb], fin_j = f[j][n]
//   odd step:  fin_i = f[j][nb], fin_j = f[i][n]
// Half-way bounce-back in place: when the source is a wall, the incoming
// value is this cell's own outgoing opposite population of the previous
// step, which sits in the other slot of the same address -- the load swaps
// the direction index.  Moving walls add 6 w_k rho (c_k . u_wall)
// (reference src/lbm/d2q9.cpp:220-223) with rho this cell's pre-correction
// density.
template <class L, class S, bool FLAGS, int P = 0>
__device__ __forceinline__ void gather_pairs(const LbmArgs& a, const typename S::T* __restrict__ f, long long n,
                                             const Nbr& o, unsigned walls, bool odd, typename S::R* fin) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const long long nb = n + nbr_off<L, j>(o);
        const bool sb = FLAGS ? ((walls >> (2 * P)) & 1U) != 0U : false;
        const bool sf = FLAGS ? ((walls >> (2 * P + 1)) & 1U) != 0U : false;
        const std::size_t N = a.N;
        const typename S::T* pb = f + ((odd != sb) ? j : i) * N + nb;
        const typename S::T* pn = f + ((odd != sf) ? i : j) * N + n;
        fin[i] = ld<S, L, i>(pb, a);
        fin[j] = ld<S, L, j>(pn, a);
        gather_pairs<L, S, FLAGS, P + 1>(a, f, n, o, walls, odd, fin);
    }
}

template <class L, int P = 0>
__device__ __forceinline__ unsigned wall_links(const LbmArgs& a, long long n, const Nbr& o) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const unsigned b = (a.flags[n + nbr_off<L, j>(o)] & kFlagTypeMask) != 0 ? 1U : 0U;
        const unsigned fw = (a.flags[n + nbr_off<L, i>(o)] & kFlagTypeMask) != 0 ? 1U : 0U;
        return (b << (2 * P)) | (fw << (2 * P + 1)) | wall_links<L, P + 1>(a, n, o);
    } else {
        return 0U;
    }
}

template <class L, class R, int P = 0>
__device__ __forceinline__ void moving_wall_pairs(const LbmArgs& a, long long n, const Nbr& o, R rw, R* fin) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const int idb = a.flags[n + nbr_off<L, j>(o)] & kFlagTypeMask;
        if (idb >= 2) {
            const R cu = R(L::cx(i)) * R(a.wall_u[idb][0]) + R(L::cy(i)) * R(a.wall_u[idb][1]) +
                         R(L::cz(i)) * R(a.wall_u[idb][2]);
            fin[i] += R(6.0) * R(L::w(i)) * rw * cu;
        }
        const int idf = a.flags[n + nbr_off<L, i>(o)] & kFlagTypeMask;
        if (idf >= 2) {
            const R cu = R(L::cx(j)) * R(a.wall_u[idf][0]) + R(L::cy(j)) * R(a.wall_u[idf][1]) +
                         R(L::cz(j)) * R(a.wall_u[idf][2]);
            fin[j] += R(6.0) * R(L::w(j)) * rw * cu;
        }
        moving_wall_pairs<L, R, P + 1>(a, n, o, rw, fin);
    }
}

template <class L, class S, bool FLAGS>
__device__ __forceinline__ void gather(const LbmArgs& a, const typename S::T* __restrict__ f, long long n,
                                       const Nbr& o, std::uint8_t flag, typename S::R* fin) {
    using R = typename S::R;
    const bool odd = a.odd != 0;
    unsigned walls = 0U;
    if constexpr (FLAGS) {
        if (flag & kFlagNearWall) walls = wall_links<L>(a, n, o);
    }
    fin[0] = ld<S, L, 0>(f + n, a);
    gather_pairs<L, S, FLAGS>(a, f, n, o, walls, odd, fin);
    if constexpr (FLAGS) {
        if (flag & kFlagNearMoving) {
            R rho0 = R(0);
#pragma unroll
            for (int d = 0; d < L::Q; ++d) rho0 += fin[d];
            const R rw = rho0 > R(1.0e-8) ? rho0 : R(1.0e-8);
            moving_wall_pairs<L, R>(a, n, o, rw, fin);
        }
    }
}

// ------------------------------------------------------------------ scatter
// Post-collision values go back to the slots the pair was read from
// (reference esoteric_pull.hpp:367-382):
//   even step: f[j][n] = fout_i, f[i][nb] = fout_j
//   odd step:  f[i][n] = fout_i, f[j][nb] = fout_j
template <class L, class S, int P = 0>
__device__ __forceinline__ void scatter_pairs(const LbmArgs& a, typename S::T* __restrict__ f, long long n,
                                              const Nbr& o, bool odd, const typename S::R* fout) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const long long nb = n + nbr_off<L, j>(o);
        const std::size_t N = a.N;
        st<S, L, i>(f + (odd ? i : j) * N + n, fout[i], a);
        st<S, L, j>(f + (odd ? j : i) * N + nb, fout[j], a);
        scatter_pairs<L, S, P + 1>(a, f, n, o, odd, fout);
    }
}

// ---------------------------------------------------------------- moments
template <class L, class R>
__device__ __forceinline__ void moments(const R* fin, R& rho, R& ux, R& uy, R& uz) {
    R r = R(0), jx = R(0), jy = R(0), jz = R(0);
#pragma unroll
    for (int d = 0; d < L::Q; ++d) {
        r += fin[d];
        if (L::cx(d) > 0) jx += fin[d];
        if (L::cx(d) < 0) jx -= fin[d];
        if (L::cy(d) > 0) jy += fin[d];
        if (L::cy(d) < 0) jy -= fin[d];
        if (L::cz(d) > 0) jz += fin[d];
        if (L::cz(d) < 0) jz -= fin[d];
    }
    // reference esoteric_pull.hpp:397-405: u = 0 when rho <= 0
    const R inv = r > R(0) ? R(1) / r : R(0);
    rho = r;
    ux = jx * inv;
    uy = jy * inv;
    uz = jz * inv;
}

template <class R>
__device__ __forceinline__ void cell_acceleration(const LbmArgs& a, long long n, R& ax, R& ay, R& az) {
    ax = R(a.ax);
    ay = R(a.ay);
    az = R(a.az);
    if (a.local_a) {
        ax += R(a.local_a[n]);
        ay += R(a.local_a[a.N + n]);
        az += R(a.local_a[2 * a.N + n]);
    }
}

// Smagorinsky relaxation time (reference esoteric_pull.hpp:72-97 with the
// coefficient K = 18 sqrt(2) Cs^2 as a parameter).  The non-equilibrium
// momentum flux is formed as sum c_a c_b f - rho (delta_ab / 3 + u_a u_b),
// which equals sum c_a c_b (f - feq) on D3Q19/D3Q27 (both lattices are
// fourth-order isotropic) and needs no per-direction equilibria.
template <class L, class R>
__device__ __forceinline__ R les_tau(const R* fin, R rho, R ux, R uy, R uz, R tau, R k) {
    if (!(rho > R(0))) return tau;
    R sxx = R(0), syy = R(0), szz = R(0), sxy = R(0), sxz = R(0), syz = R(0);
#pragma unroll
    for (int d = 1; d < L::Q; ++d) {
        if (L::cx(d) != 0) sxx += fin[d];
        if (L::cy(d) != 0) syy += fin[d];
        if (L::cz(d) != 0) szz += fin[d];
        if (L::cx(d) * L::cy(d) > 0) sxy += fin[d];
        if (L::cx(d) * L::cy(d) < 0) sxy -= fin[d];
        if (L::cx(d) * L::cz(d) > 0) sxz += fin[d];
        if (L::cx(d) * L::cz(d) < 0) sxz -= fin[d];
        if (L::cy(d) * L::cz(d) > 0) syz += fin[d];
        if (L::cy(d) * L::cz(d) < 0) syz -= fin[d];
    }
    const R third = R(1.0 / 3.0);
    const R pxx = sxx - rho * (third + ux * ux);
    const R pyy = syy - rho * (third + uy * uy);
    const R pzz = szz - rho * (third + uz * uz);
    const R pxy = sxy - rho * ux * uy;
    const R pxz = sxz - rho * ux * uz;
    const R pyz = syz - rho * uy * uz;
    const R q = pxx * pxx + pyy * pyy + pzz * pzz + R(2) * (pxy * pxy + pxz * pxz + pyz * pyz);
    return R(0.5) * (tau + sqrt(tau * tau + k * sqrt(q) / rho));
}

// ---------------------------------------------------------------- collision
// BGK (reference esoteric_pull.hpp:408-432) or TRT (reference
// one_step_pull.hpp:187-204), both with Guo forcing, written per opposite
// pair (i, j): the equilibrium splits into a symmetric part
// w rho (1 - 1.5 u^2 + 4.5 (c.u)^2) and an antisymmetric part 3 w rho (c.u),
// the Guo source into w (9 (c.u)(c.F) - 3 u.F) and 3 w (c.F).  Gray-LBM
// partial bounce-back then mixes in the incoming opposite population:
// f_i <- (1 - n_s) f_i* + n_s fin_j (Walsh, Burwinkle & Saar 2009).
template <class L, class R, int COLL, bool GRAY, int P = 0>
__device__ __forceinline__ void collide_pairs(R* f, R rho, R ux, R uy, R uz, R fx, R fy, R fz, R usq15, R uf3,
                                              R omega, R omega_m, R gp, R gm, R ns) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        constexpr R w = R(L::w(i));
        const R cu = R(L::cx(i)) * ux + R(L::cy(i)) * uy + R(L::cz(i)) * uz;
        const R cf = R(L::cx(i)) * fx + R(L::cy(i)) * fy + R(L::cz(i)) * fz;
        const R wr = w * rho;
        const R eqp = wr * (R(1) - usq15 + R(4.5) * cu * cu);
        const R eqm = wr * (R(3) * cu);
        const R fp = w * (R(9) * cu * cf - uf3);
        const R fm = w * (R(3) * cf);
        const R fi = f[i], fj = f[j];
        R oi, oj;
        if constexpr (COLL == kBGK) {
            oi = fi - omega * (fi - (eqp + eqm)) + gp * (fp + fm);
            oj = fj - omega * (fj - (eqp - eqm)) + gp * (fp - fm);
        } else {
            const R sp = R(0.5) * (fi + fj) - eqp;
            const R sm = R(0.5) * (fi - fj) - eqm;
            const R common = gp * fp - omega * sp;
            const R anti = gm * fm - omega_m * sm;
            oi = fi + common + anti;
            oj = fj + common - anti;
        }
        if constexpr (GRAY) {
            oi = (R(1) - ns) * oi + ns * fj;
            oj = (R(1) - ns) * oj + ns * fi;
        }
        f[i] = oi;
        f[j] = oj;
        collide_pairs<L, R, COLL, GRAY, P + 1>(f, rho, ux, uy, uz, fx, fy, fz, usq15, uf3, omega, omega_m, gp, gm,
                                               ns);
    }
}

template <class L, class R, int COLL, bool LES, bool GRAY>
__device__ __forceinline__ void collide(const LbmArgs& a, long long n, R* f) {
    R rho, ux, uy, uz, ax, ay, az;
    moments<L, R>(f, rho, ux, uy, uz);
    cell_acceleration<R>(a, n, ax, ay, az);
    ux += R(0.5) * ax;
    uy += R(0.5) * ay;
    uz += R(0.5) * az;
    R tau = R(a.tau);
    if constexpr (LES) tau = les_tau<L, R>(f, rho, ux, uy, uz, tau, R(a.les_k));
    const R omega = R(1) / tau;
    R omega_m = omega;
    if constexpr (COLL == kTRT) {
        // tau- = 1/2 + Lambda / (tau+ - 1/2): omega- = (tau+ - 1/2) / (Lambda + (tau+ - 1/2) / 2)
        if (a.omega_minus > 0.0) {
            omega_m = R(a.omega_minus);
        } else {
            const R sp = tau - R(0.5);
            omega_m = sp / (R(a.trt_magic) + R(0.5) * sp);
        }
    }
    const R fx = rho * ax, fy = rho * ay, fz = rho * az;
    const R usq15 = R(1.5) * (ux * ux + uy * uy + uz * uz);
    const R uf3 = R(3) * (ux * fx + uy * fy + uz * fz);
    const R gp = R(1) - R(0.5) * omega;
    const R gm = R(1) - R(0.5) * omega_m;
    R ns = R(0);
    if constexpr (GRAY) ns = R(a.ns[n]);
    // rest population
    {
        constexpr R w0 = R(L::w(0));
        const R f0 = f[0];
        R o0 = f0 - omega * (f0 - w0 * rho * (R(1) - usq15)) - gp * w0 * uf3;
        if constexpr (GRAY) o0 = (R(1) - ns) * o0 + ns * f0;
        f[0] = o0;
    }
    collide_pairs<L, R, COLL, GRAY>(f, rho, ux, uy, uz, fx, fy, fz, usq15, uf3, omega, omega_m, gp, gm, ns);
}

// ------------------------------------------------------------------ kernels
template <class L, class S, int COLL, bool LES, bool FLAGS, bool GRAY>
__global__ void __launch_bounds__(256) k_step(const __grid_constant__ LbmArgs a) {
    using R = typename S::R;
    const long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long y = static_cast<long long>(blockIdx.y) * blockDim.y + threadIdx.y;
    const long long z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const long long n = (z * a.ny + y) * a.nx + x;
    std::uint8_t flag = 0;
    if constexpr (FLAGS) {
        flag = a.flags[n];
        if (flag & kFlagTypeMask) return; // walls hold no populations of their own
    }
    const Nbr o = make_nbr(a, x, y, z);
    typename S::T* f = static_cast<typename S::T*>(a.f);
    R fin[L::Q];
    gather<L, S, FLAGS>(a, f, n, o, flag, fin);
    collide<L, R, COLL, LES, GRAY>(a, n, fin);
    scatter_pairs<L, S>(a, f, n, o, a.odd != 0, fin);
    st<S, L, 0>(f + n, fin[0], a);
}

// Equilibrium initialisation into the esoteric slots of time step 0
// (reference esoteric_pull.hpp:312-333; Taylor-Green field :121-137).  Wall
// links additionally seed the partner slot, so that the first step's bounced
// loads see the cell's own equilibrium exactly as the reference's first
// solid step does.
template <class L, class S, bool FLAGS, int P = 0>
__device__ __forceinline__ void init_pairs(const LbmArgs& a, typename S::T* f, long long n, const Nbr& o,
                                           unsigned walls, typename S::R rho, typename S::R ux, typename S::R uy,
                                           typename S::R uz, typename S::R usq15) {
    using R = typename S::R;
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const R cu = R(L::cx(i)) * ux + R(L::cy(i)) * uy + R(L::cz(i)) * uz;
        const R wr = R(L::w(i)) * rho;
        const R fi = wr * (R(1) + R(3) * cu + R(4.5) * cu * cu - usq15);
        const R fj = wr * (R(1) - R(3) * cu + R(4.5) * cu * cu - usq15);
        const long long nb = n + nbr_off<L, j>(o);
        const std::size_t N = a.N;
        st<S, L, i>(f + i * N + nb, fi, a);
        st<S, L, j>(f + j * N + n, fj, a);
        if constexpr (FLAGS) {
            if ((walls >> (2 * P)) & 1U) st<S, L, j>(f + j * N + nb, fi, a);
            if ((walls >> (2 * P + 1)) & 1U) st<S, L, i>(f + i * N + n, fj, a);
        }
        init_pairs<L, S, FLAGS, P + 1>(a, f, n, o, walls, rho, ux, uy, uz, usq15);
    }
}

template <class L, class S, bool FLAGS>
__global__ void __launch_bounds__(256) k_init(const __grid_constant__ LbmArgs a, const InitSpec s) {
    using R = typename S::R;
    const long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long y = static_cast<long long>(blockIdx.y) * blockDim.y + threadIdx.y;
    const long long z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const long long n = (z * a.ny + y) * a.nx + x;
    unsigned walls = 0U;
    const Nbr o = make_nbr(a, x, y, z);
    if constexpr (FLAGS) {
        const std::uint8_t flag = a.flags[n];
        if (flag & kFlagTypeMask) return;
        if (flag & kFlagNearWall) walls = wall_links<L>(a, n, o);
    }
    R rho, ux, uy, uz;
    if (s.kind == 0) {
        rho = R(s.rho);
        ux = R(s.ux);
        uy = R(s.uy);
        uz = R(s.uz);
    } else if (s.kind == 1) {
        const float two_pi = 2.0F * 3.14159265358979323846F;
        const float xf = (static_cast<float>(x) + 0.5F) / static_cast<float>(a.nx);
        const float yf = (static_cast<float>(y) + 0.5F) / static_cast<float>(a.ny);
        const float zf = (static_cast<float>(z) + 0.5F) / static_cast<float>(a.nz);
        const float sx = sinf(two_pi * xf), cx = cosf(two_pi * xf);
        const float sy = sinf(two_pi * yf), cy = cosf(two_pi * yf);
        const float cz = cosf(two_pi * zf);
        rho = R(1);
        ux = R(s.amplitude * sx * cy * cz);
        uy = R(-s.amplitude * cx * sy * cz);
        uz = R(0);
    } else {
        rho = R(s.fields[n]);
        ux = R(s.fields[a.N + n]);
        uy = R(s.fields[2 * a.N + n]);
        uz = R(s.fields[3 * a.N + n]);
    }
    typename S::T* f = static_cast<typename S::T*>(a.f);
    const R usq15 = R(1.5) * (ux * ux + uy * uy + uz * uz);
    st<S, L, 0>(f + n, R(L::w(0)) * rho * (R(1) - usq15), a);
    init_pairs<L, S, FLAGS>(a, f, n, o, walls, rho, ux, uy, uz, usq15);
}

// Macroscopic fields rho and u + a/2 (reference esoteric_pull.hpp:180-209 and
// esoteric_pull_sycl.hpp:229-307); wall cells report rho = 0, u = 0.
template <class L, class S, bool FLAGS, class OutT>
__global__ void __launch_bounds__(256) k_macro(const __grid_constant__ LbmArgs a, OutT* rho_out, OutT* ux_out,
                                               OutT* uy_out, OutT* uz_out) {
    using R = typename S::R;
    const long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long y = static_cast<long long>(blockIdx.y) * blockDim.y + threadIdx.y;
    const long long z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const long long n = (z * a.ny + y) * a.nx + x;
    std::uint8_t flag = 0;
    if constexpr (FLAGS) {
        flag = a.flags[n];
        if (flag & kFlagTypeMask) {
            rho_out[n] = OutT(0);
            ux_out[n] = OutT(0);
            uy_out[n] = OutT(0);
            uz_out[n] = OutT(0);
            return;
        }
    }
    const Nbr o = make_nbr(a, x, y, z);
    R fin[L::Q];
    gather<L, S, FLAGS>(a, static_cast<const typename S::T*>(a.f), n, o, flag, fin);
    R rho, ux, uy, uz, ax, ay, az;
    moments<L, R>(fin, rho, ux, uy, uz);
    cell_acceleration<R>(a, n, ax, ay, az);
    rho_out[n] = OutT(rho);
    ux_out[n] = OutT(ux + R(0.5) * ax);
    uy_out[n] = OutT(uy + R(0.5) * ay);
    uz_out[n] = OutT(uz + R(0.5) * az);
}

// Parity-independent populations [d][n] (reference esoteric_pull.hpp:257-267).
template <class L, class S, bool FLAGS, class OutT>
__global__ void __launch_bounds__(256) k_logical(const __grid_constant__ LbmArgs a, OutT* out) {
    using R = typename S::R;
    const long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long y = static_cast<long long>(blockIdx.y) * blockDim.y + threadIdx.y;
    const long long z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const long long n = (z * a.ny + y) * a.nx + x;
    R fin[L::Q];
    std::uint8_t flag = 0;
    bool wall = false;
    if constexpr (FLAGS) {
        flag = a.flags[n];
        wall = (flag & kFlagTypeMask) != 0;
    }
    if (!wall) {
        const Nbr o = make_nbr(a, x, y, z);
        gather<L, S, FLAGS>(a, static_cast<const typename S::T*>(a.f), n, o, flag, fin);
    }
#pragma unroll
    for (int d = 0; d < L::Q; ++d) out[static_cast<std::size_t>(d) * a.N + n] = wall ? OutT(0) : OutT(fin[d]);
}

// Fluid-cell reduction with FP64 accumulation (reference
// esoteric_pull.hpp:211-255 accumulates per-cell FP32 sums in FP64; the
// reference's SYCL total_mass, esoteric_pull_sycl.hpp:327-339, used FP32).
// Each block writes its partial sums to scratch; k_reduce_final combines
// them in a fixed order, so results are bitwise reproducible for a given grid.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v += __shfl_down_sync(0xffffffffU, v, s);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffU, v, s));
    return v;
}

constexpr int kReduceThreads = 256;

// Combines kReduceFields values over the block; thread 0 gets the result.
__device__ __forceinline__ void block_combine(double (&acc)[kReduceFields]) {
    __shared__ double sm[kReduceThreads / 32][kReduceFields];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kReduceFields; ++k) acc[k] = k == 5 ? warp_max(acc[k]) : warp_sum(acc[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < kReduceFields; ++k) sm[warp][k] = acc[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < kReduceFields; ++k) {
            double v = lane < kReduceThreads / 32 ? sm[lane][k] : (k == 5 ? 0.0 : 0.0);
            acc[k] = k == 5 ? warp_max(v) : warp_sum(v);
        }
    }
}

template <class L, class S, bool FLAGS>
__global__ void __launch_bounds__(kReduceThreads) k_reduce(const __grid_constant__ LbmArgs a, double* partials) {
    using R = typename S::R;
    double acc[kReduceFields] = {0, 0, 0, 0, 0, 0, 0};
    const long long rows = a.ny * a.nz;
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
        const long long y = row % a.ny, z = row / a.ny;
        for (long long x = threadIdx.x; x < a.nx; x += blockDim.x) {
            const long long n = row * a.nx + x;
            std::uint8_t flag = 0;
            if constexpr (FLAGS) {
                flag = a.flags[n];
                if (flag & kFlagTypeMask) continue;
            }
            const Nbr o = make_nbr(a, x, y, z);
            R fin[L::Q];
            gather<L, S, FLAGS>(a, static_cast<const typename S::T*>(a.f), n, o, flag, fin);
            R rho, ux, uy, uz, ax, ay, az;
            moments<L, R>(fin, rho, ux, uy, uz);
            cell_acceleration<R>(a, n, ax, ay, az);
            ux += R(0.5) * ax;
            uy += R(0.5) * ay;
            uz += R(0.5) * az;
            const double dr = double(rho), dx = double(ux), dy = double(uy), dz = double(uz);
            acc[0] += dr;
            acc[1] += dr * dx;
            acc[2] += dr * dy;
            acc[3] += dr * dz;
            acc[4] += dr * (dx * dx + dy * dy + dz * dz);
            const double speed = double(sqrt(ux * ux + uy * uy + uz * uz));
            acc[5] = fmax(acc[5], speed);
            if (!isfinite(dr) || !isfinite(dx) || !isfinite(dy) || !isfinite(dz)) acc[6] += 1.0;
        }
    }
    block_combine(acc);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < kReduceFields; ++k) partials[static_cast<std::size_t>(blockIdx.x) * kReduceFields + k] = acc[k];
}

static __global__ void __launch_bounds__(kReduceThreads) k_reduce_final(const double* partials, int blocks, double* out) {
    double acc[kReduceFields] = {0, 0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < blocks; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < kReduceFields; ++k) {
            const double v = partials[static_cast<std::size_t>(b) * kReduceFields + k];
            acc[k] = k == 5 ? fmax(acc[k], v) : acc[k] + v;
        }
    block_combine(acc);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < kReduceFields; ++k) out[k] = acc[k];
}

// Derives the internal flag byte (wall id, near-wall bits) from the caller's
// flags.  Near-wall bits let interior cells skip all neighbour-flag loads.
template <class L>
__global__ void __launch_bounds__(256) k_prepare_flags(const __grid_constant__ LbmArgs a, const std::uint8_t* user,
                                                       std::uint8_t* out) {
    const long long x = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long long y = static_cast<long long>(blockIdx.y) * blockDim.y + threadIdx.y;
    const long long z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const long long n = (z * a.ny + y) * a.nx + x;
    const std::uint8_t t = user[n] & kFlagTypeMask;
    if (t != 0) {
        out[n] = t;
        return;
    }
    const Nbr o = make_nbr(a, x, y, z);
    std::uint8_t b = 0;
#pragma unroll
    for (int d = 1; d < L::Q; ++d) {
        long long m = n + o.ox[L::cx(d) + 1] + o.oy[L::cy(d) + 1] + o.oz[L::cz(d) + 1];
        const std::uint8_t u = user[m] & kFlagTypeMask;
        if (u != 0) b |= kFlagNearWall;
        if (u >= 2) b |= kFlagNearMoving;
    }
    out[n] = b;
}

} // namespace cfdx
