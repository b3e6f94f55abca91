// Device side of the in-place Esoteric-Pull lattice-Boltzmann step (sm_100a).
//
// One thread owns CPT cells stacked in z.  Every launch reads and writes each
// population slot exactly once: a cell reads the q slots its pairs own at this
// parity and writes the post-collision values back into the same q slots, so
// the update is race-free with a single lattice in HBM (access pattern:
// Lehmann, Computation 10(6) 92, 2022; reference esoteric_pull.hpp:349-382).
//
// Layout in HBM: populations are a structure of arrays f[d][n] with
// n = (z*ny + y)*nx + x (reference esoteric_pull.hpp:304-310), so a warp
// reads 32 consecutive x cells of one direction: c_x = 0 directions are
// aligned rows, c_x = +-1 directions are shifted by one element and share
// their edge sector with the neighbouring warp, which L1/L2 absorb.
//
// The step is HBM-bound (no tensor-core work: it is a stencil, not a
// contraction).  What limits it is bytes in flight per SM and instruction
// issue: all loads of a thread's CPT cells are issued before the first
// collision; addressing is 32-bit off per-parity slot tables held in the
// parameter bank (no parity selects, no 64-bit offsets in registers); the
// collision works on opposite-pair sums and differences.
#pragma once

#include <cuda_fp16.h>

#include <cstdint>
#include <type_traits>

#include "lattice.cuh"
#include "lbm_args.h"

namespace cfdx {

using u32 = std::uint32_t;

// ------------------------------------------------------------- storage traits
// `delta` storage types hand the kernels the deviation f - w_d from the rest
// weight instead of f itself; the collision then works in deviation space
// (see collide), so decoding and encoding are one multiply each.
struct StF32 {
    using T = float;
    using R = float;
    static constexpr bool delta = false;
    static constexpr bool scaled = false;
};
struct StF64 {
    using T = double;
    using R = double;
    static constexpr bool delta = false;
    static constexpr bool scaled = false;
};
// FP16 shifted storage: h = half((f - w_d) * s_d); kernels see f - w_d = h / s_d.
// Scales are equal within an opposite pair, so a bounced load that reads the
// partner direction's slot decodes with the same constant.
// The step kernel keeps FP16 populations in storage units h (`scaled`) and
// applies the scales per weight class (collide_scaled).
struct StF16 {
    using T = __half;
    using R = float;
    static constexpr bool delta = true;
    static constexpr bool scaled = true;
};

// RAW: FP16 values stay in storage units h (no scale applied).
template <class S, class L, int D, bool RAW = false>
__device__ __forceinline__ typename S::R ld(const typename S::T* p, const LbmArgs& a) {
    if constexpr (sizeof(typename S::T) == 2) {
        if constexpr (RAW)
            return __half2float(*p);
        else
            return __half2float(*p) * a.inv_scale[D];
    } else {
        return *p;
    }
}

template <class S, class L, int D, bool RAW = false>
__device__ __forceinline__ void st(typename S::T* p, typename S::R v, const LbmArgs& a) {
    if constexpr (sizeof(typename S::T) == 2) {
        if constexpr (RAW)
            *p = __float2half_rn(v);
        else
            *p = __float2half_rn(v * a.scale[D]);
    } else {
        *p = v;
    }
}

// ------------------------------------------------------- FP16 store rounding
// FP16 stores go through sm_100a's cvt.rs (stochastic rounding): it converts
// two FP32 values to an FP16 pair, adding rbits[12:0] (low half) and
// rbits[28:16] (high half) below the FP16 mantissa and truncating.  Uniform
// random bits make the rounding unbiased, so increments smaller than half an
// FP16 step -- a small body force, a slow flow -- survive on average instead
// of being rounded away every step.  Constant bits 0x1000 in both fields give
// round-half-away-from-zero (the "nearest" mode).  The bits come from a hash
// of the cell index and a per-step seed (LbmArgs::round_*), with one 32-bit
// word per opposite pair: the same bits for a (cell, direction) in every
// kernel, so the one-cell, paired and out-of-place steps stay bitwise equal.

// lowbias32 integer hash (C. Wellons, "hash-prospector", public domain).
__device__ __forceinline__ u32 round_hash(const LbmArgs& a, u32 n) {
    u32 x = n ^ a.round_seed;
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x & a.round_mask;
}

// Rounding word of pair slot k (0: rest, p + 1: pair p) of a cell with hash h:
// bits [12:0] round the pair's first direction 2p+1 (or the rest population),
// bits [28:16] its second direction 2p+2.
__device__ __forceinline__ u32 round_bits(const LbmArgs& a, u32 h, int k) {
    return h * (0x9E3779B9U * (2U * static_cast<u32>(k) + 1U)) + a.round_add;
}

// (hi, lo) -> FP16 pair, rounded with rbits (see above).
__device__ __forceinline__ u32 f16x2_rs(float hi, float lo, u32 rbits) {
    u32 d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    return d;
}

// One FP16 store rounded with rbits[12:0].
__device__ __forceinline__ void st_h16(__half* p, float v, u32 rbits) {
    *reinterpret_cast<unsigned short*>(p) = static_cast<unsigned short>(f16x2_rs(0.0F, v, rbits));
}

// Value the kernels hold for an absolute population f of direction D.
template <class S, class L, int D> __device__ __forceinline__ typename S::R held(typename S::R f) {
    if constexpr (S::delta) {
        return f - typename S::R(L::w(D));
    } else {
        return f;
    }
}

// Absolute population from a held value.
template <class S, class L> __device__ __forceinline__ typename S::R absolute(typename S::R v, int d) {
    if constexpr (S::delta) {
        return v + typename S::R(L::w(d));
    } else {
        return v;
    }
}

// ------------------------------------------------------- periodic neighbours
// Offsets of the x-1/x/x+1, y-1/y/y+1, z-1/z/z+1 neighbours with periodic wrap
// (reference esoteric_pull.hpp:40-46), indexed by c + 1.  Unsigned wrap-around
// arithmetic keeps n + offset exact because the true neighbour index is in [0, N).
struct Nbr {
    u32 ox[3], oy[3], oz[3];
};

__device__ __forceinline__ Nbr make_nbr(const LbmArgs& a, u32 x, u32 y, u32 z) {
    Nbr o;
    const u32 plane = a.nx * a.ny;
    o.ox[0] = x == 0 ? a.nx - 1U : 0xffffffffU;
    o.ox[1] = 0U;
    o.ox[2] = x == a.nx - 1U ? 1U - a.nx : 1U;
    o.oy[0] = y == 0 ? (a.ny - 1U) * a.nx : 0U - a.nx;
    o.oy[1] = 0U;
    o.oy[2] = y == a.ny - 1U ? 0U - (a.ny - 1U) * a.nx : a.nx;
    o.oz[0] = z == 0 ? (a.nz - 1U) * plane : 0U - plane;
    o.oz[1] = 0U;
    o.oz[2] = z == a.nz - 1U ? 0U - (a.nz - 1U) * plane : plane;
    return o;
}

template <class L, int D> __device__ __forceinline__ u32 nbr_off(const Nbr& o) {
    return o.ox[L::cx(D) + 1] + o.oy[L::cy(D) + 1] + o.oz[L::cz(D) + 1];
}

// ------------------------------------------------------------------- gather
// Incoming (post-streaming, pre-collision) populations of fluid cell n.
// Pair p = (i, j = i+1), nb = n + c_j is the source of direction i,
// nf = n + c_i the source of direction j.
//   even step: fin_i = f[i][nb], fin_j = f[j][n]
//   odd step:  fin_i = f[j][nb], fin_j = f[i][n]
// i.e. fin_i = pa[p][nb], fin_j = pb[p][n] with the per-parity tables.
// Half-way bounce-back in place: when the source is a wall, the incoming
// value is this cell's own outgoing opposite population of the previous
// step, which sits in the other slot of the same address -- the load takes
// the other table.  Moving walls add 6 w_k rho (c_k . u_wall) (reference
// src/lbm/d2q9.cpp:220-223) with rho this cell's pre-correction density.
// Slot addressing: NARROW kernels use 32-bit element offsets from one base
// pointer (q*N < 2^32: one add and one wide multiply-add per access, no
// per-access pointer loads); the wide form reads the 64-bit per-parity
// pointer tables.
template <class S, bool NARROW> struct Slots {
    using T = typename S::T;
    __device__ __forceinline__ static T* at(const LbmArgs& a, bool use_pa, int p, u32 idx) {
        if constexpr (NARROW) {
            return static_cast<T*>(a.base) + ((use_pa ? a.pa_off[p] : a.pb_off[p]) + idx);
        } else {
            return static_cast<T*>(use_pa ? a.pa[p] : a.pb[p]) + idx;
        }
    }
    __device__ __forceinline__ static T* rest(const LbmArgs& a, u32 idx) {
        if constexpr (NARROW) {
            return static_cast<T*>(a.base) + (a.rest_off + idx);
        } else {
            return static_cast<T*>(a.rest) + idx;
        }
    }
};

template <class L, class S, bool NARROW, bool RAW = false, int P = 0>
__device__ __forceinline__ void gather_plain(const LbmArgs& a, u32 n, const Nbr& o, typename S::R* fin) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        fin[i] = ld<S, L, i, RAW>(Slots<S, NARROW>::at(a, true, P, n + nbr_off<L, j>(o)), a);
        fin[j] = ld<S, L, j, RAW>(Slots<S, NARROW>::at(a, false, P, n), a);
        gather_plain<L, S, NARROW, RAW, P + 1>(a, n, o, fin);
    }
}

template <class L, class S, bool NARROW, bool RAW = false, int P = 0>
__device__ __forceinline__ void gather_walls(const LbmArgs& a, u32 n, const Nbr& o, unsigned walls,
                                             typename S::R* fin) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const bool sb = ((walls >> (2 * P)) & 1U) != 0U;
        const bool sf = ((walls >> (2 * P + 1)) & 1U) != 0U;
        fin[i] = ld<S, L, i, RAW>(Slots<S, NARROW>::at(a, !sb, P, n + nbr_off<L, j>(o)), a);
        fin[j] = ld<S, L, j, RAW>(Slots<S, NARROW>::at(a, sf, P, n), a);
        gather_walls<L, S, NARROW, RAW, P + 1>(a, n, o, walls, fin);
    }
}

template <class L, int P = 0> __device__ __forceinline__ unsigned wall_links(const LbmArgs& a, u32 n, const Nbr& o) {
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
__device__ __forceinline__ void moving_wall_pairs(const LbmArgs& a, u32 n, const Nbr& o, R rw, R* fin) {
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

template <class L, class S, bool FLAGS, bool NARROW = false, bool RAW = false>
__device__ __forceinline__ void gather_loads(const LbmArgs& a, u32 n, const Nbr& o, std::uint8_t flag,
                                             typename S::R* fin) {
    fin[0] = ld<S, L, 0, RAW>(Slots<S, NARROW>::rest(a, n), a);
    if constexpr (FLAGS) {
        if (flag & kFlagNearWall) {
            gather_walls<L, S, NARROW, RAW>(a, n, o, wall_links<L>(a, n, o), fin);
            return;
        }
    }
    gather_plain<L, S, NARROW, RAW>(a, n, o, fin);
}

// Moving-wall correction for values held in FP16 storage units: the
// correction 6 w_k rho (c_k . u_wall) is scaled by s_k.
template <class L, int P = 0>
__device__ __forceinline__ void moving_wall_pairs_scaled(const LbmArgs& a, u32 n, const Nbr& o, float rw, float* h) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const int idb = a.flags[n + nbr_off<L, j>(o)] & kFlagTypeMask;
        if (idb >= 2) {
            const float cu = float(L::cx(i)) * a.wall_u[idb][0] + float(L::cy(i)) * a.wall_u[idb][1] +
                             float(L::cz(i)) * a.wall_u[idb][2];
            h[i] += a.scale[i] * (6.0F * float(L::w(i)) * rw * cu);
        }
        const int idf = a.flags[n + nbr_off<L, i>(o)] & kFlagTypeMask;
        if (idf >= 2) {
            const float cu = float(L::cx(j)) * a.wall_u[idf][0] + float(L::cy(j)) * a.wall_u[idf][1] +
                             float(L::cz(j)) * a.wall_u[idf][2];
            h[j] += a.scale[j] * (6.0F * float(L::w(j)) * rw * cu);
        }
        moving_wall_pairs_scaled<L, P + 1>(a, n, o, rw, h);
    }
}

template <class L>
__device__ __forceinline__ void gather_fixup_scaled(const LbmArgs& a, u32 n, const Nbr& o, std::uint8_t flag,
                                                    float* h) {
    if (flag & kFlagNearMoving) {
        float rho0 = 1.0F;
#pragma unroll
        for (int d = 0; d < L::Q; ++d) rho0 += h[d] * a.inv_scale[d];
        const float rw = rho0 > 1.0e-8F ? rho0 : 1.0e-8F;
        moving_wall_pairs_scaled<L>(a, n, o, rw, h);
    }
}

template <class L, class S, bool FLAGS>
__device__ __forceinline__ void gather_fixup(const LbmArgs& a, u32 n, const Nbr& o, std::uint8_t flag,
                                             typename S::R* fin) {
    using R = typename S::R;
    if constexpr (FLAGS) {
        if (flag & kFlagNearMoving) {
            R rho0 = S::delta ? R(1) : R(0);
#pragma unroll
            for (int d = 0; d < L::Q; ++d) rho0 += fin[d];
            const R rw = rho0 > R(1.0e-8) ? rho0 : R(1.0e-8);
            moving_wall_pairs<L, R>(a, n, o, rw, fin);
        }
    }
}

template <class L, class S, bool FLAGS>
__device__ __forceinline__ void gather(const LbmArgs& a, u32 n, const Nbr& o, std::uint8_t flag,
                                       typename S::R* fin) {
    gather_loads<L, S, FLAGS>(a, n, o, flag, fin);
    gather_fixup<L, S, FLAGS>(a, n, o, flag, fin);
}

// ------------------------------------------------------------------ scatter
// Post-collision values go back to the slots the pair was read from
// (reference esoteric_pull.hpp:367-382):
//   even step: f[j][n] = fout_i, f[i][nb] = fout_j
//   odd step:  f[i][n] = fout_i, f[j][nb] = fout_j
// i.e. fout_i -> pb[p][n], fout_j -> pa[p][nb].
template <class L, class S, bool NARROW, bool RAW = false, int P = 0>
__device__ __forceinline__ void scatter_pairs(const LbmArgs& a, u32 n, const Nbr& o, const typename S::R* fout,
                                              u32 h) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        auto* pi = Slots<S, NARROW>::at(a, false, P, n);
        auto* pj = Slots<S, NARROW>::at(a, true, P, n + nbr_off<L, j>(o));
        if constexpr (sizeof(typename S::T) == 2) {
            const float vi = RAW ? fout[i] : fout[i] * a.scale[i];
            const float vj = RAW ? fout[j] : fout[j] * a.scale[j];
            const u32 w = f16x2_rs(vj, vi, round_bits(a, h, P + 1));
            *reinterpret_cast<unsigned short*>(pi) = static_cast<unsigned short>(w);
            *reinterpret_cast<unsigned short*>(pj) = static_cast<unsigned short>(w >> 16);
        } else {
            st<S, L, i, RAW>(pi, fout[i], a);
            st<S, L, j, RAW>(pj, fout[j], a);
        }
        scatter_pairs<L, S, NARROW, RAW, P + 1>(a, n, o, fout, h);
    }
}

// h: the cell's rounding hash (round_hash; FP16 storage only).
template <class L, class S, bool NARROW, bool RAW = false>
__device__ __forceinline__ void scatter(const LbmArgs& a, u32 n, const Nbr& o, const typename S::R* fout, u32 h) {
    if constexpr (sizeof(typename S::T) == 2) {
        const float v0 = RAW ? fout[0] : fout[0] * a.scale[0];
        st_h16(Slots<S, NARROW>::rest(a, n), v0, round_bits(a, h, 0));
    } else {
        st<S, L, 0, RAW>(Slots<S, NARROW>::rest(a, n), fout[0], a);
    }
    scatter_pairs<L, S, NARROW, RAW>(a, n, o, fout, h);
}

// ------------------------------------------------------------------ helpers
// Reciprocals.  rcp: the hardware approximation (__fdividef, within 2 ulp),
// for relaxation rates, which enter a cell's mass and momentum alike.
// rcp_unbiased, for 1/rho in u = j / rho: the collision returns the momentum
// rho u, so an error in 1/rho that leans one way (an approximation's does)
// moves every cell's momentum the same way each step.  One Newton-Raphson step
// r + r (1 - x r) on the approximation leaves a symmetric error of about half
// an ulp at the cost of two fused multiply-adds.
__device__ __forceinline__ float rcp(float x) { return __fdividef(1.0F, x); }
__device__ __forceinline__ float rcp_unbiased(float x) {
    const float r = __fdividef(1.0F, x);
    return fmaf(r, fmaf(-x, r, 1.0F), r);
}
__device__ __forceinline__ double rcp_unbiased(double x) { return 1.0 / x; }
__device__ __forceinline__ double rcp(double x) { return 1.0 / x; }

// ---------------------------------------------------------------- moments
// rho and u of a cell (reference esoteric_pull.hpp:384-406), summed per
// opposite pair: s_p = f_i + f_j, d_p = f_i - f_j (c_j = -c_i).
template <class L, class R, int P = 0>
__device__ __forceinline__ void pair_sums(const R* f, R* s, R* d) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        s[P] = f[i] + f[j];
        d[P] = f[i] - f[j];
        pair_sums<L, R, P + 1>(f, s, d);
    }
}

// DELTA: the values are deviations f - w, whose rest weights sum to 1.
template <class L, class R, bool DELTA = false>
__device__ __forceinline__ void pair_moments(R f0, const R* s, const R* d, R& rho, R& jx, R& jy, R& jz) {
    R r = f0, x = R(0), y = R(0), z = R(0);
#pragma unroll
    for (int p = 0; p < L::PAIRS; ++p) {
        const int i = 2 * p + 1;
        r += s[p];
        if (L::cx(i) > 0) x += d[p];
        if (L::cx(i) < 0) x -= d[p];
        if (L::cy(i) > 0) y += d[p];
        if (L::cy(i) < 0) y -= d[p];
        if (L::cz(i) > 0) z += d[p];
        if (L::cz(i) < 0) z -= d[p];
    }
    rho = DELTA ? R(1) + r : r;
    jx = x;
    jy = y;
    jz = z;
}

template <class L, class R, bool DELTA = false>
__device__ __forceinline__ void moments(const R* fin, R& rho, R& ux, R& uy, R& uz) {
    R s[L::PAIRS], d[L::PAIRS], jx, jy, jz;
    pair_sums<L, R>(fin, s, d);
    pair_moments<L, R, DELTA>(fin[0], s, d, rho, jx, jy, jz);
    // reference esoteric_pull.hpp:397-405: u = 0 when rho <= 0
    const R inv = rho > R(0) ? rcp_unbiased(rho) : R(0);
    ux = jx * inv;
    uy = jy * inv;
    uz = jz * inv;
}

template <class R> __device__ __forceinline__ void cell_acceleration(const LbmArgs& a, u32 n, R& ax, R& ay, R& az) {
    ax = R(a.ax);
    ay = R(a.ay);
    az = R(a.az);
    if (a.ax_field) {
        ax += R(a.ax_field[n]);
        ay += R(a.ay_field[n]);
        az += R(a.az_field[n]);
    }
}

// Smagorinsky relaxation time (reference esoteric_pull.hpp:72-97 with the
// coefficient K = 18 sqrt(2) Cs^2 as a parameter).  The non-equilibrium
// momentum flux is formed as sum c_a c_b f - rho (delta_ab / 3 + u_a u_b),
// which equals sum c_a c_b (f - feq) on D3Q19/D3Q27 (both lattices are
// fourth-order isotropic) and needs no per-direction equilibria; c_a c_b is
// even in c, so the sums run over pair sums s_p.
template <class L, class R, bool DELTA = false>
__device__ __forceinline__ R les_tau(const R* s, R rho, R irho, R ux, R uy, R uz, R tau, R k) {
    if (!(rho > R(0))) return tau;
    R sxx = R(0), syy = R(0), szz = R(0), sxy = R(0), sxz = R(0), syz = R(0);
#pragma unroll
    for (int p = 0; p < L::PAIRS; ++p) {
        const int i = 2 * p + 1;
        if (L::cx(i) != 0) sxx += s[p];
        if (L::cy(i) != 0) syy += s[p];
        if (L::cz(i) != 0) szz += s[p];
        if (L::cx(i) * L::cy(i) > 0) sxy += s[p];
        if (L::cx(i) * L::cy(i) < 0) sxy -= s[p];
        if (L::cx(i) * L::cz(i) > 0) sxz += s[p];
        if (L::cx(i) * L::cz(i) < 0) sxz -= s[p];
        if (L::cy(i) * L::cz(i) > 0) syz += s[p];
        if (L::cy(i) * L::cz(i) < 0) syz -= s[p];
    }
    const R third = R(1.0 / 3.0);
    if constexpr (DELTA) { // sum_d c_a c_b w_d = delta_ab / 3
        sxx += third;
        syy += third;
        szz += third;
    }
    const R pxx = sxx - rho * (third + ux * ux);
    const R pyy = syy - rho * (third + uy * uy);
    const R pzz = szz - rho * (third + uz * uz);
    const R pxy = sxy - rho * ux * uy;
    const R pxz = sxz - rho * ux * uz;
    const R pyz = syz - rho * uy * uz;
    const R q = pxx * pxx + pyy * pyy + pzz * pzz + R(2) * (pxy * pxy + pxz * pxz + pyz * pyz);
    return R(0.5) * (tau + sqrt(tau * tau + k * sqrt(q) * irho));
}

// ---------------------------------------------------------------- collision
// Two-relaxation-time collision with Guo forcing (reference
// one_step_pull.hpp:187-204; BGK, esoteric_pull.hpp:408-432, is the case
// omega- = omega+), evaluated per opposite pair on s = f_i + f_j and
// d = f_i - f_j:
//   equilibrium  s_eq = 2 w rho t,  t = 1 - 1.5 u^2 + 4.5 (c.u)^2,   d_eq = 2 w rho (3 c.u)
//   Guo source   s_F  = 2 w (9 (c.u)(c.F) - 3 u.F),                d_F  = 6 w (c.F)
//   s' = s - omega+ (s - s_eq) + (1 - omega+/2) s_F
//   d' = d - omega- (d - d_eq) + (1 - omega-/2) d_F
//   f_i' = (s' + d') / 2,  f_j' = (s' - d') / 2
// The halves s'/2 and d'/2 are formed directly with per-weight-class
// coefficients computed once per cell, so a pair costs a handful of fused
// multiply-adds.  With DELTA the values are deviations f - w: s_eq becomes
// 2 w (rho t - 1) (w_i = w_j within a pair, so d is unchanged).  Gray-LBM
// partial bounce-back then mixes in the incoming opposite population:
// f_i <- (1 - n_s) f_i' + n_s fin_j (Walsh, Burwinkle & Saar 2009).
//
// Rounding: the mass and momentum coefficients both derive from the per-cell
// product w rho (rounded differently in every cell), then times omega+ or
// omega-.  A coefficient formed from constants alone (3 omega- w) carries one
// rounding error shared by every cell and every step, which the collision
// turns into a steady gain or loss of momentum against mass: with
// 3 omega- w rho, a 64^3 Taylor-Green vortex in FP32 gained kinetic energy at
// 2.3e-7 relative per step against FP64.  What remains is the representation
// error of the FP32 weights themselves, as in the reference.
template <class R> struct ClassCoef {
    R a;  // omega+ w rho          (s'/2 equilibrium term: a * t)
    R a0; // omega+ w              (DELTA: subtracted)
    R c;  // omega- w rho          (d'/2 equilibrium term: c * (3 c.u))
    R g1; // 3 (1 - omega+/2) w    (s'/2 force term: g1 * ((3 c.u)(c.F) - u.F))
    R g2; // 3 (1 - omega-/2) w    (d'/2 force term)
};

template <class L, class R, bool FORCE, bool GRAY, bool DELTA, int P = 0>
__device__ __forceinline__ void collide_pairs(R* f, const R* s, const R* d, const ClassCoef<R>* cc, R ux3, R uy3,
                                              R uz3, R ux15, R uy15, R uz15, R fx, R fy, R fz, R base, R uf, R a1,
                                              R b1, R ns) {
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const ClassCoef<R>& k = cc[weight_class<L>(i)];
        const R cu3 = R(L::cx(i)) * ux3 + R(L::cy(i)) * uy3 + R(L::cz(i)) * uz3;     // 3 c.u
        const R cu15 = R(L::cx(i)) * ux15 + R(L::cy(i)) * uy15 + R(L::cz(i)) * uz15; // 1.5 c.u
        const R t = cu3 * cu15 + base;
        R sp = DELTA ? k.a * t + (a1 * s[P] - k.a0) : k.a * t + a1 * s[P];
        R dp = k.c * cu3 + b1 * d[P];
        if constexpr (FORCE) {
            const R cf = R(L::cx(i)) * fx + R(L::cy(i)) * fy + R(L::cz(i)) * fz;
            sp += k.g1 * (cu3 * cf - uf);
            dp += k.g2 * cf;
        }
        R oi = sp + dp;
        R oj = sp - dp;
        if constexpr (GRAY) {
            const R fi = R(0.5) * (s[P] + d[P]);
            const R fj = R(0.5) * (s[P] - d[P]);
            oi = (R(1) - ns) * oi + ns * fj;
            oj = (R(1) - ns) * oj + ns * fi;
        }
        f[i] = oi;
        f[j] = oj;
        collide_pairs<L, R, FORCE, GRAY, DELTA, P + 1>(f, s, d, cc, ux3, uy3, uz3, ux15, uy15, uz15, fx, fy, fz, base,
                                                       uf, a1, b1, ns);
    }
}

// Relaxation rates of a cell: omega+ from tau (LES-adjusted) and omega- by
// the configured rule.
template <class R> __device__ __forceinline__ R omega_minus_of(const LbmArgs& a, R tau, R omega) {
    if (a.omega_minus > 0.0) return R(a.omega_minus); // fixed TRT antisymmetric rate
    if (a.omega_minus < 0.0) return omega;           // BGK
    // TRT magic: tau- = 1/2 + Lambda / (tau+ - 1/2)
    const R sp = tau - R(0.5);
    return sp * rcp(R(a.trt_magic) + R(0.5) * sp);
}

// Per weight class coefficients; `scale` multiplies every term (FP16 storage
// units), 1 otherwise.
template <class L, class R>
__device__ __forceinline__ void class_coefficients(ClassCoef<R>* cc, R rho, R omega, R omega_m, R gp, R gm,
                                                   const R* scale) {
    constexpr int K = L::Q == 27 ? 3 : 2;
#pragma unroll
    for (int k = 1; k <= K; ++k) {
        const R w = R(L::w(class_rep(k))) * scale[k];
        const R wr = w * rho;
        cc[k].a0 = omega * w;
        cc[k].a = omega * wr;
        cc[k].c = omega_m * wr;
        cc[k].g1 = R(3) * gp * w;
        cc[k].g2 = R(3) * gm * w;
    }
}

template <class L, class R, bool LES, bool GRAY, bool FORCE, bool DELTA = false>
__device__ __forceinline__ void collide(const LbmArgs& a, u32 n, R* f) {
    R s[L::PAIRS], d[L::PAIRS];
    pair_sums<L, R>(f, s, d);
    R rho, jx, jy, jz;
    pair_moments<L, R, DELTA>(f[0], s, d, rho, jx, jy, jz);
    const R inv = rho > R(0) ? rcp_unbiased(rho) : R(0);
    R ux = jx * inv, uy = jy * inv, uz = jz * inv;
    R ax = R(0), ay = R(0), az = R(0);
    if constexpr (FORCE) {
        cell_acceleration<R>(a, n, ax, ay, az);
        ux += R(0.5) * ax;
        uy += R(0.5) * ay;
        uz += R(0.5) * az;
    }
    R tau = R(a.tau);
    if constexpr (LES) tau = les_tau<L, R, DELTA>(s, rho, inv, ux, uy, uz, tau, R(a.les_k));
    const R omega = rcp(tau);
    const R omega_m = omega_minus_of<R>(a, tau, omega);
    const R base = R(1) - R(1.5) * (ux * ux + uy * uy + uz * uz);
    R fx = R(0), fy = R(0), fz = R(0), uf = R(0);
    if constexpr (FORCE) {
        fx = rho * ax;
        fy = rho * ay;
        fz = rho * az;
        uf = ux * fx + uy * fy + uz * fz;
    }
    const R gp = R(1) - R(0.5) * omega;
    const R gm = R(1) - R(0.5) * omega_m;
    R ns = R(0);
    if constexpr (GRAY) ns = R(a.ns[n]);
    {
        constexpr R w0 = R(L::w(0));
        const R f0 = f[0];
        R o0 = (R(1) - omega) * f0 + omega * (DELTA ? w0 * (rho * base - R(1)) : (w0 * rho) * base);
        if constexpr (FORCE) o0 -= gp * w0 * (R(3) * uf);
        if constexpr (GRAY) o0 = (R(1) - ns) * o0 + ns * f0;
        f[0] = o0;
    }
    ClassCoef<R> cc[4];
    const R unit[4] = {R(1), R(1), R(1), R(1)};
    class_coefficients<L, R>(cc, rho, omega, omega_m, gp, gm, unit);
    collide_pairs<L, R, FORCE, GRAY, DELTA>(f, s, d, cc, R(3) * ux, R(3) * uy, R(3) * uz, R(1.5) * ux, R(1.5) * uy,
                                            R(1.5) * uz, fx, fy, fz, base, uf, R(0.5) * (R(1) - omega),
                                            R(0.5) * (R(1) - omega_m), ns);
}

// --------------------------------------------------- FP16 scaled collision
// The same TRT/Guo/gray update as collide, for values held in FP16 storage
// units h = (f - w) s_k, with s_k constant within each weight class k.
// Pair sums stay in storage units: the moments scale each class's partial
// sums once, and the scales are folded into the per-class coefficients
// (ClassCoef scaled by s_k), so decoding and encoding cost only the
// half <-> float conversions.
template <class L, bool LES, bool GRAY, bool FORCE>
__device__ __forceinline__ void collide_scaled(const LbmArgs& a, u32 n, float* h) {
    float sh[L::PAIRS], dh[L::PAIRS];
    pair_sums<L, float>(h, sh, dh);
    // Per weight class partial sums (classes 1..3), scaled once each.
    float S[4] = {0, 0, 0, 0}, JX[4] = {0, 0, 0, 0}, JY[4] = {0, 0, 0, 0}, JZ[4] = {0, 0, 0, 0};
    float XX[4] = {0, 0, 0, 0}, YY[4] = {0, 0, 0, 0}, ZZ[4] = {0, 0, 0, 0};
    float XY[4] = {0, 0, 0, 0}, XZ[4] = {0, 0, 0, 0}, YZ[4] = {0, 0, 0, 0};
#pragma unroll
    for (int p = 0; p < L::PAIRS; ++p) {
        const int i = 2 * p + 1;
        const int k = weight_class<L>(i);
        S[k] += sh[p];
        if (L::cx(i) > 0) JX[k] += dh[p];
        if (L::cx(i) < 0) JX[k] -= dh[p];
        if (L::cy(i) > 0) JY[k] += dh[p];
        if (L::cy(i) < 0) JY[k] -= dh[p];
        if (L::cz(i) > 0) JZ[k] += dh[p];
        if (L::cz(i) < 0) JZ[k] -= dh[p];
        if constexpr (LES) {
            if (L::cx(i) != 0) XX[k] += sh[p];
            if (L::cy(i) != 0) YY[k] += sh[p];
            if (L::cz(i) != 0) ZZ[k] += sh[p];
            if (L::cx(i) * L::cy(i) > 0) XY[k] += sh[p];
            if (L::cx(i) * L::cy(i) < 0) XY[k] -= sh[p];
            if (L::cx(i) * L::cz(i) > 0) XZ[k] += sh[p];
            if (L::cx(i) * L::cz(i) < 0) XZ[k] -= sh[p];
            if (L::cy(i) * L::cz(i) > 0) YZ[k] += sh[p];
            if (L::cy(i) * L::cz(i) < 0) YZ[k] -= sh[p];
        }
    }
    constexpr int K = L::Q == 27 ? 3 : 2;
    float inv[4];
#pragma unroll
    for (int k = 0; k <= K; ++k) inv[k] = a.inv_scale[class_rep(k)];
    float rho = h[0] * inv[0], jx = 0.0F, jy = 0.0F, jz = 0.0F;
#pragma unroll
    for (int k = 1; k <= K; ++k) {
        rho += S[k] * inv[k];
        jx += JX[k] * inv[k];
        jy += JY[k] * inv[k];
        jz += JZ[k] * inv[k];
    }
    rho += 1.0F;
    const float irho = rho > 0.0F ? rcp_unbiased(rho) : 0.0F;
    float ux = jx * irho, uy = jy * irho, uz = jz * irho;
    float ax = 0.0F, ay = 0.0F, az = 0.0F;
    if constexpr (FORCE) {
        cell_acceleration<float>(a, n, ax, ay, az);
        ux += 0.5F * ax;
        uy += 0.5F * ay;
        uz += 0.5F * az;
    }
    float tau = float(a.tau);
    if constexpr (LES) {
        if (rho > 0.0F) {
            const float third = 1.0F / 3.0F;
            float sxx = third, syy = third, szz = third, sxy = 0.0F, sxz = 0.0F, syz = 0.0F;
#pragma unroll
            for (int k = 1; k <= K; ++k) {
                sxx += XX[k] * inv[k];
                syy += YY[k] * inv[k];
                szz += ZZ[k] * inv[k];
                sxy += XY[k] * inv[k];
                sxz += XZ[k] * inv[k];
                syz += YZ[k] * inv[k];
            }
            const float pxx = sxx - rho * (third + ux * ux);
            const float pyy = syy - rho * (third + uy * uy);
            const float pzz = szz - rho * (third + uz * uz);
            const float pxy = sxy - rho * ux * uy;
            const float pxz = sxz - rho * ux * uz;
            const float pyz = syz - rho * uy * uz;
            const float q = pxx * pxx + pyy * pyy + pzz * pzz + 2.0F * (pxy * pxy + pxz * pxz + pyz * pyz);
            tau = 0.5F * (tau + sqrtf(tau * tau + float(a.les_k) * sqrtf(q) * irho));
        }
    }
    const float omega = rcp(tau);
    const float omega_m = omega_minus_of<float>(a, tau, omega);
    const float base = 1.0F - 1.5F * (ux * ux + uy * uy + uz * uz);
    float fx = 0.0F, fy = 0.0F, fz = 0.0F, uf = 0.0F;
    if constexpr (FORCE) {
        fx = rho * ax;
        fy = rho * ay;
        fz = rho * az;
        uf = ux * fx + uy * fy + uz * fz;
    }
    const float gp = 1.0F - 0.5F * omega;
    const float gm = 1.0F - 0.5F * omega_m;
    float ns = 0.0F;
    if constexpr (GRAY) ns = a.ns[n];
    {
        constexpr float w0 = float(L::w(0));
        const float h0 = h[0];
        float o0 = (1.0F - omega) * h0 + a.scale[0] * (omega * w0 * (rho * base - 1.0F));
        if constexpr (FORCE) o0 -= a.scale[0] * (gp * w0 * (3.0F * uf));
        if constexpr (GRAY) o0 = (1.0F - ns) * o0 + ns * h0;
        h[0] = o0;
    }
    ClassCoef<float> cc[4];
    float scl[4];
#pragma unroll
    for (int k = 0; k <= K; ++k) scl[k] = a.scale[class_rep(k)];
    class_coefficients<L, float>(cc, rho, omega, omega_m, gp, gm, scl);
    collide_pairs<L, float, FORCE, GRAY, true>(h, sh, dh, cc, 3.0F * ux, 3.0F * uy, 3.0F * uz, 1.5F * ux, 1.5F * uy,
                                               1.5F * uz, fx, fy, fz, base, uf, 0.5F * (1.0F - omega),
                                               0.5F * (1.0F - omega_m), ns);
}

// ---------------------------------------------------------------- the step
// CPT cells per thread (stacked in z): the loads of all of a thread's cells are
// issued before the first collision.  One cell per thread measured best on
// B200 (more cells cost occupancy through registers), and the launcher uses 1.
// Minimum resident 128-thread blocks per SM the step kernels are compiled for;
// it caps registers at 65536 / (128 * blocks).  The step is latency bound at
// the occupancy its natural register count allows: measured on B200 at 512^3,
// 10 blocks (48 registers, a few spilled words that stay in L1) beat the
// uncapped 64-96 registers by 10-55% for FP32 and FP16 storage; FP64 storage
// keeps its full register set.  The macros exist for tuning builds.
#ifndef CFDX_STEP_MIN_BLOCKS_Q19
#define CFDX_STEP_MIN_BLOCKS_Q19 10
#endif
#ifndef CFDX_STEP_MIN_BLOCKS_Q27_F16
#define CFDX_STEP_MIN_BLOCKS_Q27_F16 10
#endif
#ifndef CFDX_STEP_MIN_BLOCKS_Q27_F32
#define CFDX_STEP_MIN_BLOCKS_Q27_F32 8
#endif
#ifndef CFDX_PAIR_MIN_BLOCKS
#define CFDX_PAIR_MIN_BLOCKS 8
#endif

template <class L, class S> constexpr int step_min_blocks() {
    return sizeof(typename S::T) == 8 ? 1
         : (L::Q == 19 ? CFDX_STEP_MIN_BLOCKS_Q19
                       : (sizeof(typename S::T) == 2 ? CFDX_STEP_MIN_BLOCKS_Q27_F16 : CFDX_STEP_MIN_BLOCKS_Q27_F32));
}
template <class S> constexpr int pair_min_blocks() { return sizeof(typename S::T) == 8 ? 1 : CFDX_PAIR_MIN_BLOCKS; }

template <class L, class S, bool LES, bool FLAGS, bool GRAY, int CPT, bool NARROW>
__global__ void __launch_bounds__(128, step_min_blocks<L, S>()) k_step(const __grid_constant__ LbmArgs a) {
    using R = typename S::R;
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z0 = blockIdx.z * CPT;
    if (x >= a.nx || y >= a.ny) return;
    R fin[CPT][L::Q];
    std::uint8_t flag[CPT];
    bool live[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        const u32 z = z0 + c;
        const u32 n = (z * a.ny + y) * a.nx + x;
        live[c] = z < a.nz;
        flag[c] = 0;
        if constexpr (FLAGS) {
            if (live[c]) {
                flag[c] = a.flags[n];
                live[c] = (flag[c] & kFlagTypeMask) == 0; // walls hold no populations of their own
            }
        }
        if (live[c]) gather_loads<L, S, FLAGS, NARROW, S::scaled>(a, n, make_nbr(a, x, y, z), flag[c], fin[c]);
    }
    const bool force = a.has_force != 0;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        if (!live[c]) continue;
        const u32 z = z0 + c;
        const u32 n = (z * a.ny + y) * a.nx + x;
        const Nbr o = make_nbr(a, x, y, z);
        if constexpr (S::scaled) {
            if constexpr (FLAGS) gather_fixup_scaled<L>(a, n, o, flag[c], fin[c]);
            if (force)
                collide_scaled<L, LES, GRAY, true>(a, n, fin[c]);
            else
                collide_scaled<L, LES, GRAY, false>(a, n, fin[c]);
        } else {
            gather_fixup<L, S, FLAGS>(a, n, o, flag[c], fin[c]);
            if (force)
                collide<L, R, LES, GRAY, true, S::delta>(a, n, fin[c]);
            else
                collide<L, R, LES, GRAY, false, S::delta>(a, n, fin[c]);
        }
        const u32 h = sizeof(typename S::T) == 2 ? round_hash(a, n) : 0U;
        scatter<L, S, NARROW, S::scaled>(a, n, o, fin[c], h);
    }
}

// Equilibrium initialisation into the esoteric slots of time step 0
// (reference esoteric_pull.hpp:312-333; Taylor-Green field :121-137).  Wall
// links additionally seed the partner slot, so that the first step's bounced
// loads see the cell's own equilibrium exactly as the reference's first
// solid step does.  Uses the parity-0 tables.
template <class L, class S, bool FLAGS, int P = 0>
__device__ __forceinline__ void init_pairs(const LbmArgs& a, u32 n, const Nbr& o, unsigned walls, typename S::R rho,
                                           typename S::R ux, typename S::R uy, typename S::R uz,
                                           typename S::R usq15) {
    using R = typename S::R;
    if constexpr (P < L::PAIRS) {
        constexpr int i = 2 * P + 1, j = i + 1;
        const R cu = R(L::cx(i)) * ux + R(L::cy(i)) * uy + R(L::cz(i)) * uz;
        const R wr = R(L::w(i)) * rho;
        const R fi = wr * (R(1) + R(3) * cu + R(4.5) * cu * cu - usq15);
        const R fj = wr * (R(1) - R(3) * cu + R(4.5) * cu * cu - usq15);
        const u32 nb = n + nbr_off<L, j>(o);
        const R hi = held<S, L, i>(fi), hj = held<S, L, j>(fj);
        st<S, L, i>(static_cast<typename S::T*>(a.fd[i]) + nb, hi, a);
        st<S, L, j>(static_cast<typename S::T*>(a.fd[j]) + n, hj, a);
        if constexpr (FLAGS) {
            if ((walls >> (2 * P)) & 1U) st<S, L, j>(static_cast<typename S::T*>(a.fd[j]) + nb, hi, a);
            if ((walls >> (2 * P + 1)) & 1U) st<S, L, i>(static_cast<typename S::T*>(a.fd[i]) + n, hj, a);
        }
        init_pairs<L, S, FLAGS, P + 1>(a, n, o, walls, rho, ux, uy, uz, usq15);
    }
}

template <class L, class S, bool FLAGS>
__global__ void __launch_bounds__(128) k_init(const __grid_constant__ LbmArgs a, const InitSpec s) {
    using R = typename S::R;
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const u32 n = (z * a.ny + y) * a.nx + x;
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
        // Evaluated in the arithmetic type, as the reference's FP32
        // (esoteric_pull.hpp:121-137) and FP64 (precision_pull.hpp:75-95) solvers do.
        const R two_pi = R(2) * R(3.14159265358979323846);
        const R xf = (R(x) + R(0.5)) / R(a.nx);
        const R yf = (R(y) + R(0.5)) / R(a.ny);
        const R zf = (R(z) + R(0.5)) / R(a.nz);
        const R sx = sin(two_pi * xf), cx = cos(two_pi * xf);
        const R sy = sin(two_pi * yf), cy = cos(two_pi * yf);
        const R cz = cos(two_pi * zf);
        const R amp = R(s.amplitude);
        rho = R(1);
        ux = amp * sx * cy * cz;
        uy = -amp * cx * sy * cz;
        uz = R(0);
    } else {
        rho = R(s.fields[n]);
        ux = R(s.fields[std::size_t(a.N) + n]);
        uy = R(s.fields[2 * std::size_t(a.N) + n]);
        uz = R(s.fields[3 * std::size_t(a.N) + n]);
    }
    const R usq15 = R(1.5) * (ux * ux + uy * uy + uz * uz);
    st<S, L, 0>(static_cast<typename S::T*>(a.fd[0]) + n, held<S, L, 0>(R(L::w(0)) * rho * (R(1) - usq15)), a);
    init_pairs<L, S, FLAGS>(a, n, o, walls, rho, ux, uy, uz, usq15);
}

// Macroscopic fields rho and u + a/2 (reference esoteric_pull.hpp:180-209 and
// esoteric_pull_sycl.hpp:229-307); wall cells report rho = 0, u = 0.
template <class L, class S, bool FLAGS, class OutT>
__global__ void __launch_bounds__(128) k_macro(const __grid_constant__ LbmArgs a, OutT* rho_out, OutT* ux_out,
                                               OutT* uy_out, OutT* uz_out) {
    using R = typename S::R;
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const u32 n = (z * a.ny + y) * a.nx + x;
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
    R fin[L::Q];
    gather<L, S, FLAGS>(a, n, make_nbr(a, x, y, z), flag, fin);
    R rho, ux, uy, uz, ax, ay, az;
    moments<L, R, S::delta>(fin, rho, ux, uy, uz);
    cell_acceleration<R>(a, n, ax, ay, az);
    rho_out[n] = OutT(rho);
    ux_out[n] = OutT(ux + R(0.5) * ax);
    uy_out[n] = OutT(uy + R(0.5) * ay);
    uz_out[n] = OutT(uz + R(0.5) * az);
}

// Parity-independent populations [d][n] (reference esoteric_pull.hpp:257-267).
template <class L, class S, bool FLAGS, class OutT>
__global__ void __launch_bounds__(128) k_logical(const __grid_constant__ LbmArgs a, OutT* out) {
    using R = typename S::R;
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const u32 n = (z * a.ny + y) * a.nx + x;
    R fin[L::Q];
    std::uint8_t flag = 0;
    bool wall = false;
    if constexpr (FLAGS) {
        flag = a.flags[n];
        wall = (flag & kFlagTypeMask) != 0;
    }
    if (!wall) gather<L, S, FLAGS>(a, n, make_nbr(a, x, y, z), flag, fin);
#pragma unroll
    for (int d = 0; d < L::Q; ++d)
        out[static_cast<std::size_t>(d) * a.N + n] = wall ? OutT(0) : OutT(absolute<S, L>(fin[d], d));
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
            const double v = lane < kReduceThreads / 32 ? sm[lane][k] : 0.0;
            acc[k] = k == 5 ? warp_max(v) : warp_sum(v);
        }
    }
}

template <class L, class S, bool FLAGS>
__global__ void __launch_bounds__(kReduceThreads) k_reduce(const __grid_constant__ LbmArgs a, double* partials) {
    using R = typename S::R;
    double acc[kReduceFields] = {0, 0, 0, 0, 0, 0, 0};
    const u32 rows = a.ny * a.nz;
    for (u32 row = blockIdx.x; row < rows; row += gridDim.x) {
        const u32 y = row % a.ny, z = row / a.ny;
        for (u32 x = threadIdx.x; x < a.nx; x += blockDim.x) {
            const u32 n = row * a.nx + x;
            std::uint8_t flag = 0;
            if constexpr (FLAGS) {
                flag = a.flags[n];
                if (flag & kFlagTypeMask) continue;
            }
            R fin[L::Q];
            gather<L, S, FLAGS>(a, n, make_nbr(a, x, y, z), flag, fin);
            R rho, ux, uy, uz, ax, ay, az;
            moments<L, R, S::delta>(fin, rho, ux, uy, uz);
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

static __global__ void __launch_bounds__(kReduceThreads) k_reduce_final(const double* partials, int blocks,
                                                                        double* out) {
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
__global__ void __launch_bounds__(128) k_prepare_flags(const __grid_constant__ LbmArgs a, const std::uint8_t* user,
                                                       std::uint8_t* out) {
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (x >= a.nx || y >= a.ny) return;
    const u32 n = (z * a.ny + y) * a.nx + x;
    const std::uint8_t t = user[n] & kFlagTypeMask;
    if (t != 0) {
        out[n] = t;
        return;
    }
    const Nbr o = make_nbr(a, x, y, z);
    std::uint8_t b = 0;
#pragma unroll
    for (int d = 1; d < L::Q; ++d) {
        const u32 m = n + o.ox[L::cx(d) + 1] + o.oy[L::cy(d) + 1] + o.oz[L::cz(d) + 1];
        const std::uint8_t u = user[m] & kFlagTypeMask;
        if (u != 0) b |= kFlagNearWall;
        if (u >= 2) b |= kFlagNearMoving;
    }
    out[n] = b;
}

} // namespace cfdx
