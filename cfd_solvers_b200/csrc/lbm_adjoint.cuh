// Discrete adjoint of the gray-LBM step (sm_100a).
//
// Forward (logical form): x^t(n,i) = C(x^{t-1}(n - c_i))_i, or C(x^{t-1}(n))_{opp i}
// when n - c_i is a wall, with C the per-cell TRT/BGK + Guo collision followed
// by gray partial bounce-back C_i = (1 - n_s) f*_i + n_s x_{opp i} (Walsh,
// Burwinkle & Saar 2009).  Its adjoint runs backwards in time:
//   mu(m,k) = lambda^t(m + c_k, k)   (lambda^t(m, opp k) at a wall)
//   lambda^{t-1}(m,.) = [dC/dx at x^{t-1}(m,.)]^T mu(m,.)
//   dJ/dn_s(m) += mu . dC/dn_s,   dJ/dtau += mu . dC/dtau
//
// Storage.  Kept with its directions flipped, nu(n,i) = lambda(n, opp i), the
// adjoint streams exactly like the forward: nu is gathered by a pull along
// +c (gathered nu_in(m,k) = mu(m, opp k)) and written back by the same
// in-place Esoteric-Pull scatter, bounce-back links included.  So the adjoint
// lattice uses the forward's slot tables, at its own parity, and the
// kernels below reuse the forward's gather/scatter unchanged.
//
// Forward states.  The Jacobian and dC/dn_s need the full incoming
// populations of every step.  The forward keeps a checkpoint every k steps;
// the reverse sweep recomputes a segment out of place (k_step_oop: read one
// frame, write the next, so each frame stays readable), then walks it
// backwards.  A frame written by k_step_oop is gather-ready at the same
// parity as its source: the step gathers with the tables of parity P and
// scatters with those of parity P ^ 1, which is exactly the layout parity P
// reads (the slots a parity-P^1 gather would read).
//
// Jacobian of C at x (rho = sum x, u~ = j / rho, u = u~ + a/2, F = rho a):
//   dC_i/dx_k = (1 - n_s) [A_ik + dG_i/drho + dG_i/du . (c_k - u~) / rho] + n_s delta(opp i, k)
//   A_ik = delta_ik (1 - (w+ + w-)/2) - delta(opp i, k) (w+ - w-)/2
//   G_i  = w+ feq+_i + w- feq-_i + (1 - w+/2) F+_i + (1 - w-/2) F-_i
// G is linear in rho at fixed u, so with the moments of mu
//   m0 = sum w mu, m = sum w mu c, M = sum w mu c c^T
// the contractions are
//   P  = sum mu dG/drho = w+ (m0 (1 - 1.5 u^2) + 4.5 u.M.u) + 3 w- m.u + g+ (9 u.M.a - 3 m0 u.a) + 3 g- m.a
//   Vr = sum mu dG/du / rho = 9 M v - 3 m0 v + 3 w- m,   v = w+ u + g+ a
// and in opposite-pair space (sigma = mu_i + mu_j, delta = mu_i - mu_j):
//   lambda_i + lambda_j = (1 - n_s)(sigma (1 - w+) + 2 P - 2 Vr.u~) + n_s sigma
//   lambda_i - lambda_j = (1 - n_s)(delta (1 - w-) + 2 Vr.c_i)     - n_s delta
//   lambda_0            = (1 - n_s)(mu_0 (1 - w+) + P - Vr.u~)       + n_s mu_0
// Scope: BGK/TRT, uniform or per-cell force, gray n_s, stationary walls,
// periodic faces.  Smagorinsky LES (tau depends on the populations) and
// moving walls are rejected by the host.
#pragma once

#include "lbm_device.cuh"

namespace cfdx {

// Adjoint lattice storage: FP64 next to FP64 forward storage, FP32 otherwise.
template <class S> struct AdjointStorage {
    using type = StF32;
};
template <> struct AdjointStorage<StF64> {
    using type = StF64;
};

// Absolute populations from what gather_loads returns (deviations for FP16).
template <class L, class S, int D = 0>
__device__ __forceinline__ void to_absolute(typename S::R* f) {
    if constexpr (D < L::Q) {
        if constexpr (S::delta) f[D] += typename S::R(L::w(D));
        to_absolute<L, S, D + 1>(f);
    }
}

// Compile-time loop: f(std::integral_constant<int, k>) for k in [B, E).
template <int B, int E, class F> __device__ __forceinline__ void static_for(F&& f) {
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

template <class R> struct CellState {
    R rho, irho, utx, uty, utz, ux, uy, uz, ax, ay, az;
};

// x: absolute populations, or deviations f - w when DELTA.
template <class L, class R, bool DELTA = false>
__device__ __forceinline__ CellState<R> cell_state(const LbmArgs& a, u32 n, const R* x, bool force) {
    CellState<R> c;
    R r = x[0], jx = R(0), jy = R(0), jz = R(0);
    static_for<0, L::PAIRS>([&](auto P) {
        constexpr int i = 2 * decltype(P)::value + 1, j = i + 1;
        const R s = x[i] + x[j], d = x[i] - x[j];
        r += s;
        if constexpr (L::cx(i) > 0) jx += d;
        if constexpr (L::cx(i) < 0) jx -= d;
        if constexpr (L::cy(i) > 0) jy += d;
        if constexpr (L::cy(i) < 0) jy -= d;
        if constexpr (L::cz(i) > 0) jz += d;
        if constexpr (L::cz(i) < 0) jz -= d;
    });
    c.rho = DELTA ? r + R(1) : r;
    c.irho = rcp_unbiased(c.rho);
    c.utx = jx * c.irho;
    c.uty = jy * c.irho;
    c.utz = jz * c.irho;
    c.ax = c.ay = c.az = R(0);
    if (force) cell_acceleration<R>(a, n, c.ax, c.ay, c.az);
    c.ux = c.utx + R(0.5) * c.ax;
    c.uy = c.uty + R(0.5) * c.ay;
    c.uz = c.utz + R(0.5) * c.az;
    return c;
}

// One cell of the adjoint step: nin are the gathered adjoint values
// (nin_k = mu_{opp k}), x the forward's incoming populations (absolute, or
// the deviations f - w when DELTA: FP16-shifted frames, whose deviations are
// what the loads decode and which keep the non-equilibrium differences below
// free of the weights' cancellation).  Writes the flipped result nout
// (nout_i = lambda_{opp i}) and this cell's dJ/dn_s and dJ/dtau contributions.
template <class L, class R, bool DELTA>
__device__ __forceinline__ void adjoint_cell(const LbmArgs& a, u32 n, const R* x, const R* nin, R* nout, bool force,
                                             R dwp, R dwm, double& g_ns, double& g_tau) {
    const CellState<R> c = cell_state<L, R, DELTA>(a, n, x, force);
    const R tau = p_tau<R>(a);
    const R wp = rcp(tau);
    const R wm = omega_minus_of<R>(a, tau, wp);
    const R gp = R(1) - R(0.5) * wp, gm = R(1) - R(0.5) * wm;
    const R ns = a.ns ? R(a.ns[n]) : R(0);
    const R ux = c.ux, uy = c.uy, uz = c.uz;
    const R Fx = c.rho * c.ax, Fy = c.rho * c.ay, Fz = c.rho * c.az;
    const R base = R(1) - R(1.5) * (ux * ux + uy * uy + uz * uz);
    const R uF = ux * Fx + uy * Fy + uz * Fz;

    // rest direction: forward pieces and adjoint moments
    constexpr R w0 = R(L::w(0));
    const R mu0 = nin[0];
    // x_0 - w0 rho base; with deviations x_0 - w0 (rho base - 1)
    const R neq0 = DELTA ? x[0] - w0 * (c.rho * base - R(1)) : x[0] - w0 * c.rho * base;
    const R F0 = -R(3) * w0 * uF;
    // Pair sums for dC/dn_s and dC/dtau: with s, d the pair sum and
    // difference of x and sneq = s - 2 w rho (base + 4.5 (c.u)^2),
    // dneq = d - 6 w rho c.u their non-equilibrium parts,
    //   SA = sum sigma sneq,  SB = sum delta dneq,  SD = sum delta d.
    // The pairs' Guo terms sF = 2 w (9 (c.u)(c.F) - 3 u.F), dF = 6 w c.F enter
    // only through sum sigma sF = 18 u.M.F - 6 u.F m0' and sum delta dF = 6 m.F,
    // with m0' = m0 - w0 mu0 the pairs' share of m0, so no per-pair force term.
    R SA = R(0), SB = R(0), SD = R(0);
    R m0p = R(0), mx = R(0), my = R(0), mz = R(0);
    R Mxx = R(0), Myy = R(0), Mzz = R(0), Mxy = R(0), Mxz = R(0), Myz = R(0);
    R ms[L::PAIRS], md[L::PAIRS];
    static_for<0, L::PAIRS>([&](auto PP) {
        constexpr int p = decltype(PP)::value;
        constexpr int i = 2 * p + 1, j = i + 1;
        constexpr int cx = L::cx(i), cy = L::cy(i), cz = L::cz(i);
        const R w = R(L::w(i));
        // mu_i = nin_j, mu_j = nin_i
        const R sg = nin[i] + nin[j];
        const R dl = nin[j] - nin[i];
        ms[p] = sg;
        md[p] = dl;
        const R ws = w * sg, wd = w * dl;
        m0p += ws;
        mx += signed_sum<cx, 0, 0>(wd, R(0), R(0));
        my += signed_sum<cy, 0, 0>(wd, R(0), R(0));
        mz += signed_sum<cz, 0, 0>(wd, R(0), R(0));
        if constexpr (cx != 0) Mxx += ws;
        if constexpr (cy != 0) Myy += ws;
        if constexpr (cz != 0) Mzz += ws;
        Mxy += signed_sum<cx * cy, 0, 0>(ws, R(0), R(0));
        Mxz += signed_sum<cx * cz, 0, 0>(ws, R(0), R(0));
        Myz += signed_sum<cy * cz, 0, 0>(ws, R(0), R(0));
        const R s = x[i] + x[j], d = x[i] - x[j];
        const R cu = cdot<L, i>(ux, uy, uz);
        const R t = base + R(4.5) * cu * cu;
        // s - 2 w rho t, with deviations s - 2 w (rho t - 1); d has no weight part
        const R sneq = DELTA ? s - (R(2) * w) * (c.rho * t - R(1)) : s - (R(2) * w * c.rho) * t;
        const R dneq = d - (R(6) * w * c.rho) * cu;
        SA += sg * sneq;
        SB += dl * dneq;
        SD += dl * d;
    });
    const R m0 = w0 * mu0 + m0p;
    const R ax = c.ax, ay = c.ay, az = c.az;
    const R Mux = Mxx * ux + Mxy * uy + Mxz * uz;
    const R Muy = Mxy * ux + Myy * uy + Myz * uz;
    const R Muz = Mxz * ux + Myz * uy + Mzz * uz;
    const R Max = Mxx * ax + Mxy * ay + Mxz * az;
    const R May = Mxy * ax + Myy * ay + Myz * az;
    const R Maz = Mxz * ax + Myz * ay + Mzz * az;
    // F = rho a: u.M.F = rho u.M.a, m.F = rho m.a
    const R uMa = ux * Max + uy * May + uz * Maz;
    const R ma = mx * ax + my * ay + mz * az;
    const R SF = R(18) * c.rho * uMa - R(6) * uF * m0p;
    const R DF = R(6) * c.rho * ma;
    // x_0 - C_0 = wp neq0 - gp F0, and per pair s - sst = wp sneq - gp sF,
    // d + dst = 2 d - wm dneq + gm dF
    const R gns = mu0 * (wp * neq0 - gp * F0) + R(0.5) * (wp * SA - gp * SF - R(2) * SD + wm * SB - gm * DF);
    const R gtp = mu0 * (-neq0 - R(0.5) * F0) - R(0.5) * SA - R(0.25) * SF;
    const R gtm = -R(0.5) * SB - R(0.25) * DF;
    g_ns = double(gns);
    g_tau = double((R(1) - ns) * (dwp * gtp + dwm * gtm));

    const R P = wp * (m0 * base + R(4.5) * (ux * Mux + uy * Muy + uz * Muz)) +
                R(3) * wm * (mx * ux + my * uy + mz * uz) +
                gp * (R(9) * uMa - R(3) * m0 * (ux * ax + uy * ay + uz * az)) + R(3) * gm * ma;
    const R vx = wp * ux + gp * ax, vy = wp * uy + gp * ay, vz = wp * uz + gp * az;
    const R Vx = R(9) * (wp * Mux + gp * Max) - R(3) * m0 * vx + R(3) * wm * mx;
    const R Vy = R(9) * (wp * Muy + gp * May) - R(3) * m0 * vy + R(3) * wm * my;
    const R Vz = R(9) * (wp * Muz + gp * Maz) - R(3) * m0 * vz + R(3) * wm * mz;
    const R Vu = Vx * c.utx + Vy * c.uty + Vz * c.utz;
    const R keep = R(1) - ns;
    nout[0] = keep * (mu0 * (R(1) - wp) + P - Vu) + ns * mu0;
    // Per pair, with ls = keep (sigma (1 - wp) + 2 (P - Vu)) + ns sigma and
    // ld = keep (delta (1 - wm) + 2 V.c_i) - ns delta: lambda_i = (ls + ld) / 2
    // is stored in slot j (flipped), lambda_j = (ls - ld) / 2 in slot i.  The
    // halves fold into per-cell coefficients.
    const R as = R(0.5) * (keep * (R(1) - wp) + ns), bs = keep * (P - Vu);
    const R ad = R(0.5) * (keep * (R(1) - wm) - ns);
    const R kVx = keep * Vx, kVy = keep * Vy, kVz = keep * Vz;
    static_for<0, L::PAIRS>([&](auto PP) {
        constexpr int p = decltype(PP)::value;
        constexpr int i = 2 * p + 1, j = i + 1;
        const R hs = ms[p] * as + bs;
        const R hd = md[p] * ad + cdot<L, i>(kVx, kVy, kVz);
        nout[i] = hs - hd;
        nout[j] = hs + hd;
    });
}

// Deterministic FP64 block sum of v added to partials[block] (every thread of
// the block must call it).
__device__ __forceinline__ void block_accumulate(double v, double* partials) {
    __shared__ double warp_sum[32];
    const unsigned tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const unsigned nthreads = blockDim.x * blockDim.y * blockDim.z;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffU, v, off);
    if ((tid & 31U) == 0U) warp_sum[tid >> 5] = v;
    __syncthreads();
    if (tid == 0U) {
        double s = 0.0;
        for (unsigned w = 0; w < (nthreads + 31U) / 32U; ++w) s += warp_sum[w];
        const unsigned b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        partials[b] += s;
    }
}

// Out-of-place forward step for the segment recompute: gather from f (parity
// P tables, source frame), collide exactly as k_step does, scatter through s
// (parity P ^ 1 tables, destination frame).
// Resident blocks per SM of the out-of-place recompute step.  It carries two
// argument blocks, and at the one-cell step's cap for D3Q19 (12 blocks, 40
// registers) its forms spilled up to 152 bytes.  Measured on B200, 128^3 FP32
// gray TRT channel, reverse sweep per step: 12 blocks 191 us, 10 blocks (48
// registers) 172 us, 8 blocks (64 registers) 173 us.
#ifndef CFDX_OOP_MIN_BLOCKS_Q19
#define CFDX_OOP_MIN_BLOCKS_Q19 10
#endif
template <class L, class S, bool GRAY> constexpr int oop_min_blocks() {
    return L::Q == 19 && sizeof(typename S::T) != 8 ? CFDX_OOP_MIN_BLOCKS_Q19 : step_min_blocks<L, S, GRAY>();
}

template <class L, class S, bool FLAGS, bool GRAY>
__global__ void __launch_bounds__(128, oop_min_blocks<L, S, GRAY>()) k_step_oop(const __grid_constant__ LbmArgs f,
                                                                          const __grid_constant__ LbmArgs s) {
    using R = typename S::R;
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (x >= f.nx || y >= f.ny) return;
    const u32 n = (z * f.ny + y) * f.nx + x;
    std::uint8_t flag = 0;
    if constexpr (FLAGS) {
        flag = f.flags[n];
        if (flag & kFlagTypeMask) return;
    }
    const Nbr o = make_nbr(f, x, y, z);
    R fin[L::Q];
    gather_loads<L, S, FLAGS, true, S::scaled>(f, n, o, flag, fin);
    if constexpr (S::scaled) {
        if (f.has_force)
            collide_scaled<L, false, GRAY, true>(f, n, fin);
        else
            collide_scaled<L, false, GRAY, false>(f, n, fin);
    } else {
        if (f.has_force)
            collide<L, R, false, GRAY, true, S::delta>(f, n, fin);
        else
            collide<L, R, false, GRAY, false, S::delta>(f, n, fin);
    }
    // rounding bits of the forward's step at this time (seed in f)
    scatter<L, S, true, S::scaled>(s, n, o, fin, sizeof(typename S::T) == 2 ? round_hash(f, n) : 0U);
}

// lambda^T from dJ/d(rho, u) of the state the forward left: for every fluid
// cell, lambda_k = g_rho + g_u . (c_k - u~) / rho (u = u~ + a/2 is what the
// macroscopic output reports), scattered flipped into the adjoint lattice
// through A.l (parity 1 tables, so the first adjoint step gathers at parity 0).
template <class L, class S, bool FLAGS>
__global__ void __launch_bounds__(128) k_adjoint_seed(const __grid_constant__ AdjointArgs A) {
    using R = typename S::R;
    using LS = typename AdjointStorage<S>::type;
    const LbmArgs& f = A.f;
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    if (x >= f.nx || y >= f.ny) return;
    const u32 n = (z * f.ny + y) * f.nx + x;
    std::uint8_t flag = 0;
    if constexpr (FLAGS) {
        flag = f.flags[n];
        if (flag & kFlagTypeMask) return;
    }
    const Nbr o = make_nbr(f, x, y, z);
    R xin[L::Q];
    gather_loads<L, S, FLAGS, true, false>(f, n, o, flag, xin);
    to_absolute<L, S>(xin);
    const CellState<R> c = cell_state<L, R>(f, n, xin, false);
    const R gr = A.g_rho ? R(A.g_rho[n]) : R(0);
    const R gx = R(A.g_ux[n]) * c.irho, gy = R(A.g_uy[n]) * c.irho, gz = R(A.g_uz[n]) * c.irho;
    const R g0 = gr - (gx * c.utx + gy * c.uty + gz * c.utz);
    R nout[L::Q];
    nout[0] = g0;
    static_for<0, L::PAIRS>([&](auto PP) {
        constexpr int i = 2 * decltype(PP)::value + 1, j = i + 1;
        const R cg = cdot<L, i>(gx, gy, gz);
        nout[i] = g0 - cg; // lambda_j, stored flipped in slot i
        nout[j] = g0 + cg; // lambda_i
    });
    scatter<L, LS, true, false>(A.l, n, o, nout, 0U);
}

// One reverse step: gather the adjoint (A.l, in place at its parity) and the
// forward's incoming populations of the matching forward step (A.f, a frame),
// apply the transposed collision, scatter the adjoint back, accumulate the
// gradients.
// Resident blocks per SM the reverse step is compiled for (register cap
// 65536 / (128 * blocks)).  Measured on B200 (adjoint step alone): D3Q19 at 8
// blocks (64 registers) 0.098 ms vs 0.125 uncapped at 128^3 FP32 (reverse sweep
// per step 173.4 us, against 174.0 at 7 blocks and 183.8 at 6, which spill less;
// with the moment form of the gradient terms 160.5 us at 8, 164.9 at 7, 175.4 at 6);
// D3Q27 FP16 at 256^3, reverse sweep per step: 1597 us at 6 blocks (80 registers,
// no spill once the gradient terms came from the moments), 1654 at 5, 1670 at 7.
#ifndef CFDX_ADJOINT_MIN_BLOCKS_Q19
#define CFDX_ADJOINT_MIN_BLOCKS_Q19 8
#endif
#ifndef CFDX_ADJOINT_MIN_BLOCKS_Q27
#define CFDX_ADJOINT_MIN_BLOCKS_Q27 6
#endif
template <class L, class S> constexpr int adjoint_min_blocks() {
    return sizeof(typename S::T) == 8 ? 1 : (L::Q == 19 ? CFDX_ADJOINT_MIN_BLOCKS_Q19 : CFDX_ADJOINT_MIN_BLOCKS_Q27);
}

template <class L, class S, bool FLAGS>
__global__ void __launch_bounds__(128, adjoint_min_blocks<L, S>()) k_adjoint_step(const __grid_constant__ AdjointArgs A) {
    using R = typename S::R;
    using LS = typename AdjointStorage<S>::type;
    const LbmArgs& f = A.f;
    const u32 x = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 y = blockIdx.y * blockDim.y + threadIdx.y;
    const u32 z = blockIdx.z;
    double g_tau = 0.0;
    if (x < f.nx && y < f.ny) {
        const u32 n = (z * f.ny + y) * f.nx + x;
        std::uint8_t flag = 0;
        bool fluid = true;
        if constexpr (FLAGS) {
            flag = f.flags[n];
            fluid = (flag & kFlagTypeMask) == 0;
        }
        if (fluid) {
            const Nbr o = make_nbr(f, x, y, z);
            R xin[L::Q], nin[L::Q], nout[L::Q];
            gather_loads<L, S, FLAGS, true, false>(f, n, o, flag, xin);
            gather_loads<L, LS, FLAGS, true, false>(A.l, n, o, flag, nin);
            double g_ns = 0.0;
            adjoint_cell<L, R, S::delta>(f, n, xin, nin, nout, f.has_force != 0, R(A.dwp), R(A.dwm), g_ns, g_tau);
            scatter<L, LS, true, false>(A.l, n, o, nout, 0U);
            A.grad_ns[n] += g_ns;
        }
    }
    block_accumulate(g_tau, A.tau_partials);
}

// Sum of `count` FP64 partials in a fixed order (one block).
static __global__ void __launch_bounds__(256) k_sum_partials(const double* partials, std::size_t count, double* out) {
    __shared__ double part[256];
    double s = 0.0;
    for (std::size_t i = threadIdx.x; i < count; i += blockDim.x) s += partials[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (unsigned w = blockDim.x / 2U; w > 0U; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0U) *out = part[0];
}

} // namespace cfdx
