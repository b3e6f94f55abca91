// Template dispatch from a runtime KernelKey to the kernel instantiations of
// one storage type.  Included by lbm_kernels_{f32,f16s,f64}.cu only.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <type_traits>

#include "lbm_adjoint.cuh"
#include "lbm_device.cuh"
#include "lbm_launch.h"
#include "lbm_step_h2.cuh"
#include "lbm_step_w2.cuh"
#include "lbm_step_x2.cuh"

namespace cfdx {

template <int STORAGE> struct StorageOf;
template <> struct StorageOf<kStoreF32> {
    using type = StF32;
};
template <> struct StorageOf<kStoreF64> {
    using type = StF64;
};
template <> struct StorageOf<kStoreF16S> {
    using type = StF16;
};

template <class F> cudaError_t with_lattice(int q, F&& f) {
    if (q == 19) return f(D3Q19{});
    if (q == 27) return f(D3Q27{});
    return cudaErrorInvalidValue;
}

// One-cell step kernel; NARROW (32-bit slot offsets) whenever q*N < 2^32.
template <class L, class S, bool LES, bool FL, bool GR>
cudaError_t step_single(bool narrow, const LbmArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    if (narrow)
        k_step<L, S, LES, FL, GR, 1, true><<<g, b, 0, s>>>(a);
    else
        k_step<L, S, LES, FL, GR, 1, false><<<g, b, 0, s>>>(a);
    return cudaGetLastError();
}

// Paired-cell kernels: a thread owns x0 = 2t and x0 + 1 (FP16: k_step_h2,
// packed f32x2 collision; FP32: k_step_x2).
template <class L, class S, bool LES, bool FL, bool GR>
cudaError_t step_paired(const LbmArgs& a, dim3 b, cudaStream_t s) {
    if constexpr (sizeof(typename S::T) == 8) {
        return cudaErrorInvalidValue;
    } else {
        const unsigned pairs = (a.nx + 1U) / 2U;
        dim3 g((pairs + b.x - 1U) / b.x, (a.ny + b.y - 1U) / b.y, a.z_end - a.z_first);
        if constexpr (sizeof(typename S::T) == 2) {
            // interior pairs two cells per thread, then the pairs with walls one cell per thread
            k_step_h2<L, LES, FL, GR><<<g, b, 0, s>>>(a);
            if constexpr (FL) {
                if (a.near_count > 0U) {
                    const cudaError_t e = cudaGetLastError();
                    if (e != cudaSuccess) return e;
                    k_step_list<L, S, LES, GR><<<(a.near_count + 127U) / 128U, 128, 0, s>>>(a);
                }
            }
        } else {
            k_step_x2<L, S, LES, FL, GR><<<g, b, 0, s>>>(a);
        }
        return cudaGetLastError();
    }
}

// Wall-aware z-marching pair kernel (FP16 storage): grid over pairs, rows and
// chunks of a.planes planes; the pipelined form stages two planes of words
// per thread in shared memory.  Its dynamic shared-memory limit (above 48 KB a
// kernel must opt in: D3Q27's stages) and its carveout (so that the blocks
// its register cap allows fit on an SM) are set once per kernel and device:
// function attributes belong to the device's context.
template <class K>
cudaError_t w2_attributes(K kernel, unsigned smem_bytes, int blocks, std::atomic<std::uint64_t>& devices_done) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    const std::uint64_t bit = device < 64 ? (1ULL << device) : 0ULL;
    if (bit != 0ULL && (devices_done.load() & bit) != 0ULL) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem_bytes));
    if (e != cudaSuccess) return e;
    const unsigned need = (smem_bytes + 1024U) * static_cast<unsigned>(blocks); // + per-block reservation
    const int pct = static_cast<int>(std::min(100U, (need * 100U + 228U * 1024U - 1U) / (228U * 1024U)));
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    if (e == cudaSuccess) devices_done.fetch_or(bit);
    return e;
}

template <class L, class S, bool LES, bool FL, bool GR>
cudaError_t step_w2(const KernelKey& k, const LbmArgs& a, dim3 b, cudaStream_t s) {
    if constexpr (sizeof(typename S::T) != 2) {
        return cudaErrorInvalidValue;
    } else {
        if (b.x * b.y != kW2Threads || b.z != 1U) return cudaErrorInvalidValue;
        const unsigned pairs = a.nx / 2U;
        const unsigned planes = a.planes == 0U ? 1U : a.planes;
        const unsigned span = a.z_end - a.z_first;
        dim3 g((pairs + b.x - 1U) / b.x, (a.ny + b.y - 1U) / b.y, (span + planes - 1U) / planes);
        if (k.w2_pipe) {
            static std::atomic<std::uint64_t> devices_done{0}; // one per kernel instantiation
            const cudaError_t e = w2_attributes(k_step_w2<L, LES, FL, GR, true>, w2_smem_bytes<L>(),
                                                w2_min_blocks<L>(), devices_done);
            if (e != cudaSuccess) return e;
            k_step_w2<L, LES, FL, GR, true><<<g, b, w2_smem_bytes<L>(), s>>>(a);
        } else {
            k_step_w2<L, LES, FL, GR, false><<<g, b, 0, s>>>(a);
        }
        return cudaGetLastError();
    }
}

template <class L, class S, bool LES, bool FL>
cudaError_t step_gray(const KernelKey& k, const LbmArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    if (k.w2) return k.gray ? step_w2<L, S, LES, FL, true>(k, a, b, s) : step_w2<L, S, LES, FL, false>(k, a, b, s);
    if (k.paired)
        return k.gray ? step_paired<L, S, LES, FL, true>(a, b, s) : step_paired<L, S, LES, FL, false>(a, b, s);
    return k.gray ? step_single<L, S, LES, FL, true>(k.narrow, a, g, b, s)
                  : step_single<L, S, LES, FL, false>(k.narrow, a, g, b, s);
}

template <class L, class S, bool LES>
cudaError_t step_flags(const KernelKey& k, const LbmArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    return k.flags ? step_gray<L, S, LES, true>(k, a, g, b, s) : step_gray<L, S, LES, false>(k, a, g, b, s);
}

// The collision operator (BGK or TRT) is a runtime parameter of the kernel
// (LbmArgs::omega_minus); the template axes are lattice, storage, LES,
// flags, gray and cells per thread.
template <int STORAGE>
cudaError_t Launcher<STORAGE>::step(const KernelKey& k, const LbmArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    using S = typename StorageOf<STORAGE>::type;
    return with_lattice(k.q, [&](auto lat) {
        using L = decltype(lat);
        return k.les ? step_flags<L, S, true>(k, a, g, b, s) : step_flags<L, S, false>(k, a, g, b, s);
    });
}

template <int STORAGE>
cudaError_t Launcher<STORAGE>::init(const KernelKey& k, const LbmArgs& a, const InitSpec& spec, dim3 g, dim3 b,
                                    cudaStream_t s) {
    using S = typename StorageOf<STORAGE>::type;
    return with_lattice(k.q, [&](auto lat) {
        using L = decltype(lat);
        if (k.flags)
            k_init<L, S, true><<<g, b, 0, s>>>(a, spec);
        else
            k_init<L, S, false><<<g, b, 0, s>>>(a, spec);
        return cudaGetLastError();
    });
}

template <int STORAGE>
cudaError_t Launcher<STORAGE>::macro(const KernelKey& k, const LbmArgs& a, void* rho, void* ux, void* uy, void* uz,
                                     bool out_f64, dim3 g, dim3 b, cudaStream_t s) {
    using S = typename StorageOf<STORAGE>::type;
    return with_lattice(k.q, [&](auto lat) {
        using L = decltype(lat);
        // 32-bit slot offsets (as the step) whenever q * cells < 2^32
        const auto run = [&](auto* r, auto* x, auto* y, auto* z) {
            using O = std::remove_pointer_t<decltype(r)>;
            if (k.narrow) {
                if (k.flags)
                    k_macro<L, S, true, O, true><<<g, b, 0, s>>>(a, r, x, y, z);
                else
                    k_macro<L, S, false, O, true><<<g, b, 0, s>>>(a, r, x, y, z);
            } else {
                if (k.flags)
                    k_macro<L, S, true, O, false><<<g, b, 0, s>>>(a, r, x, y, z);
                else
                    k_macro<L, S, false, O, false><<<g, b, 0, s>>>(a, r, x, y, z);
            }
        };
        if (out_f64)
            run(static_cast<double*>(rho), static_cast<double*>(ux), static_cast<double*>(uy),
                static_cast<double*>(uz));
        else
            run(static_cast<float*>(rho), static_cast<float*>(ux), static_cast<float*>(uy), static_cast<float*>(uz));
        return cudaGetLastError();
    });
}

template <int STORAGE>
cudaError_t Launcher<STORAGE>::logical(const KernelKey& k, const LbmArgs& a, float* out, dim3 g, dim3 b,
                                       cudaStream_t s) {
    using S = typename StorageOf<STORAGE>::type;
    return with_lattice(k.q, [&](auto lat) {
        using L = decltype(lat);
        if (k.flags)
            k_logical<L, S, true, float><<<g, b, 0, s>>>(a, out);
        else
            k_logical<L, S, false, float><<<g, b, 0, s>>>(a, out);
        return cudaGetLastError();
    });
}

template <int STORAGE>
cudaError_t Launcher<STORAGE>::reduce(const KernelKey& k, const LbmArgs& a, double* partials, int blocks, double* out,
                                      cudaStream_t s) {
    using S = typename StorageOf<STORAGE>::type;
    return with_lattice(k.q, [&](auto lat) {
        using L = decltype(lat);
        if (k.flags)
            k_reduce<L, S, true><<<blocks, kReduceThreads, 0, s>>>(a, partials);
        else
            k_reduce<L, S, false><<<blocks, kReduceThreads, 0, s>>>(a, partials);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        k_reduce_final<<<1, kReduceThreads, 0, s>>>(partials, blocks, out);
        return cudaGetLastError();
    });
}

template <int STORAGE>
cudaError_t Launcher<STORAGE>::step_oop(const KernelKey& k, const LbmArgs& src, const LbmArgs& dst, dim3 g, dim3 b,
                                        cudaStream_t s) {
    using S = typename StorageOf<STORAGE>::type;
    return with_lattice(k.q, [&](auto lat) {
        using L = decltype(lat);
        if (k.flags)
            k.gray ? k_step_oop<L, S, true, true><<<g, b, 0, s>>>(src, dst)
                   : k_step_oop<L, S, true, false><<<g, b, 0, s>>>(src, dst);
        else
            k.gray ? k_step_oop<L, S, false, true><<<g, b, 0, s>>>(src, dst)
                   : k_step_oop<L, S, false, false><<<g, b, 0, s>>>(src, dst);
        return cudaGetLastError();
    });
}

template <int STORAGE>
cudaError_t Launcher<STORAGE>::adjoint_seed(const KernelKey& k, const AdjointArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    using S = typename StorageOf<STORAGE>::type;
    return with_lattice(k.q, [&](auto lat) {
        using L = decltype(lat);
        if (k.flags)
            k_adjoint_seed<L, S, true><<<g, b, 0, s>>>(a);
        else
            k_adjoint_seed<L, S, false><<<g, b, 0, s>>>(a);
        return cudaGetLastError();
    });
}

template <int STORAGE>
cudaError_t Launcher<STORAGE>::adjoint_step(const KernelKey& k, const AdjointArgs& a, dim3 g, dim3 b, cudaStream_t s) {
    using S = typename StorageOf<STORAGE>::type;
    return with_lattice(k.q, [&](auto lat) {
        using L = decltype(lat);
        if (k.flags)
            k_adjoint_step<L, S, true><<<g, b, 0, s>>>(a);
        else
            k_adjoint_step<L, S, false><<<g, b, 0, s>>>(a);
        return cudaGetLastError();
    });
}

template <int STORAGE>
cudaError_t Launcher<STORAGE>::slot_io(const KernelKey& k, const LbmArgs& a, int d, float* buf, bool in, dim3 g,
                                       dim3 b, cudaStream_t s) {
    using S = typename StorageOf<STORAGE>::type;
    return with_lattice(k.q, [&](auto lat) {
        using L = decltype(lat);
        if (in) {
            if (k.flags)
                k_slot_in<L, S, true><<<g, b, 0, s>>>(a, d, buf);
            else
                k_slot_in<L, S, false><<<g, b, 0, s>>>(a, d, buf);
        } else {
            if (k.flags)
                k_slot_out<L, S, true><<<g, b, 0, s>>>(a, d, buf);
            else
                k_slot_out<L, S, false><<<g, b, 0, s>>>(a, d, buf);
        }
        return cudaGetLastError();
    });
}

} // namespace cfdx
