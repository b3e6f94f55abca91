// Copy kernel of the z-slab halo messages (halo.h): pack (lattice plane runs
// -> message buffer), unpack (buffer -> plane runs) and the direct cut
// exchange between two slabs of one process (plane runs -> plane runs, one
// launch for both directions).  HBM-bound: each chunk is one contiguous run,
// copied in the widest unit that every address and the chunk size allow.
#include "halo.h"

#include <algorithm>
#include <cstdint>

namespace cfdx {
namespace {

template <class U>
__global__ void __launch_bounds__(256) k_halo_copy(const __grid_constant__ HaloCopy c, std::uint32_t units) {
    const int k = static_cast<int>(blockIdx.y);
    const U* src = static_cast<const U*>(c.src[k]);
    U* dst = static_cast<U*>(c.dst[k]);
    const std::uint32_t stride = gridDim.x * blockDim.x;
    for (std::uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < units; e += stride) dst[e] = src[e];
}

template <class U> cudaError_t launch_as(const HaloCopy& c, std::size_t chunk_bytes, cudaStream_t s) {
    const std::size_t units = chunk_bytes / sizeof(U);
    // ~4 CTAs of 256 threads per SM over the whole copy (148 SMs)
    const std::size_t want = (units + 255) / 256;
    const std::size_t cap = std::max<std::size_t>(1, 592 / static_cast<std::size_t>(c.chunks));
    const dim3 grid(static_cast<unsigned>(std::min(want, cap)), static_cast<unsigned>(c.chunks), 1U);
    k_halo_copy<U><<<grid, 256, 0, s>>>(c, static_cast<std::uint32_t>(units));
    return cudaGetLastError();
}

} // namespace

cudaError_t launch_halo_copy(const HaloCopy& c, std::size_t chunk_bytes, cudaStream_t s) {
    if (c.chunks <= 0 || c.chunks > 2 * kMaxHaloChunks || chunk_bytes == 0 || chunk_bytes / 2 > 0xffffffffULL)
        return cudaErrorInvalidValue;
    std::uintptr_t bits = static_cast<std::uintptr_t>(chunk_bytes);
    for (int k = 0; k < c.chunks; ++k) {
        if (c.src[k] == nullptr || c.dst[k] == nullptr) return cudaErrorInvalidValue;
        bits |= reinterpret_cast<std::uintptr_t>(c.src[k]) | reinterpret_cast<std::uintptr_t>(c.dst[k]);
    }
    if ((bits & 15U) == 0U && chunk_bytes / 16 <= 0xffffffffULL) return launch_as<uint4>(c, chunk_bytes, s);
    if ((bits & 7U) == 0U && chunk_bytes / 8 <= 0xffffffffULL) return launch_as<uint2>(c, chunk_bytes, s);
    if ((bits & 3U) == 0U && chunk_bytes / 4 <= 0xffffffffULL) return launch_as<std::uint32_t>(c, chunk_bytes, s);
    if ((bits & 1U) == 0U) return launch_as<std::uint16_t>(c, chunk_bytes, s);
    return cudaErrorInvalidValue;
}

} // namespace cfdx
