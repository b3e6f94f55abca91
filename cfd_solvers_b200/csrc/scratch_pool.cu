// Temporary buffers of single calls come from a memory pool the library keeps
// per device (stream-ordered cudaMallocFromPoolAsync / cudaFreeAsync).  With
// cudaMalloc / cudaFree per call, every call mapped its memory anew and every
// cudaFree synchronised the whole device; repeated calls -- a body
// re-voxelized every few steps, a Q-criterion written every output frame --
// now reuse mapped memory.  The pool keeps up to kScratchKeep bytes between
// calls; cfdx_release_scratch hands them back.
#include "scratch_pool.h"

#include <algorithm>
#include <mutex>

namespace cfdx {
namespace {

constexpr int kMaxDevices = 64;
std::mutex g_guard;
cudaMemPool_t g_pools[kMaxDevices] = {};

cudaError_t pool_of(int device, cudaMemPool_t* pool, bool create) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    const std::lock_guard<std::mutex> lock(g_guard);
    if (!g_pools[device] && create) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t created = nullptr;
        cudaError_t e = cudaMemPoolCreate(&created, &props);
        if (e != cudaSuccess) return e;
        std::uint64_t keep = kScratchKeep;
        e = cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(created);
            return e;
        }
        g_pools[device] = created;
    }
    *pool = g_pools[device];
    return cudaSuccess;
}

} // namespace

cudaError_t scratch_pool(cudaMemPool_t* pool) {
    int device = 0;
    const cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    return pool_of(device, pool, true);
}

cudaError_t scratch_alloc(void** p, std::size_t bytes, cudaStream_t s) {
    cudaMemPool_t pool = nullptr;
    const cudaError_t e = scratch_pool(&pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(p, std::max<std::size_t>(bytes, 16), pool, s);
}

void scratch_free(void* p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

cudaError_t scratch_release(int device) {
    cudaMemPool_t pool = nullptr;
    const cudaError_t e = pool_of(device, &pool, false);
    if (e != cudaSuccess || !pool) return e;
    return cudaMemPoolTrimTo(pool, 0);
}

} // namespace cfdx
