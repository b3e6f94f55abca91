// cfdx_lbm_reduce_noalloc: the FP64 fluid-cell reduction without any
// allocation.
//
// cfdx_lbm_reduce() allocates its per-block partial sums (and a pinned host
// buffer) the first time it runs on a handle.  Some callers cannot allow that
// allocation: a process whose device memory is already held by another
// allocator (a framework's caching allocator or a pool sized to the whole
// GPU), where a fresh cudaMalloc fails or forces memory to be released;
// monitoring loops that must not pay the device-wide synchronisation that
// cudaMalloc and cudaFree imply; and foreign-language callers (ctypes, cgo)
// that have no CUDA allocation API of their own with which to hand the
// library a scratch buffer.  This entry point keeps its scratch in a fixed
// file-scope device array instead, so it calls no cudaMalloc, cudaFree or
// other allocating routine; the caller passes the lattice (a handle created
// beforehand) and a host output buffer of CFDX_REDUCE_COUNT doubles.
//
// Scratch: the reduction runs min(ny*nz, 4096) blocks over the ny*nz x-rows
// (block b sums rows b, b + blocks, ...), each writing its 7 partial sums; a
// final block combines them in a fixed order and writes the 7 results.  The
// array holds the partials of those at most 4096 blocks plus the results, so
// any lattice size is accepted.  Every GPU that loads this library holds the
// array (229,432 bytes) until the process exits.
#include "cfdx_lbm.h"

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "handle_access.h"
#include "lbm_device.cuh"

namespace {

using namespace cfdx;

constexpr unsigned kMaxBlocks = 4096;
constexpr int kMaxDevices = 64;
constexpr std::size_t kScratchDoubles = (static_cast<std::size_t>(kMaxBlocks) + 1U) * kReduceFields;

// Partial sums of up to kMaxBlocks blocks followed by the 7 final values.
static __device__ __align__(256) double g_reduce_scratch[kScratchDoubles];

std::mutex g_setup_mutex;
void* g_scratch_address[kMaxDevices] = {};

// Device address of g_reduce_scratch on `device`, which must be current.  In
// host code the array's name is only a host-side stand-in; the address comes
// from cudaGetSymbolAddress, once per device, on the first call there.  The
// cached address belongs to the device's primary context as it was then: a
// process that resets the device (cudaDeviceReset) must not call this entry
// point again afterwards.
int scratch_address(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) return record_error(CFDX_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_address[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_reduce_scratch);
        if (e != cudaSuccess) {
            const std::string m = std::string("cudaGetSymbolAddress (reduction scratch): ") + cudaGetErrorString(e);
            return record_error(CFDX_ERR_CUDA, m.c_str());
        }
        g_scratch_address[device] = p;
    }
    *out = static_cast<double*>(g_scratch_address[device]);
    return CFDX_OK;
}

template <class S, class L>
cudaError_t launch(const ReduceView& v, double* partials, unsigned blocks, double* result) {
    if (v.key.flags)
        k_reduce<L, S, true><<<blocks, kReduceThreads, 0, v.stream>>>(v.args, partials);
    else
        k_reduce<L, S, false><<<blocks, kReduceThreads, 0, v.stream>>>(v.args, partials);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_reduce_final<<<1, kReduceThreads, 0, v.stream>>>(partials, static_cast<int>(blocks), result);
    return cudaGetLastError();
}

template <class S> cudaError_t launch_storage(const ReduceView& v, double* partials, unsigned blocks, double* result) {
    if (v.key.q == 19) return launch<S, D3Q19>(v, partials, blocks, result);
    if (v.key.q == 27) return launch<S, D3Q27>(v, partials, blocks, result);
    return cudaErrorInvalidValue;
}

} // namespace

extern "C" CFDX_API int cfdx_lbm_reduce_noalloc(cfdx_lbm* lbm, double* out) {
    ReduceView v{};
    int rc = handle_reduce_view(lbm, &v);
    if (rc != CFDX_OK) return rc;
    if (!out) return record_error(CFDX_ERR_INVALID, "null output buffer");
    // a fixed block count for every lattice shape, so thin lattices reduce on many SMs
    const unsigned long long rows = static_cast<unsigned long long>(v.args.ny) * v.args.nz;
    const unsigned blocks = static_cast<unsigned>(rows < kMaxBlocks ? rows : kMaxBlocks);
    double* scratch = nullptr;
    rc = scratch_address(v.device, &scratch);
    if (rc != CFDX_OK) return rc;
    double* result = scratch + static_cast<std::size_t>(kMaxBlocks) * kReduceFields;
    // Every block writes all of its partial slots and the final block writes
    // every result slot, so nothing left by an earlier call is read.
    cudaError_t e;
    switch (v.key.storage) {
    case kStoreF32: e = launch_storage<StF32>(v, scratch, blocks, result); break;
    case kStoreF64: e = launch_storage<StF64>(v, scratch, blocks, result); break;
    case kStoreF16S: e = launch_storage<StF16>(v, scratch, blocks, result); break;
    default: e = cudaErrorInvalidValue; break;
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, result, sizeof(double) * kReduceFields, cudaMemcpyDeviceToHost, v.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(v.stream);
    if (e != cudaSuccess) {
        const std::string m = std::string("cfdx_lbm_reduce_noalloc: ") + cudaGetErrorString(e);
        return record_error(CFDX_ERR_CUDA, m.c_str());
    }
    record_download(lbm, sizeof(double) * kReduceFields);
    out[CFDX_REDUCE_KINETIC_ENERGY] *= 0.5;
    if (out[CFDX_REDUCE_NONFINITE] > 0.0)
        return record_error(CFDX_ERR_NONFINITE, "non-finite populations in fluid cells");
    return CFDX_OK;
}
