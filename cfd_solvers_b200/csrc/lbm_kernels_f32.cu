// Kernel instantiations for one population storage type (compiled separately
// to keep build times parallel).
#include "lbm_launch_impl.cuh"

namespace cfdx {
template struct Launcher<kStoreF32>;
} // namespace cfdx

namespace cfdx {

// The FP64 partial-sum kernel of the adjoint does not depend on the storage type.
cudaError_t launch_sum_partials(const double* partials, std::size_t count, double* out, cudaStream_t s) {
    k_sum_partials<<<1, 256, 0, s>>>(partials, count, out);
    return cudaGetLastError();
}

// Flag preparation does not depend on the storage type; it lives here once.
cudaError_t launch_prepare_flags(int q, const LbmArgs& a, const std::uint8_t* user, std::uint8_t* out,
                                 std::uint32_t* mask, bool ghost, dim3 g, dim3 b, cudaStream_t s) {
    if (q == 19)
        k_prepare_flags<D3Q19><<<g, b, 0, s>>>(a, user, out, mask, ghost ? 1 : 0);
    else if (q == 27)
        k_prepare_flags<D3Q27><<<g, b, 0, s>>>(a, user, out, mask, ghost ? 1 : 0);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

} // namespace cfdx
