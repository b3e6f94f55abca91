// Kernel instantiations for one population storage type (compiled separately
// to keep build times parallel).
#include "lbm_launch_impl.cuh"

namespace cfdx {
template struct Launcher<kStoreF16S>;
} // namespace cfdx
