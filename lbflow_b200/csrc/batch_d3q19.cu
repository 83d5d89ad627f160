// Batched-sweep instantiations for D3Q19.
#include "batch_kernels.cuh"

namespace lbf {
LBF_INSTANTIATE_BATCH(VS_D3Q19)
}  // namespace lbf
