// Batched-sweep instantiations for D3Q27.
#include "batch_kernels.cuh"

namespace lbf {
LBF_INSTANTIATE_BATCH(VS_D3Q27)
}  // namespace lbf
