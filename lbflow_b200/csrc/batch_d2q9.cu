// Batched-sweep instantiations for D2Q9.
#include "batch_kernels.cuh"

namespace lbf {
LBF_INSTANTIATE_BATCH(VS_D2Q9)
}  // namespace lbf
