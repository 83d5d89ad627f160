// Kernel instantiations for D3Q27.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE(VS_D3Q27, 1)
}  // namespace lbf
