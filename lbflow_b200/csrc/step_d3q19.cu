// Kernel instantiations for D3Q19.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE(VS_D3Q19, 0)
}  // namespace lbf
