// Step-kernel instantiations for D3Q19 with TRT collision.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE_COLL(VS_D3Q19, COLL_TRT)
}  // namespace lbf
