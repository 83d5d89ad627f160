// Step-kernel instantiations for D3Q27 with MRT collision.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE_COLL(VS_D3Q27, COLL_MRT)
}  // namespace lbf
