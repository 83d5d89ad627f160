// Step-kernel instantiations for D3Q27 with BGK collision.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE_COLL(VS_D3Q27, COLL_BGK)
}  // namespace lbf
