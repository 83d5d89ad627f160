// Step-kernel instantiations for D3Q27 with the central-moment collision.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE_COLL(VS_D3Q27, COLL_CENTRAL)
}  // namespace lbf
