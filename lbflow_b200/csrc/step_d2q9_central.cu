// Step-kernel instantiations for D2Q9 with the central-moment collision.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE_COLL(VS_D2Q9, COLL_CENTRAL)
}  // namespace lbf
