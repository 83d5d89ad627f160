// Kernel instantiations for D2Q9.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE(VS_D2Q9, 1)
}  // namespace lbf
