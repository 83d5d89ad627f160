// Sparse-layout step kernels with explicit faces and the scalar: D2Q9, central moments.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE_SPARSE_FS(VS_D2Q9, COLL_CENTRAL)
}  // namespace lbf
