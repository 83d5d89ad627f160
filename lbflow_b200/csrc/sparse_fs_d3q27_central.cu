// Sparse-layout step kernels with explicit faces and the scalar: D3Q27, central moments.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE_SPARSE_FS(VS_D3Q27, COLL_CENTRAL)
}  // namespace lbf
