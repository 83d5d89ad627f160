// Sparse-layout step kernels with explicit faces and the scalar: D2Q9, MRT.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE_SPARSE_FS(VS_D2Q9, COLL_MRT)
}  // namespace lbf
