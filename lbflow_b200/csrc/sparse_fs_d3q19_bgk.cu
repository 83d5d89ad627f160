// Sparse-layout step kernels with explicit faces and the scalar: D3Q19, BGK.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE_SPARSE_FS(VS_D3Q19, COLL_BGK)
}  // namespace lbf
