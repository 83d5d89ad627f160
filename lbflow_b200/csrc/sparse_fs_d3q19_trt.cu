// Sparse-layout step kernels with explicit faces and the scalar: D3Q19, TRT.
#include "dispatch.cuh"

namespace lbf {
LBF_INSTANTIATE_SPARSE_FS(VS_D3Q19, COLL_TRT)
}  // namespace lbf
