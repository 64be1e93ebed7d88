// Instantiations of the fused 2-D step for BF16 distribution storage, Allen-Cahn phase field.
#include "fused2d_impl.cuh"

namespace ipcu {
namespace f2d {
IPCU_F2D_INSTANTIATE(__nv_bfloat16, pf_bf16, 1)
}  // namespace f2d
}  // namespace ipcu
