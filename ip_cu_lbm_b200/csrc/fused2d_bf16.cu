// Instantiations of the fused 2-D step for BF16 distribution storage, salinity scalar.
#include "fused2d_impl.cuh"

namespace ipcu {
namespace f2d {
IPCU_F2D_INSTANTIATE(__nv_bfloat16, bf16, 0)
}  // namespace f2d
}  // namespace ipcu
