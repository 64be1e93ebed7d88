// Instantiations of the fused 2-D step for float distribution storage, Allen-Cahn phase field.
#include "fused2d_impl.cuh"

namespace ipcu {
namespace f2d {
IPCU_F2D_INSTANTIATE(float, pf_f32, 1)
}  // namespace f2d
}  // namespace ipcu
