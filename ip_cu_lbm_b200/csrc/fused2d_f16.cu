// Instantiations of the fused 2-D step for FP16 distribution storage, salinity scalar.
#include "fused2d_impl.cuh"

namespace ipcu {
namespace f2d {
IPCU_F2D_INSTANTIATE(__half, f16, 0)
}  // namespace f2d
}  // namespace ipcu
