// Instantiations of the fused 2-D step for __nv_bfloat16 distribution storage.
#include "fused2d_impl.cuh"

namespace ipcu {
namespace f2d {

int launch_bf16(const Params &p, int qs, int geo, cudaStream_t s, bool prep) {
  switch (qs) {
    case 0: return launch_g<__nv_bfloat16, 0>(p, geo, s, prep);
    case 5: return launch_g<__nv_bfloat16, 5>(p, geo, s, prep);
    case 9: return launch_g<__nv_bfloat16, 9>(p, geo, s, prep);
  }
  return IPCU_ERR_UNSUPPORTED;
}

int launch_batched_bf16(const Params *ps, const WorkItem *work, int nwork, int parity, int qs, int geo, int grid,
                        cudaStream_t s, bool prep) {
  switch (qs) {
    case 0: return launch_bg<__nv_bfloat16, 0>(ps, work, nwork, parity, geo, grid, s, prep);
    case 5: return launch_bg<__nv_bfloat16, 5>(ps, work, nwork, parity, geo, grid, s, prep);
    case 9: return launch_bg<__nv_bfloat16, 9>(ps, work, nwork, parity, geo, grid, s, prep);
  }
  return IPCU_ERR_UNSUPPORTED;
}

}  // namespace f2d
}  // namespace ipcu
