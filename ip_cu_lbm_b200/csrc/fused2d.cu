// Storage-type dispatch of the fused 2-D step (instantiations live in
// fused2d_f32.cu, fused2d_f16.cu, fused2d_bf16.cu so they build in parallel).
#include "fused2d.cuh"

namespace ipcu {
namespace f2d {

int launch_f32(const Params &p, int qs, int geo, cudaStream_t s, bool prep);
int launch_f16(const Params &p, int qs, int geo, cudaStream_t s, bool prep);
int launch_bf16(const Params &p, int qs, int geo, cudaStream_t s, bool prep);

int launch_step(const Params &p, int storage, int qs, int geo, cudaStream_t s, bool prepare_only) {
  switch (storage) {
    case IPCU_STORE_F32: return launch_f32(p, qs, geo, s, prepare_only);
    case IPCU_STORE_F16: return launch_f16(p, qs, geo, s, prepare_only);
    case IPCU_STORE_BF16: return launch_bf16(p, qs, geo, s, prepare_only);
  }
  return IPCU_ERR_UNSUPPORTED;
}

}  // namespace f2d
}  // namespace ipcu
