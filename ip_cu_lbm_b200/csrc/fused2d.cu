// Storage-type dispatch of the fused 2-D step (instantiations live in
// fused2d_f32.cu, fused2d_f16.cu, fused2d_bf16.cu so they build in parallel).
#include "fused2d.cuh"

namespace ipcu {
namespace f2d {

int launch_f32(const Params &p, int qs, int geo, cudaStream_t s, bool prep);
int launch_f16(const Params &p, int qs, int geo, cudaStream_t s, bool prep);
int launch_bf16(const Params &p, int qs, int geo, cudaStream_t s, bool prep);

int launch_batched_f32(const Params *, const WorkItem *, int, int, int, int, int, cudaStream_t, bool);
int launch_batched_f16(const Params *, const WorkItem *, int, int, int, int, int, cudaStream_t, bool);
int launch_batched_bf16(const Params *, const WorkItem *, int, int, int, int, int, cudaStream_t, bool);

int launch_batched(const Params *ps, const WorkItem *work, int nwork, int parity, int storage, int qs, int geo,
                   int grid, cudaStream_t s, bool prep) {
  switch (storage) {
    case IPCU_STORE_F32: return launch_batched_f32(ps, work, nwork, parity, qs, geo, grid, s, prep);
    case IPCU_STORE_F16: return launch_batched_f16(ps, work, nwork, parity, qs, geo, grid, s, prep);
    case IPCU_STORE_BF16: return launch_batched_bf16(ps, work, nwork, parity, qs, geo, grid, s, prep);
  }
  return IPCU_ERR_UNSUPPORTED;
}

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
