// Storage-type and scalar-physics dispatch of the fused 2-D step. The
// instantiations live in fused2d_{f32,f16,bf16}.cu (salinity) and
// fused2d_pf_{f32,f16,bf16}.cu (phase field) so that they build in parallel.
#include "fused2d.cuh"

namespace ipcu {
namespace f2d {

#define IPCU_F2D_DECL(NAME)                                                                        \
  int launch_##NAME(const Params &p, int qs, int geo, cudaStream_t s, bool prep);                  \
  int launch_batched_##NAME(const Params *, const WorkItem *, int, int, int, int, int, cudaStream_t, bool, bool, bool);
IPCU_F2D_DECL(f32)
IPCU_F2D_DECL(f16)
IPCU_F2D_DECL(bf16)
IPCU_F2D_DECL(pf_f32)
IPCU_F2D_DECL(pf_f16)
IPCU_F2D_DECL(pf_bf16)
#undef IPCU_F2D_DECL

int launch_batched(const Params *ps, const WorkItem *work, int nwork, int parity, int storage, int qs, int geo,
                   int pf, int grid, cudaStream_t s, bool prep, bool tma, bool pdl) {
  switch (storage) {
    case IPCU_STORE_F32:
      return pf ? launch_batched_pf_f32(ps, work, nwork, parity, qs, geo, grid, s, prep, tma, pdl)
                : launch_batched_f32(ps, work, nwork, parity, qs, geo, grid, s, prep, tma, pdl);
    case IPCU_STORE_F16:
      return pf ? launch_batched_pf_f16(ps, work, nwork, parity, qs, geo, grid, s, prep, tma, pdl)
                : launch_batched_f16(ps, work, nwork, parity, qs, geo, grid, s, prep, tma, pdl);
    case IPCU_STORE_BF16:
      return pf ? launch_batched_pf_bf16(ps, work, nwork, parity, qs, geo, grid, s, prep, tma, pdl)
                : launch_batched_bf16(ps, work, nwork, parity, qs, geo, grid, s, prep, tma, pdl);
  }
  return IPCU_ERR_UNSUPPORTED;
}

int launch_step(const Params &p, int storage, int qs, int geo, cudaStream_t s, bool prepare_only) {
  if (p.lean && p.push && storage == IPCU_STORE_F32 && qs == 0 && !p.pf) return launch_push(p, s, prepare_only);
  switch (storage) {
    case IPCU_STORE_F32: return p.pf ? launch_pf_f32(p, qs, geo, s, prepare_only) : launch_f32(p, qs, geo, s, prepare_only);
    case IPCU_STORE_F16: return p.pf ? launch_pf_f16(p, qs, geo, s, prepare_only) : launch_f16(p, qs, geo, s, prepare_only);
    case IPCU_STORE_BF16:
      return p.pf ? launch_pf_bf16(p, qs, geo, s, prepare_only) : launch_bf16(p, qs, geo, s, prepare_only);
  }
  return IPCU_ERR_UNSUPPORTED;
}

}  // namespace f2d
}  // namespace ipcu
