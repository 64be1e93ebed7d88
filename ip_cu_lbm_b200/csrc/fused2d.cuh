// Parameters of the fused 2-D step kernel (fused2d.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ipcu.h"

namespace ipcu {
namespace f2d {

constexpr int kTX = 32;  // tile width along x (one warp per row)
constexpr int kTZ = 16;  // tile height along z
constexpr int kThreads = 256;
constexpr int kMinBlocks = 4;  // resident CTAs per SM the register budget is sized for

struct Params {
  int nx, nz;
  int mrt, wall;  // mrt: 0 BGK, 1 general MRT, 2 MRT with unit non-shear rates (two-moment form)
  // ping-pong state; a step reads buffer (cur ^ parity) and writes the other
  void *fbuf[2];
  void *gbuf[2];
  float *mbuf[2];  // [3][N]: S, ux, uz
  int cur;
  // interpolated axis: weights [2][NA][NS], fin scale [2][NA], fout scale [NA],
  // and the interior cells' combined flux weights [2][NS+1][NA]
  const float *wA, *scin, *scout, *wC;
  // 1/(x_{i+1} - x_{i-1} + dz/1000) with clamped neighbours (density gradient)
  const float *ginvx, *ginvz;
  float c, dt, tau, taus;
  float fk3, hdt;  // 3 dt / c (forcing term per unit density) and dt / 2
  float rhoL, rhoH, phi;
  double rho_sal, g_bouss;
  float fscale, inv_fscale, gscale, inv_gscale, s_ref;
  float MM[81];   // Minv diag(S) M with the shear rates zeroed
  float Ms[18];   // shear rows 7, 8 of M
  float Mis[18];  // shear columns 7, 8 of Minv, [a][2]
  int8_t slipB9[16 * 9], slipK9[16 * 9];  // per wall class: owner neighbour and population
  int8_t slipB5[16 * 9], slipK5[16 * 9];
  unsigned *status;
};

// prepare_only: set the kernel's shared-memory attribute (call once before any capture)
int launch_step(const Params &p, int storage, int qs, int geo, cudaStream_t s, bool prepare_only = false);

// One work item of a batched step: simulation index and tile coordinates.
struct WorkItem {
  int sim, tx, tz, pad;
};
// Advances every simulation referenced by `work` (all of the same storage,
// scalar lattice and geometry) by one step; `params` and `work` are device
// arrays; `parity` flips the ping-pong buffers of all of them. `grid` CTAs
// loop over the work list.
int launch_batched(const Params *params, const WorkItem *work, int nwork, int parity, int storage, int qs, int geo,
                   int grid, cudaStream_t s, bool prepare_only = false);

}  // namespace f2d
}  // namespace ipcu
