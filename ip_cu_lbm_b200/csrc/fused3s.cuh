// Parameters of the fused 3-D step on stretched x and y axes (fused3s.cu).
#pragma once
#include <cuda_runtime.h>

#include "ipcu.h"

namespace ipcu {
namespace f3s {

constexpr int kTX = 32, kTY = 16, kThreads = kTX * kTY;
constexpr int kMinBlocks = 1;  // one 512-thread CTA per SM (its rings take ~190 KB of shared memory)

// Flux-form tables of one stretched axis (n cells), built on the host like
// the 2-D solver's (sim.cu axis_tables): node weights wA [2][n][NS] (sign of
// the population's motion, cell, node), fin scale scin [2][n], fout scale
// scout [n] = dz / D, combined interior weights wC [2][NS+1][n], and the
// density-gradient factors ginv [n] = 1/(x_{i+1} - x_{i-1} + dz/1000)
// (clamped neighbours).
struct Axis {
  const float *wA, *scin, *scout, *wC, *ginv;
};

struct Params3S {
  int nx, ny, nz, zchunk;  // z cells per CTA
  // populations f [19][N] and g [7][N] in the storage type (FP32, or the
  // 16-bit deviations of store3d.cuh), the force F [3][N] in FP32
  const void *f_in, *g_in;
  const float *F_in;
  void *f_out, *g_out;
  float *F_out;
  // 16-bit storage: the reference planes [5][N] (p, u_x/c, u_y/c, u_z/c, S)
  // of the state read and of the state written, the deviations' scale, and
  // the largest finite stored magnitude (status bit 2 beyond it)
  int store;  // IPCU_STORE_*
  const void *r_in;
  void *r_out;
  float scale, inv_scale, store_max;
  Axis ax, ay;
  float c, dt, itau, omg_s;  // 1/tau, 1 - 1/tau_s
  float fk3, hdt;            // 3 dt / c, dt / 2
  float rho0, rsal, gb;      // rho = rho0 + rsal S; buoyancy -gb S
  float giz_in, giz_wall;    // z (uniform): 1/(2dz + dz/1000), 1/(dz + dz/1000)
  int mrt;
  unsigned *status;
  const float *fext;  // [3][N] immersed-boundary force density added to the force, or null
  // the box outside which that density is zero (i0, j0, k0, wi, wj, wk; wi 0:
  // none), device memory the body update rewrites
  const int *fext_box;
};

// ns: 3 (quadratic upwind) or 5 (the reference's stencil); p.store selects
// the storage instantiation
int launch3s(const Params3S &p, int ns, cudaStream_t s, bool prepare_only = false);

}  // namespace f3s
}  // namespace ipcu
