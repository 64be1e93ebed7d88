// Parameters of the fused 3-D step kernel (fused3d.cu).
#pragma once
#include <cuda_runtime.h>

#include "ipcu.h"

namespace ipcu {
namespace f3d {

struct Params3 {
  int nx, ny, nz, zchunk;  // z cells per CTA
  const float *f_in, *g_in, *F_in;
  float *f_out, *g_out, *F_out;
  float c, dt, itau, omg_s;  // 1/tau, 1 - 1/tau_s
  float fk3, hdt;            // 3 dt / c, dt / 2
  float rho0, rsal, gb;      // rho = rho0 + rsal S; buoyancy -gb S
  float gi_in, gi_wall;      // 1/(2dz + dz/1000), 1/(dz + dz/1000) (clamped central differences)
  int mrt;
  unsigned *status;
  const float *fext;  // [3][N] immersed-boundary force density added to the force, or null
  // the box outside which that density is zero (i0, j0, k0, wi, wj, wk; wi 0:
  // none), device memory the body update rewrites
  const int *fext_box;
};

int launch3d(const Params3 &p, cudaStream_t s);

}  // namespace f3d
}  // namespace ipcu
