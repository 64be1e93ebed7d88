// Shared device helpers for the IP_CU_LBM B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ipcu.h"

namespace ipcu {

// Parameter-block slots of the reference's float/double items[] array
// (ref: itemIndex.hpp:4-33). Scalars first, then w[Q], cx[Q], cy[Q], cz[Q].
enum ItemSlot : int {
  IT_dz = 0, IT_dt = 1, IT_c = 2, IT_nx = 3, IT_ny = 4, IT_nz = 5, IT_Q = 6, IT_ratiox = 7,
  IT_ratioy = 8, IT_PFthick = 9, IT_num_calc = 10, IT_num_wall = 11, IT_num_IBPoints = 12,
  IT_dIBM = 13, IT_nu = 14, IT_alpha = 15, IT_sigma = 16, IT_tau = 17, IT_taus = 18,
  IT_wall1 = 19, IT_vec = 25
};

// Per-launch view of the parameter block: counts converted once to integers,
// lattice vectors read through the read-only path.
template <class T>
struct Items {
  const T *__restrict__ it;
  int Q;
  long long nc, nw;
  T dz, dt, c;
  __device__ __forceinline__ explicit Items(const T *items)
      : it(items), Q((int)__ldg(items + IT_Q)), nc((long long)__ldg(items + IT_num_calc)),
        nw((long long)__ldg(items + IT_num_wall)), dz(__ldg(items + IT_dz)), dt(__ldg(items + IT_dt)),
        c(__ldg(items + IT_c)) {}
  __device__ __forceinline__ T w(int k) const { return __ldg(it + IT_vec + k); }
  __device__ __forceinline__ T cx(int k) const { return __ldg(it + IT_vec + Q + k); }
  __device__ __forceinline__ T cy(int k) const { return __ldg(it + IT_vec + 2 * Q + k); }
  __device__ __forceinline__ T cz(int k) const { return __ldg(it + IT_vec + 3 * Q + k); }
  __device__ __forceinline__ T scal(int slot) const { return __ldg(it + slot); }
};

// Direction tables of the reference's D2Q9 (x-z plane) and D3Q27 orderings
// (ref: function/basic.cu:78-97,112-153). Index 0 = Q9, 1 = Q27.
struct DirTables {
  int8_t kinv[2][27];  // opposite direction
  int8_t cp[2][27];    // downstream partner used by the flux form (0 = self)
  int8_t cm[2][27];    // upstream partner
  int8_t cip[27], cim[27];        // Q27 corner partners of the xy tensor stencil
  int8_t cxp[27], cxm[27], cyp[27], cym[27];
};
// One copy per translation unit (no relocatable device code); each unit
// fills its copy on first use per device via ensure_tables().
static __constant__ DirTables c_dirs;
DirTables host_dir_tables();

__host__ __device__ __forceinline__ int qsel(int Q) { return Q == 27 ? 1 : 0; }

// grid-stride loop over [lo, hi)
#define IPCU_FOR(i, lo, hi)                                                                   \
  for (long long i = (long long)(lo) + (long long)blockIdx.x * blockDim.x + threadIdx.x;       \
       i < (long long)(hi); i += (long long)gridDim.x * blockDim.x)

// Launch geometry: `nthreads` > 0 mirrors the reference's numBlocks*blockSize
// coverage; otherwise a persistent grid of 4 CTAs per SM is used and the
// kernel's grid-stride loop covers whatever counts items[] holds.
struct Launch {
  dim3 grid, block;
};
Launch launch_for(long long nthreads);

int status_from_cuda(cudaError_t e);

// Fills this translation unit's constant tables once per device. The first
// launch on a device therefore issues one synchronous constant copy and
// should happen outside stream capture.
static inline void ensure_tables() {
  static bool done[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  if (!done[dev]) {
    DirTables t = host_dir_tables();
    cudaMemcpyToSymbol(c_dirs, &t, sizeof t);
    done[dev] = true;
  }
}

}  // namespace ipcu
