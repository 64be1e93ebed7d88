// Parameters of the fused 2-D step kernel (fused2d.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "ipcu.h"

namespace ipcu {
namespace f2d {

constexpr int kTX = 32;  // tile width along x (one warp per row)
constexpr int kTZ = 16;  // tile height along z
constexpr int kThreads = 256;
constexpr int kMinBlocks = 4;  // resident CTAs per SM the register budget is sized for
constexpr int kTmaBoxX = kTX + 8;     // TMA box width, FP32: [x0-4, x0+kTX+4), 16-byte aligned start
constexpr int kTmaBoxX16 = kTX + 16;  // TMA box width, 16-bit: [x0-8, x0+kTX+8)

// halo rows of the streaming stencil along z (1 unless z is the interpolated axis)
inline int halo_z(int geo) { return geo == IPCU_GEO_Z5 ? 3 : (geo == IPCU_GEO_Z3 ? 2 : 1); }

struct alignas(64) Params {
  // TMA descriptors of the ping-pong buffers (FP32 storage with nx % 4 == 0,
  // 16-bit storage with nx % 8 == 0): f [9][nz][nx], g [q][nz][nx],
  // macroscopic [3 or 4][nz][nx]; boxes sized for the tile + halo (f, g) and
  // the salinity ring rows (macroscopic)
  CUtensorMap tm_f[2], tm_g[2], tm_m[2];
  int tma;  // 1: the single-simulation kernel stages with the maps above
  int nx, nz;
  int mrt, wall;  // mrt: 0 BGK, 1 general MRT, 2 MRT with unit non-shear rates (two-moment form)
  // ping-pong state; a step reads buffer (cur ^ parity) and writes the other
  void *fbuf[2];
  void *gbuf[2];
  float *mbuf[2];  // [3][N]: S, ux, uz; 16-bit storage adds p* as a 4th plane
  int cur;
  // interpolated axis: weights [2][NA][NS], fin scale [2][NA], fout scale [NA],
  // and the interior cells' combined flux weights [2][NS+1][NA]
  const float *wA, *scin, *scout, *wC;
  // 1/(x_{i+1} - x_{i-1} + dz/1000) with clamped neighbours (density gradient);
  // gconst bit 0 (x) / bit 1 (z): the table is first, mid..., last, given
  // in gix3 / giz3, so the kernel needs no load for it
  const float *ginvx, *ginvz;
  float gix3[3], giz3[3];
  int gconst;
  float c, dt, tau, taus;
  float fk3, hdt;  // 3 dt / c (forcing term per unit density) and dt / 2
  // rho = rho_base + rho_sal_f * S: salinity (base rhoL + (rhoH - rhoL) phi)
  // or the phase field phi (base rhoL, slope rhoH - rhoL)
  float rho_base;
  // phase field: obuf[2] = [2][N] phi u, phi w of the previous step;
  // ilx2, ilz2 = 1/dx^2, 1/dz^2 per column / row (Laplacian of phi);
  // 4 beta = 48 sigma / W, kappa = 1.5 sigma W, 1/W,
  // (tau_phi - 1/2)/tau_phi, gravity
  float *obuf[2];
  const float *ilx2, *ilz2;
  float pf_beta4, pf_kap, pf_invw, pf_lam, grav;
  int pf;
  float rhoL, rhoH, phi;
  double rho_sal, g_bouss;
  float rho_sal_f, g_bouss_f;
  // 16-bit storage: stored = (value - equilibrium) * scale; store_max is the
  // largest finite stored magnitude (FP16 65504)
  float fscale, inv_fscale, gscale, inv_gscale, store_max;
  float MM[81];   // Minv diag(S) M with the shear rates zeroed
  float Ms[18];   // shear rows 7, 8 of M
  float Mis[18];  // shear columns 7, 8 of Minv, [a][2]
  int8_t slipB9[16 * 9], slipK9[16 * 9];  // per wall class: owner neighbour and population
  int8_t slipB5[16 * 9], slipK5[16 * 9];
  unsigned *status;
  // immersed boundaries: force density [2][N] added to the cell force where
  // the cell's tile is flagged by some body in ibflag ([ibnb bodies][ntz][ibtx]:
  // some cell of the tile or of its halo carries that body's force); null
  // without a body
  const float *fext;
  const uint8_t *ibflag;
  int ibtx, ibnb;
  // Lean flow-only step (FP32 storage, TMA staging, no scalar lattice, S
  // uniform): the S plane is constant and never read or written; the
  // velocity planes of buffer b hold a tile's values only where
  // ustore[b][tile] = 1 (tiles that carried an immersed-boundary force in
  // the step that wrote b). Elsewhere the velocity is c j + F0 dt / 2 rho,
  // recomputed from the populations (F0 = (0, -s_uni g_bouss)), bit for bit
  // what the step would have stored.
  uint8_t *ustore[2];
  int lean, ntx, ntz;
  float s_uni;
  // Push form of the lean step (push2d.cu; bounce-back walls, two-moment
  // MRT): each cell collides its own populations in registers and pushes
  // them to the cells they stream into, so the velocity of the new state is
  // never formed or stored.
  int push;
  // ib_uform (FP32 storage, no scalar lattice, uniform S): a body update
  // leaves the velocity c j + (F0 + f_ib) dt / 2 rho in the cells it
  // forced, with f_ib its new force density -- the state's velocity
  // is then fma(F0 + f_ib, dt / 2 rho, c j) in every cell, f_ib as it
  // stands (lean_velocity).
  int ib_uform;
};

// p*, j_x, j_z of nine populations in the one summation order every kernel
// and the host use (k = 0..8, starting from zero), so that a velocity
// recomputed from stored populations equals the one stored beside them.
__host__ __device__ __forceinline__ void moments9(const float (&f)[9], float &pr, float &jx, float &jz) {
  constexpr int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1}, ez[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
  pr = 0.f;
  jx = 0.f;
  jz = 0.f;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    pr += f[k];
    if (ex[k] > 0) jx += f[k];
    if (ex[k] < 0) jx -= f[k];
    if (ez[k] > 0) jz += f[k];
    if (ez[k] < 0) jz -= f[k];
  }
}

// prepare_only: set the kernel's shared-memory attribute (call once before any capture);
// p.pf selects the phase-field kernels
int launch_step(const Params &p, int storage, int qs, int geo, cudaStream_t s, bool prepare_only = false);
// The push form of the lean flow-only step (FP32, no scalar lattice, uniform
// grid and S, bounce-back, p.mrt == 2).
int launch_push(const Params &p, cudaStream_t s, bool prepare_only = false);

// Velocity of cell ci of buffer b of a lean simulation: the planes where
// the step that wrote b stored them (ustore 1), elsewhere c j + F dt / 2 rho
// from the populations with F = F0 + f_ib, F0 = (0, -S g') and f_ib the
// immersed-boundary force density as it stands -- the force that step
// applied, or, once a body update has run, the update's new force (ib_uform)
// -- bit for bit the value the full step and the body update store.
__device__ __forceinline__ void lean_velocity(const Params &p, int b, long long ci, long long N, float &ux,
                                              float &uz) {
  const int x = (int)(ci % p.nx), z = (int)(ci / p.nx);
  if (p.ustore[b][(z / kTZ) * p.ntx + x / kTX] == 1) {
    ux = p.mbuf[b][N + ci];
    uz = p.mbuf[b][2 * N + ci];
    return;
  }
  const float *fb = static_cast<const float *>(p.fbuf[b]);
  float fv[9];
#pragma unroll
  for (int k = 0; k < 9; k++) fv[k] = fb[k * N + ci];
  float pr, jx, jz;
  moments9(fv, pr, jx, jz);
  const float h0 = __fdividef(p.hdt, fmaf(p.s_uni, p.rho_sal_f, p.rho_base));
  float Fx = 0.0f, Fz = 0.0f;
  Fz -= __fmul_rn(p.s_uni, p.g_bouss_f);
  if (p.fext != nullptr) {
    Fx += p.fext[ci];
    Fz += p.fext[N + ci];
  }
  ux = fmaf(Fx, h0, p.c * jx);
  uz = fmaf(Fz, h0, p.c * jz);
}

// One work item of a batched step: simulation index and tile coordinates.
struct WorkItem {
  int sim, tx, tz, pad;
};
// Advances every simulation referenced by `work` (all of the same storage,
// scalar lattice and geometry) by one step; `params` and `work` are device
// arrays; `parity` flips the ping-pong buffers of all of them. `grid` CTAs
// loop over the work list. tma: every one of them has tensor maps (staged
// with TMA box loads, the maps read from `params`). pdl: launched as a
// programmatic dependent of the previous launch, a batch of body updates
// (ib2d::launch_batched): the tiles those bodies flagged wait for it, the
// rest of the work list runs beside it.
int launch_batched(const Params *params, const WorkItem *work, int nwork, int parity, int storage, int qs, int geo,
                   int pf, int grid, cudaStream_t s, bool prepare_only, bool tma, bool pdl = false);

}  // namespace f2d
}  // namespace ipcu
