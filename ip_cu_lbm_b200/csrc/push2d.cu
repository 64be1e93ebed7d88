// Push form of the lean flow-only 2-D step: D2Q9 two-moment MRT with
// forcing on a uniform grid with bounce-back walls, FP32 storage, no scalar
// lattice, uniform S (the settling-ellipse configuration). The state is the
// same as the tile kernel's (post-streaming populations f, SoA, x fastest),
// and so is every result, bit for bit: each cell loads its own nine
// populations (coalesced, no halo, no shared memory), forms its moments and
// velocity, collides in registers with the collision the tile kernel uses
// (collide_mrt2), and pushes each post-collision population to the cell it
// streams into -- or, where that cell lies outside the box, into its own
// opposite slot (halfway bounce-back, the tile kernel's rule for sources
// outside the box: ref function/propagation.cu, set_wall_propagation).
//
// The velocity of a cell is c j + F dt / 2 rho with F = F0 + f_ib, F0 =
// (0, -S g') and f_ib the body's force density as it stands, which is this
// step's force (lean_velocity in fused2d.cuh: a body update leaves that
// velocity in the cells it forces), so no velocity plane is read or
// written: 72 bytes per cell and step.
//
// Tiles are the tile kernel's 32 x 16 cells (the immersed-body flags and the
// ustore marks are per tile); 256 threads, two rows each. With a body the
// kernel is a programmatic dependent of the previous body update: flagged
// tiles wait for it (griddepcontrol.wait) before they read the force, the
// rest run beside it. It also releases the next body update, which waits
// for this step to complete before it reads anything, as soon as all its
// CTAs have started.
#include "fused2d_impl.cuh"

namespace ipcu {
namespace f2d {
namespace {

constexpr int kPushRows = kThreads / kTX;  // 8 rows of 32 threads; each thread takes rows r and r + 8

__global__ void __launch_bounds__(kThreads, 6) push_kernel(const __grid_constant__ Params p) {
  const int nx = p.nx, nz = p.nz;
  const long long N = (long long)nx * nz;
  const int tile_x = blockIdx.x, tile_z = blockIdx.y;
  const int bi = p.cur, bo = bi ^ 1;
  const float *__restrict__ f_in = static_cast<const float *>(p.fbuf[bi]);
  float *__restrict__ f_out = static_cast<float *>(p.fbuf[bo]);
  const int tile = tile_z * p.ntx + tile_x;

  // the body update after this step may be scheduled once every CTA of it
  // has started (it waits for this step's completion before it reads)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  bool ibt = false;
  if (p.fext != nullptr) {
    const long long tiles = (long long)p.ibtx * p.ntz;
    for (int b = 0; b < p.ibnb; b++)
      ibt |= *reinterpret_cast<const volatile uint8_t *>(p.ibflag + b * tiles + tile) != 0;
  }
  if (ibt) asm volatile("griddepcontrol.wait;" ::: "memory");
  const uint8_t us = p.ustore[bi][tile];

  const float c = p.c, ic = 1.0f / c;
  const float om_shear = 1.0f - 1.0f / p.tau;
  const float S = p.s_uni, rho = fmaf(S, p.rho_sal_f, p.rho_base);
  const float h0 = __fdividef(p.hdt, rho);
  const float fden = __fdividef(p.fk3, rho);
  const float gS = __fmul_rn(S, p.g_bouss_f);
  unsigned bad = 0;

  const int ix = threadIdx.x % kTX, r0 = threadIdx.x / kTX;
  const int gx = tile_x * kTX + ix;
#pragma unroll
  for (int rr = 0; rr < kTZ / kPushRows; rr++) {
    const int gz = tile_z * kTZ + r0 + rr * kPushRows;
    if (gx >= nx || gz >= nz) continue;
    const long long ci = (long long)gz * nx + gx;
    float f[9];
#pragma unroll
    for (int k = 0; k < 9; k++) f[k] = __ldcs(f_in + k * N + ci);
    float pr, jx, jz;
    moments9(f, pr, jx, jz);
    // this step's force: buoyancy of the uniform S and the body's force
    // density (zero outside the flagged tiles)
    float Fx = 0.0f, Fz = 0.0f;
    Fz -= gS;
    if (ibt) {
      Fx += p.fext[ci];
      Fz += p.fext[N + ci];
    }
    // velocity of the state: the stored planes after an upload, else
    // c j + F dt / 2 rho with this force
    float u, w;
    if (us == 1) {
      u = p.mbuf[bi][N + ci];
      w = p.mbuf[bi][2 * N + ci];
    } else {
      u = fmaf(Fx, h0, c * jx);
      w = fmaf(Fz, h0, c * jz);
    }
    const float uc = u * ic, wc = w * ic;
    float o[9];
    collide_mrt2<false>(f, pr, uc, wc, fden, Fx, Fz, om_shear, o);
    bad |= !(isfinite(u) && isfinite(w) && isfinite(pr));
    // push: population k to the cell it streams into, or back into this
    // cell's opposite slot at a wall
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const int tx = gx + ex(k), tz = gz + ez(k);
      if (tx >= 0 && tx < nx && tz >= 0 && tz < nz)
        __stcs(f_out + k * N + ci + ex(k) + (long long)ez(k) * nx, o[k]);
      else
        __stcs(f_out + kinv(k) * N + ci, o[k]);
    }
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(p.status, 1u);
  if (threadIdx.x == 0) p.ustore[bo][tile] = 0;
}

}  // namespace

int launch_push(const Params &p, cudaStream_t s, bool prepare_only) {
  if (prepare_only) return IPCU_OK;
  const dim3 grid((p.nx + kTX - 1) / kTX, (p.nz + kTZ - 1) / kTZ);
  if (p.fext) return launch_pdl(push_kernel, grid, 0, s, p);
  push_kernel<<<grid, kThreads, 0, s>>>(p);
  return status_from_cuda(cudaGetLastError());
}

}  // namespace f2d
}  // namespace ipcu
