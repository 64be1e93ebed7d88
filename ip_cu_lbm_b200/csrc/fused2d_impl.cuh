// Fused collide-and-stream step for 2-D boxes (D2Q9 flow in the x-z plane +
// D2Q5 or Q9 salinity), the B200 path of the reference's per-step chain
//   equ_f -> Force -> col_f_MRT -> IP_process(f) -> col_g_reg -> IP_process(g)
//   -> update_scalar -> update_rho -> set_wall_rho
// (ref: LockExchange/LockExchange.cu:220-236; kernels in function/collision.cu,
// function/adv.cu, function/set_bound.cu, function/propagation.cu).
//
// One launch per time step. A CTA owns a kTX x kTZ tile. Phase 0 stages the
// tile, its streaming halo (HX cells along x, HZ along z) and the salinity
// ring one cell wider: with FP32 storage and nx a multiple of 4 as three TMA
// box loads (f, g and the S/u_x/u_z planes, cp.async.bulk.tensor completing
// on one mbarrier), otherwise the ring through registers while phase 1 loads
// f, g, u itself. Phase 1 collides tile + halo into shared memory, phase 2
// evaluates the reference's conservative interpolated streaming for the
// interior from shared memory, forms the moments and writes the new state.
// Every stored value is read from HBM once and written once per step (halo
// re-reads hit L2). Storage is structure-of-arrays, x fastest. With 16-bit
// storage the populations are kept as deviations from the local
// equilibrium (storage.cuh).
//
// The streaming reproduces IP_process on a rectilinear box exactly:
//   ftmp(j,k) = f*(j+a,k) + (fin(j,k) - fout(j+a,k))        (adv.cu:234-244)
//   fout(j,k) = I_k(j) dz/D_j,  fin(j,k) = I_k(j) dz/D_{j+a}  (adv.cu:76-87)
//   f_new(c,k) = ftmp(c - e_k, k)                               (propagation.cu)
// with I_k the Lagrange interpolant along the interpolated axis evaluated at
// x_j + s(D_j - dz)/2 (weights precomputed per axis index on the host, ghost
// nodes clamped as set_posl_x does), ghost values equal to the owner
// (set_wall_f), wall partners mirrored (set_wall_f_inv), and sources outside
// the box taken from the owner's bounce-back (k -> -k) or specular slip
// partner (set_wall_propagation with the set_bound2D tables).
//
// Cells whose whole stencil lies inside the box take a clamp-free path with
// compile-time shared-memory offsets; cells next to a wall take the general
// path with the ghost rules.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstddef>
#include <type_traits>

#include "fused2d.cuh"
#include "ipcu_common.cuh"
#include "storage.cuh"

namespace ipcu {
namespace f2d {

// D2Q9 in the x-z plane in the reference's order (ref: function/basic.cu:78-87);
// D2Q5 is its first five directions.
__host__ __device__ constexpr int ex(int k) { return (k == 1 || k == 5 || k == 8) ? 1 : ((k == 3 || k == 6 || k == 7) ? -1 : 0); }
__host__ __device__ constexpr int ez(int k) { return (k == 2 || k == 5 || k == 6) ? 1 : ((k == 4 || k == 7 || k == 8) ? -1 : 0); }
__host__ __device__ constexpr int kinv(int k) { return k == 0 ? 0 : (k <= 4 ? ((k + 1) % 4) + 1 : ((k - 5 + 2) % 4) + 5); }
__host__ __device__ constexpr int mirx(int k) {
  return k == 1 ? 3 : k == 3 ? 1 : k == 5 ? 6 : k == 6 ? 5 : k == 7 ? 8 : k == 8 ? 7 : k;
}
__host__ __device__ constexpr int mirz(int k) {
  return k == 2 ? 4 : k == 4 ? 2 : k == 5 ? 8 : k == 8 ? 5 : k == 6 ? 7 : k == 7 ? 6 : k;
}
__host__ __device__ constexpr float w9(int k) { return k == 0 ? 4.0f / 9.0f : (k <= 4 ? 1.0f / 9.0f : 1.0f / 36.0f); }
__host__ __device__ constexpr float w5(int k) { return k == 0 ? 1.0f / 3.0f : 1.0f / 6.0f; }
template <int Q>
__host__ __device__ constexpr float wq(int k) { return Q == 5 ? w5(k) : w9(k); }

// Tile geometry. TMA staging needs the smem box to start on a 16-byte
// boundary in x, so its rows span [x0-4, x0+kTX+4) (40 floats); register
// staging keeps just the halo columns.
template <int GEO, bool TMA>
struct Geo {
  static constexpr int AX = (GEO == IPCU_GEO_X5 || GEO == IPCU_GEO_X3) ? 0 : ((GEO == IPCU_GEO_Z5 || GEO == IPCU_GEO_Z3) ? 1 : -1);
  static constexpr int NS = (GEO == IPCU_GEO_X5 || GEO == IPCU_GEO_Z5) ? 5 : ((GEO == IPCU_GEO_X3 || GEO == IPCU_GEO_Z3) ? 3 : 1);
  static constexpr int H = NS == 5 ? 3 : (NS == 3 ? 2 : 1);
  static constexpr int HX = AX == 0 ? H : 1;
  static constexpr int HZ = AX == 1 ? H : 1;
  static constexpr int XO = TMA ? 4 : HX;               // smem column of the tile's first cell
  static constexpr int EX = TMA ? kTX + 8 : kTX + 2 * HX;
  static constexpr int EZ = kTZ + 2 * HZ, NE = EX * EZ;
  static constexpr int CX0 = XO - HX, CW = kTX + 2 * HX;  // columns that are collided
  static constexpr int NC = CW * EZ;
  // salinity ring (rows z0-HZ-1 .. z0+kTZ+HZ): TMA shares the tile's columns,
  // register staging keeps one extra column on each side
  static constexpr int RX = TMA ? EX : EX + 2, RO = TMA ? 0 : 1, SZ = EZ + 2;
  static constexpr int NWA = AX == 0 ? EX : (AX == 1 ? EZ : 0);
  static constexpr int WREC = NS + 2;                     // NS weights, fin scale, fout scale
  static_assert(!TMA || EX == kTmaBoxX, "tensor-map box width");
};

// Cells next to a wall are queued in shared memory and processed after the
// interior cells by a compacted set of threads (up to kQueue per tile; more
// are processed in place). At the C2 size a tile has at most ~80 of them.
constexpr int kQueue = 111;

// Shared-memory layout in floats; TMA destinations start on 128-byte boundaries.
// SB: bytes of a stored population. TMA staging of 16-bit storage lands the
// f and g boxes ([planes][EZ][kTmaBoxX16] 16-bit values, starting at
// x0 - 8 so the x coordinate stays 16-byte aligned) in their own area H0,
// from which the collision phase reads them into the float tile, and stages
// four macroscopic planes (S, u_x, u_z, p*).
template <int QS, int GEO, bool TMA, int SB = 4>
struct Smem {
  using G = Geo<GEO, TMA>;
  static constexpr int al(int v, int a) { return (v + a - 1) / a * a; }
  static constexpr bool H16 = TMA && SB == 2;
  static constexpr int G0 = al(9 * G::NE, 32);                   // g tile
  static constexpr int S0 = al(G0 + QS * G::NE, 32);             // ring (TMA: S, u_x, u_z [, p*] planes)
  static constexpr int F0 = S0 + (TMA ? (H16 ? 4 : 3) : 1) * G::SZ * G::RX;  // registers: interior force
  static constexpr int W0 = F0 + (TMA ? 0 : 2 * kTX * kTZ);      // axis weights
  static constexpr int C0 = W0 + 2 * G::WREC * G::NWA;            // combined interior weights
  static constexpr int GI0 = C0 + 2 * (G::NS + 1) * G::NWA;       // density-gradient factors of the rows [EZ]
  static constexpr int B0 = al(GI0 + G::EZ, 2);                     // mbarrier
  static constexpr int Q0 = B0 + 4;                                // wall-cell queue: count + kQueue slots
  static constexpr int E16 = G::EZ * kTmaBoxX16;                   // 16-bit values per staged plane
  static constexpr int H0 = al(Q0 + 1 + kQueue, 32);               // 16-bit staging: f planes, then g
  static constexpr int HG = al(H0 + 9 * E16 / 2, 32);              // TMA destinations: 128-byte aligned
  static constexpr size_t bytes = sizeof(float) * (size_t)(H16 ? HG + QS * E16 / 2 : Q0 + 1 + kQueue);
};
template <int QS, int GEO, bool TMA, int SB = 4>
constexpr size_t smem_bytes() { return Smem<QS, GEO, TMA, SB>::bytes; }

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Acquires a tensor map written to global memory by the generic proxy (the
// batched kernel's parameter array is rewritten between launches)
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap *map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
               : "memory");
}
// 3-D tiled TMA load (no multicast) into this CTA's shared memory
__device__ __forceinline__ void tma_load_3d(unsigned dst, const CUtensorMap *map, int x, int y, int z, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}
// Waits for phase `phase` of the barrier, giving up after `limit` clock cycles.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned phase, long long limit) {
  const long long t0 = clock64();
  while (true) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred P;\n mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n selp.u32 %0, 1, 0, P;\n}"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
  }
}
constexpr long long kWaitLimit = 2000000000LL;  // ~1 s at the B200 boost clock

// storage conversion: value = stored*inv_scale
template <class ST>
__device__ __forceinline__ float ld(const ST *p, long long i, float inv_scale) {
  if constexpr (sizeof(ST) == 4) {
    return reinterpret_cast<const float *>(p)[i];
  } else if constexpr (std::is_same<ST, __half>::value) {
    return __half2float(p[i]) * inv_scale;
  } else {
    return __bfloat162float(p[i]) * inv_scale;
  }
}
template <class ST>
__device__ __forceinline__ void st(ST *p, long long i, float v, float scale) {
  if constexpr (sizeof(ST) == 4) {
    reinterpret_cast<float *>(p)[i] = v;
  } else if constexpr (std::is_same<ST, __half>::value) {
    p[i] = __float2half_rn(v * scale);
  } else {
    p[i] = __float2bfloat16_rn(v * scale);
  }
}

// Two-moment MRT collision with forcing (unit non-shear rates, the
// reference's S file): the non-shear moments relax to equilibrium in one
// step, so
//   f*_k = feq_k + Fk_k / 2 + (1 - 1/tau) (Minv_s M_s d)_k,  d = f - feq + Fk/2
// (ref: collision.cu:115-150), whose shear moments reduce to (Lallemand-Luo
// rows 7, 8)
//   p_xx = (f1 + f3 - f2 - f4) - (u^2 - w^2)/c^2,  p_xz = (f5 + f7 - f6 - f8) - u w/c^2
// (the forcing parts cancel pairwise); feq + Fk/2 is formed per opposite pair
// from A = p* - 1.5 u^2 + 4.5 (e.u)^2, B = 3 e.u + e.F fden/2. uc, wc: u/c;
// RES: f holds f - feq (16-bit storage), whose shear sums are the moments.
// Shared by the tile kernel and the push kernel (push2d.cu); the sums of two
// products are written as explicit fmas, so that both kernels round alike
// whatever the compiler contracts around them.
template <bool RES>
__device__ __forceinline__ void collide_mrt2(const float (&f)[9], float pr, float uc, float wc, float fden, float Fx,
                                             float Fz, float om_shear, float (&o)[9]) {
  const float usq = fmaf(uc, uc, wc * wc);
  const float P0 = fmaf(-1.5f, usq, pr);
  const float hx = 0.5f * fden * Fx, hz = 0.5f * fden * Fz;
  const float m7 = 0.25f * om_shear * (RES ? (f[1] + f[3]) - (f[2] + f[4])
                                           : ((f[1] + f[3]) - (f[2] + f[4])) - fmaf(uc, uc, -(wc * wc)));
  const float m8 = 0.25f * om_shear * (RES ? (f[5] + f[7]) - (f[6] + f[8])
                                           : ((f[5] + f[7]) - (f[6] + f[8])) - uc * wc);
  o[0] = w9(0) * P0;
  {
    const float A = fmaf(4.5f * uc, uc, P0), B = fmaf(3.0f, uc, hx);
    o[1] = fmaf(w9(1), A + B, m7);
    o[3] = fmaf(w9(3), A - B, m7);
  }
  {
    const float A = fmaf(4.5f * wc, wc, P0), B = fmaf(3.0f, wc, hz);
    o[2] = fmaf(w9(2), A + B, -m7);
    o[4] = fmaf(w9(4), A - B, -m7);
  }
  {
    const float eu = uc + wc;
    const float A = fmaf(4.5f * eu, eu, P0), B = fmaf(3.0f, eu, hx + hz);
    o[5] = fmaf(w9(5), A + B, m8);
    o[7] = fmaf(w9(7), A - B, m8);
  }
  {
    const float eu = wc - uc;
    const float A = fmaf(4.5f * eu, eu, P0), B = fmaf(3.0f, eu, hz - hx);
    o[6] = fmaf(w9(6), A + B, -m8);
    o[8] = fmaf(w9(8), A - B, -m8);
  }
}

// Clamp-free pull for an interior cell: lc is the cell's local index; W
// holds the combined flux weights of its axis position for both signs of
// the axis velocity (see axis_tables on the host), so the flux form is one
// dot product over the NS+1 nodes around the source cell.
template <int GEO, bool TMA, int K>
struct Fast {
  using G = Geo<GEO, TMA>;
  static constexpr int DA = G::AX == 0 ? 1 : G::EX;   // one cell along the interpolated axis
  static constexpr int A = G::AX == 0 ? ex(K) : (G::AX == 1 ? ez(K) : 0);
  static constexpr int BX = G::AX == 0 ? 0 : ex(K);   // shift-axis part of e_K
  static constexpr int BZ = G::AX == 1 ? 0 : ez(K);
  __device__ __forceinline__ static float pull(const float *arr, int lc, const float (&W)[2][G::NS + 1]) {
    constexpr int NE = G::NE;
    if constexpr (G::AX < 0 || A == 0) {
      return arr[K * NE + lc - ex(K) - ez(K) * G::EX];
    } else {
      constexpr int s = A > 0 ? 0 : 1, sg = A > 0 ? 1 : -1, h = G::NS / 2;
      const float *src = arr + K * NE + lc - BX - BZ * G::EX;  // c' = c - (shift part of e_K)
      float acc = 0.f;
#pragma unroll
      for (int q = 0; q <= G::NS; q++) acc = fmaf(W[s][q], src[sg * (q - h - 1) * DA], acc);
      return acc;
    }
  }
};

// One tile of one step; shared by the single-simulation kernel (parameters in
// the kernel's constant bank) and the batched kernel (parameters in global
// memory). TMA: stage with tensor-map box loads (single-simulation FP32
// kernel; the tensor maps live in the __grid_constant__ parameters).
// tm: the tensor maps (tm_f[2], tm_g[2], tm_m[2], contiguous) of the
// simulation, in parameter or global memory (TMA staging only).
// LEAN: the lean flow-only step (Params::lean; FP32, TMA, no scalar lattice).
template <class ST, int QS, int GEO, bool TMA, int PHYS, bool LEAN = false>
__device__ __forceinline__ void step_tile(const Params &p, int parity, int tile_x, int tile_z, float *smem,
                                          const CUtensorMap *tm = nullptr) {
  static_assert(!LEAN || (TMA && QS == 0 && PHYS == 0 && sizeof(ST) == 4), "lean step: FP32 TMA flow only");
  using G = Geo<GEO, TMA>;
  using SL = Smem<QS, GEO, TMA, (int)sizeof(ST)>;
  constexpr int HZ = G::HZ, EX = G::EX, NE = G::NE, SZ = G::SZ, RX = G::RX, RO = G::RO;
  constexpr int XO = G::XO, NWA = G::NWA, WREC = G::WREC;
  // RES (16-bit storage): f and g hold deviations from the local
  // equilibrium, p* comes from its own FP32 plane
  constexpr bool RES = sizeof(ST) == 2;

  float *sf = smem;            // [9][EZ][EX] f, collided in place
  float *sg = smem + SL::G0;   // [QS][EZ][EX] g
  float *sS = smem + SL::S0;   // [SZ][RX] salinity ring (TMA: then the u_x, u_z planes)
  float *sF = smem + SL::F0;   // registers: [2][kTZ][kTX] interior force
  float *sW = smem + SL::W0;   // [2][WREC][NWA] axis weights
  float *sC = smem + SL::C0;   // [2][NS+1][NWA] combined interior weights
  float *sGI = smem + SL::GI0;  // gradient factors of the tile's rows [EZ]
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + SL::B0);
  int *qcount = reinterpret_cast<int *>(smem + SL::Q0), *queue = qcount + 1;

  const int nx = p.nx, nz = p.nz;
  const long long N = (long long)nx * nz;
  const int x0 = tile_x * kTX, z0 = tile_z * kTZ;
  const int ox = x0 - XO, oz = z0 - HZ;  // global coords of smem (0,0)
  const int tid = threadIdx.x;
  const int bi = p.cur ^ parity, bo = bi ^ 1;
  const ST *__restrict__ f_in = static_cast<const ST *>(p.fbuf[bi]);
  const ST *__restrict__ g_in = static_cast<const ST *>(p.gbuf[bi]);
  ST *__restrict__ f_out = static_cast<ST *>(p.fbuf[bo]);
  ST *__restrict__ g_out = static_cast<ST *>(p.gbuf[bo]);
  const float *__restrict__ mac_in = p.mbuf[bi];
  float *__restrict__ mac_out = p.mbuf[bo];

  // density from the scalar, in FP32 (ref: collision.cu:251): salinity
  // rhoL + (rhoH - rhoL) phi + rho_sal S, or the phase-field mixture
  // rhoL + (rhoH - rhoL) phi(x) (PHYS 1: the scalar is phi)
  static_assert(PHYS == 0 || QS > 0, "the phase field lives on the scalar lattice");
  const float rho0 = p.rho_base, rsal = p.rho_sal_f;
  auto rho_of = [&](float S) { return fmaf(S, rsal, rho0); };
  // immersed-boundary force on this tile (block-uniform). The body's update
  // of the previous step may still be running (programmatic dependent
  // launch): a flagged tile waits for it before it reads anything. The flag
  // is read past L1 (the update sets it just before it lets this kernel go).
  bool ibt = false;
  if (p.fext != nullptr) {
    const long long tiles = (long long)p.ibtx * p.ntz;
    for (int b = 0; b < p.ibnb; b++)
      ibt |= *reinterpret_cast<const volatile uint8_t *>(p.ibflag + b * tiles + tile_z * p.ibtx + tile_x) != 0;
  }
  if (ibt) asm volatile("griddepcontrol.wait;" ::: "memory");
  // lean step: which of the 3 x 3 tiles around this one hold their velocity
  // planes in the input buffer (bit (dz + 1) * 3 + (dx + 1)); the staged
  // macroscopic box is loaded only when one of them does. The mask sits in
  // the spare word after the mbarrier (no static shared memory: the z3 tile
  // fills four CTAs' share of the SM exactly).
  unsigned &lean_nbf = *reinterpret_cast<unsigned *>(smem + SL::B0 + 2);
  if constexpr (LEAN) {
    if (tid == 0) {
      unsigned m = 0;
      const uint8_t *us = p.ustore[bi];
      for (int dzz = -1; dzz <= 1; dzz++)
        for (int dxx = -1; dxx <= 1; dxx++) {
          const int tx = tile_x + dxx, tz = tile_z + dzz;
          if (tx >= 0 && tx < p.ntx && tz >= 0 && tz < p.ntz && us[tz * p.ntx + tx]) m |= 1u << ((dzz + 1) * 3 + dxx + 1);
        }
      lean_nbf = m;
    }
  }

  // ---- phase 0: stage the tile (TMA) or the salinity ring, and the axis weights
  if (tid == 0) *qcount = 0;
  unsigned bar_a = 0;
  if constexpr (TMA) {
    bar_a = smem_u32(bar);
    if (tid == 0) mbar_init(bar_a, 1);
    __syncthreads();
    if (tid == 0) {
      if constexpr (RES) {
        // 16-bit boxes from x0 - 8 (= ox - 4), four FP32 macroscopic planes
        constexpr unsigned bytes = 2u * (unsigned)((9 + QS) * SL::E16) + 4u * (unsigned)(4 * SZ * RX);
        mbar_expect_tx(bar_a, bytes);
        tma_load_3d(smem_u32(smem + SL::H0), &tm[bi], ox - 4, oz, 0, bar_a);
        if constexpr (QS > 0) tma_load_3d(smem_u32(smem + SL::HG), &tm[2 + bi], ox - 4, oz, 0, bar_a);
        tma_load_3d(smem_u32(sS), &tm[4 + bi], ox, oz - 1, 0, bar_a);
      } else if constexpr (LEAN) {
        const bool need_mac = lean_nbf != 0;
        const unsigned bytes = 4u * (unsigned)(9 * NE + (need_mac ? 3 * SZ * RX : 0));
        mbar_expect_tx(bar_a, bytes);
        tma_load_3d(smem_u32(sf), &tm[bi], ox, oz, 0, bar_a);
        if (need_mac) tma_load_3d(smem_u32(sS), &tm[4 + bi], ox, oz - 1, 0, bar_a);
      } else {
        constexpr unsigned bytes = 4u * (unsigned)((9 + QS) * NE + 3 * SZ * RX);
        mbar_expect_tx(bar_a, bytes);
        tma_load_3d(smem_u32(sf), &tm[bi], ox, oz, 0, bar_a);
        if constexpr (QS > 0) tma_load_3d(smem_u32(sg), &tm[2 + bi], ox, oz, 0, bar_a);
        tma_load_3d(smem_u32(sS), &tm[4 + bi], ox, oz - 1, 0, bar_a);
      }
    }
  } else {
    for (int e = tid; e < SZ * RX; e += kThreads) {
      const int lz = e / RX, lx = e - lz * RX;
      const int gx = min(max(ox - RO + lx, 0), nx - 1), gz = min(max(oz - 1 + lz, 0), nz - 1);
      sS[e] = mac_in[(long long)gz * nx + gx];
    }
  }
  // the density-gradient factors 1/(z_{k+1} - z_{k-1} + dz/1000) of the
  // tile's rows, so the collision reads no table from memory (an evenly
  // spaced x axis uses its three constants, a stretched one its table)
  for (int e = tid; e < G::EZ; e += kThreads) {
    const int gz = min(max(oz + e, 0), nz - 1);
    sGI[e] = (p.gconst & 2) ? (gz == 0 ? p.giz3[0] : (gz == nz - 1 ? p.giz3[2] : p.giz3[1])) : __ldg(p.ginvz + gz);
  }
  if constexpr (G::AX >= 0) {
    const int NA = (G::AX == 0) ? nx : nz, oA = (G::AX == 0) ? ox : oz;
    for (int e = tid; e < 2 * WREC * NWA; e += kThreads) {
      const int la = e % NWA, r = e / NWA, m = r % WREC, s = r / WREC;
      const int gA = min(max(oA + la, 0), NA - 1);
      float v;
      if (m < G::NS) v = __ldg(p.wA + ((long long)s * NA + gA) * G::NS + m);
      else if (m == G::NS) v = __ldg(p.scin + (long long)s * NA + gA);
      else v = __ldg(p.scout + gA);
      sW[e] = v;
    }
    constexpr int NQ = G::NS + 1;
    for (int e = tid; e < 2 * NQ * NWA; e += kThreads) {
      const int la = e % NWA, r = e / NWA;  // r = s * NQ + q
      sC[e] = __ldg(p.wC + (long long)r * NA + min(max(oA + la, 0), NA - 1));
    }
  }
  if constexpr (TMA) {
    // every thread observes the barrier phase itself; the decision to go on
    // is made block-wide so that all threads leave together on a timeout
    const bool ok = __syncthreads_and(mbar_wait(bar_a, 0, kWaitLimit));
    if (!ok) {
      if (tid == 0) atomicOr(p.status, 4u);
      mbar_wait(bar_a, 0, kWaitLimit);  // let copies still in flight land before the CTA exits
      return;
    }
    // the box reads zeros outside the domain: give the ring's outside cells
    // their clamped (owner) salinity, as the ghosts carry it (the lean step
    // reads no salinity)
    if (!LEAN && (ox < 0 || ox + EX > nx || oz - 1 < 0 || oz - 1 + SZ > nz)) {
      for (int e = tid; e < SZ * RX; e += kThreads) {
        const int lz = e / RX, lx = e - lz * RX;
        const int gx = ox + lx, gz = oz - 1 + lz;
        if (gx >= 0 && gx < nx && gz >= 0 && gz < nz) continue;
        const int cx = min(max(gx, 0), nx - 1) - ox, cz = min(max(gz, 0), nz - 1) - (oz - 1);
        sS[e] = sS[cz * RX + cx];
      }
    }
  }
  __syncthreads();

  const float c = p.c, c2 = c * c, ic = 1.0f / c;
  const float itau = 1.0f / p.tau, omg = 1.0f - 1.0f / p.taus;
  const float ifs = p.inv_fscale, igs = p.inv_gscale;
  const float om_shear = 1.0f - itau;

  // ---- phase 1: collide tile + halo in shared memory
  for (int i = tid; i < G::NC; i += kThreads) {
    const int lz = i / G::CW, lx = G::CX0 + (i - lz * G::CW);
    const int gx = ox + lx, gz = oz + lz;
    if (gx < 0 || gx >= nx || gz < 0 || gz >= nz) continue;
    const int e = lz * EX + lx;              // tile slot
    const int rs = (lz + 1) * RX + lx + RO;  // ring slot
    float f[9], g[QS > 0 ? QS : 1], u, w, pr = 0.f;
    if constexpr (TMA) {
      if constexpr (RES) {
        const ST *h16 = reinterpret_cast<const ST *>(smem + SL::H0);
        const int e16 = lz * kTmaBoxX16 + lx + 4;  // the 16-bit box starts 4 columns left of the float tile
#pragma unroll
        for (int k = 0; k < 9; k++) f[k] = ld(h16, k * SL::E16 + e16, ifs);
        const ST *g16 = reinterpret_cast<const ST *>(smem + SL::HG);
#pragma unroll
        for (int k = 0; k < QS; k++) g[k] = ld(g16, k * SL::E16 + e16, igs);
        pr = sS[3 * SZ * RX + rs];
      } else {
#pragma unroll
        for (int k = 0; k < 9; k++) f[k] = sf[k * NE + e];
#pragma unroll
        for (int k = 0; k < QS; k++) g[k] = sg[k * NE + e];
      }
      if constexpr (LEAN) {
        // the owner tile's velocity planes, or the velocity its last step
        // formed without a body force: c j + F0 dt / 2 rho
        const int otx = lx < XO ? 0 : (lx >= XO + kTX ? 2 : 1), otz = lz < HZ ? 0 : (lz >= HZ + kTZ ? 2 : 1);
        if ((lean_nbf >> (otz * 3 + otx)) & 1u) {
          u = sS[SZ * RX + rs];
          w = sS[2 * SZ * RX + rs];
        } else {
          float p0, jx0, jz0;
          moments9(f, p0, jx0, jz0);
          const float h0 = __fdividef(p.hdt, rho_of(p.s_uni));
          u = fmaf(0.0f, h0, c * jx0);
          w = fmaf(-(p.s_uni * p.g_bouss_f), h0, c * jz0);
        }
      } else {
        u = sS[SZ * RX + rs];
        w = sS[2 * SZ * RX + rs];
      }
    } else {
      const long long ci = (long long)gz * nx + gx;
#pragma unroll
      for (int k = 0; k < 9; k++) f[k] = ld(f_in, k * N + ci, ifs);
#pragma unroll
      for (int k = 0; k < QS; k++) g[k] = ld(g_in, k * N + ci, igs);
      u = mac_in[N + ci];
      w = mac_in[2 * N + ci];
      if constexpr (RES) pr = mac_in[3 * N + ci];
    }
    const float S = LEAN ? p.s_uni : sS[rs], rho = rho_of(S);
    // p* (ref: collision.cu:244-246)
    if constexpr (!RES) {
#pragma unroll
      for (int k = 0; k < 9; k++) pr += f[k];
    }
    // force: buoyancy (salinity) or surface tension + weight (phase field),
    // plus the pressure gradient on the density (ref: collision.cu:57-112)
    const float pc = pr * c2 / 3.0f;
    const float gix = (p.gconst & 1) ? (gx == 0 ? p.gix3[0] : (gx == nx - 1 ? p.gix3[2] : p.gix3[1]))
                                     : __ldg(p.ginvx + gx);
    const float giz = sGI[lz];
    // (uniform S in the lean step: no density gradient)
    float Fx = LEAN ? 0.0f : -pc * ((rho_of(sS[rs + 1]) - rho_of(sS[rs - 1])) * gix);
    float Fz = LEAN ? 0.0f : -pc * ((rho_of(sS[rs + RX]) - rho_of(sS[rs - RX])) * giz);
    float dpx = 0.f, dpz = 0.f;  // grad(phi) (phase field)
    if constexpr (PHYS == 1) {
      // chemical potential of the double well, mu = 4 beta phi (phi - 1)(phi - 1/2)
      // - kappa lap(phi), beta = 12 sigma / W, kappa = 3 sigma W / 2; the
      // Laplacian divides by the cell's own dx^2 and dz^2 (ref: collision.cu:65-76)
      const float Sxp = sS[rs + 1], Sxm = sS[rs - 1], Szp = sS[rs + RX], Szm = sS[rs - RX];
      dpx = (Sxp - Sxm) * gix;
      dpz = (Szp - Szm) * giz;
      const float lap = (Sxp - 2.0f * S + Sxm) * __ldg(p.ilx2 + gx) + (Szp - 2.0f * S + Szm) * __ldg(p.ilz2 + gz);
      const float mu = p.pf_beta4 * S * (S - 1.0f) * (S - 0.5f) - p.pf_kap * lap;
      Fx += mu * dpx;
      Fz += mu * dpz - rho * p.grav;  // the mixture's weight (Boussi_flag off)
    } else {
      Fz -= S * p.g_bouss_f;  // Boussinesq buoyancy of the salinity
    }
    if (ibt) {  // immersed-boundary force density of the previous coupled step
      const long long ci = (long long)gz * nx + gx;
      Fx += p.fext[ci];
      Fz += p.fext[N + ci];
    }
    const float uc = u * ic, wc = w * ic;
    const float usq = uc * uc + wc * wc;
    // forcing term Fk_k = w_k (e_k . F) fden (ref: collision.cu:102-110)
    const float fden = __fdividef(p.fk3, rho);
    if (p.mrt == 2) {
      // MRT with unit non-shear rates (the reference's S file): the
      // non-shear moments relax to equilibrium in one step, so
      //   f*_k = feq_k + Fk_k / 2 + (1 - 1/tau) (Minv_s M_s d)_k,
      //   d = f - feq + Fk/2 (ref: collision.cu:115-150),
      // whose shear moments reduce to (Lallemand-Luo rows 7, 8)
      //   p_xx = (f1 + f3 - f2 - f4) - (u^2 - w^2)/c^2, p_xz = (f5 + f7 - f6 - f8) - u w/c^2
      // (the forcing parts cancel pairwise); feq + Fk/2 is formed per
      // opposite pair from A = p* - 1.5 u^2 + 4.5 (e.u)^2, B = 3 e.u + e.F fden/2.
      // (16-bit storage holds f - feq already, whose shear sums are these)
      float o[9];
      collide_mrt2<RES>(f, pr, uc, wc, fden, Fx, Fz, om_shear, o);
#pragma unroll
      for (int k = 0; k < 9; k++) sf[k * NE + e] = o[k];
    } else {
      // equilibrium (ref: collision.cu:3-14), d = f - feq + Fk/2; d goes to
      // shared memory (this cell's own slots) so that only the outputs stay
      // in registers while the 9x9 operator is applied
      auto feq_of = [&](int k) {
        const float eu = (ex(k) ? ex(k) * uc : 0.f) + (ez(k) ? ez(k) * wc : 0.f);
        return w9(k) * (pr + 3.0f * eu + 4.5f * eu * eu - 1.5f * usq);
      };
      if constexpr (RES) {
        const float u2 = rstore::usq(uc, wc);
#pragma unroll
        for (int k = 0; k < 9; k++) f[k] += rstore::feq(k, pr, uc, wc, u2);
      }
      auto fk_of = [&](int k) {
        const float ef = (ex(k) ? ex(k) * Fx : 0.f) + (ez(k) ? ez(k) * Fz : 0.f);
        return w9(k) * ef * fden;
      };
#pragma unroll
      for (int k = 0; k < 9; k++) sf[k * NE + e] = f[k] - feq_of(k) + 0.5f * fk_of(k);
      if (p.mrt == 1) {
        // f* = f - (MM + Minv_s M_s / tau) d + Fk (ref: collision.cu:115-150),
        // with f = d + feq - Fk/2
        float m7 = 0.f, m8 = 0.f;
#pragma unroll
        for (int k = 0; k < 9; k++) {
          m7 += p.Ms[k] * sf[k * NE + e];
          m8 += p.Ms[9 + k] * sf[k * NE + e];
        }
        // general relaxation rates: the 9x9 product runs as a rolled loop
        // over d's components so that only the nine outputs stay live
        float o[9];
#pragma unroll
        for (int a = 0; a < 9; a++) o[a] = 0.f;
#pragma unroll 1
        for (int k = 0; k < 9; k++) {
          const float dk = sf[k * NE + e];
#pragma unroll
          for (int a = 0; a < 9; a++) o[a] += p.MM[a * 9 + k] * dk;
        }
#pragma unroll
        for (int a = 0; a < 9; a++) {
          const float acc = o[a] + (p.Mis[a * 2] * m7 + p.Mis[a * 2 + 1] * m8) * itau;
          o[a] = sf[a * NE + e] + feq_of(a) + 0.5f * fk_of(a) - acc;
        }
#pragma unroll
        for (int a = 0; a < 9; a++) sf[a * NE + e] = o[a];
      } else {
        // BGK with forcing (ref: collision.cu:151-165): f* = f - d/tau + Fk
#pragma unroll
        for (int k = 0; k < 9; k++) {
          const float d = sf[k * NE + e];
          sf[k * NE + e] = d + feq_of(k) + 0.5f * fk_of(k) - d * itau;
        }
      }
    }
    if constexpr (PHYS == 1) {
      // conservative Allen-Cahn collision (ref: collision.cu:190-223):
      //   g*_k = g_k - (g_k - geq_k)/tau_phi + (tau_phi - 1/2)/tau_phi Fp_k,
      //   Fp_k = dt w_k [(1 - 4 (phi - 1/2)^2)/W c e_k.grad(phi)/|grad(phi)|
      //                  + 3 e_k.d(phi u)/dt / c] = w_k e_k.V
      // with d(phi u)/dt against the previous step's phi u kept in obuf.
      const float *__restrict__ old_in = p.obuf[bi];
      const long long ci = (long long)gz * nx + gx;
      const float nbx = (S * u - old_in[ci]) / p.dt, nbz = (S * w - old_in[N + ci]) / p.dt;
      const float nrm = sqrtf(dpx * dpx + dpz * dpz + 1e-8f);
      const float sh = S - 0.5f, A = p.dt * (1.0f - 4.0f * sh * sh) * p.pf_invw * c / nrm, B = 3.0f * p.dt * ic;
      const float Vx = A * dpx + B * nbx, Vz = A * dpz + B * nbz;
      const float u2 = rstore::usq(uc, wc);
#pragma unroll
      for (int k = 0; k < QS; k++) {
        const float geq = QS == 5 ? rstore::geq5(k, S, uc, wc) : rstore::geq9(k, S, uc, wc, u2);
        const float r = RES ? g[k] : g[k] - geq;  // 16-bit storage holds g - geq already
        const float ev = (ex(k) ? ex(k) * Vx : 0.f) + (ez(k) ? ez(k) * Vz : 0.f);
        sg[k * NE + e] = geq + omg * r + p.pf_lam * wq<QS>(k) * ev;
      }
      // this step's phi u for the next one (each interior cell by its own tile)
      if (lx >= XO && lx < XO + kTX && lz >= HZ && lz < HZ + kTZ) {
        float *__restrict__ old_out = p.obuf[bo];
        old_out[ci] = S * u;
        old_out[N + ci] = S * w;
      }
    } else if constexpr (QS == 5) {
      // regularised D2Q5 collision (ref: collision.cu:167-188 on the D2Q5
      // lattice, linear equilibrium w S (1 + 3 e.u/c)): the first moment of
      // g - geq is j = (g1 - g3, g2 - g4) - S u/c, and
      //   g*_k = w_k (S + 3 e_k . (S u/c + (1 - 1/tau_s) j)).
      const float jx = RES ? g[1] - g[3] : (g[1] - g[3]) - S * uc;
      const float jz = RES ? g[2] - g[4] : (g[2] - g[4]) - S * wc;
      const float ax3 = 3.0f * fmaf(omg, jx, S * uc), az3 = 3.0f * fmaf(omg, jz, S * wc);
      sg[e] = w5(0) * S;
      sg[1 * NE + e] = w5(1) * (S + ax3);
      sg[3 * NE + e] = w5(3) * (S - ax3);
      sg[2 * NE + e] = w5(2) * (S + az3);
      sg[4 * NE + e] = w5(4) * (S - az3);
    } else if constexpr (QS == 9) {
      // regularised scalar collision on the reference's Q9 scalar lattice (ref: collision.cu:167-188)
      if constexpr (RES) {
        const float u2 = rstore::usq(uc, wc);
#pragma unroll
        for (int k = 0; k < QS; k++) g[k] += rstore::geq9(k, S, uc, wc, u2);
      }
      float ge[QS], jx = 0.f, jz = 0.f;
#pragma unroll
      for (int k = 0; k < QS; k++) {
        const float eu = (ex(k) ? ex(k) * uc : 0.f) + (ez(k) ? ez(k) * wc : 0.f);
        ge[k] = wq<QS>(k) * S * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * usq);
        const float ne = g[k] - ge[k];
        if (ex(k)) jx += ex(k) * ne;
        if (ez(k)) jz += ez(k) * ne;
      }
#pragma unroll
      for (int k = 0; k < QS; k++) {
        const float ej = (ex(k) ? ex(k) * jx : 0.f) + (ez(k) ? ez(k) * jz : 0.f);
        sg[k * NE + e] = ge[k] + omg * (wq<QS>(k) * 3.0f * ej);
      }
    }
    if constexpr (TMA) {
      // u, w of this slot have been read; the slot keeps the force for phase 2
      sS[SZ * RX + rs] = Fx;
      sS[2 * SZ * RX + rs] = Fz;
    } else if (lx >= XO && lx < XO + kTX && lz >= HZ && lz < HZ + kTZ) {
      const int ii = (lz - HZ) * kTX + (lx - XO);
      sF[ii] = Fx;
      sF[kTX * kTZ + ii] = Fz;
    }
  }
  __syncthreads();

  // ---- phase 2: interpolated streaming, moments, store
  auto L = [&](int gx, int gz) { return (gz - oz) * EX + (gx - ox); };
  const int NA = (G::AX == 0) ? nx : nz;
  // general path (cells next to a wall): clamped nodes, mirrored partners,
  // bounce-back / slip ghosts
  auto interp = [&](const float *arr, int k, int s, int gx, int gz) -> float {
    const int gA = (G::AX == 0) ? gx : gz, la = gA - ((G::AX == 0) ? ox : oz);
    float acc = 0.f;
#pragma unroll
    for (int m = 0; m < G::NS; m++) {
      const int off = (s == 0 ? 1 : -1) * (m - G::NS / 2);
      const int q = min(max(gA + off, 0), NA - 1);
      const float v = (G::AX == 0) ? arr[k * NE + L(q, gz)] : arr[k * NE + L(gx, q)];
      acc += sW[(s * WREC + m) * NWA + la] * v;
    }
    return acc;
  };
  auto ftmp = [&](const float *arr, int k, int gx, int gz) -> float {
    if constexpr (G::AX < 0) {
      return arr[k * NE + L(gx, gz)];
    } else {
      const int a = (G::AX == 0) ? ex(k) : ez(k);
      if (a == 0) return arr[k * NE + L(gx, gz)];
      const int s = a > 0 ? 0 : 1;
      const int gA = (G::AX == 0) ? gx : gz, la = gA - ((G::AX == 0) ? ox : oz);
      const float fin = interp(arr, k, s, gx, gz) * sW[(s * WREC + G::NS) * NWA + la];
      const int gP = gA + a;
      if (gP >= 0 && gP < NA) {
        const int px = (G::AX == 0) ? gP : gx, pz = (G::AX == 0) ? gz : gP;
        const float fout = interp(arr, k, s, px, pz) * sW[(s * WREC + G::NS + 1) * NWA + la + a];
        return arr[k * NE + L(px, pz)] + (fin - fout);
      } else {
        const int km = (G::AX == 0) ? mirx(k) : mirz(k);
        const float fout = interp(arr, km, 1 - s, gx, gz) * sW[(s * WREC + G::NS + 1) * NWA + la];
        return arr[km * NE + L(gx, gz)] + (fin - fout);
      }
    }
  };
  auto pull = [&](const float *arr, int k, int gx, int gz, int cls, const int8_t *slipB, const int8_t *slipK) -> float {
    const int sx = gx - ex(k), sz = gz - ez(k);
    if (sx >= 0 && sx < nx && sz >= 0 && sz < nz) return ftmp(arr, k, sx, sz);
    if (p.wall == IPCU_WALL_BB) return ftmp(arr, kinv(k), gx, gz);
    const int nb = slipB[cls * 9 + k], kk = slipK[cls * 9 + k];
    return ftmp(arr, kk, gx + ex(nb), gz + ez(nb));
  };

  // moments and store of one cell from its streamed populations
  auto finish = [&](int e, long long ci, int rc, const float (&fv)[9], const float (&gv)[QS > 0 ? QS : 1]) {
    float pr, jx, jz;
    moments9(fv, pr, jx, jz);
    float S = 0.f;
    if constexpr (QS > 0) {
#pragma unroll
      for (int k = 0; k < QS; k++) S += gv[k];
    } else if constexpr (LEAN) {
      S = p.s_uni;
    } else {
      S = sS[rc];
    }
    // moments (ref: collision.cu:244-254)
    const float h = __fdividef(p.hdt, rho_of(S));
    const float Fx = TMA ? sS[SZ * RX + rc] : sF[e], Fz = TMA ? sS[2 * SZ * RX + rc] : sF[kTX * kTZ + e];
    const float ux = fmaf(Fx, h, c * jx), uz = fmaf(Fz, h, c * jz);
    if constexpr (RES) {
      // deviations from the equilibrium of the moments stored beside them
      const float ucn = ux * ic, wcn = uz * ic, u2 = rstore::usq(ucn, wcn);
      float amax = 0.f;
#pragma unroll
      for (int k = 0; k < 9; k++) {
        const float r = fv[k] - rstore::feq(k, pr, ucn, wcn, u2);
        amax = fmaxf(amax, fabsf(r) * p.fscale);
        st(f_out, k * N + ci, r, p.fscale);
      }
#pragma unroll
      for (int k = 0; k < QS; k++) {
        const float r = gv[k] - (QS == 5 ? rstore::geq5(k, S, ucn, wcn) : rstore::geq9(k, S, ucn, wcn, u2));
        amax = fmaxf(amax, fabsf(r) * p.gscale);
        st(g_out, k * N + ci, r, p.gscale);
      }
      mac_out[3 * N + ci] = pr;
      if (amax > p.store_max) atomicOr(p.status, 2u);  // beyond the 16-bit range
    } else {
#pragma unroll
      for (int k = 0; k < 9; k++) st(f_out, k * N + ci, fv[k], 1.0f);
#pragma unroll
      for (int k = 0; k < QS; k++) st(g_out, k * N + ci, gv[k], 1.0f);
    }
    if constexpr (LEAN) {
      // velocity planes only where a body force acted (recomputable elsewhere)
      if (ibt) {
        mac_out[N + ci] = ux;
        mac_out[2 * N + ci] = uz;
      }
    } else {
      mac_out[ci] = S;
      mac_out[N + ci] = ux;
      mac_out[2 * N + ci] = uz;
    }
    if (!(isfinite(ux) && isfinite(uz) && isfinite(S) && isfinite(pr))) atomicOr(p.status, 1u);
  };
  // general path: clamped stencils, ghost rules (cells next to a wall)
  auto general = [&](int e) {
    const int iz = e / kTX, ix = e - iz * kTX;
    const int gx = x0 + ix, gz = z0 + iz;
    const long long ci = (long long)gz * nx + gx;
    const int rc = (iz + HZ + 1) * RX + ix + XO + RO;
    float fv[9], gv[QS > 0 ? QS : 1];
    const int cls = (gx == 0 ? 1 : 0) | (gx == nx - 1 ? 2 : 0) | (gz == 0 ? 4 : 0) | (gz == nz - 1 ? 8 : 0);
#pragma unroll
    for (int k = 0; k < 9; k++) fv[k] = pull(sf, k, gx, gz, cls, p.slipB9, p.slipK9);
#pragma unroll
    for (int k = 0; k < QS; k++)
      gv[k] = pull(sg, k, gx, gz, cls, QS == 9 ? p.slipB9 : p.slipB5, QS == 9 ? p.slipK9 : p.slipK5);
    finish(e, ci, rc, fv, gv);
  };

  for (int e = tid; e < kTX * kTZ; e += kThreads) {
    const int iz = e / kTX, ix = e - iz * kTX;
    const int gx = x0 + ix, gz = z0 + iz;
    if (gx >= nx || gz >= nz) continue;
    const int gA = G::AX == 0 ? gx : gz, gB = G::AX == 0 ? gz : gx, NB = G::AX == 0 ? nz : nx;
    // interior: every source and stencil node inside the box
    const bool fast = (G::AX < 0) ? (gx >= 1 && gx <= nx - 2 && gz >= 1 && gz <= nz - 2)
                                  : (gA >= G::H && gA <= NA - 1 - G::H && gB >= 1 && gB <= NB - 2);
    if (!fast) {
      const int slot = atomicAdd(qcount, 1);
      if (slot < kQueue) queue[slot] = e;
      else general(e);  // queue full (tiles of very small boxes)
      continue;
    }
    const long long ci = (long long)gz * nx + gx;
    const int lc = (iz + HZ) * EX + ix + XO;
    const int rc = (iz + HZ + 1) * RX + ix + XO + RO;  // ring slot of the cell
    const int la = G::AX == 0 ? ix + XO : iz + HZ;
    float fv[9], gv[QS > 0 ? QS : 1];
    float W[2][G::NS + 1];
    if constexpr (G::AX >= 0) {
#pragma unroll
      for (int sidx = 0; sidx < 2; sidx++)
#pragma unroll
        for (int q = 0; q <= G::NS; q++) W[sidx][q] = sC[(sidx * (G::NS + 1) + q) * NWA + la];
    }
    fv[0] = Fast<GEO, TMA, 0>::pull(sf, lc, W);
    fv[1] = Fast<GEO, TMA, 1>::pull(sf, lc, W);
    fv[2] = Fast<GEO, TMA, 2>::pull(sf, lc, W);
    fv[3] = Fast<GEO, TMA, 3>::pull(sf, lc, W);
    fv[4] = Fast<GEO, TMA, 4>::pull(sf, lc, W);
    fv[5] = Fast<GEO, TMA, 5>::pull(sf, lc, W);
    fv[6] = Fast<GEO, TMA, 6>::pull(sf, lc, W);
    fv[7] = Fast<GEO, TMA, 7>::pull(sf, lc, W);
    fv[8] = Fast<GEO, TMA, 8>::pull(sf, lc, W);
    if constexpr (QS > 0) {
      gv[0] = Fast<GEO, TMA, 0>::pull(sg, lc, W);
      gv[1] = Fast<GEO, TMA, 1>::pull(sg, lc, W);
      gv[2] = Fast<GEO, TMA, 2>::pull(sg, lc, W);
      gv[3] = Fast<GEO, TMA, 3>::pull(sg, lc, W);
      gv[4] = Fast<GEO, TMA, 4>::pull(sg, lc, W);
      if constexpr (QS == 9) {
        gv[5] = Fast<GEO, TMA, 5>::pull(sg, lc, W);
        gv[6] = Fast<GEO, TMA, 6>::pull(sg, lc, W);
        gv[7] = Fast<GEO, TMA, 7>::pull(sg, lc, W);
        gv[8] = Fast<GEO, TMA, 8>::pull(sg, lc, W);
      }
    }
    finish(e, ci, rc, fv, gv);
  }
  // the queued wall cells, spread over the CTA's threads
  __syncthreads();
  const int nq = min(*qcount, kQueue);
  for (int j = tid; j < nq; j += kThreads) general(queue[j]);
  if constexpr (LEAN) {
    if (tid == 0) p.ustore[bo][tile_z * p.ntx + tile_x] = ibt ? 1 : 0;
  }
}

// Resident CTAs per SM the single-run kernel's registers are sized for. The
// FP32 TMA flow-only tile (36 KB of shared memory) fits 48 registers with a
// 4-byte spill and runs 5 CTAs per SM: the step is bound by the latency of
// staging a tile, and a fifth CTA hides more of it (+4.7 % MLUPS on an
// 800 x 3000 box). The scalar lattices spill 30-70 bytes at 48 registers
// and stay at 4.
template <class ST, int QS, bool TMA>
constexpr int step_min_blocks() {
  return (QS == 0 && TMA && sizeof(ST) == 4) ? 5 : kMinBlocks;
}

template <class ST, int QS, int GEO, bool TMA, int PHYS, bool LEAN = false>
__global__ void __launch_bounds__(kThreads, step_min_blocks<ST, QS, TMA>())
    step_kernel(const __grid_constant__ Params p) {
  extern __shared__ __align__(128) float smem[];
  step_tile<ST, QS, GEO, TMA, PHYS, LEAN>(p, 0, blockIdx.x, blockIdx.y, smem, p.tm_f);
}

// The batched kernel copies each work item's parameters (past the tensor
// maps, which register staging does not use) into shared memory, so that
// the tile reads them as shared loads rather than global ones.
// TMA: stage with each simulation's tensor maps, read in place from the
// global parameter array (all simulations of the launch have them).
template <class ST, int QS, int GEO, bool TMA, int PHYS>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
    step_kernel_batched(const Params *__restrict__ ps, const WorkItem *__restrict__ work, int nwork, int parity) {
  extern __shared__ __align__(128) float smem[];
  __shared__ Params sp;
  constexpr int kSkip = offsetof(Params, tma) / 4, kWords = sizeof(Params) / 4;
  int cur_sim = -1;
  for (int i = blockIdx.x; i < nwork; i += gridDim.x) {
    const WorkItem w = work[i];
    if (w.sim != cur_sim) {  // consecutive items of one simulation share the copy
      const uint32_t *src = reinterpret_cast<const uint32_t *>(ps + w.sim);
      uint32_t *dst = reinterpret_cast<uint32_t *>(&sp);
      for (int j = kSkip + threadIdx.x; j < kWords; j += kThreads) dst[j] = src[j];
      if (TMA && threadIdx.x < 6) tensormap_acquire(ps[w.sim].tm_f + threadIdx.x);
      cur_sim = w.sim;
      __syncthreads();
    }
    step_tile<ST, QS, GEO, TMA, PHYS>(sp, parity, w.tx, w.tz, smem, ps[w.sim].tm_f);
    __syncthreads();  // the next item reuses shared memory
  }
  // Launched as a programmatic dependent of a batch of body updates, the
  // kernel ends only after them, so that whatever follows it on the stream
  // follows them too (a no-op after a plain launch).
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Launch that may begin while the previous kernel on the stream (a body's
// update) still runs; the kernel orders itself with griddepcontrol.wait.
template <class K, class... A>
int launch_pdl(K kernel, dim3 grid, size_t smem, cudaStream_t s, A... args) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.gridDim = grid;
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return status_from_cuda(cudaLaunchKernelEx(&cfg, kernel, args...));
}

// pdl: the previous launch on the stream is a batch of body updates, which
// the flagged tiles wait for (griddepcontrol.wait) while the rest run.
template <class ST, int QS, int GEO, bool TMA, int PHYS>
int launch_b1(const Params *ps, const WorkItem *work, int nwork, int parity, int grid, cudaStream_t s, bool prep,
              bool pdl) {
  constexpr size_t sm = smem_bytes<QS, GEO, TMA, (int)sizeof(ST)>();
  if (prep)
    return status_from_cuda(cudaFuncSetAttribute(step_kernel_batched<ST, QS, GEO, TMA, PHYS>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  if (nwork <= 0) return IPCU_OK;
  if (pdl) return launch_pdl(step_kernel_batched<ST, QS, GEO, TMA, PHYS>, dim3(grid), sm, s, ps, work, nwork, parity);
  step_kernel_batched<ST, QS, GEO, TMA, PHYS><<<grid, kThreads, sm, s>>>(ps, work, nwork, parity);
  return status_from_cuda(cudaGetLastError());
}
// tma: every simulation of the launch has tensor maps
template <class ST, int QS, int GEO, int PHYS>
int launch_b(const Params *ps, const WorkItem *work, int nwork, int parity, int grid, cudaStream_t s, bool prep,
             bool tma, bool pdl) {
  if (prep) {
    const int st = launch_b1<ST, QS, GEO, false, PHYS>(ps, work, nwork, parity, grid, s, true, false);
    return st ? st : launch_b1<ST, QS, GEO, true, PHYS>(ps, work, nwork, parity, grid, s, true, false);
  }
  if (tma) return launch_b1<ST, QS, GEO, true, PHYS>(ps, work, nwork, parity, grid, s, false, pdl);
  return launch_b1<ST, QS, GEO, false, PHYS>(ps, work, nwork, parity, grid, s, false, pdl);
}

template <class ST, int QS, int PHYS>
int launch_bg(const Params *ps, const WorkItem *work, int nwork, int parity, int geo, int grid, cudaStream_t s,
              bool prep, bool tma, bool pdl) {
  switch (geo) {
    case IPCU_GEO_UNIFORM: return launch_b<ST, QS, IPCU_GEO_UNIFORM, PHYS>(ps, work, nwork, parity, grid, s, prep, tma, pdl);
    case IPCU_GEO_X5: return launch_b<ST, QS, IPCU_GEO_X5, PHYS>(ps, work, nwork, parity, grid, s, prep, tma, pdl);
    case IPCU_GEO_X3: return launch_b<ST, QS, IPCU_GEO_X3, PHYS>(ps, work, nwork, parity, grid, s, prep, tma, pdl);
    case IPCU_GEO_Z5: return launch_b<ST, QS, IPCU_GEO_Z5, PHYS>(ps, work, nwork, parity, grid, s, prep, tma, pdl);
    case IPCU_GEO_Z3: return launch_b<ST, QS, IPCU_GEO_Z3, PHYS>(ps, work, nwork, parity, grid, s, prep, tma, pdl);
  }
  return IPCU_ERR_UNSUPPORTED;
}

template <class ST, int QS, int GEO, bool TMA, int PHYS, bool LEAN = false>
int launch_t1(const Params &p, cudaStream_t s, bool prepare_only) {
  constexpr size_t sm = smem_bytes<QS, GEO, TMA, (int)sizeof(ST)>();
  if (prepare_only) {  // once per sim, outside any stream capture
    return status_from_cuda(cudaFuncSetAttribute(step_kernel<ST, QS, GEO, TMA, PHYS, LEAN>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  }
  dim3 grid((p.nx + kTX - 1) / kTX, (p.nz + kTZ - 1) / kTZ);
  if (p.fext) return launch_pdl(step_kernel<ST, QS, GEO, TMA, PHYS, LEAN>, grid, sm, s, p);
  step_kernel<ST, QS, GEO, TMA, PHYS, LEAN><<<grid, kThreads, sm, s>>>(p);
  return status_from_cuda(cudaGetLastError());
}

// TMA staging for FP32 storage when the host built the tensor maps (p.tma);
// the lean flow-only step where the host enabled it (p.lean)
template <class ST, int QS, int GEO, int PHYS>
int launch_t(const Params &p, cudaStream_t s, bool prepare_only) {
  if constexpr (QS == 0 && PHYS == 0 && sizeof(ST) == 4) {
    if (p.tma && (p.lean || prepare_only)) {
      const int st = launch_t1<ST, QS, GEO, true, PHYS, true>(p, s, prepare_only);
      if (!prepare_only || st) return st;
    }
  }
  if (p.tma) return launch_t1<ST, QS, GEO, true, PHYS>(p, s, prepare_only);
  return launch_t1<ST, QS, GEO, false, PHYS>(p, s, prepare_only);
}

template <class ST, int QS, int PHYS>
int launch_g(const Params &p, int geo, cudaStream_t s, bool prep) {
  switch (geo) {
    case IPCU_GEO_UNIFORM: return launch_t<ST, QS, IPCU_GEO_UNIFORM, PHYS>(p, s, prep);
    case IPCU_GEO_X5: return launch_t<ST, QS, IPCU_GEO_X5, PHYS>(p, s, prep);
    case IPCU_GEO_X3: return launch_t<ST, QS, IPCU_GEO_X3, PHYS>(p, s, prep);
    case IPCU_GEO_Z5: return launch_t<ST, QS, IPCU_GEO_Z5, PHYS>(p, s, prep);
    case IPCU_GEO_Z3: return launch_t<ST, QS, IPCU_GEO_Z3, PHYS>(p, s, prep);
  }
  return IPCU_ERR_UNSUPPORTED;
}

// Entry points of one instantiation unit: storage ST, scalar physics PHYS
// (the phase field needs a scalar lattice, q = 5 or 9).
template <class ST, int PHYS>
int launch_q(const Params &p, int qs, int geo, cudaStream_t s, bool prep) {
  if (qs == 0) {
    if constexpr (PHYS == 0) return launch_g<ST, 0, 0>(p, geo, s, prep);
    return IPCU_ERR_UNSUPPORTED;
  }
  if (qs == 5) return launch_g<ST, 5, PHYS>(p, geo, s, prep);
  if (qs == 9) return launch_g<ST, 9, PHYS>(p, geo, s, prep);
  return IPCU_ERR_UNSUPPORTED;
}
template <class ST, int PHYS>
int launch_bq(const Params *ps, const WorkItem *work, int nwork, int parity, int qs, int geo, int grid,
              cudaStream_t s, bool prep, bool tma, bool pdl) {
  if (qs == 0) {
    if constexpr (PHYS == 0) return launch_bg<ST, 0, 0>(ps, work, nwork, parity, geo, grid, s, prep, tma, pdl);
    return IPCU_ERR_UNSUPPORTED;
  }
  if (qs == 5) return launch_bg<ST, 5, PHYS>(ps, work, nwork, parity, geo, grid, s, prep, tma, pdl);
  if (qs == 9) return launch_bg<ST, 9, PHYS>(ps, work, nwork, parity, geo, grid, s, prep, tma, pdl);
  return IPCU_ERR_UNSUPPORTED;
}
#define IPCU_F2D_INSTANTIATE(ST, NAME, PHYS)                                                              \
  int launch_##NAME(const Params &p, int qs, int geo, cudaStream_t s, bool prep) {                        \
    return launch_q<ST, PHYS>(p, qs, geo, s, prep);                                                       \
  }                                                                                                       \
  int launch_batched_##NAME(const Params *ps, const WorkItem *work, int nwork, int parity, int qs, int geo, \
                            int grid, cudaStream_t s, bool prep, bool tma, bool pdl) {                    \
    return launch_bq<ST, PHYS>(ps, work, nwork, parity, qs, geo, grid, s, prep, tma, pdl);                \
  }

}  // namespace f2d
}  // namespace ipcu
