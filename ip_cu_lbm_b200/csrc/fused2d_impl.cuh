// Fused collide-and-stream step for 2-D boxes (D2Q9 flow in the x-z plane +
// D2Q5 or Q9 salinity), the B200 path of the reference's per-step chain
//   equ_f -> Force -> col_f_MRT -> IP_process(f) -> col_g_reg -> IP_process(g)
//   -> update_scalar -> update_rho -> set_wall_rho
// (ref: LockExchange/LockExchange.cu:220-236; kernels in function/collision.cu,
// function/adv.cu, function/set_bound.cu, function/propagation.cu).
//
// One launch per time step. A CTA owns a kTX x kTZ tile; phase 0 stages the
// salinity/density ring and the tile's axis weights, phase 1 collides the
// tile plus its streaming halo (HX cells along x, HZ along z) straight from
// HBM into shared memory, phase 2 evaluates the reference's conservative
// interpolated streaming for the interior from shared memory, forms the
// moments and writes the new state. Every stored value is read from HBM once
// and written once per step (halo re-reads hit L2). Storage is
// structure-of-arrays, x fastest, so each warp touches 128-byte lines.
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

#include <type_traits>

#include "fused2d.cuh"
#include "ipcu_common.cuh"

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

template <int GEO>
struct Geo {
  static constexpr int AX = (GEO == IPCU_GEO_X5 || GEO == IPCU_GEO_X3) ? 0 : ((GEO == IPCU_GEO_Z5 || GEO == IPCU_GEO_Z3) ? 1 : -1);
  static constexpr int NS = (GEO == IPCU_GEO_X5 || GEO == IPCU_GEO_Z5) ? 5 : ((GEO == IPCU_GEO_X3 || GEO == IPCU_GEO_Z3) ? 3 : 1);
  static constexpr int H = NS == 5 ? 3 : (NS == 3 ? 2 : 1);
  static constexpr int HX = AX == 0 ? H : 1;
  static constexpr int HZ = AX == 1 ? H : 1;
  static constexpr int EX = kTX + 2 * HX, EZ = kTZ + 2 * HZ, NE = EX * EZ;
  static constexpr int SX = EX + 2, SZ = EZ + 2;  // density ring for the gradient
  static constexpr int NWA = AX == 0 ? EX : (AX == 1 ? EZ : 0);
  static constexpr int WREC = NS + 2;             // NS weights, fin scale, fout scale
};

template <class ST, int QS, int GEO>
constexpr size_t smem_bytes() {
  using G = Geo<GEO>;
  return sizeof(float) * ((9 + QS) * G::NE + 2 * G::SX * G::SZ + 2 * kTX * kTZ + 2 * G::NWA * G::WREC +
                          2 * G::NWA * (G::NS + 1));
}

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

// Clamp-free pull for an interior cell: lc is the cell's local index; W
// holds the combined flux weights of its axis position for both signs of
// the axis velocity (see axis_tables on the host), so the flux form is one
// dot product over the NS+1 nodes around the source cell.
template <int GEO, int K>
struct Fast {
  using G = Geo<GEO>;
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
// the kernel's constant bank) and the batched kernel (parameters in global memory).
template <class ST, int QS, int GEO>
__device__ __forceinline__ void step_tile(const Params &p, int parity, int tile_x, int tile_z, float *smem) {
  using G = Geo<GEO>;
  constexpr int HX = G::HX, HZ = G::HZ, EX = G::EX, NE = G::NE, SX = G::SX, SZ = G::SZ;
  constexpr int NWA = G::NWA, WREC = G::WREC;
  float *sf = smem;                       // [9][EZ][EX] post-collision f
  float *sg = sf + 9 * NE;                // [QS][EZ][EX] post-collision g
  float *sS = sg + QS * NE;               // [SZ][SX] salinity
  float *sR = sS + SZ * SX;               // [SZ][SX] density
  float *sF = sR + SZ * SX;               // [2][kTZ][kTX] interior force
  float *sW = sF + 2 * kTX * kTZ;         // [2][WREC][NWA] axis weights
  float *sC = sW + 2 * WREC * NWA;        // [2][NS+1][NWA] combined interior weights

  const int nx = p.nx, nz = p.nz;
  const long long N = (long long)nx * nz;
  const int x0 = tile_x * kTX, z0 = tile_z * kTZ;
  const int ox = x0 - HX, oz = z0 - HZ;  // global coords of local (0,0)
  const int tid = threadIdx.x;
  const int bi = p.cur ^ parity, bo = bi ^ 1;
  const ST *__restrict__ f_in = static_cast<const ST *>(p.fbuf[bi]);
  const ST *__restrict__ g_in = static_cast<const ST *>(p.gbuf[bi]);
  ST *__restrict__ f_out = static_cast<ST *>(p.fbuf[bo]);
  ST *__restrict__ g_out = static_cast<ST *>(p.gbuf[bo]);
  const float *__restrict__ mac_in = p.mbuf[bi];
  float *__restrict__ mac_out = p.mbuf[bo];

  // density as the reference forms it: float base plus a double salinity
  // term, rounded once (ref: collision.cu:251)
  const float rho0 = p.rhoL + (p.rhoH - p.rhoL) * p.phi;

  // ---- phase 0: stage the salinity/density ring and the axis weights
  for (int e = tid; e < SX * SZ; e += kThreads) {
    const int lz = e / SX, lx = e - lz * SX;
    const int gx = min(max(ox - 1 + lx, 0), nx - 1), gz = min(max(oz - 1 + lz, 0), nz - 1);
    const float S = mac_in[(long long)gz * nx + gx];
    sS[e] = S;
    sR[e] = (float)((double)rho0 + (double)S * p.rho_sal);
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
  __syncthreads();

  const float c = p.c, c2 = c * c, ic = 1.0f / c, dt = p.dt;
  const float itau = 1.0f / p.tau, omg = 1.0f - 1.0f / p.taus;
  const float ifs = p.inv_fscale, igs = p.inv_gscale;
  const float om_shear = 1.0f - itau;

  // ---- phase 1: collide tile + halo into shared memory
  for (int e = tid; e < NE; e += kThreads) {
    const int lz = e / EX, lx = e - lz * EX;
    const int gx = ox + lx, gz = oz + lz;
    if (gx < 0 || gx >= nx || gz < 0 || gz >= nz) continue;
    float f[9], g[QS > 0 ? QS : 1];
    const long long ci = (long long)gz * nx + gx;
#pragma unroll
    for (int k = 0; k < 9; k++) f[k] = ld(f_in, k * N + ci, ifs);
#pragma unroll
    for (int k = 0; k < QS; k++) g[k] = ld(g_in, k * N + ci, igs) + wq<QS>(k) * p.s_ref;
    const float u = mac_in[N + ci], w = mac_in[2 * N + ci];
    const int rs = (lz + 1) * SX + lx + 1;
    const float S = sS[rs], rho = sR[rs];
    // p* (ref: collision.cu:244-246)
    float pr = 0.f;
#pragma unroll
    for (int k = 0; k < 9; k++) pr += f[k];
    // force: buoyancy + pressure gradient on the density (ref: collision.cu:77-88)
    const float pc = pr * c2 / 3.0f;
    const float Fx = -pc * ((sR[rs + 1] - sR[rs - 1]) * __ldg(p.ginvx + gx));
    const float Fz = (float)(-(double)S * p.g_bouss) - pc * ((sR[rs + SX] - sR[rs - SX]) * __ldg(p.ginvz + gz));
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
      const float P0 = pr - 1.5f * usq;
      const float hx = 0.5f * fden * Fx, hz = 0.5f * fden * Fz;
      const float m7 = 0.25f * om_shear * (((f[1] + f[3]) - (f[2] + f[4])) - (uc * uc - wc * wc));
      const float m8 = 0.25f * om_shear * (((f[5] + f[7]) - (f[6] + f[8])) - uc * wc);
      sf[e] = w9(0) * P0;
      {
        const float A = fmaf(4.5f * uc, uc, P0), B = fmaf(3.0f, uc, hx);
        sf[1 * NE + e] = fmaf(w9(1), A + B, m7);
        sf[3 * NE + e] = fmaf(w9(3), A - B, m7);
      }
      {
        const float A = fmaf(4.5f * wc, wc, P0), B = fmaf(3.0f, wc, hz);
        sf[2 * NE + e] = fmaf(w9(2), A + B, -m7);
        sf[4 * NE + e] = fmaf(w9(4), A - B, -m7);
      }
      {
        const float eu = uc + wc;
        const float A = fmaf(4.5f * eu, eu, P0), B = fmaf(3.0f, eu, hx + hz);
        sf[5 * NE + e] = fmaf(w9(5), A + B, m8);
        sf[7 * NE + e] = fmaf(w9(7), A - B, m8);
      }
      {
        const float eu = wc - uc;
        const float A = fmaf(4.5f * eu, eu, P0), B = fmaf(3.0f, eu, hz - hx);
        sf[6 * NE + e] = fmaf(w9(6), A + B, -m8);
        sf[8 * NE + e] = fmaf(w9(8), A - B, -m8);
      }
    } else {
      // equilibrium (ref: collision.cu:3-14), d = f - feq + Fk/2; d goes to
      // shared memory (this cell's own slots) so that only the outputs stay
      // in registers while the 9x9 operator is applied
      auto feq_of = [&](int k) {
        const float eu = (ex(k) ? ex(k) * uc : 0.f) + (ez(k) ? ez(k) * wc : 0.f);
        return w9(k) * (pr + 3.0f * eu + 4.5f * eu * eu - 1.5f * usq);
      };
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
    if constexpr (QS == 5) {
      // regularised D2Q5 collision (ref: collision.cu:167-188 on the D2Q5
      // lattice, linear equilibrium w S (1 + 3 e.u/c)): the first moment of
      // g - geq is j = (g1 - g3, g2 - g4) - S u/c, and
      //   g*_k = w_k (S + 3 e_k . (S u/c + (1 - 1/tau_s) j)).
      const float jx = (g[1] - g[3]) - S * uc, jz = (g[2] - g[4]) - S * wc;
      const float ax3 = 3.0f * fmaf(omg, jx, S * uc), az3 = 3.0f * fmaf(omg, jz, S * wc);
      sg[e] = w5(0) * S;
      sg[1 * NE + e] = w5(1) * (S + ax3);
      sg[3 * NE + e] = w5(3) * (S - ax3);
      sg[2 * NE + e] = w5(2) * (S + az3);
      sg[4 * NE + e] = w5(4) * (S - az3);
    } else if constexpr (QS == 9) {
      // regularised scalar collision on the reference's Q9 scalar lattice (ref: collision.cu:167-188)
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
    if (lx >= HX && lx < HX + kTX && lz >= HZ && lz < HZ + kTZ) {
      const int ii = (lz - HZ) * kTX + (lx - HX);
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

  for (int e = tid; e < kTX * kTZ; e += kThreads) {
    const int iz = e / kTX, ix = e - iz * kTX;
    const int gx = x0 + ix, gz = z0 + iz;
    if (gx >= nx || gz >= nz) continue;
    const long long ci = (long long)gz * nx + gx;
    const int lc = (iz + HZ) * EX + ix + HX;
    const int gA = G::AX == 0 ? gx : gz, gB = G::AX == 0 ? gz : gx, NB = G::AX == 0 ? nz : nx;
    const int la = G::AX == 0 ? ix + HX : iz + HZ;
    // interior: every source and stencil node inside the box
    const bool fast = (G::AX < 0) ? (gx >= 1 && gx <= nx - 2 && gz >= 1 && gz <= nz - 2)
                                  : (gA >= G::H && gA <= NA - 1 - G::H && gB >= 1 && gB <= NB - 2);
    float fv[9], gv[QS > 0 ? QS : 1];
    if (fast) {
      float W[2][G::NS + 1];
      if constexpr (G::AX >= 0) {
#pragma unroll
        for (int sidx = 0; sidx < 2; sidx++)
#pragma unroll
          for (int q = 0; q <= G::NS; q++) W[sidx][q] = sC[(sidx * (G::NS + 1) + q) * NWA + la];
      }
      fv[0] = Fast<GEO, 0>::pull(sf, lc, W);
      fv[1] = Fast<GEO, 1>::pull(sf, lc, W);
      fv[2] = Fast<GEO, 2>::pull(sf, lc, W);
      fv[3] = Fast<GEO, 3>::pull(sf, lc, W);
      fv[4] = Fast<GEO, 4>::pull(sf, lc, W);
      fv[5] = Fast<GEO, 5>::pull(sf, lc, W);
      fv[6] = Fast<GEO, 6>::pull(sf, lc, W);
      fv[7] = Fast<GEO, 7>::pull(sf, lc, W);
      fv[8] = Fast<GEO, 8>::pull(sf, lc, W);
      if constexpr (QS > 0) {
        gv[0] = Fast<GEO, 0>::pull(sg, lc, W);
        gv[1] = Fast<GEO, 1>::pull(sg, lc, W);
        gv[2] = Fast<GEO, 2>::pull(sg, lc, W);
        gv[3] = Fast<GEO, 3>::pull(sg, lc, W);
        gv[4] = Fast<GEO, 4>::pull(sg, lc, W);
        if constexpr (QS == 9) {
          gv[5] = Fast<GEO, 5>::pull(sg, lc, W);
          gv[6] = Fast<GEO, 6>::pull(sg, lc, W);
          gv[7] = Fast<GEO, 7>::pull(sg, lc, W);
          gv[8] = Fast<GEO, 8>::pull(sg, lc, W);
        }
      }
    } else {
      const int cls = (gx == 0 ? 1 : 0) | (gx == nx - 1 ? 2 : 0) | (gz == 0 ? 4 : 0) | (gz == nz - 1 ? 8 : 0);
#pragma unroll
      for (int k = 0; k < 9; k++) fv[k] = pull(sf, k, gx, gz, cls, p.slipB9, p.slipK9);
#pragma unroll
      for (int k = 0; k < QS; k++)
        gv[k] = pull(sg, k, gx, gz, cls, QS == 9 ? p.slipB9 : p.slipB5, QS == 9 ? p.slipK9 : p.slipK5);
    }
    float pr = 0.f, jx = 0.f, jz = 0.f;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const float v = fv[k];
      pr += v;
      if (ex(k)) jx += ex(k) * v;
      if (ez(k)) jz += ez(k) * v;
      st(f_out, k * N + ci, v, p.fscale);
    }
    float S = 0.f;
    if constexpr (QS > 0) {
#pragma unroll
      for (int k = 0; k < QS; k++) {
        S += gv[k];
        st(g_out, k * N + ci, gv[k] - wq<QS>(k) * p.s_ref, p.gscale);
      }
    } else {
      S = sS[(iz + HZ + 1) * SX + (ix + HX + 1)];
    }
    // moments (ref: collision.cu:244-254)
    const float rho = (float)((double)rho0 + (double)S * p.rho_sal);
    const float h = __fdividef(p.hdt, rho);
    const float ux = c * jx + sF[e] * h, uz = c * jz + sF[kTX * kTZ + e] * h;
    mac_out[ci] = S;
    mac_out[N + ci] = ux;
    mac_out[2 * N + ci] = uz;
    if (!(isfinite(ux) && isfinite(uz) && isfinite(S) && isfinite(pr))) atomicOr(p.status, 1u);
  }
}

template <class ST, int QS, int GEO>
__global__ void __launch_bounds__(kThreads, kMinBlocks) step_kernel(const __grid_constant__ Params p) {
  extern __shared__ float smem[];
  step_tile<ST, QS, GEO>(p, 0, blockIdx.x, blockIdx.y, smem);
}

template <class ST, int QS, int GEO>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
    step_kernel_batched(const Params *__restrict__ ps, const WorkItem *__restrict__ work, int nwork, int parity) {
  extern __shared__ float smem[];
  for (int i = blockIdx.x; i < nwork; i += gridDim.x) {
    const WorkItem w = work[i];
    step_tile<ST, QS, GEO>(ps[w.sim], parity, w.tx, w.tz, smem);
    __syncthreads();  // the next item reuses shared memory
  }
}

template <class ST, int QS, int GEO>
int launch_b(const Params *ps, const WorkItem *work, int nwork, int parity, int grid, cudaStream_t s, bool prep) {
  constexpr size_t sm = smem_bytes<ST, QS, GEO>();
  if (prep)
    return status_from_cuda(cudaFuncSetAttribute(step_kernel_batched<ST, QS, GEO>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  if (nwork <= 0) return IPCU_OK;
  step_kernel_batched<ST, QS, GEO><<<grid, kThreads, sm, s>>>(ps, work, nwork, parity);
  return status_from_cuda(cudaGetLastError());
}

template <class ST, int QS>
int launch_bg(const Params *ps, const WorkItem *work, int nwork, int parity, int geo, int grid, cudaStream_t s,
              bool prep) {
  switch (geo) {
    case IPCU_GEO_UNIFORM: return launch_b<ST, QS, IPCU_GEO_UNIFORM>(ps, work, nwork, parity, grid, s, prep);
    case IPCU_GEO_X5: return launch_b<ST, QS, IPCU_GEO_X5>(ps, work, nwork, parity, grid, s, prep);
    case IPCU_GEO_X3: return launch_b<ST, QS, IPCU_GEO_X3>(ps, work, nwork, parity, grid, s, prep);
    case IPCU_GEO_Z5: return launch_b<ST, QS, IPCU_GEO_Z5>(ps, work, nwork, parity, grid, s, prep);
    case IPCU_GEO_Z3: return launch_b<ST, QS, IPCU_GEO_Z3>(ps, work, nwork, parity, grid, s, prep);
  }
  return IPCU_ERR_UNSUPPORTED;
}

template <class ST, int QS, int GEO>
int launch_t(const Params &p, cudaStream_t s, bool prepare_only) {
  constexpr size_t sm = smem_bytes<ST, QS, GEO>();
  if (prepare_only) {  // once per sim, outside any stream capture
    return status_from_cuda(
        cudaFuncSetAttribute(step_kernel<ST, QS, GEO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  }
  dim3 grid((p.nx + kTX - 1) / kTX, (p.nz + kTZ - 1) / kTZ);
  step_kernel<ST, QS, GEO><<<grid, kThreads, sm, s>>>(p);
  return status_from_cuda(cudaGetLastError());
}

template <class ST, int QS>
int launch_g(const Params &p, int geo, cudaStream_t s, bool prep) {
  switch (geo) {
    case IPCU_GEO_UNIFORM: return launch_t<ST, QS, IPCU_GEO_UNIFORM>(p, s, prep);
    case IPCU_GEO_X5: return launch_t<ST, QS, IPCU_GEO_X5>(p, s, prep);
    case IPCU_GEO_X3: return launch_t<ST, QS, IPCU_GEO_X3>(p, s, prep);
    case IPCU_GEO_Z5: return launch_t<ST, QS, IPCU_GEO_Z5>(p, s, prep);
    case IPCU_GEO_Z3: return launch_t<ST, QS, IPCU_GEO_Z3>(p, s, prep);
  }
  return IPCU_ERR_UNSUPPORTED;
}

}  // namespace f2d
}  // namespace ipcu
