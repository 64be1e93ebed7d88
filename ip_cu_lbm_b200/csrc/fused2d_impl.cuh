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

// FP32 storage stages the raw tile (f, g, u_x, u_z) into shared memory with
// asynchronous copies before colliding it in place; reduced-precision storage
// loads through registers (cp.async moves 4, 8 or 16 bytes, not 2).
template <class ST>
constexpr bool kStageAsync = sizeof(ST) == 4;

template <class ST, int QS, int GEO>
constexpr size_t smem_bytes() {
  using G = Geo<GEO>;
  return sizeof(float) * ((9 + QS + (kStageAsync<ST> ? 2 : 0)) * G::NE + 2 * G::SX * G::SZ + 2 * kTX * kTZ +
                          2 * G::NWA * G::WREC);
}

__device__ __forceinline__ void cp_async4(float *dst, const float *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
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

// Clamp-free pull for an interior cell. lc: local index of the cell; la:
// its local index along the interpolated axis; sW layout [s][m][la].
template <int GEO, int K, bool AMOVE>
struct Fast {
  using G = Geo<GEO>;
  static constexpr int DA = G::AX == 0 ? 1 : G::EX;   // one cell along the interpolated axis
  static constexpr int A = G::AX == 0 ? ex(K) : (G::AX == 1 ? ez(K) : 0);
  static constexpr int BX = G::AX == 0 ? 0 : ex(K);   // shift-axis part of e_K
  static constexpr int BZ = G::AX == 1 ? 0 : ez(K);
  __device__ __forceinline__ static float pull(const float *arr, int lc, int la, const float *sW) {
    constexpr int NE = G::NE;
    if constexpr (G::AX < 0 || A == 0) {
      return arr[K * NE + lc - ex(K) - ez(K) * G::EX];
    } else {
      constexpr int s = A > 0 ? 0 : 1, sg = A > 0 ? 1 : -1, h = G::NS / 2;
      const int cp = lc - BX - BZ * G::EX;  // c' = c - (shift part of e_K)
      float v[G::NS + 1];
#pragma unroll
      for (int q = 0; q <= G::NS; q++) v[q] = arr[K * NE + cp + sg * (q - h - 1) * DA];
      const float *wj = sW + (s * G::WREC) * G::NWA + (la - A);  // weights of j = c' - a
      const float *wc = sW + (s * G::WREC) * G::NWA + la;        // weights of c'
      float Ij = 0.f, Ic = 0.f;
#pragma unroll
      for (int m = 0; m < G::NS; m++) {
        Ij += wj[m * G::NWA] * v[m];
        Ic += wc[m * G::NWA] * v[m + 1];
      }
      return v[h + 1] + (Ij * wj[G::NS * G::NWA] - Ic * wc[(G::NS + 1) * G::NWA]);
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
  float *sU = sW + 2 * WREC * NWA;        // [2][EZ][EX] staged u_x, u_z (FP32 storage)

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

  // ---- phase 0: start the asynchronous copy of the raw tile + halo (FP32
  // storage), then stage the salinity/density ring and the axis weights
  if constexpr (kStageAsync<ST>) {
    const float *fin32 = reinterpret_cast<const float *>(f_in);
    const float *gin32 = reinterpret_cast<const float *>(g_in);
    for (int e = tid; e < NE; e += kThreads) {
      const int lz = e / EX, lx = e - lz * EX;
      const int gx = ox + lx, gz = oz + lz;
      if (gx < 0 || gx >= nx || gz < 0 || gz >= nz) continue;
      const long long ci = (long long)gz * nx + gx;
#pragma unroll
      for (int k = 0; k < 9; k++) cp_async4(sf + k * NE + e, fin32 + k * N + ci);
#pragma unroll
      for (int k = 0; k < QS; k++) cp_async4(sg + k * NE + e, gin32 + k * N + ci);
      cp_async4(sU + e, mac_in + N + ci);
      cp_async4(sU + NE + e, mac_in + 2 * N + ci);
    }
  }
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
  }
  if constexpr (kStageAsync<ST>) cp_async_wait_all();
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
    float f[9], g[QS > 0 ? QS : 1], u, w;
    if constexpr (kStageAsync<ST>) {
#pragma unroll
      for (int k = 0; k < 9; k++) f[k] = sf[k * NE + e];
#pragma unroll
      for (int k = 0; k < QS; k++) g[k] = sg[k * NE + e];
      u = sU[e];
      w = sU[NE + e];
    } else {
      const long long ci = (long long)gz * nx + gx;
#pragma unroll
      for (int k = 0; k < 9; k++) f[k] = ld(f_in, k * N + ci, ifs);
#pragma unroll
      for (int k = 0; k < QS; k++) g[k] = ld(g_in, k * N + ci, igs) + wq<QS>(k) * p.s_ref;
      u = mac_in[N + ci];
      w = mac_in[2 * N + ci];
    }
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
    // equilibrium (ref: collision.cu:3-14) and forcing term (ref: collision.cu:102-110)
    const float uc = u * ic, wc = w * ic;
    const float usq = uc * uc + wc * wc;
    const float fden = dt * c * 3.0f / (rho * c2);
    float d[9], fk[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const float eu = (ex(k) ? ex(k) * uc : 0.f) + (ez(k) ? ez(k) * wc : 0.f);
      const float feq = w9(k) * (pr + 3.0f * eu + 4.5f * eu * eu - 1.5f * usq);
      const float ef = (ex(k) ? ex(k) * Fx : 0.f) + (ez(k) ? ez(k) * Fz : 0.f);
      fk[k] = w9(k) * ef * fden;
      d[k] = f[k] - feq + 0.5f * fk[k];
    }
    if (p.mrt == 2) {
      // unit non-shear rates: f* = f - d + (1 - 1/tau) Minv_s M_s d + Fk, with
      // the Lallemand-Luo shear moments p_xx = d1-d2+d3-d4, p_xz = d5-d6+d7-d8
      const float m7 = 0.25f * om_shear * ((d[1] - d[2]) + (d[3] - d[4]));
      const float m8 = 0.25f * om_shear * ((d[5] - d[6]) + (d[7] - d[8]));
      const float sgn7[9] = {0, 1, -1, 1, -1, 0, 0, 0, 0}, sgn8[9] = {0, 0, 0, 0, 0, 1, -1, 1, -1};
#pragma unroll
      for (int a = 0; a < 9; a++) sf[a * NE + e] = f[a] - d[a] + fk[a] + sgn7[a] * m7 + sgn8[a] * m8;
    } else if (p.mrt == 1) {
      // f* = f - (MM + Minv_s M_s / tau) d + Fk (ref: collision.cu:115-150)
      float m7 = 0.f, m8 = 0.f;
#pragma unroll
      for (int k = 0; k < 9; k++) {
        m7 += p.Ms[k] * d[k];
        m8 += p.Ms[9 + k] * d[k];
      }
#pragma unroll
      for (int a = 0; a < 9; a++) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 9; k++) acc += p.MM[a * 9 + k] * d[k];
        acc += (p.Mis[a * 2] * m7 + p.Mis[a * 2 + 1] * m8) * itau;
        sf[a * NE + e] = f[a] - acc + fk[a];
      }
    } else {
#pragma unroll
      for (int k = 0; k < 9; k++) sf[k * NE + e] = f[k] - d[k] * itau + fk[k];
    }
    if constexpr (QS > 0) {
      // regularised scalar collision (ref: collision.cu:167-188)
      float ge[QS], jx = 0.f, jz = 0.f;
#pragma unroll
      for (int k = 0; k < QS; k++) {
        const float eu = (ex(k) ? ex(k) * uc : 0.f) + (ez(k) ? ez(k) * wc : 0.f);
        const float shape = (QS == 9) ? (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * usq) : (1.0f + 3.0f * eu);
        ge[k] = wq<QS>(k) * S * shape;
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
      fv[0] = Fast<GEO, 0, false>::pull(sf, lc, la, sW);
      fv[1] = Fast<GEO, 1, true>::pull(sf, lc, la, sW);
      fv[2] = Fast<GEO, 2, true>::pull(sf, lc, la, sW);
      fv[3] = Fast<GEO, 3, true>::pull(sf, lc, la, sW);
      fv[4] = Fast<GEO, 4, true>::pull(sf, lc, la, sW);
      fv[5] = Fast<GEO, 5, true>::pull(sf, lc, la, sW);
      fv[6] = Fast<GEO, 6, true>::pull(sf, lc, la, sW);
      fv[7] = Fast<GEO, 7, true>::pull(sf, lc, la, sW);
      fv[8] = Fast<GEO, 8, true>::pull(sf, lc, la, sW);
      if constexpr (QS > 0) {
        gv[0] = Fast<GEO, 0, false>::pull(sg, lc, la, sW);
        gv[1] = Fast<GEO, 1, true>::pull(sg, lc, la, sW);
        gv[2] = Fast<GEO, 2, true>::pull(sg, lc, la, sW);
        gv[3] = Fast<GEO, 3, true>::pull(sg, lc, la, sW);
        gv[4] = Fast<GEO, 4, true>::pull(sg, lc, la, sW);
        if constexpr (QS == 9) {
          gv[5] = Fast<GEO, 5, true>::pull(sg, lc, la, sW);
          gv[6] = Fast<GEO, 6, true>::pull(sg, lc, la, sW);
          gv[7] = Fast<GEO, 7, true>::pull(sg, lc, la, sW);
          gv[8] = Fast<GEO, 8, true>::pull(sg, lc, la, sW);
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
    const float h = dt / (2.0f * rho);
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
