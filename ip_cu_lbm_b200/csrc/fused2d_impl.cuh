// Fused collide-and-stream step for 2-D boxes (D2Q9 flow in the x-z plane +
// D2Q5 or Q9 salinity), the B200 path of the reference's per-step chain
//   equ_f -> Force -> col_f_MRT -> IP_process(f) -> col_g_reg -> IP_process(g)
//   -> update_scalar -> update_rho -> set_wall_rho
// (ref: LockExchange/LockExchange.cu:220-236; kernels in function/collision.cu,
// function/adv.cu, function/set_bound.cu, function/propagation.cu).
//
// One launch per time step. A CTA owns a TX x TZ tile; phase 1 collides the
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
// (set_wall_f), x-wall partners mirrored (set_wall_f_inv), and sources
// outside the box taken from the owner's bounce-back (k -> -k) or specular
// slip partner (set_wall_propagation with the set_bound2D tables).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#pragma once
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
};

// storage conversion: value = stored*inv_scale + shift
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

template <class ST, int QS, int GEO>
__global__ void __launch_bounds__(kThreads) step_kernel(const Params p) {
  using G = Geo<GEO>;
  constexpr int HX = G::HX, HZ = G::HZ, EX = kTX + 2 * HX, EZ = kTZ + 2 * HZ, NE = EX * EZ;
  constexpr int SX = EX + 2, SZ = EZ + 2;  // salinity ring for the density gradient
  extern __shared__ float smem[];
  float *sf = smem;                       // [9][EZ][EX] post-collision f
  float *sg = sf + 9 * NE;                // [QS][EZ][EX] post-collision g
  float *sS = sg + QS * NE;               // [SZ][SX] salinity
  float *sF = sS + SZ * SX;               // [2][kTZ][kTX] interior force
  float *sW = sF + 2 * kTX * kTZ;         // weights of the tile's axis range

  const int nx = p.nx, nz = p.nz;
  const long long N = (long long)nx * nz;
  const int x0 = blockIdx.x * kTX, z0 = blockIdx.y * kTZ;
  const int ox = x0 - HX, oz = z0 - HZ;  // global coords of local (0,0)
  const int tid = threadIdx.x;
  const ST *__restrict__ f_in = static_cast<const ST *>(p.f_in);
  const ST *__restrict__ g_in = static_cast<const ST *>(p.g_in);
  ST *__restrict__ f_out = static_cast<ST *>(p.f_out);
  ST *__restrict__ g_out = static_cast<ST *>(p.g_out);

  // ---- phase 0: salinity ring and the interpolation weights of this tile
  for (int e = tid; e < SX * SZ; e += kThreads) {
    int lx = e % SX, lz = e / SX;
    int gx = min(max(ox - 1 + lx, 0), nx - 1), gz = min(max(oz - 1 + lz, 0), nz - 1);
    sS[e] = p.mac_in[(long long)gz * nx + gx];
  }
  constexpr int NWA = (G::AX == 0) ? EX : ((G::AX == 1) ? EZ : 0);
  constexpr int WREC = G::NS + 2;  // NS weights, fin scale, fout scale
  if constexpr (G::AX >= 0) {
    const int NA = (G::AX == 0) ? nx : nz, oA = (G::AX == 0) ? ox : oz;
    for (int e = tid; e < 2 * NWA * WREC; e += kThreads) {
      int s = e / (NWA * WREC), r = e % (NWA * WREC), la = r / WREC, m = r % WREC;
      int gA = min(max(oA + la, 0), NA - 1);
      float v;
      if (m < G::NS) v = __ldg(p.wA + ((long long)s * NA + gA) * G::NS + m);
      else if (m == G::NS) v = __ldg(p.scin + (long long)s * NA + gA);
      else v = __ldg(p.scout + gA);
      sW[e] = v;
    }
  }
  __syncthreads();

  const float c = p.c, c2 = c * c, dt = p.dt;
  const float itau = 1.0f / p.tau, omg = 1.0f - 1.0f / p.taus;
  // density as the reference forms it: float base plus a double salinity
  // term, rounded once (ref: collision.cu:251)
  const float rho0 = p.rhoL + (p.rhoH - p.rhoL) * p.phi;
  auto rho_of = [&](float S) -> float { return (float)((double)rho0 + (double)S * p.rho_sal); };
  const float ifs = p.inv_fscale, igs = p.inv_gscale;

  // ---- phase 1: collide tile + halo into shared memory
  for (int e = tid; e < NE; e += kThreads) {
    const int lx = e % EX, lz = e / EX;
    const int gx = ox + lx, gz = oz + lz;
    if (gx < 0 || gx >= nx || gz < 0 || gz >= nz) continue;
    const long long ci = (long long)gz * nx + gx;
    float f[9];
#pragma unroll
    for (int k = 0; k < 9; k++) f[k] = ld(f_in, k * N + ci, ifs);
    const float S = sS[(lz + 1) * SX + lx + 1];
    const float u = p.mac_in[N + ci], w = p.mac_in[2 * N + ci];
    // p* and rho (ref: collision.cu:244-251)
    float pr = 0.f;
#pragma unroll
    for (int k = 0; k < 9; k++) pr += f[k];
    const float rho = rho_of(S);
    // force: buoyancy + pressure gradient on the density (ref: collision.cu:77-88)
    const float rxp = rho_of(sS[(lz + 1) * SX + lx + 2]), rxm = rho_of(sS[(lz + 1) * SX + lx]);
    const float rzp = rho_of(sS[(lz + 2) * SX + lx + 1]), rzm = rho_of(sS[lz * SX + lx + 1]);
    const float pc = pr * c2 / 3.0f;
    const float Fx = -pc * ((rxp - rxm) * __ldg(p.ginvx + gx));
    const float Fz = (float)(-(double)S * p.g_bouss) - pc * ((rzp - rzm) * __ldg(p.ginvz + gz));
    const float usq = (u * u + w * w) / c2;
    const float fden = dt / (rho * c2 / 3.0f);
    float d[9], fk[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const float eu = c * (ex(k) * u + ez(k) * w) / c2;
      const float feq = w9(k) * (pr + 3.0f * eu + 4.5f * eu * eu - 1.5f * usq);
      fk[k] = w9(k) * c * (ex(k) * Fx + ez(k) * Fz) * fden;
      d[k] = f[k] - feq + 0.5f * fk[k];
    }
    if (p.mrt) {
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
        const float eu = c * (ex(k) * u + ez(k) * w) / c2;
        const float shape = (QS == 9) ? (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * usq) : (1.0f + 3.0f * eu);
        ge[k] = wq<QS>(k) * S * shape;
        const float ne = ld(g_in, k * N + ci, igs) + wq<QS>(k) * p.s_ref - ge[k];
        jx += ne * (c * ex(k));
        jz += ne * (c * ez(k));
      }
#pragma unroll
      for (int k = 0; k < QS; k++)
        sg[k * NE + e] = ge[k] + omg * (wq<QS>(k) * 3.0f * (jx * c * ex(k) + jz * c * ez(k)) / c2);
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
  // Lagrange interpolant of direction k (sign s) at cell (gx,gz) along the axis
  auto interp = [&](const float *arr, int k, int s, int gx, int gz) -> float {
    const int gA = (G::AX == 0) ? gx : gz, la = gA - ((G::AX == 0) ? ox : oz);
    const float *wr = sW + (s * NWA + la) * WREC;
    float acc = 0.f;
#pragma unroll
    for (int m = 0; m < G::NS; m++) {
      const int off = (s == 0 ? 1 : -1) * (m - G::NS / 2);
      const int q = min(max(gA + off, 0), NA - 1);
      const float v = (G::AX == 0) ? arr[k * NE + L(q, gz)] : arr[k * NE + L(gx, q)];
      acc += wr[m] * v;
    }
    return acc;
  };
  // the reference's ftmp (post set_tmp) of direction k at an in-box cell
  auto ftmp = [&](const float *arr, int k, int gx, int gz) -> float {
    if constexpr (G::AX < 0) {
      return arr[k * NE + L(gx, gz)];
    } else {
      const int a = (G::AX == 0) ? ex(k) : ez(k);
      if (a == 0) return arr[k * NE + L(gx, gz)];
      const int s = a > 0 ? 0 : 1;
      const int gA = (G::AX == 0) ? gx : gz, la = gA - ((G::AX == 0) ? ox : oz);
      const float fin = interp(arr, k, s, gx, gz) * sW[(s * NWA + la) * WREC + G::NS];
      const int gP = gA + a;
      if (gP >= 0 && gP < NA) {
        const int px = (G::AX == 0) ? gP : gx, pz = (G::AX == 0) ? gz : gP;
        const float fout = interp(arr, k, s, px, pz) * sW[(s * NWA + la + a) * WREC + G::NS + 1];
        return arr[k * NE + L(px, pz)] + (fin - fout);
      } else {
        const int km = (G::AX == 0) ? mirx(k) : mirz(k);
        const float fout = interp(arr, km, 1 - s, gx, gz) * sW[(s * NWA + la) * WREC + G::NS + 1];
        return arr[km * NE + L(gx, gz)] + (fin - fout);
      }
    }
  };
  // value pulled into (gx,gz) for direction k
  auto pull = [&](const float *arr, int k, int gx, int gz, int cls, const int8_t *slipB, const int8_t *slipK) -> float {
    const int sx = gx - ex(k), sz = gz - ez(k);
    if (sx >= 0 && sx < nx && sz >= 0 && sz < nz) return ftmp(arr, k, sx, sz);
    if (p.wall == IPCU_WALL_BB) return ftmp(arr, kinv(k), gx, gz);
    const int nb = slipB[cls * 9 + k], kk = slipK[cls * 9 + k];
    return ftmp(arr, kk, gx + ex(nb), gz + ez(nb));
  };

  for (int e = tid; e < kTX * kTZ; e += kThreads) {
    const int ix = e % kTX, iz = e / kTX;
    const int gx = x0 + ix, gz = z0 + iz;
    if (gx >= nx || gz >= nz) continue;
    const long long ci = (long long)gz * nx + gx;
    const int cls = (gx == 0 ? 1 : 0) | (gx == nx - 1 ? 2 : 0) | (gz == 0 ? 4 : 0) | (gz == nz - 1 ? 8 : 0);
    float pr = 0.f, jx = 0.f, jz = 0.f;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const float v = pull(sf, k, gx, gz, cls, p.slipB9, p.slipK9);
      pr += v;
      jx += (c * ex(k)) * v;
      jz += (c * ez(k)) * v;
      st(f_out, k * N + ci, v, p.fscale);
    }
    float S = 0.f;
    if constexpr (QS > 0) {
#pragma unroll
      for (int k = 0; k < QS; k++) {
        const float v = pull(sg, k, gx, gz, cls, QS == 9 ? p.slipB9 : p.slipB5, QS == 9 ? p.slipK9 : p.slipK5);
        S += v;
        st(g_out, k * N + ci, v - wq<QS>(k) * p.s_ref, p.gscale);
      }
    } else {
      S = sS[(gz - oz + 1) * SX + (gx - ox + 1)];
    }
    const float rho = rho_of(S);
    const float h = dt / (2.0f * rho);
    const float ux = jx + sF[e] * h, uz = jz + sF[kTX * kTZ + e] * h;
    p.mac_out[ci] = S;
    p.mac_out[N + ci] = ux;
    p.mac_out[2 * N + ci] = uz;
    if (!(isfinite(ux) && isfinite(uz) && isfinite(S) && isfinite(pr))) atomicOr(p.status, 1u);
  }
}

template <class ST, int QS, int GEO>
int launch_t(const Params &p, cudaStream_t s, bool prepare_only) {
  using G = Geo<GEO>;
  constexpr int EX = kTX + 2 * G::HX, EZ = kTZ + 2 * G::HZ, NE = EX * EZ;
  constexpr int NWA = (G::AX == 0) ? EX : ((G::AX == 1) ? EZ : 0);
  constexpr size_t sm = sizeof(float) * ((9 + QS) * NE + (EX + 2) * (EZ + 2) + 2 * kTX * kTZ + 2 * NWA * (G::NS + 2));
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
