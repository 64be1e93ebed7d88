// Fused 3-D step on a box whose x and y axes are stretched (z uniform):
// D3Q19 MRT flow and D3Q7 salinity with the reference's conservative
// interpolated streaming (ref: function/adv.cu:50-257) along x and y, in the
// reference's step order (moments -> Force -> collision -> streaming ->
// moments; ref: LockExchange/LockExchange.cu:220-236, collision.cu:3-257).
//
// Streaming of a population that moves
//   * along z only: an exact shift;
//   * along x (or y) in-plane, with any z part: the 1-D flux form of
//     set_out's first loops, ftmp(c) = f*(c+a) + fin(c) - fout(c+a);
//   * along an xy diagonal: set_out's corner-transport form (adv.cu:100-145),
//     fout = fx dz/DX + fy dz/DY - fxy dz^2/(DX DY) and the three fin
//     contributions of cells c, c+x, c+y.
// then f(c) = ftmp(c - e) (propagation). In the interior the diagonal form
// equals the tensor product of the two 1-D flux-form operators, so every
// interior population is one dot product over its (NS+1) or (NS+1)^2 nodes
// with combined weights precomputed per axis index (held in registers per
// thread). Cells within the halo of an x or y wall, and the first and last
// z planes, take the general path: clamped nodes (ghosts carry their
// owner's value), mirror-image ghosts across x and y walls for the partner
// and flux quantities (set_wall_f_inv's mirror, applied to every quantity
// the flux form reads), halfway bounce-back for sources outside the box.
//
// A CTA owns a 32 x 8 column of cells and marches along a chunk of z. Each
// plane is collided once into shared memory, tile + halo (H cells in x and
// y); the post-collision populations are kept by the direction of their z
// motion: those moving up (needed by the plane above) in a ring of three
// planes, those staying in-plane in two, those moving down in two (the
// extra slots hold what a bounce-back at a z wall reads). A ring of three
// salinity planes one cell wider feeds the density gradient. Every stored
// value is read from HBM once and written once per step (halo re-reads hit
// L2): f [19][N], g [7][N] and the force F [3][N], 232 B per cell in FP32.
#include <cuda_runtime.h>

#include "d3q19.cuh"
#include "fused3s.cuh"
#include "ipcu_common.cuh"

namespace ipcu {
namespace f3s {

using namespace d3;

template <int NS>
struct G {
  static constexpr int h = NS / 2;
  static constexpr int H = h + 1;  // halo: nodes of the stencils around the partners
  static constexpr int RX = kTX + 2 * H, RY = kTY + 2 * H, RC = RX * RY;
  static constexpr int SX = RX + 2, SY = RY + 2, SC = SX * SY;  // salinity ring plane
  static constexpr int UP0 = 0;                                 // [3][6][RC]
  static constexpr int MID0 = UP0 + 3 * 6 * RC;                 // [2][14][RC]
  static constexpr int DN0 = MID0 + 2 * 14 * RC;                // [2][6][RC]
  static constexpr int S0 = DN0 + 2 * 6 * RC;                   // [3][SC]
  static constexpr int FR0 = S0 + 3 * SC;                       // [2][3][kTX * kTY] force of the tile cells
  static constexpr int NF = FR0 + 2 * 3 * kTX * kTY;
  static constexpr size_t bytes = sizeof(float) * (size_t)NF;
};

// slot of a population within its z-motion class: f (D3Q19) and g (D3Q7)
__host__ __device__ constexpr int fidx(int k) {
  constexpr int t[19] = {0, 1, 2, 3, 4, 0, 0, 5, 6, 7, 8, 1, 1, 2, 2, 3, 3, 4, 4};
  return t[k];
}
__host__ __device__ constexpr int gidx(int k) { return k < 5 ? 9 + k : 5; }

template <int NS>
__device__ __forceinline__ int cls_base(int k, int plane) {
  using Gm = G<NS>;
  if (cz(k) > 0) return Gm::UP0 + (plane % 3) * 6 * Gm::RC;
  if (cz(k) < 0) return Gm::DN0 + (plane & 1) * 6 * Gm::RC;
  return Gm::MID0 + (plane & 1) * 14 * Gm::RC;
}
// shared-memory offset of population k (g: isg) of plane `plane` at region cell (lx, ly)
template <int NS>
__device__ __forceinline__ int pofs(int k, bool isg, int plane) {
  return cls_base<NS>(k, plane) + (isg ? gidx(k) : fidx(k)) * G<NS>::RC;
}

template <int NS>
__global__ void __launch_bounds__(kThreads, 2) step3s_kernel(const __grid_constant__ Params3S p) {
  using Gm = G<NS>;
  constexpr int h = Gm::h, H = Gm::H, RX = Gm::RX, RC = Gm::RC, SX = Gm::SX, SC = Gm::SC;
  extern __shared__ __align__(16) float sm[];
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const long long N = (long long)nx * ny * nz, P = (long long)nx * ny;
  const int tid = threadIdx.x, tx = tid % kTX, ty = tid / kTX;
  const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
  const int zb = blockIdx.z * p.zchunk, ze = min(zb + p.zchunk, nz);
  const int rx0 = x0 - H, ry0 = y0 - H;  // global coordinates of region cell (0, 0)
  const float c = p.c, ic = 1.0f / c, c2 = c * c;
  auto clx = [&](int v) { return min(max(v, 0), nx - 1); };
  auto cly = [&](int v) { return min(max(v, 0), ny - 1); };

  // salinity S = sum g of plane q (clamped into the box), region + 1 cell
  auto form_S = [&](int q) {
    const int qz = min(max(q, 0), nz - 1);
    float *dst = sm + Gm::S0 + ((q % 3) + 3) % 3 * SC;
    for (int e = tid; e < SC; e += kThreads) {
      const int ly = e / SX, lx = e - ly * SX;
      const long long i = (long long)qz * P + (long long)cly(ry0 - 1 + ly) * nx + clx(rx0 - 1 + lx);
      float S = 0.f;
#pragma unroll
      for (int k = 0; k < 7; k++) S += p.g_in[k * N + i];
      dst[e] = S;
    }
  };

  // collide plane q (tile + halo, cells inside the box) into the class rings
  auto collide = [&](int q) {
    const float *Sq = sm + Gm::S0 + (q % 3) * SC;
    const float *Sm = sm + Gm::S0 + ((q + 2) % 3) * SC;
    const float *Sp = sm + Gm::S0 + ((q + 1) % 3) * SC;
    const float gz = (q == 0 || q == nz - 1) ? p.giz_wall : p.giz_in;
    for (int e = tid; e < RC; e += kThreads) {
      const int ly = e / RX, lx = e - ly * RX;
      const int gx = rx0 + lx, gy = ry0 + ly;
      if (gx < 0 || gx >= nx || gy < 0 || gy >= ny) continue;
      const long long i = (long long)q * P + (long long)gy * nx + gx;
      float f[19], g[7];
#pragma unroll
      for (int k = 0; k < 19; k++) f[k] = p.f_in[k * N + i];
#pragma unroll
      for (int k = 0; k < 7; k++) g[k] = p.g_in[k * N + i];
      const float Fpx = p.F_in[i], Fpy = p.F_in[N + i], Fpz = p.F_in[2 * N + i];
      float pr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
      for (int k = 0; k < 19; k++) {
        pr += f[k];
        if (cx(k)) jx += cx(k) * f[k];
        if (cy(k)) jy += cy(k) * f[k];
        if (cz(k)) jz += cz(k) * f[k];
      }
      const int se = (ly + 1) * SX + lx + 1;  // ring slot of the cell
      const float S = Sq[se];
      auto rs = [&](float s) { return fmaf(s, p.rsal, p.rho0); };
      const float rho = rs(S);
      const float hh = __fdividef(p.hdt, rho);
      const float uc = (c * jx + Fpx * hh) * ic, vc = (c * jy + Fpy * hh) * ic, wc = (c * jz + Fpz * hh) * ic;
      // force: buoyancy + pressure gradient over clamped neighbours (ref: collision.cu:77-88)
      const float pc = pr * c2 / 3.0f;
      const float Fx = -pc * ((rs(Sq[se + 1]) - rs(Sq[se - 1])) * __ldg(p.ax.ginv + gx));
      const float Fy = -pc * ((rs(Sq[se + SX]) - rs(Sq[se - SX])) * __ldg(p.ay.ginv + gy));
      const float Fz = -S * p.gb - pc * ((rs(q + 1 < nz ? Sp[se] : S) - rs(q > 0 ? Sm[se] : S)) * gz);
      const float fden = __fdividef(p.fk3, rho);
      float fo[19], go[7];
      collide19(f, g, pr, S, uc, vc, wc, 0.5f * fden * Fx, 0.5f * fden * Fy, 0.5f * fden * Fz, p.itau, p.omg_s,
                p.mrt != 0, fo, go);
      const int le = ly * RX + lx;
#pragma unroll
      for (int k = 0; k < 19; k++) sm[pofs<NS>(k, false, q) + le] = fo[k];
#pragma unroll
      for (int k = 0; k < 7; k++) sm[pofs<NS>(k, true, q) + le] = go[k];
      if (lx >= H && lx < H + kTX && ly >= H && ly < H + kTY) {
        float *Fr = sm + Gm::FR0 + (q & 1) * 3 * kTX * kTY + (ly - H) * kTX + (lx - H);
        Fr[0] = Fx;
        Fr[kTX * kTY] = Fy;
        Fr[2 * kTX * kTY] = Fz;
      }
      if (!(isfinite(uc) && isfinite(vc) && isfinite(wc) && isfinite(S) && isfinite(pr))) atomicOr(p.status, 1u);
    }
  };

  // ---- per-thread output column and its combined interior weights
  const int ox = x0 + tx, oy = y0 + ty;
  const bool own = ox < nx && oy < ny;
  const bool inx = ox >= H && ox <= nx - 1 - H, iny = oy >= H && oy <= ny - 1 - H;
  float Wx[2][NS + 1], Wy[2][NS + 1];
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int q = 0; q <= NS; q++) {
      Wx[s][q] = __ldg(p.ax.wC + (long long)(s * (NS + 1) + q) * nx + clx(ox));
      Wy[s][q] = __ldg(p.ay.wC + (long long)(s * (NS + 1) + q) * ny + cly(oy));
    }

  // ---- general path (walls): values, 1-D and tensor interpolants, flux form
  auto V = [&](int k, bool isg, int plane, int gx, int gy) -> float {
    return sm[pofs<NS>(k, isg, plane) + (gy - ry0) * RX + (gx - rx0)];
  };
  auto Ix = [&](int k, bool isg, int plane, int s, int gx, int gy) -> float {
    const int sg = s == 0 ? 1 : -1;
    float acc = 0.f;
#pragma unroll
    for (int m = 0; m < NS; m++)
      acc += __ldg(p.ax.wA + ((long long)s * nx + gx) * NS + m) * V(k, isg, plane, clx(gx + sg * (m - h)), gy);
    return acc;
  };
  auto Iy = [&](int k, bool isg, int plane, int s, int gx, int gy) -> float {
    const int sg = s == 0 ? 1 : -1;
    float acc = 0.f;
#pragma unroll
    for (int m = 0; m < NS; m++)
      acc += __ldg(p.ay.wA + ((long long)s * ny + gy) * NS + m) * V(k, isg, plane, gx, cly(gy + sg * (m - h)));
    return acc;
  };
  auto Ixy = [&](int k, int plane, int sxi, int syi, int gx, int gy) -> float {
    const int sgx = sxi == 0 ? 1 : -1, sgy = syi == 0 ? 1 : -1;
    float acc = 0.f;
#pragma unroll
    for (int n = 0; n < NS; n++) {
      float row = 0.f;
      const int yy = cly(gy + sgy * (n - h));
#pragma unroll
      for (int m = 0; m < NS; m++)
        row += __ldg(p.ax.wA + ((long long)sxi * nx + gx) * NS + m) * V(k, false, plane, clx(gx + sgx * (m - h)), yy);
      acc += __ldg(p.ay.wA + ((long long)syi * ny + gy) * NS + n) * row;
    }
    return acc;
  };
  // ftmp of population k of plane `plane` at cell (gx, gy) inside the box
  auto ftmp = [&](int k, bool isg, int plane, int gx, int gy) -> float {
    const int ax = cx(k), ay = cy(k);
    if (ax == 0 && ay == 0) return V(k, isg, plane, gx, gy);
    if (ay == 0) {  // along x
      const int s = ax > 0 ? 0 : 1, px = gx + ax;
      const float fin = Ix(k, isg, plane, s, gx, gy) * __ldg(p.ax.scin + (long long)s * nx + gx);
      if (px >= 0 && px < nx)
        return V(k, isg, plane, px, gy) + (fin - Ix(k, isg, plane, s, px, gy) * __ldg(p.ax.scout + px));
      const int km = mir(k, true, false);
      return V(km, isg, plane, gx, gy) + (fin - Ix(km, isg, plane, 1 - s, gx, gy) * __ldg(p.ax.scout + gx));
    }
    if (ax == 0) {  // along y
      const int s = ay > 0 ? 0 : 1, py = gy + ay;
      const float fin = Iy(k, isg, plane, s, gx, gy) * __ldg(p.ay.scin + (long long)s * ny + gy);
      if (py >= 0 && py < ny)
        return V(k, isg, plane, gx, py) + (fin - Iy(k, isg, plane, s, gx, py) * __ldg(p.ay.scout + py));
      const int km = mir(k, false, true);
      return V(km, isg, plane, gx, gy) + (fin - Iy(km, isg, plane, 1 - s, gx, gy) * __ldg(p.ay.scout + gy));
    }
    // xy diagonal: the quantities of (possibly ghost) cells, ghosts mirrored
    auto Q = [&](int type, int px, int py) -> float {
      const bool mx = px < 0 || px >= nx, my = py < 0 || py >= ny;
      const int kk = mir(k, mx, my), qx = clx(px), qy = cly(py);
      const int sxi = cx(kk) > 0 ? 0 : 1, syi = cy(kk) > 0 ? 0 : 1;
      if (type == 0) return V(kk, false, plane, qx, qy);
      if (type == 1) return Ix(kk, false, plane, sxi, qx, qy);
      if (type == 2) return Iy(kk, false, plane, syi, qx, qy);
      return Ixy(kk, plane, sxi, syi, qx, qy);
    };
    const float axs = __ldg(p.ax.scout + clx(gx + ax)), ays = __ldg(p.ay.scout + cly(gy + ay));
    const float fin = (axs * ays) * Q(3, gx, gy) + ays * (Q(2, gx + ax, gy) - axs * Q(3, gx + ax, gy)) +
                      axs * (Q(1, gx, gy + ay) - ays * Q(3, gx, gy + ay));
    const float fout = axs * Q(1, gx + ax, gy + ay) + ays * Q(2, gx + ax, gy + ay) - (axs * ays) * Q(3, gx + ax, gy + ay);
    return Q(0, gx + ax, gy + ay) + (fin - fout);
  };
  // streamed value of population k at output cell (gx, gy, z): pull from
  // c - e, or bounce back where that source lies outside the box
  auto general = [&](int k, bool isg, int z, int gx, int gy) -> float {
    const int sx = gx - cx(k), sy = gy - cy(k), sz = z - cz(k);
    if (sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz) return ftmp(k, isg, sz, sx, sy);
    return ftmp(opp(k), isg, z, gx, gy);
  };
  // interior path: combined weights, nodes around the cell itself
  auto fast = [&](int k, bool isg, int z) -> float {
    const int lx = tx + H, ly = ty + H;
    const float *b = sm + pofs<NS>(k, isg, z - cz(k)) + ly * RX + lx;
    const int ax = cx(k), ay = cy(k);
    if (ax == 0 && ay == 0) return b[0];
    if (ay == 0) {
      const int s = ax > 0 ? 0 : 1;
      float acc = 0.f;
#pragma unroll
      for (int q = 0; q <= NS; q++) acc = fmaf(Wx[s][q], b[(q - h - 1) * ax], acc);
      return acc;
    }
    if (ax == 0) {
      const int s = ay > 0 ? 0 : 1;
      float acc = 0.f;
#pragma unroll
      for (int r = 0; r <= NS; r++) acc = fmaf(Wy[s][r], b[(r - h - 1) * ay * RX], acc);
      return acc;
    }
    const int sx = ax > 0 ? 0 : 1, sy = ay > 0 ? 0 : 1;
    float acc = 0.f;
#pragma unroll
    for (int r = 0; r <= NS; r++) {
      float row = 0.f;
#pragma unroll
      for (int q = 0; q <= NS; q++) row = fmaf(Wx[sx][q], b[(r - h - 1) * ay * RX + (q - h - 1) * ax], row);
      acc = fmaf(Wy[sy][r], row, acc);
    }
    return acc;
  };

  // ---- march along z: planes zb - 1 (its upward populations) and zb first
  if (zb > 0) {
    form_S(zb - 2);
    form_S(zb - 1);
    form_S(zb);
    __syncthreads();
    collide(zb - 1);
    __syncthreads();
    form_S(zb + 1);  // the ring slot of plane zb - 2
  } else {
    form_S(zb - 1);
    form_S(zb);
    form_S(zb + 1);
  }
  __syncthreads();
  collide(zb);
  __syncthreads();
  for (int z = zb; z < ze; z++) {
    form_S(z + 2);  // the ring slot of plane z - 1, no longer read
    __syncthreads();
    if (z + 1 < nz) collide(z + 1);
    __syncthreads();
    if (own) {
      const bool interior = inx && iny && z >= 1 && z <= nz - 2;
      const long long i = (long long)z * P + (long long)oy * nx + ox;
      float pr = 0.f, S = 0.f;
#pragma unroll
      for (int k = 0; k < 19; k++) {
        const float v = interior ? fast(k, false, z) : general(k, false, z, ox, oy);
        p.f_out[k * N + i] = v;
        pr += v;
      }
#pragma unroll
      for (int k = 0; k < 7; k++) {
        const float v = interior ? fast(k, true, z) : general(k, true, z, ox, oy);
        p.g_out[k * N + i] = v;
        S += v;
      }
      const float *Fr = sm + Gm::FR0 + (z & 1) * 3 * kTX * kTY + ty * kTX + tx;
      p.F_out[i] = Fr[0];
      p.F_out[N + i] = Fr[kTX * kTY];
      p.F_out[2 * N + i] = Fr[2 * kTX * kTY];
      if (!(isfinite(pr) && isfinite(S))) atomicOr(p.status, 1u);
    }
    __syncthreads();  // the next collide overwrites the oldest ring slots
  }
}

size_t smem3s(int ns) { return ns == 5 ? G<5>::bytes : G<3>::bytes; }

template <int NS>
int launch_ns(const Params3S &p, cudaStream_t s, bool prep) {
  constexpr size_t sm = G<NS>::bytes;
  if (prep)
    return status_from_cuda(
        cudaFuncSetAttribute(step3s_kernel<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  dim3 grid((p.nx + kTX - 1) / kTX, (p.ny + kTY - 1) / kTY, (p.nz + p.zchunk - 1) / p.zchunk);
  step3s_kernel<NS><<<grid, kThreads, sm, s>>>(p);
  return status_from_cuda(cudaGetLastError());
}

int launch3s(const Params3S &p, int ns, cudaStream_t s, bool prepare_only) {
  if (ns == 3) return launch_ns<3>(p, s, prepare_only);
  if (ns == 5) return launch_ns<5>(p, s, prepare_only);
  return IPCU_ERR_UNSUPPORTED;
}

}  // namespace f3s
}  // namespace ipcu
