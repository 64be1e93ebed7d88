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
// A CTA owns a 32 x 16 column of cells and marches along a chunk of z. Each
// plane is collided once into shared memory, tile + halo (H cells in x and
// y); the post-collision populations are kept by the direction of their z
// motion: those moving up (needed by the plane above) in a ring of three
// planes, those staying in-plane in two, those moving down in two (the
// extra slots hold what a bounce-back at a z wall reads). A ring of three
// salinity planes one cell wider feeds the density gradient. Every stored
// value is read from HBM once and written once per step (halo re-reads hit
// L2): f [19][N], g [7][N] and the force F [3][N], 232 B per cell in FP32.
//
// With 16-bit storage (store3d.cuh) the kernel decodes a cell's populations
// where it loads them (the collision of tile and halo cells, the salinity
// ring) and encodes them where it stores them, against the reference of
// each cell: the p and u/c its collision of this step left in shared memory
// and its salinity from the ring; 148 B per cell.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "d3q19.cuh"
#include "fused3s.cuh"
#include "ipcu_common.cuh"
#include "store3d.cuh"

namespace ipcu {
namespace f3s {

using namespace d3;

template <int NS, bool R16 = false>
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
  static constexpr int Q0 = FR0 + 2 * 3 * kTX * kTY;            // wall-cell queue: count + kTX * kTY cells
  // 16-bit storage: [2][4][kTX * kTY] reference values (p, u/c) of the tile
  // cells in the storage type, two to a slot
  static constexpr int RF0 = Q0 + 4 + kTX * kTY;
  static constexpr int NF = RF0 + (R16 ? 4 * kTX * kTY : 0);
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


// salinity S = sum g of cell i, in the order of load_cell's values
template <class T>
__device__ __forceinline__ float cell_S(const Params3S &p, long long i, long long N) {
  float S = 0.f;
  if constexpr (std::is_same<T, float>::value) {
    const float *gi = static_cast<const float *>(p.g_in);
#pragma unroll
    for (int k = 0; k < 7; k++) S += gi[k * N + i];
  } else {
    const T *gi = static_cast<const T *>(p.g_in), *ri = static_cast<const T *>(p.r_in);
    const s3::Ref r{0.f, s3::to_f(ri[N + i]), s3::to_f(ri[2 * N + i]), s3::to_f(ri[3 * N + i]), s3::to_f(ri[4 * N + i])};
#pragma unroll
    for (int k = 0; k < 7; k++) S += s3::dec(gi[k * N + i], p.inv_scale, s3::rg(k, r));
  }
  return S;
}

// Collision of cell i (column gx, gy; its salinity S and the clamped
// neighbours' along x, y and z; gz the z gradient factor of its plane): the
// reference's moments -> Force -> collision on the D3Q19 / D3Q7 subsets
// (ref: function/collision.cu:57-257). mo: the cell's pressure and u/c.
// Returns true where the state is not finite.
template <class T>
__device__ __forceinline__ bool collide_cell(const Params3S &p, long long i, long long N, int gx, int gy, float S,
                                             float Sxm, float Sxp, float Sym, float Syp, float Szm, float Szp,
                                             float gz, float (&fo)[19], float (&go)[7], float &Fx, float &Fy,
                                             float &Fz, bool ext, float (&mo)[4]) {
  const float c = p.c, ic = 1.0f / c, c2 = c * c;
  float f[19], g[7];
  s3::load_cell<T>(p.f_in, p.g_in, p.r_in, i, N, p.inv_scale, f, g);
  const float Fpx = p.F_in[i], Fpy = p.F_in[N + i], Fpz = p.F_in[2 * N + i];
  float pr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
  for (int k = 0; k < 19; k++) {
    pr += f[k];
    if (cx(k)) jx += cx(k) * f[k];
    if (cy(k)) jy += cy(k) * f[k];
    if (cz(k)) jz += cz(k) * f[k];
  }
  auto rs = [&](float s) { return fmaf(s, p.rsal, p.rho0); };
  const float rho = rs(S);
  const float hh = __fdividef(p.hdt, rho);
  const float uc = fmaf(c, jx, Fpx * hh) * ic, vc = fmaf(c, jy, Fpy * hh) * ic, wc = fmaf(c, jz, Fpz * hh) * ic;
  // force: buoyancy + pressure gradient over clamped neighbours (ref: collision.cu:77-88)
  const float pc = pr * c2 / 3.0f;
  Fx = -pc * ((rs(Sxp) - rs(Sxm)) * __ldg(p.ax.ginv + gx));
  Fy = -pc * ((rs(Syp) - rs(Sym)) * __ldg(p.ay.ginv + gy));
  Fz = fmaf(-S, p.gb, -(pc * ((rs(Szp) - rs(Szm)) * gz)));
  if (ext) {  // immersed-boundary force density of the last body update (inside its box)
    Fx += p.fext[i];
    Fy += p.fext[N + i];
    Fz += p.fext[2 * N + i];
  }
  const float fden = __fdividef(p.fk3, rho);
  collide19(f, g, pr, S, uc, vc, wc, 0.5f * fden * Fx, 0.5f * fden * Fy, 0.5f * fden * Fz, p.itau, p.omg_s,
            p.mrt != 0, fo, go);
  mo[0] = pr;
  mo[1] = uc;
  mo[2] = vc;
  mo[3] = wc;
  return !(isfinite(uc) && isfinite(vc) && isfinite(wc) && isfinite(S) && isfinite(pr));
}

// The wall path: populations of the boundary-layer cells (first and last
// cell along x, y or z) whose source c - e lies outside the box bounce back,
// f(c, k) = ftmp(c, -k), and the partner of that ftmp is across the wall:
// the flux form with mirror-image ghosts across x and y walls for every
// quantity it reads, and clamped nodes. The boundary-layer cells of a plane
// are queued and taken as (population, cell) pairs, consecutive lanes on one
// population, whose code is instantiated per population (compile-time
// direction tables; only the mirror choice is decided at run time).
//
// Src is where the post-collision populations live (RingSrc: the kernel's
// shared-memory plane rings, by z-motion class).
template <int NS>
struct RingSrc {
  using Gm = G<NS>;
  const float *sm;
  int rx0, ry0;
  // plane slot of the z-motion class CZ
  template <int CZ>
  __device__ __forceinline__ const float *slot(int plane) const {
    return sm + (CZ > 0 ? Gm::UP0 + (plane % 3) * 6 * Gm::RC
                        : (CZ < 0 ? Gm::DN0 + (plane & 1) * 6 * Gm::RC : Gm::MID0 + (plane & 1) * 14 * Gm::RC));
  }
  // value of slot row `idx` (population within the class) at (gx, gy)
  __device__ __forceinline__ float V(const float *b, int idx, int gx, int gy) const {
    return b[idx * Gm::RC + (gy - ry0) * Gm::RX + (gx - rx0)];
  }
};

template <int NS, class Src>
struct Wall {
  static constexpr int h = NS / 2;
  Src src;
  const Params3S *p;
  int nx, ny, nz;

  __device__ __forceinline__ int clx(int v) const { return min(max(v, 0), nx - 1); }
  __device__ __forceinline__ int cly(int v) const { return min(max(v, 0), ny - 1); }
  template <int CZ>
  __device__ __forceinline__ const float *slot(int plane) const {
    return src.template slot<CZ>(plane);
  }
  __device__ __forceinline__ float V(const float *b, int idx, int gx, int gy) const { return src.V(b, idx, gx, gy); }
  __device__ __forceinline__ float Ix(const float *b, int idx, int s, int gx, int gy) const {
    const int sg = s == 0 ? 1 : -1;
    const float *w = p->ax.wA + ((long long)s * nx + gx) * NS;
    float acc = 0.f;
#pragma unroll
    for (int m = 0; m < NS; m++) acc = fmaf(__ldg(w + m), V(b, idx, clx(gx + sg * (m - h)), gy), acc);
    return acc;
  }
  __device__ __forceinline__ float Iy(const float *b, int idx, int s, int gx, int gy) const {
    const int sg = s == 0 ? 1 : -1;
    const float *w = p->ay.wA + ((long long)s * ny + gy) * NS;
    float acc = 0.f;
#pragma unroll
    for (int m = 0; m < NS; m++) acc = fmaf(__ldg(w + m), V(b, idx, gx, cly(gy + sg * (m - h))), acc);
    return acc;
  }
  __device__ __forceinline__ float Ixy(const float *b, int idx, int sxi, int syi, int gx, int gy) const {
    const int sgx = sxi == 0 ? 1 : -1, sgy = syi == 0 ? 1 : -1;
    const float *wx = p->ax.wA + ((long long)sxi * nx + gx) * NS;
    const float *wy = p->ay.wA + ((long long)syi * ny + gy) * NS;
    int xs[NS];
#pragma unroll
    for (int m = 0; m < NS; m++) xs[m] = clx(gx + sgx * (m - h));
    float acc = 0.f;
#pragma unroll
    for (int n = 0; n < NS; n++) {
      const int yy = cly(gy + sgy * (n - h));
      float row = 0.f;
#pragma unroll
      for (int m = 0; m < NS; m++) row = fmaf(__ldg(wx + m), V(b, idx, xs[m], yy), row);
      acc = fmaf(__ldg(wy + n), row, acc);
    }
    return acc;
  }
  // ftmp of population K (g: ISG) of plane `plane` at cell (gx, gy) inside the box
  template <int K, bool ISG>
  __device__ __forceinline__ float ftmp(int plane, int gx, int gy) const {
    constexpr int ax = cx(K), ay = cy(K);
    const float *b = slot<cz(K)>(plane);
    constexpr int idx = ISG ? gidx(K) : fidx(K);
    if constexpr (ax == 0 && ay == 0) {
      return V(b, idx, gx, gy);
    } else if constexpr (ay == 0) {  // along x
      constexpr int s = ax > 0 ? 0 : 1, km = mir(K, true, false);
      constexpr int im = ISG ? gidx(km) : fidx(km);
      const int px = gx + ax;
      const float fin = Ix(b, idx, s, gx, gy) * __ldg(p->ax.scin + (long long)s * nx + gx);
      if (px >= 0 && px < nx) return V(b, idx, px, gy) + (fin - Ix(b, idx, s, px, gy) * __ldg(p->ax.scout + px));
      return V(b, im, gx, gy) + (fin - Ix(b, im, 1 - s, gx, gy) * __ldg(p->ax.scout + gx));
    } else if constexpr (ax == 0) {  // along y
      constexpr int s = ay > 0 ? 0 : 1, km = mir(K, false, true);
      constexpr int im = ISG ? gidx(km) : fidx(km);
      const int py = gy + ay;
      const float fin = Iy(b, idx, s, gx, gy) * __ldg(p->ay.scin + (long long)s * ny + gy);
      if (py >= 0 && py < ny) return V(b, idx, gx, py) + (fin - Iy(b, idx, s, gx, py) * __ldg(p->ay.scout + py));
      return V(b, im, gx, gy) + (fin - Iy(b, im, 1 - s, gx, gy) * __ldg(p->ay.scout + gy));
    } else {  // xy diagonal (corner transport, adv.cu:100-145); f populations only
      // a quantity (0 f*, 1 fx, 2 fy, 3 fxy) at a possibly ghost cell: the
      // owner's, for the population mirrored across the crossed walls
      auto Q = [&](int type, int px, int py) -> float {
        const bool mx = px < 0 || px >= nx, my = py < 0 || py >= ny;
        const int qx = clx(px), qy = cly(py);
        const int i = mx ? (my ? fidx(mir(K, true, true)) : fidx(mir(K, true, false)))
                         : (my ? fidx(mir(K, false, true)) : fidx(K));
        const int sxi = (ax > 0) != mx ? 0 : 1, syi = (ay > 0) != my ? 0 : 1;
        if (type == 0) return V(b, i, qx, qy);
        if (type == 1) return Ix(b, i, sxi, qx, qy);
        if (type == 2) return Iy(b, i, syi, qx, qy);
        return Ixy(b, i, sxi, syi, qx, qy);
      };
      const float axs = __ldg(p->ax.scout + clx(gx + ax)), ays = __ldg(p->ay.scout + cly(gy + ay));
      // (explicit fmas: the rounding does not depend on what the compiler
      // contracts around the call)
      const float fin = fmaf(axs * ays, Q(3, gx, gy),
                             fmaf(ays, fmaf(-axs, Q(3, gx + ax, gy), Q(2, gx + ax, gy)),
                                  axs * fmaf(-ays, Q(3, gx, gy + ay), Q(1, gx, gy + ay))));
      const float fout = fmaf(axs, Q(1, gx + ax, gy + ay),
                              fmaf(ays, Q(2, gx + ax, gy + ay), -((axs * ays) * Q(3, gx + ax, gy + ay))));
      return Q(0, gx + ax, gy + ay) + (fin - fout);
    }
  }
  // streamed value of population K at output cell (gx, gy, z) whose source
  // c - e lies outside the box: halfway bounce-back, ftmp of the opposite
  // population at the cell itself (its partner is then across the wall)
  __device__ float bounce_any(int kk, int z, int gx, int gy) const {
    switch (kk) {
#define IPCU_W3(k) \
  case k: return ftmp<opp(k), false>(z, gx, gy);
      IPCU_W3(0) IPCU_W3(1) IPCU_W3(2) IPCU_W3(3) IPCU_W3(4) IPCU_W3(5) IPCU_W3(6) IPCU_W3(7) IPCU_W3(8)
      IPCU_W3(9) IPCU_W3(10) IPCU_W3(11) IPCU_W3(12) IPCU_W3(13) IPCU_W3(14) IPCU_W3(15) IPCU_W3(16)
      IPCU_W3(17) IPCU_W3(18)
#undef IPCU_W3
#define IPCU_W3G(k) \
  case 19 + k: return ftmp<opp(k), true>(z, gx, gy);
      IPCU_W3G(0) IPCU_W3G(1) IPCU_W3G(2) IPCU_W3G(3) IPCU_W3G(4) IPCU_W3G(5) IPCU_W3G(6)
#undef IPCU_W3G
    }
    return 0.f;
  }
};

template <int NS, class T>
__global__ void __launch_bounds__(kThreads, kMinBlocks) step3s_kernel(const __grid_constant__ Params3S p) {
  constexpr bool R16 = !std::is_same<T, float>::value;
  using Gm = G<NS, R16>;
  constexpr int h = Gm::h, H = Gm::H, RX = Gm::RX, RC = Gm::RC, SX = Gm::SX, SC = Gm::SC;
  extern __shared__ __align__(16) float sm[];
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const long long N = (long long)nx * ny * nz, P = (long long)nx * ny;
  const int tid = threadIdx.x, tx = tid % kTX, ty = tid / kTX;
  const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
  const int zb = blockIdx.z * p.zchunk, ze = min(zb + p.zchunk, nz);
  const int rx0 = x0 - H, ry0 = y0 - H;  // global coordinates of region cell (0, 0)
  auto clx = [&](int v) { return min(max(v, 0), nx - 1); };
  auto cly = [&](int v) { return min(max(v, 0), ny - 1); };

  // the immersed-boundary force density is read only inside its box
  int fb[6] = {0, 0, 0, 0, 0, 0};
  if (p.fext != nullptr)
#pragma unroll
    for (int a = 0; a < 6; a++) fb[a] = p.fext_box[a];

  // salinity S = sum g of plane q (clamped into the box), region + 1 cell
  auto form_S = [&](int q) {
    const int qz = min(max(q, 0), nz - 1);
    float *dst = sm + Gm::S0 + ((q % 3) + 3) % 3 * SC;
    for (int e = tid; e < SC; e += kThreads) {
      const int ly = e / SX, lx = e - ly * SX;
      const long long i = (long long)qz * P + (long long)cly(ry0 - 1 + ly) * nx + clx(rx0 - 1 + lx);
      dst[e] = cell_S<T>(p, i, N);
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
      const int se = (ly + 1) * SX + lx + 1;  // ring slot of the cell
      const float S = Sq[se];
      float fo[19], go[7], Fx, Fy, Fz, mo[4];
      const bool ext = fb[3] > 0 && gx >= fb[0] && gx < fb[0] + fb[3] && gy >= fb[1] && gy < fb[1] + fb[4] &&
                       q >= fb[2] && q < fb[2] + fb[5];
      const bool bad = collide_cell<T>(p, i, N, gx, gy, S, Sq[se - 1], Sq[se + 1], Sq[se - SX], Sq[se + SX],
                                       q > 0 ? Sm[se] : S, q + 1 < nz ? Sp[se] : S, gz, fo, go, Fx, Fy, Fz, ext, mo);
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
        if constexpr (R16) {  // the reference the cell's stored populations will be encoded against
          T *rf = reinterpret_cast<T *>(sm + Gm::RF0) + (q & 1) * 4 * kTX * kTY + (ly - H) * kTX + (lx - H);
#pragma unroll
          for (int a = 0; a < 4; a++) rf[a * kTX * kTY] = s3::from_f<T>(mo[a]);
        }
      }
      if (bad) atomicOr(p.status, 1u);
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

  // combined-weight path, nodes around the cell itself. By linearity the
  // flux form of a population whose source lies inside the box is this dot
  // product also next to a wall, with the node addresses clamped into the
  // box as the ghosts carry their owner's value (CL: the cell lies within
  // the halo of an x or y wall).
  auto fast = [&](int k, bool isg, int z, auto clamp_tag) -> float {
    constexpr bool CL = decltype(clamp_tag)::value;
    const int lx = tx + H, ly = ty + H;
    const float *b0 = sm + pofs<NS>(k, isg, z - cz(k));
    auto nx_ = [&](int off) { return CL ? clx(ox + off) - rx0 : lx + off; };
    auto ny_ = [&](int off) { return CL ? cly(oy + off) - ry0 : ly + off; };
    const int ax = cx(k), ay = cy(k);
    if (ax == 0 && ay == 0) return b0[ly * RX + lx];
    if (ay == 0) {
      const int s = ax > 0 ? 0 : 1;
      const float *b = b0 + ly * RX;
      float acc = 0.f;
#pragma unroll
      for (int q = 0; q <= NS; q++) acc = fmaf(Wx[s][q], b[nx_((q - h - 1) * ax)], acc);
      return acc;
    }
    if (ax == 0) {
      const int s = ay > 0 ? 0 : 1;
      float acc = 0.f;
#pragma unroll
      for (int r = 0; r <= NS; r++) acc = fmaf(Wy[s][r], b0[ny_((r - h - 1) * ay) * RX + lx], acc);
      return acc;
    }
    const int sx = ax > 0 ? 0 : 1, sy = ay > 0 ? 0 : 1;
    float acc = 0.f;
#pragma unroll
    for (int r = 0; r <= NS; r++) {
      const float *b = b0 + ny_((r - h - 1) * ay) * RX;
      float row = 0.f;
#pragma unroll
      for (int q = 0; q <= NS; q++) row = fmaf(Wx[sx][q], b[nx_((q - h - 1) * ax)], row);
      acc = fmaf(Wy[sy][r], row, acc);
    }
    return acc;
  };

  // ---- storage of the output populations. 16-bit: the reference of tile
  // cell `cell` of plane z (its collision's p and u/c from shared memory, S
  // from the salinity ring) in the storage type; i >= 0 also writes the
  // cell's reference planes
  auto tile_ref = [&](int cell, int z, long long i) -> s3::Ref {
    s3::Ref R{};
    if constexpr (R16) {
      const T *rf = reinterpret_cast<const T *>(sm + Gm::RF0) + (z & 1) * 4 * kTX * kTY + cell;
      const int se = (cell / kTX + H + 1) * SX + cell % kTX + H + 1;
      const T Sh = s3::from_f<T>(sm[Gm::S0 + (z % 3) * SC + se]);
      R = s3::Ref{s3::to_f(rf[0]), s3::to_f(rf[kTX * kTY]), s3::to_f(rf[2 * kTX * kTY]), s3::to_f(rf[3 * kTX * kTY]),
                  s3::to_f(Sh)};
      if (i >= 0) {
        T *ro = static_cast<T *>(p.r_out);
#pragma unroll
        for (int a = 0; a < 4; a++) ro[a * N + i] = rf[a * kTX * kTY];
        ro[4 * N + i] = Sh;
      }
    }
    return R;
  };
  auto put = [&](bool isg, int k, long long i, float v, const s3::Ref &R, float &amax) {
    if constexpr (R16) {
      const float x = s3::mul(s3::add(v, -(isg ? s3::rg(k, R) : s3::rf(k, R))), p.scale);
      amax = fmaxf(amax, fabsf(x));
      static_cast<T *>(isg ? p.g_out : p.f_out)[k * N + i] = s3::from_f<T>(x);
    } else {
      static_cast<float *>(isg ? p.g_out : p.f_out)[k * N + i] = v;
    }
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
    int *qcount = reinterpret_cast<int *>(sm + Gm::Q0), *queue = qcount + 4;
    if (tid == 0) *qcount = 0;
    __syncthreads();
    // populations whose source lies outside the box (boundary layer only)
    // are left to the wall path below
    const bool zlo = z == 0, zhi = z == nz - 1;
    const bool xlo = ox == 0, xhi = ox == nx - 1, ylo = oy == 0, yhi = oy == ny - 1;
    auto src_in = [&](int k) {
      return !((cx(k) > 0 && xlo) || (cx(k) < 0 && xhi) || (cy(k) > 0 && ylo) || (cy(k) < 0 && yhi) ||
               (cz(k) > 0 && zlo) || (cz(k) < 0 && zhi));
    };
    if (own) {
      const long long i = (long long)z * P + (long long)oy * nx + ox;
      const float *Fr = sm + Gm::FR0 + (z & 1) * 3 * kTX * kTY + ty * kTX + tx;
      p.F_out[i] = Fr[0];
      p.F_out[N + i] = Fr[kTX * kTY];
      p.F_out[2 * N + i] = Fr[2 * kTX * kTY];
      if (xlo || xhi || ylo || yhi || zlo || zhi) queue[atomicAdd(qcount, 1)] = tid;
      float pr = 0.f, S = 0.f, amax = 0.f;
      s3::Ref R{};
      if constexpr (R16) {  // the cell's reference planes
        R = tile_ref(tid, z, i);
        amax = fmaxf(fmaxf(fabsf(R.p), fabsf(R.S)), fmaxf(fmaxf(fabsf(R.ux), fabsf(R.uy)), fabsf(R.uz)));
      }
      auto all = [&](auto tag) {
#pragma unroll
        for (int k = 0; k < 19; k++)
          if (src_in(k)) {
            const float v = fast(k, false, z, tag);
            put(false, k, i, v, R, amax);
            pr += v;
          }
#pragma unroll
        for (int k = 0; k < 7; k++)
          if (src_in(k)) {
            const float v = fast(k, true, z, tag);
            put(true, k, i, v, R, amax);
            S += v;
          }
      };
      if (inx && iny) all(std::false_type{});
      else all(std::true_type{});
      if (!(isfinite(pr) && isfinite(S))) atomicOr(p.status, 1u);
      if (R16 && !(amax <= p.store_max)) atomicOr(p.status, 4u);
    }
    // the wall cells of the plane: one (cell, population) pair per thread
    __syncthreads();
    {
      const Wall<NS, RingSrc<NS>> wp{RingSrc<NS>{sm, rx0, ry0}, &p, nx, ny, nz};
      const int nq = *qcount, nw = nq * 26;
#pragma unroll 1
      for (int w = tid; w < nw; w += kThreads) {
        const int kk = w / nq, cell = queue[w - kk * nq];  // consecutive lanes: one population
        const int gx = x0 + cell % kTX, gy = y0 + cell / kTX;
        const int k = kk >= 19 ? kk - 19 : kk;
        const int sx = gx - cx(k), sy = gy - cy(k), sz = z - cz(k);
        if (sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz) continue;  // done above
        const float v = wp.bounce_any(kk, z, gx, gy);
        const long long i = (long long)z * P + (long long)gy * nx + gx;
        float amax = 0.f;
        s3::Ref R{};
        if constexpr (R16) R = tile_ref(cell, z, -1);
        put(kk >= 19, k, i, v, R, amax);
        if (!isfinite(v)) atomicOr(p.status, 1u);
        if (R16 && !(amax <= p.store_max)) atomicOr(p.status, 4u);
      }
    }
    __syncthreads();  // the next collide overwrites the oldest ring slots
  }
}

template <int NS, class T>
int launch_ns(const Params3S &p, cudaStream_t s, bool prep) {
  constexpr size_t sm = G<NS, !std::is_same<T, float>::value>::bytes;
  static_assert(sm <= 227 * 1024, "shared memory of the 3-D step");
  if (prep)
    return status_from_cuda(
        cudaFuncSetAttribute(step3s_kernel<NS, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  dim3 grid((p.nx + kTX - 1) / kTX, (p.ny + kTY - 1) / kTY, (p.nz + p.zchunk - 1) / p.zchunk);
  step3s_kernel<NS, T><<<grid, kThreads, sm, s>>>(p);
  return status_from_cuda(cudaGetLastError());
}

template <int NS>
int launch_st(const Params3S &p, cudaStream_t s, bool prep) {
  if (p.store == IPCU_STORE_F32) return launch_ns<NS, float>(p, s, prep);
  if (p.store == IPCU_STORE_F16) return launch_ns<NS, __half>(p, s, prep);
  if (p.store == IPCU_STORE_BF16) return launch_ns<NS, __nv_bfloat16>(p, s, prep);
  return IPCU_ERR_ARG;
}

int launch3s(const Params3S &p, int ns, cudaStream_t s, bool prepare_only) {
  if (ns == 3) return launch_st<3>(p, s, prepare_only);
  if (ns == 5) return launch_st<5>(p, s, prepare_only);
  return IPCU_ERR_UNSUPPORTED;
}

}  // namespace f3s
}  // namespace ipcu
