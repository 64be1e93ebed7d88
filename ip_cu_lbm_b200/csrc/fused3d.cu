// Fused 3-D step on a uniform box: D3Q19 flow with MRT collision and a
// D3Q7 passive salinity, in the reference's step order
//   moments -> Force (Boussinesq buoyancy + pressure gradient) -> MRT
//   collision -> regularised scalar collision -> streaming -> moments
// (ref: LockExchange/LockExchange.cu:220-236; function/collision.cu:3-188,
// 238-257; propagation.cu; set_bound.cu:164-183 for halfway bounce-back),
// restricted to the D3Q19 / D3Q7 subsets of the reference's D3Q27 order
// (ref: function/basic.cu:88-97).
//
// Layout: structure-of-arrays, x fastest, then y, then z: f [19][N],
// g [7][N], and the previous step's force F [3][N] (u = c sum e f +
// F dt / 2 rho needs it, as update_rho adds the force of the step that
// produced f). Ping-pong buffers; each population is read once from its
// cell and written once to the cell it streams into (push), bounced back
// into its own cell's opposite slot where that cell lies outside the box.
//
// A CTA owns a 32 x 8 column of cells and marches along a chunk of z. The
// density gradient needs the salinity S = sum g one cell around each cell:
// a ring of three S planes (34 x 10, one cell of halo in x and y) slides
// along z in shared memory, each plane formed once per CTA.
//
// MRT with the reference's unit non-shear rates (its S file): every moment
// but the five shear moments of the d'Humieres basis relaxes to equilibrium
// in one step, so
//   f*_k = feq_k + Fk_k/2 + (1 - 1/tau) sum_m (M_m.(f - feq)) M_mk / |M_m|^2
// over m in {3p_xx, p_ww, p_xy, p_yz, p_xz} (the forcing part of the shear
// moments vanishes by parity), with M_m.feq = (2u^2 - v^2 - w^2, v^2 - w^2,
// uv, vw, uw)/c^2 and |M_m|^2 = 36, 12, 4, 4, 4.
#include <cuda_runtime.h>

#include "fused3d.cuh"
#include "ipcu_common.cuh"

namespace ipcu {
namespace f3d {

constexpr int kTX = 32, kTY = 8, kThreads = kTX * kTY;
constexpr int kRX = kTX + 2, kRY = kTY + 2;  // S ring plane with one cell of halo

// D3Q19 = the reference's D3Q27 order truncated (rest, 6 axes, 12 edges)
__host__ __device__ constexpr int cx(int k) {
  return (k == 1 || k == 7 || k == 8 || k == 11 || k == 12) ? 1 : ((k == 3 || k == 9 || k == 10 || k == 13 || k == 14) ? -1 : 0);
}
__host__ __device__ constexpr int cy(int k) {
  return (k == 2 || k == 7 || k == 9 || k == 15 || k == 16) ? 1 : ((k == 4 || k == 8 || k == 10 || k == 17 || k == 18) ? -1 : 0);
}
__host__ __device__ constexpr int cz(int k) {
  return (k == 5 || k == 11 || k == 13 || k == 15 || k == 17) ? 1 : ((k == 6 || k == 12 || k == 14 || k == 16 || k == 18) ? -1 : 0);
}
// opposite direction: axis pairs (1,3) (2,4) (5,6); edge pairs sum to 17, 25, 33
__host__ __device__ constexpr int opp(int k) {
  return k == 0 ? 0 : (k <= 4 ? ((k + 1) % 4) + 1 : (k <= 6 ? 11 - k : (k <= 10 ? 17 - k : (k <= 14 ? 25 - k : 33 - k))));
}
__host__ __device__ constexpr float w19(int k) { return k == 0 ? 1.0f / 3.0f : (k <= 6 ? 1.0f / 18.0f : 1.0f / 36.0f); }
__host__ __device__ constexpr float w7(int k) { return k == 0 ? 0.25f : 0.125f; }
// shear rows of the d'Humieres basis
__host__ __device__ constexpr int m1(int k) { return 2 * cx(k) * cx(k) - cy(k) * cy(k) - cz(k) * cz(k); }
__host__ __device__ constexpr int m2(int k) { return cy(k) * cy(k) - cz(k) * cz(k); }
__host__ __device__ constexpr int m3(int k) { return cx(k) * cy(k); }
__host__ __device__ constexpr int m4(int k) { return cy(k) * cz(k); }
__host__ __device__ constexpr int m5(int k) { return cx(k) * cz(k); }

constexpr bool check_opp() {
  for (int k = 0; k < 19; k++)
    if (cx(opp(k)) != -cx(k) || cy(opp(k)) != -cy(k) || cz(opp(k)) != -cz(k)) return false;
  return true;
}
static_assert(check_opp(), "D3Q19 opposite table");

__global__ void __launch_bounds__(kThreads, 4) step3d_kernel(const __grid_constant__ Params3 p) {
  __shared__ float sS[3][kRY][kRX];
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const long long N = (long long)nx * ny * nz, P = (long long)nx * ny;
  const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
  const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
  const int zb = blockIdx.z * p.zchunk, ze = min(zb + p.zchunk, nz);
  const int x = x0 + tx, y = y0 + ty;
  const bool own = x < nx && y < ny;
  // the immersed-boundary force density is read only inside its box
  int fb[6] = {0, 0, 0, 0, 0, 0};
  if (p.fext != nullptr)
#pragma unroll
    for (int a = 0; a < 6; a++) fb[a] = p.fext_box[a];
  const bool fcol = fb[3] > 0 && x >= fb[0] && x < fb[0] + fb[3] && y >= fb[1] && y < fb[1] + fb[4];

  // S of plane z (clamped into the box) for the ring slot z mod 3
  auto form_plane = [&](int z) {
    const int zc = min(max(z, 0), nz - 1);
    for (int e = threadIdx.x; e < kRX * kRY; e += kThreads) {
      const int ly = e / kRX, lx = e - ly * kRX;
      const int gx = min(max(x0 - 1 + lx, 0), nx - 1), gy = min(max(y0 - 1 + ly, 0), ny - 1);
      const float *__restrict__ gp = p.g_in + ((long long)zc * P + (long long)gy * nx + gx);
      float S = 0.f;
#pragma unroll
      for (int k = 0; k < 7; k++) S += gp[k * N];
      sS[((z % 3) + 3) % 3][ly][lx] = S;
    }
  };
  form_plane(zb - 1);
  form_plane(zb);

  const float c = p.c, ic = 1.0f / c, c2 = c * c;
  for (int z = zb; z < ze; z++) {
    form_plane(z + 1);
    __syncthreads();
    if (own) {
      const long long i = (long long)z * P + (long long)y * nx + x;
      // per-cell base pointers: every access below is base + a warp-uniform offset
      const float *__restrict__ fi = p.f_in + i;
      const float *__restrict__ gi = p.g_in + i;
      const float *__restrict__ Fi = p.F_in + i;
      float f[19], g[7];
#pragma unroll
      for (int k = 0; k < 19; k++) f[k] = fi[k * N];
#pragma unroll
      for (int k = 0; k < 7; k++) g[k] = gi[k * N];
      const float Fpx = Fi[0], Fpy = Fi[N], Fpz = Fi[2 * N];
      const int s0 = z % 3, sm = (z + 2) % 3, sp = (z + 1) % 3;
      const int lx = tx + 1, ly = ty + 1;
      // moments (ref: collision.cu:238-257): p*, S, u with the previous force
      float pr = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
      for (int k = 0; k < 19; k++) {
        pr += f[k];
        if (cx(k)) jx += cx(k) * f[k];
        if (cy(k)) jy += cy(k) * f[k];
        if (cz(k)) jz += cz(k) * f[k];
      }
      const float S = sS[s0][ly][lx];
      const float rho = fmaf(S, p.rsal, p.rho0);
      const float h = __fdividef(p.hdt, rho);
      const float uc = fmaf(c, jx, Fpx * h) * ic, vc = fmaf(c, jy, Fpy * h) * ic, wc = fmaf(c, jz, Fpz * h) * ic;
      // force: buoyancy + pressure gradient, clamped central differences (ref: collision.cu:77-88)
      auto rs = [&](float s) { return fmaf(s, p.rsal, p.rho0); };
      const float gx = (x == 0 || x == nx - 1) ? p.gi_wall : p.gi_in;
      const float gy = (y == 0 || y == ny - 1) ? p.gi_wall : p.gi_in;
      const float gz = (z == 0 || z == nz - 1) ? p.gi_wall : p.gi_in;
      const float pc = pr * c2 / 3.0f;
      float Fx = -pc * ((rs(sS[s0][ly][x + 1 < nx ? lx + 1 : lx]) - rs(sS[s0][ly][x > 0 ? lx - 1 : lx])) * gx);
      float Fy = -pc * ((rs(sS[s0][y + 1 < ny ? ly + 1 : ly][lx]) - rs(sS[s0][y > 0 ? ly - 1 : ly][lx])) * gy);
      float Fz =
          fmaf(-S, p.gb, -(pc * ((rs(sS[z + 1 < nz ? sp : s0][ly][lx]) - rs(sS[z > 0 ? sm : s0][ly][lx])) * gz)));
      if (fcol && z >= fb[2] && z < fb[2] + fb[5]) {  // immersed-boundary force density of the last body update
        Fx += p.fext[i];
        Fy += p.fext[N + i];
        Fz += p.fext[2 * N + i];
      }
      // collision
      const float fden = __fdividef(p.fk3, rho);
      const float hx = 0.5f * fden * Fx, hy = 0.5f * fden * Fy, hz = 0.5f * fden * Fz;
      const float usq = uc * uc + vc * vc + wc * wc;
      const float P0 = pr - 1.5f * usq;
      float fo[19];
      if (p.mrt) {
        // shear moments of f - feq, divided by the row norms
        float a1 = 0.f, a2 = 0.f, a3 = 0.f, a4 = 0.f, a5 = 0.f;
#pragma unroll
        for (int k = 0; k < 19; k++) {
          if (m1(k)) a1 += m1(k) * f[k];
          if (m2(k)) a2 += m2(k) * f[k];
          if (m3(k)) a3 += m3(k) * f[k];
          if (m4(k)) a4 += m4(k) * f[k];
          if (m5(k)) a5 += m5(k) * f[k];
        }
        const float om = 1.0f - p.itau;
        a1 = om * (a1 - (2.0f * uc * uc - vc * vc - wc * wc)) * (1.0f / 36.0f);
        a2 = om * (a2 - (vc * vc - wc * wc)) * (1.0f / 12.0f);
        a3 = om * (a3 - uc * vc) * 0.25f;
        a4 = om * (a4 - vc * wc) * 0.25f;
        a5 = om * (a5 - uc * wc) * 0.25f;
#pragma unroll
        for (int k = 0; k < 19; k++) {
          const float eu = (cx(k) ? cx(k) * uc : 0.f) + (cy(k) ? cy(k) * vc : 0.f) + (cz(k) ? cz(k) * wc : 0.f);
          const float eh = (cx(k) ? cx(k) * hx : 0.f) + (cy(k) ? cy(k) * hy : 0.f) + (cz(k) ? cz(k) * hz : 0.f);
          float sh = 0.f;
          if (m1(k)) sh += m1(k) * a1;
          if (m2(k)) sh += m2(k) * a2;
          if (m3(k)) sh += m3(k) * a3;
          if (m4(k)) sh += m4(k) * a4;
          if (m5(k)) sh += m5(k) * a5;
          fo[k] = fmaf(w19(k), fmaf(4.5f * eu, eu, P0) + fmaf(3.0f, eu, eh), sh);
        }
      } else {
        // BGK with forcing (ref: collision.cu:151-165): f* = f - (f - feq + Fk/2)/tau + Fk
#pragma unroll
        for (int k = 0; k < 19; k++) {
          const float eu = (cx(k) ? cx(k) * uc : 0.f) + (cy(k) ? cy(k) * vc : 0.f) + (cz(k) ? cz(k) * wc : 0.f);
          const float eh = (cx(k) ? cx(k) * hx : 0.f) + (cy(k) ? cy(k) * hy : 0.f) + (cz(k) ? cz(k) * hz : 0.f);
          const float feq = w19(k) * (fmaf(4.5f * eu, eu, P0) + 3.0f * eu);
          const float fk2 = w19(k) * eh;  // Fk / 2
          fo[k] = f[k] - (f[k] - feq + fk2) * p.itau + 2.0f * fk2;
        }
      }
      // regularised D3Q7 collision, cs^2 = 1/4: g*_k = w_k (S + 4 e_k.(S u/c + (1 - 1/tau_s) j))
      const float jgx = (g[1] - g[3]) - S * uc, jgy = (g[2] - g[4]) - S * vc, jgz = (g[5] - g[6]) - S * wc;
      const float bx = 4.0f * fmaf(p.omg_s, jgx, S * uc), by = 4.0f * fmaf(p.omg_s, jgy, S * vc),
                  bz = 4.0f * fmaf(p.omg_s, jgz, S * wc);
      float go[7];
      go[0] = w7(0) * S;
      go[1] = w7(1) * (S + bx);
      go[3] = w7(3) * (S - bx);
      go[2] = w7(2) * (S + by);
      go[4] = w7(4) * (S - by);
      go[5] = w7(5) * (S + bz);
      go[6] = w7(6) * (S - bz);
      // push streaming with halfway bounce-back (ref: propagation.cu, set_bound.cu:155-159):
      // population k goes to the cell e_k away, or back into this cell's
      // opposite slot where that cell lies outside the box
      float *__restrict__ fo_ = p.f_out + i;
      float *__restrict__ go_ = p.g_out + i;
      const bool bx0 = x > 0, bx1 = x < nx - 1, by0 = y > 0, by1 = y < ny - 1, bz0 = z > 0, bz1 = z < nz - 1;
      auto inside = [&](int k) {
        return (cx(k) > 0 ? bx1 : (cx(k) < 0 ? bx0 : true)) && (cy(k) > 0 ? by1 : (cy(k) < 0 ? by0 : true)) &&
               (cz(k) > 0 ? bz1 : (cz(k) < 0 ? bz0 : true));
      };
#pragma unroll
      for (int k = 0; k < 19; k++) {
        if (inside(k)) fo_[k * N + cz(k) * P + cy(k) * nx + cx(k)] = fo[k];
        else fo_[opp(k) * N] = fo[k];
      }
#pragma unroll
      for (int k = 0; k < 7; k++) {
        if (inside(k)) go_[k * N + cz(k) * P + cy(k) * nx + cx(k)] = go[k];
        else go_[opp(k) * N] = go[k];
      }
      float *__restrict__ Fo = p.F_out + i;
      Fo[0] = Fx;
      Fo[N] = Fy;
      Fo[2 * N] = Fz;
      if (!(isfinite(uc) && isfinite(wc) && isfinite(S) && isfinite(pr))) atomicOr(p.status, 1u);
    }
    __syncthreads();  // the ring slot of z - 1 is overwritten next
  }
}

int launch3d(const Params3 &p, cudaStream_t s) {
  dim3 grid((p.nx + kTX - 1) / kTX, (p.ny + kTY - 1) / kTY, (p.nz + p.zchunk - 1) / p.zchunk);
  step3d_kernel<<<grid, kThreads, 0, s>>>(p);
  return status_from_cuda(cudaGetLastError());
}

}  // namespace f3d
}  // namespace ipcu
