// Moving rigid sphere on the 3-D solver: one 1024-thread CTA per body after
// each fluid step, working in a window box that covers the markers' 4x4x4
// stencils and the previous update's (global-memory scratch, L2-resident):
//   1. markers: position, velocity, stencil origin and Peskin-4 weights per
//      axis, evaluated in index space (a marker at x lies at the continuous
//      cell index s = i + (x - x_i)/(x_{i+1} - x_i); on a uniform axis this
//      is x/dz - 1/2);
//   2. the window cells' velocity u* = c j + (F - f_ib) dt/2rho from the
//      state the fluid step wrote (its force F carries the previous IB
//      force f_ib, which multi-direct forcing finds again as a whole);
//   3. each window cell's (marker, node) pairs, counted, scanned and listed
//      in pair order, so every sum below runs in a fixed order;
//   4. multi-direct forcing, `iters` times: U*_l = sum phi u*,
//      dF_l = 2 rho_f (U_b,l - U*_l)/dt, df = sum dF phi dA / V per cell,
//      u* += df dt/2rho;
//   5. the state's force becomes F - f_ib + f_ib' (so the next step's
//      velocity is the corrected one) and f_ib' replaces f_ib;
//   6. FP64 sums: marker force and torque, fluid momentum and angular
//      momentum inside the sphere (volume fractions clamp(1/2 - d/dz, 0, 1),
//      d = |x - X| - R);
//   7. FP64 body step (one thread): the reaction of the mean of this and the
//      previous step's IB force, buoyancy (1 - rho_f/rho_s) m g along -z
//      (ref: function/ibm.cu:383-396), the change of the fluid momentum
//      inside (Kempe & Froehlich 2012), forward Euler; the orientation
//      advances by the mean angular velocity (Rodrigues), the markers follow
//      (ref: update_IBpoint, ibm.cu:426-447).
// One CTA: the phases synchronise with block barriers; nothing waits on
// another kernel. The marker arrays and the window's pair counts and offsets
// live in shared memory (100 B per marker, 8 B per window cell); the
// window's velocities and force sums and the pair lists in global scratch.
#include <cuda_runtime.h>

#include <climits>

#include "d3q19.cuh"
#include "ibm3d.cuh"
#include "ipcu_common.cuh"

namespace ipcu {
namespace ib3d {
namespace {

constexpr int kWarps = kThreads / 32;

// 4-point Peskin kernel (ref: function/ibm.cu:61-66), r in cell units
__device__ __forceinline__ float peskin4(float r) {
  r = fabsf(r);
  if (r < 1.0f) return (3.0f - 2.0f * r + sqrtf(fmaxf(1.0f + 4.0f * r - 4.0f * r * r, 0.0f))) * 0.125f;
  if (r < 2.0f) return (5.0f - 2.0f * r - sqrtf(fmaxf(-7.0f + 12.0f * r - 4.0f * r * r, 0.0f))) * 0.125f;
  return 0.0f;
}

// continuous cell index of x among n ascending cell centres (linear between
// centres, extended beyond the first and last pair)
__device__ double index_coord(const double *c, int n, double x) {
  int lo = 0, hi = n;  // number of centres <= x
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (c[mid] <= x) lo = mid + 1;
    else hi = mid;
  }
  const int i = min(max(lo - 1, 0), n - 2);
  return i + (x - c[i]) / (c[i + 1] - c[i]);
}

// block sum of v[0..11] (FP64), returned to every thread
__device__ void block_sum12(double (&v)[12], double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < 12; a++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[a] += __shfl_down_sync(0xffffffffu, v[a], o);
  }
  if (lane == 0)
#pragma unroll
    for (int a = 0; a < 12; a++) red[warp * 12 + a] = v[a];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int a = 0; a < 12; a++) {
      double t = 0.0;
      for (int w = 0; w < kWarps; w++) t += red[w * 12 + a];
      red[kWarps * 12 + a] = t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int a = 0; a < 12; a++) v[a] = red[kWarps * 12 + a];
}

// dynamic shared memory of the update: the 227 KB a block may hold, less
// room for its static shared memory (body state, reductions)
constexpr size_t kSmem = 227 * 1024 - 4096;

__global__ void __launch_bounds__(kThreads, 1) ib3d_kernel(const __grid_constant__ Job j) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ Body B;
  __shared__ int bnd[6], bnew[6], s_fail;
  __shared__ int wtot[kWarps];
  __shared__ double red[(kWarps + 1) * 12];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nx = j.nx, ny = j.ny, nz = j.nz, nl = j.nl;
  const long long P = (long long)nx * ny, N = P * nz;
  const double dz = j.dz;
  // shared memory: marker arrays, then the window's counts and offsets
  float *sw = reinterpret_cast<float *>(dsm);  // [nl][12] weights
  int *sorg = reinterpret_cast<int *>(sw + 12 * nl);  // [nl][3]
  float *sub = reinterpret_cast<float *>(sorg + 3 * nl), *sft = sub + 3 * nl, *sdf = sft + 3 * nl;
  float *sdA = sdf + 3 * nl;  // [nl]
  int *soff = reinterpret_cast<int *>(sdA + nl);  // [W + 1]
  const long long wcap = ((long long)kSmem - 100LL * nl) / 8 - 1;  // window cells that fit
  if (tid == 0) {
    B = *j.body;
    for (int a = 0; a < 3; a++) {
      bnew[2 * a] = INT_MAX;
      bnew[2 * a + 1] = INT_MIN;
    }
    s_fail = (nl <= 0 || nl > kMaxMarkers) ? 1 : 0;
  }
  __syncthreads();
  if (s_fail) {
    if (tid == 0) atomicOr(j.status, 8u);
    return;
  }

  // ---- 1. markers
  for (int l = tid; l < nl; l += kThreads) {
    const double r0x = j.r0[3 * l], r0y = j.r0[3 * l + 1], r0z = j.r0[3 * l + 2];
    const double rx = B.R[0] * r0x + B.R[1] * r0y + B.R[2] * r0z;
    const double ry = B.R[3] * r0x + B.R[4] * r0y + B.R[5] * r0z;
    const double rz = B.R[6] * r0x + B.R[7] * r0y + B.R[8] * r0z;
    const double X = B.X[0] + rx, Y = B.X[1] + ry, Z = B.X[2] + rz;
    const double sx = index_coord(j.xc, nx, X), sy = index_coord(j.yc, ny, Y), sz = Z / dz - 0.5;
    const int i0 = (int)floor(sx) - 1, j0 = (int)floor(sy) - 1, k0 = (int)floor(sz) - 1;
    sorg[3 * l] = i0;
    sorg[3 * l + 1] = j0;
    sorg[3 * l + 2] = k0;
#pragma unroll
    for (int a = 0; a < 4; a++) {
      sw[12 * l + a] = peskin4((float)((double)(i0 + a) - sx));
      sw[12 * l + 4 + a] = peskin4((float)((double)(j0 + a) - sy));
      sw[12 * l + 8 + a] = peskin4((float)((double)(k0 + a) - sz));
    }
    sub[3 * l] = (float)(B.U[0] + (B.om[1] * rz - B.om[2] * ry));
    sub[3 * l + 1] = (float)(B.U[1] + (B.om[2] * rx - B.om[0] * rz));
    sub[3 * l + 2] = (float)(B.U[2] + (B.om[0] * ry - B.om[1] * rx));
    sft[3 * l] = sft[3 * l + 1] = sft[3 * l + 2] = 0.f;
    sdA[l] = (float)j.dA[l];
    atomicMin(&bnew[0], i0);
    atomicMax(&bnew[1], i0 + 3);
    atomicMin(&bnew[2], j0);
    atomicMax(&bnew[3], j0 + 3);
    atomicMin(&bnew[4], k0);
    atomicMax(&bnew[5], k0 + 3);
  }
  __syncthreads();
  // the window: the new stencils' box and the previous update's, clipped to the box
  if (tid == 0) {
    for (int a = 0; a < 6; a++) bnd[a] = bnew[a];
    if (B.win[3] > 0) {
      bnd[0] = min(bnd[0], B.win[0]);
      bnd[1] = max(bnd[1], B.win[0] + B.win[3] - 1);
      bnd[2] = min(bnd[2], B.win[1]);
      bnd[3] = max(bnd[3], B.win[1] + B.win[4] - 1);
      bnd[4] = min(bnd[4], B.win[2]);
      bnd[5] = max(bnd[5], B.win[2] + B.win[5] - 1);
    }
    bnd[0] = max(bnd[0], 0);
    bnd[1] = min(bnd[1], nx - 1);
    bnd[2] = max(bnd[2], 0);
    bnd[3] = min(bnd[3], ny - 1);
    bnd[4] = max(bnd[4], 0);
    bnd[5] = min(bnd[5], nz - 1);
    const long long W = (long long)(bnd[1] - bnd[0] + 1) * (bnd[3] - bnd[2] + 1) * (bnd[5] - bnd[4] + 1);
    s_fail = (bnd[1] < bnd[0] || bnd[3] < bnd[2] || bnd[5] < bnd[4] || W > kMaxWin || W > wcap) ? 1 : 0;
  }
  __syncthreads();
  if (s_fail) {
    if (tid == 0) atomicOr(j.status, 8u);
    return;
  }
  const int wi0 = bnd[0], wj0 = bnd[2], wk0 = bnd[4];
  const int WX = bnd[1] - wi0 + 1, WY = bnd[3] - wj0 + 1, WZ = bnd[5] - wk0 + 1;
  const int W = WX * WY * WZ;
  auto cell_of = [&](int c) -> long long {
    const int k = c / (WX * WY), r = c - k * (WX * WY), jj = r / WX, i = r - jj * WX;
    return (long long)(wk0 + k) * P + (long long)(wj0 + jj) * nx + (wi0 + i);
  };

  // ---- 2. window cells: u* from the state, counts and sums cleared
  const float c = j.c;
  for (int cw = tid; cw < W; cw += kThreads) {
    const long long ci = cell_of(cw);
    float jx = 0.f, jy = 0.f, jzm = 0.f, S = 0.f;
#pragma unroll
    for (int k = 0; k < 19; k++) {
      const float v = j.f[k * N + ci];
      if (d3::cx(k)) jx += d3::cx(k) * v;
      if (d3::cy(k)) jy += d3::cy(k) * v;
      if (d3::cz(k)) jzm += d3::cz(k) * v;
    }
#pragma unroll
    for (int k = 0; k < 7; k++) S += j.g[k * N + ci];
    const float h = __fdividef(j.hdt, fmaf(S, j.rsal, j.rho0));
    const float cj[3] = {c * jx, c * jy, c * jzm};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float Fa = j.F[a * N + ci], fe = j.fext[a * N + ci];
      j.wu[a * kMaxWin + cw] = fmaf(Fa, h, cj[a]) - fe * h;
      j.wj[a * kMaxWin + cw] = cj[a];
      j.wf[a * kMaxWin + cw] = 0.f;
    }
    const int k = cw / (WX * WY), r = cw - k * (WX * WY), jj = r / WX, i = r - jj * WX;
    j.wh[cw] = h;
    j.wv[cw] = j.wx[wi0 + i] * j.wy[wj0 + jj] * (float)dz;
    soff[cw] = 0;
  }
  __syncthreads();

  // ---- 3. pairs: count per window cell, scan, list in pair order
  auto pair_cell = [&](int e) -> int {  // window index of pair e = 64 l + node, or -1 outside the box
    const int l = e >> 6, a = e & 63;
    const int i = sorg[3 * l] + (a & 3), jj = sorg[3 * l + 1] + ((a >> 2) & 3), k = sorg[3 * l + 2] + (a >> 4);
    if (i < 0 || i >= nx || jj < 0 || jj >= ny || k < 0 || k >= nz) return -1;
    return ((k - wk0) * WY + (jj - wj0)) * WX + (i - wi0);
  };
  for (int e = tid; e < 64 * nl; e += kThreads) {
    const int cw = pair_cell(e);
    if (cw >= 0) atomicAdd(&soff[cw], 1);
  }
  __syncthreads();
  {
    // exclusive scan of the counts in place: consecutive chunks per thread,
    // then across lanes and warps (the fill cursors start from the offsets)
    const int per = (W + kThreads - 1) / kThreads, b0 = tid * per, b1 = min(b0 + per, W);
    int sum = 0;
    for (int q = b0; q < b1; q++) sum += soff[q];
    int x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wtot[warp] = x;
    __syncthreads();
    if (tid == 0) {
      int run = 0;
      for (int w = 0; w < kWarps; w++) {
        const int t = wtot[w];
        wtot[w] = run;
        run += t;
      }
      soff[W] = run;
    }
    __syncthreads();
    int base = wtot[warp] + x - sum;
    for (int q = b0; q < b1; q++) {
      const int cq = soff[q];
      soff[q] = base;
      j.cur[q] = base;
      base += cq;
    }
  }
  __syncthreads();
  for (int e = tid; e < 64 * nl; e += kThreads) {
    const int cw = pair_cell(e);
    if (cw >= 0) j.list[atomicAdd(&j.cur[cw], 1)] = e;
  }
  __syncthreads();
  for (int cw = tid; cw < W; cw += kThreads) {  // insertion sort of each cell's short list
    const int a0 = soff[cw], a1 = soff[cw + 1];
    for (int a = a0 + 1; a < a1; a++) {
      const int v = j.list[a];
      int b2 = a - 1;
      while (b2 >= a0 && j.list[b2] > v) {
        j.list[b2 + 1] = j.list[b2];
        b2--;
      }
      j.list[b2 + 1] = v;
    }
  }
  __syncthreads();

  // ---- 4. multi-direct forcing
  const float two_rf_dt = (float)(2.0 * j.rho_f / j.dt);
  auto node_w = [&](int l, int a) {
    return sw[12 * l + (a & 3)] * sw[12 * l + 4 + ((a >> 2) & 3)] * sw[12 * l + 8 + (a >> 4)];
  };
  for (int it = 0; it < j.iters; it++) {
    for (int l = tid; l < nl; l += kThreads) {
      float v[3] = {0.f, 0.f, 0.f};
      for (int a = 0; a < 64; a++) {
        const int cw = pair_cell(64 * l + a);
        if (cw < 0) continue;
        const float w = node_w(l, a);
#pragma unroll
        for (int q = 0; q < 3; q++) v[q] = fmaf(w, j.wu[q * kMaxWin + cw], v[q]);
      }
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const float d = two_rf_dt * (sub[3 * l + q] - v[q]);
        sdf[3 * l + q] = d;
        sft[3 * l + q] += d;
      }
    }
    __syncthreads();
    for (int cw = tid; cw < W; cw += kThreads) {
      const int a0 = soff[cw], a1 = soff[cw + 1];
      if (a0 == a1) continue;
      float fx = 0.f, fy = 0.f, fz = 0.f;
      for (int a = a0; a < a1; a++) {
        const int e = j.list[a], l = e >> 6;
        const float wd = node_w(l, e & 63) * sdA[l];
        fx = fmaf(sdf[3 * l], wd, fx);
        fy = fmaf(sdf[3 * l + 1], wd, fy);
        fz = fmaf(sdf[3 * l + 2], wd, fz);
      }
      const float iv = 1.0f / j.wv[cw], h = j.wh[cw];
      fx *= iv;
      fy *= iv;
      fz *= iv;
      j.wu[cw] = fmaf(fx, h, j.wu[cw]);
      j.wu[kMaxWin + cw] = fmaf(fy, h, j.wu[kMaxWin + cw]);
      j.wu[2 * kMaxWin + cw] = fmaf(fz, h, j.wu[2 * kMaxWin + cw]);
      j.wf[cw] += fx;
      j.wf[kMaxWin + cw] += fy;
      j.wf[2 * kMaxWin + cw] += fz;
    }
    __syncthreads();
  }

  // ---- 5. write back: the state's force carries the new IB force
  bool bad = false;
  for (int cw = tid; cw < W; cw += kThreads) {
    const long long ci = cell_of(cw);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float fn = j.wf[a * kMaxWin + cw];
      j.F[a * N + ci] = (j.F[a * N + ci] - j.fext[a * N + ci]) + fn;
      j.fext[a * N + ci] = fn;
      bad |= !isfinite(fn);
    }
  }
  if (bad) atomicOr(j.status, 1u);
  __syncthreads();

  // ---- 6. FP64 sums
  double acc[12];
#pragma unroll
  for (int a = 0; a < 12; a++) acc[a] = 0.0;
  for (int l = tid; l < nl; l += kThreads) {
    const double r0x = j.r0[3 * l], r0y = j.r0[3 * l + 1], r0z = j.r0[3 * l + 2];
    const double rx = B.R[0] * r0x + B.R[1] * r0y + B.R[2] * r0z;
    const double ry = B.R[3] * r0x + B.R[4] * r0y + B.R[5] * r0z;
    const double rz = B.R[6] * r0x + B.R[7] * r0y + B.R[8] * r0z;
    const double fx = (double)sft[3 * l] * j.dA[l], fy = (double)sft[3 * l + 1] * j.dA[l],
                 fz = (double)sft[3 * l + 2] * j.dA[l];
    acc[0] += fx;
    acc[1] += fy;
    acc[2] += fz;
    acc[3] += ry * fz - rz * fy;
    acc[4] += rz * fx - rx * fz;
    acc[5] += rx * fy - ry * fx;
  }
  for (int cw = tid; cw < W; cw += kThreads) {
    const int k = cw / (WX * WY), r = cw - k * (WX * WY), jj = r / WX, i = r - jj * WX;
    const double dx = j.xc[wi0 + i] - B.X[0], dy = j.yc[wj0 + jj] - B.X[1], dzz = (wk0 + k + 0.5) * dz - B.X[2];
    const double d = sqrt(dx * dx + dy * dy + dzz * dzz) - j.radius;
    const double al = fmin(fmax(0.5 - d / dz, 0.0), 1.0) * (double)j.wv[cw];
    if (al > 0.0) {
      const long long ci = cell_of(cw);
      const float h = j.wh[cw];
      const double ux = fmaf(j.F[ci], h, j.wj[cw]), uy = fmaf(j.F[N + ci], h, j.wj[kMaxWin + cw]),
                   uz = fmaf(j.F[2 * N + ci], h, j.wj[2 * kMaxWin + cw]);
      acc[6] += al * ux;
      acc[7] += al * uy;
      acc[8] += al * uz;
      acc[9] += al * (dy * uz - dzz * uy);
      acc[10] += al * (dzz * ux - dx * uz);
      acc[11] += al * (dx * uy - dy * ux);
    }
  }
  block_sum12(acc, red);

  // ---- 7. rigid-body step (FP64, one thread)
  if (tid == 0) {
    Body nb = B;
    const double dt = j.dt, rf = j.rho_f;
    double Fb[3], Tb[3];
    for (int a = 0; a < 3; a++) {
      Fb[a] = -(acc[a] + B.Fib[a]) / 2;
      Tb[a] = -(acc[3 + a] + B.Tib[a]) / 2;
    }
    Fb[2] += -(1.0 - rf / j.rho_s) * j.m * j.grav;
    double om_mean[3];
    for (int a = 0; a < 3; a++) {
      const double P0 = B.have_prev ? B.P[a] : acc[6 + a], L0 = B.have_prev ? B.L[a] : acc[9 + a];
      nb.U[a] = B.U[a] + (dt * Fb[a] + rf * (acc[6 + a] - P0)) / j.m;
      nb.om[a] = B.om[a] + (dt * Tb[a] + rf * (acc[9 + a] - L0)) / j.I;
      nb.X[a] = B.X[a] + dt * (B.U[a] + nb.U[a]) / 2;
      om_mean[a] = dt * (B.om[a] + nb.om[a]) / 2;
      nb.P[a] = acc[6 + a];
      nb.L[a] = acc[9 + a];
      nb.Fib[a] = acc[a];
      nb.Tib[a] = acc[3 + a];
    }
    // R' = rot(om_mean) R (Rodrigues)
    const double th = sqrt(om_mean[0] * om_mean[0] + om_mean[1] * om_mean[1] + om_mean[2] * om_mean[2]);
    if (th > 0.0) {
      const double kx = om_mean[0] / th, ky = om_mean[1] / th, kz = om_mean[2] / th;
      const double s = sin(th), c1 = 1.0 - cos(th);
      const double K[9] = {0, -kz, ky, kz, 0, -kx, -ky, kx, 0};
      double Q[9];
      for (int r = 0; r < 3; r++)
        for (int q = 0; q < 3; q++) {
          double kk = 0.0;
          for (int t = 0; t < 3; t++) kk += K[3 * r + t] * K[3 * t + q];
          Q[3 * r + q] = (r == q ? 1.0 : 0.0) + s * K[3 * r + q] + c1 * kk;
        }
      for (int r = 0; r < 3; r++)
        for (int q = 0; q < 3; q++) {
          double v = 0.0;
          for (int t = 0; t < 3; t++) v += Q[3 * r + t] * B.R[3 * t + q];
          nb.R[3 * r + q] = v;
        }
    }
    // the window whose cells now hold the IB force: the new stencils' box
    nb.win[0] = max(bnew[0], 0);
    nb.win[1] = max(bnew[2], 0);
    nb.win[2] = max(bnew[4], 0);
    nb.win[3] = min(bnew[1], nx - 1) - nb.win[0] + 1;
    nb.win[4] = min(bnew[3], ny - 1) - nb.win[1] + 1;
    nb.win[5] = min(bnew[5], nz - 1) - nb.win[2] + 1;
    if (nb.win[3] <= 0 || nb.win[4] <= 0 || nb.win[5] <= 0) nb.win[3] = 0;
    nb.have_prev = 1;
    *j.body = nb;
  }
}

}  // namespace

int prepare() {
  return status_from_cuda(cudaFuncSetAttribute(ib3d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
}

int launch(const Job &j, cudaStream_t s) {
  ib3d_kernel<<<1, kThreads, kSmem, s>>>(j);
  return status_from_cuda(cudaGetLastError());
}

}  // namespace ib3d
}  // namespace ipcu
