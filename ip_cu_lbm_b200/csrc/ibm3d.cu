// Moving rigid sphere on the 3-D solver, after each fluid step, as a chain
// of kernels (one CTA where a phase is serial, a grid where it is wide), in
// a window box that covers every marker's 4x4x4 stencil (the sphere's box
// in index space) and the previous update's:
//   1. set-up (one CTA): the plan (window and stencil-origin bin boxes);
//      markers: position, velocity, stencil origin and Peskin-4 weights per
//      axis, evaluated in index space (a marker at x lies at the continuous
//      cell index s = i + (x - x_i)/(x_{i+1} - x_i); on a uniform axis this
//      is x/dz - 1/2), binned by stencil origin, each bin in marker order;
//   2. window (grid): u* = c j + (F - f_ib) dt/2rho from the state the fluid
//      step wrote (its force F carries the previous IB force f_ib, which
//      multi-direct forcing finds again as a whole), and each window cell's
//      contributions (marker, node) from the bins, by node then marker, so
//      every sum below runs in a fixed order;
//   3. multi-direct forcing, `iters` times: interpolation (grid over the
//      markers) U*_l = sum phi u*, dF_l = 2 rho_f (U_b,l - U*_l)/dt; spread
//      (grid over the window) df = sum dF phi dA / V, u* += df dt/2rho;
//   4. write-back (grid): the state's force becomes F - f_ib + f_ib' (so the
//      next step's velocity is the corrected one) and f_ib' replaces f_ib;
//   5. FP64 sums: partials in fixed blocks (grid), added in a fixed order by
//      one CTA: marker force and torque, fluid momentum and angular momentum
//      inside the sphere (volume fractions clamp(1/2 - d/dz, 0, 1),
//      d = |x - X| - R);
//   6. FP64 body step (one thread): the reaction of the mean of this and the
//      previous step's IB force, buoyancy (1 - rho_f/rho_s) m g along -z
//      (ref: function/ibm.cu:383-396), the change of the fluid momentum
//      inside (Kempe & Froehlich 2012), forward Euler; the orientation
//      advances by the mean angular velocity (Rodrigues), the markers follow
//      (ref: update_IBpoint, ibm.cu:426-447).
// Every kernel is ordered after the previous one on the stream; nothing
// waits on another kernel.
#include <cuda_runtime.h>

#include <climits>

#include "d3q19.cuh"
#include "ibm3d.cuh"
#include "ipcu_common.cuh"
#include "store3d.cuh"

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

// The cells a sphere's marker stencils can touch: along each axis
// [floor(s(X - R)) - 1, floor(s(X + R)) + 2] with s the continuous cell index
// (monotonic, so every marker's 4-node stencil lies inside), unclipped.
__device__ void sphere_box(const Job &j, const double *X, int (&lo)[3], int (&hi)[3]) {
  const double R = j.radius;
  const double s0[3] = {index_coord(j.xc, j.nx, X[0] - R), index_coord(j.yc, j.ny, X[1] - R), (X[2] - R) / j.dz - 0.5};
  const double s1[3] = {index_coord(j.xc, j.nx, X[0] + R), index_coord(j.yc, j.ny, X[1] + R), (X[2] + R) / j.dz - 0.5};
  for (int a = 0; a < 3; a++) {
    lo[a] = (int)floor(s0[a]) - 1;
    hi[a] = (int)floor(s1[a]) + 2;
  }
}

__device__ __forceinline__ float node_weight(const float *mw, int l, int a) {
  return mw[12 * l + (a & 3)] * mw[12 * l + 4 + ((a >> 2) & 3)] * mw[12 * l + 8 + (a >> 4)];
}

// ---- 1. set-up: plan, markers, origin bins (one CTA)
__global__ void __launch_bounds__(kThreads, 1) ib3d_setup_kernel(const __grid_constant__ Job j) {
  __shared__ Body B;
  __shared__ Plan pl;
  __shared__ int wtot[kWarps];
  extern __shared__ int bcur[];  // [kMaxBins] counts, then fill cursors
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nx = j.nx, ny = j.ny, nz = j.nz, nl = j.nl;
  if (tid == 0) {
    B = *j.body;
    int lo[3], hi[3];
    sphere_box(j, B.X, lo, hi);
    int w0[3], w1[3];
    const int n3[3] = {nx, ny, nz};
    bool ok = nl > 0 && nl <= kMaxMarkers;
    for (int a = 0; a < 3; a++) {
      pl.olo[a] = lo[a];
      pl.on[a] = hi[a] - 3 - lo[a] + 1;
      w0[a] = lo[a];
      w1[a] = hi[a];
      if (B.win[3] > 0) {
        w0[a] = min(w0[a], B.win[a]);
        w1[a] = max(w1[a], B.win[a] + B.win[3 + a] - 1);
      }
      w0[a] = max(w0[a], 0);
      w1[a] = min(w1[a], n3[a] - 1);
      ok = ok && w1[a] >= w0[a];
      pl.win[a] = w0[a];
      pl.win[3 + a] = w1[a] - w0[a] + 1;
    }
    const long long W = (long long)pl.win[3] * pl.win[4] * pl.win[5];
    const long long NB = (long long)pl.on[0] * pl.on[1] * pl.on[2];
    ok = ok && W <= kMaxWin && NB <= kMaxBins;
    pl.W = ok ? (int)W : 0;
    pl.NB = ok ? (int)NB : 0;
    pl.ok = ok ? 1 : 0;
    *j.plan = pl;
    if (!ok) atomicOr(j.status, 8u);
  }
  __syncthreads();
  if (!pl.ok) return;
  const int OX = pl.on[0], OY = pl.on[1], NB = pl.NB;
  for (int b = tid; b < NB; b += kThreads) bcur[b] = 0;
  __syncthreads();
  const double dz = j.dz;
  for (int l = tid; l < nl; l += kThreads) {
    const double r0x = j.r0[3 * l], r0y = j.r0[3 * l + 1], r0z = j.r0[3 * l + 2];
    const double rx = B.R[0] * r0x + B.R[1] * r0y + B.R[2] * r0z;
    const double ry = B.R[3] * r0x + B.R[4] * r0y + B.R[5] * r0z;
    const double rz = B.R[6] * r0x + B.R[7] * r0y + B.R[8] * r0z;
    const double X = B.X[0] + rx, Y = B.X[1] + ry, Z = B.X[2] + rz;
    const double sx = index_coord(j.xc, nx, X), sy = index_coord(j.yc, ny, Y), sz = Z / dz - 0.5;
    const int i0 = (int)floor(sx) - 1, j0 = (int)floor(sy) - 1, k0 = (int)floor(sz) - 1;
    j.morg[3 * l] = i0;
    j.morg[3 * l + 1] = j0;
    j.morg[3 * l + 2] = k0;
#pragma unroll
    for (int a = 0; a < 4; a++) {
      j.mw[12 * l + a] = peskin4((float)((double)(i0 + a) - sx));
      j.mw[12 * l + 4 + a] = peskin4((float)((double)(j0 + a) - sy));
      j.mw[12 * l + 8 + a] = peskin4((float)((double)(k0 + a) - sz));
    }
    j.mub[3 * l] = (float)(B.U[0] + (B.om[1] * rz - B.om[2] * ry));
    j.mub[3 * l + 1] = (float)(B.U[1] + (B.om[2] * rx - B.om[0] * rz));
    j.mub[3 * l + 2] = (float)(B.U[2] + (B.om[0] * ry - B.om[1] * rx));
    j.mft[3 * l] = j.mft[3 * l + 1] = j.mft[3 * l + 2] = 0.f;
    atomicAdd(&bcur[((k0 - pl.olo[2]) * OY + (j0 - pl.olo[1])) * OX + (i0 - pl.olo[0])], 1);
  }
  __syncthreads();
  {
    // exclusive scan of the bin counts: consecutive chunks per thread, then
    // across lanes and warps; the cursors start at the offsets
    const int per = (NB + kThreads - 1) / kThreads, b0 = tid * per, b1 = min(b0 + per, NB);
    int sum = 0;
    for (int q = b0; q < b1; q++) sum += bcur[q];
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
      j.bstart[NB] = run;
    }
    __syncthreads();
    int base = wtot[warp] + x - sum;
    for (int q = b0; q < b1; q++) {
      const int cq = bcur[q];
      j.bstart[q] = base;
      bcur[q] = base;
      base += cq;
    }
  }
  __syncthreads();
  for (int l = tid; l < nl; l += kThreads) {
    const int b = ((j.morg[3 * l + 2] - pl.olo[2]) * OY + (j.morg[3 * l + 1] - pl.olo[1])) * OX +
                  (j.morg[3 * l] - pl.olo[0]);
    j.blist[atomicAdd(&bcur[b], 1)] = l;
  }
  __syncthreads();
  for (int b = tid; b < NB; b += kThreads) {  // each bin's few markers in index order
    const int a0 = j.bstart[b], a1 = j.bstart[b + 1];
    for (int a = a0 + 1; a < a1; a++) {
      const int v = j.blist[a];
      int b2 = a - 1;
      while (b2 >= a0 && j.blist[b2] > v) {
        j.blist[b2 + 1] = j.blist[b2];
        b2--;
      }
      j.blist[b2 + 1] = v;
    }
  }
}

// ---- 2. window cells (grid): u*, and the contribution lists
__global__ void __launch_bounds__(256) ib3d_window_kernel(const __grid_constant__ Job j) {
  const Plan pl = *j.plan;
  if (!pl.ok) return;
  const int WX = pl.win[3], WY = pl.win[4], W = pl.W;
  const int OX = pl.on[0], OY = pl.on[1], OZ = pl.on[2];
  const long long P = (long long)j.nx * j.ny, N = P * j.nz;
  const float c = j.c;
  for (int cw = blockIdx.x * blockDim.x + threadIdx.x; cw < W; cw += gridDim.x * blockDim.x) {
    const int k = cw / (WX * WY), r = cw - k * (WX * WY), jj = r / WX, i = r - jj * WX;
    const int gi = pl.win[0] + i, gj = pl.win[1] + jj, gk = pl.win[2] + k;
    const long long ci = (long long)gk * P + (long long)gj * j.nx + gi;
    float jx = 0.f, jy = 0.f, jzm = 0.f, S = 0.f;
    float f[19], g[7];
    if (j.store == IPCU_STORE_F16) s3::load_cell<__half>(j.f, j.g, j.r, ci, N, j.inv_scale, f, g);
    else if (j.store == IPCU_STORE_BF16) s3::load_cell<__nv_bfloat16>(j.f, j.g, j.r, ci, N, j.inv_scale, f, g);
    else s3::load_cell<float>(j.f, j.g, j.r, ci, N, j.inv_scale, f, g);
#pragma unroll
    for (int q = 0; q < 19; q++) {
      const float v = f[q];
      if (d3::cx(q)) jx += d3::cx(q) * v;
      if (d3::cy(q)) jy += d3::cy(q) * v;
      if (d3::cz(q)) jzm += d3::cz(q) * v;
    }
#pragma unroll
    for (int q = 0; q < 7; q++) S += g[q];
    const float h = __fdividef(j.hdt, fmaf(S, j.rsal, j.rho0));
    const float cj[3] = {c * jx, c * jy, c * jzm};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float Fa = j.F[a * N + ci], fe = j.fext[a * N + ci];
      j.wu[a * kMaxWin + cw] = fmaf(Fa, h, cj[a]) - fe * h;
      j.wj[a * kMaxWin + cw] = cj[a];
      j.wf[a * kMaxWin + cw] = 0.f;
    }
    j.wh[cw] = h;
    j.wv[cw] = j.wx[gi] * j.wy[gj] * (float)j.dz;
    // contributions: the markers whose stencil origin is this cell less a
    // node offset, by node and then marker index
    int t = 0;
    for (int a = 0; a < 64; a++) {
      const int oi = gi - (a & 3) - pl.olo[0], oj = gj - ((a >> 2) & 3) - pl.olo[1], ok = gk - (a >> 4) - pl.olo[2];
      if (oi < 0 || oi >= OX || oj < 0 || oj >= OY || ok < 0 || ok >= OZ) continue;
      const int b = (ok * OY + oj) * OX + oi;
      for (int q = j.bstart[b]; q < j.bstart[b + 1]; q++) {
        if (t < kSlots) j.clist[(long long)cw * kSlots + t] = (j.blist[q] << 6) | a;
        t++;
      }
    }
    if (t > kSlots) atomicOr(j.status, 8u);
    j.ccnt[cw] = min(t, kSlots);
  }
}

// ---- 3a. interpolation at the markers (grid over markers)
__global__ void __launch_bounds__(256) ib3d_interp_kernel(const __grid_constant__ Job j) {
  const Plan pl = *j.plan;
  if (!pl.ok) return;
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= j.nl) return;
  const int WX = pl.win[3], WY = pl.win[4];
  const int i0 = j.morg[3 * l], j0 = j.morg[3 * l + 1], k0 = j.morg[3 * l + 2];
  float v[3] = {0.f, 0.f, 0.f};
#pragma unroll 8
  for (int a = 0; a < 64; a++) {
    const int i = i0 + (a & 3), jj = j0 + ((a >> 2) & 3), k = k0 + (a >> 4);
    if (i < 0 || i >= j.nx || jj < 0 || jj >= j.ny || k < 0 || k >= j.nz) continue;
    const int cw = ((k - pl.win[2]) * WY + (jj - pl.win[1])) * WX + (i - pl.win[0]);
    const float w = node_weight(j.mw, l, a);
#pragma unroll
    for (int q = 0; q < 3; q++) v[q] = fmaf(w, j.wu[q * kMaxWin + cw], v[q]);
  }
  const float two_rf_dt = (float)(2.0 * j.rho_f / j.dt);
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const float d = two_rf_dt * (j.mub[3 * l + q] - v[q]);
    j.mdf[3 * l + q] = d;
    j.mft[3 * l + q] += d;
  }
}

// ---- 3b. spread to the window cells (grid over the window)
__global__ void __launch_bounds__(256) ib3d_spread_kernel(const __grid_constant__ Job j) {
  const Plan pl = *j.plan;
  if (!pl.ok) return;
  for (int cw = blockIdx.x * blockDim.x + threadIdx.x; cw < pl.W; cw += gridDim.x * blockDim.x) {
    const int nc = j.ccnt[cw];
    if (nc == 0) continue;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    for (int t = 0; t < nc; t++) {
      const int e = j.clist[(long long)cw * kSlots + t], l = e >> 6;
      const float wd = node_weight(j.mw, l, e & 63) * (float)j.dA[l];
      fx = fmaf(j.mdf[3 * l], wd, fx);
      fy = fmaf(j.mdf[3 * l + 1], wd, fy);
      fz = fmaf(j.mdf[3 * l + 2], wd, fz);
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
}

// ---- 4. write back and 5. partial sums (grid of kParts CTAs, fixed
// blocks of window cells and markers each)
__global__ void __launch_bounds__(256) ib3d_writeback_kernel(const __grid_constant__ Job j) {
  __shared__ double red[8 * 12];
  const Plan pl = *j.plan;
  if (!pl.ok) return;
  const int WX = pl.win[3], WY = pl.win[4], W = pl.W;
  const long long P = (long long)j.nx * j.ny, N = P * j.nz;
  const Body *B = j.body;
  const double X0 = B->X[0], X1 = B->X[1], X2 = B->X[2], dz = j.dz;
  double acc[12];
#pragma unroll
  for (int a = 0; a < 12; a++) acc[a] = 0.0;
  bool bad = false;
  const int chunk = (W + kParts - 1) / kParts, c0 = blockIdx.x * chunk, c1 = min(c0 + chunk, W);
  for (int cw = c0 + threadIdx.x; cw < c1; cw += blockDim.x) {
    const int k = cw / (WX * WY), r = cw - k * (WX * WY), jj = r / WX, i = r - jj * WX;
    const long long ci = (long long)(pl.win[2] + k) * P + (long long)(pl.win[1] + jj) * j.nx + (pl.win[0] + i);
    float Fn[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const float fn = j.wf[a * kMaxWin + cw];
      Fn[a] = (j.F[a * N + ci] - j.fext[a * N + ci]) + fn;
      j.F[a * N + ci] = Fn[a];
      j.fext[a * N + ci] = fn;
      bad |= !isfinite(fn);
    }
    // fluid momentum inside the sphere, from the corrected state
    const double dx = j.xc[pl.win[0] + i] - X0, dy = j.yc[pl.win[1] + jj] - X1, dzz = (pl.win[2] + k + 0.5) * dz - X2;
    const double d = sqrt(dx * dx + dy * dy + dzz * dzz) - j.radius;
    const double al = fmin(fmax(0.5 - d / dz, 0.0), 1.0) * (double)j.wv[cw];
    if (al > 0.0) {
      const float h = j.wh[cw];
      const double ux = fmaf(Fn[0], h, j.wj[cw]), uy = fmaf(Fn[1], h, j.wj[kMaxWin + cw]),
                   uz = fmaf(Fn[2], h, j.wj[2 * kMaxWin + cw]);
      acc[6] += al * ux;
      acc[7] += al * uy;
      acc[8] += al * uz;
      acc[9] += al * (dy * uz - dzz * uy);
      acc[10] += al * (dzz * ux - dx * uz);
      acc[11] += al * (dx * uy - dy * ux);
    }
  }
  if (bad) atomicOr(j.status, 1u);
  // marker force and torque, in the same fixed blocks
  const int mchunk = (j.nl + kParts - 1) / kParts, m0 = blockIdx.x * mchunk, m1 = min(m0 + mchunk, j.nl);
  for (int l = m0 + threadIdx.x; l < m1; l += blockDim.x) {
    const double r0x = j.r0[3 * l], r0y = j.r0[3 * l + 1], r0z = j.r0[3 * l + 2];
    const double rx = B->R[0] * r0x + B->R[1] * r0y + B->R[2] * r0z;
    const double ry = B->R[3] * r0x + B->R[4] * r0y + B->R[5] * r0z;
    const double rz = B->R[6] * r0x + B->R[7] * r0y + B->R[8] * r0z;
    const double fx = (double)j.mft[3 * l] * j.dA[l], fy = (double)j.mft[3 * l + 1] * j.dA[l],
                 fz = (double)j.mft[3 * l + 2] * j.dA[l];
    acc[0] += fx;
    acc[1] += fy;
    acc[2] += fz;
    acc[3] += ry * fz - rz * fy;
    acc[4] += rz * fx - rx * fz;
    acc[5] += rx * fy - ry * fx;
  }
  // block sum in a fixed order: warps, then the block's warps in sequence
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int a = 0; a < 12; a++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[a] += __shfl_down_sync(0xffffffffu, acc[a], o);
  }
  if (lane == 0)
#pragma unroll
    for (int a = 0; a < 12; a++) red[warp * 12 + a] = acc[a];
  __syncthreads();
  if (threadIdx.x < 12) {
    double t = 0.0;
    for (int w = 0; w < 8; w++) t += red[w * 12 + threadIdx.x];
    j.part[blockIdx.x * 12 + threadIdx.x] = t;
  }
}

// ---- 6. the partials added in block order, and the body step (one CTA)
__global__ void __launch_bounds__(32) ib3d_body_kernel(const __grid_constant__ Job j) {
  const Plan pl = *j.plan;
  if (!pl.ok) return;
  __shared__ double acc[12];
  if (threadIdx.x < 12) {
    double t = 0.0;
    for (int b = 0; b < kParts; b++) t += j.part[b * 12 + threadIdx.x];
    acc[threadIdx.x] = t;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const Body B = *j.body;
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
  // the cells that now hold the IB force: this update's sphere box, clipped
  {
    int lo[3], hi[3];
    sphere_box(j, B.X, lo, hi);
    const int n3[3] = {j.nx, j.ny, j.nz};
    nb.win[3] = 1;
    for (int a = 0; a < 3; a++) {
      lo[a] = max(lo[a], 0);
      hi[a] = min(hi[a], n3[a] - 1);
      nb.win[a] = lo[a];
      nb.win[3 + a] = hi[a] - lo[a] + 1;
      if (hi[a] < lo[a]) nb.win[3] = 0;
    }
  }
  nb.have_prev = 1;
  *j.body = nb;
}

}  // namespace

int prepare() {
  return status_from_cuda(cudaFuncSetAttribute(ib3d_setup_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)(sizeof(int) * kMaxBins)));
}

int launch(const Job &j, cudaStream_t s) {
  const int wgrid = 148 * 2;  // window cells: up to 64K, ~2 CTAs per SM looping
  ib3d_setup_kernel<<<1, kThreads, sizeof(int) * kMaxBins, s>>>(j);
  ib3d_window_kernel<<<wgrid, 256, 0, s>>>(j);
  for (int it = 0; it < j.iters; it++) {
    ib3d_interp_kernel<<<(j.nl + 255) / 256, 256, 0, s>>>(j);
    ib3d_spread_kernel<<<wgrid, 256, 0, s>>>(j);
  }
  ib3d_writeback_kernel<<<kParts, 256, 0, s>>>(j);
  ib3d_body_kernel<<<1, 32, 0, s>>>(j);
  return status_from_cuda(cudaGetLastError());
}

}  // namespace ib3d
}  // namespace ipcu
