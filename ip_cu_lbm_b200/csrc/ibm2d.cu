// Moving immersed boundary for the fused 2-D solver: one CTA per body runs,
// after each fluid step, the whole coupled update on the body's footprint.
//
// The fluid step added the previous IB force density f_ib to the cell force
// (fused kernel), so the new velocity u = c j + (F + f_ib) dt / 2 rho holds
// half of it. The update (uniform lattice, cell centres (i + 1/2) dz):
//   1. markers X_l = X + R(theta) X0_l, U_b,l = U + omega x r_l (FP64, as
//      update_IBpoint, ref: function/ibm.cu:426-447), and their 4x4 Peskin
//      stencils (ref: function/ibm.cu:61-66 weightFunction);
//   2. the cells of the previous and the new stencils get shared-memory
//      slots (a window map over their bounding box); the old force's half
//      is taken out of u there and f_ib restarts at zero;
//   3. multi-direct forcing, `iters` times: U*_l = sum phi u (one thread
//      per marker, a fixed pairwise sum over its 16 nodes), dF_l = 2 rho_f
//      (U_b,l - U*_l) / dt,
//      spread df = dF_l phi dS_l / dz^2 onto f_ib and df dt / 2 rho onto u,
//      F_l += dF_l; each slot gathers its (marker, cell) pairs from a list
//      sorted by pair index, so every sum runs in a fixed order and a
//      body's update is the same whatever runs beside it;
//   4. u and f_ib go back to HBM (16-bit storage re-expresses the stored
//      deviations about the new u, so the populations stay as they were).
//      The tile flags the fluid kernel reads follow the footprint. The
//      next fluid step may run beside this update (programmatic dependent
//      launch; the update lets it go at its start): its flagged tiles wait
//      for the update, the others run on. It needs flags on the previous
//      and this step's footprints, the cells this update writes; both are
//      set one update ahead, since each update ends by flagging the
//      footprint its successor will have (the successor starts from the
//      body state this one leaves). The first update flags its own
//      footprint before it lets the fluid step go. Tiles of the footprint
//      two steps back that none of the previous, current and next
//      footprints covers are unflagged;
//   5. FP64 sums: F_ib = sum F_l dS_l, T_ib = sum r_l x F_l dS_l and the
//      fluid momentum P, angular momentum L inside the body, each cell
//      weighted by its volume fraction alpha = clamp(1/2 - d/dz, 0, 1), d the
//      signed distance of its centre from the ellipse (first-order estimate
//      F/|grad F| of F = (x/a)^2 + (z/b)^2 - 1 in the body frame; a binary
//      inside test would kick the body whenever a centre crosses the outline);
//   6. one thread steps the body in FP64 (update_IBbody's force, torque and
//      buoyancy (1 - rho_f/rho_s) m g, ref: function/ibm.cu:367-424): the
//      body takes the reaction of the mean of this step's and the previous
//      step's IB force (the fluid's momentum changes by that mean) plus the
//      change of the fluid momentum inside it, with forward Euler for the
//      velocities and the trapezoidal rule for position and angle:
//        m (U' - U) = -dt (F_ib + F_ib,old)/2 + rho_f (P - P_old) + buoyancy,
//        I (w' - w) = -dt (T_ib + T_ib,old)/2 + rho_f (L - L_old).
// Overflow of the marker, window or slot capacity sets status bit 8 and
// leaves the state untouched.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "fused2d_impl.cuh"
#include "ibm2d.cuh"
#include "ipcu_common.cuh"
#include "storage.cuh"

namespace ipcu {
namespace ib2d {

namespace {

// Velocity of cell ci in buffer b, the one the fluid step wrote: its
// velocity planes, or, after a lean flow-only step, c j + F dt / 2 rho from
// the populations and the force that step applied (f2d::lean_velocity: the
// value the full step would have stored, bit for bit).
__device__ __forceinline__ void vel_at(const f2d::Params &p, int b, const float *mac, long long ci, long long N,
                                       float &ux, float &uz) {
  if (p.lean) {
    f2d::lean_velocity(p, b, ci, N, ux, uz);
    return;
  }
  ux = mac[N + ci];
  uz = mac[2 * N + ci];
}

constexpr int kWarps = kThreads / 32;
constexpr int kTileMap = 1024;          // tiles tracked around the footprints for the flag clean-up

// 4-point Peskin kernel (ref: function/ibm.cu:61-66), r in lattice spacings
__device__ __forceinline__ float peskin4(float r) {
  r = fabsf(r);
  if (r < 1.0f) return (3.0f - 2.0f * r + sqrtf(fmaxf(1.0f + 4.0f * r - 4.0f * r * r, 0.0f))) * 0.125f;
  if (r < 2.0f) return (5.0f - 2.0f * r - sqrtf(fmaxf(-7.0f + 12.0f * r - 4.0f * r * r, 0.0f))) * 0.125f;
  return 0.0f;
}

struct Layout {
  // markers
  static constexpr size_t I0 = 0;                                   // int [nl] stencil origin x
  static constexpr size_t K0 = I0 + 4 * kMaxMarkers;                 // int [nl] origin z
  static constexpr size_t WX = K0 + 4 * kMaxMarkers;                 // float [nl][4]
  static constexpr size_t WZ = WX + 16 * kMaxMarkers;                // float [nl][4]
  static constexpr size_t UB = WZ + 16 * kMaxMarkers;                // float [nl][2] body velocity at the marker
  static constexpr size_t DF = UB + 8 * kMaxMarkers;                 // float [nl][2] this iteration's force
  static constexpr size_t FT = DF + 8 * kMaxMarkers;                 // float [nl][2] accumulated force
  static constexpr size_t DS = FT + 8 * kMaxMarkers;                 // float [nl] dS / dz^2
  // slots
  static constexpr size_t CELL = DS + 4 * kMaxMarkers;               // int [slots] cell index
  static constexpr size_t SU = CELL + 4 * kMaxSlots;                 // float [slots] u_x
  static constexpr size_t SW = SU + 4 * kMaxSlots;                   // float [slots] u_z
  static constexpr size_t SFX = SW + 4 * kMaxSlots;                  // float [slots] f_ib x
  static constexpr size_t SFZ = SFX + 4 * kMaxSlots;                 // float [slots] f_ib z
  static constexpr size_t SH = SFZ + 4 * kMaxSlots;                  // float [slots] dt / 2 rho
  static constexpr size_t OFF = SH + 4 * kMaxSlots;                  // int [slots + 1] first pair of a slot
  static constexpr size_t CUR = OFF + 4 * (kMaxSlots + 1);           // int [slots] count, then write cursor
  static constexpr size_t LIST = CUR + 4 * kMaxSlots;                // short [16 nl] pairs l*16+q by slot
  static constexpr size_t PS = LIST + 2 * 16 * kMaxMarkers;          // short [16 nl] slot of each pair (-1 outside)
  static constexpr size_t MAP = PS + 2 * 16 * kMaxMarkers;           // short [window] slot of a window cell
  static constexpr size_t WL = (MAP + 2 * kMaxWindow + 15) / 16 * 16;  // float [16 nl] spread weight of each list entry
  static constexpr size_t RED = WL + 4 * 16 * kMaxMarkers;              // double [kWarps][6]
  static constexpr size_t BYTES = RED + 8 * 6 * kWarps;
};
static_assert(Layout::BYTES + 2048 <= 227 * 1024, "the update's dynamic and static shared memory");

template <class ST, int QS>
__device__ void coupled_update(const Job &j, int parity) {
  extern __shared__ __align__(16) unsigned char sm[];
  int *sI0 = reinterpret_cast<int *>(sm + Layout::I0);
  int *sK0 = reinterpret_cast<int *>(sm + Layout::K0);
  float *sWX = reinterpret_cast<float *>(sm + Layout::WX);
  float *sWZ = reinterpret_cast<float *>(sm + Layout::WZ);
  float *sUB = reinterpret_cast<float *>(sm + Layout::UB);
  float *sDF = reinterpret_cast<float *>(sm + Layout::DF);
  float *sFT = reinterpret_cast<float *>(sm + Layout::FT);
  float *sDS = reinterpret_cast<float *>(sm + Layout::DS);
  int *sCell = reinterpret_cast<int *>(sm + Layout::CELL);
  float *sU = reinterpret_cast<float *>(sm + Layout::SU);
  float *sW = reinterpret_cast<float *>(sm + Layout::SW);
  float *sFX = reinterpret_cast<float *>(sm + Layout::SFX);
  float *sFZ = reinterpret_cast<float *>(sm + Layout::SFZ);
  float *sH = reinterpret_cast<float *>(sm + Layout::SH);
  int *sOff = reinterpret_cast<int *>(sm + Layout::OFF);
  int *sCur = reinterpret_cast<int *>(sm + Layout::CUR);
  short *sList = reinterpret_cast<short *>(sm + Layout::LIST);
  short *sPS = reinterpret_cast<short *>(sm + Layout::PS);
  short *sMap = reinterpret_cast<short *>(sm + Layout::MAP);
  float *sWL = reinterpret_cast<float *>(sm + Layout::WL);
  double *sRed = reinterpret_cast<double *>(sm + Layout::RED);
  __shared__ Body B;
  __shared__ int bnd[4];   // window bounds imin, imax, kmin, kmax
  __shared__ int bnd2[4];  // bounds of the footprint two steps back
  __shared__ int bnd3[4];  // bounds of the next step's footprint
  __shared__ uint8_t tmap[kTileMap];  // tiles of the previous, current and next footprints
  __shared__ int nslot, fail;

  const f2d::Params &p = j.fp;
  // launched as a programmatic dependent of the fluid step: nothing is read
  // before that step has completed (a no-op for an ordinary launch)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nx = p.nx, nz = p.nz, nl = j.nl;
  const long long N = (long long)nx * nz;
  const int b = p.cur ^ parity ^ 1;  // the buffer the fluid step wrote
  float *mac = p.mbuf[b];
  const double dz = j.dz, idz = 1.0 / dz;

  // this thread's marker (nl <= kMaxMarkers = kThreads: at most one),
  // loaded while thread 0 fetches the body
  double px0 = 0.0, pz0 = 0.0, pdS = 0.0;
  int porg[4] = {0, 0, 0, 0};
  if (tid < nl) {
    px0 = j.X0[2 * tid];
    pz0 = j.X0[2 * tid + 1];
    pdS = j.dS[tid];
    porg[0] = j.org[2 * tid];
    porg[1] = j.org[2 * tid + 1];
    porg[2] = j.org2[2 * tid];
    porg[3] = j.org2[2 * tid + 1];
  }
  if (tid == 0) {
    B = *j.body;
    bnd[0] = bnd[2] = bnd2[0] = bnd2[2] = bnd3[0] = bnd3[2] = INT_MAX;
    bnd[1] = bnd[3] = bnd2[1] = bnd2[3] = bnd3[1] = bnd3[3] = INT_MIN;
    nslot = 0;
    fail = nl > kMaxMarkers ? 1 : 0;
  }
  __syncthreads();
  if (fail) {
    if (tid == 0) atomicOr(p.status, 8u);
    return;
  }
  const bool have_prev = B.have_prev != 0, have_prev2 = B.have_prev2 != 0;
  // the footprint of this step was flagged by the previous update
  if (have_prev) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const double cth = cos(B.th), sth = sin(B.th);

  // window bounds: each thread's own, then one shared atomic per warp
  int bx[12] = {INT_MAX, INT_MIN, INT_MAX, INT_MIN, INT_MAX, INT_MIN, INT_MAX, INT_MIN,
                INT_MAX, INT_MIN, INT_MAX, INT_MIN};
  auto take_box = [&](int *box, int i0, int k0) {
    box[0] = min(box[0], i0);
    box[1] = max(box[1], i0 + 3);
    box[2] = min(box[2], k0);
    box[3] = max(box[3], k0 + 3);
  };
  auto merge_box = [&](const int *box, int *dst) {
    const int a = __reduce_min_sync(0xffffffffu, box[0]), b2 = __reduce_max_sync(0xffffffffu, box[1]);
    const int c = __reduce_min_sync(0xffffffffu, box[2]), d = __reduce_max_sync(0xffffffffu, box[3]);
    if (lane == 0) {
      atomicMin(&dst[0], a);
      atomicMax(&dst[1], b2);
      atomicMin(&dst[2], c);
      atomicMax(&dst[3], d);
    }
  };

  // ---- 1. markers: position, velocity, stencil origin and weights
  static_assert(kMaxMarkers <= kThreads, "one marker per thread at most");
  if (tid < nl) {
    const int l = tid;
    const double x0 = px0, z0 = pz0;
    const double rx = cth * x0 - sth * z0, rz = sth * x0 + cth * z0;
    const double X = B.X[0] + rx, Z = B.X[1] + rz;
    const double xs = X * idz - 0.5, zs = Z * idz - 0.5;  // in cell-index units
    const int i0 = (int)floor(xs) - 1, k0 = (int)floor(zs) - 1;
    sI0[l] = i0;
    sK0[l] = k0;
#pragma unroll
    for (int a = 0; a < 4; a++) {
      sWX[4 * l + a] = peskin4((float)((double)(i0 + a) - xs));
      sWZ[4 * l + a] = peskin4((float)((double)(k0 + a) - zs));
    }
    sUB[2 * l] = (float)(B.U[0] - B.om * rz);
    sUB[2 * l + 1] = (float)(B.U[1] + B.om * rx);
    sFT[2 * l] = sFT[2 * l + 1] = 0.f;
    sDS[l] = (float)(pdS * idz * idz);
    take_box(bx, i0, k0);
    if (have_prev2) take_box(bx + 4, porg[2], porg[3]);
    if (have_prev) take_box(bx, porg[0], porg[1]);
  }
  merge_box(bx, bnd);
  merge_box(bx + 4, bnd2);
  __syncthreads();
  const int wi0 = bnd[0], wk0 = bnd[2], WW = bnd[1] - bnd[0] + 1, WH = bnd[3] - bnd[2] + 1;
  if (nl == 0 || (long long)WW * WH > kMaxWindow) {
    if (tid == 0 && nl > 0) atomicOr(p.status, 8u);
    return;
  }
  const int nwin = WW * WH;

  // ---- 2. slots for the cells of the old and new stencils inside the box
  for (int e = tid; e < nwin; e += kThreads) sMap[e] = -1;
  __syncthreads();
  for (int e = tid; e < 16 * nl; e += kThreads) {
    const int l = e >> 4, i = sI0[l] + (e & 3), k = sK0[l] + ((e >> 2) & 3);
    if (i >= 0 && i < nx && k >= 0 && k < nz) sMap[(k - wk0) * WW + (i - wi0)] = -2;
  }
  if (have_prev)
    for (int e = tid; e < 16 * nl; e += kThreads) {
      const int l = e >> 4, i = j.org[2 * l] + (e & 3), k = j.org[2 * l + 1] + ((e >> 2) & 3);
      if (i >= 0 && i < nx && k >= 0 && k < nz) sMap[(k - wk0) * WW + (i - wi0)] = -2;
    }
  __syncthreads();
  for (int e = tid; e < nwin; e += kThreads) {
    if (sMap[e] != -2) continue;
    const int s = atomicAdd(&nslot, 1);
    if (s < kMaxSlots) {
      sMap[e] = (short)s;
      const int k = wk0 + e / WW, i = wi0 + e % WW;
      sCell[s] = k * nx + i;
    }
  }
  __syncthreads();
  const int ns = nslot;
  if (ns > kMaxSlots) {
    if (tid == 0) atomicOr(p.status, 8u);
    return;
  }
  // tiles whose halo may reach a marker's 4x4 stencil: the stencil widened
  // by the margin spans at most two tiles per axis, those of its ends
  const int ibtx = p.ibtx;
  auto corners = [&](int i0, int k0, int (&tx)[2], int (&tz)[2]) {
    tx[0] = min(max(i0 - kHalo, 0), nx - 1) / f2d::kTX;
    tx[1] = min(max(i0 + 3 + kHalo, 0), nx - 1) / f2d::kTX;
    tz[0] = min(max(k0 - kHalo, 0), nz - 1) / f2d::kTZ;
    tz[1] = min(max(k0 + 3 + kHalo, 0), nz - 1) / f2d::kTZ;
  };
  if (!have_prev) {  // the first update flags its own footprint before the next fluid step may start
    for (int l = tid; l < nl; l += kThreads) {
      int tx[2], tz[2];
      corners(sI0[l], sK0[l], tx, tz);
#pragma unroll
      for (int c = 0; c < 4; c++) j.flag[tz[c >> 1] * ibtx + tx[c & 1]] = 1;
    }
    __threadfence();
    __syncthreads();
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  }
  const float rho0 = p.rho_base, rsal = p.rho_sal_f, hdt = p.hdt;
  for (int s = tid; s < ns; s += kThreads) {
    const long long ci = sCell[s];
    const float S = p.lean ? p.s_uni : mac[ci];
    const float h = hdt / fmaf(S, rsal, rho0);
    float ux, uz;
    vel_at(p, b, mac, ci, N, ux, uz);
    sH[s] = h;
    sU[s] = ux - j.fext[ci] * h;
    sW[s] = uz - j.fext[N + ci] * h;
    sFX[s] = sFZ[s] = 0.f;
    sCur[s] = 0;
  }
  __syncthreads();

  // ---- pairs of the new stencils: their slots, then listed by slot in pair order
  for (int e = tid; e < 16 * nl; e += kThreads) {
    const int l = e >> 4, i = sI0[l] + (e & 3), k = sK0[l] + ((e >> 2) & 3);
    const int s = (i < 0 || i >= nx || k < 0 || k >= nz) ? -1 : sMap[(k - wk0) * WW + (i - wi0)];
    sPS[e] = (short)s;
    if (s >= 0) atomicAdd(&sCur[s], 1);
  }
  __syncthreads();
  {
    // exclusive scan of the counts: kPer consecutive slots per thread, then
    // across lanes and warps
    constexpr int kPer = (kMaxSlots + kThreads - 1) / kThreads;
    int *wtot = reinterpret_cast<int *>(sRed);
    int loc[kPer], sum = 0;
#pragma unroll
    for (int i = 0; i < kPer; i++) {
      const int s = tid * kPer + i;
      loc[i] = sum;
      sum += s < ns ? sCur[s] : 0;
    }
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
      sOff[ns] = run;
    }
    __syncthreads();
    const int base = wtot[warp] + x - sum;
    __syncthreads();  // every warp has read wtot before sRed is reused
#pragma unroll
    for (int i = 0; i < kPer; i++) {
      const int s = tid * kPer + i;
      if (s < ns) sOff[s] = base + loc[i];
    }
  }
  __syncthreads();
  for (int s = tid; s < ns; s += kThreads) sCur[s] = sOff[s];
  __syncthreads();
  // each slot's pairs, first in arrival order (into the window map, free
  // from here on), then each pair at its rank in pair order: the lists come
  // out sorted, so every sum over them runs in a fixed order
  short *sTmp = sMap;
  for (int e = tid; e < 16 * nl; e += kThreads) {
    const int s = sPS[e];
    if (s >= 0) sTmp[atomicAdd(&sCur[s], 1)] = (short)e;
  }
  __syncthreads();
  // (one thread per list position: neighbouring lanes mostly share a slot,
  // so they scan the same entries together)
  for (int a = tid; a < sOff[ns]; a += kThreads) {
    const int e = sTmp[a], s = sPS[e];
    const int a0 = sOff[s], a1 = sOff[s + 1];
    int r = 0;
    for (int b2 = a0; b2 < a1; b2++) r += sTmp[b2] < e;
    sList[a0 + r] = (short)e;
    const int l = e >> 4;
    sWL[a0 + r] = sWX[4 * l + (e & 3)] * sWZ[4 * l + ((e >> 2) & 3)] * sDS[l];  // kernel weight x marker area
  }
  __syncthreads();

  // ---- 3. multi-direct forcing
  const float two_rf_dt = (float)(2.0 * j.rho_f / j.dt);
  for (int it = 0; it < j.iters; it++) {
    // one thread per marker: the velocity at its 16 nodes, summed in a
    // fixed pairwise order (explicit rounding: the order and the roundings
    // do not depend on the compiler), then the marker's force
    for (int l = tid; l < nl; l += kThreads) {
      float wx[4], wz[4], vx[16], vz[16];
#pragma unroll
      for (int a = 0; a < 4; a++) {
        wx[a] = sWX[4 * l + a];
        wz[a] = sWZ[4 * l + a];
      }
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int s = sPS[16 * l + q];
        vx[q] = vz[q] = 0.f;
        if (s >= 0) {
          const float w = __fmul_rn(wx[q & 3], wz[q >> 2]);
          vx[q] = __fmul_rn(w, sU[s]);
          vz[q] = __fmul_rn(w, sW[s]);
        }
      }
#pragma unroll
      for (int o = 8; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < o; q++) {
          vx[q] = __fadd_rn(vx[q], vx[q + o]);
          vz[q] = __fadd_rn(vz[q], vz[q + o]);
        }
      const float dfx = two_rf_dt * (sUB[2 * l] - vx[0]), dfz = two_rf_dt * (sUB[2 * l + 1] - vz[0]);
      sDF[2 * l] = dfx;
      sDF[2 * l + 1] = dfz;
      sFT[2 * l] += dfx;
      sFT[2 * l + 1] += dfz;
    }
    __syncthreads();
    for (int s = tid; s < ns; s += kThreads) {
      float fx = 0.f, fz = 0.f;
      for (int a = sOff[s]; a < sOff[s + 1]; a++) {
        const int l = sList[a] >> 4;
        const float wd = sWL[a];
        fx = fmaf(sDF[2 * l], wd, fx);
        fz = fmaf(sDF[2 * l + 1], wd, fz);
      }
      sFX[s] += fx;
      sFZ[s] += fz;
      sU[s] = fmaf(fx, sH[s], sU[s]);
      sW[s] = fmaf(fz, sH[s], sW[s]);
    }
    __syncthreads();
  }

  // ---- 4. write back
  constexpr bool RES = sizeof(ST) == 2;
  const float ic = 1.0f / p.c;
  for (int s = tid; s < ns; s += kThreads) {
    const long long ci = sCell[s];
    float un = sU[s], wn = sW[s];
    if (!RES && p.ib_uform) {
      // uniform S, no scalar lattice: the velocity the forcing leaves, in the
      // form the lean steps recompute it (f2d::lean_velocity), c j + (F0 +
      // f_ib) dt / 2 rho with this update's force f_ib
      const float *fb = static_cast<const float *>(p.fbuf[b]);
      float fv[9];
#pragma unroll
      for (int k = 0; k < 9; k++) fv[k] = fb[k * N + ci];
      float pr, jx, jz;
      f2d::moments9(fv, pr, jx, jz);
      const float S = p.lean ? p.s_uni : mac[ci];
      const float hf = __fdividef(p.hdt, fmaf(S, p.rho_sal_f, p.rho_base));
      float Fx = 0.0f, Fz = 0.0f;
      Fz -= __fmul_rn(S, p.g_bouss_f);
      Fx += sFX[s];
      Fz += sFZ[s];
      un = fmaf(Fx, hf, p.c * jx);
      wn = fmaf(Fz, hf, p.c * jz);
    }
    if constexpr (RES) {
      // re-express the stored deviations about the new velocity
      ST *fb = static_cast<ST *>(p.fbuf[b]);
      const float uo = mac[N + ci] * ic, wo = mac[2 * N + ci] * ic, u2o = rstore::usq(uo, wo);
      const float uc = un * ic, wc = wn * ic, u2 = rstore::usq(uc, wc);
      const float pr = mac[3 * N + ci];
      float amax = 0.f;
#pragma unroll
      for (int k = 0; k < 9; k++) {
        const float fv = f2d::ld(fb, k * N + ci, p.inv_fscale) + rstore::feq(k, pr, uo, wo, u2o);
        const float r = fv - rstore::feq(k, pr, uc, wc, u2);
        amax = fmaxf(amax, fabsf(r) * p.fscale);
        f2d::st(fb, k * N + ci, r, p.fscale);
      }
      if constexpr (QS > 0) {
        ST *gb = static_cast<ST *>(p.gbuf[b]);
        const float S = mac[ci];
#pragma unroll
        for (int k = 0; k < QS; k++) {
          const float eo = QS == 5 ? rstore::geq5(k, S, uo, wo) : rstore::geq9(k, S, uo, wo, u2o);
          const float en = QS == 5 ? rstore::geq5(k, S, uc, wc) : rstore::geq9(k, S, uc, wc, u2);
          const float r = f2d::ld(gb, k * N + ci, p.inv_gscale) + eo - en;
          amax = fmaxf(amax, fabsf(r) * p.gscale);
          f2d::st(gb, k * N + ci, r, p.gscale);
        }
      }
      if (amax > p.store_max) atomicOr(p.status, 2u);
    }
    mac[N + ci] = un;
    mac[2 * N + ci] = wn;
    j.fext[ci] = sFX[s];
    j.fext[N + ci] = sFZ[s];
    if (!(isfinite(un) && isfinite(wn))) atomicOr(p.status, 1u);
  }
  __syncthreads();

  // ---- 5. FP64 sums: marker force and torque, fluid momentum inside the body
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int l = tid; l < nl; l += kThreads) {
    const double x0 = j.X0[2 * l], z0 = j.X0[2 * l + 1];
    const double rx = cth * x0 - sth * z0, rz = sth * x0 + cth * z0;
    const double fx = (double)sFT[2 * l] * j.dS[l], fz = (double)sFT[2 * l + 1] * j.dS[l];
    j.fmark[2 * l] = (float)fx;
    j.fmark[2 * l + 1] = (float)fz;
    acc[0] += fx;
    acc[1] += fz;
    acc[2] += rx * fz - rz * fx;
  }
  {
    const double a = j.semi_a, bb = j.semi_b, ra = 1.0 / a, rb = 1.0 / bb;
    // half extents of the ellipse, widened by one cell for the fraction ramp
    const double hx = sqrt(a * a * cth * cth + bb * bb * sth * sth) + dz;
    const double hz = sqrt(a * a * sth * sth + bb * bb * cth * cth) + dz;
    const int ia = max((int)ceil((B.X[0] - hx) * idz - 0.5), 0), ib = min((int)floor((B.X[0] + hx) * idz - 0.5), nx - 1);
    const int ka = max((int)ceil((B.X[1] - hz) * idz - 0.5), 0), kb = min((int)floor((B.X[1] + hz) * idz - 0.5), nz - 1);
    const int bw = ib - ia + 1, bh = kb - ka + 1;
    const double dA = dz * dz;
    if (bw > 0 && bh > 0) {
      // kC cells per thread at a time: their fractions first, then all
      // their velocity loads in flight together, then the sums in cell order
      constexpr int kC = 4;
      for (int e0 = tid; e0 < bw * bh; e0 += kC * kThreads) {
        double al[kC], dxs[kC], dzs[kC];
        long long cis[kC];
#pragma unroll
        for (int c = 0; c < kC; c++) {
          const int e = e0 + c * kThreads;
          al[c] = 0.0;
          dxs[c] = dzs[c] = 0.0;
          cis[c] = 0;
          if (e < bw * bh) {
            const int i = ia + e % bw, k = ka + e / bw;
            const double dx = (i + 0.5) * dz - B.X[0], dzz = (k + 0.5) * dz - B.X[1];
            const double xb = cth * dx + sth * dzz, zb = -sth * dx + cth * dzz;
            const double xa = xb * ra, zc = zb * rb;
            const double F = xa * xa + zc * zc - 1.0;
            const double G = 2.0 * hypot(xa * ra, zc * rb);
            al[c] = fmin(fmax(0.5 - F / fmax(G, 1e-300) * idz, 0.0), 1.0) * dA;
            dxs[c] = dx;
            dzs[c] = dzz;
            cis[c] = (long long)k * nx + i;
          }
        }
        float uxf[kC], uzf[kC];
#pragma unroll
        for (int c = 0; c < kC; c++) {
          uxf[c] = uzf[c] = 0.f;
          if (al[c] > 0.0) vel_at(p, b, mac, cis[c], N, uxf[c], uzf[c]);
        }
#pragma unroll
        for (int c = 0; c < kC; c++)
          if (al[c] > 0.0) {
            const double ux = uxf[c], uz = uzf[c];
            acc[3] += al[c] * ux;
            acc[4] += al[c] * uz;
            acc[5] += al[c] * (dxs[c] * uz - dzs[c] * ux);
          }
      }
    }
  }
#pragma unroll
  for (int v = 0; v < 6; v++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[v] += __shfl_down_sync(0xffffffffu, acc[v], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int v = 0; v < 6; v++) sRed[warp * 6 + v] = acc[v];
  }
  __syncthreads();

  // ---- 6. rigid-body step (FP64, one thread)
  if (tid == 0) {
    double t[6] = {0, 0, 0, 0, 0, 0};
    for (int w = 0; w < kWarps; w++)
      for (int v = 0; v < 6; v++) t[v] += sRed[w * 6 + v];
    Body nb = B;
    const double dt = j.dt, rf = j.rho_f;
    double Fb[2] = {-(t[0] + B.Fib[0]) / 2, -(t[1] + B.Fib[1]) / 2};
    const double Tb = -(t[2] + B.Tib) / 2;
    Fb[1] += -(1.0 - rf / j.rho_s) * j.m * j.grav;
    const double P0 = have_prev ? B.P[0] : t[3], P1 = have_prev ? B.P[1] : t[4], L0 = have_prev ? B.L : t[5];
    nb.U[0] = B.U[0] + (dt * Fb[0] + rf * (t[3] - P0)) / j.m;
    nb.U[1] = B.U[1] + (dt * Fb[1] + rf * (t[4] - P1)) / j.m;
    nb.om = B.om + (dt * Tb + rf * (t[5] - L0)) / j.I;
    nb.X[0] = B.X[0] + dt * (B.U[0] + nb.U[0]) / 2;
    nb.X[1] = B.X[1] + dt * (B.U[1] + nb.U[1]) / 2;
    nb.th = B.th + dt * (B.om + nb.om) / 2;
    nb.P[0] = t[3];
    nb.P[1] = t[4];
    nb.L = t[5];
    nb.Fib[0] = t[0];
    nb.Fib[1] = t[1];
    nb.Tib = t[2];
    nb.have_prev2 = B.have_prev;
    nb.have_prev = 1;
    *j.body = nb;
    B = nb;
  }
  __syncthreads();

  // ---- 7. flags for the next step's footprint (from the body state just
  // written, as the next update will compute it), clean-up two steps back,
  // and the footprints move back one step
  int *sPI = reinterpret_cast<int *>(sUB);  // predicted stencil origins [nl][2]
  {
    const double c2 = cos(B.th), s2 = sin(B.th);
    for (int l = tid; l < nl; l += kThreads) {
      const double x0 = j.X0[2 * l], z0 = j.X0[2 * l + 1];
      const double X = B.X[0] + (c2 * x0 - s2 * z0), Z = B.X[1] + (s2 * x0 + c2 * z0);
      const int pi = (int)floor(X * idz - 0.5) - 1, pk = (int)floor(Z * idz - 0.5) - 1;
      sPI[2 * l] = pi;
      sPI[2 * l + 1] = pk;
      take_box(bx + 8, pi, pk);
    }
    merge_box(bx + 8, bnd3);
  }
  __syncthreads();
  const int lo_i = min(min(wi0, bnd2[0]), bnd3[0]), hi_i = max(max(wi0 + WW - 1, bnd2[1]), bnd3[1]);
  const int lo_k = min(min(wk0, bnd2[2]), bnd3[2]), hi_k = max(max(wk0 + WH - 1, bnd2[3]), bnd3[3]);
  const int tx0 = min(max(lo_i - kHalo, 0), nx - 1) / f2d::kTX, tz0 = min(max(lo_k - kHalo, 0), nz - 1) / f2d::kTZ;
  const int tmw = min(max(hi_i + kHalo, 0), nx - 1) / f2d::kTX - tx0 + 1;
  const int tmh = min(max(hi_k + kHalo, 0), nz - 1) / f2d::kTZ - tz0 + 1;
  const bool tmap_ok = tmw > 0 && tmh > 0 && tmw * tmh <= kTileMap;
  if (tmap_ok)
    for (int e = tid; e < tmw * tmh; e += kThreads) tmap[e] = 0;
  __syncthreads();
  // previous, current and next footprints: kept (the next one flagged now)
  for (int e = tid; e < 3 * nl; e += kThreads) {
    const int which = e / nl, l = e - which * nl;
    if (which == 0 && !have_prev) continue;
    const int i0 = which == 0 ? j.org[2 * l] : (which == 1 ? sI0[l] : sPI[2 * l]);
    const int k0 = which == 0 ? j.org[2 * l + 1] : (which == 1 ? sK0[l] : sPI[2 * l + 1]);
    int tx[2], tz[2];
    corners(i0, k0, tx, tz);
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int x = tx[c & 1], z = tz[c >> 1];
      if (which == 2) j.flag[z * ibtx + x] = 1;
      if (tmap_ok) tmap[(z - tz0) * tmw + (x - tx0)] = 1;
    }
  }
  __syncthreads();
  if (have_prev2 && tmap_ok) {
    for (int l = tid; l < nl; l += kThreads) {
      int tx[2], tz[2];
      corners(j.org2[2 * l], j.org2[2 * l + 1], tx, tz);
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const int x = tx[c & 1], z = tz[c >> 1];
        if (!tmap[(z - tz0) * tmw + (x - tx0)]) j.flag[z * ibtx + x] = 0;
      }
    }
  }
  __syncthreads();
  for (int l = tid; l < nl; l += kThreads) {
    j.org2[2 * l] = j.org[2 * l];
    j.org2[2 * l + 1] = j.org[2 * l + 1];
    j.org[2 * l] = sI0[l];
    j.org[2 * l + 1] = sK0[l];
  }
}

template <class ST, int QS>
__global__ void __launch_bounds__(kThreads, 1) ib_kernel(const __grid_constant__ Job j, int parity) {
  coupled_update<ST, QS>(j, parity);
}

template <class ST, int QS>
__global__ void __launch_bounds__(kThreads, 1) ib_kernel_batched(const Job *__restrict__ jobs, int parity) {
  coupled_update<ST, QS>(jobs[blockIdx.x], parity);
}

template <class ST, int QS>
int prep1() {
  cudaError_t e = cudaFuncSetAttribute(ib_kernel<ST, QS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Layout::BYTES);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(ib_kernel_batched<ST, QS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Layout::BYTES);
  return status_from_cuda(e);
}

template <class ST>
int prep_q() {
  int st = prep1<ST, 0>();
  if (!st) st = prep1<ST, 5>();
  if (!st) st = prep1<ST, 9>();
  return st;
}

template <class ST, int QS>
int go(const Job *jp, const Job *jobs, int njobs, int parity, cudaStream_t s) {
  if (jp) {
    // a programmatic dependent of the fluid step before it: its launch
    // overlaps that step's last wave, and it waits (griddepcontrol.wait,
    // first thing) for the step to complete before it reads anything
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = Layout::BYTES;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return status_from_cuda(cudaLaunchKernelEx(&cfg, ib_kernel<ST, QS>, *jp, parity));
  }
  ib_kernel_batched<ST, QS><<<njobs, kThreads, Layout::BYTES, s>>>(jobs, parity);
  return status_from_cuda(cudaGetLastError());
}

template <class ST>
int go_q(const Job *jp, const Job *jobs, int njobs, int parity, int qs, cudaStream_t s) {
  switch (qs) {
    case 0: return go<ST, 0>(jp, jobs, njobs, parity, s);
    case 5: return go<ST, 5>(jp, jobs, njobs, parity, s);
    case 9: return go<ST, 9>(jp, jobs, njobs, parity, s);
  }
  return IPCU_ERR_UNSUPPORTED;
}

int dispatch(const Job *jp, const Job *jobs, int njobs, int parity, int storage, int qs, cudaStream_t s) {
  switch (storage) {
    case IPCU_STORE_F32: return go_q<float>(jp, jobs, njobs, parity, qs, s);
    case IPCU_STORE_F16: return go_q<__half>(jp, jobs, njobs, parity, qs, s);
    case IPCU_STORE_BF16: return go_q<__nv_bfloat16>(jp, jobs, njobs, parity, qs, s);
  }
  return IPCU_ERR_UNSUPPORTED;
}

}  // namespace

size_t smem_bytes() { return Layout::BYTES; }

int prepare() {
  int st = prep_q<float>();
  if (!st) st = prep_q<__half>();
  if (!st) st = prep_q<__nv_bfloat16>();
  return st;
}

int launch(const Job &j, int parity, int storage, int qs, cudaStream_t s) {
  return dispatch(&j, nullptr, 1, parity, storage, qs, s);
}

int launch_batched(const Job *jobs, int njobs, int parity, int storage, int qs, cudaStream_t s) {
  if (njobs <= 0) return IPCU_OK;
  return dispatch(nullptr, jobs, njobs, parity, storage, qs, s);
}

}  // namespace ib2d
}  // namespace ipcu
