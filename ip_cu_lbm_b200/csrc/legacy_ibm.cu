// Reference-compatible kernel entries, immersed-boundary family
// (ref: function/ibm.cu). Markers are few (10^2-10^3), so the marker kernels
// are latency-bound: one warp lane per marker for the stencil work, and a
// single thread block with warp-shuffle reductions (accumulated in FP64)
// for the rigid-body force/torque sums that the reference does serially on
// one thread.
#include "ipcu_common.cuh"

namespace ipcu {
namespace {

// Peskin-type kernel of the reference, float arithmetic (ref: function/ibm.cu:61-66)
__device__ __forceinline__ float peskin4(float dx, float x, float xl) {
  float r = fabsf(x - xl) / dx;
  if (r < 1.0f) return (3.0f - 2.0f * r + sqrtf(1.0f + 4.0f * r - 4.0f * r * r)) * 0.125f;
  if (r <= 2.0f) return (5.0f - 2.0f * r - sqrtf(-7.0f + 12.0f * r - 4.0f * r * r)) * 0.125f;
  return 0.0f;
}

template <class T>
__device__ __forceinline__ void lag3(T *cf, const T *pl, T xa) {
#pragma unroll
  for (int a = 0; a < 3; a++) {
    T v = T(1);
#pragma unroll
    for (int b = 0; b < 3; b++)
      if (b != a) v *= (xa - pl[b]) / (pl[a] - pl[b]);
    cf[a] = v;
  }
}

template <class T>
__host__ __device__ __forceinline__ void quat_rot(T q0, T q1, T q2, T q3, T *R) {
  R[0] = q0 * q0 - q2 * q2 - q3 * q3 + q1 * q1;
  R[1] = T(2) * (q1 * q2 - q0 * q3);
  R[2] = T(2) * (q1 * q3 + q0 * q2);
  R[3] = T(2) * (q1 * q2 + q0 * q3);
  R[4] = q0 * q0 - q3 * q3 - q1 * q1 + q2 * q2;
  R[5] = T(2) * (q2 * q3 - q0 * q1);
  R[6] = T(2) * (q1 * q3 - q0 * q2);
  R[7] = T(2) * (q2 * q3 + q0 * q1);
  R[8] = q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3;
}

// Stencil direction for the 3x3(x3) marker neighbourhood (ref: function/ibm.cu:132-142).
// Q9 (x-z plane): index (i, l) -> direction with (ex, ez) = (i-1, l-1), except
// for the corner noted below.
__device__ __forceinline__ int ib_dir(int Q, int i, int j, int l) {
  // The reference's table maps (i,l) = (0,0) to direction 5, not 7; kept.
  if (Q == 9) {
    const int t[3][3] = {{5, 3, 6}, {4, 0, 2}, {8, 1, 5}};
    return t[i][l];
  }
  // D3Q27 direction with velocity (i-1, j-1, l-1)
  const int t[3][3][3] = {{{26, 10, 25}, {14, 3, 13}, {24, 9, 23}},
                          {{18, 4, 17}, {6, 0, 5}, {16, 2, 15}},
                          {{22, 8, 21}, {12, 1, 11}, {20, 7, 19}}};
  return t[i][j][l];
}

// ---- get_IBMGw2: Suzuki-Yoshino stress-jump marker force, interpolation
// of all populations on the 3x3(x3) stencil and spreading to F
// (ref: function/ibm.cu:124-274)
template <class T, int Q>
__device__ void ibm_gw2_body(const Items<T> &P, const int *lid, const int *nb, const T *f, const T *tau,
                             const T *px, const T *py, const T *pz, const T *posw, const T *nB,
                             const T *velw, T *Fx, T *Fy, T *Fz, T *Gw, T rhof) {
  constexpr int qs = (Q == 27) ? 1 : 0, j0 = (Q == 9) ? 1 : 0, j1 = (Q == 9) ? 2 : 3, dim = (Q == 9) ? 2 : 3;
  const long long np = (long long)P.scal(IT_num_IBPoints);
  const T dIBM = P.scal(IT_dIBM);
  IPCU_FOR(m, 0, np) {
    const long long L = lid[m];
    auto N = [&](int d) -> long long { return (long long)nb[L * Q + d]; };
    const T uw = velw[m * 3], vw = velw[m * 3 + 1], ww = velw[m * 3 + 2];
    const T nbx = nB[m * 3], nby = nB[m * 3 + 1], nbz = nB[m * 3 + 2];
    T cx[3], cy[3], cz[3];
    const int xs[3] = {3, 0, 1};
#pragma unroll
    for (int a = 0; a < 3; a++)
      cx[a] = (T)peskin4((float)P.dz, (float)posw[m * 3], (float)px[N(xs[a])]) * T(N(xs[a]) < P.nc);
    if (Q == 27) {
      T pl[3] = {py[N(4)], py[N(0)], py[N(2)]};
      lag3(cy, pl, posw[m * 3 + 1]);
      T ql[3] = {pz[N(6)], pz[N(0)], pz[N(5)]};
      lag3(cz, ql, posw[m * 3 + 2]);
    } else {
      cy[0] = T(0);
      cy[1] = T(1);
      cy[2] = T(0);
      const int zs[3] = {4, 0, 2};
#pragma unroll
      for (int a = 0; a < 3; a++)
        cz[a] = (T)peskin4((float)P.dz, (float)posw[m * 3 + 2], (float)pz[N(zs[a])]) * T(N(zs[a]) < P.nc);
      T s = cx[0] + cx[1] + cx[2];
#pragma unroll
      for (int a = 0; a < 3; a++) cx[a] /= s;
      s = cz[0] + cz[1] + cz[2];
#pragma unroll
      for (int a = 0; a < 3; a++) cz[a] /= s;
    }
    T fw[Q];
#pragma unroll
    for (int k = 0; k < Q; k++) fw[k] = T(0);
    for (int i = 0; i < 3; i++)
      for (int j = j0; j < j1; j++)
        for (int l = 0; l < 3; l++) {
          long long id = N(ib_dir(Q, i, j, l));
          if (id < P.nc) {
            T wgt = cx[i] * cy[j] * cz[l];
#pragma unroll
            for (int k = 0; k < Q; k++) fw[k] += wgt * f[id * Q + k];
          }
        }
    // split into the two sides of the surface with the 22.5 degree blend
    const T sa = sin(T(22.5 / 180.0 * 3.14159));
    T fw1[Q], fw2[Q];
#pragma unroll
    for (int k = 0; k < Q; k++) {
      const int ki = c_dirs.kinv[qs][k];
      T t = (nbx * P.cx(k) + nby * P.cy(k) + nbz * P.cz(k)) / P.c;
      T t2 = sqrt(P.cx(k) * P.cx(k) + P.cy(k) * P.cy(k) + P.cz(k) * P.cz(k)) / P.c * sa;
      T t3 = T(6) * P.w(k) * (P.cx(k) * uw + P.cy(k) * vw + P.cz(k) * ww) / (P.c * P.c);
      T be = fabs(t) / (t2 + T(1e-10f));
      T mix = (T(1) - be) * fw[k] + be * (fw[ki] + t3), refl = fw[ki] + t3;
      fw1[k] = (t <= T(0)) ? fw[k] : ((t <= t2) ? mix : refl);
      fw2[k] = (t >= T(0)) ? fw[k] : ((t >= -t2) ? mix : refl);
    }
    const T tl = tau[L], a1 = T(0.5) / tl, a2 = T(1) - T(0.5) / tl;
    const T U[3] = {uw, vw, ww}, n3[3] = {nbx, nby, nbz};
    auto traction = [&](bool jump, T *g) {
#pragma unroll
      for (int a = 0; a < 3; a++) {
        T sig[3] = {0, 0, 0};
#pragma unroll
        for (int k = 0; k < Q; k++) {
          const T ck[3] = {P.cx(k), P.cy(k), P.cz(k)};
          T df = jump ? fw1[k] - fw2[k] : fw1[k];
#pragma unroll
          for (int b = 0; b < 3; b++)
            sig[b] -= a1 * df * T(a == b) +
                      a2 * T(3) * (df * (ck[a] - U[a]) * (ck[b] - U[b]) - (df - P.w(k)) * U[a] * U[b]) / (P.c * P.c);
        }
        g[a] = sig[0] * n3[0] + sig[1] * n3[1] + sig[2] * n3[2];
      }
    };
    T g[3];
    traction(true, g);
    const T sc = (T)powf((float)(dIBM / P.dz), (float)(dim - 1)) / P.dz;
    for (int i = 0; i < 3; i++)
      for (int j = j0; j < j1; j++)
        for (int l = 0; l < 3; l++) {
          long long id = N(ib_dir(Q, i, j, l));
          if (id < P.nc) {
            T wgt = cx[i] * cy[j] * cz[l];
            atomicAdd(&Fx[id], -g[0] * sc * wgt);
            atomicAdd(&Fy[id], -g[1] * sc * wgt);
            atomicAdd(&Fz[id], -g[2] * sc * wgt);
          }
        }
    traction(false, g);
    const T gs = rhof * P.c * P.c / T(3) * (T)powf((float)dIBM, (float)(dim - 1));
    Gw[m * 3] = g[0] * gs;
    Gw[m * 3 + 1] = g[1] * gs;
    Gw[m * 3 + 2] = g[2] * gs;
  }
}
template <class T>
__global__ void k_get_IBMGw2(const T *it, const int *lid, const int *nb, const T *f, const T *tau, const T *px,
                             const T *py, const T *pz, const T *posw, const T *nB, const T *velw, T *Fx, T *Fy,
                             T *Fz, T *Gw, T rhof) {
  Items<T> P(it);
  if (P.Q == 9) ibm_gw2_body<T, 9>(P, lid, nb, f, tau, px, py, pz, posw, nB, velw, Fx, Fy, Fz, Gw, rhof);
  else if (P.Q == 27) ibm_gw2_body<T, 27>(P, lid, nb, f, tau, px, py, pz, posw, nB, velw, Fx, Fy, Fz, Gw, rhof);
}

// ---- IB_directForcing: classic direct forcing (ref: function/ibm.cu:276-344)
__global__ void k_IB_directForcing(const float *it, const int *lid, const int *nb, const float *px, const float *py,
                                   const float *pz, const float *posw, const float *u, const float *v,
                                   const float *w, const float *velw, float *Fx, float *Fy, float *Fz, float *Gw) {
  Items<float> P(it);
  const int Q = P.Q, j0 = (Q == 9) ? 1 : 0, j1 = (Q == 9) ? 2 : 3, dim = (Q == 9) ? 2 : 3;
  const long long np = (long long)P.scal(IT_num_IBPoints);
  const float dIBM = P.scal(IT_dIBM);
  IPCU_FOR(m, 0, np) {
    const long long L = lid[m];
    auto N = [&](int d) -> long long { return (long long)nb[L * Q + d]; };
    float cx[3], cy[3], cz[3];
    float pl[3] = {px[N(3)], px[N(0)], px[N(1)]};
    lag3(cx, pl, posw[m * 3]);
    if (Q == 27) {
      float a[3] = {py[N(4)], py[N(0)], py[N(2)]};
      lag3(cy, a, posw[m * 3 + 1]);
      float b[3] = {pz[N(6)], pz[N(0)], pz[N(5)]};
      lag3(cz, b, posw[m * 3 + 2]);
    } else {
      cy[0] = 0.f;
      cy[1] = 1.f;
      cy[2] = 0.f;
      float b[3] = {pz[N(4)], pz[N(0)], pz[N(2)]};
      lag3(cz, b, posw[m * 3 + 2]);
    }
    float uw[3] = {0.f, 0.f, 0.f};
    for (int i = 0; i < 3; i++)
      for (int j = j0; j < j1; j++)
        for (int l = 0; l < 3; l++) {
          long long id = N(ib_dir(Q, i, j, l));
          if (id < P.nc) {
            float wgt = cx[i] * cy[j] * cz[l];
            uw[0] += wgt * u[id];
            uw[1] += wgt * v[id];
            uw[2] += wgt * w[id];
          }
        }
    float gw[3];
    for (int a = 0; a < 3; a++) gw[a] = (velw[m * 3 + a] - uw[a]) / P.dt;
    const float sc = powf(dIBM / P.dz, (float)(dim - 1)) * 3.0f / (P.c * P.c);
    for (int i = 0; i < 3; i++)
      for (int j = j0; j < j1; j++)
        for (int l = 0; l < 3; l++) {
          long long id = N(ib_dir(Q, i, j, l));
          if (id < P.nc) {
            float wgt = cx[i] * cy[j] * cz[l] * sc;
            atomicAdd(&Fx[id], gw[0] * wgt);
            atomicAdd(&Fy[id], gw[1] * wgt);
            atomicAdd(&Fz[id], gw[2] * wgt);
          }
        }
    const float gs = 1000.0f * powf(dIBM, (float)(dim - 1)) * P.dz;
    for (int a = 0; a < 3; a++) Gw[m * 3 + a] += -gw[a] * gs;
  }
}

// ---- update_velIBM: post-stream forcing f += w dt (e.F), then p*, u
// (ref: function/ibm.cu:346-365)
template <class T, int Q>
__device__ void velibm_body(const Items<T> &P, T *f, T *pr, T *u, T *v, T *w, const T *Fx, const T *Fy,
                            const T *Fz) {
  IPCU_FOR(i, 0, P.nc) {
    T a = 0, b = 0, c = 0, d = 0, fx = Fx[i], fy = Fy[i], fz = Fz[i];
#pragma unroll
    for (int k = 0; k < Q; k++) {
      T fk = f[i * Q + k] + P.w(k) * P.dt * (P.cx(k) * fx + P.cy(k) * fy + P.cz(k) * fz);
      f[i * Q + k] = fk;
      a += fk;
      b += P.cx(k) * fk;
      c += P.cy(k) * fk;
      d += P.cz(k) * fk;
    }
    pr[i] = a;
    u[i] = b;
    v[i] = c;
    w[i] = d;
  }
}
template <class T>
__global__ void k_update_velIBM(const T *it, T *f, T *pr, T *u, T *v, T *w, const T *Fx, const T *Fy,
                                const T *Fz) {
  Items<T> P(it);
  if (P.Q == 9) velibm_body<T, 9>(P, f, pr, u, v, w, Fx, Fy, Fz);
  else if (P.Q == 27) velibm_body<T, 27>(P, f, pr, u, v, w, Fx, Fy, Fz);
}

// ---- update_IBbody: force/torque sums over markers, AB2 translation and
// rotation, quaternion AB2 (ref: function/ibm.cu:367-424). One block: the
// marker sums are warp-shuffle reductions in FP64; thread 0 then applies
// the reference's update (including its reading of quatold at offset 0).
template <class T>
__global__ void k_update_IBbody(const T *it, int ib, const T *massB, const T *densB, const T *inertia, T *FB,
                                T *posB, T *Tq, T *velB, T *quat, T *quaS, T *angleVB, const T *posw, const T *Gw,
                                T *quatold, T rhof) {
  Items<T> P(it);
  const long long np = (long long)P.scal(IT_num_IBPoints);
  const T cx = posB[ib * 3], cy = posB[ib * 3 + 1], cz = posB[ib * 3 + 2];
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (long long m = threadIdx.x; m < np; m += blockDim.x) {
    const T *g = Gw + m * 3, *x = posw + m * 3;
    s[0] += (double)g[0];
    s[1] += (double)g[1];
    s[2] += (double)g[2];
    s[3] += (double)((x[1] - cy) * g[2] - (x[2] - cz) * g[1]);
    s[4] += (double)((x[2] - cz) * g[0] - (x[0] - cx) * g[2]);
    s[5] += (double)((x[0] - cx) * g[1] - (x[1] - cy) * g[0]);
  }
  __shared__ double red[32][6];
#pragma unroll
  for (int a = 0; a < 6; a++)
    for (int o = 16; o > 0; o >>= 1) s[a] += __shfl_down_sync(0xffffffffu, s[a], o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int a = 0; a < 6; a++) red[wid][a] = s[a];
  __syncthreads();
  if (threadIdx.x != 0) return;
  for (int a = 0; a < 6; a++) {
    double t = 0;
    for (int q = 0; q < (int)((blockDim.x + 31) / 32); q++) t += red[q][a];
    s[a] = t;
  }
  const T dt = P.dt;
  T Ro[9], Fo[3], To[3], vo[3], wo[3];
  quat_rot(quatold[ib * 4], quatold[ib * 4 + 1], quatold[ib * 4 + 2], quatold[ib * 4 + 3], Ro);
  for (int a = 0; a < 3; a++) {
    Fo[a] = FB[ib * 3 + a];
    To[a] = Tq[ib * 3 + a];
    vo[a] = velB[ib * 3 + a];
    wo[a] = angleVB[ib * 3 + a];
    FB[ib * 3 + a] = (T)s[a];
    Tq[ib * 3 + a] = (T)s[3 + a];
  }
  FB[ib * 3 + 2] += (T(1) - rhof / densB[ib]) * massB[ib] * T(9.81);
  for (int a = 0; a < 3; a++) {
    velB[ib * 3 + a] += dt * (T(3) * FB[ib * 3 + a] - Fo[a]) / massB[ib] / T(2);
    posB[ib * 3 + a] += dt * (T(3) * velB[ib * 3 + a] - vo[a]) / T(2);
  }
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++)
      angleVB[ib * 3 + a] +=
          dt * (T(3) * quaS[ib * 3 + b * 3 + a] * Tq[ib * 3 + b] - Ro[b * 3 + a] * To[b]) / inertia[ib * 3 + a] / T(2);
  T q[4], w[3];
  for (int a = 0; a < 4; a++) q[a] = quat[ib * 4 + a];
  for (int a = 0; a < 3; a++) w[a] = angleVB[ib * 3 + a];
  T *Qn = quat + ib * 4;
  Qn[0] += dt * T(3) * (-w[0] * q[1] - w[1] * q[2] - w[2] * q[3]) / T(4);
  Qn[1] += dt * T(3) * (w[0] * q[0] + w[2] * q[2] - w[1] * q[3]) / T(4);
  Qn[2] += dt * T(3) * (w[1] * q[0] - w[2] * q[1] + w[0] * q[3]) / T(4);
  Qn[3] += dt * T(3) * (w[2] * q[0] + w[1] * q[1] - w[0] * q[2]) / T(4);
  const T qo[4] = {quatold[0], quatold[1], quatold[2], quatold[3]};
  Qn[0] -= dt * (-wo[0] * qo[1] - wo[1] * qo[2] - wo[2] * qo[3]) / T(4);
  Qn[1] -= dt * (wo[0] * qo[0] + wo[2] * qo[2] - wo[1] * qo[3]) / T(4);
  Qn[2] -= dt * (wo[1] * qo[0] - wo[2] * qo[1] + wo[0] * qo[3]) / T(4);
  Qn[3] -= dt * (wo[2] * qo[0] + wo[1] * qo[1] - wo[0] * qo[2]) / T(4);
  for (int a = 0; a < 4; a++) quatold[ib * 4 + a] = q[a];
  quat_rot(Qn[0], Qn[1], Qn[2], Qn[3], quaS);
}

// ---- update_IBpoint: marker position, normal, velocity from the body state
// (ref: function/ibm.cu:426-447)
template <class T>
__global__ void k_update_IBpoint(const T *it, int ib, const T *posB, const T *velB, const T *om, const T *R, T *posw,
                                 const T *op, T *nB, const T *onB, T *velw) {
  Items<T> P(it);
  const long long np = (long long)P.scal(IT_num_IBPoints);
  const T *Rb = R + ib * 9, *w = om + ib * 3;
  IPCU_FOR(m, 0, np) {
    const T r[3] = {op[m * 3], op[m * 3 + 1], op[m * 3 + 2]};
    const T nr[3] = {onB[m * 3], onB[m * 3 + 1], onB[m * 3 + 2]};
    const T wr[3] = {w[1] * r[2] - w[2] * r[1], w[2] * r[0] - w[0] * r[2], w[0] * r[1] - w[1] * r[0]};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      T x = posB[ib * 3 + a], n = T(0);
#pragma unroll
      for (int b = 0; b < 3; b++) {
        x += Rb[a * 3 + b] * r[b];
        n += Rb[a * 3 + b] * nr[b];
      }
      posw[m * 3 + a] = x;
      nB[m * 3 + a] = n;
      velw[m * 3 + a] = velB[ib * 3 + a] + Rb[a * 3] * wr[0] + Rb[a * 3 + 1] * wr[1] + Rb[a * 3 + 2] * wr[2];
    }
  }
}

// ---- search_IBlattice: nearest of the Q neighbours (ref: function/ibm.cu:449-463)
template <class T>
__global__ void k_search_IBlattice(const T *it, int *lid, const int *nb, const T *px, const T *py, const T *pz,
                                   const T *posw) {
  Items<T> P(it);
  const long long np = (long long)P.scal(IT_num_IBPoints);
  const int Q = P.Q;
  IPCU_FOR(m, 0, np) {
    const T mx = posw[m * 3], my = posw[m * 3 + 1], mz = posw[m * 3 + 2];
    long long id = lid[m], best = id;
    T a = px[id] - mx, b = py[id] - my, c = pz[id] - mz;
    T d1 = a * a + b * b + c * c;
    for (int k = 1; k < Q; k++) {
      long long n = nb[id * Q + k];
      a = px[n] - mx;
      b = py[n] - my;
      c = pz[n] - mz;
      T d2 = a * a + b * b + c * c;
      if (d2 < d1) {
        best = n;
        d1 = d2;
      }
    }
    lid[m] = (int)best;
  }
}

// ---- SPM: smoothed-profile forcing of a disc (ref: function/ibm.cu:44-49,68-85)
template <class T>
__global__ void k_SPM(const T *it, T R, const T *posB, T *f, T *ftmp, const T *px, const T *py, T *Fx, T *Fy,
                      T *Fz, const T *u, const T *v, const T *w, const T *velw) {
  Items<T> P(it);
  const int Q = P.Q;
  IPCU_FOR(i, 0, P.nc) {
    float dz = (float)P.dz;
    float dx_ = (float)(px[i] - posB[0]), dy_ = (float)(py[i] - posB[1]);
    float r = (float)R - 0.5f * dz - sqrtf(dx_ * dx_ + dy_ * dy_);
    float pr = (r < -0.5f * dz) ? 0.0f : (fabsf(r) <= 0.5f * dz ? 0.5f * (sinf(3.14159f * r / dz) + 1.0f) : 1.0f);
    T fx = (T)pr * (velw[0] - u[i]) / P.dz, fy = (T)pr * (velw[1] - v[i]) / P.dz, fz = (T)pr * (velw[2] - w[i]) / P.dz;
    for (int k = 0; k < Q; k++) {
      T fk = ftmp[i * Q + k] + P.w(k) * P.dt * T(3) * (P.cx(k) * fx + P.cy(k) * fy + P.cz(k) * fz) / (P.c * P.c);
      f[i * Q + k] = fk;
      ftmp[i * Q + k] = fk;
    }
    Fx[i] = T(0);
    Fy[i] = T(0);
    Fz[i] = T(0);
  }
}

// ---- SPM_ellipse: smoothed-profile forcing of an ellipse (ref: function/ibm.cu:50-59,87-122)
__device__ __forceinline__ float spm_profile2(float lim, float r) {
  float in_l = 1.0f - lim + (lim / 2) * (lim / 2), out_l = 1.0f + lim + (lim / 2) * (lim / 2);
  if (out_l < r) return 0.0f;
  if (in_l <= r) return 0.5f * (sinf(3.14159f * r / lim) + 1.0f);
  return 1.0f;
}
__global__ void k_SPM_ellipse(const float *it, float Ra, float Rb, const float *quaS, const float *posB, float *f,
                              const float *px, const float *py, const float *pz, const float *u, const float *v,
                              const float *w, const float *velB) {
  Items<float> P(it);
  const int Q = P.Q;
  IPCU_FOR(i, 0, P.nc) {
    float rx = px[i] - posB[0], ry = py[i] - posB[1], rz = pz[i] - posB[2];
    float X1 = quaS[0] * rx + quaS[1] * ry + quaS[2] * rz;
    float Y1 = quaS[3] * rx + quaS[4] * ry + quaS[5] * rz;
    float Z1 = quaS[6] * rx + quaS[7] * ry + quaS[8] * rz;
    if (Q == 27) Z1 = Y1;
    float d = (X1 / Ra) * (X1 / Ra) + (Z1 / Rb) * (Z1 / Rb);
    float pr = spm_profile2(P.dz / Ra, d);
    float fx = pr * (velB[0] - u[i]) / P.dt, fy = pr * (velB[1] - v[i]) / P.dt, fz = pr * (velB[2] - w[i]) / P.dt;
    for (int k = 0; k < Q; k++)
      f[i * Q + k] += P.w(k) * P.dt * 3.0f * (P.cx(k) * fx + P.cy(k) * fy + P.cz(k) * fz) / (P.c * P.c);
  }
}

}  // namespace
}  // namespace ipcu

using namespace ipcu;

#define LAUNCH(kern, ...)                                                     \
  do {                                                                        \
    ensure_tables();                                                          \
    Launch L_ = launch_for(nthreads);                                         \
    kern<<<L_.grid, L_.block, 0, (cudaStream_t)stream>>>(__VA_ARGS__);        \
    return status_from_cuda(cudaGetLastError());                              \
  } while (0)

#define DEF(T, S)                                                                                       \
  extern "C" int ipcu_get_IBMGw2_##S(T *items, int *lattice_id, int *neib, T *f, T *tau, T *posx, T *posy, \
                                     T *posz, T *posw, T *posB, T *nBvec, T *velx, T *vely, T *velz,    \
                                     T *velw, T *Fx, T *Fy, T *Fz, T *Gw, T rhof, int64_t nthreads,     \
                                     ipcu_stream_t stream) {                                           \
    (void)posB; (void)velx; (void)vely; (void)velz;                                                     \
    if (!items || !lattice_id || !neib || !f || !tau || !posw || !nBvec || !velw || !Gw) return IPCU_ERR_ARG; \
    LAUNCH(k_get_IBMGw2<T>, items, lattice_id, neib, f, tau, posx, posy, posz, posw, nBvec, velw, Fx, Fy, Fz, Gw, rhof); \
  }                                                                                                     \
  extern "C" int ipcu_update_velIBM_##S(T *items, int *lattice_id, T *f, T *ftmp, T *pressure, T *tau,   \
                                        T *velx, T *vely, T *velz, T *velx_old, T *vely_old,            \
                                        T *velz_old, T *Fx, T *Fy, T *Fz, int64_t nthreads,             \
                                        ipcu_stream_t stream) {                                        \
    (void)lattice_id; (void)ftmp; (void)tau; (void)velx_old; (void)vely_old; (void)velz_old;            \
    if (!items || !f || !pressure || !velx || !vely || !velz || !Fx || !Fy || !Fz) return IPCU_ERR_ARG; \
    LAUNCH(k_update_velIBM<T>, items, f, pressure, velx, vely, velz, Fx, Fy, Fz);                       \
  }                                                                                                     \
  extern "C" int ipcu_update_IBbody_##S(T *items, int IB_index, T *massB, T *densB, T *inertia, T *FB,   \
                                        T *posB, T *Torque, T *velB, T *quat, T *quaS, T *angleVB,      \
                                        T *posw, T *Gw, T *quatold, T rhof, int64_t nthreads,           \
                                        ipcu_stream_t stream) {                                        \
    (void)nthreads;                                                                                     \
    if (!items || !massB || !densB || !inertia || !FB || !posB || !Torque || !velB || !quat || !quaS || \
        !angleVB || !posw || !Gw || !quatold || IB_index < 0)                                           \
      return IPCU_ERR_ARG;                                                                              \
    ensure_tables();                                                                                    \
    k_update_IBbody<T><<<1, 256, 0, (cudaStream_t)stream>>>(items, IB_index, massB, densB, inertia, FB, \
                                                            posB, Torque, velB, quat, quaS, angleVB,    \
                                                            posw, Gw, quatold, rhof);                   \
    return status_from_cuda(cudaGetLastError());                                                        \
  }                                                                                                     \
  extern "C" int ipcu_update_IBpoint_##S(T *items, int IB_index, T *posB, T *velB, T *angleVB, T *quaS,   \
                                         T *posw, T *oposw, T *nBvec, T *onBvec, T *velw,               \
                                         int64_t nthreads, ipcu_stream_t stream) {                     \
    if (!items || IB_index < 0 || !posB || !velB || !angleVB || !quaS || !posw || !oposw || !nBvec ||   \
        !onBvec || !velw)                                                                               \
      return IPCU_ERR_ARG;                                                                              \
    LAUNCH(k_update_IBpoint<T>, items, IB_index, posB, velB, angleVB, quaS, posw, oposw, nBvec, onBvec, velw); \
  }                                                                                                     \
  extern "C" int ipcu_search_IBlattice_##S(T *items, int IB_index, int *lattice_id, int *neib, T *posx,  \
                                           T *posy, T *posz, T *posw, int64_t nthreads,                \
                                           ipcu_stream_t stream) {                                     \
    (void)IB_index;                                                                                     \
    if (!items || !lattice_id || !neib || !posx || !posy || !posz || !posw) return IPCU_ERR_ARG;        \
    LAUNCH(k_search_IBlattice<T>, items, lattice_id, neib, posx, posy, posz, posw);                     \
  }                                                                                                     \
  extern "C" int ipcu_SPM_##S(T *items, T Radius, T *posB, T *f, T *ftmp, T *tau, T *posx, T *posy,      \
                              T *Fx, T *Fy, T *Fz, T *velx, T *vely, T *velz, T *velw, int64_t nthreads, \
                              ipcu_stream_t stream) {                                                  \
    (void)tau;                                                                                          \
    if (!items || !posB || !f || !ftmp || !posx || !posy || !Fx || !velw) return IPCU_ERR_ARG;          \
    LAUNCH(k_SPM<T>, items, Radius, posB, f, ftmp, posx, posy, Fx, Fy, Fz, velx, vely, velz, velw);      \
  }

DEF(float, f32)
DEF(double, f64)
#undef DEF

extern "C" int ipcu_IB_directForcing_f32(float *items, int *lattice_id, int *neib, float *posx, float *posy,
                                         float *posz, float *posw, float *velx, float *vely, float *velz,
                                         float *velw, float *Fx, float *Fy, float *Fz, float *Gw,
                                         int64_t nthreads, ipcu_stream_t stream) {
  if (!items || !lattice_id || !neib || !posw || !velw || !Gw) return IPCU_ERR_ARG;
  LAUNCH(k_IB_directForcing, items, lattice_id, neib, posx, posy, posz, posw, velx, vely, velz, velw, Fx, Fy, Fz, Gw);
}

extern "C" int ipcu_SPM_ellipse_f32(float *items, float Rada, float Radb, float *quaS, float *posB, float *f,
                                    float *tau, float *posx, float *posy, float *posz, float *velx, float *vely,
                                    float *velz, float *velB, float *angleVB, int64_t nthreads,
                                    ipcu_stream_t stream) {
  (void)tau;
  (void)angleVB;
  if (!items || !quaS || !posB || !f || !posx || !posy || !posz || !velB) return IPCU_ERR_ARG;
  LAUNCH(k_SPM_ellipse, items, Rada, Radb, quaS, posB, f, posx, posy, posz, velx, vely, velz, velB);
}

// host-side rotation matrix (ref: function/ibm.cu:16-43)
extern "C" void ipcu_set_quaternionS_f64(int IB_index, double q0, double q1, double q2, double q3, double *quaS) {
  quat_rot(q0, q1, q2, q3, quaS + IB_index * 9);
}
extern "C" void ipcu_set_quaternionS_f32(int IB_index, float q0, float q1, float q2, float q3, float *quaS) {
  quat_rot(q0, q1, q2, q3, quaS + IB_index * 9);
}
