// Reference-compatible kernel entries, collision family.
//
// Each kernel keeps the argument order and the buffer contracts of the
// reference's function/collision.cu (array-of-structures f[cell*Q+k] over
// the compacted cell list, parameters in the items[] block) so a caller of
// the reference links against these unchanged. Inside, the kernels are
// written for sm_100a: Q is a compile-time constant (9 or 27, dispatched once
// per thread block from items[]), counts are converted once, loops are
// grid-stride over a grid sized from the caller's coverage, and every launch
// goes to the caller's stream.
#include "ipcu_common.cuh"

namespace ipcu {
namespace {

template <class T, int Q>
__device__ __forceinline__ T eq_term(const Items<T> &P, int k, T u, T v, T w, T usq_c2) {
  T eu = (P.cx(k) * u + P.cy(k) * v + P.cz(k) * w) / (P.c * P.c);
  return T(3) * eu + T(4.5) * eu * eu - T(1.5) * usq_c2;
}

// ---- equ_f: pressure-form equilibrium (ref: function/collision.cu:3-14)
template <class T, int Q>
__device__ void equ_f_body(const Items<T> &P, T *feq, const T *p, const T *u, const T *v, const T *w) {
  IPCU_FOR(i, 0, P.nc) {
    T ui = u[i], vi = v[i], wi = w[i], pi = p[i];
    T us = (ui * ui + vi * vi + wi * wi) / (P.c * P.c);
#pragma unroll
    for (int k = 0; k < Q; k++) feq[i * Q + k] = P.w(k) * (pi + eq_term<T, Q>(P, k, ui, vi, wi, us));
  }
}
template <class T>
__global__ void k_equ_f(const T *it, T *feq, const T *p, const T *u, const T *v, const T *w) {
  Items<T> P(it);
  if (P.Q == 9) equ_f_body<T, 9>(P, feq, p, u, v, w);
  else if (P.Q == 27) equ_f_body<T, 27>(P, feq, p, u, v, w);
}

// ---- equ_g: scalar equilibrium (ref: function/collision.cu:16-27)
template <class T, int Q>
__device__ void equ_g_body(const Items<T> &P, T *feq, const T *s, const T *u, const T *v, const T *w) {
  IPCU_FOR(i, 0, P.nc) {
    T ui = u[i], vi = v[i], wi = w[i], si = s[i];
    T us = (ui * ui + vi * vi + wi * wi) / (P.c * P.c);
#pragma unroll
    for (int k = 0; k < Q; k++) feq[i * Q + k] = P.w(k) * si * (T(1) + eq_term<T, Q>(P, k, ui, vi, wi, us));
  }
}
template <class T>
__global__ void k_equ_g(const T *it, T *feq, const T *s, const T *u, const T *v, const T *w) {
  Items<T> P(it);
  if (P.Q == 9) equ_g_body<T, 9>(P, feq, s, u, v, w);
  else if (P.Q == 27) equ_g_body<T, 27>(P, feq, s, u, v, w);
}

// ---- wall_function: Spalding law of the wall, Newton iterations for u_tau
// (ref: function/collision.cu:28-55)
template <class T>
__global__ void k_wall_function(const T *it, const T *dX, const T *dY, int x, int y, int z, int nw,
                                const int *wall, const T *u, const T *v, const T *w, T *Fx, T *Fy,
                                const T *rho) {
  Items<T> P(it);
  const T nu = P.scal(IT_nu);
  const T kap = T(0.41), B = T(5.5);
  const T eb = exp(-kap * B);
  IPCU_FOR(e, 0, nw) {
    int id = wall[e];
    T vol = dX[id] * dY[id] * P.dz;
    T au = sqrt(u[id] * u[id] + v[id] * v[id] + w[id] * w[id]);
    T eta = au * T(1e-7f) + T(1e-20f);
    T yd = T(x) * dX[id] / T(2) + T(y) * dY[id] / T(2) + T(z) * P.dz / T(2);
    T area = vol / (yd * T(2));
    T ut = au * T(0.11);
    for (int n = 0; n < 15; n++) {
      T t = kap * au / (ut + eta);
      T et = exp(t);
      T fv = au / (ut + eta) - yd * ut / nu + eb * (et - T(1) - t - t * t / T(2) - t * t * t / T(6));
      T dv = -yd / nu - au / (ut * ut + eta) + eb * t / (ut + eta) * (-et + T(1) + t + t * t / T(2)) + eta;
      ut += -(fv / dv);
    }
    T s = ut * ut * rho[id] * (area / vol) / (au + eta);
    Fx[id] += -u[id] * s;
    Fy[id] += -v[id] * s;
  }
}

// ---- Force: surface tension, buoyancy, pressure gradient; lattice
// projection Fk (ref: function/collision.cu:57-112)
template <class T, int Q>
__device__ void force_body(const Items<T> &P, bool bouss, const int *nb, T *Fk, T *Fx, T *Fy, T *Fz,
                           const T *pr, const T *rho, const T *sal, const T *phi, const T *u,
                           const T *v, const T *w, const T *dX, const T *px, const T *py, const T *pz) {
  constexpr int up = (Q == 27) ? 5 : 2, dn = (Q == 27) ? 6 : 4;
  const T reg = P.dz / T(1000);
  const T sig = P.scal(IT_sigma), W = P.scal(IT_PFthick);
  const T beta = T(12) * sig / W, kap = T(3) * sig * W / T(2);
  IPCU_FOR(i, 0, P.nc) {
    const int *n = nb + i * Q;
    const int n1 = n[1], n3 = n[3], n2 = n[2], n4 = n[4], nu_ = n[up], nd = n[dn];
    T gx = (phi[n1] - phi[n3]) / (px[n1] - px[n3] + reg);
    T gy = (Q == 27) ? (phi[n2] - phi[n4]) / (py[n2] - py[n4] + reg) : T(0);
    T gz = (phi[nu_] - phi[nd]) / (pz[nu_] - pz[nd] + reg);
    T ph = phi[i];
    T lap = (phi[n1] - T(2) * ph + phi[n3]) / (dX[i] * dX[i]) + (phi[n2] - T(2) * ph + phi[n4]) / (P.dz * P.dz);
    T st = T(4) * beta * ph * (ph - T(1)) * (ph - T(0.5)) - kap * lap;
    T fx = Fx[i] + st * gx, fy = Fy[i] + st * gy, fz = Fz[i] + st * gz;
    fz += bouss ? -sal[i] * T(0.824493) * T(9.81) : -rho[i] * T(9.81);
    gx = (rho[n1] - rho[n3]) / (px[n1] - px[n3] + reg);
    gy = (Q == 27) ? (rho[n2] - rho[n4]) / (py[n2] - py[n4] + reg) : T(0);
    gz = (rho[nu_] - rho[nd]) / (pz[nu_] - pz[nd] + reg);
    T pc = pr[i] * P.c * P.c / T(3);
    fx += -pc * gx;
    fy += -pc * gy;
    fz += -pc * gz;
    Fx[i] = fx;
    Fy[i] = fy;
    Fz[i] = fz;
    T den = rho[i] * P.c * P.c / T(3);
#pragma unroll
    for (int k = 0; k < Q; k++) Fk[i * Q + k] = P.w(k) * P.dt * (P.cx(k) * fx + P.cy(k) * fy + P.cz(k) * fz) / den;
  }
}
template <class T>
__global__ void k_Force(const T *it, int bouss, const int *nb, T *Fk, T *Fx, T *Fy, T *Fz, const T *pr,
                        const T *rho, const T *sal, const T *phi, const T *u, const T *v, const T *w,
                        const T *dX, const T *px, const T *py, const T *pz) {
  Items<T> P(it);
  if (P.Q == 9) force_body<T, 9>(P, bouss != 0, nb, Fk, Fx, Fy, Fz, pr, rho, sal, phi, u, v, w, dX, px, py, pz);
  else if (P.Q == 27) force_body<T, 27>(P, bouss != 0, nb, Fk, Fx, Fy, Fz, pr, rho, sal, phi, u, v, w, dX, px, py, pz);
}

// ---- col_f_MRT: f <- f - (MM + Minv[:,s] M[s,:]/tau)(f - feq + Fk/2) + Fk,
// shear rows s = {7,8} (Q9) or {5..9} (Q27); post-collision state to ftmp,
// f and feq zeroed (ref: function/collision.cu:115-150). The per-cell
// operator is assembled in shared memory-free registers: the shear
// projector rows are hoisted out of the Q loop.
template <class T, int Q>
__device__ void mrt_body(const Items<T> &P, const T *tau, T *f, T *ftmp, T *feq, const T *Fk, const T *M,
                         const T *Mi, const T *MM) {
  constexpr int s0 = (Q == 27) ? 5 : 7, ns = (Q == 27) ? 5 : 2;
  IPCU_FOR(i, 0, P.nc) {
    T d[Q], fi[Q], fk[Q];
    const T it_ = T(1) / tau[i];
#pragma unroll
    for (int k = 0; k < Q; k++) {
      fi[k] = f[i * Q + k];
      fk[k] = Fk[i * Q + k];
      d[k] = fi[k] - feq[i * Q + k] + fk[k] / T(2);
    }
    // shear moments m_l = M[s0+l,:] . d
    T m[ns];
#pragma unroll
    for (int l = 0; l < ns; l++) {
      T a = 0;
#pragma unroll
      for (int k = 0; k < Q; k++) a += __ldg(M + (s0 + l) * Q + k) * d[k];
      m[l] = a;
    }
#pragma unroll 1
    for (int a = 0; a < Q; a++) {
      T acc = 0;
#pragma unroll
      for (int k = 0; k < Q; k++) acc += __ldg(MM + a * Q + k) * d[k];
#pragma unroll
      for (int l = 0; l < ns; l++) acc += __ldg(Mi + a * Q + s0 + l) * m[l] * it_;
      ftmp[i * Q + a] = fi[a] - acc + fk[a];
    }
#pragma unroll
    for (int k = 0; k < Q; k++) {
      feq[i * Q + k] = T(0);
      f[i * Q + k] = T(0);
    }
  }
}
template <class T>
__global__ void k_col_f_MRT(const T *it, const T *tau, T *f, T *ftmp, T *feq, const T *Fk, const T *M,
                            const T *Mi, const T *MM) {
  Items<T> P(it);
  if (P.Q == 9) mrt_body<T, 9>(P, tau, f, ftmp, feq, Fk, M, Mi, MM);
  else if (P.Q == 27) mrt_body<T, 27>(P, tau, f, ftmp, feq, Fk, M, Mi, MM);
}

// ---- col_f_SRT (ref: function/collision.cu:151-165)
template <class T>
__global__ void k_col_f_SRT(const T *it, const T *tau, T *f, T *ftmp, T *feq, const T *Fk) {
  Items<T> P(it);
  const int Q = P.Q;
  IPCU_FOR(j, 0, P.nc * Q) {
    long long i = j / Q;
    T fj = f[j], fk = Fk[j];
    ftmp[j] = fj - (fj - feq[j] + fk / T(2)) / tau[i] + fk;
    f[j] = T(0);
    feq[j] = T(0);
  }
}

// ---- col_g_reg: regularised scalar collision (ref: function/collision.cu:167-188)
template <class T, int Q>
__device__ void greg_body(const Items<T> &P, const T *taus, T *g, T *gtmp, T *geq, const T *s, const T *u,
                          const T *v, const T *w) {
  IPCU_FOR(i, 0, P.nc) {
    T ui = u[i], vi = v[i], wi = w[i], si = s[i];
    T us = (ui * ui + vi * vi + wi * wi) / (P.c * P.c);
    T ge[Q], jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int k = 0; k < Q; k++) {
      ge[k] = P.w(k) * si * (T(1) + eq_term<T, Q>(P, k, ui, vi, wi, us));
      T ne = g[i * Q + k] - ge[k];
      jx += ne * P.cx(k);
      jy += ne * P.cy(k);
      jz += ne * P.cz(k);
    }
    const T om = T(1) - T(1) / taus[i];
#pragma unroll
    for (int k = 0; k < Q; k++) {
      T neq = P.w(k) * T(3) * (jx * P.cx(k) + jy * P.cy(k) + jz * P.cz(k)) / (P.c * P.c);
      gtmp[i * Q + k] = ge[k] + om * neq;
      geq[i * Q + k] = T(0);
      g[i * Q + k] = T(0);
    }
  }
}
template <class T>
__global__ void k_col_g_reg(const T *it, const T *taus, T *g, T *gtmp, T *geq, const T *s, const T *u,
                            const T *v, const T *w) {
  Items<T> P(it);
  if (P.Q == 9) greg_body<T, 9>(P, taus, g, gtmp, geq, s, u, v, w);
  else if (P.Q == 27) greg_body<T, 27>(P, taus, g, gtmp, geq, s, u, v, w);
}

// ---- col_PF: conservative Allen-Cahn collision (ref: function/collision.cu:190-223).
// Relaxation 0.5+0.08 and source weight 0.08 are the reference's constants.
template <class T, int Q>
__device__ void pf_body(const Items<T> &P, const int *nb, T *g, T *gtmp, T *geq, const T *phi, const T *u,
                        const T *v, const T *w, T *po, T *uo, T *vo, T *wo, const T *px, const T *py,
                        const T *pz) {
  constexpr int up = (Q == 27) ? 5 : 2, dn = (Q == 27) ? 6 : 4;
  const T reg = P.dz / T(1000), W = P.scal(IT_PFthick);
  IPCU_FOR(i, 0, P.nc) {
    const int *n = nb + i * Q;
    T gx = (phi[n[1]] - phi[n[3]]) / (px[n[1]] - px[n[3]] + reg);
    T gy = (Q == 27) ? (phi[n[2]] - phi[n[4]]) / (py[n[2]] - py[n[4]] + reg) : T(0);
    T gz = (phi[n[up]] - phi[n[dn]]) / (pz[n[up]] - pz[n[dn]] + reg);
    T ph = phi[i], ui = u[i], vi = v[i], wi = w[i];
    T du = (ph * ui - po[i] * uo[i]) / P.dt, dv = (ph * vi - po[i] * vo[i]) / P.dt, dw = (ph * wi - po[i] * wo[i]) / P.dt;
    po[i] = ph;
    uo[i] = ui;
    vo[i] = vi;
    wo[i] = wi;
    T inv_n = T(1) / sqrt(gx * gx + gy * gy + gz * gz + T(1e-8f));
    T us = (ui * ui + vi * vi + wi * wi) / (P.c * P.c);
    T lead = (T(1) - T(4) * (ph - T(0.5)) * (ph - T(0.5))) / W;
#pragma unroll
    for (int k = 0; k < Q; k++) {
      T ge = P.w(k) * ph * (T(1) + eq_term<T, Q>(P, k, ui, vi, wi, us));
      T src = P.dt * P.w(k) *
              (lead * (P.cx(k) * gx + P.cy(k) * gy + P.cz(k) * gz) * inv_n +
               T(3) * (P.cx(k) * du + P.cy(k) * dv + P.cz(k) * dw) / (P.c * P.c));
      T gk = g[i * Q + k];
      gtmp[i * Q + k] = gk - (gk - ge - src * T(0.08)) / (T(0.5) + T(0.08));
      geq[i * Q + k] = T(0);
      g[i * Q + k] = T(0);
    }
  }
}
template <class T>
__global__ void k_col_PF(const T *it, const int *nb, T *g, T *gtmp, T *geq, const T *phi, const T *u,
                         const T *v, const T *w, T *po, T *uo, T *vo, T *wo, const T *px, const T *py,
                         const T *pz) {
  Items<T> P(it);
  if (P.Q == 9) pf_body<T, 9>(P, nb, g, gtmp, geq, phi, u, v, w, po, uo, vo, wo, px, py, pz);
  else if (P.Q == 27) pf_body<T, 27>(P, nb, g, gtmp, geq, phi, u, v, w, po, uo, vo, wo, px, py, pz);
}

// ---- update_scalar (ref: function/collision.cu:225-236)
template <class T>
__global__ void k_update_scalar(const T *it, const T *g, T *s) {
  Items<T> P(it);
  const int Q = P.Q;
  IPCU_FOR(i, 0, P.nc) {
    T a = 0;
    for (int k = 0; k < Q; k++) a += g[i * Q + k];
    s[i] = a;
  }
}

// ---- update_rho: p*, u (+ F dt / 2 rho), rho(phi, S) (ref: function/collision.cu:238-257)
template <class T, int Q>
__device__ void rho_body(const Items<T> &P, T rhoL, T rhoH, const T *f, const T *Fx, const T *Fy, const T *Fz,
                         T *pr, const T *sal, const T *phi, T *rho, T *u, T *v, T *w) {
  IPCU_FOR(i, 0, P.nc) {
    T a = 0, b = 0, c = 0, d = 0;
#pragma unroll
    for (int k = 0; k < Q; k++) {
      T fk = f[i * Q + k];
      a += fk;
      b += P.cx(k) * fk;
      c += P.cy(k) * fk;
      d += P.cz(k) * fk;
    }
    T r = rhoL + (rhoH - rhoL) * phi[i] + sal[i] * T(0.824493);
    pr[i] = a;
    rho[i] = r;
    T h = P.dt / (T(2) * r);
    u[i] = b + Fx[i] * h;
    v[i] = c + Fy[i] * h;
    w[i] = d + Fz[i] * h;
  }
}
template <class T>
__global__ void k_update_rho(const T *it, T rhoL, T rhoH, const T *f, const T *Fx, const T *Fy, const T *Fz,
                             T *pr, const T *sal, const T *phi, T *rho, T *u, T *v, T *w) {
  Items<T> P(it);
  if (P.Q == 9) rho_body<T, 9>(P, rhoL, rhoH, f, Fx, Fy, Fz, pr, sal, phi, rho, u, v, w);
  else if (P.Q == 27) rho_body<T, 27>(P, rhoL, rhoH, f, Fx, Fy, Fz, pr, sal, phi, rho, u, v, w);
}

// ---- resetF (ref: function/collision.cu:258-264)
template <class T>
__global__ void k_resetF(T *Fx, T *Fy, T *Fz, int n) {
  IPCU_FOR(i, 0, n) {
    Fx[i] = T(0);
    Fy[i] = T(0);
    Fz[i] = T(0);
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
  extern "C" int ipcu_equ_f_##S(T *items, T *feq, T *pressure, T *velx, T *vely, T *velz,               \
                                int64_t nthreads, ipcu_stream_t stream) {                              \
    if (!items || !feq || !pressure || !velx || !vely || !velz) return IPCU_ERR_ARG;                    \
    LAUNCH(k_equ_f<T>, items, feq, pressure, velx, vely, velz);                                         \
  }                                                                                                     \
  extern "C" int ipcu_equ_g_##S(T *items, T *feq, T *sal, T *velx, T *vely, T *velz, int64_t nthreads,  \
                                ipcu_stream_t stream) {                                                \
    if (!items || !feq || !sal || !velx || !vely || !velz) return IPCU_ERR_ARG;                         \
    LAUNCH(k_equ_g<T>, items, feq, sal, velx, vely, velz);                                              \
  }                                                                                                     \
  extern "C" int ipcu_wall_function_##S(T *items, T *delX, T *delY, int x, int y, int z, int wall_number, \
                                        int *wall, T *velx, T *vely, T *velz, T *Fx, T *Fy, T *rho,     \
                                        int64_t nthreads, ipcu_stream_t stream) {                      \
    if (!items || (wall_number > 0 && !wall)) return IPCU_ERR_ARG;                                      \
    if (wall_number <= 0) return IPCU_OK;                                                               \
    LAUNCH(k_wall_function<T>, items, delX, delY, x, y, z, wall_number, wall, velx, vely, velz, Fx, Fy, rho); \
  }                                                                                                     \
  extern "C" int ipcu_Force_##S(T *items, int Boussi_flag, int *neib, T *f, T *feq, T *tau, T *Fk, T *Fx,  \
                                T *Fy, T *Fz, T *pressure, T *rho, T *sal, T *phi, T *velx, T *vely,   \
                                T *velz, T *delX, T *delY, T *posx, T *posy, T *posz, int64_t nthreads, \
                                ipcu_stream_t stream) {                                                \
    (void)f; (void)feq; (void)tau; (void)delY;                                                          \
    if (!items || !neib || !Fk || !Fx || !Fy || !Fz) return IPCU_ERR_ARG;                               \
    LAUNCH(k_Force<T>, items, Boussi_flag, neib, Fk, Fx, Fy, Fz, pressure, rho, sal, phi, velx, vely,   \
           velz, delX, posx, posy, posz);                                                               \
  }                                                                                                     \
  extern "C" int ipcu_col_f_MRT_##S(T *items, T *tau, T *f, T *ftmp, T *feq, T *Fk, T *M, T *M_inv, T *S_, \
                                    T *Mconst, int64_t nthreads, ipcu_stream_t stream) {               \
    (void)S_;                                                                                           \
    if (!items || !tau || !f || !ftmp || !feq || !Fk || !M || !M_inv || !Mconst) return IPCU_ERR_ARG;   \
    LAUNCH(k_col_f_MRT<T>, items, tau, f, ftmp, feq, Fk, M, M_inv, Mconst);                             \
  }                                                                                                     \
  extern "C" int ipcu_col_f_SRT_##S(T *items, T *tau, T *f, T *ftmp, T *feq, T *Fk, int64_t nthreads,   \
                                    ipcu_stream_t stream) {                                            \
    if (!items || !tau || !f || !ftmp || !feq || !Fk) return IPCU_ERR_ARG;                              \
    LAUNCH(k_col_f_SRT<T>, items, tau, f, ftmp, feq, Fk);                                               \
  }                                                                                                     \
  extern "C" int ipcu_col_g_reg_##S(T *items, T *taus, T *g, T *gtmp, T *geq, T *sal, T *velx, T *vely, \
                                    T *velz, int64_t nthreads, ipcu_stream_t stream) {                 \
    if (!items || !taus || !g || !gtmp || !geq || !sal) return IPCU_ERR_ARG;                            \
    LAUNCH(k_col_g_reg<T>, items, taus, g, gtmp, geq, sal, velx, vely, velz);                           \
  }                                                                                                     \
  extern "C" int ipcu_col_PF_##S(T *items, int *neib, T *taus, T *g, T *gtmp, T *geq, T *phi, T *velx,  \
                                 T *vely, T *velz, T *phiold, T *uold, T *vold, T *wold, T *posx,       \
                                 T *posy, T *posz, int64_t nthreads, ipcu_stream_t stream) {           \
    (void)taus;                                                                                         \
    if (!items || !neib || !g || !gtmp || !geq || !phi) return IPCU_ERR_ARG;                            \
    LAUNCH(k_col_PF<T>, items, neib, g, gtmp, geq, phi, velx, vely, velz, phiold, uold, vold, wold,     \
           posx, posy, posz);                                                                           \
  }                                                                                                     \
  extern "C" int ipcu_update_scalar_##S(T *items, T *g, T *scalar, int64_t nthreads,                    \
                                        ipcu_stream_t stream) {                                        \
    if (!items || !g || !scalar) return IPCU_ERR_ARG;                                                   \
    LAUNCH(k_update_scalar<T>, items, g, scalar);                                                       \
  }                                                                                                     \
  extern "C" int ipcu_update_rho_##S(T *items, T rhoL, T rhoH, T *f, T *Fx, T *Fy, T *Fz, T *pressure,  \
                                     T *sal, T *phi, T *rho, T *velx, T *vely, T *velz,                 \
                                     int64_t nthreads, ipcu_stream_t stream) {                         \
    if (!items || !f || !pressure || !rho) return IPCU_ERR_ARG;                                         \
    LAUNCH(k_update_rho<T>, items, rhoL, rhoH, f, Fx, Fy, Fz, pressure, sal, phi, rho, velx, vely, velz); \
  }                                                                                                     \
  extern "C" int ipcu_resetF_##S(T *items, T *Fx, T *Fy, T *Fz, int num_F, int64_t nthreads,            \
                                 ipcu_stream_t stream) {                                               \
    (void)items;                                                                                        \
    if (!Fx || !Fy || !Fz) return IPCU_ERR_ARG;                                                         \
    if (num_F <= 0) return IPCU_OK;                                                                     \
    if (nthreads <= 0) nthreads = num_F;                                                                \
    LAUNCH(k_resetF<T>, Fx, Fy, Fz, num_F);                                                             \
  }

DEF(float, f32)
DEF(double, f64)
#undef DEF
