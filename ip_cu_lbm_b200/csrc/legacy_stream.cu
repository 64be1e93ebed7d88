// Reference-compatible kernel entries, streaming family: the conservative
// interpolated streaming pass IP_process and its ten stages, the pull
// propagation, ghost-cell boundaries, and the small per-cell utilities of
// function/basic.cu. Argument order and buffer roles follow the reference
// (ref: function/adv.cu, propagation.cu, set_bound.cu, basic.cu).
#include "ipcu_common.cuh"

namespace ipcu {
namespace {

// ---- set_wall_f: ghost <- copy of its owner (ref: function/adv.cu:3-13)
template <class T>
__global__ void k_set_wall_f(const T *it, const int *nb, T *f) {
  Items<T> P(it);
  const int Q = P.Q;
  IPCU_FOR(j, P.nc * Q, (P.nc + P.nw) * Q) {
    long long g = j / Q;
    int k = (int)(j - g * Q);
    f[j] = f[(long long)nb[g * Q] * Q + k];
  }
}

// Ghost stencil nodes carry their owner's coordinate; they are placed one
// lattice spacing beyond the previous node (ref: function/adv.cu:16-28).
template <class T>
__device__ __forceinline__ void clamp5(T *pl, T s, T dz) {
  if (s == T(1)) {
    pl[1] = fmin(pl[1], pl[2] - dz);
    pl[0] = fmin(pl[0], pl[1] - dz);
    pl[3] = fmax(pl[3], pl[2] + dz);
    pl[4] = fmax(pl[4], pl[3] + dz);
  } else if (s == T(-1)) {
    pl[1] = fmax(pl[1], pl[2] + dz);
    pl[0] = fmax(pl[0], pl[1] + dz);
    pl[3] = fmin(pl[3], pl[2] - dz);
    pl[4] = fmin(pl[4], pl[3] - dz);
  } else {
#pragma unroll
    for (int a = 0; a < 5; a++) pl[a] = T(0);
  }
}
// 5-point Lagrange weights at xa (ref: function/adv.cu:40-48)
template <class T>
__device__ __forceinline__ void lag5(T *cf, const T *pl, T xa) {
#pragma unroll
  for (int a = 0; a < 5; a++) {
    T v = T(1);
#pragma unroll
    for (int b = 0; b < 5; b++)
      if (b != a) v *= (xa - pl[b]) / (pl[a] - pl[b]);
    cf[a] = v;
  }
}

// ---- set_out: conservative flux form of the interpolated streaming
// (ref: function/adv.cu:50-147). fout = I(x_c + s(dx_c - dz)/2) dz/dx_c,
// fin = same dz/dx_{c+}; Q27 xy-diagonals use the 5x5 tensor stencil and
// scatter corner fluxes with atomics into fin / finy.
template <class T, int Q>
__device__ void set_out_body(const Items<T> &P, const int *nb, const T *ftmp, T *fout, T *fin, T *finy,
                             const T *px, const T *py, const T *dX, const T *dY) {
  constexpr int qs = (Q == 27) ? 1 : 0;
  auto N = [&](long long cell, int d) -> long long { return (long long)nb[cell * Q + d]; };
  IPCU_FOR(i, 0, P.nc) {
    const long long b = i * Q;
    const T dz = P.dz;
    auto axis = [&](int k, const T *pos, const T *del, T s) {
      long long a1 = N(i, c_dirs.cm[qs][k]), b1 = N(i, c_dirs.cp[qs][k]);
      long long a2 = N(a1, c_dirs.cm[qs][k]), b2 = N(b1, c_dirs.cp[qs][k]);
      T xa = pos[i] + s * (del[i] - dz) / T(2);
      T pl[5] = {pos[a2], pos[a1], pos[i], pos[b1], pos[b2]};
      clamp5(pl, s, dz);
      T cf[5];
      lag5(cf, pl, xa);
      T val = cf[0] * ftmp[a2 * Q + k] + cf[1] * ftmp[a1 * Q + k] + cf[2] * ftmp[b + k] + cf[3] * ftmp[b1 * Q + k] +
              cf[4] * ftmp[b2 * Q + k];
      fin[b + k] = val * (dz / del[b1]);
      fout[b + k] = val * (dz / del[i]);
    };
    if (Q == 9) {
      fout[b + 0] = fin[b + 0] = ftmp[b + 0];
      fout[b + 2] = fin[b + 2] = ftmp[b + 2];
      fout[b + 4] = fin[b + 4] = ftmp[b + 4];
      const int kx[6] = {1, 3, 5, 6, 7, 8};
#pragma unroll
      for (int e = 0; e < 6; e++) axis(kx[e], px, dX, P.cx(kx[e]) / P.c);
    } else {
      fout[b + 0] = fin[b + 0] = ftmp[b + 0];
      fout[b + 5] = fin[b + 5] = ftmp[b + 5];
      fout[b + 6] = fin[b + 6] = ftmp[b + 6];
      const int kx[6] = {1, 3, 11, 13, 12, 14}, ky[6] = {2, 4, 15, 17, 16, 18};
      for (int e = 0; e < 6; e++) axis(kx[e], px, dX, P.cx(kx[e]) / P.c);
      for (int e = 0; e < 6; e++) axis(ky[e], py, dY, P.cy(ky[e]) / P.c);
      for (int e = 0; e < 12; e++) {
        const int k = (e < 4) ? 7 + e : (e < 8 ? 19 + (e - 4) : 23 + (e - 8));
        long long id[25];
        id[12] = i;
        id[13] = N(i, c_dirs.cxp[k]);
        id[14] = N(id[13], c_dirs.cxp[k]);
        id[11] = N(i, c_dirs.cxm[k]);
        id[10] = N(id[11], c_dirs.cxm[k]);
        id[17] = N(i, c_dirs.cyp[k]);
        id[22] = N(id[17], c_dirs.cyp[k]);
        id[7] = N(i, c_dirs.cym[k]);
        id[2] = N(id[7], c_dirs.cym[k]);
        id[18] = N(i, c_dirs.cp[1][k]);
        id[24] = N(id[18], c_dirs.cp[1][k]);
        id[6] = N(i, c_dirs.cm[1][k]);
        id[0] = N(id[6], c_dirs.cm[1][k]);
        id[8] = N(i, c_dirs.cip[k]);
        id[4] = N(id[8], c_dirs.cip[k]);
        id[16] = N(i, c_dirs.cim[k]);
        id[20] = N(id[16], c_dirs.cim[k]);
        id[19] = N(id[14], c_dirs.cyp[k]);
        id[9] = N(id[14], c_dirs.cym[k]);
        id[15] = N(id[10], c_dirs.cyp[k]);
        id[5] = N(id[10], c_dirs.cym[k]);
        id[23] = N(id[22], c_dirs.cxp[k]);
        id[21] = N(id[22], c_dirs.cxm[k]);
        id[3] = N(id[2], c_dirs.cxp[k]);
        id[1] = N(id[2], c_dirs.cxm[k]);
        T sx = P.cx(k) / P.c, sy = P.cy(k) / P.c;
        T pl[5] = {px[id[10]], px[id[11]], px[i], px[id[13]], px[id[14]]}, cxw[5], cyw[5];
        clamp5(pl, sx, dz);
        lag5(cxw, pl, (T)(px[i] + sx * (dX[i] - dz) / T(2)));
        T ql[5] = {py[id[2]], py[id[7]], py[i], py[id[17]], py[id[22]]};
        clamp5(ql, sy, dz);
        lag5(cyw, ql, (T)(py[i] + sy * (dY[i] - dz) / T(2)));
        T fx = 0, fy = 0, fxy = 0;
#pragma unroll
        for (int a = 0; a < 5; a++) {
          fx += cxw[a] * ftmp[id[10 + a] * Q + k];
          fy += cyw[a] * ftmp[id[2 + 5 * a] * Q + k];
        }
#pragma unroll
        for (int a = 0; a < 5; a++)
#pragma unroll
          for (int c = 0; c < 5; c++) fxy += cxw[a] * cyw[c] * ftmp[id[a + 5 * c] * Q + k];
        fout[b + k] = fx * dz / dX[i] + fy * dz / dY[i] - fxy * (dz * dz) / (dX[i] * dY[i]);
        atomicAdd(&fin[b + k], fxy * (dz * dz) / (dX[id[13]] * dY[id[17]]));
        atomicAdd(&fin[N(i, c_dirs.cxm[k]) * Q + k], (fy - fxy * dz / dX[id[17]]) * dz / dY[id[17]]);
        atomicAdd(&finy[N(i, c_dirs.cym[k]) * Q + k], (fx - fxy * dz / dY[id[13]]) * dz / dX[id[13]]);
      }
    }
  }
}
template <class T>
__global__ void k_set_out(const T *it, const int *nb, const T *ftmp, T *fout, T *fin, T *finy, const T *px,
                          const T *py, const T *dX, const T *dY) {
  Items<T> P(it);
  if (P.Q == 9) set_out_body<T, 9>(P, nb, ftmp, fout, fin, finy, px, py, dX, dY);
  else if (P.Q == 27) set_out_body<T, 27>(P, nb, ftmp, fout, fin, finy, px, py, dX, dY);
}

// ---- set_fin: Q27 only, ghost-cell fluxes handed to the fluid neighbour
// (ref: function/adv.cu:148-175). The (1 - n/g) factor is 1 when the
// neighbour is the owner and 0 when it is the ghost itself.
template <class T>
__global__ void k_set_fin(const T *it, const int *nb, T *fin, T *finy) {
  Items<T> P(it);
  if (P.Q != 27) return;
  constexpr int Q = 27;
  const int nk[8] = {9, 8, 10, 7, 7, 10, 8, 9}, nkz[8] = {19, 20, 21, 22, 23, 24, 25, 26},
            nn[8] = {1, 2, 1, 4, 3, 2, 3, 4};
  IPCU_FOR(g, P.nc, P.nc + P.nw) {
    const long long b = g * Q;
    for (int k = 0; k < 4; k++) {
      const int k0 = 7 + k, k4 = 19 + 2 * k, k8 = 20 + 2 * k;
      long long A = nb[b + nn[2 * k]];
      T fa = T(1 - A / g);
      int d0 = nk[2 * (k0 - 7)];
      fin[A * Q + d0] += fin[b + k0] * fa;
      fin[A * Q + nkz[2 * (d0 - 7)]] += fin[b + k4] * fa;
      fin[A * Q + nkz[2 * (d0 - 7) + 1]] += fin[b + k8] * fa;
      long long B = nb[b + nn[2 * k + 1]];
      T fb = T(1 - B / g);
      int d1 = nk[2 * (k0 - 7) + 1];
      finy[B * Q + d1] += finy[b + k0] * fb;
      finy[B * Q + nkz[2 * (d1 - 7)]] += finy[b + k4] * fb;
      finy[B * Q + nkz[2 * (d1 - 7) + 1]] += finy[b + k8] * fb;
    }
  }
}

// ---- reset_f: fin += finy; f <- ftmp (ref: function/adv.cu:176-187)
template <class T>
__global__ void k_reset_f(const T *it, const T *ftmp, T *fin, T *f) {
  Items<T> P(it);
  IPCU_FOR(j, 0, P.nc * P.Q) {
    fin[j] += f[j];
    f[j] = ftmp[j];
  }
}

// ---- set_wall_f_inv: ghost <- owner mirrored across the x (and y) wall
// (ref: function/adv.cu:188-232). In D2Q9 directions 2 and 4 map to the
// owner's rest population, as in the reference table.
template <class T>
__global__ void k_set_wall_f_inv(const T *it, const int *nb, const int *nextB, const int *nextK, T *f) {
  Items<T> P(it);
  const int Q = P.Q;
  IPCU_FOR(g, P.nc, P.nc + P.nw) {
    const long long b = g * Q, o = nb[b];
    if (Q == 9) {
      const int mx[9] = {0, 3, 0, 1, 0, 6, 5, 8, 7};
#pragma unroll
      for (int k = 1; k < 9; k++) f[b + k] = f[o * Q + mx[k]];
    } else if (Q == 27) {
      const int nkz[8] = {20, 19, 22, 21, 24, 23, 26, 25};
      const int mxy[19] = {0, 3, 4, 1, 2, 0, 0, 0, 0, 0, 0, 13, 14, 11, 12, 17, 18, 15, 16};
      for (int e = 0; e < 15; e++) {
        int k = (e < 7) ? e : (e < 14 ? 11 + (e - 7) : 18);
        f[b + k] = f[o * Q + mxy[k]];
      }
      const long long wb = (g - P.nc) * Q;
      for (int k = 0; k < 4; k++) {
        const int k0 = 7 + k, k4 = 19 + 2 * k, k8 = 20 + 2 * k;
        const int ik = c_dirs.kinv[1][k0];
        int nk = c_dirs.kinv[1][nextK[wb + ik]], neB = nextB[wb + ik];
        long long s = nb[o * Q + neB];
        f[b + k0] = f[s * Q + nk];
        f[b + k4] = f[s * Q + nkz[2 * (nk - 7) + 1]];
        f[b + k8] = f[s * Q + nkz[2 * (nk - 7)]];
      }
    }
  }
}

// ---- set_tmp: candidate post-stream value f(c+) + (fin(c) - fout(c+))
// (ref: function/adv.cu:234-244)
template <class T>
__global__ void k_set_tmp(const T *it, const int *nb, const T *f, T *ftmp, const T *fout, const T *fin) {
  Items<T> P(it);
  const int Q = P.Q, qs = qsel(Q);
  IPCU_FOR(j, 0, P.nc * Q) {
    long long i = j / Q;
    int k = (int)(j - i * Q);
    long long s = nb[i * Q + c_dirs.cp[qs][k]];
    ftmp[j] = f[s * Q + k] + (fin[j] - fout[s * Q + k]);
  }
}

// ---- set_wall_propagation: bounce-back (1) or specular slip (0) ghosts
// (ref: function/set_bound.cu:164-183)
template <class T>
__global__ void k_set_wall_propagation(const T *it, int bc, const int *nb, const int *nextK, const int *nextB,
                                       T *ftmp) {
  Items<T> P(it);
  const int Q = P.Q, qs = qsel(Q);
  IPCU_FOR(g, P.nc, P.nc + P.nw) {
    const long long b = g * Q, o = nb[b], wb = (g - P.nc) * Q;
    if (bc == 1) {
      for (int k = 1; k < Q; k++) ftmp[b + k] = ftmp[o * Q + c_dirs.kinv[qs][k]];
    } else if (bc == 0) {
      for (int k = 1; k < Q; k++) {
        long long s = nb[o * Q + nextB[wb + k]];
        ftmp[b + k] = ftmp[s * Q + nextK[wb + k]];
      }
    }
  }
}

// ---- propagation: pull shift f(c) <- ftmp(neib(c, -k)) (ref: function/propagation.cu:2-12)
template <class T>
__global__ void k_propagation(const T *it, const int *nb, T *f, const T *ftmp) {
  Items<T> P(it);
  const int Q = P.Q, qs = qsel(Q);
  IPCU_FOR(j, 0, P.nc * Q) {
    long long i = j / Q;
    int k = (int)(j - i * Q);
    f[j] = ftmp[(long long)nb[i * Q + c_dirs.kinv[qs][k]] * Q + k];
  }
}

// ---- reset_wall_fin (ref: function/basic.cu:274-284)
template <class T>
__global__ void k_reset_wall_fin(const T *it, T *fin, T *finy) {
  Items<T> P(it);
  IPCU_FOR(j, P.nc * P.Q, (P.nc + P.nw) * P.Q) {
    fin[j] = T(0);
    finy[j] = T(0);
  }
}

// ---- set_wall_rho: ghost copies its owner's value (ref: function/basic.cu:254-261)
template <class T>
__global__ void k_set_wall_rho(const T *it, const int *nb, T *rho) {
  Items<T> P(it);
  IPCU_FOR(g, P.nc, P.nc + P.nw) rho[g] = rho[nb[g * P.Q]];
}

// ---- reset_pressure: rescale p* and re-equilibrate f after a dt change
// (ref: function/basic.cu:262-273)
template <class T>
__global__ void k_reset_pressure(const T *it, T *pr, T *f, const T *u, const T *v, const T *w, T alpha) {
  Items<T> P(it);
  const int Q = P.Q;
  IPCU_FOR(i, 0, P.nc) {
    T p = pr[i] / (alpha * alpha);
    pr[i] = p;
    T ui = u[i], vi = v[i], wi = w[i];
    T us = (ui * ui + vi * vi + wi * wi) / (P.c * P.c);
    for (int k = 0; k < Q; k++) {
      T eu = (P.cx(k) * ui + P.cy(k) * vi + P.cz(k) * wi) / (P.c * P.c);
      f[i * Q + k] = P.w(k) * (p + T(3) * eu + T(4.5) * eu * eu - T(1.5) * us);
    }
  }
}

// ---- LES: coherent-structure Smagorinsky sub-grid viscosity -> tau, taus
// (ref: function/basic.cu:285-339). In D2Q9 the reference's z-gradient
// stencil uses the same neighbour twice (up = down = 2), so it is zero.
template <class T>
__global__ void k_LES(const T *it, const int *nb, T *tau, T *taus, const T *phi, const T *rho, T muL, T muH,
                      const T *u, const T *v, const T *w, const T *px, const T *py, const T *pz) {
  Items<T> P(it);
  const int Q = P.Q, up = (Q == 27) ? 5 : 2, dn = (Q == 27) ? 6 : 2;
  const T reg = P.dz / T(1000);
  IPCU_FOR(i, 0, P.nc) {
    const int *n = nb + i * Q;
    const T *vel[3] = {u, v, w};
    T g[3][3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      g[0][a] = (vel[a][n[1]] - vel[a][n[3]]) / (px[n[1]] - px[n[3]] + reg);
      g[1][a] = (Q == 27) ? (vel[a][n[2]] - vel[a][n[4]]) / (py[n[2]] - py[n[4]] + reg) : T(0);
      g[2][a] = (vel[a][n[up]] - vel[a][n[dn]]) / (pz[n[up]] - pz[n[dn]] + reg);
    }
    T S = 0, Qc = 0, sum = 0;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) {
        T sab = (g[a][b] + g[b][a]) / T(2);
        S += sqrt(T(2) * sab * sab);
        Qc += g[a][b] * g[b][a];
        sum += g[a][b];
      }
    Qc *= T(-0.5);
    T E = T(1) / (T(2) * sum * sum + T(1e-40f));
    T Fcs = fmax(T(-1), fmin(Qc / E, T(1)));
    T C = T(0.05) * pow(fabs(Fcs), T(1.5));
    tau[i] = T(3) * ((muL + phi[i] * (muH - muL)) / rho[i] + C * S * P.dz * P.dz) / (P.c * P.c * P.dt) + T(0.5);
    taus[i] = T(3) * (T(1e-9f) + C * S * P.dz * P.dz / T(1000)) / (P.c * P.c * P.dt) + T(0.5);
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
  extern "C" int ipcu_set_wall_f_##S(T *items, int *neib, T *f, int64_t nthreads, ipcu_stream_t stream) { \
    if (!items || !neib || !f) return IPCU_ERR_ARG;                                                     \
    LAUNCH(k_set_wall_f<T>, items, neib, f);                                                            \
  }                                                                                                     \
  extern "C" int ipcu_set_out_##S(T *items, int *neib, T *ftmp, T *fout, T *fin, T *finy, T *posx,       \
                                  T *posy, T *delX, T *delY, int64_t nthreads, ipcu_stream_t stream) { \
    if (!items || !neib || !ftmp || !fout || !fin || !finy || !posx || !delX) return IPCU_ERR_ARG;      \
    LAUNCH(k_set_out<T>, items, neib, ftmp, fout, fin, finy, posx, posy, delX, delY);                   \
  }                                                                                                     \
  extern "C" int ipcu_set_fin_##S(T *items, int *neib, int *nextK, T *fin, T *finy, int64_t nthreads,   \
                                  ipcu_stream_t stream) {                                              \
    (void)nextK;                                                                                        \
    if (!items || !neib || !fin || !finy) return IPCU_ERR_ARG;                                          \
    LAUNCH(k_set_fin<T>, items, neib, fin, finy);                                                       \
  }                                                                                                     \
  extern "C" int ipcu_reset_f_##S(T *items, T *ftmp, T *fin, T *f, int64_t nthreads, ipcu_stream_t stream) { \
    if (!items || !ftmp || !fin || !f) return IPCU_ERR_ARG;                                             \
    LAUNCH(k_reset_f<T>, items, ftmp, fin, f);                                                          \
  }                                                                                                     \
  extern "C" int ipcu_set_wall_f_inv_##S(T *items, int *neib, int *nextB, int *nextK, T *f,             \
                                         int64_t nthreads, ipcu_stream_t stream) {                     \
    if (!items || !neib || !f) return IPCU_ERR_ARG;                                                     \
    LAUNCH(k_set_wall_f_inv<T>, items, neib, nextB, nextK, f);                                          \
  }                                                                                                     \
  extern "C" int ipcu_set_tmp_##S(T *items, int *neib, T *f, T *ftmp, T *fout, T *fin, int64_t nthreads, \
                                  ipcu_stream_t stream) {                                              \
    if (!items || !neib || !f || !ftmp || !fout || !fin) return IPCU_ERR_ARG;                           \
    LAUNCH(k_set_tmp<T>, items, neib, f, ftmp, fout, fin);                                              \
  }                                                                                                     \
  extern "C" int ipcu_set_wall_propagation_##S(T *items, int boundary_condition, int *neib, int *nextK,  \
                                               int *nextB, T *ftmp, int64_t nthreads,                  \
                                               ipcu_stream_t stream) {                                 \
    if (!items || !neib || !ftmp) return IPCU_ERR_ARG;                                                  \
    if (boundary_condition == 0 && (!nextK || !nextB)) return IPCU_ERR_ARG;                             \
    LAUNCH(k_set_wall_propagation<T>, items, boundary_condition, neib, nextK, nextB, ftmp);             \
  }                                                                                                     \
  extern "C" int ipcu_propagation_##S(T *items, int *neib, T *f, T *ftmp, int64_t nthreads,             \
                                      ipcu_stream_t stream) {                                          \
    if (!items || !neib || !f || !ftmp) return IPCU_ERR_ARG;                                            \
    LAUNCH(k_propagation<T>, items, neib, f, ftmp);                                                     \
  }                                                                                                     \
  extern "C" int ipcu_reset_wall_fin_##S(T *items, T *fin, T *finy, int64_t nthreads,                   \
                                         ipcu_stream_t stream) {                                       \
    if (!items || !fin || !finy) return IPCU_ERR_ARG;                                                   \
    LAUNCH(k_reset_wall_fin<T>, items, fin, finy);                                                      \
  }                                                                                                     \
  extern "C" int ipcu_set_wall_rho_##S(T *items, int *neib, T *rho, int64_t nthreads,                   \
                                       ipcu_stream_t stream) {                                         \
    if (!items || !neib || !rho) return IPCU_ERR_ARG;                                                   \
    LAUNCH(k_set_wall_rho<T>, items, neib, rho);                                                        \
  }                                                                                                     \
  extern "C" int ipcu_reset_pressure_##S(T *items, T *pressure, T *f, T *velx, T *vely, T *velz, T alpha, \
                                         int64_t nthreads, ipcu_stream_t stream) {                     \
    if (!items || !pressure || !f) return IPCU_ERR_ARG;                                                 \
    LAUNCH(k_reset_pressure<T>, items, pressure, f, velx, vely, velz, alpha);                           \
  }                                                                                                     \
  extern "C" int ipcu_LES_##S(T *items, int *neib, T *tau, T *taus, T *phi, T *rho, T muL, T muH,        \
                              T *velx, T *vely, T *velz, T *posx, T *posy, T *posz, int64_t nthreads,   \
                              ipcu_stream_t stream) {                                                  \
    if (!items || !neib || !tau || !taus) return IPCU_ERR_ARG;                                          \
    LAUNCH(k_LES<T>, items, neib, tau, taus, phi, rho, muL, muH, velx, vely, velz, posx, posy, posz);   \
  }                                                                                                     \
  /* The ten-stage streaming pass (ref: function/adv.cu:245-257). feq is   */                           \
  /* reused as fin and f as finy; numBlocks*blockSize is the coverage.     */                           \
  extern "C" int ipcu_IP_process_##S(T *d_items, int numBlocks, int blockSize, int *d_neib, T *d_f,      \
                                     T *d_feq, T *d_ftmp, T *d_fout, int *d_nextB, int *d_nextK,        \
                                     T *d_posx, T *d_posy, T *d_delX, T *d_delY, int slip,               \
                                     ipcu_stream_t stream) {                                           \
    if (!d_items || !d_neib || !d_f || !d_feq || !d_ftmp || !d_fout || !d_posx || !d_delX)              \
      return IPCU_ERR_ARG;                                                                              \
    if (slip == 0 && (!d_nextB || !d_nextK)) return IPCU_ERR_ARG;                                       \
    int64_t nthreads = (int64_t)numBlocks * (int64_t)blockSize;                                         \
    int st;                                                                                             \
    if ((st = ipcu_set_wall_f_##S(d_items, d_neib, d_ftmp, nthreads, stream))) return st;               \
    if ((st = ipcu_set_out_##S(d_items, d_neib, d_ftmp, d_fout, d_feq, d_f, d_posx, d_posy, d_delX,     \
                               d_delY, nthreads, stream)))                                              \
      return st;                                                                                        \
    if ((st = ipcu_set_fin_##S(d_items, d_neib, d_nextK, d_feq, d_f, nthreads, stream))) return st;     \
    if ((st = ipcu_reset_f_##S(d_items, d_ftmp, d_feq, d_f, nthreads, stream))) return st;              \
    if ((st = ipcu_set_wall_f_inv_##S(d_items, d_neib, d_nextB, d_nextK, d_f, nthreads, stream))) return st; \
    if ((st = ipcu_set_wall_f_inv_##S(d_items, d_neib, d_nextB, d_nextK, d_fout, nthreads, stream))) return st; \
    if ((st = ipcu_set_tmp_##S(d_items, d_neib, d_f, d_ftmp, d_fout, d_feq, nthreads, stream))) return st; \
    if ((st = ipcu_set_wall_propagation_##S(d_items, slip, d_neib, d_nextK, d_nextB, d_ftmp, nthreads, stream))) \
      return st;                                                                                        \
    if ((st = ipcu_propagation_##S(d_items, d_neib, d_f, d_ftmp, nthreads, stream))) return st;         \
    return ipcu_reset_wall_fin_##S(d_items, d_feq, d_f, nthreads, stream);                              \
  }

DEF(float, f32)
DEF(double, f64)
#undef DEF
