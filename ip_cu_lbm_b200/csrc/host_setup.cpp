// Host-side set-up helpers of the reference kernel library, re-expressed
// behind the C ABI (plain pointers and sizes instead of std::vector
// growth): lattice constants (Items::setc), MRT matrices (read_M / set_M),
// ghost cells (set_neibghor_wall), wall lists (set_walln) and the slip
// tables (set_bound2D / set_bound3D), plus a structured box-grid builder
// that reproduces the case drivers' cell numbering.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "ipcu.h"

namespace {

const int kKinv9[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
const int kKinv27[27] = {0, 3, 4, 1, 2, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15, 26, 25, 24, 23, 22, 21, 20, 19};
inline const int *kinv_of(int Q) { return Q == 27 ? kKinv27 : kKinv9; }

// Unit lattice vectors: D2Q9 in the x-z plane and D3Q27 (ref: function/basic.cu:78-97)
void unit_vectors(int Q, int *ex, int *ey, int *ez, double *w) {
  for (int k = 0; k < 27; k++) ex[k] = ey[k] = ez[k] = 0, w[k] = 0;
  if (Q == 9) {
    const int x[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1}, z[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    for (int k = 0; k < 9; k++) {
      ex[k] = x[k];
      ez[k] = z[k];
      w[k] = k == 0 ? 4.0 / 9.0 : (k < 5 ? 1.0 / 9.0 : 1.0 / 36.0);
    }
  } else {
    const int v[27][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {-1, 0, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1},
                          {1, 1, 0}, {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, 0, 1}, {1, 0, -1}, {-1, 0, 1},
                          {-1, 0, -1}, {0, 1, 1}, {0, 1, -1}, {0, -1, 1}, {0, -1, -1}, {1, 1, 1}, {1, 1, -1},
                          {1, -1, 1}, {1, -1, -1}, {-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
    for (int k = 0; k < 27; k++) {
      ex[k] = v[k][0];
      ey[k] = v[k][1];
      ez[k] = v[k][2];
      int n = std::abs(v[k][0]) + std::abs(v[k][1]) + std::abs(v[k][2]);
      w[k] = n == 0 ? 8.0 / 27.0 : (n == 1 ? 2.0 / 27.0 : (n == 2 ? 1.0 / 54.0 : 1.0 / 216.0));
    }
  }
}

template <class T>
struct ItemView {
  const T *it;
  int Q;
  long long nc, nw;
  T c;
  explicit ItemView(const T *items)
      : it(items), Q((int)items[6]), nc((long long)items[10]), nw((long long)items[11]), c(items[2]) {}
  int ex(int k) const { return (int)(it[25 + Q + k] / c); }
  int ey(int k) const { return (int)(it[25 + 2 * Q + k] / c); }
  int ez(int k) const { return (int)(it[25 + 3 * Q + k] / c); }
};

// set_walln (ref: function/set_bound.cu:23-38)
template <class T>
int walln(const T *items, const int *neib, int64_t cap, int *const *wall_out, int *sizes) {
  ItemView<T> v(items);
  int d[6];
  if (v.Q == 9) {
    const int a[6] = {1, 0, 3, 0, 2, 4};
    std::memcpy(d, a, sizeof a);
  } else if (v.Q == 27) {
    const int a[6] = {1, 2, 3, 4, 5, 6};
    std::memcpy(d, a, sizeof a);
  } else {
    return IPCU_ERR_ARG;
  }
  for (int a = 0; a < 6; a++) sizes[a] = 0;
  for (long long i = 0; i < v.nc; i++)
    for (int a = 0; a < 6; a++)
      if (neib[i * v.Q + d[a]] >= (int)v.nc) {
        if (sizes[a] >= cap) return IPCU_ERR_CAPACITY;
        if (wall_out && wall_out[a]) wall_out[a][sizes[a]] = (int)i;
        sizes[a]++;
      }
  return IPCU_OK;
}

// set_bound2D (ref: function/set_bound.cu:40-73): for each ghost and
// direction, the neighbour of the owner (nextB) and the population (nextK)
// a specular (slip) wall reflects into the ghost.
template <class T>
int bound2d(const T *items, int nb, const int *neib, int *nextK, int *nextB) {
  ItemView<T> v(items);
  if (v.Q != 9) return IPCU_ERR_ARG;
  int nei[2][2][9] = {}, kv[2][2][9] = {};
  for (int k = 0; k < 9; k++) {
    kv[std::abs(v.ex(k))][std::abs(v.ez(k))][k] = kKinv9[k];
    kv[0][0][k] = kKinv9[k];
  }
  // reflections off a z wall (index [1][0]) and an x wall ([0][1])
  nei[1][0][5] = 3; nei[0][1][5] = 4; nei[1][0][6] = 1; nei[0][1][6] = 4;
  nei[1][0][7] = 1; nei[0][1][7] = 2; nei[1][0][8] = 3; nei[0][1][8] = 2;
  kv[1][0][5] = 8; kv[0][1][5] = 6; kv[1][0][6] = 7; kv[0][1][6] = 5;
  kv[1][0][7] = 6; kv[0][1][7] = 8; kv[1][0][8] = 5; kv[0][1][8] = 7;
  for (long long g = 0; g < v.nw; g++) {
    const long long o = (long long)neib[(nb + g) * 9] * 9;
    nextB[g * 9] = 0;
    nextK[g * 9] = 0;
    for (int k = 1; k < 9; k++) {
      int cx = v.ex(k), cz = v.ez(k);
      if (neib[o + kKinv9[k]] >= nb) {
        if ((neib[o + 1] >= nb && cx == -1) || (neib[o + 3] >= nb && cx == 1)) cx = 0;
        if ((neib[o + 2] >= nb && cz == -1) || (neib[o + 4] >= nb && cz == 1)) cz = 0;
      }
      nextB[g * 9 + k] = nei[std::abs(cx)][std::abs(cz)][k];
      nextK[g * 9 + k] = kv[std::abs(cx)][std::abs(cz)][k];
    }
  }
  return IPCU_OK;
}

// set_bound3D (ref: function/set_bound.cu:75-162)
template <class T>
int bound3d(const T *items, int nb, const int *neib, int *nextK, int *nextB) {
  ItemView<T> v(items);
  if (v.Q != 27) return IPCU_ERR_ARG;
  static int nei[2][2][2][27], kv[2][2][2][27];
  std::memset(nei, 0, sizeof nei);
  std::memset(kv, 0, sizeof kv);
  for (int k = 0; k < 27; k++) {
    kv[std::abs(v.ex(k))][std::abs(v.ey(k))][std::abs(v.ez(k))][k] = kKinv27[k];
    kv[0][0][0][k] = kKinv27[k];
  }
  // Per direction k: which owner neighbour (nextB) and which population
  // (nextK) a reflection across the x ([1][0][0]), y ([0][1][0]), z
  // ([0][0][1]) walls, or across an edge ([1][1][0], [1][0][1], [0][1][1]),
  // draws from.
  struct R { int k, a, b, c, n, q; };
  static const R rules[] = {
      {7, 1, 0, 0, 3, 8}, {7, 0, 1, 0, 4, 9}, {8, 1, 0, 0, 3, 7}, {8, 0, 1, 0, 2, 10},
      {9, 1, 0, 0, 1, 10}, {9, 0, 1, 0, 4, 7}, {10, 1, 0, 0, 1, 9}, {10, 0, 1, 0, 2, 8},
      {11, 1, 0, 0, 3, 12}, {11, 0, 0, 1, 6, 13}, {12, 1, 0, 0, 3, 11}, {12, 0, 0, 1, 5, 14},
      {13, 1, 0, 0, 1, 14}, {13, 0, 0, 1, 6, 11}, {14, 1, 0, 0, 1, 13}, {14, 0, 0, 1, 5, 12},
      {15, 0, 1, 0, 4, 16}, {15, 0, 0, 1, 6, 17}, {16, 0, 1, 0, 4, 15}, {16, 0, 0, 1, 5, 18},
      {17, 0, 1, 0, 2, 18}, {17, 0, 0, 1, 6, 15}, {18, 0, 1, 0, 2, 17}, {18, 0, 0, 1, 5, 16},
      {19, 1, 0, 0, 3, 22}, {19, 0, 1, 0, 4, 24}, {19, 0, 0, 1, 6, 25}, {19, 1, 1, 0, 10, 20}, {19, 1, 0, 1, 14, 21}, {19, 0, 1, 1, 18, 23},
      {20, 1, 0, 0, 3, 21}, {20, 0, 1, 0, 4, 23}, {20, 0, 0, 1, 5, 26}, {20, 1, 1, 0, 10, 19}, {20, 1, 0, 1, 13, 22}, {20, 0, 1, 1, 17, 24},
      {21, 1, 0, 0, 3, 20}, {21, 0, 1, 0, 2, 26}, {21, 0, 0, 1, 6, 23}, {21, 1, 1, 0, 9, 22}, {21, 1, 0, 1, 14, 19}, {21, 0, 1, 1, 16, 25},
      {22, 1, 0, 0, 3, 19}, {22, 0, 1, 0, 2, 25}, {22, 0, 0, 1, 5, 24}, {22, 1, 1, 0, 9, 21}, {22, 1, 0, 1, 13, 20}, {22, 0, 1, 1, 15, 26},
      {23, 1, 0, 0, 1, 26}, {23, 0, 1, 0, 4, 20}, {23, 0, 0, 1, 6, 21}, {23, 1, 1, 0, 8, 24}, {23, 1, 0, 1, 12, 25}, {23, 0, 1, 1, 18, 19},
      {24, 1, 0, 0, 1, 25}, {24, 0, 1, 0, 4, 19}, {24, 0, 0, 1, 5, 22}, {24, 1, 1, 0, 8, 23}, {24, 1, 0, 1, 11, 26}, {24, 0, 1, 1, 17, 20},
      {25, 1, 0, 0, 1, 24}, {25, 0, 1, 0, 2, 22}, {25, 0, 0, 1, 6, 19}, {25, 1, 1, 0, 7, 26}, {25, 1, 0, 1, 12, 23}, {25, 0, 1, 1, 16, 21},
      {26, 1, 0, 0, 1, 23}, {26, 0, 1, 0, 2, 21}, {26, 0, 0, 1, 5, 20}, {26, 1, 1, 0, 7, 25}, {26, 1, 0, 1, 11, 24}, {26, 0, 1, 1, 15, 22},
  };
  for (const R &r : rules) {
    nei[r.a][r.b][r.c][r.k] = r.n;
    kv[r.a][r.b][r.c][r.k] = r.q;
  }
  for (long long g = 0; g < v.nw; g++) {
    const long long o = (long long)neib[(nb + g) * 27] * 27;
    nextB[g * 27] = 0;
    nextK[g * 27] = 0;
    for (int k = 1; k < 27; k++) {
      const int ex = v.ex(k), ey = v.ey(k), ez = v.ez(k);
      int cx = ex, cy = ey, cz = ez;
      auto W = [&](int d) { return neib[o + d] >= nb; };
      if (W(kKinv27[k])) {
        if ((W(1) && cx == -1) || (W(3) && cx == 1)) cx = 0;
        if ((W(2) && cy == -1) || (W(4) && cy == 1)) cy = 0;
        if ((W(5) && cz == -1) || (W(6) && cz == 1)) cz = 0;
        // an open edge neighbour restores the component pair
        if ((!W(11) && ex == -1 && ez == -1) || (!W(14) && ex == 1 && ez == 1)) { cx = ex; cz = ez; }
        if ((!W(12) && ex == -1 && ez == 1) || (!W(13) && ex == 1 && ez == -1)) { cx = ex; cz = ez; }
        if ((!W(15) && ey == -1 && ez == -1) || (!W(18) && ey == 1 && ez == 1)) { cy = ey; cz = ez; }
        if ((!W(16) && ey == -1 && ez == 1) || (!W(17) && ey == 1 && ez == -1)) { cy = ey; cz = ez; }
        // a walled edge neighbour removes it
        if ((W(11) && cx == -1 && cz == -1) || (W(14) && cx == 1 && cz == 1)) { cx = 0; cz = 0; }
        if ((W(12) && cx == -1 && cz == 1) || (W(13) && cx == 1 && cz == -1)) { cx = 0; cz = 0; }
        if ((W(15) && cy == -1 && cz == -1) || (W(18) && cy == 1 && cz == 1)) { cy = 0; cz = 0; }
        if ((W(16) && cy == -1 && cz == 1) || (W(17) && cy == 1 && cz == -1)) { cy = 0; cz = 0; }
      }
      nextB[g * 27 + k] = nei[std::abs(cx)][std::abs(cy)][std::abs(cz)][k];
      nextK[g * 27 + k] = kv[std::abs(cx)][std::abs(cy)][std::abs(cz)][k];
    }
  }
  return IPCU_OK;
}

bool read_matrix(const std::string &fn, int rows, int cols, double *out) {
  std::ifstream in(fn);
  if (!in) return false;
  std::string line;
  for (int i = 0; i < rows; i++) {
    if (!std::getline(in, line)) return false;
    std::stringstream ss(line);
    std::string cell;
    for (int j = 0; j < cols; j++) {
      if (!std::getline(ss, cell, ',')) return false;
      out[i * cols + j] = std::stod(cell);
    }
  }
  return true;
}

}  // namespace

// ---------------------------------------------------------------- lattice constants
extern "C" int ipcu_setc(int Q, double dx, double dt, int alpha, double *c, double *tau, double *taus, double *cx,
                         double *cy, double *cz, double *w) {
  if (Q != 9 && Q != 27) return IPCU_ERR_ARG;
  if (!c || !tau || !taus || !cx || !cy || !cz || !w || dt == 0) return IPCU_ERR_ARG;
  int ex[27], ey[27], ez[27];
  double ww[27];
  unit_vectors(Q, ex, ey, ez, ww);
  // c = dx/dt; tau from a water viscosity of 1e-6; taus from 1.4e-alpha (ref: function/basic.cu:70-77)
  *c = dx / dt;
  *tau = 1.0 * 3.0 * std::pow(10.0, -6) / (*c) / (*c) / dt + 0.5;
  *taus = 1.4 * 3.0 * std::pow(10.0, -alpha) / (*c) / (*c) / dt + 0.5;
  for (int k = 0; k < 27; k++) {
    cx[k] = ex[k] * (*c);
    cy[k] = ey[k] * (*c);
    cz[k] = ez[k] * (*c);
    w[k] = ww[k];
  }
  return IPCU_OK;
}

// ---------------------------------------------------------------- MRT matrices
// read_M (ref: function/basic.cu:157-170): input/{MRT,S,Minv}_D3Q<Q>.csv under `dir`.
extern "C" int ipcu_read_M_csv(const char *dir, int Q, double *M, double *S, double *Minv) {
  if (!dir || !M || !S || !Minv || (Q != 9 && Q != 27)) return IPCU_ERR_ARG;
  std::string d(dir);
  char b[64];
  std::snprintf(b, sizeof b, "/input/MRT_D3Q%d.csv", Q);
  if (!read_matrix(d + b, Q, Q, M)) return IPCU_ERR_IO;
  std::snprintf(b, sizeof b, "/input/Minv_D3Q%d.csv", Q);
  if (!read_matrix(d + b, Q, Q, Minv)) return IPCU_ERR_IO;
  std::snprintf(b, sizeof b, "/input/S_D3Q%d.csv", Q);
  if (!read_matrix(d + b, 1, Q, S)) return IPCU_ERR_IO;
  return IPCU_OK;
}

// set_M (ref: function/basic.cu:171-201): the shear rows' rates are zeroed
// in S (Q9: 7,8; Q27: 5..9) and MM = Minv diag(S) M is formed; M, Minv are
// returned as read.
extern "C" int ipcu_set_M(int Q, const double *M_in, const double *S_in, const double *Minv_in, double *M,
                          double *S, double *Minv, double *MM) {
  if (!M_in || !S_in || !Minv_in || !M || !S || !Minv || !MM || (Q != 9 && Q != 27)) return IPCU_ERR_ARG;
  std::vector<double> s(S_in, S_in + Q), sm((size_t)Q * Q);
  if (Q == 9) s[7] = s[8] = 0;
  else
    for (int i = 5; i < 10; i++) s[i] = 0;
  for (int i = 0; i < Q; i++)
    for (int j = 0; j < Q; j++) sm[i * Q + j] = s[i] * M_in[i * Q + j];
  for (int i = 0; i < Q; i++)
    for (int j = 0; j < Q; j++) {
      double a = 0;
      for (int k = 0; k < Q; k++) a += Minv_in[i * Q + k] * sm[k * Q + j];
      MM[i * Q + j] = a;
    }
  std::memcpy(M, M_in, sizeof(double) * Q * Q);
  std::memcpy(Minv, Minv_in, sizeof(double) * Q * Q);
  std::memcpy(S, s.data(), sizeof(double) * Q);
  return IPCU_OK;
}

// ---------------------------------------------------------------- ghost cells
// set_neibghor_wall (ref: function/basic.cu:203-237). `neib` holds room
// for `cap` cells; its first num_calc*Q entries are the fluid table with -1
// for missing neighbours. One ghost is appended per fluid cell that has a
// missing neighbour, scanning the nx*ny*nz numbering `lnum` (-1 = solid) in
// order; the ghost's own entries point to itself except towards its owner,
// and the owner's missing entries point to the ghost. owner_out[g] receives
// the owner of ghost g. Returns the ghost count, or a negative status.
extern "C" int64_t ipcu_set_neibghor_wall(int Q, int nx, int ny, int nz, int64_t num_calc, const int *lnum,
                                          int *neib, int64_t cap, int *owner_out) {
  if ((Q != 9 && Q != 27) || !lnum || !neib || nx <= 0 || ny <= 0 || nz <= 0) return IPCU_ERR_ARG;
  const int *ki = kinv_of(Q);
  int64_t ng = 0;
  const int64_t ncell = (int64_t)nx * ny * nz;
  for (int64_t idx = 0; idx < ncell; idx++) {
    const int64_t c = lnum[idx];
    if (c < 0) continue;
    bool open = false;
    for (int k = 1; k < Q; k++)
      if (neib[c * Q + k] == -1) {
        open = true;
        break;
      }
    if (!open) continue;
    const int64_t g = num_calc + ng;
    if (g >= cap) return IPCU_ERR_CAPACITY;
    for (int k = 0; k < Q; k++) neib[g * Q + k] = (int)g;
    neib[g * Q] = (int)c;
    for (int k = 1; k < Q; k++)
      if (neib[c * Q + k] == -1) {
        neib[c * Q + k] = (int)g;
        neib[g * Q + ki[k]] = (int)c;
      }
    if (owner_out) owner_out[ng] = (int)c;
    ng++;
  }
  return ng;
}

#define WALL_DEFS(T, S)                                                                               \
  extern "C" int ipcu_set_walln_##S(const T *items, const int *neib, int64_t cap, int *const *wall_out, \
                                    int *sizes) {                                                    \
    if (!items || !neib || !sizes) return IPCU_ERR_ARG;                                               \
    return walln<T>(items, neib, cap, wall_out, sizes);                                               \
  }                                                                                                   \
  extern "C" int ipcu_set_bound2D_##S(const T *items, int num_block, const int *neib, int *nextK,      \
                                      int *nextB) {                                                  \
    if (!items || !neib || !nextK || !nextB) return IPCU_ERR_ARG;                                     \
    return bound2d<T>(items, num_block, neib, nextK, nextB);                                          \
  }                                                                                                   \
  extern "C" int ipcu_set_bound3D_##S(const T *items, int num_block, const int *neib, int *nextK,      \
                                      int *nextB) {                                                  \
    if (!items || !neib || !nextK || !nextB) return IPCU_ERR_ARG;                                     \
    return bound3d<T>(items, num_block, neib, nextK, nextB);                                          \
  }
WALL_DEFS(float, f32)
WALL_DEFS(double, f64)
#undef WALL_DEFS

// ---------------------------------------------------------------- box grid builder
// Fluid numbering and neighbour table of a rectangular box with per-column
// x refinement divx[nx0] and y refinement divy[ny0] and nz uniform layers,
// as the case drivers build it (ref: LockExchange/LockExchange.cu:34-127):
// cells are numbered x-major, then y, then z (z fastest); posx/posy/posz
// are cell centres and delX/delY the refined widths. Outputs are sized for
// the refined grid (NX = sum divx, NY = sum divy): lnum[NX*NY*nz],
// neib[num_calc*Q] (-1 where the neighbour lies outside the box) and the
// per-cell geometry arrays (num_calc each). Returns num_calc.
extern "C" int64_t ipcu_build_box_grid(int Q, int nx0, int ny0, int nz, double dx, double ratiox, double ratioy,
                                       const int *divx, const int *divy, int *lnum, int *neib, double *posx,
                                       double *posy, double *posz, double *delX, double *delY) {
  if ((Q != 9 && Q != 27) || nx0 <= 0 || ny0 <= 0 || nz <= 0 || !divx || !divy) return IPCU_ERR_ARG;
  int ex[27], ey[27], ez[27];
  double w[27];
  unit_vectors(Q, ex, ey, ez, w);
  int64_t NX = 0, NY = 0;
  for (int i = 0; i < nx0; i++) NX += divx[i];
  for (int j = 0; j < ny0; j++) NY += divy[j];
  int64_t n = 0;
  for (int i = 0; i < nx0; i++)
    for (int di = 0; di < divx[i]; di++)
      for (int j = 0; j < ny0; j++)
        for (int dj = 0; dj < divy[j]; dj++)
          for (int l = 0; l < nz; l++) {
            if (lnum) lnum[n] = (int)n;
            if (posx) {
              posx[n] = (i + (2.0 * di + 1.0) / (2.0 * divx[i])) * dx * ratiox;
              posy[n] = (j + (2.0 * dj + 1.0) / (2.0 * divy[j])) * dx * ratioy;
              posz[n] = (l + 0.5) * dx;
              delX[n] = dx * ratiox / divx[i];
              delY[n] = dx * ratioy / divy[j];
            }
            n++;
          }
  if (neib) {
    for (int64_t I = 0; I < NX; I++)
      for (int64_t J = 0; J < NY; J++)
        for (int64_t L = 0; L < nz; L++) {
          const int64_t c = (I * NY + J) * nz + L;
          for (int k = 0; k < Q; k++) {
            int64_t a = I + ex[k], b = J + ey[k], d = L + ez[k];
            neib[c * Q + k] = (a >= 0 && a < NX && b >= 0 && b < NY && d >= 0 && d < nz) ? (int)((a * NY + b) * nz + d) : -1;
          }
        }
  }
  return n;
}
