// Host-side tables of a stretched axis, shared by the 2-D and 3-D solvers:
// the flux-form weights of the reference's interpolated streaming and the
// density-gradient factors.
#pragma once
#include <algorithm>
#include <vector>

namespace ipcu {

// Stencil weights of the conservative flux form along one axis, for every
// cell and both travel directions. Nodes beyond a wall take the wall cell's
// coordinate and are then pushed one lattice spacing past the previous node
// (ref: function/adv.cu:16-21 set_posl_x; 41-48 Lagrange_interpolation;
// 76-86 evaluation point and flux scales).
inline void axis_tables(const std::vector<double> &X, const std::vector<double> &D, double dz, int ns, std::vector<float> &w,
                 std::vector<float> &scin, std::vector<float> &scout, std::vector<float> &wc) {
  const int n = (int)X.size();
  std::vector<double> wd((size_t)2 * n * ns, 0.0), sid((size_t)2 * n, 0.0), sod(n, 0.0);
  auto cl = [&](int i) { return std::min(std::max(i, 0), n - 1); };
  for (int j = 0; j < n; j++) {
    sod[j] = dz / D[j];
    for (int s = 0; s < 2; s++) {
      const int sg = s == 0 ? 1 : -1;
      const double xa = X[j] + sg * (D[j] - dz) / 2.0;
      double pl[5];
      const int h = ns / 2;
      for (int m = 0; m < ns; m++) pl[m] = X[cl(j + sg * (m - h))];
      // walk outwards from the centre node, each node at least dz beyond its inner neighbour
      for (int m = h - 1; m >= 0; m--) pl[m] = sg > 0 ? std::min(pl[m], pl[m + 1] - dz) : std::max(pl[m], pl[m + 1] + dz);
      for (int m = h + 1; m < ns; m++) pl[m] = sg > 0 ? std::max(pl[m], pl[m - 1] + dz) : std::min(pl[m], pl[m - 1] - dz);
      for (int a = 0; a < ns; a++) {
        double v = 1.0;
        for (int b = 0; b < ns; b++)
          if (b != a) v *= (xa - pl[b]) / (pl[a] - pl[b]);
        wd[((size_t)s * n + j) * ns + a] = v;
      }
      sid[(size_t)s * n + j] = dz / D[cl(j + sg)];
    }
  }
  w.resize(wd.size());
  scin.resize(sid.size());
  scout.resize(sod.size());
  for (size_t i = 0; i < wd.size(); i++) w[i] = (float)wd[i];
  for (size_t i = 0; i < sid.size(); i++) scin[i] = (float)sid[i];
  for (size_t i = 0; i < sod.size(); i++) scout[i] = (float)sod[i];
  // Interior cells (stencils clear of the walls) take the flux form as one
  // dot product over the NS+1 nodes c'+sg*(q-h-1), q = 0..NS, around the
  // source cell c' (axis index j): the centre value, plus fin of the
  // upstream cell j-sg, minus fout of c'. wc layout [2][NS+1][n].
  const int nq = ns + 1, h = ns / 2;
  wc.assign((size_t)2 * nq * n, 0.f);
  for (int j = 0; j < n; j++)
    for (int s = 0; s < 2; s++) {
      const int sg = s == 0 ? 1 : -1, ju = cl(j - sg);
      for (int q = 0; q < nq; q++) {
        double v = (q == h + 1) ? 1.0 : 0.0;
        if (q < ns) v += sid[(size_t)s * n + ju] * wd[((size_t)s * n + ju) * ns + q];
        if (q >= 1) v -= sod[j] * wd[((size_t)s * n + j) * ns + q - 1];
        wc[((size_t)s * nq + q) * n + j] = (float)v;
      }
    }
}


// 1/(x_{i+1} - x_{i-1} + dz/1000) in float, clamped neighbours
// (ref: function/collision.cu:82-85; ghosts carry their owner's position)
inline std::vector<float> grad_inv(const std::vector<double> &X, double dz) {
  const int n = (int)X.size();
  std::vector<float> r(n);
  const float reg = (float)dz / 1000.0f;
  for (int i = 0; i < n; i++) {
    float a = (float)X[std::min(i + 1, n - 1)], b = (float)X[std::max(i - 1, 0)];
    r[i] = 1.0f / (a - b + reg);
  }
  return r;
}

}  // namespace ipcu
