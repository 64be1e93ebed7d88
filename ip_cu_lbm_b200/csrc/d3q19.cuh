// D3Q19 / D3Q7 lattice facts shared by the 3-D step kernels: the reference's
// D3Q27 velocity order truncated (rest, 6 axes, 12 edges; D3Q7 = its first
// seven directions; ref: function/basic.cu:88-97), weights, opposites,
// mirrors and the five shear rows of the d'Humieres moment basis.
#pragma once

namespace ipcu {
namespace d3 {

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
__host__ __device__ constexpr int find19(int a, int b, int c) {
  for (int k = 0; k < 19; k++)
    if (cx(k) == a && cy(k) == b && cz(k) == c) return k;
  return -1;
}
// the population mirrored across an x wall (mx), a y wall (my) or both
__host__ __device__ constexpr int mir(int k, bool mx, bool my) {
  return find19(mx ? -cx(k) : cx(k), my ? -cy(k) : cy(k), cz(k));
}
__host__ __device__ constexpr float w19(int k) { return k == 0 ? 1.0f / 3.0f : (k <= 6 ? 1.0f / 18.0f : 1.0f / 36.0f); }
__host__ __device__ constexpr float w7(int k) { return k == 0 ? 0.25f : 0.125f; }
// shear rows of the d'Humieres basis
__host__ __device__ constexpr int m1(int k) { return 2 * cx(k) * cx(k) - cy(k) * cy(k) - cz(k) * cz(k); }
__host__ __device__ constexpr int m2(int k) { return cy(k) * cy(k) - cz(k) * cz(k); }
__host__ __device__ constexpr int m3(int k) { return cx(k) * cy(k); }
__host__ __device__ constexpr int m4(int k) { return cy(k) * cz(k); }
__host__ __device__ constexpr int m5(int k) { return cx(k) * cz(k); }

constexpr bool check_tables() {
  for (int k = 0; k < 19; k++) {
    if (cx(opp(k)) != -cx(k) || cy(opp(k)) != -cy(k) || cz(opp(k)) != -cz(k)) return false;
    if (mir(k, true, true) < 0 || mir(mir(k, true, false), true, false) != k) return false;
  }
  return true;
}
static_assert(check_tables(), "D3Q19 opposite / mirror tables");

// Collision of one cell (ref: function/collision.cu:57-188 on the D3Q19 /
// D3Q7 subsets): MRT with the reference's unit non-shear rates, whose
// operator reduces to
//   f*_k = feq_k + Fk_k/2 + (1 - 1/tau) sum_m (M_m.(f - feq)) M_mk / |M_m|^2
// over the five shear rows (the forcing part of the shear moments vanishes
// by parity), or BGK; the regularised D3Q7 scalar collision with cs^2 = 1/4,
//   g*_k = w_k (S + 4 e_k.(S u/c + (1 - 1/tau_s) j)).
// uc, vc, wc: velocity over c; h3 = F fden / 2 (the half forcing term);
// itau = 1/tau; omg_s = 1 - 1/tau_s.
__device__ __forceinline__ void collide19(const float (&f)[19], const float (&g)[7], float pr, float S, float uc,
                                          float vc, float wc, float hx, float hy, float hz, float itau, float omg_s,
                                          bool mrt, float (&fo)[19], float (&go)[7]) {
  // (sums of two products as explicit fmas: every kernel that inlines this
  // rounds alike, whatever the compiler contracts around it)
  const float usq = fmaf(uc, uc, fmaf(vc, vc, wc * wc));
  const float P0 = fmaf(-1.5f, usq, pr);
  if (mrt) {
    float a1 = 0.f, a2 = 0.f, a3 = 0.f, a4 = 0.f, a5 = 0.f;
#pragma unroll
    for (int k = 0; k < 19; k++) {
      if (m1(k)) a1 += m1(k) * f[k];
      if (m2(k)) a2 += m2(k) * f[k];
      if (m3(k)) a3 += m3(k) * f[k];
      if (m4(k)) a4 += m4(k) * f[k];
      if (m5(k)) a5 += m5(k) * f[k];
    }
    const float om = 1.0f - itau;
    a1 = om * (a1 - fmaf(2.0f * uc, uc, -fmaf(vc, vc, wc * wc))) * (1.0f / 36.0f);
    a2 = om * (a2 - fmaf(vc, vc, -(wc * wc))) * (1.0f / 12.0f);
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
#pragma unroll
    for (int k = 0; k < 19; k++) {
      const float eu = (cx(k) ? cx(k) * uc : 0.f) + (cy(k) ? cy(k) * vc : 0.f) + (cz(k) ? cz(k) * wc : 0.f);
      const float eh = (cx(k) ? cx(k) * hx : 0.f) + (cy(k) ? cy(k) * hy : 0.f) + (cz(k) ? cz(k) * hz : 0.f);
      const float feq = w19(k) * (fmaf(4.5f * eu, eu, P0) + 3.0f * eu);
      const float fk2 = w19(k) * eh;  // Fk / 2
      fo[k] = f[k] - (f[k] - feq + fk2) * itau + 2.0f * fk2;
    }
  }
  const float jgx = (g[1] - g[3]) - S * uc, jgy = (g[2] - g[4]) - S * vc, jgz = (g[5] - g[6]) - S * wc;
  const float bx = 4.0f * fmaf(omg_s, jgx, S * uc), by = 4.0f * fmaf(omg_s, jgy, S * vc),
              bz = 4.0f * fmaf(omg_s, jgz, S * wc);
  go[0] = w7(0) * S;
  go[1] = w7(1) * (S + bx);
  go[3] = w7(3) * (S - bx);
  go[2] = w7(2) * (S + by);
  go[4] = w7(4) * (S - by);
  go[5] = w7(5) * (S + bz);
  go[6] = w7(6) * (S - bz);
}

}  // namespace d3
}  // namespace ipcu
