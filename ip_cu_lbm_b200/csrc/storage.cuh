// Reduced-precision (FP16/BF16) storage of the structured solver's
// distributions as deviations from the local equilibrium.
//
// A stored population is r_k = f_k - feq_k(p*, u) with p*, u the cell's own
// FP32 moments, which are kept beside it (macroscopic planes S, u_x, u_z, p*);
// the scalar lattice likewise stores g_k - geq_k(S, u). Only the
// non-equilibrium part then carries the 16-bit rounding, so the velocity and
// salinity the kernel forms from the populations keep FP32 accuracy in their
// equilibrium part. Store (kernel phase 2, host set_state) and load (kernel
// phase 1, host get) evaluate the equilibria with the functions below, whose
// explicit rounding makes the two sides agree bit for bit on host and device.
#pragma once
#include <cmath>

namespace ipcu {
namespace rstore {

__host__ __device__ __forceinline__ float mul(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
__host__ __device__ __forceinline__ float add(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
__host__ __device__ __forceinline__ float fma(float a, float b, float c) {
#ifdef __CUDA_ARCH__
  return __fmaf_rn(a, b, c);
#else
  return std::fmaf(a, b, c);
#endif
}

// e_k . u / c for the reference's D2Q9 (x-z plane) order; D2Q5 is k < 5
__host__ __device__ __forceinline__ float eu(int k, float uc, float wc) {
  switch (k) {
    case 1: return uc;
    case 2: return wc;
    case 3: return -uc;
    case 4: return -wc;
    case 5: return add(uc, wc);
    case 6: return add(wc, -uc);
    case 7: return -add(uc, wc);
    case 8: return -add(wc, -uc);
  }
  return 0.f;
}
__host__ __device__ __forceinline__ float w9(int k) { return k == 0 ? 4.0f / 9.0f : (k <= 4 ? 1.0f / 9.0f : 1.0f / 36.0f); }
__host__ __device__ __forceinline__ float w5(int k) { return k == 0 ? 1.0f / 3.0f : 1.0f / 6.0f; }

__host__ __device__ __forceinline__ float usq(float uc, float wc) { return fma(uc, uc, mul(wc, wc)); }

// pressure-form D2Q9 equilibrium w_k (p* + 3 e.u + 4.5 (e.u)^2 - 1.5 u^2) (u in units of c)
__host__ __device__ __forceinline__ float feq(int k, float pr, float uc, float wc, float u2) {
  const float e = eu(k, uc, wc);
  const float t = fma(mul(4.5f, e), e, fma(3.0f, e, fma(-1.5f, u2, pr)));
  return mul(w9(k), t);
}
// scalar equilibria: D2Q5 linear w S (1 + 3 e.u); Q9 second order
__host__ __device__ __forceinline__ float geq5(int k, float S, float uc, float wc) {
  return mul(mul(w5(k), S), fma(3.0f, eu(k, uc, wc), 1.0f));
}
__host__ __device__ __forceinline__ float geq9(int k, float S, float uc, float wc, float u2) {
  const float e = eu(k, uc, wc);
  const float t = fma(mul(4.5f, e), e, fma(3.0f, e, fma(-1.5f, u2, 1.0f)));
  return mul(mul(w9(k), S), t);
}

}  // namespace rstore
}  // namespace ipcu
