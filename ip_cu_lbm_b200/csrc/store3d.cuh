// Reduced-precision (FP16/BF16) storage of the 3-D solver's populations as
// deviations from a per-cell reference equilibrium.
//
// Each cell stores five reference values in the storage type, (p, u_x/c,
// u_y/c, u_z/c, S): the pressure, velocity and salinity its own collision
// formed in the step that wrote it. Against them a population is stored as
//   f_k:  (f_k - w_k (p + 3 e_k.u)) * scale
//   g_k:  (g_k - w_k S (1 + 4 e_k.u)) * scale
// so only the non-equilibrium part and the cell's change over one step carry
// the 16-bit rounding; the equilibrium part is exact to the reference's own
// rounding, which the deviation absorbs (the decoder forms the same
// reference from the same stored bits). FP16 scales the deviations by 2^12
// and keeps the reference values unscaled; BF16 scales nothing.
//
// Encoding (kernel store, host set_state) and decoding (kernel load, host
// get, the sphere update) use the functions below, whose explicit rounding
// gives the same bits on host and device.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <type_traits>

#include "d3q19.cuh"
#include "storage.cuh"

namespace ipcu {
namespace s3 {

using rstore::add;
using rstore::fma;
using rstore::mul;

template <class T>
__host__ __device__ __forceinline__ float to_f(T v) {
  if constexpr (std::is_same<T, __half>::value) return __half2float(v);
  else return __bfloat162float(v);
}
template <class T>
__host__ __device__ __forceinline__ T from_f(float v) {
  if constexpr (std::is_same<T, __half>::value) return __float2half_rn(v);
  else return __float2bfloat16_rn(v);
}

// decoded reference of one cell
struct Ref {
  float p, ux, uy, uz, S;
};

// e_k . u for direction k of D3Q19 (D3Q7: k < 7), components added in x, y, z order
__host__ __device__ __forceinline__ float eu(int k, const Ref &r) {
  float e = 0.f;
  bool any = false;
  auto term = [&](int c, float u) {
    if (!c) return;
    const float t = c > 0 ? u : -u;
    e = any ? add(e, t) : t;
    any = true;
  };
  term(d3::cx(k), r.ux);
  term(d3::cy(k), r.uy);
  term(d3::cz(k), r.uz);
  return e;
}
// reference equilibria: linear in u
__host__ __device__ __forceinline__ float rf(int k, const Ref &r) { return mul(d3::w19(k), fma(3.0f, eu(k, r), r.p)); }
__host__ __device__ __forceinline__ float rg(int k, const Ref &r) {
  return mul(mul(d3::w7(k), r.S), fma(4.0f, eu(k, r), 1.0f));
}

// stored deviation -> value, and back
template <class T>
__host__ __device__ __forceinline__ float dec(T h, float inv_scale, float ref) {
  return fma(to_f(h), inv_scale, ref);
}
template <class T>
__host__ __device__ __forceinline__ T enc(float v, float scale, float ref) {
  return from_f<T>(mul(add(v, -ref), scale));
}
// the reference planes store the values themselves
template <class T>
__host__ __device__ __forceinline__ Ref ref_of(const T *r, long long i, long long N) {
  return Ref{to_f(r[i]), to_f(r[N + i]), to_f(r[2 * N + i]), to_f(r[3 * N + i]), to_f(r[4 * N + i])};
}

// populations of cell i in FP32: f [19][N] and g [7][N] in the storage
// type T (float: the values; 16-bit: deviations decoded against the
// reference planes r [5][N])
template <class T>
__host__ __device__ __forceinline__ void load_cell(const void *f, const void *g, const void *r, long long i, long long N,
                                                   float inv_scale, float (&fo)[19], float (&go)[7]) {
  if constexpr (std::is_same<T, float>::value) {
    const float *fi = static_cast<const float *>(f), *gi = static_cast<const float *>(g);
#pragma unroll
    for (int k = 0; k < 19; k++) fo[k] = fi[k * N + i];
#pragma unroll
    for (int k = 0; k < 7; k++) go[k] = gi[k * N + i];
  } else {
    const T *fi = static_cast<const T *>(f), *gi = static_cast<const T *>(g);
    const Ref rr = ref_of(static_cast<const T *>(r), i, N);
#pragma unroll
    for (int k = 0; k < 19; k++) fo[k] = dec(fi[k * N + i], inv_scale, rf(k, rr));
#pragma unroll
    for (int k = 0; k < 7; k++) go[k] = dec(gi[k * N + i], inv_scale, rg(k, rr));
  }
}

}  // namespace s3
}  // namespace ipcu
