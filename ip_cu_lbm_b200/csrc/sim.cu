// Structured-grid solver object (ipcu_sim_*): device-resident state,
// host-precomputed axis tables, stepping (direct or CUDA-graph replay),
// field I/O and FP64 conservation totals.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <tuple>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fused2d.cuh"
#include "ipcu_common.cuh"

using namespace ipcu;

struct ipcu_sim {
  ipcu_sim_config cfg;
  int nx, nz;
  long long N;
  cudaStream_t stream;
  size_t esz;  // bytes per stored distribution value
  void *f[2] = {nullptr, nullptr};
  void *g[2] = {nullptr, nullptr};
  float *mac[2] = {nullptr, nullptr};
  float *wA = nullptr, *scin = nullptr, *scout = nullptr, *wC = nullptr, *ginvx = nullptr, *ginvz = nullptr;
  unsigned *status = nullptr;
  double *partials = nullptr;
  int cur = 0;
  f2d::Params P;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // per starting parity
  int graph_chunk = 0;
  std::vector<double> X, Z, DX, DZ;
  std::vector<double> M, Minv, Srates;  // MRT matrices as given (for snapshots)
  long long steps = 0;                  // time steps taken since creation / restore
};

namespace {

constexpr int ex9[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
constexpr int ez9[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
constexpr int kinv9[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
constexpr double w9d[9] = {4.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 36, 1.0 / 36, 1.0 / 36, 1.0 / 36};
constexpr double w5d[5] = {1.0 / 3, 1.0 / 6, 1.0 / 6, 1.0 / 6, 1.0 / 6};

inline int geo_axis(int geo) {
  return (geo == IPCU_GEO_X5 || geo == IPCU_GEO_X3) ? 0 : ((geo == IPCU_GEO_Z5 || geo == IPCU_GEO_Z3) ? 1 : -1);
}
inline int geo_ns(int geo) {
  return (geo == IPCU_GEO_X5 || geo == IPCU_GEO_Z5) ? 5 : ((geo == IPCU_GEO_X3 || geo == IPCU_GEO_Z3) ? 3 : 1);
}

// Stencil weights of the conservative flux form along one axis, for every
// cell and both travel directions. Nodes beyond a wall take the wall cell's
// coordinate and are then pushed one lattice spacing past the previous node
// (ref: function/adv.cu:16-21 set_posl_x; 41-48 Lagrange_interpolation;
// 76-86 evaluation point and flux scales).
void axis_tables(const std::vector<double> &X, const std::vector<double> &D, double dz, int ns, std::vector<float> &w,
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
std::vector<float> grad_inv(const std::vector<double> &X, double dz) {
  const int n = (int)X.size();
  std::vector<float> r(n);
  const float reg = (float)dz / 1000.0f;
  for (int i = 0; i < n; i++) {
    float a = (float)X[std::min(i + 1, n - 1)], b = (float)X[std::max(i - 1, 0)];
    r[i] = 1.0f / (a - b + reg);
  }
  return r;
}

// Specular-slip partner tables per wall class (bit 0 left x wall, 1 right,
// 2 bottom z wall, 3 top), following set_bound2D (ref: function/set_bound.cu:40-73).
void slip_tables(int q, int8_t *B, int8_t *K) {
  int nei[2][2][9] = {}, kv[2][2][9] = {};
  for (int k = 0; k < q; k++) {
    kv[std::abs(ex9[k])][std::abs(ez9[k])][k] = kinv9[k];
    kv[0][0][k] = kinv9[k];
  }
  if (q == 9) {
    nei[1][0][5] = 3; nei[0][1][5] = 4; nei[1][0][6] = 1; nei[0][1][6] = 4;
    nei[1][0][7] = 1; nei[0][1][7] = 2; nei[1][0][8] = 3; nei[0][1][8] = 2;
    kv[1][0][5] = 8; kv[0][1][5] = 6; kv[1][0][6] = 7; kv[0][1][6] = 5;
    kv[1][0][7] = 6; kv[0][1][7] = 8; kv[1][0][8] = 5; kv[0][1][8] = 7;
  }
  for (int cls = 0; cls < 16; cls++) {
    const bool L = cls & 1, R = cls & 2, Bo = cls & 4, T = cls & 8;
    for (int k = 0; k < 9; k++) {
      int b = 0, kk = 0;
      if (k > 0 && k < q) {
        int cx = ex9[k], cz = ez9[k];
        const bool out = (cx == 1 && L) || (cx == -1 && R) || (cz == 1 && Bo) || (cz == -1 && T);
        if (out) {
          if ((R && cx == -1) || (L && cx == 1)) cx = 0;
          if ((T && cz == -1) || (Bo && cz == 1)) cz = 0;
        }
        b = nei[std::abs(cx)][std::abs(cz)][k];
        kk = kv[std::abs(cx)][std::abs(cz)][k];
      }
      B[cls * 9 + k] = (int8_t)b;
      K[cls * 9 + k] = (int8_t)kk;
    }
  }
}

template <class ST>
void to_store(const double *src, void *dst_host, long long n, double scale, double shift_w, const double *wk, int q,
              long long N) {
  ST *d = (ST *)dst_host;
  for (long long i = 0; i < n; i++) {
    double v = src[i];
    if (wk) v -= wk[i / N] * shift_w;
    if constexpr (sizeof(ST) == 4) d[i] = (float)v;
    else if constexpr (std::is_same<ST, __half>::value) d[i] = __float2half_rn((float)(v * scale));
    else d[i] = __float2bfloat16_rn((float)(v * scale));
  }
  (void)q;
}
template <class ST>
void from_store(const void *src_host, double *dst, long long n, double inv_scale, double shift_w, const double *wk,
                long long N) {
  const ST *s = (const ST *)src_host;
  for (long long i = 0; i < n; i++) {
    double v;
    if constexpr (sizeof(ST) == 4) v = (double)((const float *)s)[i];
    else if constexpr (std::is_same<ST, __half>::value) v = (double)__half2float(s[i]) * inv_scale;
    else v = (double)__bfloat162float(s[i]) * inv_scale;
    if (wk) v += wk[i / N] * shift_w;
    dst[i] = v;
  }
}

// FP64 area-weighted sums of p* (sum of f) and S, two-pass deterministic
// (per-block partials, then one block in fixed order).
template <class ST>
__global__ void k_totals(const ST *f, const float *mac, const float *wx, const float *wz, int nx, int nz,
                         float inv_fs, double *part) {
  const long long N = (long long)nx * nz;
  double sp = 0, ss = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), z = (int)(i / nx);
    const double a = (double)wx[x] * (double)wz[z];
    double p = 0;
    for (int k = 0; k < 9; k++) {
      if constexpr (sizeof(ST) == 4) p += (double)((const float *)f)[k * N + i];
      else if constexpr (std::is_same<ST, __half>::value) p += (double)__half2float(f[k * N + i]) * inv_fs;
      else p += (double)__bfloat162float(f[k * N + i]) * inv_fs;
    }
    sp += p * a;
    ss += (double)mac[i] * a;
  }
  __shared__ double r[2][256];
  r[0][threadIdx.x] = sp;
  r[1][threadIdx.x] = ss;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      r[0][threadIdx.x] += r[0][threadIdx.x + o];
      r[1][threadIdx.x] += r[1][threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = r[0][0];
    part[2 * blockIdx.x + 1] = r[1][0];
  }
}
__global__ void k_totals_final(const double *part, int nb, double *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double a = 0, b = 0;
    for (int i = 0; i < nb; i++) {
      a += part[2 * i];
      b += part[2 * i + 1];
    }
    out[0] = a;
    out[1] = b;
  }
}

constexpr int kTotBlocks = 296;

void free_sim(ipcu_sim *s) {
  if (!s) return;
  for (int i = 0; i < 2; i++) {
    if (s->graph[i]) cudaGraphExecDestroy(s->graph[i]);
    cudaFree(s->f[i]);
    cudaFree(s->g[i]);
    cudaFree(s->mac[i]);
  }
  cudaFree(s->wA);
  cudaFree(s->scin);
  cudaFree(s->scout);
  cudaFree(s->wC);
  cudaFree(s->ginvx);
  cudaFree(s->ginvz);
  cudaFree(s->status);
  cudaFree(s->partials);
  delete s;
}

template <class V>
int upload(V **dst, const std::vector<V> &src) {
  if (src.empty()) return IPCU_OK;
  if (cudaMalloc((void **)dst, sizeof(V) * src.size()) != cudaSuccess) return IPCU_ERR_NOMEM;
  return cudaMemcpy(*dst, src.data(), sizeof(V) * src.size(), cudaMemcpyHostToDevice) == cudaSuccess ? IPCU_OK
                                                                                                      : IPCU_ERR_CUDA;
}

}  // namespace

extern "C" int ipcu_version(void) { return 100; }

extern "C" int ipcu_sim_create(const ipcu_sim_config *cfg, const double *s0, ipcu_stream_t stream, ipcu_sim **out) {
  if (!cfg || !out) return IPCU_ERR_ARG;
  *out = nullptr;
  const ipcu_sim_config &c = *cfg;
  if (c.nx < 1 || c.nz < 1 || c.dz <= 0 || c.dt <= 0 || c.tau <= 0.5) return IPCU_ERR_ARG;
  if (c.q_scalar != 0 && c.q_scalar != 5 && c.q_scalar != 9) return IPCU_ERR_ARG;
  if (c.q_scalar != 0 && c.taus <= 0.5) return IPCU_ERR_ARG;
  if (c.geometry < IPCU_GEO_UNIFORM || c.geometry > IPCU_GEO_Z3) return IPCU_ERR_ARG;
  if (c.storage < IPCU_STORE_F32 || c.storage > IPCU_STORE_BF16) return IPCU_ERR_ARG;
  if (c.wall != IPCU_WALL_BB && c.wall != IPCU_WALL_SLIP) return IPCU_ERR_ARG;
  if (c.mrt && (!c.M || !c.Minv || !c.S)) return IPCU_ERR_ARG;
  ipcu_sim *s = new ipcu_sim();
  s->cfg = c;
  s->cfg.x = s->cfg.z = s->cfg.wx = s->cfg.wz = nullptr;
  s->cfg.M = s->cfg.Minv = s->cfg.S = nullptr;
  s->nx = c.nx;
  s->nz = c.nz;
  s->N = (long long)c.nx * c.nz;
  s->stream = (cudaStream_t)stream;
  s->esz = c.storage == IPCU_STORE_F32 ? 4 : 2;
  const double dz = c.dz;
  if (c.mrt) {
    s->M.assign(c.M, c.M + 81);
    s->Minv.assign(c.Minv, c.Minv + 81);
    s->Srates.assign(c.S, c.S + 9);
  }
  s->X.resize(c.nx);
  s->Z.resize(c.nz);
  s->DX.resize(c.nx);
  s->DZ.resize(c.nz);
  for (int i = 0; i < c.nx; i++) {
    s->X[i] = c.x ? c.x[i] : (i + 0.5) * dz;
    s->DX[i] = c.wx ? c.wx[i] : dz;
    if (s->DX[i] < dz * (1 - 1e-9)) {  // CFL <= 1 on the interpolated axis
      free_sim(s);
      return IPCU_ERR_ARG;
    }
  }
  for (int l = 0; l < c.nz; l++) {
    s->Z[l] = c.z ? c.z[l] : (l + 0.5) * dz;
    s->DZ[l] = c.wz ? c.wz[l] : dz;
    if (s->DZ[l] < dz * (1 - 1e-9)) {
      free_sim(s);
      return IPCU_ERR_ARG;
    }
  }
  const int ax = geo_axis(c.geometry), ns = geo_ns(c.geometry);
  // a uniform geometry needs uniform widths; the interpolated axis may be anything >= dz
  for (int i = 0; i < c.nx && ax != 0; i++)
    if (std::fabs(s->DX[i] - dz) > 1e-12 * dz) {
      free_sim(s);
      return IPCU_ERR_ARG;
    }
  for (int l = 0; l < c.nz && ax != 1; l++)
    if (std::fabs(s->DZ[l] - dz) > 1e-12 * dz) {
      free_sim(s);
      return IPCU_ERR_ARG;
    }
  ensure_tables();
  int st = IPCU_OK;
  const size_t fb = s->esz * 9 * s->N, gb = s->esz * std::max(c.q_scalar, 1) * s->N, mb = sizeof(float) * 3 * s->N;
  for (int i = 0; i < 2 && st == IPCU_OK; i++) {
    if (cudaMalloc(&s->f[i], fb) != cudaSuccess || cudaMalloc(&s->g[i], gb) != cudaSuccess ||
        cudaMalloc((void **)&s->mac[i], mb) != cudaSuccess)
      st = IPCU_ERR_NOMEM;
  }
  if (st == IPCU_OK && (cudaMalloc((void **)&s->status, sizeof(unsigned)) != cudaSuccess ||
                        cudaMalloc((void **)&s->partials, sizeof(double) * (2 * kTotBlocks + 2)) != cudaSuccess))
    st = IPCU_ERR_NOMEM;
  if (st == IPCU_OK) cudaMemset(s->status, 0, sizeof(unsigned));
  if (st == IPCU_OK && ax >= 0) {
    std::vector<float> w, si, so, wc;
    axis_tables(ax == 0 ? s->X : s->Z, ax == 0 ? s->DX : s->DZ, dz, ns, w, si, so, wc);
    if ((st = upload(&s->wA, w)) == IPCU_OK && (st = upload(&s->scin, si)) == IPCU_OK &&
        (st = upload(&s->scout, so)) == IPCU_OK)
      st = upload(&s->wC, wc);
  }
  if (st == IPCU_OK) {
    std::vector<float> gx = grad_inv(s->X, dz), gz = grad_inv(s->Z, dz);
    if ((st = upload(&s->ginvx, gx)) == IPCU_OK) st = upload(&s->ginvz, gz);
  }
  if (st != IPCU_OK) {
    free_sim(s);
    return st;
  }
  // kernel parameters
  f2d::Params &P = s->P;
  std::memset(&P, 0, sizeof P);
  P.nx = c.nx;
  P.nz = c.nz;
  P.mrt = c.mrt ? 1 : 0;
  P.wall = c.wall;
  P.wA = s->wA;
  P.scin = s->scin;
  P.scout = s->scout;
  P.wC = s->wC;
  P.ginvx = s->ginvx;
  P.ginvz = s->ginvz;
  P.c = (float)(dz / c.dt);
  P.dt = (float)c.dt;
  P.fk3 = (float)(3.0 * c.dt * c.dt / dz);
  P.hdt = (float)(0.5 * c.dt);
  P.tau = (float)c.tau;
  P.taus = (float)(c.q_scalar ? c.taus : 1.0);
  P.rhoL = (float)c.rhoL;
  P.rhoH = (float)c.rhoH;
  P.phi = (float)c.phi;
  P.rho_sal = c.rho_sal;
  P.g_bouss = c.g_bouss;
  const bool lowp = c.storage != IPCU_STORE_F32;
  // reduced-precision storage: f is a pressure deviation, scaled into the
  // normal FP16 range; g is stored as the deviation from w_k * s_ref
  const double fscale = lowp ? (c.storage == IPCU_STORE_F16 ? 1024.0 : 1.0) : 1.0;
  const double gscale = lowp ? (c.storage == IPCU_STORE_F16 ? 64.0 : 1.0) : 1.0;
  P.fscale = (float)fscale;
  P.inv_fscale = (float)(1.0 / fscale);
  P.gscale = (float)gscale;
  P.inv_gscale = (float)(1.0 / gscale);
  P.s_ref = lowp ? (float)c.s_ref : 0.0f;
  if (c.mrt) {
    double Sv[9], MM[81];
    for (int i = 0; i < 9; i++) Sv[i] = c.S[i];
    Sv[7] = Sv[8] = 0;  // shear rows relax with 1/tau per cell (ref: function/basic.cu:185)
    for (int a = 0; a < 9; a++)
      for (int b = 0; b < 9; b++) {
        double acc = 0;
        for (int k = 0; k < 9; k++) acc += c.Minv[a * 9 + k] * Sv[k] * c.M[k * 9 + b];
        MM[a * 9 + b] = acc;
      }
    for (int i = 0; i < 81; i++) P.MM[i] = (float)MM[i];
    for (int k = 0; k < 9; k++) {
      P.Ms[k] = (float)c.M[7 * 9 + k];
      P.Ms[9 + k] = (float)c.M[8 * 9 + k];
      P.Mis[k * 2] = (float)c.Minv[k * 9 + 7];
      P.Mis[k * 2 + 1] = (float)c.Minv[k * 9 + 8];
    }
    // With unit non-shear rates and the Lallemand-Luo shear moments the
    // operator is f* = f - d + (1 - 1/tau) P d + Fk, P the projector on
    // p_xx = d1-d2+d3-d4 and p_xz = d5-d6+d7-d8 (weight 1/4 each): the kernel
    // then evaluates two moments instead of the 9x9 product.
    const double v7[9] = {0, 1, -1, 1, -1, 0, 0, 0, 0}, v8[9] = {0, 0, 0, 0, 0, 1, -1, 1, -1};
    double dev = 0;
    for (int a = 0; a < 9; a++)
      for (int b = 0; b < 9; b++) {
        const double pab = 0.25 * (v7[a] * v7[b] + v8[a] * v8[b]);
        double ps = 0;
        for (int l = 7; l < 9; l++) ps += c.Minv[a * 9 + l] * c.M[l * 9 + b];
        dev = std::max(dev, std::fabs(MM[a * 9 + b] - ((a == b ? 1.0 : 0.0) - pab)));
        dev = std::max(dev, std::fabs(ps - pab));
      }
    if (dev < 1e-12) P.mrt = 2;
  }
  slip_tables(9, P.slipB9, P.slipK9);
  slip_tables(5, P.slipB5, P.slipK5);
  P.status = s->status;
  for (int i = 0; i < 2; i++) {
    P.fbuf[i] = s->f[i];
    P.gbuf[i] = s->g[i];
    P.mbuf[i] = s->mac[i];
  }
  st = f2d::launch_step(P, c.storage, c.q_scalar, c.geometry, s->stream, true);
  if (st != IPCU_OK) {
    free_sim(s);
    return st;
  }
  // initial state: f = 0 (p* = 0, u = 0), g = w_k S, u = 0
  std::vector<double> S0(s->N, 0.0);
  if (s0) std::copy(s0, s0 + s->N, S0.begin());
  std::vector<double> g0((size_t)std::max(c.q_scalar, 1) * s->N, 0.0), f0((size_t)9 * s->N, 0.0), z0(s->N, 0.0);
  if (c.q_scalar)
    for (int k = 0; k < c.q_scalar; k++)
      for (long long i = 0; i < s->N; i++) g0[k * s->N + i] = (c.q_scalar == 5 ? w5d[k] : w9d[k]) * S0[i];
  *out = s;
  st = ipcu_sim_set_state(s, f0.data(), c.q_scalar ? g0.data() : nullptr, S0.data(), z0.data(), z0.data());
  if (st != IPCU_OK) {
    free_sim(s);
    *out = nullptr;
  }
  return st;
}

extern "C" void ipcu_sim_destroy(ipcu_sim *sim) {
  if (sim) cudaStreamSynchronize(sim->stream);
  free_sim(sim);
}

static int launch_one(ipcu_sim *s) {
  f2d::Params P = s->P;
  P.cur = s->cur;
  int st = f2d::launch_step(P, s->cfg.storage, s->cfg.q_scalar, s->cfg.geometry, s->stream);
  if (st == IPCU_OK) {
    s->cur ^= 1;
    s->steps++;
  }
  return st;
}

extern "C" int ipcu_sim_step(ipcu_sim *sim, int64_t nsteps) {
  if (!sim || nsteps < 0) return IPCU_ERR_ARG;
  for (int64_t i = 0; i < nsteps; i++) {
    int st = launch_one(sim);
    if (st) return st;
  }
  return IPCU_OK;
}

extern "C" int ipcu_sim_step_graph(ipcu_sim *sim, int64_t nsteps, int32_t chunk) {
  if (!sim || nsteps < 0 || chunk < 2) return IPCU_ERR_ARG;
  if (chunk % 2) chunk++;  // even, so a replay returns to the same buffer parity
  if (sim->graph_chunk != chunk) {
    for (int i = 0; i < 2; i++)
      if (sim->graph[i]) {
        cudaGraphExecDestroy(sim->graph[i]);
        sim->graph[i] = nullptr;
      }
    sim->graph_chunk = chunk;
  }
  int64_t left = nsteps;
  while (left >= chunk) {
    const int par = sim->cur;
    if (!sim->graph[par]) {
      cudaStream_t cs;
      if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return IPCU_ERR_CUDA;
      cudaStream_t keep = sim->stream;
      sim->stream = cs;
      cudaGraph_t gr;
      if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        sim->stream = keep;
        cudaStreamDestroy(cs);
        return IPCU_ERR_CUDA;
      }
      int st = IPCU_OK;
      for (int i = 0; i < chunk && st == IPCU_OK; i++) st = launch_one(sim);
      cudaError_t e = cudaStreamEndCapture(cs, &gr);
      sim->stream = keep;
      cudaStreamDestroy(cs);
      sim->cur = par;  // capture does not execute
      sim->steps -= chunk;
      if (st != IPCU_OK || e != cudaSuccess) return IPCU_ERR_CUDA;
      e = cudaGraphInstantiate(&sim->graph[par], gr, 0);
      cudaGraphDestroy(gr);
      if (e != cudaSuccess) return IPCU_ERR_CUDA;
    }
    if (cudaGraphLaunch(sim->graph[par], sim->stream) != cudaSuccess) return IPCU_ERR_CUDA;
    sim->steps += chunk;
    left -= chunk;
  }
  return ipcu_sim_step(sim, left);
}

extern "C" int64_t ipcu_sim_cells(const ipcu_sim *sim) { return sim ? sim->N : 0; }

extern "C" int64_t ipcu_sim_bytes_per_cell(const ipcu_sim *sim) {
  if (!sim) return 0;
  // every stored distribution and the three macroscopic fields are read once and written once
  return 2 * ((int64_t)sim->esz * (9 + sim->cfg.q_scalar) + 4 * 3);
}

extern "C" int ipcu_sim_device_state(ipcu_sim *sim, void **f, void **g, float **mac) {
  if (!sim) return IPCU_ERR_ARG;
  if (f) *f = sim->f[sim->cur];
  if (g) *g = sim->g[sim->cur];
  if (mac) *mac = sim->mac[sim->cur];
  return IPCU_OK;
}

static const double *wk_of(int q) { return q == 5 ? w5d : w9d; }

extern "C" int ipcu_sim_set_state(ipcu_sim *s, const double *f, const double *g, const double *S, const double *ux,
                                  const double *uz) {
  if (!s) return IPCU_ERR_ARG;
  const long long N = s->N;
  const int q = s->cfg.q_scalar;
  const double fs = s->P.fscale, gs = s->P.gscale, sref = s->P.s_ref;
  std::vector<unsigned char> buf;
  if (f) {
    buf.resize(s->esz * 9 * N);
    if (s->cfg.storage == IPCU_STORE_F32) to_store<float>(f, buf.data(), 9 * N, fs, 0, nullptr, 9, N);
    else if (s->cfg.storage == IPCU_STORE_F16) to_store<__half>(f, buf.data(), 9 * N, fs, 0, nullptr, 9, N);
    else to_store<__nv_bfloat16>(f, buf.data(), 9 * N, fs, 0, nullptr, 9, N);
    if (cudaMemcpy(s->f[s->cur], buf.data(), buf.size(), cudaMemcpyHostToDevice) != cudaSuccess) return IPCU_ERR_CUDA;
  }
  if (g && q) {
    buf.resize(s->esz * q * N);
    if (s->cfg.storage == IPCU_STORE_F32) to_store<float>(g, buf.data(), q * N, gs, sref, wk_of(q), q, N);
    else if (s->cfg.storage == IPCU_STORE_F16) to_store<__half>(g, buf.data(), q * N, gs, sref, wk_of(q), q, N);
    else to_store<__nv_bfloat16>(g, buf.data(), q * N, gs, sref, wk_of(q), q, N);
    if (cudaMemcpy(s->g[s->cur], buf.data(), buf.size(), cudaMemcpyHostToDevice) != cudaSuccess) return IPCU_ERR_CUDA;
  }
  const double *src[3] = {S, ux, uz};
  std::vector<float> m(N);
  for (int a = 0; a < 3; a++) {
    if (!src[a]) continue;
    for (long long i = 0; i < N; i++) m[i] = (float)src[a][i];
    if (cudaMemcpy(s->mac[s->cur] + a * N, m.data(), sizeof(float) * N, cudaMemcpyHostToDevice) != cudaSuccess)
      return IPCU_ERR_CUDA;
  }
  return IPCU_OK;
}

extern "C" int ipcu_sim_get(ipcu_sim *s, const char *field, double *out, int64_t n) {
  if (!s || !field || !out) return IPCU_ERR_ARG;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  const long long N = s->N;
  const int q = s->cfg.q_scalar;
  std::string fd(field);
  auto get_dist = [&](void *dev, int qq, double scale, double shift, const double *wk, double *dst) -> int {
    std::vector<unsigned char> buf(s->esz * qq * N);
    if (cudaMemcpy(buf.data(), dev, buf.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return IPCU_ERR_CUDA;
    if (s->cfg.storage == IPCU_STORE_F32) from_store<float>(buf.data(), dst, qq * N, 1.0 / scale, shift, wk, N);
    else if (s->cfg.storage == IPCU_STORE_F16) from_store<__half>(buf.data(), dst, qq * N, 1.0 / scale, shift, wk, N);
    else from_store<__nv_bfloat16>(buf.data(), dst, qq * N, 1.0 / scale, shift, wk, N);
    return IPCU_OK;
  };
  if (fd == "f") {
    if (n < 9 * N) return IPCU_ERR_CAPACITY;
    return get_dist(s->f[s->cur], 9, s->P.fscale, 0, nullptr, out);
  }
  if (fd == "g") {
    if (!q) return IPCU_ERR_ARG;
    if (n < q * N) return IPCU_ERR_CAPACITY;
    return get_dist(s->g[s->cur], q, s->P.gscale, s->P.s_ref, wk_of(q), out);
  }
  if (n < N) return IPCU_ERR_CAPACITY;
  if (fd == "p") {
    std::vector<double> f(9 * N);
    int st = get_dist(s->f[s->cur], 9, s->P.fscale, 0, nullptr, f.data());
    if (st) return st;
    for (long long i = 0; i < N; i++) {
      float a = 0.f;  // p* in the kernel's float order
      for (int k = 0; k < 9; k++) a += (float)f[k * N + i];
      out[i] = a;
    }
    return IPCU_OK;
  }
  int slot = fd == "S" ? 0 : (fd == "ux" ? 1 : (fd == "uz" ? 2 : (fd == "rho" ? 0 : -1)));
  if (slot < 0) return IPCU_ERR_ARG;
  std::vector<float> m(N);
  if (cudaMemcpy(m.data(), s->mac[s->cur] + slot * N, sizeof(float) * N, cudaMemcpyDeviceToHost) != cudaSuccess)
    return IPCU_ERR_CUDA;
  if (fd == "rho") {
    const float rho0 = s->P.rhoL + (s->P.rhoH - s->P.rhoL) * s->P.phi;
    for (long long i = 0; i < N; i++) out[i] = (float)((double)rho0 + (double)m[i] * s->P.rho_sal);
  } else {
    for (long long i = 0; i < N; i++) out[i] = m[i];
  }
  return IPCU_OK;
}

extern "C" int ipcu_sim_status(ipcu_sim *s, uint32_t *flags) {
  if (!s || !flags) return IPCU_ERR_ARG;
  unsigned v = 0;
  if (cudaMemcpyAsync(&v, s->status, sizeof v, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  *flags = v;
  return v ? IPCU_ERR_NONFINITE : IPCU_OK;
}

extern "C" int ipcu_sim_totals(ipcu_sim *s, double *sum_p, double *sum_s) {
  if (!s) return IPCU_ERR_ARG;
  // area weights (dx dz / dz^2) from the cell widths, FP32 copies on the device
  std::vector<float> wx(s->nx), wz(s->nz);
  for (int i = 0; i < s->nx; i++) wx[i] = (float)(s->DX[i] / s->cfg.dz);
  for (int l = 0; l < s->nz; l++) wz[l] = (float)(s->DZ[l] / s->cfg.dz);
  float *dwx = nullptr, *dwz = nullptr;
  if (upload(&dwx, wx) || upload(&dwz, wz)) {
    cudaFree(dwx);
    cudaFree(dwz);
    return IPCU_ERR_NOMEM;
  }
  const float ifs = s->P.inv_fscale;
  if (s->cfg.storage == IPCU_STORE_F32)
    k_totals<float><<<kTotBlocks, 256, 0, s->stream>>>((const float *)s->f[s->cur], s->mac[s->cur], dwx, dwz, s->nx, s->nz, ifs, s->partials);
  else if (s->cfg.storage == IPCU_STORE_F16)
    k_totals<__half><<<kTotBlocks, 256, 0, s->stream>>>((const __half *)s->f[s->cur], s->mac[s->cur], dwx, dwz, s->nx, s->nz, ifs, s->partials);
  else
    k_totals<__nv_bfloat16><<<kTotBlocks, 256, 0, s->stream>>>((const __nv_bfloat16 *)s->f[s->cur], s->mac[s->cur], dwx, dwz, s->nx, s->nz, ifs, s->partials);
  k_totals_final<<<1, 32, 0, s->stream>>>(s->partials, kTotBlocks, s->partials + 2 * kTotBlocks);
  double h[2] = {0, 0};
  cudaError_t e = cudaMemcpyAsync(h, s->partials + 2 * kTotBlocks, sizeof h, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(dwx);
  cudaFree(dwz);
  if (e != cudaSuccess) return IPCU_ERR_CUDA;
  if (sum_p) *sum_p = h[0];
  if (sum_s) *sum_s = h[1];
  return IPCU_OK;
}

extern "C" int ipcu_sim_upload(ipcu_sim *s, const void *f, const void *g, const float *mac) {
  if (!s) return IPCU_ERR_ARG;
  const long long N = s->N;
  cudaError_t e = cudaSuccess;
  if (f) e = cudaMemcpyAsync(s->f[s->cur], f, s->esz * 9 * N, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess && g && s->cfg.q_scalar)
    e = cudaMemcpyAsync(s->g[s->cur], g, s->esz * s->cfg.q_scalar * N, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess && mac) e = cudaMemcpyAsync(s->mac[s->cur], mac, sizeof(float) * 3 * N, cudaMemcpyHostToDevice, s->stream);
  return e == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

extern "C" int ipcu_sim_download(ipcu_sim *s, void *f, void *g, float *mac) {
  if (!s) return IPCU_ERR_ARG;
  const long long N = s->N;
  cudaError_t e = cudaSuccess;
  if (f) e = cudaMemcpyAsync(f, s->f[s->cur], s->esz * 9 * N, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess && g && s->cfg.q_scalar)
    e = cudaMemcpyAsync(g, s->g[s->cur], s->esz * s->cfg.q_scalar * N, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess && mac) e = cudaMemcpyAsync(mac, s->mac[s->cur], sizeof(float) * 3 * N, cudaMemcpyDeviceToHost, s->stream);
  return e == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

extern "C" int ipcu_sim_sync(ipcu_sim *s) {
  if (!s) return IPCU_ERR_ARG;
  return cudaStreamSynchronize(s->stream) == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

extern "C" int32_t ipcu_sim_storage_bytes(const ipcu_sim *s) { return s ? (int32_t)s->esz : 0; }

// ---------------------------------------------------------------------------
// Allocation-free totals. Some callers cannot allocate device memory at the
// point where they need the conservation check: code running inside CUDA
// graph capture (an allocation is not a capturable stream operation), hosts
// that hand all device memory to their own pool at start-up, and real-time
// loops that must not hit the driver's allocator. This entry point runs the
// same two-pass reduction as ipcu_sim_totals but keeps its per-block partial
// sums in a file-scope device array instead of allocated scratch.
//
// Limit: kNoAllocBlocks partials of kNoAllocCells cells each, i.e. at most
// 1024 * 16384 = 16,777,216 cells; larger fields are rejected with
// IPCU_ERR_CAPACITY. The array occupies 16.4 KB on every device that loads
// the library, until the process exits. Every call shares it and it keeps
// the last call's contents: each call writes every partial it reads, so
// nothing needs clearing, but calls whose kernels overlap on the GPU (two
// streams, or two host threads) race on it and must be serialised by the
// caller.
constexpr int kNoAllocBlocks = 1024;
constexpr long long kNoAllocCells = 16384;
static __device__ __align__(256) double g_noalloc_partials[2 * kNoAllocBlocks + 2];

extern "C" int ipcu_totals_noalloc_f32(const float *f, const float *mac, const float *wx, const float *wz, int nx,
                                       int nz, double *out, ipcu_stream_t stream) {
  if (!f || !mac || !wx || !wz || !out || nx < 1 || nz < 1) return IPCU_ERR_ARG;
  const long long N = (long long)nx * nz;
  if (N > (long long)kNoAllocBlocks * kNoAllocCells) return IPCU_ERR_CAPACITY;
  // host code cannot use the array's name as a device address: resolve it
  // once per device (the first call on a device does this set-up, so it
  // should come before any stream capture)
  static double *dev_ptr[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return IPCU_ERR_CUDA;
  if (!dev_ptr[dev]) {
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_partials) != cudaSuccess || !ptr) return IPCU_ERR_CUDA;
    dev_ptr[dev] = static_cast<double *>(ptr);
  }
  const int nb = (int)((N + kNoAllocCells - 1) / kNoAllocCells);
  k_totals<float><<<nb, 256, 0, (cudaStream_t)stream>>>(f, mac, wx, wz, nx, nz, 1.0f, dev_ptr[dev]);
  k_totals_final<<<1, 32, 0, (cudaStream_t)stream>>>(dev_ptr[dev], nb, out);
  return status_from_cuda(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Checkpoint / restore: a versioned binary snapshot of the configuration,
// the axis geometry, the MRT matrices, the step count and the raw state in
// its storage format (replaces the reference's unused text save_status,
// ref: function/basic.cu:31-56, which had no reader).
namespace {
constexpr char kMagic[8] = {'I', 'P', 'C', 'U', 'S', 'I', 'M', '1'};
constexpr int32_t kSnapVersion = 1;
template <class T>
bool wr(FILE *f, const T *p, size_t n) { return fwrite(p, sizeof(T), n, f) == n; }
template <class T>
bool rd(FILE *f, T *p, size_t n) { return fread(p, sizeof(T), n, f) == n; }
}  // namespace

extern "C" int64_t ipcu_sim_steps(const ipcu_sim *s) { return s ? s->steps : -1; }

extern "C" int ipcu_sim_save(ipcu_sim *s, const char *path) {
  if (!s || !path) return IPCU_ERR_ARG;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  const long long N = s->N;
  const int q = s->cfg.q_scalar;
  std::vector<unsigned char> fb(s->esz * 9 * N), gb(s->esz * (size_t)q * N);
  std::vector<float> mb(3 * N);
  if (cudaMemcpy(fb.data(), s->f[s->cur], fb.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return IPCU_ERR_CUDA;
  if (q && cudaMemcpy(gb.data(), s->g[s->cur], gb.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return IPCU_ERR_CUDA;
  if (cudaMemcpy(mb.data(), s->mac[s->cur], sizeof(float) * 3 * N, cudaMemcpyDeviceToHost) != cudaSuccess)
    return IPCU_ERR_CUDA;
  FILE *f = fopen(path, "wb");
  if (!f) return IPCU_ERR_IO;
  ipcu_sim_config c = s->cfg;
  c.x = c.z = c.wx = c.wz = c.M = c.Minv = c.S = nullptr;
  bool ok = wr(f, kMagic, 8) && wr(f, &kSnapVersion, 1) && wr(f, &c, 1) && wr(f, &s->steps, 1) &&
            wr(f, s->X.data(), s->X.size()) && wr(f, s->Z.data(), s->Z.size()) && wr(f, s->DX.data(), s->DX.size()) &&
            wr(f, s->DZ.data(), s->DZ.size());
  if (ok && c.mrt) ok = wr(f, s->M.data(), 81) && wr(f, s->Minv.data(), 81) && wr(f, s->Srates.data(), 9);
  ok = ok && wr(f, fb.data(), fb.size()) && wr(f, gb.data(), gb.size()) && wr(f, mb.data(), mb.size());
  ok = (fclose(f) == 0) && ok;
  return ok ? IPCU_OK : IPCU_ERR_IO;
}

extern "C" int ipcu_sim_load(const char *path, ipcu_stream_t stream, ipcu_sim **out) {
  if (!path || !out) return IPCU_ERR_ARG;
  *out = nullptr;
  FILE *f = fopen(path, "rb");
  if (!f) return IPCU_ERR_IO;
  char mg[8];
  int32_t ver = 0;
  ipcu_sim_config c;
  long long steps = 0;
  bool ok = rd(f, mg, 8) && std::memcmp(mg, kMagic, 8) == 0 && rd(f, &ver, 1) && ver == kSnapVersion && rd(f, &c, 1) &&
            rd(f, &steps, 1) && c.nx > 0 && c.nz > 0;
  std::vector<double> X(ok ? c.nx : 0), Z(ok ? c.nz : 0), DX(X.size()), DZ(Z.size()), M(81), Mi(81), S(9);
  ok = ok && rd(f, X.data(), X.size()) && rd(f, Z.data(), Z.size()) && rd(f, DX.data(), DX.size()) &&
       rd(f, DZ.data(), DZ.size());
  if (ok && c.mrt) ok = rd(f, M.data(), 81) && rd(f, Mi.data(), 81) && rd(f, S.data(), 9);
  if (!ok) {
    fclose(f);
    return IPCU_ERR_IO;
  }
  c.x = X.data();
  c.z = Z.data();
  c.wx = DX.data();
  c.wz = DZ.data();
  c.M = c.mrt ? M.data() : nullptr;
  c.Minv = c.mrt ? Mi.data() : nullptr;
  c.S = c.mrt ? S.data() : nullptr;
  ipcu_sim *s = nullptr;
  int st = ipcu_sim_create(&c, nullptr, stream, &s);
  if (st != IPCU_OK) {
    fclose(f);
    return st;
  }
  const long long N = s->N;
  const int q = c.q_scalar;
  std::vector<unsigned char> fb(s->esz * 9 * N), gb(s->esz * (size_t)q * N);
  std::vector<float> mb(3 * N);
  ok = rd(f, fb.data(), fb.size()) && rd(f, gb.data(), gb.size()) && rd(f, mb.data(), mb.size());
  fclose(f);
  if (!ok) {
    ipcu_sim_destroy(s);
    return IPCU_ERR_IO;
  }
  if (cudaMemcpy(s->f[s->cur], fb.data(), fb.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      (q && cudaMemcpy(s->g[s->cur], gb.data(), gb.size(), cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemcpy(s->mac[s->cur], mb.data(), sizeof(float) * 3 * N, cudaMemcpyHostToDevice) != cudaSuccess) {
    ipcu_sim_destroy(s);
    return IPCU_ERR_CUDA;
  }
  s->steps = steps;
  *out = s;
  return IPCU_OK;
}

// Field CSV in the reference's column order (ref: function/basic.cu:16-28):
// "num_calc,N" then x,y,z,delx,dely,pressure,salinity,phi,rho,u,v,w,Fx,Fy,Fz
// per cell in the reference's cell order (x-major, z fastest). Fx, Fz are the
// force the next step applies to the current state (buoyancy + pressure
// gradient); the reference wrote the one applied to the previous state.
extern "C" int ipcu_sim_write_csv(ipcu_sim *s, const char *path) {
  if (!s || !path) return IPCU_ERR_ARG;
  const long long N = s->N;
  std::vector<double> p(N), S(N), ux(N), uz(N), rho(N);
  int st;
  if ((st = ipcu_sim_get(s, "p", p.data(), N)) || (st = ipcu_sim_get(s, "S", S.data(), N)) ||
      (st = ipcu_sim_get(s, "ux", ux.data(), N)) || (st = ipcu_sim_get(s, "uz", uz.data(), N)) ||
      (st = ipcu_sim_get(s, "rho", rho.data(), N)))
    return st;
  FILE *f = fopen(path, "w");
  if (!f) return IPCU_ERR_IO;
  const int nx = s->nx, nz = s->nz;
  const double c2 = (double)s->P.c * s->P.c, reg = s->cfg.dz / 1000.0;
  fprintf(f, "num_calc,%lld\n", N);
  fprintf(f, "x       ,y       ,z       ,delx    ,dely    ,pressure,salinity ,phi     ,rho     ,u       ,v       ,w       ,Fx      ,Fy      ,Fz      \n");
  for (int i = 0; i < nx; i++)
    for (int l = 0; l < nz; l++) {
      const long long c = (long long)l * nx + i;
      const int ip = std::min(i + 1, nx - 1), im = std::max(i - 1, 0), lp = std::min(l + 1, nz - 1), lm = std::max(l - 1, 0);
      const double pc = p[c] * c2 / 3.0;
      const double Fx = -pc * (rho[(long long)l * nx + ip] - rho[(long long)l * nx + im]) / (s->X[ip] - s->X[im] + reg);
      const double Fz = -S[c] * s->cfg.g_bouss -
                        pc * (rho[(long long)lp * nx + i] - rho[(long long)lm * nx + i]) / (s->Z[lp] - s->Z[lm] + reg);
      fprintf(f, "%f,%f,%f,%f,%f,%f,%f,%f,%f,%f,%f,%f,%f,%f,%f\n", s->X[i], 0.5 * s->cfg.dz, s->Z[l], s->DX[i],
              s->cfg.dz, p[c], S[c], s->cfg.phi, rho[c], ux[c], 0.0, uz[c], Fx, 0.0, Fz);
    }
  return fclose(f) == 0 ? IPCU_OK : IPCU_ERR_IO;
}

// ---------------------------------------------------------------------------
// Batched stepping: many resident simulations advanced together, one launch
// per step for each (storage, scalar lattice, geometry) class, CTAs walking a
// device work list of (simulation, tile) items. Each simulation's arithmetic
// is the single-run kernel's, tile by tile, so a simulation's result does not
// depend on what it is batched with.
struct ipcu_batch {
  cudaStream_t stream;
  f2d::Params *d_params = nullptr;
  f2d::WorkItem *d_work = nullptr;
  size_t cap_params = 0, cap_work = 0;
  int grid_cap = 0;
};

extern "C" int ipcu_batch_create(ipcu_stream_t stream, ipcu_batch **out) {
  if (!out) return IPCU_ERR_ARG;
  ipcu_batch *b = new ipcu_batch();
  b->stream = (cudaStream_t)stream;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  b->grid_cap = sms * f2d::kMinBlocks;
  *out = b;
  return IPCU_OK;
}

extern "C" void ipcu_batch_destroy(ipcu_batch *b) {
  if (!b) return;
  cudaStreamSynchronize(b->stream);
  cudaFree(b->d_params);
  cudaFree(b->d_work);
  delete b;
}

extern "C" int ipcu_batch_step(ipcu_batch *b, ipcu_sim *const *sims, int n, int64_t nsteps) {
  if (!b || (n > 0 && !sims) || nsteps < 0) return IPCU_ERR_ARG;
  if (n == 0 || nsteps == 0) return IPCU_OK;
  for (int i = 0; i < n; i++) {
    if (!sims[i]) return IPCU_ERR_ARG;
    // the batch stream takes over: the simulation's own work must be finished
    if (cudaStreamSynchronize(sims[i]->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  }
  // group by kernel class, keeping order
  std::vector<int> order(n);
  for (int i = 0; i < n; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
    const ipcu_sim_config &A = sims[a]->cfg, &C = sims[c]->cfg;
    return std::make_tuple(A.storage, A.q_scalar, A.geometry) < std::make_tuple(C.storage, C.q_scalar, C.geometry);
  });
  std::vector<f2d::Params> hp(n);
  std::vector<f2d::WorkItem> hw;
  struct Group { int storage, qs, geo, w0, w1; };
  std::vector<Group> groups;
  for (int oi = 0; oi < n; oi++) {
    ipcu_sim *s = sims[order[oi]];
    hp[oi] = s->P;
    hp[oi].cur = s->cur;
    const ipcu_sim_config &c = s->cfg;
    if (groups.empty() || groups.back().storage != c.storage || groups.back().qs != c.q_scalar ||
        groups.back().geo != c.geometry)
      groups.push_back({c.storage, c.q_scalar, c.geometry, (int)hw.size(), (int)hw.size()});
    const int tx = (s->nx + f2d::kTX - 1) / f2d::kTX, tz = (s->nz + f2d::kTZ - 1) / f2d::kTZ;
    for (int z = 0; z < tz; z++)
      for (int x = 0; x < tx; x++) hw.push_back({oi, x, z, 0});
    groups.back().w1 = (int)hw.size();
  }
  if (hp.size() > b->cap_params) {
    cudaFree(b->d_params);
    if (cudaMalloc((void **)&b->d_params, sizeof(f2d::Params) * hp.size()) != cudaSuccess) return IPCU_ERR_NOMEM;
    b->cap_params = hp.size();
  }
  if (hw.size() > b->cap_work) {
    cudaFree(b->d_work);
    if (cudaMalloc((void **)&b->d_work, sizeof(f2d::WorkItem) * hw.size()) != cudaSuccess) return IPCU_ERR_NOMEM;
    b->cap_work = hw.size();
  }
  if (cudaMemcpyAsync(b->d_params, hp.data(), sizeof(f2d::Params) * hp.size(), cudaMemcpyHostToDevice, b->stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(b->d_work, hw.data(), sizeof(f2d::WorkItem) * hw.size(), cudaMemcpyHostToDevice, b->stream) !=
          cudaSuccess)
    return IPCU_ERR_CUDA;
  for (const Group &g : groups) {
    int st = f2d::launch_batched(nullptr, nullptr, 0, 0, g.storage, g.qs, g.geo, 0, b->stream, true);
    if (st) return st;
  }
  for (int64_t k = 0; k < nsteps; k++) {
    for (const Group &g : groups) {
      const int nw = g.w1 - g.w0;
      const int grid = std::min(nw, b->grid_cap);
      int st = f2d::launch_batched(b->d_params, b->d_work + g.w0, nw, (int)(k & 1), g.storage, g.qs, g.geo, grid,
                                   b->stream, false);
      if (st) return st;
    }
  }
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  for (int i = 0; i < n; i++) {
    sims[i]->cur ^= (int)(nsteps & 1);
    sims[i]->steps += nsteps;
  }
  return IPCU_OK;
}

extern "C" int64_t ipcu_sim_device_bytes(const ipcu_sim *s) {
  if (!s) return 0;
  const long long N = s->N;
  return 2 * ((long long)s->esz * (9 + std::max(s->cfg.q_scalar, 1)) * N + 4LL * 3 * N) +
         4LL * (3 * (s->nx + s->nz) + 2 * 5 * std::max(s->nx, s->nz)) + 2048;
}
