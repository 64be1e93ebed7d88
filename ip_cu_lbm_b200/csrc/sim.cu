// Structured-grid solver object (ipcu_sim_*): device-resident state,
// host-precomputed axis tables, stepping (direct or CUDA-graph replay),
// field I/O and FP64 conservation totals.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <array>
#include <map>
#include <tuple>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "axis_tables.hpp"
#include "fused2d.cuh"
#include "ibm2d.cuh"
#include "ipcu_common.cuh"
#include "storage.cuh"

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
  float *obuf[2] = {nullptr, nullptr};     // phase field: previous step's phi u, phi w
  float *ilx2 = nullptr, *ilz2 = nullptr;  // phase field: 1/dx^2, 1/dz^2
  unsigned *status = nullptr;
  double *partials = nullptr;
  cudaEvent_t ready = nullptr;  // recorded on the stream before a batch takes the simulation
  int cur = 0;
  f2d::Params P;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // per starting parity
  int graph_chunk = 0;
  std::vector<double> X, Z, DX, DZ;
  std::vector<double> M, Minv, Srates;  // MRT matrices as given (for snapshots)
  long long steps = 0;                  // time steps taken since creation / restore
  // moving immersed boundaries (empty without a body): each body's device
  // state and coupled-update parameters (fp filled per launch); the force
  // density and the tile flags ([bodies][tiles]) they share; with several
  // bodies, device copies of the job list per starting buffer parity
  std::vector<ib2d::Job *> ibs;
  float *ibfext = nullptr;
  uint8_t *ibflags = nullptr;
  ib2d::Job *d_jobs[2] = {nullptr, nullptr};
  bool jobs_dirty = true;
  // lean flow-only step (f2d::Params::lean): per-parity tile flags of
  // stored velocity planes; lean_ok: the configuration allows it
  uint8_t *ustore[2] = {nullptr, nullptr};
  bool lean_ok = false;
  int ntiles = 0;
  // area weights dx dz / dz^2 per column and row (conservation totals)
  float *twx = nullptr, *twz = nullptr;
  // the attached bodies' descriptions as given (snapshots re-attach them)
  std::vector<ipcu_ib_body2d> ib_cfg;
  std::vector<std::vector<double>> ib_X0, ib_dS;
};

// Macroscopic planes: S, u_x, u_z (+ p* with 16-bit storage)
static int nmac(const ipcu_sim *s) { return s->cfg.storage == IPCU_STORE_F32 ? 3 : 4; }

namespace {

constexpr int ex9[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
constexpr int ez9[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
constexpr int kinv9[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};

inline int geo_axis(int geo) {
  return (geo == IPCU_GEO_X5 || geo == IPCU_GEO_X3) ? 0 : ((geo == IPCU_GEO_Z5 || geo == IPCU_GEO_Z3) ? 1 : -1);
}
inline int geo_ns(int geo) {
  return (geo == IPCU_GEO_X5 || geo == IPCU_GEO_Z5) ? 5 : ((geo == IPCU_GEO_X3 || geo == IPCU_GEO_Z3) ? 3 : 1);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); null when the driver does not provide it
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Planes [planes][nz][nx] of 4-byte (FP32) or 2-byte (16-bit storage, moved
// as raw bits) values read as boxes of [planes][rows][kTmaBoxX] or
// [planes][rows][kTmaBoxX16]; cells outside the array read as zero
bool encode_planes(CUtensorMap *map, void *base, int nx, int nz, int planes, int rows, int esz = 4) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc || (nx * esz) % 16 != 0) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)nz, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)nx * esz, (cuuint64_t)nx * nz * esz};
  const cuuint32_t box[3] = {(cuuint32_t)(esz == 4 ? f2d::kTmaBoxX : f2d::kTmaBoxX16), (cuuint32_t)rows,
                             (cuuint32_t)planes};
  const cuuint32_t es[3] = {1, 1, 1};
  return enc(map, esz == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16, 3, base, dims,
             strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
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

// FP32 <-> stored value (16-bit storage multiplies by `scale` first)
template <class ST>
inline void enc(const float *src, void *dst, long long n, float scale) {
  ST *d = (ST *)dst;
  for (long long i = 0; i < n; i++) {
    if constexpr (sizeof(ST) == 4) d[i] = src[i];
    else if constexpr (std::is_same<ST, __half>::value) d[i] = __float2half_rn(src[i] * scale);
    else d[i] = __float2bfloat16_rn(src[i] * scale);
  }
}
template <class ST>
inline void dec(const void *src, float *dst, long long n, float inv_scale) {
  const ST *d = (const ST *)src;
  for (long long i = 0; i < n; i++) {
    if constexpr (sizeof(ST) == 4) dst[i] = ((const float *)d)[i];
    else if constexpr (std::is_same<ST, __half>::value) dst[i] = __half2float(d[i]) * inv_scale;
    else dst[i] = __bfloat162float(d[i]) * inv_scale;
  }
}

// FP32 scalar lattice at rest: g_k = w_k S (the product in double, rounded once)
__global__ void k_init_g(const float *S, int q, float *g, long long N) {
  IPCU_FOR(i, 0, N) {
    const double v = S[i];
    for (int k = 0; k < q; k++) {
      const double w = q == 5 ? (k == 0 ? 1.0 / 3 : 1.0 / 6) : (k == 0 ? 4.0 / 9 : (k <= 4 ? 1.0 / 9 : 1.0 / 36));
      g[k * N + i] = (float)(w * v);
    }
  }
}

// Lean flow-only step: completes the velocity planes of buffer b in the
// tiles whose last step did not store them (ustore[b][tile] 0 or 2), with
// the value that step formed, c j + F dt / 2 rho from the populations
// (f2d::lean_velocity).
__global__ void k_lean_fill(const __grid_constant__ f2d::Params P, int b) {
  const long long N = (long long)P.nx * P.nz;
  float *mac = P.mbuf[b];
  IPCU_FOR(i, 0, N) {
    const int x = (int)(i % P.nx), z = (int)(i / P.nx);
    if (P.ustore[b][(z / f2d::kTZ) * P.ntx + x / f2d::kTX] == 1) continue;
    float ux, uz;
    f2d::lean_velocity(P, b, i, N, ux, uz);
    mac[N + i] = ux;
    mac[2 * N + i] = uz;
  }
}

// FP64 area-weighted sums of p* (sum of f) and S, two-pass deterministic
// (per-block partials, then one block in fixed order).
// (16-bit storage keeps p* in the 4th macroscopic plane; pass f = nullptr)
__global__ void k_totals(const float *f, const float *mac, const float *wx, const float *wz, int nx, int nz,
                         double *part) {
  const long long N = (long long)nx * nz;
  double sp = 0, ss = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), z = (int)(i / nx);
    const double a = (double)wx[x] * (double)wz[z];
    double p = 0;
    if (f) {
      for (int k = 0; k < 9; k++) p += (double)f[k * N + i];
    } else {
      p = (double)mac[3 * N + i];
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
constexpr int kMaxBodies = 16;  // bodies per simulation

// A simulation's device memory comes from the device's stream-ordered pool
// (cudaMallocAsync on the simulation's stream): creating and retiring many
// simulations, as a server does, then neither synchronises the device nor
// returns memory to the driver in between. The pool keeps freed memory
// for reuse (release threshold raised once per device, for this process).
void retain_pool() {
  static bool done[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done[dev] = true;
}
template <class V>
bool salloc(ipcu_sim *s, V **p, size_t bytes) {
  return cudaMallocAsync((void **)p, bytes, s->stream) == cudaSuccess;
}
template <class V>
int supload(ipcu_sim *s, V **dst, const std::vector<V> &src) {
  if (src.empty()) return IPCU_OK;
  if (!salloc(s, dst, sizeof(V) * src.size())) return IPCU_ERR_NOMEM;
  // pageable source: the call returns once the source has been staged
  return cudaMemcpyAsync(*dst, src.data(), sizeof(V) * src.size(), cudaMemcpyHostToDevice, s->stream) == cudaSuccess
             ? IPCU_OK
             : IPCU_ERR_CUDA;
}

void free_sim(ipcu_sim *s) {
  if (!s) return;
  auto fr = [&](void *p) {
    if (p) cudaFreeAsync(p, s->stream);
  };
  for (int i = 0; i < 2; i++) {
    if (s->graph[i]) cudaGraphExecDestroy(s->graph[i]);
    fr(s->f[i]);
    fr(s->g[i]);
    fr(s->mac[i]);
  }
  fr(s->wA);
  fr(s->scin);
  fr(s->scout);
  fr(s->wC);
  fr(s->ginvx);
  fr(s->ginvz);
  fr(s->status);
  fr(s->partials);
  fr(s->obuf[0]);
  fr(s->obuf[1]);
  fr(s->ilx2);
  fr(s->ilz2);
  fr(s->ustore[0]);
  fr(s->ustore[1]);
  fr(s->twx);
  fr(s->twz);
  for (ib2d::Job *j : s->ibs) {
    fr(j->body);
    fr((void *)j->X0);
    fr((void *)j->dS);
    fr(j->org);
    fr(j->org2);
    fr(j->fmark);
    delete j;
  }
  fr(s->ibfext);
  fr(s->ibflags);
  fr(s->d_jobs[0]);
  fr(s->d_jobs[1]);
  if (s->ready) cudaEventDestroy(s->ready);
  delete s;
}

template <class V>
int upload(V **dst, const std::vector<V> &src) {
  if (src.empty()) return IPCU_OK;
  if (cudaMalloc((void **)dst, sizeof(V) * src.size()) != cudaSuccess) return IPCU_ERR_NOMEM;
  return cudaMemcpy(*dst, src.data(), sizeof(V) * src.size(), cudaMemcpyHostToDevice) == cudaSuccess ? IPCU_OK
                                                                                                      : IPCU_ERR_CUDA;
}

// ---- lean flow-only step bookkeeping
// The current buffer's velocity planes made complete (before anything reads
// them from outside the lean kernels: field reads, downloads, snapshots,
// batched steps).
int lean_fill(ipcu_sim *s) {
  if (!s->P.lean) return IPCU_OK;
  const Launch L = launch_for(s->N);
  k_lean_fill<<<L.grid, L.block, 0, s->stream>>>(s->P, s->cur);
  return status_from_cuda(cudaGetLastError());
}
// Every tile of the current buffer holds its velocity planes (after an
// upload, or after batched steps).
int lean_mark_all(ipcu_sim *s) {
  if (!s->ustore[0]) return IPCU_OK;
  return status_from_cuda(cudaMemsetAsync(s->ustore[s->cur], 1, (size_t)s->ntiles, s->stream));
}
void drop_graphs(ipcu_sim *s) {
  cudaStreamSynchronize(s->stream);
  s->jobs_dirty = true;  // the parameters changed: the device job lists follow
  for (int i = 0; i < 2; i++)
    if (s->graph[i]) {
      cudaGraphExecDestroy(s->graph[i]);
      s->graph[i] = nullptr;
    }
  s->graph_chunk = 0;
}
// A new S plane was written to the current buffer: the lean step stays on
// only while S is uniform at the value it was set up with.
void lean_check_s(ipcu_sim *s, const float *S) {
  if (!s->P.ib_uform) return;
  for (long long i = 0; i < s->N; i++)
    if (S[i] != s->P.s_uni) {
      s->lean_ok = false;
      s->P.ib_uform = 0;
      if (s->P.lean) s->P.lean = 0;
      drop_graphs(s);
      return;
    }
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
  if (c.scalar_kind != IPCU_SCALAR_SALINITY && c.scalar_kind != IPCU_SCALAR_PHASE) return IPCU_ERR_ARG;
  if (c.scalar_kind == IPCU_SCALAR_PHASE && (c.q_scalar == 0 || !(c.pf_width > 0))) return IPCU_ERR_ARG;
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
  retain_pool();
  int st = cudaEventCreateWithFlags(&s->ready, cudaEventDisableTiming) == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
  const size_t fb = s->esz * 9 * s->N, gb = s->esz * std::max(c.q_scalar, 1) * s->N, mb = sizeof(float) * nmac(s) * s->N;
  for (int i = 0; i < 2 && st == IPCU_OK; i++) {
    if (!salloc(s, &s->f[i], fb) || !salloc(s, &s->g[i], gb) || !salloc(s, &s->mac[i], mb)) st = IPCU_ERR_NOMEM;
  }
  if (st == IPCU_OK &&
      (!salloc(s, &s->status, sizeof(unsigned)) || !salloc(s, &s->partials, sizeof(double) * (2 * kTotBlocks + 2))))
    st = IPCU_ERR_NOMEM;
  if (st == IPCU_OK) cudaMemsetAsync(s->status, 0, sizeof(unsigned), s->stream);
  const bool pf = c.scalar_kind == IPCU_SCALAR_PHASE;
  for (int i = 0; i < 2 && st == IPCU_OK && pf; i++) {
    if (!salloc(s, &s->obuf[i], sizeof(float) * 2 * s->N)) st = IPCU_ERR_NOMEM;
    else cudaMemsetAsync(s->obuf[i], 0, sizeof(float) * 2 * s->N, s->stream);  // u = 0 at rest
  }
  if (st == IPCU_OK && pf) {
    std::vector<float> lx(c.nx), lz(c.nz);
    for (int i = 0; i < c.nx; i++) lx[i] = (float)(1.0 / (s->DX[i] * s->DX[i]));
    for (int l = 0; l < c.nz; l++) lz[l] = (float)(1.0 / (s->DZ[l] * s->DZ[l]));
    if ((st = supload(s, &s->ilx2, lx)) == IPCU_OK) st = supload(s, &s->ilz2, lz);
  }
  if (st == IPCU_OK && ax >= 0) {
    std::vector<float> w, si, so, wc;
    axis_tables(ax == 0 ? s->X : s->Z, ax == 0 ? s->DX : s->DZ, dz, ns, w, si, so, wc);
    if ((st = supload(s, &s->wA, w)) == IPCU_OK && (st = supload(s, &s->scin, si)) == IPCU_OK &&
        (st = supload(s, &s->scout, so)) == IPCU_OK)
      st = supload(s, &s->wC, wc);
  }
  if (st == IPCU_OK) {
    std::vector<float> gx = grad_inv(s->X, dz), gz = grad_inv(s->Z, dz);
    if ((st = supload(s, &s->ginvx, gx)) == IPCU_OK) st = supload(s, &s->ginvz, gz);
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
  {
    // tables of an evenly spaced axis hold three values: first, interior, last
    auto three = [](const std::vector<float> &t, float *o) {
      const size_t n = t.size();
      if (n < 3) return false;
      for (size_t i = 2; i + 1 < n; i++)
        if (t[i] != t[1]) return false;
      o[0] = t[0];
      o[1] = t[1];
      o[2] = t[n - 1];
      return true;
    };
    const std::vector<float> tx = grad_inv(s->X, dz), tz = grad_inv(s->Z, dz);
    P.gconst = (three(tx, P.gix3) ? 1 : 0) | (three(tz, P.giz3) ? 2 : 0);
  }
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
  P.rho_sal_f = (float)c.rho_sal;
  P.g_bouss_f = (float)c.g_bouss;
  P.rho_base = std::fmaf(P.rhoH - P.rhoL, P.phi, P.rhoL);
  P.pf = pf ? 1 : 0;
  if (pf) {
    // the scalar is phi: rho = rhoL + (rhoH - rhoL) phi; surface tension
    // beta = 12 sigma / W, kappa = 3 sigma W / 2 (ref: collision.cu:71)
    P.rho_base = P.rhoL;
    P.rho_sal_f = P.rhoH - P.rhoL;
    P.pf_beta4 = (float)(48.0 * c.sigma / c.pf_width);
    P.pf_kap = (float)(1.5 * c.sigma * c.pf_width);
    P.pf_invw = (float)(1.0 / c.pf_width);
    P.pf_lam = (float)((c.taus - 0.5) / c.taus);
    P.grav = (float)c.gravity;
    P.ilx2 = s->ilx2;
    P.ilz2 = s->ilz2;
    for (int i = 0; i < 2; i++) P.obuf[i] = s->obuf[i];
  }
  // 16-bit storage holds deviations from the local equilibrium (mostly
  // 1e-8 .. 1e-1 in lattice units); FP16 scales them by 2^12 so that they sit
  // in its normal range with room up to 16 before the 65504 limit
  const double scale = c.storage == IPCU_STORE_F16 ? 4096.0 : 1.0;
  P.fscale = P.gscale = (float)scale;
  P.inv_fscale = P.inv_gscale = (float)(1.0 / scale);
  P.store_max = c.storage == IPCU_STORE_F16 ? 65504.0f : 3.0e38f;
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
  // TMA staging for FP32 storage: tile + halo rows for f and g, ring rows
  // (one more on each side) for the S, u_x, u_z planes
  // TMA staging: FP32 storage with nx % 4 == 0; 16-bit storage with
  // nx % 8 == 0 and no scalar lattice (with one, the staged 16-bit boxes
  // beside the float tile leave room for 2 CTAs per SM instead of 4, which
  // measured slower than register staging)
  P.tma = 0;
  if ((c.storage == IPCU_STORE_F32 && c.nx % 4 == 0) ||
      (c.storage != IPCU_STORE_F32 && c.nx % 8 == 0 && c.q_scalar == 0)) {
    const int rows = f2d::kTZ + 2 * f2d::halo_z(c.geometry), esz = (int)s->esz;
    bool ok = true;
    for (int i = 0; i < 2 && ok; i++) {
      ok = encode_planes(&P.tm_f[i], s->f[i], c.nx, c.nz, 9, rows, esz) &&
           encode_planes(&P.tm_m[i], s->mac[i], c.nx, c.nz, nmac(s), rows + 2) &&
           (c.q_scalar == 0 || encode_planes(&P.tm_g[i], s->g[i], c.nx, c.nz, c.q_scalar, rows, esz));
    }
    P.tma = ok ? 1 : 0;
  }
  // tiles, and the lean flow-only step where the configuration allows it:
  // FP32 storage with TMA staging, no scalar lattice, a uniform S
  P.ntx = (c.nx + f2d::kTX - 1) / f2d::kTX;
  P.ntz = (c.nz + f2d::kTZ - 1) / f2d::kTZ;
  s->ntiles = P.ntx * P.ntz;
  {
    bool uni = true;
    const float s00 = s0 ? (float)s0[0] : 0.f;
    for (long long i = 1; s0 && i < s->N && uni; i++) uni = (float)s0[i] == s00;
    s->lean_ok = c.storage == IPCU_STORE_F32 && c.q_scalar == 0 && !pf && P.tma && uni;
    P.s_uni = s00;
    P.ib_uform = (c.storage == IPCU_STORE_F32 && c.q_scalar == 0 && !pf && uni) ? 1 : 0;
    if (s->lean_ok) {
      if (!salloc(s, &s->ustore[0], (size_t)s->ntiles) || !salloc(s, &s->ustore[1], (size_t)s->ntiles)) {
        free_sim(s);
        return IPCU_ERR_NOMEM;
      }
      P.ustore[0] = s->ustore[0];
      P.ustore[1] = s->ustore[1];
      P.lean = 1;
      // the push form: bounce-back walls on a uniform grid, two-moment MRT
      P.push = (c.wall == IPCU_WALL_BB && c.geometry == IPCU_GEO_UNIFORM && P.mrt == 2) ? 1 : 0;
    }
  }
  {
    std::vector<float> wxv(c.nx), wzv(c.nz);
    for (int i = 0; i < c.nx; i++) wxv[i] = (float)(s->DX[i] / dz);
    for (int l = 0; l < c.nz; l++) wzv[l] = (float)(s->DZ[l] / dz);
    if ((st = supload(s, &s->twx, wxv)) == IPCU_OK) st = supload(s, &s->twz, wzv);
    if (st != IPCU_OK) {
      free_sim(s);
      return st;
    }
  }
  st = f2d::launch_step(P, c.storage, c.q_scalar, c.geometry, s->stream, true);
  if (st != IPCU_OK) {
    free_sim(s);
    return st;
  }
  // initial state, built on the device: f = 0 (p* = 0, u = 0), g = w_k S,
  // u = 0; with 16-bit storage the stored deviations are all zero
  {
    const long long N = s->N;
    std::vector<float> S0f(N, 0.f);
    if (s0)
      for (long long i = 0; i < N; i++) S0f[i] = (float)s0[i];
    const int cb = s->cur;
    cudaError_t e = cudaMemsetAsync(s->f[cb], 0, s->esz * 9 * N, s->stream);
    if (e == cudaSuccess && c.q_scalar) e = cudaMemsetAsync(s->g[cb], 0, s->esz * c.q_scalar * N, s->stream);
    // both buffers' macroscopic planes start at S0, u = 0 (the lean step
    // never writes the S plane)
    for (int i = 0; i < 2 && e == cudaSuccess; i++) {
      e = cudaMemsetAsync(s->mac[i], 0, sizeof(float) * nmac(s) * N, s->stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->mac[i], S0f.data(), sizeof(float) * N, cudaMemcpyHostToDevice, s->stream);
    }
    if (e == cudaSuccess && s->ustore[0]) {
      e = cudaMemsetAsync(s->ustore[cb], 1, (size_t)s->ntiles, s->stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(s->ustore[cb ^ 1], 0, (size_t)s->ntiles, s->stream);
    }
    if (e == cudaSuccess && c.q_scalar && c.storage == IPCU_STORE_F32) {
      Launch L = launch_for(N);
      k_init_g<<<L.grid, L.block, 0, s->stream>>>(s->mac[cb], c.q_scalar, (float *)s->g[cb], N);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);  // S0f is released on return
    st = e == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
  }
  if (st != IPCU_OK) {
    free_sim(s);
    return st;
  }
  *out = s;
  return IPCU_OK;
}

// Memory is returned in stream order; only a simulation that recorded CUDA
// graphs waits for its stream before the graphs are destroyed.
extern "C" void ipcu_sim_destroy(ipcu_sim *sim) {
  if (sim && (sim->graph[0] || sim->graph[1])) cudaStreamSynchronize(sim->stream);
  free_sim(sim);
}

static int launch_one(ipcu_sim *s) {
  f2d::Params P = s->P;
  P.cur = s->cur;
  int st = f2d::launch_step(P, s->cfg.storage, s->cfg.q_scalar, s->cfg.geometry, s->stream);
  if (st == IPCU_OK && s->ibs.size() == 1) {
    ib2d::Job j = *s->ibs[0];
    j.fp = P;
    st = ib2d::launch(j, 0, s->cfg.storage, s->cfg.q_scalar, s->stream);
  } else if (st == IPCU_OK && s->ibs.size() > 1) {
    // one CTA per body, side by side (bodies far enough apart never share a cell)
    st = ib2d::launch_batched(s->d_jobs[s->cur], (int)s->ibs.size(), 0, s->cfg.storage, s->cfg.q_scalar, s->stream);
  }
  if (st == IPCU_OK) {
    s->cur ^= 1;
    s->steps++;
  }
  return st;
}

// Several bodies: the device job lists (one per starting buffer parity) hold
// the simulation's current parameters (refreshed outside any capture).
static int sync_jobs(ipcu_sim *s) {
  const size_t nb = s->ibs.size();
  if (nb < 2 || !s->jobs_dirty) return IPCU_OK;
  std::vector<ib2d::Job> h(nb);
  for (int c = 0; c < 2; c++) {
    if (s->d_jobs[c]) cudaFreeAsync(s->d_jobs[c], s->stream);
    s->d_jobs[c] = nullptr;
    if (!salloc(s, &s->d_jobs[c], sizeof(ib2d::Job) * nb)) return IPCU_ERR_NOMEM;
    for (size_t b = 0; b < nb; b++) {
      h[b] = *s->ibs[b];
      h[b].fp = s->P;
      h[b].fp.cur = c;
    }
    if (cudaMemcpyAsync(s->d_jobs[c], h.data(), sizeof(ib2d::Job) * nb, cudaMemcpyHostToDevice, s->stream) !=
        cudaSuccess)
      return IPCU_ERR_CUDA;
  }
  s->jobs_dirty = false;
  return IPCU_OK;
}

extern "C" int ipcu_sim_step(ipcu_sim *sim, int64_t nsteps) {
  if (!sim || nsteps < 0) return IPCU_ERR_ARG;
  if (int st = sync_jobs(sim)) return st;
  for (int64_t i = 0; i < nsteps; i++) {
    int st = launch_one(sim);
    if (st) return st;
  }
  return IPCU_OK;
}

extern "C" int ipcu_sim_step_graph(ipcu_sim *sim, int64_t nsteps, int32_t chunk) {
  if (!sim || nsteps < 0 || chunk < 2) return IPCU_ERR_ARG;
  if (int st = sync_jobs(sim)) return st;
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

extern "C" int ipcu_stream_create(ipcu_stream_t *out) {
  if (!out) return IPCU_ERR_ARG;
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return IPCU_ERR_CUDA;
  *out = (ipcu_stream_t)s;
  return IPCU_OK;
}

extern "C" int ipcu_stream_destroy(ipcu_stream_t stream) {
  if (!stream) return IPCU_ERR_ARG;
  return cudaStreamDestroy((cudaStream_t)stream) == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Moving immersed boundaries (ibm2d.cu): up to kMaxBodies rigid bodies per
// simulation, as the reference's IB_index loop over bodies (ref:
// function/ibm.cu:367-424), each with its own markers, stencil footprints,
// tile flags and previous orientation. They share the fluid's force density;
// the body updates run side by side, so the bodies must stay apart (no
// contact model, as in the reference): at attach the new body's outline must
// be at least kBodyGap cells from every other body's.
constexpr double kBodyGap = 6.0;  // two 4-point stencils and a cell of motion

static double outline_radius(const double *markers, int n) {
  double r = 0.0;
  for (int l = 0; l < n; l++) r = std::max(r, std::hypot(markers[2 * l], markers[2 * l + 1]));
  return r;
}

static int attach_body(ipcu_sim *s, const ipcu_ib_body2d *bd, const double *markers, const double *dS, int32_t n,
                       bool check_gap) {
  if (!s || !bd || !markers || !dS || n <= 0) return IPCU_ERR_ARG;
  if ((int)s->ibs.size() >= kMaxBodies) return IPCU_ERR_CAPACITY;
  if (n > ib2d::kMaxMarkers) return IPCU_ERR_CAPACITY;
  if (s->cfg.geometry != IPCU_GEO_UNIFORM || s->cfg.scalar_kind == IPCU_SCALAR_PHASE) return IPCU_ERR_UNSUPPORTED;
  if (!(bd->rho_s > 0 && bd->rho_f > 0 && bd->area > 0 && bd->inertia > 0 && bd->semi_a > 0 && bd->semi_b > 0 &&
        bd->iters >= 0 && bd->iters <= 64))
    return IPCU_ERR_ARG;
  for (int i = 0; i < n; i++)
    if (!(dS[i] > 0) || !std::isfinite(markers[2 * i]) || !std::isfinite(markers[2 * i + 1])) return IPCU_ERR_ARG;
  if (check_gap && !s->ibs.empty()) {
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) return IPCU_ERR_CUDA;
    const double r = outline_radius(markers, n);
    for (size_t b = 0; b < s->ibs.size(); b++) {
      ib2d::Body o;
      if (cudaMemcpy(&o, s->ibs[b]->body, sizeof o, cudaMemcpyDeviceToHost) != cudaSuccess) return IPCU_ERR_CUDA;
      const double d = std::hypot(bd->xc - o.X[0], bd->zc - o.X[1]);
      if (d < r + outline_radius(s->ib_X0[b].data(), s->ibs[b]->nl) + kBodyGap * s->cfg.dz) return IPCU_ERR_ARG;
    }
  }
  {
    static bool prepared[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return IPCU_ERR_CUDA;
    if (!prepared[dev]) {
      const int st = ib2d::prepare();
      if (st) return st;
      prepared[dev] = true;
    }
  }
  // recorded graphs hold the parameters without the body: drop them
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  for (int i = 0; i < 2; i++)
    if (s->graph[i]) {
      cudaGraphExecDestroy(s->graph[i]);
      s->graph[i] = nullptr;
    }
  s->graph_chunk = 0;
  ib2d::Job *j = new ib2d::Job();
  std::memset(j, 0, sizeof *j);
  const long long N = s->N;
  const int tx = (s->nx + f2d::kTX - 1) / f2d::kTX, tz = (s->nz + f2d::kTZ - 1) / f2d::kTZ;
  ib2d::Body b0;
  std::memset(&b0, 0, sizeof b0);
  b0.X[0] = bd->xc;
  b0.X[1] = bd->zc;
  b0.U[0] = bd->u;
  b0.U[1] = bd->w;
  b0.th = bd->theta;
  b0.om = bd->omega;
  std::vector<double> X0(markers, markers + 2 * n), dSv(dS, dS + n);
  const size_t tiles = (size_t)tx * tz;
  const int nb = (int)s->ibs.size();  // bodies already attached
  bool ok = salloc(s, &j->body, sizeof(ib2d::Body)) && salloc(s, &j->org, sizeof(int) * 2 * n) &&
            salloc(s, &j->org2, sizeof(int) * 2 * n) && salloc(s, &j->fmark, sizeof(float) * 2 * n);
  double *dX0 = nullptr, *ddS = nullptr;
  ok = ok && salloc(s, &dX0, sizeof(double) * 2 * n) && salloc(s, &ddS, sizeof(double) * n);
  j->X0 = dX0;
  j->dS = ddS;
  s->ibs.push_back(j);  // freed with the simulation from here on
  if (!ok) return IPCU_ERR_NOMEM;
  // the shared force density (first body), and the tile flags grown by one
  // body's slice, the existing slices copied over
  if (!s->ibfext) {
    if (!salloc(s, &s->ibfext, sizeof(float) * 2 * N)) return IPCU_ERR_NOMEM;
    if (cudaMemsetAsync(s->ibfext, 0, sizeof(float) * 2 * N, s->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  }
  uint8_t *flags = nullptr;
  if (!salloc(s, &flags, tiles * (nb + 1))) return IPCU_ERR_NOMEM;
  if (nb > 0 && cudaMemcpyAsync(flags, s->ibflags, tiles * nb, cudaMemcpyDeviceToDevice, s->stream) != cudaSuccess)
    return IPCU_ERR_CUDA;
  if (s->ibflags) cudaFreeAsync(s->ibflags, s->stream);
  s->ibflags = flags;
  for (int b = 0; b <= nb; b++) {
    s->ibs[b]->flag = flags + tiles * b;
    s->ibs[b]->fext = s->ibfext;
  }
  cudaError_t e = cudaMemcpyAsync(j->body, &b0, sizeof b0, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dX0, X0.data(), sizeof(double) * 2 * n, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ddS, dSv.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(j->org, 0, sizeof(int) * 2 * n, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(j->org2, 0, sizeof(int) * 2 * n, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(j->fmark, 0, sizeof(float) * 2 * n, s->stream);
  // the tiles whose halo may reach the initial markers' 4x4 stencils are
  // flagged from the start, as each update flags its successor's footprint:
  // the first fluid step then already stores the velocity the first update
  // reads there (lean flow-only step)
  std::vector<uint8_t> fl((size_t)tx * tz, 0);
  {
    const double ct = std::cos(bd->theta), sn = std::sin(bd->theta), idz = 1.0 / s->cfg.dz;
    auto tile_of = [&](int v, int nmax, int t) { return std::min(std::max(v, 0), nmax - 1) / t; };
    for (int l = 0; l < n; l++) {
      const double X = bd->xc + ct * markers[2 * l] - sn * markers[2 * l + 1];
      const double Z = bd->zc + sn * markers[2 * l] + ct * markers[2 * l + 1];
      const int i0 = (int)std::floor(X * idz - 0.5) - 1, k0 = (int)std::floor(Z * idz - 0.5) - 1;
      const int xa = tile_of(i0 - ib2d::kHalo, s->nx, f2d::kTX), xb = tile_of(i0 + 3 + ib2d::kHalo, s->nx, f2d::kTX);
      const int za = tile_of(k0 - ib2d::kHalo, s->nz, f2d::kTZ), zb = tile_of(k0 + 3 + ib2d::kHalo, s->nz, f2d::kTZ);
      for (int zt : {za, zb})
        for (int xt : {xa, xb}) fl[(size_t)zt * tx + xt] = 1;
    }
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(j->flag, fl.data(), fl.size(), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return IPCU_ERR_CUDA;
  s->ib_cfg.push_back(*bd);
  s->ib_X0.emplace_back(markers, markers + 2 * n);
  s->ib_dS.emplace_back(dS, dS + n);
  j->nl = n;
  j->iters = bd->iters;
  j->m = bd->rho_s * bd->area;
  j->I = bd->rho_s * bd->inertia;
  j->rho_s = bd->rho_s;
  j->rho_f = bd->rho_f;
  j->grav = bd->gravity;
  j->semi_a = bd->semi_a;
  j->semi_b = bd->semi_b;
  j->dz = s->cfg.dz;
  j->dt = s->cfg.dt;
  s->P.fext = s->ibfext;
  s->P.ibflag = s->ibflags;
  s->P.ibtx = tx;
  s->P.ibnb = nb + 1;
  s->jobs_dirty = true;
  return IPCU_OK;
}

extern "C" int ipcu_sim_ib_attach(ipcu_sim *s, const ipcu_ib_body2d *bd, const double *markers, const double *dS,
                                  int32_t n) {
  return attach_body(s, bd, markers, dS, n, true);
}

extern "C" int32_t ipcu_sim_ib_count(const ipcu_sim *s) { return s ? (int32_t)s->ibs.size() : 0; }

extern "C" int ipcu_sim_ib_body_at(ipcu_sim *s, int32_t index, double *out) {
  if (!s || !out || index < 0 || index >= (int)s->ibs.size()) return IPCU_ERR_ARG;
  ib2d::Body b;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess ||
      cudaMemcpy(&b, s->ibs[index]->body, sizeof b, cudaMemcpyDeviceToHost) != cudaSuccess)
    return IPCU_ERR_CUDA;
  const double v[9] = {b.X[0], b.X[1], b.U[0], b.U[1], b.th, b.om, b.Fib[0], b.Fib[1], b.Tib};
  std::memcpy(out, v, sizeof v);
  return IPCU_OK;
}

extern "C" int ipcu_sim_ib_body(ipcu_sim *s, double *out) { return ipcu_sim_ib_body_at(s, 0, out); }

// Markers of a body as the reference's IB_csv writes them (ref:
// function/ibm.cu:3-14): position, velocity and the force each marker put on
// the fluid in the last update, 9 values per marker (x, y, z, u, v, w, Fx,
// Fy, Fz; the body moves in the x-z plane, y = dz/2).
extern "C" int32_t ipcu_sim_ib_markers_at(ipcu_sim *s, int32_t index, double *out, int32_t cap) {
  if (!s || !out || index < 0 || index >= (int)s->ibs.size()) return IPCU_ERR_ARG;
  const ib2d::Job *j = s->ibs[index];
  const int n = j->nl;
  if (cap < n) return IPCU_ERR_CAPACITY;
  ib2d::Body b;
  std::vector<float> fm(2 * (size_t)n);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess ||
      cudaMemcpy(&b, j->body, sizeof b, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(fm.data(), j->fmark, sizeof(float) * fm.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
    return IPCU_ERR_CUDA;
  const double c = std::cos(b.th), sn = std::sin(b.th);
  const std::vector<double> &X0 = s->ib_X0[index];
  for (int l = 0; l < n; l++) {
    const double x0 = X0[2 * l], z0 = X0[2 * l + 1];
    const double rx = c * x0 - sn * z0, rz = sn * x0 + c * z0;
    double *o = out + 9 * (size_t)l;
    o[0] = b.X[0] + rx;
    o[1] = 0.5 * s->cfg.dz;
    o[2] = b.X[1] + rz;
    o[3] = b.U[0] - b.om * rz;
    o[4] = 0.0;
    o[5] = b.U[1] + b.om * rx;
    o[6] = fm[2 * l];
    o[7] = 0.0;
    o[8] = fm[2 * l + 1];
  }
  return n;
}

extern "C" int32_t ipcu_sim_ib_markers(ipcu_sim *s, double *out, int32_t cap) {
  return ipcu_sim_ib_markers_at(s, 0, out, cap);
}

// every body's markers, body after body, in the IB_csv columns
extern "C" int ipcu_sim_write_ib_csv(ipcu_sim *s, const char *path) {
  if (!s || !path || s->ibs.empty()) return IPCU_ERR_ARG;
  std::vector<double> m;
  for (int b = 0; b < (int)s->ibs.size(); b++) {
    const int n = s->ibs[b]->nl;
    std::vector<double> mb(9 * (size_t)n);
    if (const int st = ipcu_sim_ib_markers_at(s, b, mb.data(), n); st < 0) return st;
    m.insert(m.end(), mb.begin(), mb.end());
  }
  FILE *f = fopen(path, "w");
  if (!f) return IPCU_ERR_IO;
  fprintf(f, "x,y,z,velx,vely,velz,ax,ay,az\n");
  for (size_t l = 0; l < m.size() / 9; l++) {
    const double *o = m.data() + 9 * l;
    fprintf(f, "%g,%g,%g,%g,%g,%g,%g,%g,%g\n", o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7], o[8]);
  }
  return fclose(f) == 0 ? IPCU_OK : IPCU_ERR_IO;
}

extern "C" int64_t ipcu_sim_bytes_per_cell(const ipcu_sim *sim) {
  if (!sim) return 0;
  // every stored distribution and the macroscopic planes are read once and written once
  // (the phase field also reads and writes the previous step's phi u, phi w)
  const int old = sim->cfg.scalar_kind == IPCU_SCALAR_PHASE ? 2 : 0;
  // (the lean flow-only step reads and writes the nine populations only)
  if (sim->P.lean) return 2 * (int64_t)sim->esz * 9;
  return 2 * ((int64_t)sim->esz * (9 + sim->cfg.q_scalar) + 4 * (nmac(sim) + old));
}

extern "C" int ipcu_sim_device_state(ipcu_sim *sim, void **f, void **g, float **mac) {
  if (!sim) return IPCU_ERR_ARG;
  if (int st = lean_fill(sim)) return st;
  if (f) *f = sim->f[sim->cur];
  if (g) *g = sim->g[sim->cur];
  if (mac) *mac = sim->mac[sim->cur];
  return IPCU_OK;
}

// The physical state in FP32 on the host: f [9][N], g [q][N], mac [4][N]
// (S, u_x, u_z, p*), converted from / to the storage layout.
struct HostState {
  std::vector<float> f, g, mac;
};

static int state_download(ipcu_sim *s, HostState &h) {
  const long long N = s->N;
  const int q = s->cfg.q_scalar, nm = nmac(s);
  std::vector<unsigned char> fb(s->esz * 9 * N), gb(s->esz * (size_t)q * N);
  h.f.resize(9 * N);
  h.g.resize((size_t)q * N);
  h.mac.assign(4 * N, 0.f);
  if (int st = lean_fill(s)) return st;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess ||
      cudaMemcpy(fb.data(), s->f[s->cur], fb.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
      (q && cudaMemcpy(gb.data(), s->g[s->cur], gb.size(), cudaMemcpyDeviceToHost) != cudaSuccess) ||
      cudaMemcpy(h.mac.data(), s->mac[s->cur], sizeof(float) * nm * N, cudaMemcpyDeviceToHost) != cudaSuccess)
    return IPCU_ERR_CUDA;
  const float ifs = s->P.inv_fscale, igs = s->P.inv_gscale;
  switch (s->cfg.storage) {
    case IPCU_STORE_F32: dec<float>(fb.data(), h.f.data(), 9 * N, 1.f), dec<float>(gb.data(), h.g.data(), q * N, 1.f); break;
    case IPCU_STORE_F16: dec<__half>(fb.data(), h.f.data(), 9 * N, ifs), dec<__half>(gb.data(), h.g.data(), q * N, igs); break;
    default: dec<__nv_bfloat16>(fb.data(), h.f.data(), 9 * N, ifs), dec<__nv_bfloat16>(gb.data(), h.g.data(), q * N, igs);
  }
  const float ic = 1.0f / s->P.c;
  for (long long i = 0; i < N; i++) {
    if (nm == 3) {  // p* in the kernel's float order
      float a = 0.f;
      for (int k = 0; k < 9; k++) a += h.f[k * N + i];
      h.mac[3 * N + i] = a;
      continue;
    }
    // 16-bit storage: deviations plus the equilibrium of the stored moments
    const float S = h.mac[i], uc = h.mac[N + i] * ic, wc = h.mac[2 * N + i] * ic, pr = h.mac[3 * N + i];
    const float u2 = rstore::usq(uc, wc);
    for (int k = 0; k < 9; k++) h.f[k * N + i] += rstore::feq(k, pr, uc, wc, u2);
    for (int k = 0; k < q; k++)
      h.g[k * N + i] += q == 5 ? rstore::geq5(k, S, uc, wc) : rstore::geq9(k, S, uc, wc, u2);
  }
  return IPCU_OK;
}

static int state_upload(ipcu_sim *s, const HostState &h) {
  const long long N = s->N;
  const int q = s->cfg.q_scalar, nm = nmac(s);
  std::vector<float> f = h.f, g = h.g;
  if (nm == 4) {
    const float ic = 1.0f / s->P.c;
    for (long long i = 0; i < N; i++) {
      const float S = h.mac[i], uc = h.mac[N + i] * ic, wc = h.mac[2 * N + i] * ic, pr = h.mac[3 * N + i];
      const float u2 = rstore::usq(uc, wc);
      for (int k = 0; k < 9; k++) f[k * N + i] -= rstore::feq(k, pr, uc, wc, u2);
      for (int k = 0; k < q; k++)
        g[k * N + i] -= q == 5 ? rstore::geq5(k, S, uc, wc) : rstore::geq9(k, S, uc, wc, u2);
    }
  }
  std::vector<unsigned char> fb(s->esz * 9 * N), gb(s->esz * (size_t)q * N);
  const float fs = s->P.fscale, gs = s->P.gscale;
  switch (s->cfg.storage) {
    case IPCU_STORE_F32: enc<float>(f.data(), fb.data(), 9 * N, 1.f), enc<float>(g.data(), gb.data(), q * N, 1.f); break;
    case IPCU_STORE_F16: enc<__half>(f.data(), fb.data(), 9 * N, fs), enc<__half>(g.data(), gb.data(), q * N, gs); break;
    default: enc<__nv_bfloat16>(f.data(), fb.data(), 9 * N, fs), enc<__nv_bfloat16>(g.data(), gb.data(), q * N, gs);
  }
  if (cudaStreamSynchronize(s->stream) != cudaSuccess ||
      cudaMemcpy(s->f[s->cur], fb.data(), fb.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      (q && cudaMemcpy(s->g[s->cur], gb.data(), gb.size(), cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemcpy(s->mac[s->cur], h.mac.data(), sizeof(float) * nm * N, cudaMemcpyHostToDevice) != cudaSuccess)
    return IPCU_ERR_CUDA;
  lean_check_s(s, h.mac.data());
  if (int st = lean_mark_all(s)) return st;
  if (s->obuf[s->cur]) {
    // phase field: the previous step's phi u is taken equal to this state's,
    // so the d(phi u)/dt term starts at zero (the reference driver's
    // phi_old = phi, u_old = u at start-up)
    std::vector<float> o(2 * N);
    for (long long i = 0; i < N; i++) {
      o[i] = h.mac[i] * h.mac[N + i];
      o[N + i] = h.mac[i] * h.mac[2 * N + i];
    }
    if (cudaMemcpy(s->obuf[s->cur], o.data(), sizeof(float) * 2 * N, cudaMemcpyHostToDevice) != cudaSuccess)
      return IPCU_ERR_CUDA;
  }
  return IPCU_OK;
}

extern "C" int ipcu_sim_set_state(ipcu_sim *s, const double *f, const double *g, const double *S, const double *ux,
                                  const double *uz) {
  if (!s) return IPCU_ERR_ARG;
  const long long N = s->N;
  const int q = s->cfg.q_scalar;
  HostState h;
  // fields not given keep their current physical values
  if (!(f && (g || !q) && S && ux && uz)) {
    int st = state_download(s, h);
    if (st) return st;
  } else {
    h.f.resize(9 * N);
    h.g.resize((size_t)q * N);
    h.mac.assign(4 * N, 0.f);
  }
  if (f)
    for (long long i = 0; i < 9 * N; i++) h.f[i] = (float)f[i];
  if (g && q)
    for (long long i = 0; i < q * N; i++) h.g[i] = (float)g[i];
  const double *src[3] = {S, ux, uz};
  for (int a = 0; a < 3; a++)
    if (src[a])
      for (long long i = 0; i < N; i++) h.mac[a * N + i] = (float)src[a][i];
  for (long long i = 0; i < N; i++) {  // p* in the kernel's float order
    float a = 0.f;
    for (int k = 0; k < 9; k++) a += h.f[k * N + i];
    h.mac[3 * N + i] = a;
  }
  return state_upload(s, h);
}

extern "C" int ipcu_sim_get(ipcu_sim *s, const char *field, double *out, int64_t n) {
  if (!s || !field || !out) return IPCU_ERR_ARG;
  const long long N = s->N;
  const int q = s->cfg.q_scalar;
  const std::string fd(field);
  if (fd == "ibfx" || fd == "ibfz") {  // immersed-boundary force density
    if (s->ibs.empty()) return IPCU_ERR_ARG;
    if (n < N) return IPCU_ERR_CAPACITY;
    std::vector<float> m(N);
    if (cudaStreamSynchronize(s->stream) != cudaSuccess ||
        cudaMemcpy(m.data(), s->ibfext + (fd == "ibfz" ? N : 0), sizeof(float) * N, cudaMemcpyDeviceToHost) !=
            cudaSuccess)
      return IPCU_ERR_CUDA;
    for (long long i = 0; i < N; i++) out[i] = m[i];
    return IPCU_OK;
  }
  const long long need = fd == "f" ? 9 * N : (fd == "g" ? (long long)q * N : N);
  if (fd == "g" && !q) return IPCU_ERR_ARG;
  const int slot = fd == "S" ? 0 : (fd == "ux" ? 1 : (fd == "uz" ? 2 : (fd == "rho" ? 0 : (fd == "p" ? 3 : -1))));
  if (slot < 0 && fd != "f" && fd != "g") return IPCU_ERR_ARG;
  if (n < need) return IPCU_ERR_CAPACITY;
  // macroscopic planes straight from the device; p* with FP32 storage and
  // the populations need the whole state
  if (slot >= 0 && (slot < 3 || nmac(s) == 4)) {
    if (int st = lean_fill(s)) return st;
    std::vector<float> m(N);
    if (cudaStreamSynchronize(s->stream) != cudaSuccess ||
        cudaMemcpy(m.data(), s->mac[s->cur] + (long long)slot * N, sizeof(float) * N, cudaMemcpyDeviceToHost) !=
            cudaSuccess)
      return IPCU_ERR_CUDA;
    if (fd == "rho") {
      for (long long i = 0; i < N; i++) out[i] = std::fmaf(m[i], s->P.rho_sal_f, s->P.rho_base);
    } else {
      for (long long i = 0; i < N; i++) out[i] = m[i];
    }
    return IPCU_OK;
  }
  HostState h;
  int st = state_download(s, h);
  if (st) return st;
  if (fd == "f" || fd == "g") {
    const std::vector<float> &v = fd == "f" ? h.f : h.g;
    for (long long i = 0; i < need; i++) out[i] = v[i];
  } else {
    for (long long i = 0; i < N; i++) out[i] = h.mac[slot * N + i];
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
  // area weights (dx dz / dz^2) resident on the device since creation
  const float *f32 = s->cfg.storage == IPCU_STORE_F32 ? (const float *)s->f[s->cur] : nullptr;
  k_totals<<<kTotBlocks, 256, 0, s->stream>>>(f32, s->mac[s->cur], s->twx, s->twz, s->nx, s->nz, s->partials);
  k_totals_final<<<1, 32, 0, s->stream>>>(s->partials, kTotBlocks, s->partials + 2 * kTotBlocks);
  double h[2] = {0, 0};
  cudaError_t e = cudaMemcpyAsync(h, s->partials + 2 * kTotBlocks, sizeof h, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
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
  if (e == cudaSuccess && mac) e = cudaMemcpyAsync(s->mac[s->cur], mac, sizeof(float) * nmac(s) * N, cudaMemcpyHostToDevice, s->stream);
  if (e != cudaSuccess) return IPCU_ERR_CUDA;
  if (mac) {
    lean_check_s(s, mac);  // (reads the host buffer, which the copy only reads too)
    return lean_mark_all(s);
  }
  return IPCU_OK;
}

extern "C" int ipcu_sim_download(ipcu_sim *s, void *f, void *g, float *mac) {
  if (!s) return IPCU_ERR_ARG;
  const long long N = s->N;
  if (mac) {
    if (int st = lean_fill(s)) return st;
  }
  cudaError_t e = cudaSuccess;
  if (f) e = cudaMemcpyAsync(f, s->f[s->cur], s->esz * 9 * N, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess && g && s->cfg.q_scalar)
    e = cudaMemcpyAsync(g, s->g[s->cur], s->esz * s->cfg.q_scalar * N, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess && mac) e = cudaMemcpyAsync(mac, s->mac[s->cur], sizeof(float) * nmac(s) * N, cudaMemcpyDeviceToHost, s->stream);
  return e == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

extern "C" int ipcu_sim_sync(ipcu_sim *s) {
  if (!s) return IPCU_ERR_ARG;
  return cudaStreamSynchronize(s->stream) == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

extern "C" int32_t ipcu_sim_storage_bytes(const ipcu_sim *s) { return s ? (int32_t)s->esz : 0; }

// ---------------------------------------------------------------------------
// Allocation-free totals. Some callers cannot allocate device memory at the
// point where they need the conservation check: hosts that hand all device
// memory to their own pool at start-up, and real-time loops that must not
// hit the driver's allocator. This entry point runs the same two-pass
// reduction as ipcu_sim_totals (with up to 1024 blocks instead of 296, so
// the two agree to rounding, not bit for bit) but keeps its per-block
// partial sums in a file-scope device array instead of allocated scratch.
//
// Limit: kNoAllocBlocks partials of kNoAllocCells cells each, i.e. at most
// 1024 * 16384 = 16,777,216 cells; larger fields are rejected with
// IPCU_ERR_CAPACITY. The array occupies 16 KB on every device that loads
// the library, until the process exits. Every call shares it and it keeps
// the last call's contents: each call writes every partial it reads, so
// nothing needs clearing, but calls whose kernels overlap on the GPU (two
// streams, or two host threads) race on it and must be serialised by the
// caller.
constexpr int kNoAllocBlocks = 1024;
constexpr long long kNoAllocCells = 16384;
static __device__ __align__(256) double g_noalloc_partials[2 * kNoAllocBlocks];

extern "C" int ipcu_totals_noalloc_f32(const float *f, const float *mac, const float *wx, const float *wz, int nx,
                                       int nz, double *out, ipcu_stream_t stream) {
  if (!f || !mac || !wx || !wz || !out || nx < 1 || nz < 1) return IPCU_ERR_ARG;
  const long long N = (long long)nx * nz;
  if (N > (long long)kNoAllocBlocks * kNoAllocCells) return IPCU_ERR_CAPACITY;
  // host code cannot use the array's name as a device address: resolve it
  // once per device (the first call on a device does this set-up, so it
  // should come before any stream capture). The cache is keyed on the
  // current device, which must be the one `stream` belongs to; concurrent
  // first calls write the same address.
  static double *dev_ptr[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return IPCU_ERR_CUDA;
  if (!dev_ptr[dev]) {
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_partials) != cudaSuccess || !ptr) return IPCU_ERR_CUDA;
    dev_ptr[dev] = static_cast<double *>(ptr);
  }
  const int nb = (int)((N + kNoAllocCells - 1) / kNoAllocCells);
  k_totals<<<nb, 256, 0, (cudaStream_t)stream>>>(f, mac, wx, wz, nx, nz, dev_ptr[dev]);
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
// 2: 16-bit storage as equilibrium deviations + p* plane; 3: scalar kind and
// phase-field parameters in the configuration, previous-step phi u planes;
// 4: the moving body (description and device state) after the fluid state
constexpr int32_t kSnapVersion = 5;
template <class T>
bool wr(FILE *f, const T *p, size_t n) { return fwrite(p, sizeof(T), n, f) == n; }
template <class T>
bool rd(FILE *f, T *p, size_t n) { return fread(p, sizeof(T), n, f) == n; }
}  // namespace

extern "C" int64_t ipcu_sim_steps(const ipcu_sim *s) { return s ? s->steps : -1; }

extern "C" int ipcu_sim_save(ipcu_sim *s, const char *path) {
  if (!s || !path) return IPCU_ERR_ARG;
  if (int st = lean_fill(s)) return st;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  const long long N = s->N;
  const int q = s->cfg.q_scalar;
  std::vector<unsigned char> fb(s->esz * 9 * N), gb(s->esz * (size_t)q * N);
  std::vector<float> mb((size_t)nmac(s) * N);
  if (cudaMemcpy(fb.data(), s->f[s->cur], fb.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return IPCU_ERR_CUDA;
  if (q && cudaMemcpy(gb.data(), s->g[s->cur], gb.size(), cudaMemcpyDeviceToHost) != cudaSuccess) return IPCU_ERR_CUDA;
  if (cudaMemcpy(mb.data(), s->mac[s->cur], sizeof(float) * mb.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
    return IPCU_ERR_CUDA;
  std::vector<float> ob(s->obuf[s->cur] ? 2 * N : 0);
  if (!ob.empty() &&
      cudaMemcpy(ob.data(), s->obuf[s->cur], sizeof(float) * ob.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
    return IPCU_ERR_CUDA;
  FILE *f = fopen(path, "wb");
  if (!f) return IPCU_ERR_IO;
  ipcu_sim_config c = s->cfg;
  c.x = c.z = c.wx = c.wz = c.M = c.Minv = c.S = nullptr;
  bool ok = wr(f, kMagic, 8) && wr(f, &kSnapVersion, 1) && wr(f, &c, 1) && wr(f, &s->steps, 1) &&
            wr(f, s->X.data(), s->X.size()) && wr(f, s->Z.data(), s->Z.size()) && wr(f, s->DX.data(), s->DX.size()) &&
            wr(f, s->DZ.data(), s->DZ.size());
  if (ok && c.mrt) ok = wr(f, s->M.data(), 81) && wr(f, s->Minv.data(), 81) && wr(f, s->Srates.data(), 9);
  ok = ok && wr(f, fb.data(), fb.size()) && wr(f, gb.data(), gb.size()) && wr(f, mb.data(), mb.size()) &&
       wr(f, ob.data(), ob.size());
  // the moving bodies: their count, then per body its description and its
  // device state as it stands (rigid-body state, the two previous stencil
  // footprints, its tile flags, the marker forces), then the force density
  // the bodies put on the fluid
  const int32_t nbodies = (int32_t)s->ibs.size();
  ok = ok && wr(f, &nbodies, 1);
  for (int bi = 0; ok && bi < nbodies; bi++) {
    const ib2d::Job &j = *s->ibs[bi];
    const int32_t n = j.nl;
    ib2d::Body b;
    std::vector<int> org(2 * n), org2(2 * n);
    std::vector<float> fm(2 * n);
    std::vector<uint8_t> fl((size_t)s->ntiles);
    ok = cudaMemcpy(&b, j.body, sizeof b, cudaMemcpyDeviceToHost) == cudaSuccess &&
         cudaMemcpy(org.data(), j.org, sizeof(int) * 2 * n, cudaMemcpyDeviceToHost) == cudaSuccess &&
         cudaMemcpy(org2.data(), j.org2, sizeof(int) * 2 * n, cudaMemcpyDeviceToHost) == cudaSuccess &&
         cudaMemcpy(fl.data(), j.flag, fl.size(), cudaMemcpyDeviceToHost) == cudaSuccess &&
         cudaMemcpy(fm.data(), j.fmark, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost) == cudaSuccess;
    ok = ok && wr(f, &s->ib_cfg[bi], 1) && wr(f, &n, 1) && wr(f, s->ib_X0[bi].data(), 2 * (size_t)n) &&
         wr(f, s->ib_dS[bi].data(), (size_t)n) && wr(f, &b, 1) && wr(f, org.data(), org.size()) &&
         wr(f, org2.data(), org2.size()) && wr(f, fl.data(), fl.size()) && wr(f, fm.data(), fm.size());
  }
  if (ok && nbodies > 0) {
    std::vector<float> fe(2 * N);
    ok = cudaMemcpy(fe.data(), s->ibfext, sizeof(float) * 2 * N, cudaMemcpyDeviceToHost) == cudaSuccess &&
         wr(f, fe.data(), fe.size());
  }
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
  bool ok = rd(f, mg, 8) && std::memcmp(mg, kMagic, 8) == 0 && rd(f, &ver, 1) && ver >= 3 && ver <= kSnapVersion &&
            rd(f, &c, 1) &&
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
  std::vector<float> mb((size_t)nmac(s) * N), ob(s->obuf[s->cur] ? 2 * N : 0);
  ok = rd(f, fb.data(), fb.size()) && rd(f, gb.data(), gb.size()) && rd(f, mb.data(), mb.size()) &&
       rd(f, ob.data(), ob.size());
  // versions 4 (one body, the force density inside its block) and 5 (a
  // count of bodies, the force density after them): the moving bodies,
  // re-attached and their device state restored
  struct Saved {
    ipcu_ib_body2d cfg;
    int32_t nl = 0;
    std::vector<double> X0, dS;
    ib2d::Body b;
    std::vector<int> org, org2;
    std::vector<float> fm;
    std::vector<uint8_t> fl;
  };
  int32_t nbodies = 0;
  std::vector<Saved> bodies;
  std::vector<float> fe;
  if (ok && ver >= 4) ok = rd(f, &nbodies, 1) && nbodies >= 0 && nbodies <= kMaxBodies && (ver >= 5 || nbodies <= 1);
  if (ok && nbodies > 0) {
    bodies.resize(nbodies);
    fe.resize(2 * N);
    for (int bi = 0; ok && bi < nbodies; bi++) {
      Saved &B = bodies[bi];
      ok = rd(f, &B.cfg, 1) && rd(f, &B.nl, 1) && B.nl > 0 && B.nl <= ib2d::kMaxMarkers;
      if (!ok) break;
      const size_t nl = (size_t)B.nl;
      B.X0.resize(2 * nl);
      B.dS.resize(nl);
      B.org.resize(2 * nl);
      B.org2.resize(2 * nl);
      B.fm.resize(2 * nl);
      B.fl.resize((size_t)s->ntiles);
      ok = rd(f, B.X0.data(), B.X0.size()) && rd(f, B.dS.data(), B.dS.size()) && rd(f, &B.b, 1) &&
           rd(f, B.org.data(), B.org.size()) && rd(f, B.org2.data(), B.org2.size()) &&
           (ver >= 5 || rd(f, fe.data(), fe.size())) && rd(f, B.fl.data(), B.fl.size()) &&
           rd(f, B.fm.data(), B.fm.size());
    }
    if (ok && ver >= 5) ok = rd(f, fe.data(), fe.size());
  }
  fclose(f);
  if (!ok) {
    ipcu_sim_destroy(s);
    return IPCU_ERR_IO;
  }
  if (cudaMemcpy(s->f[s->cur], fb.data(), fb.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      (q && cudaMemcpy(s->g[s->cur], gb.data(), gb.size(), cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemcpy(s->mac[s->cur], mb.data(), sizeof(float) * mb.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      (!ob.empty() &&
       cudaMemcpy(s->obuf[s->cur], ob.data(), sizeof(float) * ob.size(), cudaMemcpyHostToDevice) != cudaSuccess)) {
    ipcu_sim_destroy(s);
    return IPCU_ERR_CUDA;
  }
  lean_check_s(s, mb.data());
  if (lean_mark_all(s) != IPCU_OK) {
    ipcu_sim_destroy(s);
    return IPCU_ERR_CUDA;
  }
  for (int bi = 0; bi < nbodies; bi++) {
    const Saved &B = bodies[bi];
    st = attach_body(s, &B.cfg, B.X0.data(), B.dS.data(), B.nl, false);
    const ib2d::Job *j = st == IPCU_OK ? s->ibs[bi] : nullptr;
    if (st == IPCU_OK &&
        (cudaMemcpy(j->body, &B.b, sizeof B.b, cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(j->org, B.org.data(), sizeof(int) * B.org.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(j->org2, B.org2.data(), sizeof(int) * B.org2.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(j->flag, B.fl.data(), B.fl.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
         cudaMemcpy(j->fmark, B.fm.data(), sizeof(float) * B.fm.size(), cudaMemcpyHostToDevice) != cudaSuccess))
      st = IPCU_ERR_CUDA;
    if (st != IPCU_OK) {
      ipcu_sim_destroy(s);
      return st;
    }
  }
  if (nbodies > 0 &&
      cudaMemcpy(s->ibfext, fe.data(), sizeof(float) * fe.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    ipcu_sim_destroy(s);
    return IPCU_ERR_CUDA;
  }
  s->steps = steps;
  *out = s;
  return IPCU_OK;
}

extern "C" int ipcu_sim_set_lean(ipcu_sim *s, int enable) {
  if (!s) return IPCU_ERR_ARG;
  if (enable && !s->lean_ok) return IPCU_ERR_UNSUPPORTED;
  if ((s->P.lean != 0) == (enable != 0)) return IPCU_OK;
  if (!enable) {
    if (int st = lean_fill(s)) return st;  // the planes of the current buffer made complete
    s->P.lean = 0;
  } else {
    s->P.lean = 1;  // after full steps every plane of the current buffer is valid
    if (int st = lean_mark_all(s)) return st;
  }
  drop_graphs(s);
  return IPCU_OK;
}

extern "C" int ipcu_sim_lean(const ipcu_sim *s) { return s && s->P.lean ? 1 : 0; }

extern "C" int ipcu_sim_set_push(ipcu_sim *s, int enable) {
  if (!s) return IPCU_ERR_ARG;
  const bool ok = s->lean_ok && s->cfg.wall == IPCU_WALL_BB && s->cfg.geometry == IPCU_GEO_UNIFORM && s->P.mrt == 2;
  if (enable && !ok) return IPCU_ERR_UNSUPPORTED;
  if ((s->P.push != 0) == (enable != 0)) return IPCU_OK;
  if (!enable && s->P.lean) {
    // the tile form reads a tile's velocity planes wherever ustore is set:
    // complete them and mark every tile
    if (int st = lean_fill(s)) return st;
    if (int st = lean_mark_all(s)) return st;
  }
  s->P.push = enable ? 1 : 0;
  drop_graphs(s);
  return IPCU_OK;
}

extern "C" int ipcu_sim_push(const ipcu_sim *s) { return s && s->P.lean && s->P.push ? 1 : 0; }

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
  cudaEvent_t done = nullptr;  // recorded after each enqueue; the simulations' streams wait on it
  cudaEvent_t mark[4] = {nullptr, nullptr, nullptr, nullptr};  // ring of progress marks
  int next_mark = 0;
  f2d::Params *d_params = nullptr;
  f2d::WorkItem *d_work = nullptr;
  ib2d::Job *d_jobs = nullptr;  // coupled bodies of the listed simulations
  size_t cap_params = 0, cap_work = 0, cap_jobs = 0;
  int sms = 148;
  // CTAs per SM of the batched grid, per kernel class (storage, scalar
  // lattice, geometry, scalar kind); f2d::kMinBlocks where not set
  std::map<std::array<int, 4>, int> ctas;
  // graph mode: each enqueue's launches are captured into one CUDA graph and
  // replayed; the executable graph is updated in place while the launch
  // sequence keeps its shape, and re-instantiated when it changes. Replaced
  // executables are released once the launch that used them has completed.
  bool use_graph = false;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t exec_done = nullptr;  // recorded after the last launch of `exec`
  std::vector<std::pair<cudaGraphExec_t, cudaEvent_t>> retired;
  long long graph_updates = 0, graph_instantiations = 0;
};

extern "C" int ipcu_batch_create(ipcu_stream_t stream, ipcu_batch **out) {
  if (!out) return IPCU_ERR_ARG;
  ipcu_batch *b = new ipcu_batch();
  b->stream = (cudaStream_t)stream;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  b->sms = sms;
  bool ok = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; i < 4 && ok; i++) ok = cudaEventCreateWithFlags(&b->mark[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    ipcu_batch_destroy(b);
    return IPCU_ERR_CUDA;
  }
  *out = b;
  return IPCU_OK;
}

extern "C" void ipcu_batch_destroy(ipcu_batch *b) {
  if (!b) return;
  cudaStreamSynchronize(b->stream);
  cudaFree(b->d_params);
  cudaFree(b->d_work);
  cudaFree(b->d_jobs);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->exec_done) cudaEventDestroy(b->exec_done);
  for (auto &r : b->retired) {
    cudaGraphExecDestroy(r.first);
    cudaEventDestroy(r.second);
  }
  if (b->done) cudaEventDestroy(b->done);
  for (int i = 0; i < 4; i++)
    if (b->mark[i]) cudaEventDestroy(b->mark[i]);
  delete b;
}

// Enqueues batched steps on the batch stream -- simulation i advances by
// nsteps[i] -- and orders every listed simulation's own stream after them
// (event wait), so that later work on a simulation -- reads, more steps,
// destruction -- sees the results.
//
// Within each kernel class the simulations are laid out by decreasing step
// count, so the ones still stepping at step k own a prefix of the class's
// work list (and of its bodies): one launch per class per step, its grid the
// prefix, however ragged the counts. Classes with bodies go first, each
// fluid launch right after a batch of body updates is a programmatic
// dependent of it (only the tiles the bodies flagged wait), and a class
// without bodies follows one with bodies, so their fluid step runs beside
// the body updates.
// Graph mode: capture `launches` on the batch stream, bring the executable
// graph up to date (in place when the captured sequence has the shape of the
// previous one) and replay it.
template <class F>
static int batch_graph(ipcu_batch *b, F &&launches) {
  // release replaced executables whose last launch has completed
  for (size_t i = 0; i < b->retired.size();) {
    if (cudaEventQuery(b->retired[i].second) == cudaSuccess) {
      cudaGraphExecDestroy(b->retired[i].first);
      cudaEventDestroy(b->retired[i].second);
      b->retired.erase(b->retired.begin() + i);
    } else {
      cudaGetLastError();  // cudaErrorNotReady is not an error here
      i++;
    }
  }
  if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return IPCU_ERR_CUDA;
  const int st = launches();
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
  if (st != IPCU_OK || e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return st != IPCU_OK ? st : IPCU_ERR_CUDA;
  }
  bool ok = false;
  if (b->exec) {
    cudaGraphExecUpdateResultInfo info;
    ok = cudaGraphExecUpdate(b->exec, graph, &info) == cudaSuccess;
    if (ok) {
      b->graph_updates++;
    } else {
      cudaGetLastError();
      b->retired.emplace_back(b->exec, b->exec_done);  // in flight until exec_done completes
      b->exec = nullptr;
      b->exec_done = nullptr;
    }
  }
  if (!ok) {
    ok = cudaGraphInstantiate(&b->exec, graph, 0) == cudaSuccess &&
         cudaEventCreateWithFlags(&b->exec_done, cudaEventDisableTiming) == cudaSuccess;
    b->graph_instantiations++;
  }
  cudaGraphDestroy(graph);
  if (!ok || cudaGraphLaunch(b->exec, b->stream) != cudaSuccess ||
      cudaEventRecord(b->exec_done, b->stream) != cudaSuccess)
    return IPCU_ERR_CUDA;
  return IPCU_OK;
}

static int batch_enqueue(ipcu_batch *b, ipcu_sim *const *sims, int n, const int64_t *nsteps) {
  if (!b || (n > 0 && (!sims || !nsteps))) return IPCU_ERR_ARG;
  std::vector<int> order;
  int64_t kmax = 0;
  for (int i = 0; i < n; i++) {
    if (!sims[i] || nsteps[i] < 0) return IPCU_ERR_ARG;
    if (nsteps[i] == 0) continue;
    order.push_back(i);
    kmax = std::max(kmax, nsteps[i]);
  }
  if (order.empty()) return IPCU_OK;
  for (int i : order) {
    // the batched kernel reads and writes every plane: a simulation that
    // ran lean steps completes its velocity planes first
    if (sims[i]->P.lean) {
      if (int st = lean_fill(sims[i])) return st;
    }
    // the batch stream waits (on the device) for the simulation's own work
    if (cudaEventRecord(sims[i]->ready, sims[i]->stream) != cudaSuccess ||
        cudaStreamWaitEvent(b->stream, sims[i]->ready, 0) != cudaSuccess)
      return IPCU_ERR_CUDA;
  }
  // group by (bodies first, kernel class), then by decreasing step count
  auto key = [&](int a) {
    const ipcu_sim_config &A = sims[a]->cfg;
    return std::make_tuple(sims[a]->ibs.empty(), A.storage, A.q_scalar, A.geometry, A.scalar_kind, sims[a]->P.tma);
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
    const auto ka = key(a), kc = key(c);
    return ka < kc || (ka == kc && nsteps[a] > nsteps[c]);
  });
  const int m = (int)order.size();
  std::vector<f2d::Params> hp(m);
  std::vector<f2d::WorkItem> hw;
  std::vector<ib2d::Job> hj;
  // per class: its simulations' end offsets in the work and body lists,
  // with their step counts (decreasing)
  struct Member { int64_t steps; int w1, j1; };
  struct Group { int storage, qs, geo, pf, tma, w0, j0; std::vector<Member> mem; size_t live; };
  std::vector<Group> groups;
  for (int oi = 0; oi < m; oi++) {
    ipcu_sim *s = sims[order[oi]];
    hp[oi] = s->P;
    hp[oi].cur = s->cur;
    hp[oi].lean = 0;
    const ipcu_sim_config &c = s->cfg;
    if (oi == 0 || key(order[oi]) != key(order[oi - 1]))
      groups.push_back({c.storage, c.q_scalar, c.geometry, c.scalar_kind, s->P.tma, (int)hw.size(), (int)hj.size(),
                        {}, 0});
    const int tx = (s->nx + f2d::kTX - 1) / f2d::kTX, tz = (s->nz + f2d::kTZ - 1) / f2d::kTZ;
    for (int z = 0; z < tz; z++)
      for (int x = 0; x < tx; x++) hw.push_back({oi, x, z, 0});
    for (ib2d::Job *j : s->ibs) {
      hj.push_back(*j);
      hj.back().fp = hp[oi];
    }
    Group &g = groups.back();
    g.mem.push_back({nsteps[order[oi]], (int)hw.size(), (int)hj.size()});
    g.live = g.mem.size();
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
  if (hj.size() > b->cap_jobs) {
    cudaFree(b->d_jobs);
    if (cudaMalloc((void **)&b->d_jobs, sizeof(ib2d::Job) * hj.size()) != cudaSuccess) return IPCU_ERR_NOMEM;
    b->cap_jobs = hj.size();
  }
  if ((!hj.empty() &&
       cudaMemcpyAsync(b->d_jobs, hj.data(), sizeof(ib2d::Job) * hj.size(), cudaMemcpyHostToDevice, b->stream) !=
           cudaSuccess) ||
      cudaMemcpyAsync(b->d_params, hp.data(), sizeof(f2d::Params) * hp.size(), cudaMemcpyHostToDevice, b->stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(b->d_work, hw.data(), sizeof(f2d::WorkItem) * hw.size(), cudaMemcpyHostToDevice, b->stream) !=
          cudaSuccess)
    return IPCU_ERR_CUDA;
  for (const Group &g : groups) {
    int st = f2d::launch_batched(nullptr, nullptr, 0, 0, g.storage, g.qs, g.geo, g.pf, 0, b->stream, true, g.tma);
    if (st) return st;
  }
  auto launches = [&]() -> int {
    bool after_bodies = false;  // the last launch on the stream is a batch of body updates
    for (int64_t k = 0; k < kmax; k++) {
      for (Group &g : groups) {
        while (g.live > 0 && g.mem[g.live - 1].steps <= k) g.live--;  // members done after k steps
        if (g.live == 0) continue;
        const int nw = g.mem[g.live - 1].w1 - g.w0, nj = g.mem[g.live - 1].j1 - g.j0;
        const auto it = b->ctas.find({g.storage, g.qs, g.geo, g.pf});
        const int grid = std::min(nw, b->sms * (it == b->ctas.end() ? f2d::kMinBlocks : it->second));
        int st = f2d::launch_batched(b->d_params, b->d_work + g.w0, nw, (int)(k & 1), g.storage, g.qs, g.geo, g.pf,
                                     grid, b->stream, false, g.tma != 0, after_bodies);
        after_bodies = false;
        if (!st && nj > 0) {
          st = ib2d::launch_batched(b->d_jobs + g.j0, nj, (int)(k & 1), g.storage, g.qs, b->stream);
          after_bodies = true;
        }
        if (st) return st;
      }
    }
    return IPCU_OK;
  };
  if (!b->use_graph) {
    if (int st = launches()) return st;
  } else if (int st = batch_graph(b, launches)) {
    return st;
  }
  if (cudaEventRecord(b->done, b->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  for (int i : order) {
    if (cudaStreamWaitEvent(sims[i]->stream, b->done, 0) != cudaSuccess) return IPCU_ERR_CUDA;
    sims[i]->cur ^= (int)(nsteps[i] & 1);
    sims[i]->steps += nsteps[i];
    // the batched kernel wrote every velocity plane: the lean step's flags
    // of the new current buffer all hold
    if (int st = lean_mark_all(sims[i])) return st;
  }
  return IPCU_OK;
}

static int batch_enqueue_all(ipcu_batch *b, ipcu_sim *const *sims, int n, int64_t nsteps) {
  if (!b || n < 0 || (n > 0 && !sims) || nsteps < 0) return IPCU_ERR_ARG;
  const std::vector<int64_t> each((size_t)n, nsteps);
  return batch_enqueue(b, sims, n, each.data());
}

extern "C" int ipcu_batch_step(ipcu_batch *b, ipcu_sim *const *sims, int n, int64_t nsteps) {
  const int st = batch_enqueue_all(b, sims, n, nsteps);
  if (st != IPCU_OK || n == 0 || nsteps == 0) return st;
  return cudaStreamSynchronize(b->stream) == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

extern "C" int ipcu_batch_launch(ipcu_batch *b, ipcu_sim *const *sims, int n, int64_t nsteps) {
  return batch_enqueue_all(b, sims, n, nsteps);
}

extern "C" int ipcu_batch_launch_each(ipcu_batch *b, ipcu_sim *const *sims, const int64_t *nsteps, int n) {
  if (n < 0) return IPCU_ERR_ARG;
  return batch_enqueue(b, sims, n, nsteps);
}

extern "C" int ipcu_batch_set_graph(ipcu_batch *b, int enable) {
  if (!b) return IPCU_ERR_ARG;
  if (enable && b->stream == nullptr) return IPCU_ERR_UNSUPPORTED;  // the legacy stream cannot be captured
  b->use_graph = enable != 0;
  return IPCU_OK;
}

extern "C" int ipcu_batch_set_ctas(ipcu_batch *b, int storage, int q_scalar, int geometry, int scalar_kind,
                                   int ctas_per_sm) {
  if (!b || ctas_per_sm < 0 || ctas_per_sm > 32) return IPCU_ERR_ARG;
  const std::array<int, 4> key = {storage, q_scalar, geometry, scalar_kind};
  if (ctas_per_sm == 0) b->ctas.erase(key);
  else b->ctas[key] = ctas_per_sm;
  return IPCU_OK;
}

extern "C" int ipcu_batch_graph_stats(const ipcu_batch *b, int64_t *updates, int64_t *instantiations) {
  if (!b || !updates || !instantiations) return IPCU_ERR_ARG;
  *updates = b->graph_updates;
  *instantiations = b->graph_instantiations;
  return IPCU_OK;
}

extern "C" int ipcu_batch_mark(ipcu_batch *b) {
  if (!b) return IPCU_ERR_ARG;
  const int m = b->next_mark;
  if (cudaEventRecord(b->mark[m], b->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  b->next_mark = (m + 1) % 4;
  return m;
}

extern "C" int ipcu_batch_wait_mark(ipcu_batch *b, int mark) {
  if (!b || mark < 0 || mark >= 4) return IPCU_ERR_ARG;
  return cudaEventSynchronize(b->mark[mark]) == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

extern "C" int ipcu_batch_sync(ipcu_batch *b) {
  if (!b) return IPCU_ERR_ARG;
  return cudaStreamSynchronize(b->stream) == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

// per body: tile flags, markers (X0, dS, two footprints, marker forces),
// rigid-body state, and its entry in the two device job lists
static long long ib_bytes(const ipcu_sim *s) {
  long long t = 0;
  for (const ib2d::Job *j : s->ibs)
    t += (long long)s->ntiles + 40LL * j->nl + (long long)sizeof(ib2d::Body) +
         (s->ibs.size() > 1 ? 2LL * (long long)sizeof(ib2d::Job) : 0);
  return t;
}

extern "C" int64_t ipcu_sim_device_bytes(const ipcu_sim *s) {
  if (!s) return 0;
  const long long N = s->N;
  return 2 * ((long long)s->esz * (9 + std::max(s->cfg.q_scalar, 1)) * N + 4LL * (nmac(s) + (s->cfg.scalar_kind == IPCU_SCALAR_PHASE ? 2 : 0)) * N) +
         4LL * (3 * (s->nx + s->nz) + 2 * 5 * std::max(s->nx, s->nz)) + 2048 +
         (s->cfg.scalar_kind == IPCU_SCALAR_PHASE ? 4LL * (s->nx + s->nz) : 0) +  // 1/dx^2, 1/dz^2
         (s->ibs.empty() ? 0 : 8LL * N) + ib_bytes(s);  // immersed bodies: force density, per body below
}
