// 3-D structured solver object (ipcu_sim3d_*): device-resident state (FP32,
// or 16-bit deviations from a per-cell reference, store3d.cuh), stepping
// (direct or CUDA-graph replay), field I/O.
#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "axis_tables.hpp"
#include "d3q19.cuh"
#include "fused3d.cuh"
#include "fused3s.cuh"
#include "ibm3d.cuh"
#include "ipcu_common.cuh"
#include "store3d.cuh"

using namespace ipcu;

struct ipcu_sim3d {
  ipcu_sim3d_config cfg;
  long long N;
  cudaStream_t stream;
  // populations in the storage type, FP32 force planes, and with 16-bit
  // storage the reference planes [5][N]
  void *f[2] = {nullptr, nullptr}, *g[2] = {nullptr, nullptr}, *r[2] = {nullptr, nullptr};
  float *F[2] = {nullptr, nullptr};
  int store = IPCU_STORE_F32;
  float scale = 1.0f, inv_scale = 1.0f;
  unsigned *status = nullptr;
  int cur = 0;
  f3d::Params3 P;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // two steps, per starting buffer
  long long steps = 0;
  // stretched x and y axes (ns 3 or 5; 0: the uniform box kernel): the
  // step kernel's parameters and the axes' device tables
  int ns = 0;
  f3s::Params3S PS;
  float *tab = nullptr;
  std::vector<double> X, DX, Y, DY;
  // an attached sphere (ibm3d.cu): its job with every device array, one
  // block of memory for them, and the force density on the fluid
  ib3d::Job *ib = nullptr;
  void *ib_mem = nullptr;
};

namespace {

constexpr double w7d(int k) { return k == 0 ? 0.25 : 0.125; }
constexpr int E19[19][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {-1, 0, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1},
                            {1, 1, 0}, {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, 0, 1}, {1, 0, -1}, {-1, 0, 1},
                            {-1, 0, -1}, {0, 1, 1}, {0, 1, -1}, {0, -1, 1}, {0, -1, -1}};

// Device memory is stream-ordered on the simulation's stream (a server
// creating and releasing simulations never synchronises the device): freed
// after the work queued on that stream, allocated before it.
template <class V>
bool salloc3(ipcu_sim3d *s, V **p, size_t bytes) {
  return cudaMallocAsync((void **)p, bytes, s->stream) == cudaSuccess;
}

void free3(ipcu_sim3d *s) {
  if (!s) return;
  auto fr = [&](void *p) {
    if (p) cudaFreeAsync(p, s->stream);
  };
  for (int i = 0; i < 2; i++) {
    if (s->graph[i]) cudaGraphExecDestroy(s->graph[i]);
    fr(s->f[i]);
    fr(s->g[i]);
    fr(s->r[i]);
    fr(s->F[i]);
  }
  fr(s->status);
  fr(s->tab);
  fr(s->ib_mem);
  delete s->ib;
  delete s;
}

f3d::Params3 params_for(const ipcu_sim3d *s, int cur) {
  f3d::Params3 P = s->P;
  P.f_in = static_cast<const float *>(s->f[cur]);
  P.g_in = static_cast<const float *>(s->g[cur]);
  P.F_in = s->F[cur];
  P.f_out = static_cast<float *>(s->f[cur ^ 1]);
  P.g_out = static_cast<float *>(s->g[cur ^ 1]);
  P.F_out = s->F[cur ^ 1];
  return P;
}

// one step reading buffer `cur`: the uniform box kernel or the stretched one
int launch_one(const ipcu_sim3d *s, int cur, cudaStream_t st) {
  if (!s->ns) return f3d::launch3d(params_for(s, cur), st);
  f3s::Params3S P = s->PS;
  P.f_in = s->f[cur];
  P.g_in = s->g[cur];
  P.F_in = s->F[cur];
  P.f_out = s->f[cur ^ 1];
  P.g_out = s->g[cur ^ 1];
  P.F_out = s->F[cur ^ 1];
  P.r_in = s->r[cur];
  P.r_out = s->r[cur ^ 1];
  return f3s::launch3s(P, s->ns, st);
}

// fluid step, then the sphere's update on the state it wrote
int launch_step(const ipcu_sim3d *s, int cur, cudaStream_t st) {
  int e = launch_one(s, cur, st);
  if (e == IPCU_OK && s->ib) {
    ib3d::Job j = *s->ib;
    j.f = s->f[cur ^ 1];
    j.g = s->g[cur ^ 1];
    j.r = s->r[cur ^ 1];
    j.F = s->F[cur ^ 1];
    e = ib3d::launch(j, st);
  }
  return e;
}

// ---- host side of the storage formats (store3d.cuh): the FP32 state of
// buffer `cur` written into / read from the simulation's storage layout
template <class T>
void encode3(const ipcu_sim3d *s, const float *f, const float *g, const float *F, std::vector<T> &fh,
             std::vector<T> &gh, std::vector<T> &rh) {
  const long long N = s->N;
  const float c = s->P.c, ic = 1.0f / c;
  fh.resize(19 * N);
  gh.resize(7 * N);
  rh.resize(5 * N);
  for (long long i = 0; i < N; i++) {
    // the reference: the cell's pressure, u/c and salinity
    float pr = 0.f, j[3] = {0.f, 0.f, 0.f}, S = 0.f;
    for (int k = 0; k < 19; k++) {
      const float v = f[k * N + i];
      pr += v;
      for (int a = 0; a < 3; a++)
        if (E19[k][a]) j[a] += E19[k][a] * v;
    }
    for (int k = 0; k < 7; k++) S += g[k * N + i];
    const float h = s->P.hdt / std::fmaf(S, s->P.rsal, s->P.rho0);
    const float ref[5] = {pr, std::fmaf(c, j[0], F[i] * h) * ic, std::fmaf(c, j[1], F[N + i] * h) * ic,
                          std::fmaf(c, j[2], F[2 * N + i] * h) * ic, S};
    for (int a = 0; a < 5; a++) rh[a * N + i] = s3::from_f<T>(ref[a]);
    const s3::Ref R = s3::ref_of(rh.data(), i, N);
    for (int k = 0; k < 19; k++) fh[k * N + i] = s3::enc<T>(f[k * N + i], s->scale, s3::rf(k, R));
    for (int k = 0; k < 7; k++) gh[k * N + i] = s3::enc<T>(g[k * N + i], s->scale, s3::rg(k, R));
  }
}

template <class T>
int put16(ipcu_sim3d *s, const float *f, const float *g, const float *F) {
  std::vector<T> fh, gh, rh;
  encode3(s, f, g, F, fh, gh, rh);
  const int b = s->cur;
  const bool ok = cudaMemcpy(s->f[b], fh.data(), 2 * fh.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(s->g[b], gh.data(), 2 * gh.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(s->r[b], rh.data(), 2 * rh.size(), cudaMemcpyHostToDevice) == cudaSuccess;
  return ok ? IPCU_OK : IPCU_ERR_CUDA;
}

template <class T>
int get16(ipcu_sim3d *s, float *f, float *g) {
  const long long N = s->N;
  std::vector<T> fh(19 * N), gh(7 * N), rh(5 * N);
  const int b = s->cur;
  if (cudaMemcpy(fh.data(), s->f[b], 2 * fh.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(gh.data(), s->g[b], 2 * gh.size(), cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(rh.data(), s->r[b], 2 * rh.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
    return IPCU_ERR_CUDA;
  float fo[19], go[7];
  for (long long i = 0; i < N; i++) {
    s3::load_cell<T>(fh.data(), gh.data(), rh.data(), i, N, s->inv_scale, fo, go);
    for (int k = 0; k < 19; k++) f[k * N + i] = fo[k];
    for (int k = 0; k < 7; k++) g[k * N + i] = go[k];
  }
  return IPCU_OK;
}

// FP32 state (f [19][N], g [7][N], F [3][N]) into buffer `cur`; synchronises
int put_state(ipcu_sim3d *s, const float *f, const float *g, const float *F) {
  const long long N = s->N;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess ||
      cudaMemcpy(s->F[s->cur], F, sizeof(float) * 3 * N, cudaMemcpyHostToDevice) != cudaSuccess)
    return IPCU_ERR_CUDA;
  if (s->store == IPCU_STORE_F16) return put16<__half>(s, f, g, F);
  if (s->store == IPCU_STORE_BF16) return put16<__nv_bfloat16>(s, f, g, F);
  const bool ok = cudaMemcpy(s->f[s->cur], f, sizeof(float) * 19 * N, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(s->g[s->cur], g, sizeof(float) * 7 * N, cudaMemcpyHostToDevice) == cudaSuccess;
  return ok ? IPCU_OK : IPCU_ERR_CUDA;
}

// buffer `cur` as FP32 arrays; synchronises
int get_state(ipcu_sim3d *s, std::vector<float> &f, std::vector<float> &g, std::vector<float> &F) {
  const long long N = s->N;
  f.resize(19 * N);
  g.resize(7 * N);
  F.resize(3 * N);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess ||
      cudaMemcpy(F.data(), s->F[s->cur], sizeof(float) * F.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
    return IPCU_ERR_CUDA;
  if (s->store == IPCU_STORE_F16) return get16<__half>(s, f.data(), g.data());
  if (s->store == IPCU_STORE_BF16) return get16<__nv_bfloat16>(s, f.data(), g.data());
  const bool ok = cudaMemcpy(f.data(), s->f[s->cur], sizeof(float) * f.size(), cudaMemcpyDeviceToHost) == cudaSuccess &&
                  cudaMemcpy(g.data(), s->g[s->cur], sizeof(float) * g.size(), cudaMemcpyDeviceToHost) == cudaSuccess;
  return ok ? IPCU_OK : IPCU_ERR_CUDA;
}

}  // namespace

extern "C" int ipcu_sim3d_create(const ipcu_sim3d_config *cfg, const double *s0, ipcu_stream_t stream,
                                 ipcu_sim3d **out) {
  return ipcu_sim3d_create_stretched(cfg, nullptr, s0, stream, out);
}

extern "C" int ipcu_sim3d_create_stretched(const ipcu_sim3d_config *cfg, const ipcu_sim3d_axes *axes,
                                           const double *s0, ipcu_stream_t stream, ipcu_sim3d **out) {
  if (!cfg || !out) return IPCU_ERR_ARG;
  *out = nullptr;
  const ipcu_sim3d_config &c = *cfg;
  if (c.nx < 1 || c.ny < 1 || c.nz < 1 || !(c.dz > 0) || !(c.dt > 0) || c.tau <= 0.5 || c.taus <= 0.5)
    return IPCU_ERR_ARG;
  const bool stretched = axes && (axes->x || axes->wx || axes->y || axes->wy);
  if (stretched && axes->ns != 3 && axes->ns != 5) return IPCU_ERR_ARG;
  if (c.storage != IPCU_STORE_F32 && c.storage != IPCU_STORE_F16 && c.storage != IPCU_STORE_BF16) return IPCU_ERR_ARG;
  // 16-bit storage runs the flux-form kernel on every box (stencil 3 unless
  // the axes name one)
  const bool flux = stretched || c.storage != IPCU_STORE_F32;
  const int ns = stretched ? axes->ns : (axes && axes->ns == 5 ? 5 : 3);
  std::vector<double> X(c.nx), DX(c.nx), Y(c.ny), DY(c.ny);
  for (int i = 0; i < c.nx; i++) {
    X[i] = stretched && axes->x ? axes->x[i] : (i + 0.5) * c.dz;
    DX[i] = stretched && axes->wx ? axes->wx[i] : c.dz;
    if (DX[i] < c.dz * (1 - 1e-9)) return IPCU_ERR_ARG;  // CFL <= 1 on the interpolated axes
  }
  for (int j = 0; j < c.ny; j++) {
    Y[j] = stretched && axes->y ? axes->y[j] : (j + 0.5) * c.dz;
    DY[j] = stretched && axes->wy ? axes->wy[j] : c.dz;
    if (DY[j] < c.dz * (1 - 1e-9)) return IPCU_ERR_ARG;
  }
  ipcu_sim3d *s = new ipcu_sim3d();
  s->X = X;
  s->DX = DX;
  s->Y = Y;
  s->DY = DY;
  s->cfg = c;
  s->N = (long long)c.nx * c.ny * c.nz;
  s->stream = (cudaStream_t)stream;
  ensure_tables();
  const long long N = s->N;
  s->store = c.storage;
  // FP16 scales the deviations by 2^12 (they span about 1e-9 .. 1e-1 in
  // lattice units: FP16's normal range from 1.5e-8 up to 16); BF16 has
  // FP32's range
  s->scale = c.storage == IPCU_STORE_F16 ? 4096.0f : 1.0f;
  s->inv_scale = 1.0f / s->scale;
  const size_t es = c.storage == IPCU_STORE_F32 ? sizeof(float) : 2;
  for (int i = 0; i < 2; i++)
    if (!salloc3(s, &s->f[i], es * 19 * N) || !salloc3(s, &s->g[i], es * 7 * N) ||
        !salloc3(s, &s->F[i], sizeof(float) * 3 * N) ||
        (c.storage != IPCU_STORE_F32 && !salloc3(s, &s->r[i], 2 * 5 * N))) {
      free3(s);
      return IPCU_ERR_NOMEM;
    }
  // the set-up below uses synchronous copies: the allocations land first
  if (!salloc3(s, &s->status, sizeof(unsigned)) || cudaStreamSynchronize(s->stream) != cudaSuccess) {
    free3(s);
    return IPCU_ERR_NOMEM;
  }
  f3d::Params3 &P = s->P;
  std::memset(&P, 0, sizeof P);
  P.nx = c.nx;
  P.ny = c.ny;
  P.nz = c.nz;
  // z cells per CTA: enough CTAs for several waves on 148 SMs (chunks of
  // 12 at 160 x 160 x 640: measured 2 % faster than 24 and 8 % faster than
  // 48, the two ring planes formed per chunk notwithstanding)
  const long long cols = (long long)((c.nx + 31) / 32) * ((c.ny + 7) / 8);
  P.zchunk = (int)std::max(4LL, std::min<long long>(64, (long long)c.nz * cols / (148LL * 3 * 12)));
  const double cl = c.dz / c.dt;
  P.c = (float)cl;
  P.dt = (float)c.dt;
  P.itau = (float)(1.0 / c.tau);
  P.omg_s = (float)(1.0 - 1.0 / c.taus);
  P.fk3 = (float)(3.0 * c.dt / cl);
  P.hdt = (float)(0.5 * c.dt);
  P.rho0 = (float)c.rho0;
  P.rsal = (float)c.rho_sal;
  P.gb = (float)c.g_bouss;
  // clamped central differences: 1/(x_{i+1} - x_{i-1} + dz/1000), the ghost
  // carrying its owner's position at a wall (ref: function/collision.cu:82-85)
  const float reg = (float)c.dz / 1000.0f;
  P.gi_in = 1.0f / (2.0f * (float)c.dz + reg);
  P.gi_wall = 1.0f / ((float)c.dz + reg);
  P.mrt = c.mrt ? 1 : 0;
  P.status = s->status;
  if (flux) {
    // flux-form and gradient tables of both axes, one device block
    s->ns = ns;
    std::vector<float> wx, six, sox, wcx, wy, siy, soy, wcy;
    axis_tables(X, DX, c.dz, s->ns, wx, six, sox, wcx);
    axis_tables(Y, DY, c.dz, s->ns, wy, siy, soy, wcy);
    const std::vector<float> gx = grad_inv(X, c.dz), gy = grad_inv(Y, c.dz);
    const std::vector<float> *parts[10] = {&wx, &six, &sox, &wcx, &gx, &wy, &siy, &soy, &wcy, &gy};
    size_t total = 0;
    for (auto *v : parts) total += v->size();
    std::vector<float> all;
    all.reserve(total);
    for (auto *v : parts) all.insert(all.end(), v->begin(), v->end());
    if (!salloc3(s, &s->tab, sizeof(float) * total) || cudaStreamSynchronize(s->stream) != cudaSuccess ||
        cudaMemcpy(s->tab, all.data(), sizeof(float) * total, cudaMemcpyHostToDevice) != cudaSuccess) {
      free3(s);
      return IPCU_ERR_NOMEM;
    }
    const float *b[10];
    size_t off = 0;
    for (int i = 0; i < 10; i++) {
      b[i] = s->tab + off;
      off += parts[i]->size();
    }
    f3s::Params3S &Q = s->PS;
    std::memset(&Q, 0, sizeof Q);
    Q.nx = c.nx;
    Q.ny = c.ny;
    Q.nz = c.nz;
    // z cells per CTA: the chunk's first planes are collided twice, so
    // chunks of 32 (6 % extra) while the grid keeps several waves
    const long long cols3 = (long long)((c.nx + f3s::kTX - 1) / f3s::kTX) * ((c.ny + f3s::kTY - 1) / f3s::kTY);
    Q.zchunk = (int)std::max(4LL, std::min<long long>(32, (long long)c.nz * cols3 / (148LL * f3s::kMinBlocks * 4)));
    Q.ax = {b[0], b[1], b[2], b[3], b[4]};
    Q.ay = {b[5], b[6], b[7], b[8], b[9]};
    Q.c = P.c;
    Q.dt = P.dt;
    Q.itau = P.itau;
    Q.omg_s = P.omg_s;
    Q.fk3 = P.fk3;
    Q.hdt = P.hdt;
    Q.rho0 = P.rho0;
    Q.rsal = P.rsal;
    Q.gb = P.gb;
    Q.giz_in = P.gi_in;
    Q.giz_wall = P.gi_wall;
    Q.mrt = P.mrt;
    Q.status = s->status;
    Q.store = s->store;
    Q.scale = s->scale;
    Q.inv_scale = s->inv_scale;
    Q.store_max = c.storage == IPCU_STORE_F16 ? 65504.0f : 3.0e38f;
    const int st = f3s::launch3s(Q, s->ns, s->stream, true);
    if (st != IPCU_OK) {
      free3(s);
      return st;
    }
  }
  // state at rest: f = 0, g = w_k S0, F = 0
  std::vector<float> f0(19 * N, 0.0f), g0(7 * N), F0(3 * N, 0.0f);
  for (long long i = 0; i < N; i++) {
    const double S = s0 ? s0[i] : 0.0;
    for (int k = 0; k < 7; k++) g0[k * N + i] = (float)(w7d(k) * S);
  }
  if (cudaMemsetAsync(s->status, 0, sizeof(unsigned), s->stream) != cudaSuccess ||
      put_state(s, f0.data(), g0.data(), F0.data()) != IPCU_OK) {
    free3(s);
    return IPCU_ERR_CUDA;
  }
  *out = s;
  return IPCU_OK;
}

extern "C" void ipcu_sim3d_destroy(ipcu_sim3d *s) {
  if (s) cudaStreamSynchronize(s->stream);
  free3(s);
}

extern "C" int ipcu_sim3d_step(ipcu_sim3d *s, int64_t nsteps) {
  if (!s || nsteps < 0) return IPCU_ERR_ARG;
  for (int64_t k = 0; k < nsteps; k++) {
    const int st = launch_step(s, s->cur, s->stream);
    if (st != IPCU_OK) return st;
    s->cur ^= 1;
    s->steps++;
  }
  return IPCU_OK;
}

extern "C" int ipcu_sim3d_step_graph(ipcu_sim3d *s, int64_t nsteps) {
  if (!s || nsteps < 0) return IPCU_ERR_ARG;
  const int64_t pairs = nsteps / 2;
  if (pairs > 0) {
    cudaGraphExec_t &ge = s->graph[s->cur];
    if (!ge) {
      // record on a private stream (the simulation's may be the legacy
      // default stream, which cannot be captured), replay on the simulation's
      cudaStream_t cs;
      if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return IPCU_ERR_CUDA;
      cudaGraph_t gr;
      if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaStreamDestroy(cs);
        return IPCU_ERR_CUDA;
      }
      int st = launch_step(s, s->cur, cs);
      if (st == IPCU_OK) st = launch_step(s, s->cur ^ 1, cs);
      const cudaError_t e = cudaStreamEndCapture(cs, &gr);
      cudaStreamDestroy(cs);
      if (st != IPCU_OK || e != cudaSuccess) return st != IPCU_OK ? st : IPCU_ERR_CUDA;
      const cudaError_t ei = cudaGraphInstantiate(&ge, gr, 0);
      cudaGraphDestroy(gr);
      if (ei != cudaSuccess) return IPCU_ERR_CUDA;
    }
    for (int64_t k = 0; k < pairs; k++)
      if (cudaGraphLaunch(ge, s->stream) != cudaSuccess) return IPCU_ERR_CUDA;
    s->steps += 2 * pairs;  // two steps return to the same buffer
  }
  return ipcu_sim3d_step(s, nsteps % 2);
}

extern "C" int ipcu_sim3d_get(ipcu_sim3d *s, const char *field, double *out, int64_t n) {
  if (!s || !field || !out) return IPCU_ERR_ARG;
  const long long N = s->N;
  const std::string fd(field);
  const long long need = fd == "f" ? 19 * N : (fd == "g" ? 7 * N : (fd == "F" ? 3 * N : N));
  if (fd != "f" && fd != "g" && fd != "F" && fd != "S" && fd != "p" && fd != "ux" && fd != "uy" && fd != "uz")
    return IPCU_ERR_ARG;
  if (n < need) return IPCU_ERR_CAPACITY;
  std::vector<float> f, g, F;
  if (int st = get_state(s, f, g, F)) return st;
  const std::vector<float> *raw = fd == "f" ? &f : (fd == "g" ? &g : (fd == "F" ? &F : nullptr));
  if (raw) {
    for (long long i = 0; i < need; i++) out[i] = (*raw)[i];
    return IPCU_OK;
  }
  // moments in the kernel's float order
  const float c = s->P.c;
  for (long long i = 0; i < N; i++) {
    float pr = 0.f, j[3] = {0.f, 0.f, 0.f}, S = 0.f;
    for (int k = 0; k < 19; k++) {
      const float v = f[k * N + i];
      pr += v;
      for (int a = 0; a < 3; a++)
        if (E19[k][a]) j[a] += E19[k][a] * v;
    }
    for (int k = 0; k < 7; k++) S += g[k * N + i];
    const float rho = std::fmaf(S, s->P.rsal, s->P.rho0), h = s->P.hdt / rho;
    if (fd == "p") out[i] = pr;
    else if (fd == "S") out[i] = S;
    else {
      const int a = fd == "ux" ? 0 : (fd == "uy" ? 1 : 2);
      out[i] = c * j[a] + F[a * N + i] * h;
    }
  }
  return IPCU_OK;
}

namespace {
// S, u_x, u_y, u_z of every cell ([4][N]) from the current state, in the
// float order of ipcu_sim3d_get (explicit rounding: the same values)
template <class T>
__global__ void macro3d_kernel(const void *__restrict__ fs, const void *__restrict__ gs, const void *__restrict__ rs,
                               float inv_scale, const float *__restrict__ F, long long N, float c, float rsal,
                               float rho0, float hdt, float *__restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    float j[3] = {0.f, 0.f, 0.f}, S = 0.f, f[19], g[7];
    s3::load_cell<T>(fs, gs, rs, i, N, inv_scale, f, g);
#pragma unroll
    for (int k = 0; k < 19; k++) {
      const float v = f[k];
      if (d3::cx(k)) j[0] = __fadd_rn(j[0], d3::cx(k) > 0 ? v : -v);
      if (d3::cy(k)) j[1] = __fadd_rn(j[1], d3::cy(k) > 0 ? v : -v);
      if (d3::cz(k)) j[2] = __fadd_rn(j[2], d3::cz(k) > 0 ? v : -v);
    }
#pragma unroll
    for (int k = 0; k < 7; k++) S = __fadd_rn(S, g[k]);
    const float h = __fdiv_rn(hdt, __fmaf_rn(S, rsal, rho0));
    out[i] = S;
#pragma unroll
    for (int a = 0; a < 3; a++) out[(a + 1) * N + i] = __fadd_rn(__fmul_rn(c, j[a]), __fmul_rn(F[a * N + i], h));
  }
}
}  // namespace

extern "C" int ipcu_sim3d_macro_async(ipcu_sim3d *s, float *out) {
  if (!s || !out) return IPCU_ERR_ARG;
  const long long N = s->N;
  float *d = nullptr;
  if (cudaMallocAsync((void **)&d, sizeof(float) * 4 * N, s->stream) != cudaSuccess) return IPCU_ERR_NOMEM;
  const int blocks = (int)std::min<long long>((N + 255) / 256, 148LL * 16);
  const int b = s->cur;
  auto go = [&](auto kern) {
    kern<<<blocks, 256, 0, s->stream>>>(s->f[b], s->g[b], s->r[b], s->inv_scale, s->F[b], N, s->P.c, s->P.rsal,
                                        s->P.rho0, s->P.hdt, d);
  };
  if (s->store == IPCU_STORE_F16) go(macro3d_kernel<__half>);
  else if (s->store == IPCU_STORE_BF16) go(macro3d_kernel<__nv_bfloat16>);
  else go(macro3d_kernel<float>);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, sizeof(float) * 4 * N, cudaMemcpyDefault, s->stream);
  cudaFreeAsync(d, s->stream);
  return e == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

extern "C" int ipcu_sim3d_set_state(ipcu_sim3d *s, const double *f, const double *g, const double *F) {
  if (!s) return IPCU_ERR_ARG;
  std::vector<float> fv, gv, Fv;
  if (int st = get_state(s, fv, gv, Fv)) return st;  // the parts kept
  auto put = [&](const double *src, std::vector<float> &dst) {
    if (src)
      for (size_t i = 0; i < dst.size(); i++) dst[i] = (float)src[i];
  };
  put(f, fv);
  put(g, gv);
  put(F, Fv);
  return put_state(s, fv.data(), gv.data(), Fv.data());
}


extern "C" int ipcu_sim3d_upload(ipcu_sim3d *s, const float *f, const float *g, const float *F) {
  if (!s) return IPCU_ERR_ARG;
  if (s->store != IPCU_STORE_F32 && (f || g)) return IPCU_ERR_UNSUPPORTED;
  const long long N = s->N;
  cudaError_t e = cudaSuccess;
  if (f) e = cudaMemcpyAsync(s->f[s->cur], f, sizeof(float) * 19 * N, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess && g) e = cudaMemcpyAsync(s->g[s->cur], g, sizeof(float) * 7 * N, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess && F) e = cudaMemcpyAsync(s->F[s->cur], F, sizeof(float) * 3 * N, cudaMemcpyHostToDevice, s->stream);
  return e == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

extern "C" int ipcu_sim3d_download(ipcu_sim3d *s, float *f, float *g, float *F) {
  if (!s) return IPCU_ERR_ARG;
  if (s->store != IPCU_STORE_F32 && (f || g)) return IPCU_ERR_UNSUPPORTED;
  const long long N = s->N;
  cudaError_t e = cudaSuccess;
  if (f) e = cudaMemcpyAsync(f, s->f[s->cur], sizeof(float) * 19 * N, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess && g) e = cudaMemcpyAsync(g, s->g[s->cur], sizeof(float) * 7 * N, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess && F) e = cudaMemcpyAsync(F, s->F[s->cur], sizeof(float) * 3 * N, cudaMemcpyDeviceToHost, s->stream);
  return e == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

extern "C" int ipcu_sim3d_sync(ipcu_sim3d *s) {
  if (!s) return IPCU_ERR_ARG;
  return cudaStreamSynchronize(s->stream) == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA;
}

extern "C" int ipcu_sim3d_status(ipcu_sim3d *s, uint32_t *flags) {
  if (!s || !flags) return IPCU_ERR_ARG;
  unsigned v = 0;
  if (cudaMemcpyAsync(&v, s->status, sizeof v, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
      cudaStreamSynchronize(s->stream) != cudaSuccess)
    return IPCU_ERR_CUDA;
  *flags = v;
  return v ? IPCU_ERR_NONFINITE : IPCU_OK;
}

extern "C" int64_t ipcu_sim3d_cells(const ipcu_sim3d *s) { return s ? s->N : 0; }

extern "C" int64_t ipcu_sim3d_bytes_per_cell(const ipcu_sim3d *s) {
  if (!s) return 0;
  return s->store == IPCU_STORE_F32 ? 2 * 4 * (19 + 7 + 3) : 2 * (2 * (19 + 7 + 5) + 4 * 3);
}

// ---------------------------------------------------------------------------
// Checkpoint / restore: configuration, axes, step count and the raw state in
// its storage type (f, g, with 16-bit storage the reference planes, F); a
// restored run continues bit-identically. Version 1 files (FP32 only, the
// configuration without its storage field) still load.
namespace {
constexpr char kMagic3[8] = {'I', 'P', 'C', 'U', 'S', '3', 'D', '1'};
constexpr int32_t kSnap3Version = 2;
constexpr size_t kCfgV1 = offsetof(ipcu_sim3d_config, storage);
template <class T>
bool wr3(FILE *f, const T *p, size_t n) { return fwrite(p, sizeof(T), n, f) == n; }
template <class T>
bool rd3(FILE *f, T *p, size_t n) { return fread(p, sizeof(T), n, f) == n; }

// the raw arrays of buffer `cur`: device pointer and bytes
std::vector<std::pair<void *, size_t>> raw_parts(ipcu_sim3d *s) {
  const long long N = s->N;
  const int b = s->cur;
  const size_t es = s->store == IPCU_STORE_F32 ? sizeof(float) : 2;
  std::vector<std::pair<void *, size_t>> v = {{s->f[b], es * 19 * N}, {s->g[b], es * 7 * N}};
  if (s->store != IPCU_STORE_F32) v.push_back({s->r[b], 2 * 5 * (size_t)N});
  v.push_back({s->F[b], sizeof(float) * 3 * N});
  return v;
}
}  // namespace

extern "C" int ipcu_sim3d_save(ipcu_sim3d *s, const char *path) {
  if (!s || !path) return IPCU_ERR_ARG;
  if (s->ib) return IPCU_ERR_UNSUPPORTED;  // the sphere's state is not part of the 3-D snapshot
  const auto parts = raw_parts(s);
  std::vector<std::vector<char>> host(parts.size());
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  for (size_t a = 0; a < parts.size(); a++) {
    host[a].resize(parts[a].second);
    if (cudaMemcpy(host[a].data(), parts[a].first, parts[a].second, cudaMemcpyDeviceToHost) != cudaSuccess)
      return IPCU_ERR_CUDA;
  }
  FILE *fp = fopen(path, "wb");
  if (!fp) return IPCU_ERR_IO;
  const int32_t ns = s->ns;
  bool ok = wr3(fp, kMagic3, 8) && wr3(fp, &kSnap3Version, 1) && wr3(fp, &s->cfg, 1) && wr3(fp, &ns, 1) &&
            wr3(fp, &s->steps, 1) && wr3(fp, s->X.data(), s->X.size()) && wr3(fp, s->DX.data(), s->DX.size()) &&
            wr3(fp, s->Y.data(), s->Y.size()) && wr3(fp, s->DY.data(), s->DY.size());
  for (auto &h : host) ok = ok && wr3(fp, h.data(), h.size());
  ok = (fclose(fp) == 0) && ok;
  return ok ? IPCU_OK : IPCU_ERR_IO;
}

extern "C" int ipcu_sim3d_load(const char *path, ipcu_stream_t stream, ipcu_sim3d **out) {
  if (!path || !out) return IPCU_ERR_ARG;
  *out = nullptr;
  FILE *fp = fopen(path, "rb");
  if (!fp) return IPCU_ERR_IO;
  char mg[8];
  int32_t ver = 0, ns = 0;
  ipcu_sim3d_config c;
  std::memset(&c, 0, sizeof c);
  long long steps = 0;
  bool ok = rd3(fp, mg, 8) && std::memcmp(mg, kMagic3, 8) == 0 && rd3(fp, &ver, 1) && (ver == 1 || ver == 2) &&
            rd3(fp, reinterpret_cast<char *>(&c), ver == 1 ? kCfgV1 : sizeof c) && rd3(fp, &ns, 1) &&
            rd3(fp, &steps, 1) && c.nx > 0 && c.ny > 0 && c.nz > 0;
  std::vector<double> X(ok ? c.nx : 0), DX(X.size()), Y(ok ? c.ny : 0), DY(Y.size());
  ok = ok && rd3(fp, X.data(), X.size()) && rd3(fp, DX.data(), DX.size()) && rd3(fp, Y.data(), Y.size()) &&
       rd3(fp, DY.data(), DY.size());
  if (!ok) {
    fclose(fp);
    return IPCU_ERR_IO;
  }
  // ns 0: the uniform box kernel; else the flux-form kernel on the saved
  // axes (a 16-bit box without stretched axes saved its uniform ones)
  ipcu_sim3d_axes ax{X.data(), DX.data(), Y.data(), DY.data(), ns};
  ipcu_sim3d *s = nullptr;
  const int st = ipcu_sim3d_create_stretched(&c, ns ? &ax : nullptr, nullptr, stream, &s);
  if (st != IPCU_OK) {
    fclose(fp);
    return st;
  }
  const auto parts = raw_parts(s);
  for (auto &pt : parts) {
    std::vector<char> h(pt.second);
    ok = ok && rd3(fp, h.data(), h.size()) &&
         cudaMemcpy(pt.first, h.data(), h.size(), cudaMemcpyHostToDevice) == cudaSuccess;
  }
  fclose(fp);
  if (!ok) {
    ipcu_sim3d_destroy(s);
    return IPCU_ERR_IO;
  }
  s->steps = steps;
  *out = s;
  return IPCU_OK;
}

extern "C" int64_t ipcu_sim3d_steps(const ipcu_sim3d *s) { return s ? s->steps : -1; }

// ---------------------------------------------------------------------------
// Moving sphere (ibm3d.cu): one per simulation.
extern "C" int ipcu_sim3d_ib_attach(ipcu_sim3d *s, const ipcu_ib_sphere3d *bd, const double *markers, const double *dA,
                                    int32_t n) {
  if (!s || !bd || !markers || !dA || n <= 0) return IPCU_ERR_ARG;
  if (s->ib) return IPCU_ERR_CAPACITY;
  if (n > ib3d::kMaxMarkers) return IPCU_ERR_CAPACITY;
  if (!(bd->radius > 0 && bd->rho_s > 0 && bd->rho_f > 0 && bd->iters >= 0 && bd->iters <= 64)) return IPCU_ERR_ARG;
  for (int i = 0; i < 3 * n; i++)
    if (!std::isfinite(markers[i])) return IPCU_ERR_ARG;
  for (int i = 0; i < n; i++)
    if (!(dA[i] > 0)) return IPCU_ERR_ARG;
  {
    static bool prepared[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return IPCU_ERR_CUDA;
    if (!prepared[dev]) {
      if (int st = ib3d::prepare()) return st;
      prepared[dev] = true;
    }
  }
  const ipcu_sim3d_config &c = s->cfg;
  const long long N = s->N;
  const size_t W = ib3d::kMaxWin;
  // one block: body, markers, scratch, axes, force density (8-byte aligned parts)
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  const size_t o_body = take(sizeof(ib3d::Body)), o_r0 = take(sizeof(double) * 3 * n), o_dA = take(sizeof(double) * n);
  const size_t o_xc = take(sizeof(double) * c.nx), o_yc = take(sizeof(double) * c.ny);
  const size_t o_wx = take(sizeof(float) * c.nx), o_wy = take(sizeof(float) * c.ny);
  const size_t o_plan = take(sizeof(ib3d::Plan)), o_morg = take(sizeof(int) * 3 * n), o_mw = take(sizeof(float) * 12 * n);
  const size_t o_mub = take(sizeof(float) * 3 * n), o_mft = take(sizeof(float) * 3 * n), o_mdf = take(sizeof(float) * 3 * n);
  const size_t o_bstart = take(sizeof(int) * (ib3d::kMaxBins + 1)), o_blist = take(sizeof(int) * n);
  const size_t o_part = take(sizeof(double) * 12 * ib3d::kParts);
  const size_t o_wu = take(sizeof(float) * 3 * W), o_wf = take(sizeof(float) * 3 * W), o_wj = take(sizeof(float) * 3 * W);
  const size_t o_wh = take(sizeof(float) * W), o_wv = take(sizeof(float) * W);
  const size_t o_ccnt = take(sizeof(int) * W), o_clist = take(sizeof(int) * W * ib3d::kSlots);
  const size_t o_fext = take(sizeof(float) * 3 * (size_t)N);
  char *mem = nullptr;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return IPCU_ERR_CUDA;
  if (cudaMallocAsync((void **)&mem, off, s->stream) != cudaSuccess) return IPCU_ERR_NOMEM;
  ib3d::Job *j = new ib3d::Job();
  std::memset(j, 0, sizeof *j);
  j->nx = c.nx;
  j->ny = c.ny;
  j->nz = c.nz;
  j->c = s->P.c;
  j->hdt = s->P.hdt;
  j->rho0 = s->P.rho0;
  j->rsal = s->P.rsal;
  j->dz = c.dz;
  j->dt = c.dt;
  j->body = reinterpret_cast<ib3d::Body *>(mem + o_body);
  j->r0 = reinterpret_cast<const double *>(mem + o_r0);
  j->dA = reinterpret_cast<const double *>(mem + o_dA);
  j->xc = reinterpret_cast<const double *>(mem + o_xc);
  j->yc = reinterpret_cast<const double *>(mem + o_yc);
  j->wx = reinterpret_cast<const float *>(mem + o_wx);
  j->wy = reinterpret_cast<const float *>(mem + o_wy);
  j->plan = reinterpret_cast<ib3d::Plan *>(mem + o_plan);
  j->morg = reinterpret_cast<int *>(mem + o_morg);
  j->mw = reinterpret_cast<float *>(mem + o_mw);
  j->mub = reinterpret_cast<float *>(mem + o_mub);
  j->mft = reinterpret_cast<float *>(mem + o_mft);
  j->mdf = reinterpret_cast<float *>(mem + o_mdf);
  j->bstart = reinterpret_cast<int *>(mem + o_bstart);
  j->blist = reinterpret_cast<int *>(mem + o_blist);
  j->part = reinterpret_cast<double *>(mem + o_part);
  j->wu = reinterpret_cast<float *>(mem + o_wu);
  j->wf = reinterpret_cast<float *>(mem + o_wf);
  j->wj = reinterpret_cast<float *>(mem + o_wj);
  j->wh = reinterpret_cast<float *>(mem + o_wh);
  j->wv = reinterpret_cast<float *>(mem + o_wv);
  j->ccnt = reinterpret_cast<int *>(mem + o_ccnt);
  j->clist = reinterpret_cast<int *>(mem + o_clist);
  j->fext = reinterpret_cast<float *>(mem + o_fext);
  j->status = s->status;
  j->store = s->store;
  j->inv_scale = s->inv_scale;
  j->nl = n;
  j->iters = bd->iters;
  j->radius = bd->radius;
  const double vol = 4.0 / 3.0 * M_PI * bd->radius * bd->radius * bd->radius;
  j->m = bd->rho_s * vol;
  j->I = 0.4 * j->m * bd->radius * bd->radius;
  j->rho_s = bd->rho_s;
  j->rho_f = bd->rho_f;
  j->grav = bd->gravity;
  ib3d::Body b0;
  std::memset(&b0, 0, sizeof b0);
  b0.X[0] = bd->xc;
  b0.X[1] = bd->yc;
  b0.X[2] = bd->zc;
  b0.U[0] = bd->u;
  b0.U[1] = bd->v;
  b0.U[2] = bd->w;
  b0.R[0] = b0.R[4] = b0.R[8] = 1.0;
  std::vector<float> wxf(c.nx), wyf(c.ny);
  for (int i = 0; i < c.nx; i++) wxf[i] = (float)s->DX[i];
  for (int i = 0; i < c.ny; i++) wyf[i] = (float)s->DY[i];
  cudaError_t e = cudaMemcpyAsync(j->body, &b0, sizeof b0, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(mem + o_r0, markers, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(mem + o_dA, dA, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(mem + o_xc, s->X.data(), sizeof(double) * c.nx, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(mem + o_yc, s->Y.data(), sizeof(double) * c.ny, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(mem + o_wx, wxf.data(), sizeof(float) * c.nx, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(mem + o_wy, wyf.data(), sizeof(float) * c.ny, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(j->fext, 0, sizeof(float) * 3 * (size_t)N, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);  // the host vectors are released on return
  if (e != cudaSuccess) {
    cudaFreeAsync(mem, s->stream);
    delete j;
    return IPCU_ERR_CUDA;
  }
  // the step kernels add the force density; recorded graphs hold the old parameters
  for (int i = 0; i < 2; i++)
    if (s->graph[i]) {
      cudaGraphExecDestroy(s->graph[i]);
      s->graph[i] = nullptr;
    }
  s->P.fext = j->fext;
  s->PS.fext = j->fext;
  s->P.fext_box = s->PS.fext_box = j->body->win;
  s->ib = j;
  s->ib_mem = mem;
  return IPCU_OK;
}

extern "C" int ipcu_sim3d_ib_body(ipcu_sim3d *s, double *out) {
  if (!s || !out || !s->ib) return IPCU_ERR_ARG;
  ib3d::Body b;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess ||
      cudaMemcpy(&b, s->ib->body, sizeof b, cudaMemcpyDeviceToHost) != cudaSuccess)
    return IPCU_ERR_CUDA;
  for (int a = 0; a < 3; a++) {
    out[a] = b.X[a];
    out[3 + a] = b.U[a];
    out[6 + a] = b.om[a];
    out[9 + a] = b.Fib[a];
    out[12 + a] = b.Tib[a];
  }
  return IPCU_OK;
}
