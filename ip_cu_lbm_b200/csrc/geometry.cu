// Device-side geometry set-up: the reference builds the cell numbering, the
// neighbour table and the ghost cells on the host in O(N) serial loops, and
// searches each marker's nearest fluid cell in an O(N * Np) host loop
// (ref: LockExchange/LockExchange.cu:55-127, function/basic.cu:203-237,
// SphereFallSuzuki2018/SphereSuzuki.cu:268-274). These kernels produce the
// same arrays on the GPU: box numbering and neighbours per cell, one ghost
// per open cell numbered in the reference's scan order (a device prefix sum
// over the open flags), ghost geometry copied from the owner, and the nearest
// cell per marker with the reference's float distances and first-minimum rule.
#include <vector>

#include "ipcu_common.cuh"

namespace ipcu {
namespace {

// unit velocity of direction k: D2Q9 (x-z plane) or D3Q27 (ref: function/basic.cu:78-97)
__device__ __forceinline__ void unit_vec(int Q, int k, int &ex, int &ey, int &ez) {
  if (Q == 9) {
    const int x[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1}, z[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    ex = x[k];
    ey = 0;
    ez = z[k];
  } else {
    const signed char v[27][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {-1, 0, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1},
                                  {1, 1, 0}, {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, 0, 1}, {1, 0, -1}, {-1, 0, 1},
                                  {-1, 0, -1}, {0, 1, 1}, {0, 1, -1}, {0, -1, 1}, {0, -1, -1}, {1, 1, 1}, {1, 1, -1},
                                  {1, -1, 1}, {1, -1, -1}, {-1, 1, 1}, {-1, 1, -1}, {-1, -1, 1}, {-1, -1, -1}};
    ex = v[k][0];
    ey = v[k][1];
    ez = v[k][2];
  }
}

struct Axis {
  const int *coarse;    // refined index -> coarse index
  const int *sub;       // refined index -> subdivision index
  const int *div;       // coarse divisions
};

// numbering, geometry and neighbour table of the refined box (x-major, then y, z fastest)
template <class T>
__global__ void k_box(int Q, int NX, int NY, int nz, double dx, double rx, double ry, Axis ax, Axis ay, int *lnum,
                      int *neib, T *px, T *py, T *pz, T *dX, T *dY, int *open) {
  const long long n = (long long)NX * NY * nz;
  IPCU_FOR(c, 0, n) {
    const int L = (int)(c % nz);
    const long long t = c / nz;
    const int J = (int)(t % NY), I = (int)(t / NY);
    lnum[c] = (int)c;
    const int ic = ax.coarse[I], di = ax.sub[I], jc = ay.coarse[J], dj = ay.sub[J];
    px[c] = (T)((ic + (2.0 * di + 1.0) / (2.0 * ax.div[ic])) * dx * rx);
    py[c] = (T)((jc + (2.0 * dj + 1.0) / (2.0 * ay.div[jc])) * dx * ry);
    pz[c] = (T)((L + 0.5) * dx);
    dX[c] = (T)(dx * rx / ax.div[ic]);
    dY[c] = (T)(dx * ry / ay.div[jc]);
    int op = 0;
    for (int k = 0; k < Q; k++) {
      int ex, ey, ez;
      unit_vec(Q, k, ex, ey, ez);
      const int a = I + ex, b = J + ey, d = L + ez;
      const bool in = a >= 0 && a < NX && b >= 0 && b < NY && d >= 0 && d < nz;
      neib[c * Q + k] = in ? (int)(((long long)a * NY + b) * nz + d) : -1;
      if (!in && k > 0) op = 1;
    }
    open[c] = op;
  }
}

// exclusive scan of int flags, three passes: block sums, scan of block sums, add
constexpr int kScanBlock = 1024;
__global__ void k_scan_block(const int *in, long long n, long long *out, long long *bsum) {
  __shared__ long long s[kScanBlock];
  const long long i = (long long)blockIdx.x * kScanBlock + threadIdx.x;
  const long long v = i < n ? in[i] : 0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < kScanBlock; o <<= 1) {
    long long a = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
    __syncthreads();
    s[threadIdx.x] += a;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v;
  if (threadIdx.x == kScanBlock - 1) bsum[blockIdx.x] = s[threadIdx.x];
}
__global__ void k_scan_sums(long long *bsum, int nb, long long *total) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    long long acc = 0;
    for (int b = 0; b < nb; b++) {
      long long v = bsum[b];
      bsum[b] = acc;
      acc += v;
    }
    *total = acc;
  }
}
__global__ void k_scan_add(long long *out, long long n, const long long *bsum) {
  const long long i = (long long)blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n) out[i] += bsum[blockIdx.x];
}

// one ghost per open cell (ref: function/basic.cu:213-233): its entries point
// to itself except towards the owner; the owner's missing entries point to it;
// geometry copied from the owner
template <class T>
__global__ void k_ghosts(int Q, long long nc, const int *open, const long long *pos, int *neib, int *owner, T *px,
                         T *py, T *pz, T *dX, T *dY) {
  IPCU_FOR(c, 0, nc) {
    if (!open[c]) continue;
    const long long g = nc + pos[c];
    const int8_t *kinv = c_dirs.kinv[qsel(Q)];
    for (int k = 0; k < Q; k++) neib[g * Q + k] = (int)g;
    neib[g * Q] = (int)c;
    for (int k = 1; k < Q; k++)
      if (neib[c * Q + k] == -1) {
        neib[c * Q + k] = (int)g;
        neib[g * Q + kinv[k]] = (int)c;
      }
    owner[pos[c]] = (int)c;
    px[g] = px[c];
    py[g] = py[c];
    pz[g] = pz[c];
    dX[g] = dX[c];
    dY[g] = dY[c];
  }
}

// nearest fluid cell per marker: one block per marker, distances as the
// reference forms them (ref: SphereFallSuzuki2018/SphereSuzuki.cu:268-274:
// coordinate differences in the storage type, squares summed in double
// without contraction, rounded to float), smallest index among equal minima
// (its loop keeps the first minimum)
template <class T>
__global__ void k_nearest(const T *px, const T *py, const T *pz, long long nc, const T *posw, int nm, int *lid) {
  const int m = blockIdx.x;
  if (m >= nm) return;
  const T wx = posw[m * 3], wy = posw[m * 3 + 1], wz = posw[m * 3 + 2];
  float best = 3.4e38f;
  long long bi = 0x7fffffffffffffffLL;
  for (long long i = threadIdx.x; i < nc; i += blockDim.x) {
    const double a = (double)(T)(px[i] - wx), b = (double)(T)(py[i] - wy), c = (double)(T)(pz[i] - wz);
    const double s = __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
    const float d = (float)sqrt(s);
    if (d < best || (d == best && i < bi)) {
      best = d;
      bi = i;
    }
  }
  __shared__ float sd[256];
  __shared__ long long si[256];
  sd[threadIdx.x] = best;
  si[threadIdx.x] = bi;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      const float d2 = sd[threadIdx.x + o];
      const long long i2 = si[threadIdx.x + o];
      if (d2 < sd[threadIdx.x] || (d2 == sd[threadIdx.x] && i2 < si[threadIdx.x])) {
        sd[threadIdx.x] = d2;
        si[threadIdx.x] = i2;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) lid[m] = (int)(si[0] == 0x7fffffffffffffffLL ? 0 : si[0]);
}

template <class T>
int build_box(int Q, int nx0, int ny0, int nz, double dx, double rx, double ry, const int *divx, const int *divy,
              int *lnum, int *neib, T *px, T *py, T *pz, T *dX, T *dY, int64_t cap, int *owner, int64_t *nc_out,
              int64_t *nw_out, cudaStream_t s) {
  if ((Q != 9 && Q != 27) || nx0 < 1 || ny0 < 1 || nz < 1 || !divx || !divy || !lnum || !neib || !owner)
    return IPCU_ERR_ARG;
  std::vector<int> xc, xs, yc, ys;
  for (int i = 0; i < nx0; i++)
    for (int d = 0; d < divx[i]; d++) xc.push_back(i), xs.push_back(d);
  for (int j = 0; j < ny0; j++)
    for (int d = 0; d < divy[j]; d++) yc.push_back(j), ys.push_back(d);
  const int NX = (int)xc.size(), NY = (int)yc.size();
  const long long nc = (long long)NX * NY * nz;
  if (nc > cap) return IPCU_ERR_CAPACITY;
  ensure_tables();
  // small device tables for the axes, the open flags and the scan
  int *d_ax = nullptr, *d_open = nullptr;
  long long *d_pos = nullptr, *d_bsum = nullptr;
  const int nb = (int)((nc + kScanBlock - 1) / kScanBlock);
  size_t axn = 2 * (NX + NY) + nx0 + ny0;
  if (cudaMalloc((void **)&d_ax, sizeof(int) * axn) != cudaSuccess ||
      cudaMalloc((void **)&d_open, sizeof(int) * nc) != cudaSuccess ||
      cudaMalloc((void **)&d_pos, sizeof(long long) * nc) != cudaSuccess ||
      cudaMalloc((void **)&d_bsum, sizeof(long long) * (nb + 1)) != cudaSuccess) {
    cudaFree(d_ax);
    cudaFree(d_open);
    cudaFree(d_pos);
    cudaFree(d_bsum);
    return IPCU_ERR_NOMEM;
  }
  std::vector<int> h;
  h.insert(h.end(), xc.begin(), xc.end());
  h.insert(h.end(), xs.begin(), xs.end());
  h.insert(h.end(), divx, divx + nx0);
  h.insert(h.end(), yc.begin(), yc.end());
  h.insert(h.end(), ys.begin(), ys.end());
  h.insert(h.end(), divy, divy + ny0);
  int st = IPCU_OK;
  if (cudaMemcpyAsync(d_ax, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, s) != cudaSuccess) st = IPCU_ERR_CUDA;
  Axis ax{d_ax, d_ax + NX, d_ax + 2 * NX}, ay{d_ax + 2 * NX + nx0, d_ax + 2 * NX + nx0 + NY, d_ax + 2 * NX + nx0 + 2 * NY};
  if (st == IPCU_OK) {
    Launch L = launch_for(nc);
    k_box<T><<<L.grid, L.block, 0, s>>>(Q, NX, NY, nz, dx, rx, ry, ax, ay, lnum, neib, px, py, pz, dX, dY, d_open);
    k_scan_block<<<nb, kScanBlock, 0, s>>>(d_open, nc, d_pos, d_bsum);
    k_scan_sums<<<1, 32, 0, s>>>(d_bsum, nb, d_bsum + nb);
    k_scan_add<<<nb, kScanBlock, 0, s>>>(d_pos, nc, d_bsum);
    long long nw = 0;
    if (cudaMemcpyAsync(&nw, d_bsum + nb, sizeof nw, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      st = IPCU_ERR_CUDA;
    else if (nc + nw > cap)
      st = IPCU_ERR_CAPACITY;
    else {
      k_ghosts<T><<<L.grid, L.block, 0, s>>>(Q, nc, d_open, d_pos, neib, owner, px, py, pz, dX, dY);
      if (cudaStreamSynchronize(s) != cudaSuccess) st = IPCU_ERR_CUDA;
      *nc_out = nc;
      *nw_out = nw;
    }
  }
  cudaFree(d_ax);
  cudaFree(d_open);
  cudaFree(d_pos);
  cudaFree(d_bsum);
  return st;
}

}  // namespace
}  // namespace ipcu

using namespace ipcu;

#define GEOM_DEFS(T, S)                                                                                        \
  extern "C" int ipcu_build_box_device_##S(int Q, int nx0, int ny0, int nz, double dx, double ratiox,          \
                                           double ratioy, const int *divx, const int *divy, int *lnum,         \
                                           int *neib, T *posx, T *posy, T *posz, T *delX, T *delY,              \
                                           int64_t cap, int *owner, int64_t *num_calc, int64_t *num_wall,      \
                                           ipcu_stream_t stream) {                                             \
    if (!num_calc || !num_wall) return IPCU_ERR_ARG;                                                           \
    return build_box<T>(Q, nx0, ny0, nz, dx, ratiox, ratioy, divx, divy, lnum, neib, posx, posy, posz, delX,   \
                        delY, cap, owner, num_calc, num_wall, (cudaStream_t)stream);                           \
  }                                                                                                            \
  extern "C" int ipcu_nearest_cells_##S(const T *posx, const T *posy, const T *posz, int64_t num_calc,         \
                                        const T *posw, int num_markers, int *lattice_id,                       \
                                        ipcu_stream_t stream) {                                                \
    if (!posx || !posy || !posz || !posw || !lattice_id || num_markers < 0 || num_calc < 1)                    \
      return IPCU_ERR_ARG;                                                                                     \
    if (num_markers == 0) return IPCU_OK;                                                                      \
    k_nearest<T><<<num_markers, 256, 0, (cudaStream_t)stream>>>(posx, posy, posz, num_calc, posw, num_markers, \
                                                                 lattice_id);                                  \
    return status_from_cuda(cudaGetLastError());                                                               \
  }
GEOM_DEFS(float, f32)
GEOM_DEFS(double, f64)
#undef GEOM_DEFS
