// Direction tables, launch geometry and status helpers shared by all kernels.
#include "ipcu_common.cuh"

namespace ipcu {

DirTables host_dir_tables() {
  DirTables t{};
  // D2Q9 in the x-z plane: 0 rest; 1 +x, 2 +z, 3 -x, 4 -z; 5 (+x,+z), 6 (-x,+z),
  // 7 (-x,-z), 8 (+x,-z) (ref: function/basic.cu:78-87).
  const int ki9[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
  for (int k = 0; k < 9; k++) t.kinv[0][k] = (int8_t)ki9[k];
  // The flux form interpolates x-moving populations along x; the partner
  // is the x-neighbour the population moves towards (ref: basic.cu:123-126).
  const int xmov[6] = {1, 3, 5, 6, 7, 8}, xdir[6] = {1, 3, 1, 3, 3, 1};
  for (int i = 0; i < 6; i++) {
    t.cp[0][xmov[i]] = (int8_t)xdir[i];
    t.cm[0][xmov[i]] = (int8_t)(xdir[i] == 1 ? 3 : 1);
  }
  // D3Q27 (ref: function/basic.cu:88-97,116-137)
  const int ki27[27] = {0, 3, 4, 1, 2, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15, 26, 25, 24, 23, 22, 21, 20, 19};
  const int cp27[27] = {0, 1, 2, 3, 4, 0, 0, 7, 8, 9, 10, 1, 1, 3, 3, 2, 2, 4, 4, 7, 7, 8, 8, 9, 9, 10, 10};
  for (int k = 0; k < 27; k++) {
    t.kinv[1][k] = (int8_t)ki27[k];
    t.cp[1][k] = (int8_t)cp27[k];
    t.cm[1][k] = (int8_t)ki27[cp27[k]];
  }
  const int ip_[8] = {8, 8, 7, 7, 10, 10, 9, 9}, im_[8] = {9, 9, 10, 10, 7, 7, 8, 8};
  for (int i = 0; i < 8; i++) {
    t.cip[19 + i] = (int8_t)ip_[i];
    t.cim[19 + i] = (int8_t)im_[i];
  }
  // axis partners of the xy tensor stencil (ref: function/basic.cu:139-153)
  const int xp[27] = {0, 1, 0, 3, 0, 0, 0, 1, 1, 3, 3, 1, 1, 3, 3, 0, 0, 0, 0, 1, 1, 1, 1, 3, 3, 3, 3};
  const int yp[27] = {0, 0, 2, 0, 4, 0, 0, 2, 4, 2, 4, 0, 0, 0, 0, 2, 2, 4, 4, 2, 2, 4, 4, 2, 2, 4, 4};
  for (int k = 0; k < 27; k++) {
    t.cxp[k] = (int8_t)xp[k];
    t.cxm[k] = (int8_t)(xp[k] == 1 ? 3 : (xp[k] == 3 ? 1 : 0));
    t.cyp[k] = (int8_t)yp[k];
    t.cym[k] = (int8_t)(yp[k] == 2 ? 4 : (yp[k] == 4 ? 2 : 0));
  }
  return t;
}

Launch launch_for(long long nthreads) {
  static int sms[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (sms[dev] == 0) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    sms[dev] = v > 0 ? v : 148;
  }
  Launch L;
  L.block = dim3(256);
  long long cap = (long long)sms[dev] * 8;
  long long want = nthreads > 0 ? (nthreads + 255) / 256 : (long long)sms[dev] * 4;
  if (want < 1) want = 1;
  if (want > cap) want = cap;
  L.grid = dim3((unsigned)want);
  return L;
}

int status_from_cuda(cudaError_t e) { return e == cudaSuccess ? IPCU_OK : IPCU_ERR_CUDA; }

}  // namespace ipcu

extern "C" const char *ipcu_status_string(int code) {
  switch (code) {
    case IPCU_OK: return "ok";
    case IPCU_ERR_ARG: return "invalid argument";
    case IPCU_ERR_CUDA: return "CUDA error";
    case IPCU_ERR_NOMEM: return "out of device memory";
    case IPCU_ERR_CAPACITY: return "output capacity too small";
    case IPCU_ERR_NONFINITE: return "non-finite value detected";
    case IPCU_ERR_UNSUPPORTED: return "unsupported configuration";
    case IPCU_ERR_IO: return "file I/O error";
    case IPCU_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

extern "C" const char *ipcu_last_cuda_error(void) { return cudaGetErrorString(cudaPeekAtLastError()); }

// The pybind prototype's kernel: add a constant to every element
// (ref: pybind_LockExchange/kernel.cu:4-9, which adds 5.0f).
namespace {
__global__ void k_add_scalar(float *d, long long n, float v) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    d[i] += v;
}
}  // namespace

extern "C" int ipcu_add_scalar_f32(float *data, int64_t n, float value, ipcu_stream_t stream) {
  if (n < 0 || (n > 0 && !data)) return IPCU_ERR_ARG;
  if (n == 0) return IPCU_OK;
  ipcu::Launch L = ipcu::launch_for(n);
  k_add_scalar<<<L.grid, L.block, 0, (cudaStream_t)stream>>>(data, n, value);
  return ipcu::status_from_cuda(cudaGetLastError());
}
