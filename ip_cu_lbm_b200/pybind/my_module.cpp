// pybind11 module `my_module`: the Python boundary of the reference's
// pybind_LockExchange prototype (ref: pybind_LockExchange/wrapper.cpp:11-61,
// kernel.cu:4-17, run.py:1-13), made to build and work, plus the LockExchange
// stepping class that prototype was meant to expose, on top of libipcu's C ABI.
//
//   GPUMemory(n)            device buffer of n float32 (RAII)
//     .set(np.float32[n])   host -> device
//     .get() -> np.float32  device -> host
//     .size()
//   compute_on_gpu(mem)     adds 5 to every element (the prototype's kernel)
//   LockExchange(**config)  a structured-grid simulation (ipcu_sim_*)
//     .step(n), .step_graph(n, chunk), .get(field) -> np.float64, .totals()
#include <cuda_runtime.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "ipcu.h"

namespace py = pybind11;

extern "C" int ipcu_add_scalar_f32(float *data, int64_t n, float value, ipcu_stream_t stream);

namespace {

void check(int st, const char *what) {
  if (st != IPCU_OK) throw std::runtime_error(std::string(what) + ": " + ipcu_status_string(st));
}

class GPUMemory {
 public:
  explicit GPUMemory(size_t n) : n_(n) {
    if (n_ && cudaMalloc(&d_, n_ * sizeof(float)) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
  }
  ~GPUMemory() {
    if (d_) cudaFree(d_);
  }
  GPUMemory(const GPUMemory &) = delete;
  GPUMemory &operator=(const GPUMemory &) = delete;
  void set(py::array_t<float, py::array::c_style | py::array::forcecast> a) {
    if ((size_t)a.size() != n_) throw std::runtime_error("Size mismatch");
    if (cudaMemcpy(d_, a.data(), n_ * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
      throw std::runtime_error("cudaMemcpy H2D failed");
  }
  py::array_t<float> get() const {
    py::array_t<float> out(n_);
    if (cudaMemcpy(out.mutable_data(), d_, n_ * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
      throw std::runtime_error("cudaMemcpy D2H failed");
    return out;
  }
  size_t size() const { return n_; }
  float *data() { return d_; }

 private:
  float *d_ = nullptr;
  size_t n_ = 0;
};

void compute_on_gpu(GPUMemory &m) {
  check(ipcu_add_scalar_f32(m.data(), (int64_t)m.size(), 5.0f, nullptr), "compute_on_gpu");
  if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("compute_on_gpu: CUDA error");
}

const std::vector<std::string> kGeo = {"uniform", "x5", "x3", "z5", "z3"};
const std::vector<std::string> kStore = {"f32", "f16", "bf16"};

int index_of(const std::vector<std::string> &v, const std::string &s, const char *what) {
  for (size_t i = 0; i < v.size(); i++)
    if (v[i] == s) return (int)i;
  throw std::runtime_error(std::string("unknown ") + what + ": " + s);
}

class LockExchange {
 public:
  LockExchange(int nx, int nz, int q_scalar, const std::string &geometry, const std::string &storage,
               const std::string &wall, bool mrt, double dz, double dt, std::vector<double> x,
               std::vector<double> z, std::vector<double> wx, std::vector<double> wz, double tau, double taus,
               double rhoL, double rhoH, double phi, double rho_sal, double g_bouss, double s_ref,
               std::vector<double> M, std::vector<double> Minv, std::vector<double> S, std::vector<double> s0)
      : nx_(nx), nz_(nz), q_(q_scalar) {
    ipcu_sim_config c{};
    c.nx = nx;
    c.nz = nz;
    c.q_scalar = q_scalar;
    c.geometry = index_of(kGeo, geometry, "geometry");
    c.storage = index_of(kStore, storage, "storage");
    c.wall = wall == "bb" ? IPCU_WALL_BB : (wall == "slip" ? IPCU_WALL_SLIP : -1);
    c.mrt = mrt ? 1 : 0;
    c.dz = dz;
    c.dt = dt;
    auto opt = [](const std::vector<double> &v, size_t n) -> const double * {
      if (v.empty()) return nullptr;
      if (v.size() != n) throw std::runtime_error("coordinate/matrix array of wrong length");
      return v.data();
    };
    c.x = opt(x, nx);
    c.z = opt(z, nz);
    c.wx = opt(wx, nx);
    c.wz = opt(wz, nz);
    c.tau = tau;
    c.taus = taus;
    c.rhoL = rhoL;
    c.rhoH = rhoH;
    c.phi = phi;
    c.rho_sal = rho_sal;
    c.g_bouss = g_bouss;
    c.s_ref = s_ref;
    c.M = opt(M, 81);
    c.Minv = opt(Minv, 81);
    c.S = opt(S, 9);
    check(ipcu_sim_create(&c, opt(s0, (size_t)nx * nz), nullptr, &sim_), "ipcu_sim_create");
  }
  ~LockExchange() { ipcu_sim_destroy(sim_); }
  void step(int64_t n) { check(ipcu_sim_step(sim_, n), "step"); }
  void step_graph(int64_t n, int chunk) { check(ipcu_sim_step_graph(sim_, n, chunk), "step_graph"); }
  py::array_t<double> get(const std::string &field) {
    const int64_t N = (int64_t)nx_ * nz_;
    const int64_t q = field == "f" ? 9 : (field == "g" ? q_ : 1);
    std::vector<py::ssize_t> shape = q > 1 || field == "f" || field == "g"
                                         ? std::vector<py::ssize_t>{q, nz_, nx_}
                                         : std::vector<py::ssize_t>{nz_, nx_};
    py::array_t<double> out(shape);
    check(ipcu_sim_get(sim_, field.c_str(), out.mutable_data(), q * N), "get");
    return out;
  }
  std::pair<double, double> totals() {
    double p = 0, s = 0;
    check(ipcu_sim_totals(sim_, &p, &s), "totals");
    return {p, s};
  }
  int64_t cells() const { return ipcu_sim_cells(sim_); }

 private:
  int nx_, nz_, q_;
  ipcu_sim *sim_ = nullptr;
};

}  // namespace

PYBIND11_MODULE(my_module, m) {
  m.doc() = "IP_CU_LBM B200 Python boundary: GPUMemory, compute_on_gpu, LockExchange";
  py::class_<GPUMemory>(m, "GPUMemory")
      .def(py::init<size_t>())
      .def("set", &GPUMemory::set)
      .def("get", &GPUMemory::get)
      .def("size", &GPUMemory::size);
  m.def("compute_on_gpu", &compute_on_gpu);
  py::class_<LockExchange>(m, "LockExchange")
      .def(py::init<int, int, int, const std::string &, const std::string &, const std::string &, bool, double, double,
                    std::vector<double>, std::vector<double>, std::vector<double>, std::vector<double>, double,
                    double, double, double, double, double, double, double, std::vector<double>,
                    std::vector<double>, std::vector<double>, std::vector<double>>(),
           py::arg("nx"), py::arg("nz"), py::arg("q_scalar") = 5, py::arg("geometry") = "uniform",
           py::arg("storage") = "f32", py::arg("wall") = "bb", py::arg("mrt") = false, py::arg("dz") = 1.0,
           py::arg("dt") = 1.0, py::arg("x") = std::vector<double>{}, py::arg("z") = std::vector<double>{},
           py::arg("wx") = std::vector<double>{}, py::arg("wz") = std::vector<double>{}, py::arg("tau") = 0.53,
           py::arg("taus") = 0.503, py::arg("rhoL") = 1.0, py::arg("rhoH") = 1.0, py::arg("phi") = 1.0,
           py::arg("rho_sal") = 0.0, py::arg("g_bouss") = 1e-4, py::arg("s_ref") = 0.5,
           py::arg("M") = std::vector<double>{}, py::arg("Minv") = std::vector<double>{},
           py::arg("S") = std::vector<double>{}, py::arg("s0") = std::vector<double>{})
      .def("step", &LockExchange::step, py::arg("n") = 1)
      .def("step_graph", &LockExchange::step_graph, py::arg("n"), py::arg("chunk") = 64)
      .def("get", &LockExchange::get)
      .def("totals", &LockExchange::totals)
      .def("cells", &LockExchange::cells);
}
