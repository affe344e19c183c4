// _ftlm_core — the reference's pybind11 module (python/bindings.cpp of PeizhiMai/FTLM_extended_Hubbard:
// HubbardParams, version_string, nsites, lines 8-39) with the GPU hot path behind it on torch tensors.
//
// Kept from the reference module, same names, fields, defaults and keyword arguments:
//   HubbardParams(Lx=2, Ly=2, t=1, tp=0, U=0, V=0, phi_x=0, phi_y=0), version_string(), nsites(params).
// Added (all compute goes through the C ABI of libftlm_gpu.so, include/ftlm_gpu.h):
//   Sector(params, n_up, n_down)      FockBasis + geometry of one (N_up, N_dn) sector on the GPU
//     .dim(), .up_mask(i), .down_mask(i), .index_of(up, down)      FockBasis (include/ftlm/fock_basis.hpp:13-24)
//     .apply(x) -> y, .apply(x, out=y)  apply_extended_hubbard on CUDA complex128 tensors
//                                       (include/ftlm/hubbard_hamiltonian.hpp:13-16), torch's current stream
//     .lanczos(max_steps, seed, start) -> (alpha, beta)              lanczos_tridiagonal (include/ftlm/lanczos.hpp:55-59)
//     .ftlm(betas, n_random, lanczos_steps, seed, start) -> (ln Z, E)  ftlm_log_partition_complex
//                                                                      (include/ftlm/ftlm_thermo.hpp:41-50)
//     .batched_ftlm(betas, n_random, lanczos_steps, seed) -> (ln Z, E)  complex64 32-chain blocks
//   grand_canonical_sweep(params, n_random, lanczos_steps, seed, temperatures, mus, method, start)
//       the sector + mu loops of benchmarks/bench_ftlm_nmu_rect.cpp:138-219 -> dict of float64 tensors
//   GrandCanonicalLogZ (torch::autograd::Function) and grand_canonical_logz(theta, Lx, Ly, ...):
//       ln Z_GC at theta = (U, V, t', mu, beta) with the hand-written backward d ln Z_GC / d theta.
// Errors of the C ABI become Python RuntimeError (ValueError for FTLM_ERR_INVALID, as the
// reference's std::invalid_argument).
#include <torch/extension.h>

#include <pybind11/stl.h>

#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "ftlm/hubbard_params.hpp"
#include "ftlm/version.hpp"
#include "ftlm_gpu.h"

namespace py = pybind11;

namespace {

void check(int status) {
  if (status == FTLM_OK) return;
  const std::string msg = ftlm_gpu_last_error();
  if (status == FTLM_ERR_INVALID) throw std::invalid_argument(msg);
  throw std::runtime_error("ftlm_gpu error " + std::to_string(status) + ": " + msg);
}

ftlm_params c_params(const ftlm::HubbardParams& p) {
  return ftlm_params{p.Lx, p.Ly, p.t, p.tp, p.U, p.V, p.phi_x, p.phi_y};
}

int start_mode(const std::string& s) {
  if (s == "reference") return FTLM_START_REFERENCE;
  if (s == "philox") return FTLM_START_PHILOX;
  throw std::invalid_argument("start must be 'reference' or 'philox'");
}

int method_id(const std::string& m) {
  if (m == "plain") return 0;
  if (m == "batched") return 1;
  throw std::invalid_argument("method must be 'plain' or 'batched'");
}

torch::Tensor f64(const std::vector<double>& v) {
  return torch::tensor(v, torch::dtype(torch::kFloat64));
}

std::vector<double> host_doubles(const torch::Tensor& t) {
  torch::Tensor c = t.detach().to(torch::kCPU, torch::kFloat64).contiguous().reshape({-1});
  return std::vector<double>(c.data_ptr<double>(), c.data_ptr<double>() + c.numel());
}

// One (N_up, N_dn) sector: FockBasis + its device tables (ftlm_gpu_sector_*).
class Sector {
 public:
  Sector(const ftlm::HubbardParams& p, int n_up, int n_down) {
    const ftlm_params cp = c_params(p);
    ftlm_sector* s = nullptr;
    check(ftlm_gpu_sector_create(&cp, n_up, n_down, &s));
    h_.reset(s, [](ftlm_sector* q) { ftlm_gpu_sector_destroy(q); });
    long long d = 0;
    check(ftlm_gpu_sector_dim(s, &d));
    dim_ = d;
  }
  long long dim() const { return dim_; }
  uint64_t up_mask(long long i) const { return state(i).first; }
  uint64_t down_mask(long long i) const { return state(i).second; }
  long long index_of(uint64_t up, uint64_t dn) const {
    long long idx = -1;
    check(ftlm_gpu_sector_index_of(h_.get(), up, dn, &idx));
    return idx;
  }

  // y = H x on CUDA complex128 vectors (apply_extended_hubbard; y overwritten), torch's current stream.
  torch::Tensor apply(const torch::Tensor& x, c10::optional<torch::Tensor> out) {
    TORCH_CHECK(x.is_cuda(), "apply: x must be a CUDA tensor (the GPU path has no CPU fallback)");
    TORCH_CHECK(x.scalar_type() == torch::kComplexDouble, "apply: x must be complex128");
    TORCH_CHECK(x.is_contiguous() && x.numel() == dim_, "apply: x must be contiguous with dim() elements");
    torch::Tensor y = out.has_value() ? *out : torch::empty_like(x);
    TORCH_CHECK(y.is_cuda() && y.scalar_type() == torch::kComplexDouble && y.is_contiguous() && y.numel() == dim_ &&
                    y.device() == x.device(),
                "apply: out must be a contiguous complex128 CUDA tensor of dim() elements on x's device");
    c10::cuda::CUDAGuard guard(x.device());
    const cudaStream_t st = c10::cuda::getCurrentCUDAStream(x.device().index()).stream();
    check(ftlm_gpu_apply(h_.get(), reinterpret_cast<const double*>(x.data_ptr()), reinterpret_cast<double*>(y.data_ptr()),
                         st));
    return y;
  }

  py::tuple lanczos(int max_steps, unsigned seed, const std::string& start) {
    std::vector<double> a(static_cast<size_t>(std::max(1, max_steps))), b(a.size());
    int nb = 0, used = 0;
    check(ftlm_gpu_lanczos(h_.get(), max_steps, seed, start_mode(start), a.data(), b.data(), &nb, &used));
    a.resize(static_cast<size_t>(used));
    b.resize(static_cast<size_t>(nb));
    return py::make_tuple(f64(a), f64(b));
  }

  py::tuple ftlm(const std::vector<double>& bt, int n_random, int lanczos_steps, unsigned seed, const std::string& start) {
    std::vector<double> lnz(bt.size()), en(bt.size());
    check(ftlm_gpu_ftlm_sector(h_.get(), bt.data(), static_cast<int>(bt.size()), n_random, lanczos_steps, seed,
                               start_mode(start), lnz.data(), en.data()));
    return py::make_tuple(f64(lnz), f64(en));
  }

  py::tuple batched_ftlm(const std::vector<double>& bt, int n_random, int lanczos_steps, unsigned seed) {
    std::vector<double> lnz(bt.size()), en(bt.size());
    check(ftlm_gpu_batched_ftlm_sector(h_.get(), bt.data(), static_cast<int>(bt.size()), n_random, lanczos_steps, seed,
                                       lnz.data(), en.data()));
    return py::make_tuple(f64(lnz), f64(en));
  }

 private:
  std::pair<uint64_t, uint64_t> state(long long i) const {
    if (i < 0 || i >= dim_) throw py::index_error("state index out of range");
    uint64_t u = 0, d = 0;
    check(ftlm_gpu_sector_state(h_.get(), i, &u, &d));
    return {u, d};
  }
  std::shared_ptr<ftlm_sector> h_;
  long long dim_ = 0;
};

py::dict grand_canonical_sweep(const ftlm::HubbardParams& p, int n_random, int lanczos_steps, unsigned seed,
                               const std::vector<double>& T, const std::vector<double>& mu, const std::string& method,
                               const std::string& start) {
  std::vector<double> bt(T.size());
  for (size_t i = 0; i < T.size(); ++i) {
    if (!(T[i] > 0.0)) throw std::invalid_argument("temperatures must be > 0");
    bt[i] = 1.0 / T[i];
  }
  const int n = ftlm::nsites(p);
  const int nsec = (n + 1) * (n + 1);
  const int nb = static_cast<int>(bt.size()), nm = static_cast<int>(mu.size());
  std::vector<double> lz(static_cast<size_t>(nsec) * nb), es(lz.size()), g(static_cast<size_t>(nb) * nm),
      na(g.size()), ea(g.size());
  const ftlm_params cp = c_params(p);
  if (method_id(method) == 1)
    check(ftlm_gpu_batched_sweep(&cp, n_random, lanczos_steps, seed, bt.data(), nb, mu.data(), nm, lz.data(), es.data(),
                                 g.data(), na.data(), ea.data()));
  else
    check(ftlm_gpu_gc_sweep(&cp, n_random, lanczos_steps, seed, start_mode(start), bt.data(), nb, mu.data(), nm,
                            lz.data(), es.data(), g.data(), na.data(), ea.data()));
  py::dict d;
  d["lnz_sector"] = f64(lz).reshape({nsec, nb});
  d["energy_sector"] = f64(es).reshape({nsec, nb});
  d["lnz"] = f64(g).reshape({nb, nm});
  d["n"] = f64(na).reshape({nb, nm});
  d["energy"] = f64(ea).reshape({nb, nm});
  return d;
}

// Lattice and chain settings of one differentiable ln Z_GC evaluation.
struct GcConfig {
  int Lx = 2, Ly = 2;
  double t = 1.0, phi_x = 0.0, phi_y = 0.0;
  int R = 8, M = 40;
  unsigned seed = 1;
  int method = 1, start = FTLM_START_REFERENCE;
  ftlm_params params(const double* th) const { return ftlm_params{Lx, Ly, t, th[2], th[0], th[1], phi_x, phi_y}; }
};

// ln Z_GC(U, V, t', mu, beta): forward = ftlm_gpu_gc_logz (every sector's chains, converged
// quadrature, log-sum-exp); backward = ftlm_gpu_gc_logz_grad (d/dmu = beta <N>, d/dbeta = <mu N - E>,
// d/d(U, V, t') from the chains replayed from their seeds), scaled by the incoming gradient.
class GrandCanonicalLogZ : public torch::autograd::Function<GrandCanonicalLogZ> {
 public:
  static torch::Tensor forward(torch::autograd::AutogradContext* ctx, const torch::Tensor& theta, int64_t Lx,
                               int64_t Ly, double t, double phi_x, double phi_y, int64_t R, int64_t M, int64_t seed,
                               int64_t method, int64_t start) {
    TORCH_CHECK(theta.numel() == 5, "theta must hold (U, V, t', mu, beta)");
    GcConfig c{static_cast<int>(Lx), static_cast<int>(Ly), t, phi_x, phi_y, static_cast<int>(R), static_cast<int>(M),
               static_cast<unsigned>(seed), static_cast<int>(method), static_cast<int>(start)};
    const std::vector<double> th = host_doubles(theta);
    const int n = c.Lx * c.Ly;
    const int nsec = (n + 1) * (n + 1);
    std::vector<double> lnz(static_cast<size_t>(nsec)), en(lnz.size());
    double lnZ = 0.0;
    const ftlm_params cp = c.params(th.data());
    check(ftlm_gpu_gc_logz(&cp, th[3], th[4], c.R, c.M, c.seed, c.method, c.start, lnz.data(), en.data(), &lnZ));
    ctx->save_for_backward({theta});
    ctx->saved_data["table"] = torch::cat({f64(lnz), f64(en)});
    ctx->saved_data["cfg"] = std::vector<int64_t>{Lx, Ly, R, M, seed, method, start};
    ctx->saved_data["lat"] = std::vector<double>{t, phi_x, phi_y};
    return torch::full({}, lnZ, theta.options().dtype(torch::kFloat64));
  }

  static torch::autograd::variable_list backward(torch::autograd::AutogradContext* ctx,
                                                 torch::autograd::variable_list grad_out) {
    const torch::Tensor theta = ctx->get_saved_variables()[0];
    const std::vector<int64_t> k = ctx->saved_data["cfg"].toIntVector();
    const std::vector<double> lat = ctx->saved_data["lat"].toDoubleVector();
    GcConfig c{static_cast<int>(k[0]), static_cast<int>(k[1]), lat[0], lat[1], lat[2], static_cast<int>(k[2]),
               static_cast<int>(k[3]), static_cast<unsigned>(k[4]), static_cast<int>(k[5]), static_cast<int>(k[6])};
    const std::vector<double> table = host_doubles(ctx->saved_data["table"].toTensor());
    const size_t nsec = table.size() / 2;
    const std::vector<double> th = host_doubles(theta);
    std::vector<double> g(5);
    const ftlm_params cp = c.params(th.data());
    check(ftlm_gpu_gc_logz_grad(&cp, th[3], th[4], c.R, c.M, c.seed, c.method, c.start, table.data(),
                                table.data() + nsec, g.data()));
    torch::Tensor grad = f64(g).to(theta.device(), theta.scalar_type()).reshape(theta.sizes()) * grad_out[0];
    torch::autograd::variable_list out(11);
    out[0] = grad;
    return out;
  }
};

torch::Tensor grand_canonical_logz(const torch::Tensor& theta, int Lx, int Ly, int n_random, int lanczos_steps,
                                   unsigned seed, const std::string& method, const std::string& start, double t,
                                   double phi_x, double phi_y) {
  return GrandCanonicalLogZ::apply(theta, Lx, Ly, t, phi_x, phi_y, n_random, lanczos_steps, static_cast<int64_t>(seed),
                                   method_id(method), start_mode(start));
}

}  // namespace

PYBIND11_MODULE(_ftlm_core, m) {
  m.doc() = "ftlm_extended_hubbard core: the reference's bindings plus the B200 hot path on torch tensors";

  py::class_<ftlm::HubbardParams>(m, "HubbardParams")
      .def(py::init<>())
      .def(py::init([](int Lx, int Ly, double t, double tp, double U, double V, double phi_x, double phi_y) {
             ftlm::HubbardParams p;
             p.Lx = Lx;
             p.Ly = Ly;
             p.t = t;
             p.tp = tp;
             p.U = U;
             p.V = V;
             p.phi_x = phi_x;
             p.phi_y = phi_y;
             return p;
           }),
           py::arg("Lx") = 2, py::arg("Ly") = 2, py::arg("t") = 1.0, py::arg("tp") = 0.0, py::arg("U") = 0.0,
           py::arg("V") = 0.0, py::arg("phi_x") = 0.0, py::arg("phi_y") = 0.0)
      .def_readwrite("Lx", &ftlm::HubbardParams::Lx)
      .def_readwrite("Ly", &ftlm::HubbardParams::Ly)
      .def_readwrite("t", &ftlm::HubbardParams::t)
      .def_readwrite("tp", &ftlm::HubbardParams::tp)
      .def_readwrite("U", &ftlm::HubbardParams::U)
      .def_readwrite("V", &ftlm::HubbardParams::V)
      .def_readwrite("phi_x", &ftlm::HubbardParams::phi_x)
      .def_readwrite("phi_y", &ftlm::HubbardParams::phi_y);

  m.def("version_string", &ftlm::version_string);
  m.def("nsites", &ftlm::nsites, py::arg("params"));

  py::class_<Sector>(m, "Sector")
      .def(py::init<const ftlm::HubbardParams&, int, int>(), py::arg("params"), py::arg("n_up"), py::arg("n_down"))
      .def("dim", &Sector::dim)
      .def("up_mask", &Sector::up_mask, py::arg("idx"))
      .def("down_mask", &Sector::down_mask, py::arg("idx"))
      .def("index_of", &Sector::index_of, py::arg("up"), py::arg("down"))
      .def("apply", &Sector::apply, py::arg("x"), py::arg("out") = py::none())
      .def("lanczos", &Sector::lanczos, py::arg("max_steps"), py::arg("seed"), py::arg("start") = "reference")
      .def("ftlm", &Sector::ftlm, py::arg("betas"), py::arg("n_random"), py::arg("lanczos_steps"), py::arg("seed"),
           py::arg("start") = "reference")
      .def("batched_ftlm", &Sector::batched_ftlm, py::arg("betas"), py::arg("n_random"), py::arg("lanczos_steps"),
           py::arg("seed"));

  m.def("grand_canonical_sweep", &grand_canonical_sweep, py::arg("params"), py::arg("n_random"),
        py::arg("lanczos_steps"), py::arg("seed"), py::arg("temperatures"), py::arg("mus"),
        py::arg("method") = "plain", py::arg("start") = "reference");
  m.def("grand_canonical_logz", &grand_canonical_logz, py::arg("theta"), py::arg("Lx"), py::arg("Ly"),
        py::arg("n_random"), py::arg("lanczos_steps"), py::arg("seed"), py::arg("method") = "batched",
        py::arg("start") = "reference", py::arg("t") = 1.0, py::arg("phi_x") = 0.0, py::arg("phi_y") = 0.0);
  m.def("release_workspaces", []() { check(ftlm_gpu_batched_release()); });
}
