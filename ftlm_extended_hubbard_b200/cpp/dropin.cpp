// C++ drop-in of the reference's FTLM hot-path API (namespace ftlm) over the C ABI of
// libftlm_gpu.so.  Host orchestration only: every H·v, Lanczos step and quadrature runs in the
// library's CUDA kernels.  Errors become the reference's exceptions (std::invalid_argument for
// bad sectors, std::out_of_range for FockBasis indices, std::runtime_error otherwise).
#include <cmath>
#include <complex>
#include <cstring>
#include <exception>
#include <limits>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "ftlm/fock_basis.hpp"
#include "ftlm/ftlm_thermo.hpp"
#include "ftlm/hubbard_hamiltonian.hpp"
#include "ftlm/hubbard_params.hpp"
#include "ftlm/lanczos.hpp"
#include "ftlm/lanczos_engine.hpp"
#include "ftlm/lattice.hpp"
#include "ftlm/version.hpp"
#include "ftlm_gpu.h"

namespace ftlm {

namespace {

using cd = std::complex<double>;

void check(int rc) {
  if (rc == FTLM_OK) return;
  const std::string msg = ftlm_gpu_last_error();
  if (rc == FTLM_ERR_INVALID) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

// Device sectors keyed by everything apply_extended_hubbard depends on.
std::mutex g_cache_mu;
std::map<std::string, ftlm_sector*> g_cache;

std::string key_of(const FockBasis& b, const HubbardParams& p, const std::vector<SpinfulHopping>& h,
                   const std::vector<NearestPair>& pr) {
  std::string k;
  auto put = [&k](const void* v, size_t n) { k.append(static_cast<const char*>(v), n); };
  const int hdr[3] = {b.n_sites(), b.n_up(), b.n_down()};
  put(hdr, sizeof(hdr));
  put(&p.U, sizeof(double));
  put(&p.V, sizeof(double));
  for (const auto& x : h) {
    const int i3[3] = {x.from, x.to, x.spin};
    const double c2[2] = {x.coeff.real(), x.coeff.imag()};
    put(i3, sizeof(i3));
    put(c2, sizeof(c2));
  }
  for (const auto& x : pr) {
    const int i2[2] = {x.i, x.j};
    put(i2, sizeof(i2));
  }
  return k;
}

ftlm_sector* sector_for(const HubbardParams& p, const FockBasis& b, const std::vector<SpinfulHopping>& h,
                        const std::vector<NearestPair>& pr) {
  const std::string k = key_of(b, p, h, pr);
  std::lock_guard<std::mutex> lock(g_cache_mu);
  auto it = g_cache.find(k);
  if (it != g_cache.end()) return it->second;
  if (g_cache.size() >= 8) {
    for (auto& kv : g_cache) ftlm_gpu_sector_destroy(kv.second);
    g_cache.clear();
  }
  std::vector<ftlm_hop> hv(h.size());
  for (size_t i = 0; i < h.size(); ++i) hv[i] = ftlm_hop{h[i].from, h[i].to, h[i].spin, h[i].coeff.real(), h[i].coeff.imag()};
  std::vector<ftlm_pair> pv(pr.size());
  for (size_t i = 0; i < pr.size(); ++i) pv[i] = ftlm_pair{pr[i].i, pr[i].j};
  ftlm_sector* s = nullptr;
  check(ftlm_gpu_sector_create_hops(b.n_sites(), b.n_up(), b.n_down(), p.U, p.V, hv.data(), static_cast<int>(hv.size()),
                                    pv.data(), static_cast<int>(pv.size()), &s));
  g_cache[k] = s;
  return s;
}

// Calls a C++ operator from the C ABI's host callback; an exception is kept and rethrown after
// the C call returns (the vector handed back is zero, which ends the recurrence).
struct HostOp {
  const std::function<void(const cd*, cd*)>* f = nullptr;
  long long dim = 0;
  std::exception_ptr err;
};

void host_trampoline(const double* x, double* y, void* ctx) {
  auto* op = static_cast<HostOp*>(ctx);
  if (op->err) {
    std::memset(y, 0, static_cast<size_t>(op->dim) * 2 * sizeof(double));
    return;
  }
  try {
    (*op->f)(reinterpret_cast<const cd*>(x), reinterpret_cast<cd*>(y));
  } catch (...) {
    op->err = std::current_exception();
    std::memset(y, 0, static_cast<size_t>(op->dim) * 2 * sizeof(double));
  }
}

double log_partition(int dim, const std::function<void(const cd*, cd*)>& apply_h, double beta, const FtlmParams& par,
                     const std::function<double()>& h00) {
  if (dim <= 0) return -std::numeric_limits<double>::infinity();
  if (dim == 1) return -beta * h00();
  const int R = std::max(1, par.n_random);
  const int M = std::max(1, par.lanczos_steps);
  std::vector<double> A(static_cast<size_t>(R) * M, 0.0), B(static_cast<size_t>(R) * M, 0.0);
  std::vector<int> used(static_cast<size_t>(R), 0);
  for (int r = 0; r < R; ++r) {
    std::vector<double> a, b;
    const unsigned seed_r = par.seed + static_cast<unsigned>(r) * 100003u;
    used[static_cast<size_t>(r)] = lanczos_tridiagonal(dim, apply_h, M, seed_r, &a, &b);
    std::copy(a.begin(), a.end(), A.begin() + static_cast<long>(r) * M);
    std::copy(b.begin(), b.end(), B.begin() + static_cast<long>(r) * M);
  }
  std::vector<double> lq(static_cast<size_t>(R)), eq(static_cast<size_t>(R));
  check(ftlm_gpu_tridiag_quadrature(A.data(), B.data(), used.data(), R, M, &beta, 1, lq.data(), eq.data()));
  double lnz = 0.0, e = 0.0;
  check(ftlm_gpu_ftlm_combine(lq.data(), eq.data(), used.data(), R, 1, std::log(static_cast<double>(dim)), &lnz, &e));
  return lnz;
}

}  // namespace

int nsites(const HubbardParams& p) { return p.Lx * p.Ly; }

const char* version_string() { return ftlm_gpu_version_string(); }

void build_hubbard_geometry(const HubbardParams& p, const RectLattice& lat, std::vector<SpinfulHopping>* hoppings,
                            std::vector<NearestPair>* nn_pairs) {
  ftlm_params cp{lat.Lx, lat.Ly, p.t, p.tp, p.U, p.V, p.phi_x, p.phi_y};
  int nh = 0, np = 0;
  check(ftlm_gpu_build_geometry(&cp, nullptr, 0, &nh, nullptr, 0, &np));
  std::vector<ftlm_hop> h(static_cast<size_t>(nh));
  std::vector<ftlm_pair> q(static_cast<size_t>(np));
  check(ftlm_gpu_build_geometry(&cp, h.data(), nh, &nh, q.data(), np, &np));
  hoppings->clear();
  nn_pairs->clear();
  for (const auto& x : h) hoppings->push_back(SpinfulHopping{x.from, x.to, x.spin, cd(x.coeff_re, x.coeff_im)});
  for (const auto& x : q) nn_pairs->push_back(NearestPair{x.i, x.j});
}

FockBasis::FockBasis(int n_sites, int n_up, int n_down) : n_sites_(n_sites), n_up_(n_up), n_down_(n_down) {
  check(ftlm_gpu_sector_create_host(n_sites, n_up, n_down, 0.0, 0.0, nullptr, 0, nullptr, 0, &h_));
  long long d = 0;
  check(ftlm_gpu_sector_dim(h_, &d));
  dim_ = static_cast<int>(d);
}

FockBasis::~FockBasis() { ftlm_gpu_sector_destroy(h_); }

uint64_t FockBasis::up_mask(int idx) const {
  if (idx < 0 || idx >= dim_) throw std::out_of_range("FockBasis::up_mask");
  uint64_t u = 0, d = 0;
  check(ftlm_gpu_sector_state(h_, idx, &u, &d));
  return u;
}

uint64_t FockBasis::down_mask(int idx) const {
  if (idx < 0 || idx >= dim_) throw std::out_of_range("FockBasis::down_mask");
  uint64_t u = 0, d = 0;
  check(ftlm_gpu_sector_state(h_, idx, &u, &d));
  return d;
}

int FockBasis::index_of(uint64_t up, uint64_t down) const {
  long long i = -1;
  check(ftlm_gpu_sector_index_of(h_, up, down, &i));
  return static_cast<int>(i);
}

void apply_extended_hubbard(const HubbardParams& p, const FockBasis& basis, const std::vector<SpinfulHopping>& hoppings,
                            const std::vector<NearestPair>& nn_pairs, const cd* x, cd* y) {
  ftlm_sector* s = sector_for(p, basis, hoppings, nn_pairs);
  check(ftlm_gpu_apply_host(s, reinterpret_cast<const double*>(x), reinterpret_cast<double*>(y)));
}

int lanczos_tridiagonal(int dim, const std::function<void(const cd*, cd*)>& apply_h, int max_steps, unsigned seed,
                        std::vector<double>* alpha, std::vector<double>* beta, LanczosComplexWorkspace* ws) {
  (void)ws;
  alpha->clear();
  beta->clear();
  if (dim <= 0 || max_steps <= 0) return 0;
  std::vector<double> a(static_cast<size_t>(max_steps)), b(static_cast<size_t>(max_steps));
  int nb = 0, used = 0;
  HostOp op{&apply_h, dim, nullptr};
  const int rc = ftlm_gpu_lanczos_host_op(dim, host_trampoline, &op, max_steps, seed, FTLM_START_REFERENCE, a.data(),
                                          b.data(), &nb, &used);
  if (op.err) std::rethrow_exception(op.err);
  check(rc);
  alpha->assign(a.begin(), a.begin() + used);
  beta->assign(b.begin(), b.begin() + nb);
  return used;
}

std::pair<double, double> tridiagonal_extrema(const std::vector<double>& alpha, const std::vector<double>& beta,
                                              int steps) {
  const int n = steps;
  if (n <= 0) return {0.0, 0.0};
  if (n == 1) return {alpha[0], alpha[0]};
  std::vector<double> a(alpha.begin(), alpha.begin() + n), b(static_cast<size_t>(n), 0.0), lam(static_cast<size_t>(n)),
      w(static_cast<size_t>(n));
  for (int i = 0; i < n - 1 && i < static_cast<int>(beta.size()); ++i) b[static_cast<size_t>(i)] = beta[static_cast<size_t>(i)];
  int nn = n;
  check(ftlm_gpu_tridiag_eig(a.data(), b.data(), &nn, 1, n, 120, 1e-15, lam.data(), w.data()));
  double lo = std::numeric_limits<double>::infinity(), hi = -lo;
  for (double v : lam) {
    lo = std::min(lo, v);
    hi = std::max(hi, v);
  }
  return {lo, hi};
}

LanczosExtrema lanczos_extrema(int dim, const std::function<void(const cd*, cd*)>& apply_h, int max_steps, unsigned seed) {
  LanczosExtrema out{};
  std::vector<double> alpha, beta;
  const int used = lanczos_tridiagonal(dim, apply_h, max_steps, seed, &alpha, &beta);
  out.steps_used = used;
  if (used == 0) return out;
  std::vector<double> bt;
  if (used >= 2) bt.assign(beta.begin(), beta.begin() + (used - 1));
  const auto mm = tridiagonal_extrema(alpha, bt, used);
  out.min_eval = mm.first;
  out.max_eval = mm.second;
  return out;
}

double ftlm_log_partition_complex(int dim, const std::function<void(const cd*, cd*)>& apply_h, double beta,
                                  const FtlmParams& par) {
  return log_partition(dim, apply_h, beta, par, [&]() {
    cd x[1] = {cd(1.0, 0.0)}, y[1] = {cd(0.0, 0.0)};
    apply_h(x, y);
    return y[0].real();
  });
}

double ftlm_log_partition_real(int dim, const std::function<void(const double*, double*)>& apply_real, double beta,
                               const FtlmParams& par) {
  std::vector<double> xr, xi, yr, yi;
  if (dim > 1) {
    xr.resize(static_cast<size_t>(dim));
    xi.resize(static_cast<size_t>(dim));
    yr.resize(static_cast<size_t>(dim));
    yi.resize(static_cast<size_t>(dim));
  }
  // Real-symmetric H on a complex vector: H(re) + i H(im), two real applies per step.
  const std::function<void(const cd*, cd*)> apply_c = [&](const cd* x, cd* y) {
    for (int i = 0; i < dim; ++i) {
      xr[static_cast<size_t>(i)] = x[i].real();
      xi[static_cast<size_t>(i)] = x[i].imag();
    }
    apply_real(xr.data(), yr.data());
    apply_real(xi.data(), yi.data());
    for (int i = 0; i < dim; ++i) y[i] = cd(yr[static_cast<size_t>(i)], yi[static_cast<size_t>(i)]);
  };
  return log_partition(dim, apply_c, beta, par, [&]() {
    double x[1] = {1.0}, y[1] = {0.0};
    apply_real(x, y);
    return y[0];
  });
}

}  // namespace ftlm
