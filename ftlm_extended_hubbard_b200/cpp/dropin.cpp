// C++ drop-in of the reference's FTLM hot-path API (namespace ftlm) over the C ABI of
// libftlm_gpu.so.  Host orchestration only: every H·v, Lanczos step and quadrature runs in the
// library's CUDA kernels.  Errors become the reference's exceptions (std::invalid_argument for
// bad sectors, std::out_of_range for FockBasis indices, std::runtime_error otherwise).
#include <algorithm>
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
#include "ftlm/symmetry/orbit_k_block_basis.hpp"
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

// ---- translation-orbit momentum blocks (include/ftlm/symmetry/orbit_k_block_basis.hpp) ---------
namespace symmetry {

namespace {

// Site (x, y) = y*lx + x goes to ((y+dy) mod ly)*lx + (x+dx) mod lx.
int shift_site(int site, int lx, int ly, int dx, int dy) {
  return ((site / lx + dy) % ly) * lx + (site % lx + dx) % lx;
}

std::uint16_t shift_bits(std::uint16_t m, int lx, int ly, int dx, int dy) {
  std::uint32_t out = 0;
  for (int site = 0; site < lx * ly; ++site)
    if ((m >> site) & 1u) out |= 1u << shift_site(site, lx, ly, dx, dy);
  return static_cast<std::uint16_t>(out);
}

// (-1)^(inversions of the occupied modes 2*site+spin, in site order, after the translation).
double shift_sign(RawState s, int lx, int ly, int dx, int dy) {
  int modes[32];
  int n = 0;
  for (int site = 0; site < lx * ly; ++site) {
    const int t = shift_site(site, lx, ly, dx, dy);
    if ((s.up >> site) & 1u) modes[n++] = 2 * t;
    if ((s.dn >> site) & 1u) modes[n++] = 2 * t + 1;
  }
  int inv = 0;
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) inv += modes[i] > modes[j] ? 1 : 0;
  return (inv & 1) ? -1.0 : 1.0;
}

RawState canonical(RawState s, int lx, int ly) {
  std::uint32_t best = pack_raw_state(s);
  for (int dy = 0; dy < ly; ++dy)
    for (int dx = 0; dx < lx; ++dx) {
      const RawState t{shift_bits(s.up, lx, ly, dx, dy), shift_bits(s.dn, lx, ly, dx, dy)};
      best = std::min(best, pack_raw_state(t));
    }
  return unpack_raw_state(best);
}

ftlm_sector* bare_sector(const FockBasis& fb, int lx, int ly) {
  ftlm_sector* s = nullptr;
  check(ftlm_gpu_sector_create_hops(fb.n_sites(), fb.n_up(), fb.n_down(), 0.0, 0.0, nullptr, 0, nullptr, 0, &s));
  const int rc = ftlm_gpu_sector_set_lattice(s, lx, ly);
  if (rc != FTLM_OK) {
    const std::string msg = ftlm_gpu_last_error();
    ftlm_gpu_sector_destroy(s);
    throw std::invalid_argument(msg);
  }
  return s;
}

// Device sector + orbit block per (operator, K, tolerance); both destroyed together on eviction.
struct OrbitSlot {
  ftlm_sector* s = nullptr;
  ftlm_orbit* o = nullptr;
};
std::mutex g_orbit_mu;
std::map<std::string, OrbitSlot> g_orbits;

}  // namespace

bool OrbitKBlockBasis::build(const FockBasis& fb, MomentumSector Ksec, double survive_tol) {
  entries_.clear();
  rep_pack_to_row_.clear();
  survive_tol_ = survive_tol;
  K = Ksec;
  lx = K.lx;
  ly = K.ly;
  if (fb.n_sites() > 16)
    throw std::invalid_argument("OrbitKBlockBasis::build: n_sites must be <= 16 (RawState bit width)");
  ftlm_sector* s = bare_sector(fb, lx, ly);
  ftlm_orbit* o = nullptr;
  int rc = ftlm_gpu_orbit_create_ex(s, K.kx, K.ky, survive_tol, &o);
  if (rc != FTLM_OK) {
    ftlm_gpu_sector_destroy(s);
    check(rc);
  }
  long long d = 0;
  ftlm_gpu_orbit_dim(o, &d);
  std::vector<std::uint32_t> rep(static_cast<size_t>(d));
  std::vector<double> A(2 * static_cast<size_t>(d)), absA(static_cast<size_t>(d));
  std::vector<int> osz(static_cast<size_t>(d)), ssz(static_cast<size_t>(d));
  std::vector<long long> oidx(static_cast<size_t>(d));
  rc = ftlm_gpu_orbit_entries_ex(o, rep.data(), A.data(), absA.data(), osz.data(), ssz.data(), oidx.data());
  ftlm_gpu_orbit_destroy(o);
  ftlm_gpu_sector_destroy(s);
  check(rc);
  entries_.resize(static_cast<size_t>(d));
  for (size_t i = 0; i < entries_.size(); ++i) {
    OrbitKRepEntry& e = entries_[i];
    e.rep = unpack_raw_state(rep[i]);
    e.orbit_index = static_cast<std::size_t>(oidx[i]);
    e.orbit_size = static_cast<std::uint16_t>(osz[i]);
    e.stabilizer_size = static_cast<std::uint16_t>(ssz[i]);
    e.A_k = {A[2 * i], A[2 * i + 1]};
    e.abs_A = absA[i];
    rep_pack_to_row_[rep[i]] = i;
  }
  return true;
}

int OrbitKBlockBasis::reduced_index_of_rep(RawState rep) const {
  const auto it = rep_pack_to_row_.find(pack_raw_state(rep));
  return it == rep_pack_to_row_.end() ? -1 : static_cast<int>(it->second);
}

bool OrbitKBlockBasis::map_raw_to_rep(RawState s, int* reduced_index, int* dx, int* dy, double* eta) const {
  if (!reduced_index || !dx || !dy || !eta) return false;
  const RawState rep = canonical(s, lx, ly);
  const auto it = rep_pack_to_row_.find(pack_raw_state(rep));
  if (it == rep_pack_to_row_.end()) return false;
  for (int tdx = 0; tdx < lx; ++tdx)
    for (int tdy = 0; tdy < ly; ++tdy) {
      if (shift_bits(rep.up, lx, ly, tdx, tdy) != s.up || shift_bits(rep.dn, lx, ly, tdx, tdy) != s.dn) continue;
      *reduced_index = static_cast<int>(it->second);
      *dx = tdx;
      *dy = tdy;
      *eta = shift_sign(rep, lx, ly, tdx, tdy);
      return true;
    }
  return false;
}

void apply_orbit_k_block(const HubbardParams& p, const FockBasis& fb, const OrbitKBlockBasis& basis,
                         const std::vector<SpinfulHopping>& hoppings, const std::vector<NearestPair>& nn_pairs,
                         const std::complex<double>* x, std::complex<double>* y) {
  const int dk = basis.dim();
  if (dk <= 0) return;
  std::string k = key_of(fb, p, hoppings, nn_pairs);
  const int kk[4] = {basis.lx, basis.ly, basis.K.kx, basis.K.ky};
  const double tol = basis.survive_tol();
  k.append(reinterpret_cast<const char*>(kk), sizeof(kk));
  k.append(reinterpret_cast<const char*>(&tol), sizeof(tol));
  std::lock_guard<std::mutex> lock(g_orbit_mu);
  auto it = g_orbits.find(k);
  if (it == g_orbits.end()) {
    if (g_orbits.size() >= 4) {
      for (auto& kv : g_orbits) {
        ftlm_gpu_orbit_destroy(kv.second.o);
        ftlm_gpu_sector_destroy(kv.second.s);
      }
      g_orbits.clear();
    }
    std::vector<ftlm_hop> hv(hoppings.size());
    for (size_t i = 0; i < hoppings.size(); ++i)
      hv[i] = ftlm_hop{hoppings[i].from, hoppings[i].to, hoppings[i].spin, hoppings[i].coeff.real(),
                       hoppings[i].coeff.imag()};
    std::vector<ftlm_pair> pv(nn_pairs.size());
    for (size_t i = 0; i < nn_pairs.size(); ++i) pv[i] = ftlm_pair{nn_pairs[i].i, nn_pairs[i].j};
    OrbitSlot slot;
    check(ftlm_gpu_sector_create_hops(fb.n_sites(), fb.n_up(), fb.n_down(), p.U, p.V, hv.data(),
                                      static_cast<int>(hv.size()), pv.data(), static_cast<int>(pv.size()), &slot.s));
    int rc = ftlm_gpu_sector_set_lattice(slot.s, basis.lx, basis.ly);
    if (rc == FTLM_OK) rc = ftlm_gpu_orbit_create_ex(slot.s, basis.K.kx, basis.K.ky, tol, &slot.o);
    if (rc != FTLM_OK) {
      ftlm_gpu_sector_destroy(slot.s);
      check(rc);
    }
    it = g_orbits.emplace(k, slot).first;
  }
  long long d = 0;
  check(ftlm_gpu_orbit_dim(it->second.o, &d));
  if (d != dk) throw std::invalid_argument("apply_orbit_k_block: basis does not belong to this sector");
  check(ftlm_gpu_orbit_apply_host(it->second.o, reinterpret_cast<const double*>(x), reinterpret_cast<double*>(y)));
}

}  // namespace symmetry

}  // namespace ftlm
