// ORACLE — test infrastructure, not product code.
//
// A CPU restatement of the reference's FTLM hot path (PeizhiMai/FTLM_extended_Hubbard),
// written from the reference's documented behaviour.  Only tests/, __graft_entry__.smoke()
// and the cpu_baseline / reference legs of bench.py may load it, and only as the checker.
//
// Pinning: tests/test_oracle_pin.py checks this file against the reference library itself
// (oracle/_ref, built from the reference sources by oracle/Makefile) and against the golden
// vectors under tests/golden/ that were produced from it: bit-exact basis/geometry/matrix
// elements, bit-exact Lanczos alpha/beta in "scatter" mode, identical per-sector ln Z.
//
// Third-party arithmetic: the Lanczos start vectors come from libstdc++'s std::mt19937 and
// std::normal_distribution<double> (GCC 13.3 libstdc++; Marsaglia polar method), called here
// exactly as src/lanczos.cpp:140-169 calls them.  Elementary functions (atan2, cos, sin, exp,
// log, sqrt) are glibc's, as in the reference build.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using cd = std::complex<double>;

struct Hop {
  int from, to, spin;
  cd coeff;
};
struct Pair {
  int i, j;
};

// src/lattice.cpp:9-11 — Peierls factor e^{i(wx phi_x + wy phi_y)}.
cd peierls(int wx, int wy, double phix, double phiy) {
  return std::polar(1.0, static_cast<double>(wx) * phix + static_cast<double>(wy) * phiy);
}

// src/lattice.cpp:13-24 — both directions, both spins; coefficient -t*phase and -t*conj(phase).
void add_bond(int from, int to, cd phase, double t, std::vector<Hop>* hops) {
  if (std::abs(t) < 1e-15) return;
  const cd cij = -t * phase;
  const cd cji = -t * std::conj(phase);
  for (int s = 0; s < 2; ++s) {
    hops->push_back(Hop{from, to, s, cij});
    hops->push_back(Hop{to, from, s, cji});
  }
}

// src/lattice.cpp:38-110 — east, north, then the four diagonals of every site (so each
// diagonal bond is listed twice and each bond of a length-2 direction is listed twice).
void geometry(int Lx, int Ly, double t, double tp, double phix, double phiy, std::vector<Hop>* hops,
              std::vector<Pair>* pairs) {
  hops->clear();
  pairs->clear();
  auto site = [Lx](int x, int y) { return y * Lx + x; };
  auto nn_pair = [pairs](int a, int b) {
    if (a == b) return;
    if (a > b) std::swap(a, b);
    pairs->push_back(Pair{a, b});
  };
  for (int y = 0; y < Ly; ++y) {
    for (int x = 0; x < Lx; ++x) {
      const int i = site(x, y);
      if (Lx > 1) {
        const int nx = (x + 1 >= Lx) ? 0 : x + 1;
        const int wx = (x + 1 >= Lx) ? 1 : 0;
        const int j = site(nx, y);
        if (i != j) {
          nn_pair(i, j);
          add_bond(i, j, peierls(wx, 0, phix, phiy), t, hops);
        }
      }
      if (Ly > 1) {
        const int ny = (y + 1 >= Ly) ? 0 : y + 1;
        const int wy = (y + 1 >= Ly) ? 1 : 0;
        const int j = site(x, ny);
        if (i != j) {
          nn_pair(i, j);
          add_bond(i, j, peierls(0, wy, phix, phiy), t, hops);
        }
      }
      const int dd[4][2] = {{1, 1}, {1, -1}, {-1, 1}, {-1, -1}};
      for (const auto& d : dd) {
        int nx = x + d[0], ny = y + d[1], wx = 0, wy = 0;
        if (nx >= Lx) {
          nx -= Lx;
          wx = 1;
        } else if (nx < 0) {
          nx += Lx;
          wx = -1;
        }
        if (ny >= Ly) {
          ny -= Ly;
          wy = 1;
        } else if (ny < 0) {
          ny += Ly;
          wy = -1;
        }
        const int j = site(nx, ny);
        if (i != j) add_bond(i, j, peierls(wx, wy, phix, phiy), tp, hops);
      }
    }
  }
}

// src/fock_basis.cpp:7-15 — k-subsets of {0..n-1} in lexicographic order of the sorted
// position list (smallest position chosen first).
void combos(int n, int k, int pos, uint64_t cur, std::vector<uint64_t>* out) {
  if (k == 0) {
    out->push_back(cur);
    return;
  }
  for (int i = pos; i <= n - k; ++i) combos(n, k - 1, i + 1, cur | (1ULL << i), out);
}

// src/hubbard_hamiltonian.cpp:24-43 — fermions strictly between JW modes 2*site+spin.
int between(int ma, int mb, uint64_t up, uint64_t dn) {
  if (ma > mb) std::swap(ma, mb);
  int c = 0;
  for (int m = ma + 1; m < mb; ++m) {
    const int s = m / 2;
    c += static_cast<int>(((m % 2 == 0) ? (up >> s) : (dn >> s)) & 1ULL);
  }
  return c;
}

struct Sector {
  int Lx, Ly, n, nu, nd;
  double t, tp, U, V, phix, phiy;
  std::vector<Hop> hops;
  std::vector<Pair> pairs;
  std::vector<uint64_t> ups, dns;  // lex-ordered strings; state index = rank_up*|dns| + rank_dn
  std::vector<int32_t> rank_up, rank_dn;  // mask -> rank (n <= 24), -1 if wrong popcount
  long long dim() const { return static_cast<long long>(ups.size()) * static_cast<long long>(dns.size()); }

  // src/fock_basis.cpp:44-51 (index_of) — here by rank lookup instead of a hash map.
  long long index_of(uint64_t u, uint64_t d) const {
    if (u >= rank_up.size() || d >= rank_dn.size()) return -1;
    const int ru = rank_up[u], rd = rank_dn[d];
    if (ru < 0 || rd < 0) return -1;
    return static_cast<long long>(ru) * static_cast<long long>(dns.size()) + rd;
  }
  uint64_t up_of(long long i) const { return ups[static_cast<size_t>(i / static_cast<long long>(dns.size()))]; }
  uint64_t dn_of(long long i) const { return dns[static_cast<size_t>(i % static_cast<long long>(dns.size()))]; }

  // src/hubbard_hamiltonian.cpp:66-71 — U * #doubly occupied + V * sum_pairs n_i n_j.
  double diag(uint64_t u, uint64_t d) const {
    double v = static_cast<double>(__builtin_popcountll(u & d)) * U;
    for (const auto& pr : pairs) {
      const int oi = static_cast<int>(((u >> pr.i) & 1ULL) + ((d >> pr.i) & 1ULL));
      const int oj = static_cast<int>(((u >> pr.j) & 1ULL) + ((d >> pr.j) & 1ULL));
      v += V * static_cast<double>(oi * oj);
    }
    return v;
  }
};

Sector* make_sector(int Lx, int Ly, double t, double tp, double U, double V, double phix, double phiy, int nu,
                    int nd) {
  const int n = Lx * Ly;
  if (n <= 0 || n > 24 || nu < 0 || nd < 0 || nu > n || nd > n) return nullptr;
  auto* s = new Sector{Lx, Ly, n, nu, nd, t, tp, U, V, phix, phiy, {}, {}, {}, {}, {}, {}};
  geometry(Lx, Ly, t, tp, phix, phiy, &s->hops, &s->pairs);
  combos(n, nu, 0, 0, &s->ups);
  combos(n, nd, 0, 0, &s->dns);
  s->rank_up.assign(size_t(1) << n, -1);
  s->rank_dn.assign(size_t(1) << n, -1);
  for (size_t i = 0; i < s->ups.size(); ++i) s->rank_up[s->ups[i]] = static_cast<int32_t>(i);
  for (size_t i = 0; i < s->dns.size(); ++i) s->rank_dn[s->dns[i]] = static_cast<int32_t>(i);
  return s;
}

// src/hubbard_hamiltonian.cpp:51-108 — column scatter in the reference's order (columns
// ascending, diagonal first, then hops in list order; columns with |x|^2 < 1e-28 skipped).
void apply_scatter(const Sector& s, const cd* x, cd* y) {
  const long long dim = s.dim();
  std::fill(y, y + dim, cd(0.0, 0.0));
  for (long long col = 0; col < dim; ++col) {
    const uint64_t u = s.up_of(col), d = s.dn_of(col);
    const cd vc = x[col];
    if (std::norm(vc) < 1e-28) continue;
    y[col] += cd(s.diag(u, d), 0.0) * vc;
    for (const auto& h : s.hops) {
      uint64_t up2 = u, dn2 = d;
      const uint64_t occ = h.spin == 0 ? u : d;
      if (!((occ >> h.from) & 1ULL) || ((occ >> h.to) & 1ULL)) continue;
      if (h.spin == 0)
        up2 = u ^ (1ULL << h.from) ^ (1ULL << h.to);
      else
        dn2 = d ^ (1ULL << h.from) ^ (1ULL << h.to);
      const double sign = (between(2 * h.from + h.spin, 2 * h.to + h.spin, u, d) & 1) ? -1.0 : 1.0;
      const long long row = s.index_of(up2, dn2);
      if (row < 0) continue;
      y[row] += (sign * h.coeff) * vc;
    }
  }
}

// The same operator in gather form, rows split across threads: y[r] = sum over sources s of
// H[r,s] x[s], with the reference's source-skip rule (|x[s]|^2 < 1e-28 contributes nothing).
void apply_gather_rows(const Sector& s, const cd* x, cd* y, long long r0, long long r1) {
  for (long long r = r0; r < r1; ++r) {
    const uint64_t u2 = s.up_of(r), d2 = s.dn_of(r);
    cd acc(0.0, 0.0);
    if (std::norm(x[r]) >= 1e-28) acc += cd(s.diag(u2, d2), 0.0) * x[r];
    for (const auto& h : s.hops) {
      const uint64_t occ = h.spin == 0 ? u2 : d2;
      if (!((occ >> h.to) & 1ULL) || ((occ >> h.from) & 1ULL)) continue;
      uint64_t u = u2, d = d2;
      if (h.spin == 0)
        u = u2 ^ (1ULL << h.from) ^ (1ULL << h.to);
      else
        d = d2 ^ (1ULL << h.from) ^ (1ULL << h.to);
      const long long col = s.index_of(u, d);
      if (col < 0) continue;
      const cd vc = x[col];
      if (std::norm(vc) < 1e-28) continue;
      const double sign = (between(2 * h.from + h.spin, 2 * h.to + h.spin, u, d) & 1) ? -1.0 : 1.0;
      acc += (sign * h.coeff) * vc;
    }
    y[r] = acc;
  }
}

void apply_gather(const Sector& s, const cd* x, cd* y, int nthreads) {
  const long long dim = s.dim();
  if (nthreads <= 1 || dim < 4096) {
    apply_gather_rows(s, x, y, 0, dim);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t) {
    const long long a = dim * t / nthreads, b = dim * (t + 1) / nthreads;
    th.emplace_back([&, a, b]() { apply_gather_rows(s, x, y, a, b); });
  }
  for (auto& x_ : th) x_.join();
}

void apply_mode(const Sector& s, const cd* x, cd* y, int mode, int nthreads) {
  if (mode == 0)
    apply_scatter(s, x, y);
  else
    apply_gather(s, x, y, nthreads);
}

// src/lanczos.cpp:125-208 — Hermitian Lanczos, three vectors, no reorthogonalisation.
template <class Apply>
int lanczos(long long dim, Apply&& apply_h, int max_steps, unsigned seed, std::vector<double>* alpha,
            std::vector<double>* beta) {
  alpha->clear();
  beta->clear();
  if (dim <= 0 || max_steps <= 0) return 0;
  std::mt19937 rng(seed);
  std::normal_distribution<double> gauss(0.0, 1.0);
  std::vector<cd> q(static_cast<size_t>(dim)), qp(static_cast<size_t>(dim), cd(0.0, 0.0)),
      w(static_cast<size_t>(dim));
  for (long long i = 0; i < dim; ++i) {
    const double re = gauss(rng);
    const double im = gauss(rng);
    q[static_cast<size_t>(i)] = {re, im};
  }
  double n0 = 0.0;
  for (const auto& z : q) n0 += std::norm(z);
  n0 = std::sqrt(n0);
  if (n0 < 1e-18) {
    q[0] = {1.0, 0.0};
  } else {
    const cd sc(1.0 / n0, 0.0);
    for (auto& z : q) z *= sc;
  }
  double beta_prev = 0.0;
  int used = 0;
  for (int k = 0; k < max_steps; ++k) {
    apply_h(q.data(), w.data());
    cd z(0.0, 0.0);
    for (long long i = 0; i < dim; ++i) z += std::conj(q[static_cast<size_t>(i)]) * w[static_cast<size_t>(i)];
    const double a_k = z.real();
    for (long long i = 0; i < dim; ++i) w[static_cast<size_t>(i)] -= z * q[static_cast<size_t>(i)];
    if (k > 0)
      for (long long i = 0; i < dim; ++i) w[static_cast<size_t>(i)] -= beta_prev * qp[static_cast<size_t>(i)];
    double nw2 = 0.0;
    for (const auto& v : w) nw2 += std::norm(v);
    alpha->push_back(a_k);
    if (nw2 < 1e-24) {
      used = k + 1;
      break;
    }
    const double b_k = std::sqrt(nw2);
    beta->push_back(b_k);
    std::swap(q, qp);
    for (long long i = 0; i < dim; ++i) q[static_cast<size_t>(i)] = w[static_cast<size_t>(i)] / b_k;
    beta_prev = b_k;
    used = k + 1;
  }
  return used;
}

// src/ftlm_thermo.cpp:17-80 — classical Jacobi (largest |off-diagonal| pivot each rotation),
// row-major A, V starts at identity.  Returns rotations performed; *offmax the last pivot size.
int jacobi_all(double* A, double* Vm, int n, int max_rot, double tol, double* offmax) {
  std::fill(Vm, Vm + static_cast<size_t>(n) * n, 0.0);
  for (int i = 0; i < n; ++i) Vm[static_cast<size_t>(i) * n + i] = 1.0;
  *offmax = 0.0;
  if (n <= 1) return 0;
  int rot = 0;
  for (int sweep = 0; sweep < max_rot; ++sweep) {
    int p = 0, q = 1;
    double mx = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) {
        const double v = std::abs(A[static_cast<size_t>(i) * n + j]);
        if (v > mx) {
          mx = v;
          p = i;
          q = j;
        }
      }
    *offmax = mx;
    if (mx < tol) break;
    const double app = A[static_cast<size_t>(p) * n + p], aqq = A[static_cast<size_t>(q) * n + q],
                 apq = A[static_cast<size_t>(p) * n + q];
    const double phi = 0.5 * std::atan2(2.0 * apq, aqq - app);
    const double c = std::cos(phi), s = std::sin(phi);
    for (int k = 0; k < n; ++k) {
      if (k == p || k == q) continue;
      const double apk = A[static_cast<size_t>(p) * n + k], aqk = A[static_cast<size_t>(q) * n + k];
      const double rpk = c * apk - s * aqk, rqk = c * aqk + s * apk;
      A[static_cast<size_t>(p) * n + k] = rpk;
      A[static_cast<size_t>(k) * n + p] = rpk;
      A[static_cast<size_t>(q) * n + k] = rqk;
      A[static_cast<size_t>(k) * n + q] = rqk;
    }
    const double npp = c * c * app - 2.0 * s * c * apq + s * s * aqq;
    const double nqq = s * s * app + 2.0 * s * c * apq + c * c * aqq;
    A[static_cast<size_t>(p) * n + q] = 0.0;
    A[static_cast<size_t>(q) * n + p] = 0.0;
    A[static_cast<size_t>(p) * n + p] = npp;
    A[static_cast<size_t>(q) * n + q] = nqq;
    for (int i = 0; i < n; ++i) {
      const double vip = Vm[static_cast<size_t>(i) * n + p], viq = Vm[static_cast<size_t>(i) * n + q];
      Vm[static_cast<size_t>(i) * n + p] = c * vip - s * viq;
      Vm[static_cast<size_t>(i) * n + q] = s * vip + c * viq;
    }
    ++rot;
  }
  return rot;
}

// src/ftlm_thermo.cpp:83-146 (first half) — Ritz values lam_k and weights |V_0k|^2 of the
// tridiagonal (alpha, beta[0..n-2]) with max(3000, 120 n) Jacobi rotations at tol 1e-14.
int tridiag_eig(const double* alpha, int n, const double* beta, int nb, double* lam, double* w0, double* offmax) {
  if (n <= 0) return 0;
  if (n == 1) {
    lam[0] = alpha[0];
    w0[0] = 1.0;
    *offmax = 0.0;
    return 0;
  }
  std::vector<double> T(static_cast<size_t>(n) * n, 0.0), Vm(static_cast<size_t>(n) * n);
  for (int i = 0; i < n; ++i) T[static_cast<size_t>(i) * n + i] = alpha[i];
  for (int i = 0; i < n - 1 && i < nb; ++i) {
    T[static_cast<size_t>(i) * n + i + 1] = beta[i];
    T[static_cast<size_t>(i + 1) * n + i] = beta[i];
  }
  const int rot = jacobi_all(T.data(), Vm.data(), n, std::max(3000, 120 * n), 1e-14, offmax);
  for (int k = 0; k < n; ++k) {
    lam[k] = T[static_cast<size_t>(k) * n + k];
    w0[k] = Vm[static_cast<size_t>(k)] * Vm[static_cast<size_t>(k)];
  }
  return rot;
}

// src/ftlm_thermo.cpp:83-146 (second half) — log sum_k w_k exp(-beta lam_k), skipping w_k <= 0;
// n == 1 gives -beta*alpha_0 (:93-95).
double log_quadrature(const double* lam, const double* w0, int n, double bT) {
  if (n <= 0) return -std::numeric_limits<double>::infinity();
  if (n == 1) return -bT * lam[0];
  double mx = -std::numeric_limits<double>::infinity();
  for (int k = 0; k < n; ++k) {
    if (w0[k] <= 0.0) continue;
    mx = std::max(mx, -bT * lam[k] + std::log(w0[k]));
  }
  if (!std::isfinite(mx)) return -std::numeric_limits<double>::infinity();
  double s = 0.0;
  for (int k = 0; k < n; ++k) {
    if (w0[k] <= 0.0) continue;
    s += std::exp(-bT * lam[k] + std::log(w0[k]) - mx);
  }
  return mx + std::log(s);
}

// Energy companion of log_quadrature (not in the reference): log of sum_k w_k lam_k e^{-b lam_k}
// is not sign-definite, so return the ratio E_r = sum w lam e / sum w e with the same shift.
double quad_energy(const double* lam, const double* w0, int n, double bT) {
  if (n <= 0) return 0.0;
  if (n == 1) return lam[0];
  double mx = -std::numeric_limits<double>::infinity();
  for (int k = 0; k < n; ++k)
    if (w0[k] > 0.0) mx = std::max(mx, -bT * lam[k] + std::log(w0[k]));
  double s = 0.0, se = 0.0;
  for (int k = 0; k < n; ++k) {
    if (w0[k] <= 0.0) continue;
    const double e = std::exp(-bT * lam[k] + std::log(w0[k]) - mx);
    s += e;
    se += lam[k] * e;
  }
  return se / s;
}


// ---- translation-orbit momentum blocks (reference src/orbit_k_block_basis.cpp:70-220) -----------
// Lattice site of (x, y) is y*Lx + x; a translation by (dx, dy) sends it to
// ((y+dy) mod Ly)*Lx + (x+dx) mod Lx (include/ftlm/symmetry/occup_bits_translate.hpp:10-27).
int shifted_site(int site, int Lx, int Ly, int dx, int dy) {
  return ((site / Lx + dy) % Ly) * Lx + (site % Lx + dx) % Lx;
}

uint32_t shift_bits(uint32_t m, int Lx, int Ly, int dx, int dy) {
  uint32_t out = 0;
  for (int site = 0; site < Lx * Ly; ++site)
    if ((m >> site) & 1u) out |= 1u << shifted_site(site, Lx, Ly, dx, dy);
  return out;
}

uint32_t pack(uint32_t u, uint32_t d) { return (u << 16) | d; }

// include/ftlm/symmetry/fermionic_translation.hpp:32-54 — (-1)^(inversions) of the occupied modes
// 2*site+spin listed in site order (up before down), each sent through the translation.
double shift_sign(uint32_t u, uint32_t d, int Lx, int Ly, int dx, int dy) {
  std::vector<int> modes;
  for (int site = 0; site < Lx * Ly; ++site) {
    const int ts = shifted_site(site, Lx, Ly, dx, dy);
    if ((u >> site) & 1u) modes.push_back(2 * ts);
    if ((d >> site) & 1u) modes.push_back(2 * ts + 1);
  }
  int inv = 0;
  for (size_t i = 0; i < modes.size(); ++i)
    for (size_t j = i + 1; j < modes.size(); ++j) inv += modes[i] > modes[j] ? 1 : 0;
  return (inv & 1) ? -1.0 : 1.0;
}

// include/ftlm/symmetry/orbit.hpp:115-119 — smallest packed image over the translation group.
uint32_t orbit_min(uint32_t u, uint32_t d, int Lx, int Ly) {
  uint32_t best = pack(u, d);
  for (int dy = 0; dy < Ly; ++dy)
    for (int dx = 0; dx < Lx; ++dx)
      best = std::min(best, pack(shift_bits(u, Lx, Ly, dx, dy), shift_bits(d, Lx, Ly, dx, dy)));
  return best;
}

// include/ftlm/symmetry/momentum_sector.hpp:57-63 — chi_K^*(R) = exp(-2 pi i (kx dx/Lx + ky dy/Ly)).
cd bloch(int kx, int ky, int Lx, int Ly, int dx, int dy) {
  const double pi = std::acos(-1.0);
  const double th = -2.0 * pi *
                    (static_cast<double>(kx * dx) / static_cast<double>(Lx) +
                     static_cast<double>(ky * dy) / static_cast<double>(Ly));
  return {std::cos(th), std::sin(th)};
}

struct OrbitBlock {
  const Sector* s;
  int kx, ky;
  std::vector<uint32_t> reps;  // surviving representatives, ascending packed
  std::vector<double> absA;
  std::vector<int> size;       // orbit size
  std::unordered_map<uint32_t, int> row;
};

// src/orbit_k_block_basis.cpp:70-117 — distinct canonical representatives of the sector; stabiliser
// sum A = sum_{R in Stab} eta(rep, R) chi_K^*(R) over R in (dy outer, dx inner) order
// (include/ftlm/symmetry/translation_group.hpp:23-29); keep |A| > 1e-12.
OrbitBlock* make_orbit(const Sector* s, int kx, int ky) {
  if (s->n > 16) return nullptr;
  const int Lx = s->Lx, Ly = s->Ly;
  std::vector<uint32_t> all;
  for (long long i = 0; i < s->dim(); ++i)
    all.push_back(orbit_min(static_cast<uint32_t>(s->up_of(i)), static_cast<uint32_t>(s->dn_of(i)), Lx, Ly));
  std::sort(all.begin(), all.end());
  all.erase(std::unique(all.begin(), all.end()), all.end());
  auto* o = new OrbitBlock{s, kx, ky, {}, {}, {}, {}};
  for (uint32_t p : all) {
    const uint32_t u = p >> 16, d = p & 0xFFFFu;
    cd A(0.0, 0.0);
    int stab = 0;
    for (int dy = 0; dy < Ly; ++dy)
      for (int dx = 0; dx < Lx; ++dx) {
        if (shift_bits(u, Lx, Ly, dx, dy) != u || shift_bits(d, Lx, Ly, dx, dy) != d) continue;
        ++stab;
        A += cd(shift_sign(u, d, Lx, Ly, dx, dy), 0.0) * bloch(kx, ky, Lx, Ly, dx, dy);
      }
    const double a = std::abs(A);
    if (a <= 1e-12) continue;
    o->row[p] = static_cast<int>(o->reps.size());
    o->reps.push_back(p);
    o->absA.push_back(a);
    o->size.push_back(Lx * Ly / stab);
  }
  return o;
}

// src/orbit_k_block_basis.cpp:151-220 — scatter over source representatives beta (skipping
// |x_beta|^2 < 1e-28): diagonal, then every hop of rep(beta) in list order to s'; s' = T_R rep(alpha)
// with R the first translation in (dx outer, dy inner) order (:127-149);
// y_alpha += h * (eta * sqrt(|A_alpha|/|A_beta|)) * chi_K^*(R) * x_beta.
void orbit_apply(const OrbitBlock& o, const cd* x, cd* y) {
  const Sector& s = *o.s;
  const int Lx = s.Lx, Ly = s.Ly;
  const size_t dk = o.reps.size();
  std::fill(y, y + dk, cd(0.0, 0.0));
  for (size_t b = 0; b < dk; ++b) {
    const cd xb = x[b];
    if (std::norm(xb) < 1e-28) continue;
    const uint32_t u = o.reps[b] >> 16, d = o.reps[b] & 0xFFFFu;
    y[b] += cd(s.diag(u, d), 0.0) * xb;
    for (const auto& h : s.hops) {
      const uint32_t occ = h.spin == 0 ? u : d;
      if (!((occ >> h.from) & 1u) || ((occ >> h.to) & 1u)) continue;
      const uint32_t flip = (1u << h.from) | (1u << h.to);
      const uint32_t u2 = h.spin == 0 ? u ^ flip : u, d2 = h.spin == 0 ? d : d ^ flip;
      const double jw = (between(2 * h.from + h.spin, 2 * h.to + h.spin, u, d) & 1) ? -1.0 : 1.0;
      const cd hv = jw * h.coeff;
      const auto it = o.row.find(orbit_min(u2, d2, Lx, Ly));
      if (it == o.row.end()) continue;
      const int a = it->second;
      const uint32_t ru = o.reps[static_cast<size_t>(a)] >> 16, rd = o.reps[static_cast<size_t>(a)] & 0xFFFFu;
      for (int dx = 0, done = 0; dx < Lx && !done; ++dx)
        for (int dy = 0; dy < Ly; ++dy) {
          if (shift_bits(ru, Lx, Ly, dx, dy) != u2 || shift_bits(rd, Lx, Ly, dx, dy) != d2) continue;
          const double eta = shift_sign(ru, rd, Lx, Ly, dx, dy);
          const double nrm = std::sqrt(o.absA[static_cast<size_t>(a)] / o.absA[b]);
          y[static_cast<size_t>(a)] += hv * cd(eta * nrm, 0.0) * bloch(o.kx, o.ky, Lx, Ly, dx, dy) * xb;
          done = 1;
          break;
        }
    }
  }
}

}  // namespace

extern "C" {

int or_geometry(int Lx, int Ly, double t, double tp, double phix, double phiy, int max_hops, int* from, int* to,
                int* spin, double* coeff, int max_pairs, int* pi, int* pj, int* n_pairs) {
  std::vector<Hop> hops;
  std::vector<Pair> pairs;
  geometry(Lx, Ly, t, tp, phix, phiy, &hops, &pairs);
  for (size_t i = 0; i < hops.size() && static_cast<int>(i) < max_hops; ++i) {
    from[i] = hops[i].from;
    to[i] = hops[i].to;
    spin[i] = hops[i].spin;
    coeff[2 * i] = hops[i].coeff.real();
    coeff[2 * i + 1] = hops[i].coeff.imag();
  }
  for (size_t i = 0; i < pairs.size() && static_cast<int>(i) < max_pairs; ++i) {
    pi[i] = pairs[i].i;
    pj[i] = pairs[i].j;
  }
  *n_pairs = static_cast<int>(pairs.size());
  return static_cast<int>(hops.size());
}

long long or_enumerate(int n, int k, uint64_t* out) {
  std::vector<uint64_t> v;
  if (n < 0 || k < 0 || k > n || n > 62) return 0;
  combos(n, k, 0, 0, &v);
  if (out) std::memcpy(out, v.data(), v.size() * sizeof(uint64_t));
  return static_cast<long long>(v.size());
}

void* or_sector_create(int Lx, int Ly, double t, double tp, double U, double V, double phix, double phiy, int nu,
                       int nd) {
  return make_sector(Lx, Ly, t, tp, U, V, phix, phiy, nu, nd);
}
void or_sector_destroy(void* h) { delete static_cast<Sector*>(h); }
long long or_sector_dim(void* h) { return static_cast<Sector*>(h)->dim(); }
void or_sector_masks(void* h, uint64_t* up, uint64_t* dn) {
  auto* s = static_cast<Sector*>(h);
  for (long long i = 0; i < s->dim(); ++i) {
    up[i] = s->up_of(i);
    dn[i] = s->dn_of(i);
  }
}
long long or_sector_index_of(void* h, uint64_t up, uint64_t dn) { return static_cast<Sector*>(h)->index_of(up, dn); }
double or_sector_diag(void* h, uint64_t up, uint64_t dn) { return static_cast<Sector*>(h)->diag(up, dn); }

// mode 0: reference scatter order (single thread); mode 1: row gather over `nthreads` threads.
void or_sector_apply(void* h, const double* x, double* y, int mode, int nthreads) {
  apply_mode(*static_cast<Sector*>(h), reinterpret_cast<const cd*>(x), reinterpret_cast<cd*>(y), mode, nthreads);
}

// Rows [r0, r1) of y = H x only (gather form); for bounded CPU timing samples.
void or_sector_apply_rows(void* h, const double* x, double* y, long long r0, long long r1, int nthreads) {
  auto* s = static_cast<Sector*>(h);
  const cd* xc = reinterpret_cast<const cd*>(x);
  cd* yc = reinterpret_cast<cd*>(y);
  if (nthreads <= 1) {
    apply_gather_rows(*s, xc, yc, r0, r1);
    return;
  }
  std::vector<std::thread> th;
  const long long n = r1 - r0;
  for (int t = 0; t < nthreads; ++t) {
    const long long a = r0 + n * t / nthreads, b = r0 + n * (t + 1) / nthreads;
    th.emplace_back([=]() { apply_gather_rows(*s, xc, yc, a, b); });
  }
  for (auto& x_ : th) x_.join();
}

int or_sector_lanczos(void* h, int M, unsigned seed, double* alpha, double* beta, int* n_beta, int mode,
                      int nthreads) {
  auto* s = static_cast<Sector*>(h);
  std::vector<double> a, b;
  const int used = lanczos(s->dim(), [&](const cd* x, cd* y) { apply_mode(*s, x, y, mode, nthreads); }, M, seed, &a, &b);
  std::copy(a.begin(), a.end(), alpha);
  std::copy(b.begin(), b.end(), beta);
  *n_beta = static_cast<int>(b.size());
  return used;
}

// The reference's start vector for `seed` (src/lanczos.cpp:140-175), normalised.
void or_start_vector(long long dim, unsigned seed, double* q) {
  std::mt19937 rng(seed);
  std::normal_distribution<double> gauss(0.0, 1.0);
  double n0 = 0.0;
  for (long long i = 0; i < dim; ++i) {
    q[2 * i] = gauss(rng);
    q[2 * i + 1] = gauss(rng);
    n0 += q[2 * i] * q[2 * i] + q[2 * i + 1] * q[2 * i + 1];
  }
  n0 = std::sqrt(n0);
  if (n0 < 1e-18) {
    std::fill(q, q + 2 * dim, 0.0);
    q[0] = 1.0;
    return;
  }
  const cd sc(1.0 / n0, 0.0);
  for (long long i = 0; i < dim; ++i) {
    const cd z = cd(q[2 * i], q[2 * i + 1]) * sc;
    q[2 * i] = z.real();
    q[2 * i + 1] = z.imag();
  }
}

int or_tridiag_eig(const double* alpha, int n, const double* beta, int nb, double* lam, double* w0, double* offmax) {
  return tridiag_eig(alpha, n, beta, nb, lam, w0, offmax);
}

double or_log_quadrature(const double* lam, const double* w0, int n, double bT) {
  return log_quadrature(lam, w0, n, bT);
}

double or_quad_energy(const double* lam, const double* w0, int n, double bT) { return quad_energy(lam, w0, n, bT); }

// src/lanczos.cpp:106-123 + 211-231 — lanczos_extrema: min/max Ritz value with the
// 120-rotation / 1e-15 Jacobi of tridiagonal_extrema.
int or_sector_lanczos_extrema(void* h, int M, unsigned seed, double* mn, double* mx, int mode, int nthreads) {
  auto* s = static_cast<Sector*>(h);
  std::vector<double> a, b;
  const int used = lanczos(s->dim(), [&](const cd* x, cd* y) { apply_mode(*s, x, y, mode, nthreads); }, M, seed, &a, &b);
  *mn = 0.0;
  *mx = 0.0;
  if (used == 0) return 0;
  const int n = used;
  std::vector<double> T(static_cast<size_t>(n) * n, 0.0), Vm(static_cast<size_t>(n) * n);
  for (int i = 0; i < n; ++i) T[static_cast<size_t>(i) * n + i] = a[static_cast<size_t>(i)];
  for (int i = 0; i < n - 1 && i < static_cast<int>(b.size()); ++i) {
    T[static_cast<size_t>(i) * n + i + 1] = b[static_cast<size_t>(i)];
    T[static_cast<size_t>(i + 1) * n + i] = b[static_cast<size_t>(i)];
  }
  double off = 0.0;
  if (n > 1) jacobi_all(T.data(), Vm.data(), n, 120, 1e-15, &off);
  double lo = std::numeric_limits<double>::infinity(), hi = -lo;
  for (int i = 0; i < n; ++i) {
    lo = std::min(lo, T[static_cast<size_t>(i) * n + i]);
    hi = std::max(hi, T[static_cast<size_t>(i) * n + i]);
  }
  *mn = lo;
  *mx = hi;
  return used;
}

}  // extern "C"

namespace {

// src/ftlm_thermo.cpp:213-256 — ln Tr e^{-bT H} for one sector, evaluated at n_bt temperatures
// from the same R chains (the reference re-runs the chains per temperature; the chains do not
// depend on the temperature, so the values are identical).  seed_r = seed + r*100003.
// Outputs: lnz[n_bt], energy[n_bt] (FTLM estimate of <H>_sector), lam/w0 per chain if non-null
// (R*M each, padded with w=0).
template <class Apply>
void ftlm_core(long long dim, Apply&& apply_h, double h00, const double* bts, int n_bt, int R, int M, unsigned seed,
               double* lnz, double* energy, double* lam_out, double* w_out, int* used_out) {
  R = std::max(1, R);
  M = std::max(1, M);
  if (dim <= 0) {
    for (int b = 0; b < n_bt; ++b) {
      lnz[b] = -std::numeric_limits<double>::infinity();
      energy[b] = 0.0;
    }
    return;
  }
  if (dim == 1) {  // src/ftlm_thermo.cpp:219-223
    for (int b = 0; b < n_bt; ++b) {
      lnz[b] = -bts[b] * h00;
      energy[b] = h00;
    }
    if (used_out) used_out[0] = 1;
    if (lam_out) {
      std::fill(lam_out, lam_out + static_cast<size_t>(R) * M, 0.0);
      std::fill(w_out, w_out + static_cast<size_t>(R) * M, 0.0);
      lam_out[0] = h00;
      w_out[0] = 1.0;
    }
    return;
  }
  std::vector<std::vector<double>> lams(static_cast<size_t>(R)), ws(static_cast<size_t>(R));
  std::vector<int> used(static_cast<size_t>(R), 0);
  for (int r = 0; r < R; ++r) {
    std::vector<double> a, b;
    const unsigned seed_r = seed + static_cast<unsigned>(r) * 100003u;
    used[r] = lanczos(dim, apply_h, M, seed_r, &a, &b);
    if (used[r] <= 0) continue;
    const int n = static_cast<int>(a.size());
    lams[r].resize(static_cast<size_t>(n));
    ws[r].resize(static_cast<size_t>(n));
    double off = 0.0;
    tridiag_eig(a.data(), n, b.data(), static_cast<int>(b.size()), lams[r].data(), ws[r].data(), &off);
    if (used_out) used_out[r] = used[r];
    if (lam_out) {
      for (int k = 0; k < M; ++k) {
        lam_out[static_cast<size_t>(r) * M + k] = k < n ? lams[r][static_cast<size_t>(k)] : 0.0;
        w_out[static_cast<size_t>(r) * M + k] = k < n ? ws[r][static_cast<size_t>(k)] : 0.0;
      }
    }
  }
  for (int bi = 0; bi < n_bt; ++bi) {
    const double bT = bts[bi];
    std::vector<double> lb, eb;
    for (int r = 0; r < R; ++r) {
      if (used[r] <= 0) continue;
      const int n = static_cast<int>(lams[r].size());
      lb.push_back(log_quadrature(lams[r].data(), ws[r].data(), n, bT));
      eb.push_back(quad_energy(lams[r].data(), ws[r].data(), n, bT));
    }
    if (lb.empty()) {
      lnz[bi] = -std::numeric_limits<double>::infinity();
      energy[bi] = 0.0;
      continue;
    }
    double mx = lb[0];
    for (double x : lb) mx = std::max(mx, x);
    double sm = 0.0, se = 0.0;
    for (size_t i = 0; i < lb.size(); ++i) {
      const double e = std::exp(lb[i] - mx);
      sm += e;
      se += e * eb[i];
    }
    lnz[bi] = std::log(static_cast<double>(dim)) + (mx + std::log(sm / static_cast<double>(lb.size())));
    energy[bi] = se / sm;
  }
}

}  // namespace

extern "C" {

void or_sector_ftlm(void* h, const double* bts, int n_bt, int R, int M, unsigned seed, int mode, int nthreads,
                    double* lnz, double* energy, double* lam_out, double* w_out, int* used_out) {
  auto* s = static_cast<Sector*>(h);
  const double h00 = s->dim() == 1 ? s->diag(s->up_of(0), s->dn_of(0)) : 0.0;
  ftlm_core(
      s->dim(), [&](const cd* x, cd* y) { apply_mode(*s, x, y, mode, nthreads); }, h00, bts, n_bt, R, M, seed, lnz,
      energy, lam_out, w_out, used_out);
}

// benchmarks/bench_ftlm_nmu_rect.cpp:186-219 — grand-canonical combination of sector ln Z_s
// over a (beta, mu) grid: ln Z_GC = LSE_s(ln Z_s + beta mu N_s); <n> = <N>/n_sites;
// <E> = sum_s w_s E_s / sum_s w_s.  lnz_s/e_s are [n_sec][n_bt]; outputs [n_bt][n_mu].
void or_gc_reduce(const double* lnz_s, const double* e_s, const int* N_s, int n_sec, const double* bts, int n_bt,
                  const double* mus, int n_mu, int n_sites, double* lnz_gc, double* n_avg, double* e_avg) {
  for (int b = 0; b < n_bt; ++b) {
    const double bT = bts[b];
    for (int m = 0; m < n_mu; ++m) {
      const double mu = mus[m];
      double mx = -std::numeric_limits<double>::infinity();
      for (int i = 0; i < n_sec; ++i) {
        const double lz = lnz_s[static_cast<size_t>(i) * n_bt + b];
        if (!std::isfinite(lz)) continue;
        mx = std::max(mx, lz + bT * mu * static_cast<double>(N_s[i]));
      }
      const size_t o = static_cast<size_t>(b) * n_mu + m;
      if (!std::isfinite(mx)) {
        lnz_gc[o] = -std::numeric_limits<double>::infinity();
        n_avg[o] = 0.0;
        e_avg[o] = 0.0;
        continue;
      }
      double sw = 0.0, snw = 0.0, sew = 0.0;
      for (int i = 0; i < n_sec; ++i) {
        const double lz = lnz_s[static_cast<size_t>(i) * n_bt + b];
        if (!std::isfinite(lz)) continue;
        const double w = std::exp(lz + bT * mu * static_cast<double>(N_s[i]) - mx);
        sw += w;
        snw += static_cast<double>(N_s[i]) * w;
        sew += e_s[static_cast<size_t>(i) * n_bt + b] * w;
      }
      lnz_gc[o] = mx + std::log(sw);
      n_avg[o] = (sw > 0.0) ? (snw / sw) / static_cast<double>(n_sites) : 0.0;
      e_avg[o] = (sw > 0.0) ? sew / sw : 0.0;
    }
  }
}

// Orbit momentum block of a sector (n_sites <= 16); NULL when unsupported.
void* or_orbit_create(void* sector, int kx, int ky) { return make_orbit(static_cast<Sector*>(sector), kx, ky); }
void or_orbit_destroy(void* h) { delete static_cast<OrbitBlock*>(h); }
long long or_orbit_dim(void* h) { return static_cast<long long>(static_cast<OrbitBlock*>(h)->reps.size()); }
void or_orbit_entries(void* h, uint32_t* rep, double* absA, int* orbit_size) {
  const auto* o = static_cast<OrbitBlock*>(h);
  for (size_t i = 0; i < o->reps.size(); ++i) {
    if (rep) rep[i] = o->reps[i];
    if (absA) absA[i] = o->absA[i];
    if (orbit_size) orbit_size[i] = o->size[i];
  }
}
void or_orbit_apply(void* h, const double* x, double* y) {
  orbit_apply(*static_cast<OrbitBlock*>(h), reinterpret_cast<const cd*>(x), reinterpret_cast<cd*>(y));
}
// ftlm_log_partition_complex on the block (seed_r = seed + r*100003), at n_bt temperatures.
void or_orbit_ftlm(void* h, const double* bts, int n_bt, int R, int M, unsigned seed, double* lnz, double* energy) {
  auto* o = static_cast<OrbitBlock*>(h);
  const long long dk = static_cast<long long>(o->reps.size());
  double h00 = 0.0;
  if (dk == 1) {
    cd one(1.0, 0.0), y0;
    orbit_apply(*o, &one, &y0);
    h00 = y0.real();
  }
  ftlm_core(
      dk, [&](const cd* x, cd* y) { orbit_apply(*o, x, y); }, h00, bts, n_bt, R, M, seed, lnz, energy, nullptr,
      nullptr, nullptr);
}

}  // extern "C"
