// Test infrastructure only: a C ABI over the UNMODIFIED reference C++ library
// (PeizhiMai/FTLM_extended_Hubbard), compiled together with the reference's own
// hot-path sources by oracle/Makefile into oracle/_ref/libftlm_ref.so.
//
// Nothing in the product links this file.  Tests and the CPU-baseline leg of the
// benchmark load it through ctypes to (1) pin the in-repo oracle restatement and
// (2) time the reference's own CPU implementation of the hot path.
//
// Reference entry points wrapped here (paths inside the reference project):
//   FockBasis                    include/ftlm/fock_basis.hpp:11-35, src/fock_basis.cpp:7-51
//   build_hubbard_geometry       include/ftlm/lattice.hpp:38-40, src/lattice.cpp:38-110
//   apply_extended_hubbard       include/ftlm/hubbard_hamiltonian.hpp:13-16, src/hubbard_hamiltonian.cpp:51-108
//   lanczos_tridiagonal          include/ftlm/lanczos.hpp:55-59, src/lanczos.cpp:125-208
//   lanczos_extrema              include/ftlm/lanczos.hpp:45-48, src/lanczos.cpp:211-231
//   ftlm_log_partition_real      include/ftlm/ftlm_thermo.hpp:41-43, src/ftlm_thermo.cpp:150-211
//   ftlm_log_partition_complex   include/ftlm/ftlm_thermo.hpp:47-50, src/ftlm_thermo.cpp:213-256
//   OrbitKBlockBasis/apply_orbit_k_block  include/ftlm/symmetry/orbit_k_block_basis.hpp:45-85
#include <chrono>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <thread>
#include <vector>

#include "ftlm/fock_basis.hpp"
#include "ftlm/ftlm_thermo.hpp"
#include "ftlm/hubbard_hamiltonian.hpp"
#include "ftlm/hubbard_params.hpp"
#include "ftlm/lanczos.hpp"
#include "ftlm/lattice.hpp"
#include "ftlm/symmetry/orbit_k_block_basis.hpp"

namespace {

using cd = std::complex<double>;

struct RefSector {
  ftlm::HubbardParams p;
  ftlm::FockBasis basis;
  std::vector<ftlm::SpinfulHopping> hops;
  std::vector<ftlm::NearestPair> pairs;
  RefSector(const ftlm::HubbardParams& pp, int nu, int nd) : p(pp), basis(pp.Lx * pp.Ly, nu, nd) {
    ftlm::RectLattice lat{p.Lx, p.Ly};
    ftlm::build_hubbard_geometry(p, lat, &hops, &pairs);
  }
};

ftlm::HubbardParams make_params(int Lx, int Ly, double t, double tp, double U, double V, double phix,
                                double phiy) {
  ftlm::HubbardParams p;
  p.Lx = Lx;
  p.Ly = Ly;
  p.t = t;
  p.tp = tp;
  p.U = U;
  p.V = V;
  p.phi_x = phix;
  p.phi_y = phiy;
  return p;
}

struct RefOrbit {
  const RefSector* sec;
  ftlm::symmetry::OrbitKBlockBasis ob;
};

}  // namespace

extern "C" {

// ---- geometry -------------------------------------------------------------------------------
int ref_geometry(int Lx, int Ly, double t, double tp, double U, double V, double phix, double phiy,
                 int max_hops, int* from, int* to, int* spin, double* coeff /*2*max_hops*/, int max_pairs,
                 int* pi, int* pj, int* n_pairs) {
  ftlm::HubbardParams p = make_params(Lx, Ly, t, tp, U, V, phix, phiy);
  ftlm::RectLattice lat{Lx, Ly};
  std::vector<ftlm::SpinfulHopping> hops;
  std::vector<ftlm::NearestPair> pairs;
  ftlm::build_hubbard_geometry(p, lat, &hops, &pairs);
  const int nh = static_cast<int>(hops.size());
  for (int i = 0; i < nh && i < max_hops; ++i) {
    from[i] = hops[i].from;
    to[i] = hops[i].to;
    spin[i] = hops[i].spin;
    coeff[2 * i] = hops[i].coeff.real();
    coeff[2 * i + 1] = hops[i].coeff.imag();
  }
  const int np = static_cast<int>(pairs.size());
  for (int i = 0; i < np && i < max_pairs; ++i) {
    pi[i] = pairs[i].i;
    pj[i] = pairs[i].j;
  }
  *n_pairs = np;
  return nh;
}

// ---- sector handle --------------------------------------------------------------------------
void* ref_sector_create(int Lx, int Ly, double t, double tp, double U, double V, double phix, double phiy,
                        int nu, int nd) {
  try {
    return new RefSector(make_params(Lx, Ly, t, tp, U, V, phix, phiy), nu, nd);
  } catch (...) {
    return nullptr;
  }
}

void ref_sector_destroy(void* h) { delete static_cast<RefSector*>(h); }

long long ref_sector_dim(void* h) { return static_cast<RefSector*>(h)->basis.dim(); }

void ref_sector_masks(void* h, uint64_t* up, uint64_t* dn) {
  auto* s = static_cast<RefSector*>(h);
  const int d = s->basis.dim();
  for (int i = 0; i < d; ++i) {
    up[i] = s->basis.up_mask(i);
    dn[i] = s->basis.down_mask(i);
  }
}

int ref_sector_index_of(void* h, uint64_t up, uint64_t dn) {
  return static_cast<RefSector*>(h)->basis.index_of(up, dn);
}

// y = H x, complex interleaved (re, im) doubles of length 2*dim.
void ref_sector_apply(void* h, const double* x, double* y) {
  auto* s = static_cast<RefSector*>(h);
  ftlm::apply_extended_hubbard(s->p, s->basis, s->hops, s->pairs, reinterpret_cast<const cd*>(x),
                               reinterpret_cast<cd*>(y));
}

// Timed CPU samples of the reference apply for a sector too large to apply in full on the CPU:
// `nthreads` threads each own an x/y pair (allocated once) and call apply_extended_hubbard on an
// x that is non-zero on `ncols` consecutive columns only.  The reference skips columns with
// |x|^2 < 1e-28, so one call processes exactly `ncols` columns plus its fixed O(dim) fill of y
// and scan of x.  ref_sample_run returns the wall seconds of the parallel region and the number
// of processed columns.
struct RefSample {
  RefSector* s;
  int nthreads;
  std::vector<std::vector<cd>> xs, ys;
  std::vector<long long> c0;
  long long ncols_prev = 0;
};

void* ref_sample_create(void* h, int nthreads) {
  auto* s = static_cast<RefSector*>(h);
  if (nthreads < 1) nthreads = 1;
  try {
    auto* c = new RefSample{s, nthreads, {}, {}, {}, 0};
    const size_t dim = static_cast<size_t>(s->basis.dim());
    c->xs.resize(static_cast<size_t>(nthreads));
    c->ys.resize(static_cast<size_t>(nthreads));
    c->c0.assign(static_cast<size_t>(nthreads), 0);
    for (int t = 0; t < nthreads; ++t) {
      c->xs[t].assign(dim, cd(0.0, 0.0));
      c->ys[t].assign(dim, cd(0.0, 0.0));
    }
    return c;
  } catch (...) {
    return nullptr;
  }
}

void ref_sample_destroy(void* c) { delete static_cast<RefSample*>(c); }

double ref_sample_run(void* ctx, long long col0, long long ncols, long long* cols_done) {
  auto* c = static_cast<RefSample*>(ctx);
  const long long dim = c->s->basis.dim();
  for (int t = 0; t < c->nthreads; ++t) {
    for (long long k = 0; k < c->ncols_prev; ++k) c->xs[t][static_cast<size_t>((c->c0[t] + k) % dim)] = cd(0.0, 0.0);
    c->c0[t] = (col0 + static_cast<long long>(t) * ncols) % dim;
    for (long long k = 0; k < ncols; ++k) c->xs[t][static_cast<size_t>((c->c0[t] + k) % dim)] = cd(0.5, -0.25);
  }
  c->ncols_prev = ncols;
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> th;
  for (int t = 0; t < c->nthreads; ++t) {
    th.emplace_back([c, t]() {
      ftlm::apply_extended_hubbard(c->s->p, c->s->basis, c->s->hops, c->s->pairs, c->xs[t].data(), c->ys[t].data());
    });
  }
  for (auto& x : th) x.join();
  *cols_done = static_cast<long long>(c->nthreads) * ncols;
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// lanczos_tridiagonal on this sector with the full complex apply.  alpha has room for M,
// beta for M.  Returns steps used; *n_beta receives beta.size().
int ref_sector_lanczos(void* h, int M, unsigned seed, double* alpha, double* beta, int* n_beta) {
  auto* s = static_cast<RefSector*>(h);
  std::function<void(const cd*, cd*)> ap = [s](const cd* x, cd* y) {
    ftlm::apply_extended_hubbard(s->p, s->basis, s->hops, s->pairs, x, y);
  };
  std::vector<double> a, b;
  const int used = ftlm::lanczos_tridiagonal(s->basis.dim(), ap, M, seed, &a, &b);
  for (size_t i = 0; i < a.size(); ++i) alpha[i] = a[i];
  for (size_t i = 0; i < b.size(); ++i) beta[i] = b[i];
  *n_beta = static_cast<int>(b.size());
  return used;
}

int ref_sector_lanczos_extrema(void* h, int M, unsigned seed, double* mn, double* mx) {
  auto* s = static_cast<RefSector*>(h);
  std::function<void(const cd*, cd*)> ap = [s](const cd* x, cd* y) {
    ftlm::apply_extended_hubbard(s->p, s->basis, s->hops, s->pairs, x, y);
  };
  const ftlm::LanczosExtrema e = ftlm::lanczos_extrema(s->basis.dim(), ap, M, seed);
  *mn = e.min_eval;
  *mx = e.max_eval;
  return e.steps_used;
}

double ref_sector_ftlm_complex(void* h, double beta, int R, int M, unsigned seed) {
  auto* s = static_cast<RefSector*>(h);
  std::function<void(const cd*, cd*)> ap = [s](const cd* x, cd* y) {
    ftlm::apply_extended_hubbard(s->p, s->basis, s->hops, s->pairs, x, y);
  };
  ftlm::FtlmParams par;
  par.n_random = R;
  par.lanczos_steps = M;
  par.seed = seed;
  return ftlm::ftlm_log_partition_complex(s->basis.dim(), ap, beta, par);
}

// Same real-apply wrapping as benchmarks/bench_ftlm_nmu_rect.cpp:151-162.
double ref_sector_ftlm_real(void* h, double beta, int R, int M, unsigned seed) {
  auto* s = static_cast<RefSector*>(h);
  const int dim = s->basis.dim();
  std::vector<cd> xc(static_cast<size_t>(dim)), yc(static_cast<size_t>(dim));
  auto apply_real = [&](const double* x, double* y) {
    for (int i = 0; i < dim; ++i) xc[static_cast<size_t>(i)] = {x[i], 0.0};
    ftlm::apply_extended_hubbard(s->p, s->basis, s->hops, s->pairs, xc.data(), yc.data());
    for (int i = 0; i < dim; ++i) y[i] = yc[static_cast<size_t>(i)].real();
  };
  ftlm::FtlmParams par;
  par.n_random = R;
  par.lanczos_steps = M;
  par.seed = seed;
  return ftlm::ftlm_log_partition_real(dim, apply_real, beta, par);
}

// tests/test_ftlm_thermo.cpp: diag(2,3) through ftlm_log_partition_real.
double ref_ftlm_diag_real(const double* diag, int dim, double beta, int R, int M, unsigned seed) {
  std::vector<double> d(diag, diag + dim);
  auto ap = [&](const double* x, double* y) {
    for (int i = 0; i < dim; ++i) y[i] = d[static_cast<size_t>(i)] * x[i];
  };
  ftlm::FtlmParams par;
  par.n_random = R;
  par.lanczos_steps = M;
  par.seed = seed;
  return ftlm::ftlm_log_partition_real(dim, ap, beta, par);
}

// Lanczos on an arbitrary dense Hermitian matrix (column-major complex), for quadrature pins.
int ref_dense_lanczos(const double* Hcm, int dim, int M, unsigned seed, double* alpha, double* beta, int* n_beta) {
  std::vector<cd> H(reinterpret_cast<const cd*>(Hcm), reinterpret_cast<const cd*>(Hcm) + static_cast<size_t>(dim) * dim);
  std::function<void(const cd*, cd*)> ap = [&](const cd* x, cd* y) {
    for (int i = 0; i < dim; ++i) {
      cd s(0.0, 0.0);
      for (int j = 0; j < dim; ++j) s += H[static_cast<size_t>(j) * dim + i] * x[j];
      y[i] = s;
    }
  };
  std::vector<double> a, b;
  const int used = ftlm::lanczos_tridiagonal(dim, ap, M, seed, &a, &b);
  for (size_t i = 0; i < a.size(); ++i) alpha[i] = a[i];
  for (size_t i = 0; i < b.size(); ++i) beta[i] = b[i];
  *n_beta = static_cast<int>(b.size());
  return used;
}

// ---- orbit k-block (config with translation symmetry) --------------------------------------
void* ref_orbit_create(void* sector, int kx, int ky) {
  auto* s = static_cast<RefSector*>(sector);
  try {
    auto* o = new RefOrbit{s, {}};
    ftlm::symmetry::MomentumSector K{};
    K.kx = kx;
    K.ky = ky;
    K.lx = s->p.Lx;
    K.ly = s->p.Ly;
    o->ob.build(s->basis, K);
    return o;
  } catch (...) {
    return nullptr;
  }
}

void ref_orbit_destroy(void* h) { delete static_cast<RefOrbit*>(h); }

int ref_orbit_dim(void* h) { return static_cast<RefOrbit*>(h)->ob.dim(); }

// Per reduced row: packed rep (up<<16|dn), |A|, orbit size.
void ref_orbit_entries(void* h, uint32_t* rep, double* absA, int* orbit_size) {
  auto* o = static_cast<RefOrbit*>(h);
  const auto& e = o->ob.entries();
  for (size_t i = 0; i < e.size(); ++i) {
    rep[i] = (static_cast<uint32_t>(e[i].rep.up) << 16) | e[i].rep.dn;
    absA[i] = e[i].abs_A;
    orbit_size[i] = e[i].orbit_size;
  }
}

void ref_orbit_apply(void* h, const double* x, double* y) {
  auto* o = static_cast<RefOrbit*>(h);
  ftlm::symmetry::apply_orbit_k_block(o->sec->p, o->sec->basis, o->ob, o->sec->hops, o->sec->pairs,
                                      reinterpret_cast<const cd*>(x), reinterpret_cast<cd*>(y));
}

double ref_orbit_ftlm_complex(void* h, double beta, int R, int M, unsigned seed) {
  auto* o = static_cast<RefOrbit*>(h);
  std::function<void(const cd*, cd*)> ap = [o](const cd* x, cd* y) {
    ftlm::symmetry::apply_orbit_k_block(o->sec->p, o->sec->basis, o->ob, o->sec->hops, o->sec->pairs, x, y);
  };
  ftlm::FtlmParams par;
  par.n_random = R;
  par.lanczos_steps = M;
  par.seed = seed;
  return ftlm::ftlm_log_partition_complex(o->ob.dim(), ap, beta, par);
}

}  // extern "C"
