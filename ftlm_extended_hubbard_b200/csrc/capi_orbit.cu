#include "capi_internal.hpp"

using namespace ftlm_b200;
using namespace ftlm_b200::capi;

// ---------------------------------------------------------------------------------------------
// Translation-orbit k-blocks (orbit.cu).  Reference: OrbitKBlockBasis::build and
// apply_orbit_k_block (src/orbit_k_block_basis.cpp:70-220), k-bench block loop
// (benchmarks/bench_ftlm_nmu_4x4_k.cpp:801-1081).
struct OrbitSectorData {
  int G = 0;
  DevBuf tlut, tsite, rorder, rank_u, rank_d, rep_full, reta;
  DevBuf uh_from, uh_to, uh_c, uh_own, uh_oth, dh_from, dh_to, dh_c, dh_own, dh_oth;
  int n_uh = 0, n_dh = 0;
  int64_t nreps = 0;                  // number of orbit representatives of the sector
  DevBuf reps_dev;                    // [nreps] representatives, ascending packed (up<<16 | dn)
  DevBuf reps_full_dev;               // [nreps] their full-space indices (int64)
  OrbitDev dev{};
};

struct ftlm_orbit {
  ftlm_sector* sector = nullptr;
  std::shared_ptr<OrbitSectorData> data;
  int kx = 0, ky = 0;
  int64_t dk = 0;
  std::vector<uint32_t> reps;  // surviving representatives (ascending packed)
  std::vector<double> absA;
  std::vector<double> Ak;         // A(K), 2 per representative
  std::vector<int> stab;          // stabiliser size
  std::vector<int64_t> orbit_idx; // index among all representatives of the sector (ascending packed)
  DevBuf reps_dev, sqrtA, table, chi, xs;
  OrbitApplyDev app{};
  LanczosWs ws;
  DevBuf hx, hy;
};

namespace {

template <class T>
cudaError_t upload_to(DevBuf& b, const std::vector<T>& v) {
  cudaError_t e = b.alloc(std::max<size_t>(v.size(), 1) * sizeof(T));
  if (e != cudaSuccess || v.empty()) return e;
  return cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

int build_orbit_sector(ftlm_sector* s) {
  if (s->orbit_data) return FTLM_OK;
  const SectorPlan& P = s->plan;
  if (s->Lx <= 0 || s->Ly <= 0) return fail(FTLM_ERR_UNSUPPORTED, "orbit k-blocks need a sector built from lattice parameters");
  if (P.n > 16) return fail(FTLM_ERR_INVALID, "OrbitKBlockBasis::build: n_sites must be <= 16 (RawState bit width)");
  auto D = std::make_shared<OrbitSectorData>();
  const int Lx = s->Lx, Ly = s->Ly, n = P.n, G = Lx * Ly;
  D->G = G;
  std::vector<uint16_t> tl(static_cast<size_t>(G) * 512, 0);
  std::vector<uint8_t> ts(static_cast<size_t>(G) * 16, 0), ro;
  for (int dy = 0; dy < Ly; ++dy)
    for (int dx = 0; dx < Lx; ++dx) {
      const int R = dy * Lx + dx;
      for (int site = 0; site < n; ++site) {
        const int x = site % Lx, y = site / Lx;
        ts[static_cast<size_t>(R) * 16 + site] = static_cast<uint8_t>(((y + dy) % Ly) * Lx + (x + dx) % Lx);
      }
      for (int half = 0; half < 2; ++half)
        for (int m = 0; m < 256; ++m) {
          uint16_t out = 0;
          for (int b = 0; b < 8; ++b) {
            const int site = half * 8 + b;
            if (site < n && ((m >> b) & 1)) out |= static_cast<uint16_t>(1u << ts[static_cast<size_t>(R) * 16 + site]);
          }
          tl[static_cast<size_t>(R) * 512 + half * 256 + m] = out;
        }
    }
  for (int dx = 0; dx < Lx; ++dx)
    for (int dy = 0; dy < Ly; ++dy) ro.push_back(static_cast<uint8_t>(dy * Lx + dx));  // reference search order
  std::vector<int32_t> rku(65536, -1), rkd(65536, -1);
  for (int64_t i = 0; i < P.up.D; ++i) rku[P.up.masks[static_cast<size_t>(i)]] = static_cast<int32_t>(i);
  for (int64_t i = 0; i < P.dn.D; ++i) rkd[P.dn.masks[static_cast<size_t>(i)]] = static_cast<int32_t>(i);
  CU_TRY(upload_to(D->tlut, tl));
  CU_TRY(upload_to(D->tsite, ts));
  CU_TRY(upload_to(D->rorder, ro));
  CU_TRY(upload_to(D->rank_u, rku));
  CU_TRY(upload_to(D->rank_d, rkd));
  OrbitDev& O = D->dev;
  O.n = n;
  O.Lx = Lx;
  O.Ly = Ly;
  O.G = G;
  O.Du = P.up.D;
  O.Dd = P.dn.D;
  O.dim = P.dim;
  O.umask = s->dev.umask;
  O.dmask = s->dev.dmask;
  O.rank_u = D->rank_u.as<int32_t>();
  O.rank_d = D->rank_d.as<int32_t>();
  O.tlut = D->tlut.as<uint16_t>();
  O.tsite = D->tsite.as<uint8_t>();
  O.rorder = D->rorder.as<uint8_t>();
  CU_TRY(D->rep_full.alloc(static_cast<size_t>(P.dim) * sizeof(int32_t)));
  CU_TRY(D->reta.alloc(static_cast<size_t>(P.dim)));
  CU_TRY(orbit_canon(O, D->rep_full.as<int32_t>(), D->reta.as<uint8_t>(), s->stream));
  {
    // Representatives in ascending packed order, compacted on the device: position p of that order is
    // (p / Dd)-th up string by mask value, (p % Dd)-th down string by mask value.
    std::vector<int32_t> inv_u(static_cast<size_t>(P.up.D)), inv_d(static_cast<size_t>(P.dn.D));
    for (size_t i = 0; i < inv_u.size(); ++i) inv_u[i] = static_cast<int32_t>(i);
    for (size_t i = 0; i < inv_d.size(); ++i) inv_d[i] = static_cast<int32_t>(i);
    std::sort(inv_u.begin(), inv_u.end(),
              [&P](int32_t a, int32_t b) { return P.up.masks[static_cast<size_t>(a)] < P.up.masks[static_cast<size_t>(b)]; });
    std::sort(inv_d.begin(), inv_d.end(),
              [&P](int32_t a, int32_t b) { return P.dn.masks[static_cast<size_t>(a)] < P.dn.masks[static_cast<size_t>(b)]; });
    DevBuf iu, id, counts;
    CU_TRY(upload_to(iu, inv_u));
    CU_TRY(upload_to(id, inv_d));
    CU_TRY(counts.alloc(static_cast<size_t>(orbit_compact_counts(P.dim)) * sizeof(int32_t)));
    CU_TRY(orbit_count_reps(O, D->rep_full.as<int32_t>(), iu.as<int32_t>(), id.as<int32_t>(), counts.as<int32_t>(),
                            &D->nreps, s->stream));
    CU_TRY(D->reps_dev.alloc(static_cast<size_t>(std::max<int64_t>(D->nreps, 1)) * sizeof(uint32_t)));
    CU_TRY(D->reps_full_dev.alloc(static_cast<size_t>(std::max<int64_t>(D->nreps, 1)) * sizeof(int64_t)));
    CU_TRY(orbit_write_reps(O, D->rep_full.as<int32_t>(), iu.as<int32_t>(), id.as<int32_t>(), counts.as<int32_t>(),
                            D->reps_dev.as<uint32_t>(), D->reps_full_dev.as<int64_t>(), s->stream));
    CU_TRY(cudaStreamSynchronize(s->stream));
  }
  // merged hops with their JW masks (same convention as the sector plan)
  std::vector<int32_t> f, t;
  std::vector<double2> c;
  std::vector<uint32_t> own, oth;
  for (const auto& h : P.hu) {
    f.push_back(h.from);
    t.push_back(h.to);
    c.push_back(make_double2(h.cre, h.cim));
    own.push_back(h.own_mask);
    oth.push_back(h.other_mask);
  }
  D->n_uh = static_cast<int>(f.size());
  CU_TRY(upload_to(D->uh_from, f));
  CU_TRY(upload_to(D->uh_to, t));
  CU_TRY(upload_to(D->uh_c, c));
  CU_TRY(upload_to(D->uh_own, own));
  CU_TRY(upload_to(D->uh_oth, oth));
  f.clear();
  t.clear();
  c.clear();
  own.clear();
  oth.clear();
  for (const auto& h : P.hd) {
    f.push_back(h.from);
    t.push_back(h.to);
    c.push_back(make_double2(h.cre, h.cim));
    own.push_back(h.own_mask);
    oth.push_back(h.other_mask);
  }
  D->n_dh = static_cast<int>(f.size());
  CU_TRY(upload_to(D->dh_from, f));
  CU_TRY(upload_to(D->dh_to, t));
  CU_TRY(upload_to(D->dh_c, c));
  CU_TRY(upload_to(D->dh_own, own));
  CU_TRY(upload_to(D->dh_oth, oth));
  s->orbit_data = D;
  return FTLM_OK;
}

int orbit_apply_dev(ftlm_orbit* o, const double2* x, double2* y, cudaStream_t st) {
  CU_TRY(orbit_apply(o->app, x, y, st));
  return FTLM_OK;
}

}  // namespace

extern "C" {

int ftlm_gpu_orbit_create(ftlm_sector* s, int kx, int ky, ftlm_orbit** out) {
  return ftlm_gpu_orbit_create_ex(s, kx, ky, 1e-12, out);
}

int ftlm_gpu_sector_set_lattice(ftlm_sector* s, int Lx, int Ly) {
  if (!s || Lx <= 0 || Ly <= 0 || Lx * Ly != s->plan.n)
    return fail(FTLM_ERR_INVALID, "lattice Lx*Ly must equal the sector's number of sites");
  if (s->Lx == Lx && s->Ly == Ly) return FTLM_OK;
  s->Lx = Lx;
  s->Ly = Ly;
  s->orbit_data.reset();
  return FTLM_OK;
}

int ftlm_gpu_orbit_create_ex(ftlm_sector* s, int kx, int ky, double survive_tol, ftlm_orbit** out) {
  int rc = need_device(s);
  if (rc) return rc;
  if (!out) return fail(FTLM_ERR_INVALID, "null output");
  *out = nullptr;
  if (s->Lx > 0 && (kx < 0 || ky < 0 || kx >= s->Lx || ky >= s->Ly)) return fail(FTLM_ERR_INVALID, "momentum out of range");
  rc = build_orbit_sector(s);
  if (rc) return rc;
  auto o = std::make_unique<ftlm_orbit>();
  o->sector = s;
  o->data = s->orbit_data;
  o->kx = kx;
  o->ky = ky;
  const OrbitSectorData& D = *o->data;
  // translation_bloch_phase(K, dx, dy) (include/ftlm/symmetry/momentum_sector.hpp:57-63), R = dy*Lx + dx
  std::vector<double2> chi(static_cast<size_t>(D.G));
  const double pi = std::acos(-1.0);
  for (int dy = 0; dy < s->Ly; ++dy)
    for (int dx = 0; dx < s->Lx; ++dx) {
      const double theta = -2.0 * pi *
                           (static_cast<double>(kx * dx) / static_cast<double>(s->Lx) +
                            static_cast<double>(ky * dy) / static_cast<double>(s->Ly));
      chi[static_cast<size_t>(dy * s->Lx + dx)] = make_double2(std::cos(theta), std::sin(theta));
    }
  CU_TRY(upload_to(o->chi, chi));
  const int64_t nreps = D.nreps;
  DevBuf absA, Adev, sdev, counts;
  CU_TRY(absA.alloc(std::max<int64_t>(nreps, 1) * sizeof(double)));
  CU_TRY(Adev.alloc(std::max<int64_t>(nreps, 1) * sizeof(double2)));
  CU_TRY(sdev.alloc(std::max<int64_t>(nreps, 1) * sizeof(int)));
  CU_TRY(counts.alloc(static_cast<size_t>(orbit_compact_counts(nreps)) * sizeof(int32_t)));
  CU_TRY(orbit_absA(D.dev, D.reps_dev.as<uint32_t>(), nreps, o->chi.as<double2>(), absA.as<double>(),
                    Adev.as<double2>(), sdev.as<int>(), s->stream));
  // survivors |A| > survive_tol (orbit_k_block_basis.hpp:53), compacted in order on the device
  int64_t dk = 0;
  CU_TRY(orbit_count_survivors(absA.as<double>(), nreps, survive_tol, counts.as<int32_t>(), &dk, s->stream));
  if (dk >= (1 << 24)) return fail(FTLM_ERR_UNSUPPORTED, "k-block larger than 2^24 states");
  o->dk = dk;
  const size_t n1 = static_cast<size_t>(std::max<int64_t>(dk, 1));
  DevBuf full_k, absA_k, A_k, stab_k, oidx_k;
  CU_TRY(o->reps_dev.alloc(n1 * sizeof(uint32_t)));
  CU_TRY(o->sqrtA.alloc(n1 * sizeof(double)));
  CU_TRY(full_k.alloc(n1 * sizeof(int64_t)));
  CU_TRY(absA_k.alloc(n1 * sizeof(double)));
  CU_TRY(A_k.alloc(n1 * sizeof(double2)));
  CU_TRY(stab_k.alloc(n1 * sizeof(int)));
  CU_TRY(oidx_k.alloc(n1 * sizeof(int64_t)));
  const OrbitBlockIn bin{D.reps_dev.as<uint32_t>(), D.reps_full_dev.as<int64_t>(), absA.as<double>(), Adev.as<double2>(),
                         sdev.as<int>()};
  const OrbitBlockOut bout{o->reps_dev.as<uint32_t>(), full_k.as<int64_t>(), absA_k.as<double>(), A_k.as<double2>(),
                           stab_k.as<int>(), oidx_k.as<int64_t>(), o->sqrtA.as<double>()};
  CU_TRY(orbit_write_survivors(bin, nreps, survive_tol, counts.as<int32_t>(), bout, s->stream));
  // host copies of the block's entries (ftlm_gpu_orbit_entries / _ex)
  o->reps.resize(static_cast<size_t>(dk));
  o->absA.resize(static_cast<size_t>(dk));
  o->Ak.resize(2 * static_cast<size_t>(dk));
  o->stab.resize(static_cast<size_t>(dk));
  o->orbit_idx.resize(static_cast<size_t>(dk));
  if (dk > 0) {
    CU_TRY(cudaMemcpyAsync(o->reps.data(), o->reps_dev.p, o->reps.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
    CU_TRY(cudaMemcpyAsync(o->absA.data(), absA_k.p, o->absA.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CU_TRY(cudaMemcpyAsync(o->Ak.data(), A_k.p, o->Ak.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CU_TRY(cudaMemcpyAsync(o->stab.data(), stab_k.p, o->stab.size() * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    CU_TRY(cudaMemcpyAsync(o->orbit_idx.data(), oidx_k.p, o->orbit_idx.size() * sizeof(int64_t), cudaMemcpyDeviceToHost,
                           s->stream));
  }
  {
    DevBuf red;
    CU_TRY(red.alloc(static_cast<size_t>(s->plan.dim) * sizeof(int32_t)));
    CU_TRY(cudaMemsetAsync(red.p, 0xFF, static_cast<size_t>(s->plan.dim) * sizeof(int32_t), s->stream));
    CU_TRY(orbit_scatter_index(full_k.as<int64_t>(), o->dk, red.as<int32_t>(), s->stream));
    CU_TRY(o->table.alloc(static_cast<size_t>(s->plan.dim) * sizeof(uint32_t)));
    CU_TRY(orbit_table(D.dev, D.rep_full.as<int32_t>(), D.reta.as<uint8_t>(), red.as<int32_t>(), o->table.as<uint32_t>(),
                       s->stream));
    CU_TRY(cudaStreamSynchronize(s->stream));
  }
  OrbitApplyDev& A = o->app;
  A.O = D.dev;
  A.S = s->dev;
  A.dk = o->dk;
  A.reps = o->reps_dev.as<uint32_t>();
  A.sqrtA = o->sqrtA.as<double>();
  A.table = o->table.as<uint32_t>();
  A.chi_tab = o->chi.as<double2>();
  A.uhop_from = D.uh_from.as<int32_t>();
  A.uhop_to = D.uh_to.as<int32_t>();
  A.uhop_c = D.uh_c.as<double2>();
  A.uhop_own = D.uh_own.as<uint32_t>();
  A.uhop_oth = D.uh_oth.as<uint32_t>();
  A.n_uhops = D.n_uh;
  A.dhop_from = D.dh_from.as<int32_t>();
  A.dhop_to = D.dh_to.as<int32_t>();
  A.dhop_c = D.dh_c.as<double2>();
  A.dhop_own = D.dh_own.as<uint32_t>();
  A.dhop_oth = D.dh_oth.as<uint32_t>();
  A.n_dhops = D.n_dh;
  CU_TRY(o->xs.alloc(static_cast<size_t>(std::max<int64_t>(o->dk, 1)) * sizeof(double2)));
  A.xs = o->xs.as<double2>();
  A.path = 1;
  *out = o.release();
  return FTLM_OK;
}

int ftlm_gpu_orbit_destroy(ftlm_orbit* o) {
  delete o;
  return FTLM_OK;
}

int ftlm_gpu_orbit_set_apply_path(ftlm_orbit* o, int path) {
  if (!o || (path != 0 && path != 1)) return fail(FTLM_ERR_INVALID, "path must be 0 or 1");
  o->app.path = path;
  return FTLM_OK;
}

int ftlm_gpu_orbit_dim(const ftlm_orbit* o, long long* dim) {
  if (!o || !dim) return fail(FTLM_ERR_INVALID, "null argument");
  *dim = o->dk;
  return FTLM_OK;
}

int ftlm_gpu_orbit_entries(const ftlm_orbit* o, uint32_t* rep_packed, double* absA) {
  if (!o) return fail(FTLM_ERR_INVALID, "null orbit");
  if (rep_packed) std::copy(o->reps.begin(), o->reps.end(), rep_packed);
  if (absA) std::copy(o->absA.begin(), o->absA.end(), absA);
  return FTLM_OK;
}

int ftlm_gpu_orbit_entries_ex(const ftlm_orbit* o, uint32_t* rep_packed, double* A, double* absA, int* orbit_size,
                              int* stabilizer_size, long long* orbit_index) {
  if (!o) return fail(FTLM_ERR_INVALID, "null orbit");
  const int G = o->data->G;
  for (size_t i = 0; i < o->reps.size(); ++i) {
    if (rep_packed) rep_packed[i] = o->reps[i];
    if (A) {
      A[2 * i] = o->Ak[2 * i];
      A[2 * i + 1] = o->Ak[2 * i + 1];
    }
    if (absA) absA[i] = o->absA[i];
    if (stabilizer_size) stabilizer_size[i] = o->stab[i];
    if (orbit_size) orbit_size[i] = o->stab[i] > 0 ? G / o->stab[i] : 0;
    if (orbit_index) orbit_index[i] = o->orbit_idx[i];
  }
  return FTLM_OK;
}

int ftlm_gpu_orbit_apply(ftlm_orbit* o, const double* x, double* y, void* stream) {
  if (!o || !x || !y) return fail(FTLM_ERR_INVALID, "null argument");
  if (x == y) return fail(FTLM_ERR_INVALID, "x and y must not alias");
  return orbit_apply_dev(o, reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y),
                         static_cast<cudaStream_t>(stream));
}

int ftlm_gpu_orbit_apply_host(ftlm_orbit* o, const double* x, double* y) {
  if (!o || !x || !y) return fail(FTLM_ERR_INVALID, "null argument");
  const size_t bytes = static_cast<size_t>(std::max<int64_t>(o->dk, 1)) * sizeof(double2);
  if (!o->hx.p) {
    CU_TRY(o->hx.alloc(bytes));
    CU_TRY(o->hy.alloc(bytes));
  }
  cudaStream_t st = o->sector->stream;
  CU_TRY(cudaMemcpyAsync(o->hx.p, x, o->dk * sizeof(double2), cudaMemcpyHostToDevice, st));
  const int rc = orbit_apply_dev(o, o->hx.as<double2>(), o->hy.as<double2>(), st);
  if (rc) return rc;
  CU_TRY(cudaMemcpyAsync(y, o->hy.p, o->dk * sizeof(double2), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  return FTLM_OK;
}

int ftlm_gpu_orbit_ftlm(ftlm_orbit* o, const double* bts, int n_bt, int R, int M, unsigned seed, int start_mode,
                        double* lnz, double* energy) {
  if (!o) return fail(FTLM_ERR_INVALID, "null orbit");
  if (n_bt < 0 || (n_bt > 0 && (!bts || !lnz || !energy))) return fail(FTLM_ERR_INVALID, "bad arguments");
  R = std::max(1, R);
  M = std::max(1, M);
  if (M > 160) return fail(FTLM_ERR_UNSUPPORTED, "more than 160 Lanczos steps for the on-chip Jacobi");
  const int64_t dk = o->dk;
  if (dk <= 0) {
    for (int b = 0; b < n_bt; ++b) {
      lnz[b] = -std::numeric_limits<double>::infinity();
      energy[b] = 0.0;
    }
    return FTLM_OK;
  }
  if (dk == 1) {  // src/ftlm_thermo.cpp:219-223
    const double one[2] = {1.0, 0.0};
    double h00[2] = {0.0, 0.0};
    const int rc = ftlm_gpu_orbit_apply_host(o, one, h00);
    if (rc) return rc;
    for (int b = 0; b < n_bt; ++b) {
      lnz[b] = -bts[b] * h00[0];
      energy[b] = h00[0];
    }
    return FTLM_OK;
  }
  std::vector<double> A(static_cast<size_t>(R) * M, 0.0), B(static_cast<size_t>(R) * M, 0.0);
  std::vector<int> nv(static_cast<size_t>(R), 0);
  for (int r = 0; r < R; ++r) {
    std::vector<double> a, b;
    const int rc = run_lanczos(
        dk, [o](const double2* x, double2* y, cudaStream_t st) { return orbit_apply_dev(o, x, y, st); }, o->ws, M,
        seed + static_cast<unsigned>(r) * 100003u, start_mode, o->sector->stream, &a, &b);
    if (rc) return rc;
    std::copy(a.begin(), a.end(), A.begin() + static_cast<long>(r) * M);
    std::copy(b.begin(), b.end(), B.begin() + static_cast<long>(r) * M);
    nv[static_cast<size_t>(r)] = static_cast<int>(a.size());
  }
  std::vector<double> lq(static_cast<size_t>(R) * n_bt), eq(static_cast<size_t>(R) * n_bt);
  int rc = chain_quadrature(A.data(), B.data(), nv.data(), R, M, bts, n_bt, lq.data(), eq.data(),
                            plain_quadrature_converged());
  if (rc) return rc;
  return ftlm_gpu_ftlm_combine(lq.data(), eq.data(), nv.data(), R, n_bt, std::log(static_cast<double>(dk)), lnz, energy);
}

// Batched complex64 FTLM of one block: 32-chain blocks of bt_orbit_step (Philox starts, as the
// sector path); blocks with dim <= 2M use the complex128 Philox path.
int ftlm_gpu_orbit_batched_ftlm(ftlm_orbit* o, const double* bts, int n_bt, int R, int M, unsigned seed, double* lnz,
                                double* energy) {
  if (!o) return fail(FTLM_ERR_INVALID, "null orbit");
  if (n_bt < 0 || (n_bt > 0 && (!bts || !lnz || !energy))) return fail(FTLM_ERR_INVALID, "bad arguments");
  R = std::max(1, R);
  M = std::max(1, M);
  if (M > 160) return fail(FTLM_ERR_UNSUPPORTED, "more than 160 Lanczos steps for the on-chip Jacobi");
  const int64_t dk = o->dk;
  if (dk <= 2 * static_cast<int64_t>(M)) return ftlm_gpu_orbit_ftlm(o, bts, n_bt, R, M, seed, FTLM_START_PHILOX, lnz, energy);
  const SectorPlan& P = o->sector->plan;
  if (P.max_up_deg > 120 || P.max_up_deg + ((P.max_dn_deg + 7) / 8) * 8 + 8 > 256)
    return fail(FTLM_ERR_UNSUPPORTED, "batched orbit path: more than 256 sources per representative");
  cudaStream_t st = o->sector->stream;
  const OrbitApplyDev& Adev = o->app;
  std::vector<double> A, B;
  std::vector<int> used;
  int rc = bt_run_chains_impl(
      dk, st,
      [&Adev, st](const float2* wk, const float2* wkm1, float2* y, int k, double* sd, double* part, double* al,
                  double* be, int* us, int* fl) { return bt_orbit_step(Adev, wk, wkm1, y, k, sd, part, al, be, us, fl, st); },
      R, M, seed, &A, &B, &used, nullptr);
  if (rc) return rc;
  std::vector<double> lq(static_cast<size_t>(R) * n_bt), eq(static_cast<size_t>(R) * n_bt);
  rc = chain_quadrature(A.data(), B.data(), used.data(), R, M, bts, n_bt, lq.data(), eq.data(), true);
  if (rc) return rc;
  return ftlm_gpu_ftlm_combine(lq.data(), eq.data(), used.data(), R, n_bt, std::log(static_cast<double>(dk)), lnz, energy);
}

// Exact ln Tr e^{-bT H_K} of a small block (the k-bench's exact_log_partition_small_complex,
// benchmarks/bench_ftlm_nmu_4x4_k.cpp:249-333), all on the GPU: H_K built column by column, its
// real 2dk x 2dk embedding [[Re, -Im], [Im, Re]] (each eigenvalue twice) diagonalised by the
// parallel Jacobi of symeig.cu, and ln Z = log sum_i (1/2) e^{-bT lam_i} with the energy ratio by
// the quadrature evaluation kernel (weights 1/2).  2dk <= 160.
static int orbit_block_ed(ftlm_orbit* o, const double* bts, int n_bt, double* lnz, double* energy) {
  const int64_t dk = o->dk;
  const int m = static_cast<int>(2 * dk);
  if (m > kMaxEig) return fail(FTLM_ERR_UNSUPPORTED, "exact small-block path: block dimension > 80");
  const size_t col = static_cast<size_t>(dk) * sizeof(double2);
  DevBuf X, Y, Rm, lam, w, nn, bt, lq, eq, info;
  CU_TRY(X.alloc(col * dk));
  CU_TRY(Y.alloc(col * dk));
  CU_TRY(Rm.alloc(static_cast<size_t>(m) * m * sizeof(double)));
  CU_TRY(lam.alloc(static_cast<size_t>(m) * sizeof(double)));
  CU_TRY(w.alloc(static_cast<size_t>(m) * sizeof(double)));
  CU_TRY(nn.alloc(sizeof(int)));
  CU_TRY(bt.alloc(std::max(1, n_bt) * sizeof(double)));
  CU_TRY(lq.alloc(std::max(1, n_bt) * sizeof(double)));
  CU_TRY(eq.alloc(std::max(1, n_bt) * sizeof(double)));
  CU_TRY(info.alloc(sizeof(int)));
  cudaStream_t st = o->sector->stream;
  CU_TRY(cudaMemsetAsync(X.p, 0, col * dk, st));
  const double one[2] = {1.0, 0.0};
  for (int64_t j = 0; j < dk; ++j)
    CU_TRY(cudaMemcpyAsync(X.as<double2>() + j * dk + j, one, sizeof(double2), cudaMemcpyHostToDevice, st));
  for (int64_t j = 0; j < dk; ++j) {
    const int rc = orbit_apply_dev(o, X.as<double2>() + j * dk, Y.as<double2>() + j * dk, st);
    if (rc) return rc;
  }
  const std::vector<double> half(static_cast<size_t>(m), 0.5);
  CU_TRY(cudaMemcpyAsync(w.p, half.data(), m * sizeof(double), cudaMemcpyHostToDevice, st));
  CU_TRY(cudaMemcpyAsync(nn.p, &m, sizeof(int), cudaMemcpyHostToDevice, st));
  if (n_bt > 0) CU_TRY(cudaMemcpyAsync(bt.p, bts, n_bt * sizeof(double), cudaMemcpyHostToDevice, st));
  CU_TRY(embed_hermitian(Y.as<double2>(), static_cast<int>(dk), Rm.as<double>(), st));
  CU_TRY(symeig_dense(Rm.as<double>(), nn.as<int>(), 1, m, lam.as<double>(), info.as<int>(), st));
  CU_TRY(quad_eval(lam.as<double>(), w.as<double>(), nn.as<int>(), 1, m, bt.as<double>(), n_bt, lq.as<double>(),
                   eq.as<double>(), st));
  int h_info = 0;
  CU_TRY(cudaMemcpyAsync(&h_info, info.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (n_bt > 0) {
    CU_TRY(cudaMemcpyAsync(lnz, lq.p, n_bt * sizeof(double), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaMemcpyAsync(energy, eq.p, n_bt * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CU_TRY(cudaStreamSynchronize(st));
  if (h_info != 0) return fail(FTLM_ERR_NUMERIC, "GPU Jacobi eigen-solver did not converge");
  return FTLM_OK;
}

// All momentum blocks of a sector (ky outer, kx inner): blocks with dim <= ed_cutoff exactly
// (the k-bench's --ed-cutoff, default 64), larger ones by FTLM with seed_k = seed + sector_index*257 +
// ky*17 + kx; ln Z_sector = log-sum-exp over blocks (benchmarks/bench_ftlm_nmu_4x4_k.cpp:801-1081).
static int orbit_sector_impl(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed,
                             int sector_index, int start_mode, int ed_cutoff, bool batched, double* lnz, double* energy,
                             long long* dims_k) {
  int rc = need_device(s);
  if (rc) return rc;
  if (n_bt <= 0 || !bts || !lnz || !energy) return fail(FTLM_ERR_INVALID, "bad arguments");
  rc = build_orbit_sector(s);
  if (rc) return rc;
  std::vector<double> acc(static_cast<size_t>(n_bt), -std::numeric_limits<double>::infinity());
  std::vector<double> eacc(static_cast<size_t>(n_bt), 0.0);
  std::vector<double> lk(static_cast<size_t>(n_bt)), ek(static_cast<size_t>(n_bt));
  for (int ky = 0; ky < s->Ly; ++ky)
    for (int kx = 0; kx < s->Lx; ++kx) {
      ftlm_orbit* o = nullptr;
      rc = ftlm_gpu_orbit_create(s, kx, ky, &o);
      if (rc) return rc;
      if (dims_k) dims_k[ky * s->Lx + kx] = o->dk;
      if (o->dk > 0) {
        const unsigned seed_k = seed + static_cast<unsigned>(sector_index * 257 + ky * 17 + kx);
        if (o->dk <= ed_cutoff)
          rc = o->dk == 1 ? ftlm_gpu_orbit_ftlm(o, bts, n_bt, R, M, seed_k, start_mode, lk.data(), ek.data())
                          : orbit_block_ed(o, bts, n_bt, lk.data(), ek.data());
        else if (batched)
          rc = ftlm_gpu_orbit_batched_ftlm(o, bts, n_bt, R, M, seed_k, lk.data(), ek.data());
        else
          rc = ftlm_gpu_orbit_ftlm(o, bts, n_bt, R, M, seed_k, start_mode, lk.data(), ek.data());
        if (rc) {
          ftlm_gpu_orbit_destroy(o);
          return rc;
        }
        for (int b = 0; b < n_bt; ++b) {  // running log-sum-exp, energy weighted by e^{ln Z_K}
          const double a = acc[static_cast<size_t>(b)], x = lk[static_cast<size_t>(b)];
          if (!std::isfinite(x)) continue;
          if (!std::isfinite(a)) {
            acc[static_cast<size_t>(b)] = x;
            eacc[static_cast<size_t>(b)] = ek[static_cast<size_t>(b)];
            continue;
          }
          const double m = std::max(a, x);
          const double wa = std::exp(a - m), wx = std::exp(x - m);
          acc[static_cast<size_t>(b)] = m + std::log(wa + wx);
          eacc[static_cast<size_t>(b)] = (wa * eacc[static_cast<size_t>(b)] + wx * ek[static_cast<size_t>(b)]) / (wa + wx);
        }
      }
      ftlm_gpu_orbit_destroy(o);
    }
  std::copy(acc.begin(), acc.end(), lnz);
  std::copy(eacc.begin(), eacc.end(), energy);
  return FTLM_OK;
}

int ftlm_gpu_orbit_sector_ftlm(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed,
                               int sector_index, int start_mode, int ed_cutoff, double* lnz, double* energy,
                               long long* dims_k) {
  return orbit_sector_impl(s, bts, n_bt, R, M, seed, sector_index, start_mode, ed_cutoff, false, lnz, energy, dims_k);
}

int ftlm_gpu_orbit_sector_batched_ftlm(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed,
                                       int sector_index, int ed_cutoff, double* lnz, double* energy, long long* dims_k) {
  return orbit_sector_impl(s, bts, n_bt, R, M, seed, sector_index, FTLM_START_PHILOX, ed_cutoff, true, lnz, energy,
                           dims_k);
}

}  // extern "C"
