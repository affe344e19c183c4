#include "capi_internal.hpp"

using namespace ftlm_b200;
using namespace ftlm_b200::capi;

// ---------------------------------------------------------------------------------------------
// Parameter gradient of the sector FTLM estimate (no reference counterpart).
//
// For one chain with normalised start vector r, Lanczos vectors q_i and tridiagonal T, the
// estimator term is g = e_1^T e^{-bT T} e_1 and, with r fixed, its exact derivative in the Krylov
// space is dg/dtheta = -sum_il K_il <q_i| dH/dtheta |q_l> (Duhamel; K from duhamel_weights).  The
// chains are replayed from their seed with the forward's kernels (bit-identical alpha/beta), the
// vectors kept on the device, and the three moments of dH/dU (double occupancy), dH/dV (neighbour
// pair density) and dH/dt' (the t' hopping operator) reduced by grad.cu.
namespace {

struct ChainGrad {
  bool ok = false;
  double lmin = 0.0, g = 0.0, m[3] = {0.0, 0.0, 0.0};
};

// Weight matrices of up to nc chains on the GPU (symeig.cu: Jacobi eigen-decomposition of each
// chain's tridiagonal, then K = Z P Z^T), written to g_grad.Kp in the layout [i][ld][nc] (chain
// fastest) with the scales 1/(sc_i sc_l); g and the lowest Ritz value per chain to `out`.
int fill_weights(ftlm_sector* s, int nc, int ld, double bT, const std::vector<int>& n, const std::vector<double>& A,
                 const std::vector<double>& B, const std::vector<std::vector<double>>& scale,
                 std::vector<ChainGrad>* out) {
  cudaStream_t st = s->stream;
  std::vector<double> sc(static_cast<size_t>(nc) * ld, 1.0);
  for (int c = 0; c < nc; ++c)
    for (size_t i = 0; i < scale[static_cast<size_t>(c)].size() && i < static_cast<size_t>(ld); ++i)
      sc[static_cast<size_t>(c) * ld + i] = scale[static_cast<size_t>(c)][i];
  const size_t mat = static_cast<size_t>(nc) * ld * sizeof(double);
  DevBuf da, db, dn, dsc, dl, dvt, dy, dg, dlm, di;
  CU_TRY(da.alloc(mat));
  CU_TRY(db.alloc(mat));
  CU_TRY(dn.alloc(nc * sizeof(int)));
  CU_TRY(dsc.alloc(mat));
  CU_TRY(dl.alloc(mat));
  CU_TRY(dvt.alloc(mat * ld));
  CU_TRY(dy.alloc(mat * ld));
  CU_TRY(dg.alloc(nc * sizeof(double)));
  CU_TRY(dlm.alloc(nc * sizeof(double)));
  CU_TRY(di.alloc(nc * sizeof(int)));
  CU_TRY(cudaMemcpyAsync(da.p, A.data(), mat, cudaMemcpyHostToDevice, st));
  CU_TRY(cudaMemcpyAsync(db.p, B.data(), mat, cudaMemcpyHostToDevice, st));
  CU_TRY(cudaMemcpyAsync(dn.p, n.data(), nc * sizeof(int), cudaMemcpyHostToDevice, st));
  CU_TRY(cudaMemcpyAsync(dsc.p, sc.data(), mat, cudaMemcpyHostToDevice, st));
  CU_TRY(cudaMemsetAsync(dg.p, 0, nc * sizeof(double), st));
  CU_TRY(g_grad.grow(g_grad.Kp, g_grad.kcap, static_cast<size_t>(ld) * ld * nc * sizeof(double)));
  CU_TRY(cudaMemsetAsync(g_grad.Kp.p, 0, static_cast<size_t>(ld) * ld * nc * sizeof(double), st));
  CU_TRY(symeig_tridiag(da.as<double>(), db.as<double>(), dn.as<int>(), nc, ld, dl.as<double>(), nullptr,
                        dvt.as<double>(), di.as<int>(), st));
  CU_TRY(duhamel_weights_dev(dl.as<double>(), dvt.as<double>(), dn.as<int>(), nc, ld, bT, dsc.as<double>(),
                             dy.as<double>(), g_grad.Kp.as<double>(), dg.as<double>(), dlm.as<double>(), st));
  std::vector<double> g(static_cast<size_t>(nc)), lm(static_cast<size_t>(nc));
  std::vector<int> info(static_cast<size_t>(nc));
  CU_TRY(cudaMemcpyAsync(g.data(), dg.p, nc * sizeof(double), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaMemcpyAsync(lm.data(), dlm.p, nc * sizeof(double), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaMemcpyAsync(info.data(), di.p, nc * sizeof(int), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  for (int c = 0; c < nc; ++c) {
    ChainGrad& cg = (*out)[static_cast<size_t>(c)];
    cg = ChainGrad{};
    if (n[static_cast<size_t>(c)] <= 0) continue;
    if (info[static_cast<size_t>(c)] != 0) return fail(FTLM_ERR_NUMERIC, "GPU Jacobi eigen-solver did not converge");
    cg.ok = true;
    cg.g = g[static_cast<size_t>(c)];
    cg.lmin = lm[static_cast<size_t>(c)];
  }
  return FTLM_OK;
}

// Moments of one batch of chains: Q [n][vstride], AQ likewise (or null), weights already in
// g_grad.Kp [n][ld][nc] (fill_weights).
template <class T>
int run_moments(ftlm_sector* s, const T* Q, const T* AQ, int64_t vstride, int n, int ld, int nc,
                std::vector<ChainGrad>* out) {
  cudaStream_t st = s->stream;
  CU_TRY(g_grad.grow(g_grad.part, g_grad.pcap, static_cast<size_t>(2048) * 32 * 3 * sizeof(double)));
  int grid = 0;
  cudaError_t e;
  if constexpr (sizeof(T) == sizeof(float2))
    e = grad_moments_c64(s->dev, Q, AQ ? AQ : Q, vstride, g_grad.Kp.as<double>(), n, ld, g_grad.part.as<double>(), &grid, st);
  else
    e = grad_moments_c128(s->dev, Q, AQ ? AQ : Q, vstride, g_grad.Kp.as<double>(), n, ld, g_grad.part.as<double>(), &grid,
                          st);
  if (e == cudaErrorInvalidValue)
    return fail(FTLM_ERR_UNSUPPORTED, "gradient: Lanczos vectors of one block do not fit in shared memory");
  CU_TRY(e);
  std::vector<double> hp(static_cast<size_t>(grid) * nc * 3);
  CU_TRY(cudaMemcpyAsync(hp.data(), g_grad.part.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  CU_TRY(cudaStreamSynchronize(st));
  for (int c = 0; c < nc; ++c) {
    ChainGrad& cg = (*out)[static_cast<size_t>(c)];
    for (int q = 0; q < 3; ++q) {
      double sum = 0.0;
      for (int b = 0; b < grid; ++b) sum += hp[(static_cast<size_t>(b) * nc + c) * 3 + q];
      cg.m[q] = sum;
    }
  }
  return FTLM_OK;
}

// Plain path: complex128 chains of ftlm_gpu_ftlm_sector (seed_r = seed + r*100003).
int grad_plain(ftlm_sector* s, ftlm_sector* op, double bT, int R, int M, unsigned seed, int start_mode,
               std::vector<ChainGrad>* out) {
  const int64_t dim = s->plan.dim;
  CU_TRY(g_grad.grow(g_grad.Q, g_grad.qcap, static_cast<size_t>(M) * dim * sizeof(double2)));
  if (op) CU_TRY(g_grad.grow(g_grad.AQ, g_grad.acap, static_cast<size_t>(M) * dim * sizeof(double2)));
  double2* Q = g_grad.Q.as<double2>();
  double2* AQ = op ? g_grad.AQ.as<double2>() : nullptr;
  out->assign(static_cast<size_t>(R), ChainGrad{});
  std::vector<ChainGrad> one(1);
  for (int r = 0; r < R; ++r) {
    std::vector<double> a, b;
    int rc = run_lanczos(
        dim, [s](const double2* x, double2* y, cudaStream_t st) { return s->apply(x, y, st); }, s->ws, M,
        seed + static_cast<unsigned>(r) * 100003u, start_mode, s->stream, &a, &b, Q);
    if (rc) return rc;
    const int n = static_cast<int>(a.size());
    if (n <= 0) continue;
    std::vector<double> A(static_cast<size_t>(M), 0.0), B(static_cast<size_t>(M), 0.0);
    std::copy(a.begin(), a.end(), A.begin());
    std::copy(b.begin(), b.begin() + std::min<size_t>(b.size(), static_cast<size_t>(M)), B.begin());
    if (op)
      for (int i = 0; i < n; ++i) {
        rc = op->apply(Q + static_cast<int64_t>(i) * dim, AQ + static_cast<int64_t>(i) * dim, s->stream);
        if (rc) return rc;
      }
    std::vector<std::vector<double>> scale(1, std::vector<double>(static_cast<size_t>(n), 1.0));
    rc = fill_weights(s, 1, M, bT, std::vector<int>{n}, A, B, scale, &one);
    if (rc) return rc;
    rc = run_moments<double2>(s, Q, AQ, dim, n, M, 1, &one);
    if (rc) return rc;
    (*out)[static_cast<size_t>(r)] = one[0];
  }
  return FTLM_OK;
}

// Batched path: complex64 32-chain blocks of ftlm_gpu_batched_ftlm_sector, replayed step by step.
int grad_batched(ftlm_sector* s, ftlm_sector* op, double bT, int R, int M, unsigned seed, std::vector<ChainGrad>* out) {
  const int64_t dim = s->plan.dim;
  const int64_t vs = dim * kBtChains;
  std::lock_guard<std::mutex> lock(g_bt_mu);
  CU_TRY(g_bt.ensure(dim, M));
  CU_TRY(g_grad.grow(g_grad.Q, g_grad.qcap, static_cast<size_t>(M + 1) * vs * sizeof(float2)));
  if (op) CU_TRY(g_grad.grow(g_grad.AQ, g_grad.acap, static_cast<size_t>(M) * vs * sizeof(float2)));
  if (!g_grad.stunit.p) {
    std::vector<double> unit(static_cast<size_t>(kBtFields) * kBtChains, 0.0);
    for (int c = 0; c < kBtChains; ++c) unit[static_cast<size_t>(kBtSin) * kBtChains + c] = 1.0;
    CU_TRY(g_grad.stunit.alloc(unit.size() * sizeof(double)));
    CU_TRY(cudaMemcpy(g_grad.stunit.p, unit.data(), unit.size() * sizeof(double), cudaMemcpyHostToDevice));
    CU_TRY(g_grad.zflag.alloc(sizeof(int)));
    CU_TRY(cudaMemset(g_grad.zflag.p, 0, sizeof(int)));
  }
  cudaStream_t st = s->stream;
  float2* Q = g_grad.Q.as<float2>();
  float2* AQ = op ? g_grad.AQ.as<float2>() : nullptr;
  double* sd = g_bt.st.as<double>();
  double* part = g_bt.partial.as<double>();
  double* al = g_bt.alpha.as<double>();
  double* be = g_bt.beta.as<double>();
  int* us = g_bt.used.as<int>();
  int* fl = g_bt.flags.as<int>();
  out->assign(static_cast<size_t>(R), ChainGrad{});
  std::vector<double> ha(static_cast<size_t>(M) * kBtChains), hb(static_cast<size_t>(M) * kBtChains),
      hs(static_cast<size_t>(kBtFields) * kBtChains);
  std::vector<int> hu(kBtChains);
  for (int blk = 0; blk * kBtChains < R; ++blk) {
    const unsigned seed_b = seed + static_cast<unsigned>(blk * kBtChains) * 100003u;
    CU_TRY(cudaMemsetAsync(al, 0, static_cast<size_t>(M) * kBtChains * sizeof(double), st));
    CU_TRY(cudaMemsetAsync(be, 0, static_cast<size_t>(M) * kBtChains * sizeof(double), st));
    CU_TRY(bt_start(Q, dim, seed_b, sd, part, us, fl, st, &s->dev));
    CU_TRY(cudaMemcpyAsync(hs.data(), sd, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    for (int k = 0; k < M; ++k)
      CU_TRY(bt_step(s->dev, Q + static_cast<int64_t>(k) * vs, Q + static_cast<int64_t>(k > 0 ? k - 1 : 0) * vs,
                     Q + static_cast<int64_t>(k + 1) * vs, k, sd, part, al, be, us, fl, st));
    CU_TRY(cudaMemcpyAsync(ha.data(), al, ha.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaMemcpyAsync(hb.data(), be, hb.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaMemcpyAsync(hu.data(), us, hu.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    CU_TRY(cudaStreamSynchronize(st));
    const int nc = std::min(kBtChains, R - blk * kBtChains);
    std::vector<int> n(static_cast<size_t>(kBtChains), 0);
    std::vector<double> A(static_cast<size_t>(kBtChains) * M, 0.0), B(static_cast<size_t>(kBtChains) * M, 0.0);
    std::vector<std::vector<double>> scale(static_cast<size_t>(kBtChains));
    int nmax = 0;
    for (int c = 0; c < nc; ++c) {
      const double sin0 = hs[static_cast<size_t>(kBtSin) * kBtChains + c];
      const int nn = (sin0 > 0.0) ? hu[static_cast<size_t>(c)] : 0;
      n[static_cast<size_t>(c)] = nn;
      nmax = std::max(nmax, nn);
      auto& sc = scale[static_cast<size_t>(c)];
      sc.assign(static_cast<size_t>(std::max(nn, 1)), 1.0);
      for (int k = 0; k < M; ++k) {
        A[static_cast<size_t>(c) * M + k] = ha[static_cast<size_t>(k) * kBtChains + c];
        B[static_cast<size_t>(c) * M + k] = hb[static_cast<size_t>(k) * kBtChains + c];
      }
      if (nn > 0) {  // W_0 = ||raw|| q_0, W_i = beta_{i-1} q_i
        sc[0] = 1.0 / sin0;
        for (int i = 1; i < nn; ++i) sc[static_cast<size_t>(i)] = B[static_cast<size_t>(c) * M + i - 1];
      }
    }
    if (nmax == 0) continue;
    if (op)
      for (int i = 0; i < nmax; ++i)
        CU_TRY(bt_apply(op->dev, Q + static_cast<int64_t>(i) * vs, AQ + static_cast<int64_t>(i) * vs,
                        g_grad.stunit.as<double>(), part, g_grad.zflag.as<int>(), st));
    std::vector<ChainGrad> cg(static_cast<size_t>(kBtChains));
    int rc = fill_weights(s, kBtChains, M, bT, n, A, B, scale, &cg);
    if (rc) return rc;
    rc = run_moments<float2>(s, Q, AQ, vs, nmax, M, kBtChains, &cg);
    if (rc) return rc;
    for (int c = 0; c < nc; ++c) (*out)[static_cast<size_t>(blk * kBtChains + c)] = cg[static_cast<size_t>(c)];
  }
  return FTLM_OK;
}

}  // namespace

extern "C" {

int ftlm_gpu_grad_sector(ftlm_sector* s, ftlm_sector* op_tp, double bT, int R, int M, unsigned seed, int method,
                         int start_mode, double* lnz, double* dlnz) {
  int rc = need_device(s);
  if (rc) return rc;
  if (op_tp) {
    rc = need_device(op_tp);
    if (rc) return rc;
    if (op_tp->plan.n != s->plan.n || op_tp->plan.nu != s->plan.nu || op_tp->plan.nd != s->plan.nd)
      return fail(FTLM_ERR_INVALID, "gradient operator sector has a different (n_sites, N_up, N_dn)");
  }
  if (!lnz || !dlnz || method < 0 || method > 1) return fail(FTLM_ERR_INVALID, "bad arguments");
  R = std::max(1, R);
  M = std::max(1, M);
  if (M > kMaxEig) return fail(FTLM_ERR_UNSUPPORTED, "more than 160 Lanczos steps for the GPU eigen-solver");
  const int64_t dim = s->plan.dim;
  std::vector<ChainGrad> cg;
  if (method == 1 && dim > 2 * static_cast<int64_t>(M)) {
    if (s->plan.max_up_deg > 120 || (op_tp && op_tp->plan.max_up_deg > 120))
      return fail(FTLM_ERR_UNSUPPORTED, "batched path: more than 120 up-hop sources per string");
    rc = grad_batched(s, op_tp, bT, R, M, seed, &cg);
  } else {
    rc = grad_plain(s, op_tp, bT, R, M, seed, method == 1 ? FTLM_START_PHILOX : start_mode, &cg);
  }
  if (rc) return rc;
  // ln Z = ln dim + log mean_r g_r, g_r = e^{-bT lmin_r} ghat_r; d ln Z = -sum_r e^{-bT lmin_r} m_r / sum_r g_r
  double mx = -std::numeric_limits<double>::infinity();
  int used = 0;
  for (const auto& c : cg)
    if (c.ok) {
      mx = std::max(mx, -bT * c.lmin + std::log(c.g));
      ++used;
    }
  if (used == 0) {
    *lnz = -std::numeric_limits<double>::infinity();
    dlnz[0] = dlnz[1] = dlnz[2] = 0.0;
    return FTLM_OK;
  }
  double zs = 0.0, d[3] = {0.0, 0.0, 0.0};
  for (const auto& c : cg) {
    if (!c.ok) continue;
    const double w = std::exp(-bT * c.lmin - mx);
    zs += w * c.g;
    for (int q = 0; q < 3; ++q) d[q] -= w * c.m[q];
  }
  *lnz = std::log(static_cast<double>(dim)) + mx + std::log(zs / static_cast<double>(used));
  for (int q = 0; q < 3; ++q) dlnz[q] = d[q] / zs;
  if (!op_tp) dlnz[2] = 0.0;
  return FTLM_OK;
}

// ---- differentiable grand-canonical ln Z at one (T, mu) ----------------------------------------
// Forward: every sector's chains as the FTLM entry points make them (the small sectors' chains in
// one fused launch), the converged tridiagonal quadrature, the sector combine
// (src/ftlm_thermo.cpp:246-256) and the grand-canonical log-sum-exp of
// benchmarks/bench_ftlm_nmu_rect.cpp:186-219 at a single (T, mu).  Backward: d/dmu = bT <N>,
// d/dbT = <mu N - E>, and d/d(U, V, t') = sum_s w_s d ln Z_s/dtheta from ftlm_gpu_grad_sector
// (sectors with weight w_s < 1e-13 skipped).
namespace {

constexpr double kGcWeightCutoff = 1e-13;
constexpr long long kGcFusedPlainMax = 1LL << 17;

struct SectorDeleter {
  void operator()(ftlm_sector* s) const { ftlm_gpu_sector_destroy(s); }
};
using SectorPtr = std::unique_ptr<ftlm_sector, SectorDeleter>;

int gc_check(const ftlm_params* p, double bT, int R, int M, int method, int start_mode) {
  if (!p) return fail(FTLM_ERR_INVALID, "null params");
  const int n = p->Lx * p->Ly;
  if (p->Lx <= 0 || p->Ly <= 0 || n > 32) return fail(FTLM_ERR_INVALID, "FockBasis: require 1 <= n_sites <= 32");
  if (R <= 0 || M <= 0 || M > 160) return fail(FTLM_ERR_INVALID, "require R > 0 and 0 < M <= 160");
  if (method < 0 || method > 1) return fail(FTLM_ERR_INVALID, "method must be 0 (plain) or 1 (batched)");
  if (start_mode != FTLM_START_REFERENCE && start_mode != FTLM_START_PHILOX)
    return fail(FTLM_ERR_INVALID, "unknown start_mode");
  if (!(bT > 0.0) || !std::isfinite(bT)) return fail(FTLM_ERR_INVALID, "inverse temperature must be finite and > 0");
  return FTLM_OK;
}

// ln Z_s, E_s at bT from R chains (alpha/beta [R][M], used [R]) of a sector of size dim.
int gc_quadrature(const double* A, const double* B, const int* used, int R, int M, double bT, int64_t dim,
                  double* lnz, double* en) {
  std::vector<double> lq(static_cast<size_t>(R)), eq(static_cast<size_t>(R));
  int rc = ftlm_gpu_tridiag_quadrature_exact(A, B, used, R, M, &bT, 1, lq.data(), eq.data());
  if (rc) return rc;
  return ftlm_gpu_ftlm_combine(lq.data(), eq.data(), used, R, 1, std::log(static_cast<double>(dim)), lnz, en);
}

double gc_lse(const std::vector<double>& x) {
  double mx = -std::numeric_limits<double>::infinity();
  for (double v : x) mx = std::max(mx, v);
  if (!std::isfinite(mx)) return mx;
  double s = 0.0;
  for (double v : x) s += std::exp(v - mx);
  return mx + std::log(s);
}

}  // namespace

int ftlm_gpu_gc_logz(const ftlm_params* p, double mu, double bT, int R, int M, unsigned seed, int method,
                     int start_mode, double* lnz_s, double* e_s, double* lnz_gc) {
  int rc = gc_check(p, bT, R, M, method, start_mode);
  if (rc) return rc;
  if (!lnz_s || !e_s || !lnz_gc) return fail(FTLM_ERR_INVALID, "null output");
  const int n = p->Lx * p->Ly;
  const int nsec = (n + 1) * (n + 1);
  const int st_mode = method == 1 ? FTLM_START_PHILOX : start_mode;
  const long long limit = method == 1 ? 2LL * M : kGcFusedPlainMax;
  std::vector<SectorPtr> small;
  std::vector<int> small_idx;
  std::vector<double> A, B;
  std::vector<int> used;
  for (int nu = 0; nu <= n; ++nu)
    for (int nd = 0; nd <= n; ++nd) {
      const int idx = nu * (n + 1) + nd;
      ftlm_sector* raw = nullptr;
      rc = ftlm_gpu_sector_create(p, nu, nd, &raw);
      if (rc) return rc;
      SectorPtr s(raw);
      const int64_t dim = s->plan.dim;
      if (dim <= limit) {  // chains of all small sectors in one launch below
        small.push_back(std::move(s));
        small_idx.push_back(idx);
        continue;
      }
      if (method == 1) {
        rc = need_device(s.get());
        if (rc) return rc;
        if (s->plan.max_up_deg > 120)
          return fail(FTLM_ERR_UNSUPPORTED, "batched path: more than 120 up-hop sources per string");
        rc = bt_run_chains(s.get(), R, M, seed, &A, &B, &used);
        if (rc) return rc;
      } else {
        A.assign(static_cast<size_t>(R) * M, 0.0);
        B.assign(static_cast<size_t>(R) * M, 0.0);
        used.assign(static_cast<size_t>(R), 0);
        for (int r = 0; r < R; ++r) {
          int nb = 0, u = 0;
          rc = ftlm_gpu_lanczos(s.get(), M, seed + static_cast<unsigned>(r) * 100003u, st_mode,
                                A.data() + static_cast<size_t>(r) * M, B.data() + static_cast<size_t>(r) * M, &nb, &u);
          if (rc) return rc;
          used[static_cast<size_t>(r)] = u;
        }
      }
      rc = gc_quadrature(A.data(), B.data(), used.data(), R, M, bT, dim, lnz_s + idx, e_s + idx);
      if (rc) return rc;
    }
  if (!small.empty()) {
    std::vector<ftlm_sector*> hs;
    for (auto& s : small) hs.push_back(s.get());
    const size_t ns = hs.size();
    A.assign(ns * R * M, 0.0);
    B.assign(ns * R * M, 0.0);
    used.assign(ns * R, 0);
    rc = ftlm_gpu_lanczos_sectors(hs.data(), static_cast<int>(ns), R, M, seed, st_mode, A.data(), B.data(), used.data());
    if (rc) return rc;
    for (size_t i = 0; i < ns; ++i) {
      rc = gc_quadrature(A.data() + i * R * M, B.data() + i * R * M, used.data() + i * R, R, M, bT, hs[i]->plan.dim,
                         lnz_s + small_idx[i], e_s + small_idx[i]);
      if (rc) return rc;
    }
  }
  std::vector<double> x(static_cast<size_t>(nsec));
  for (int nu = 0; nu <= n; ++nu)
    for (int nd = 0; nd <= n; ++nd) {
      const int idx = nu * (n + 1) + nd;
      x[static_cast<size_t>(idx)] = lnz_s[idx] + bT * mu * static_cast<double>(nu + nd);
    }
  *lnz_gc = gc_lse(x);
  return FTLM_OK;
}

int ftlm_gpu_gc_logz_grad(const ftlm_params* p, double mu, double bT, int R, int M, unsigned seed, int method,
                          int start_mode, const double* lnz_s, const double* e_s, double* grad) {
  int rc = gc_check(p, bT, R, M, method, start_mode);
  if (rc) return rc;
  if (!lnz_s || !e_s || !grad) return fail(FTLM_ERR_INVALID, "null argument");
  const int n = p->Lx * p->Ly;
  const int nsec = (n + 1) * (n + 1);
  std::vector<double> x(static_cast<size_t>(nsec)), N(static_cast<size_t>(nsec));
  for (int nu = 0; nu <= n; ++nu)
    for (int nd = 0; nd <= n; ++nd) {
      const int idx = nu * (n + 1) + nd;
      N[static_cast<size_t>(idx)] = static_cast<double>(nu + nd);
      x[static_cast<size_t>(idx)] = lnz_s[idx] + bT * mu * N[static_cast<size_t>(idx)];
    }
  const double lnZ = gc_lse(x);
  if (!std::isfinite(lnZ)) return fail(FTLM_ERR_NUMERIC, "grand-canonical ln Z is not finite");
  double d[3] = {0.0, 0.0, 0.0}, dmu = 0.0, dbeta = 0.0;
  ftlm_params pop = *p;  // dH/dt': the t' hopping operator alone
  pop.t = 0.0;
  pop.tp = 1.0;
  pop.U = 0.0;
  pop.V = 0.0;
  for (int nu = 0; nu <= n; ++nu)
    for (int nd = 0; nd <= n; ++nd) {
      const size_t idx = static_cast<size_t>(nu * (n + 1) + nd);
      const double w = std::exp(x[idx] - lnZ);
      if (!(w > 0.0)) continue;
      dmu += bT * w * N[idx];
      dbeta += w * (mu * N[idx] - e_s[idx]);
      if (!(w >= kGcWeightCutoff)) continue;
      ftlm_sector *rs = nullptr, *ro = nullptr;
      rc = ftlm_gpu_sector_create(p, nu, nd, &rs);
      if (rc) return rc;
      SectorPtr s(rs);
      rc = ftlm_gpu_sector_create(&pop, nu, nd, &ro);
      if (rc) return rc;
      SectorPtr op(ro);
      double lz = 0.0, g[3] = {0.0, 0.0, 0.0};
      rc = ftlm_gpu_grad_sector(s.get(), op.get(), bT, R, M, seed, method, start_mode, &lz, g);
      if (rc) return rc;
      if (!(std::fabs(lz - lnz_s[idx]) <= 1e-9 * std::max(1.0, std::fabs(lz))))
        return fail(FTLM_ERR_NUMERIC, "gradient replay of sector (" + std::to_string(nu) + "," + std::to_string(nd) +
                                          ") did not reproduce the forward ln Z");
      for (int q = 0; q < 3; ++q) d[q] += w * g[q];
    }
  grad[0] = d[0];
  grad[1] = d[1];
  grad[2] = d[2];
  grad[3] = dmu;
  grad[4] = dbeta;
  return FTLM_OK;
}

// Per-chain log quadrature and energy ratio with a converged eigen-decomposition (parallel cyclic
// Jacobi on the GPU, symeig.cu), the quadrature the gradient differentiates; same layout as
// ftlm_gpu_tridiag_quadrature.
int ftlm_gpu_tridiag_quadrature_exact(const double* alpha, const double* beta, const int* n, int nc, int ld,
                                      const double* bts, int n_bt, double* logq, double* energy) {
  if (nc < 0 || ld <= 0 || n_bt < 0 || !alpha || !beta || !n || (n_bt > 0 && (!bts || !logq || !energy)))
    return fail(FTLM_ERR_INVALID, "bad arguments");
  if (ld > kMaxEig) return fail(FTLM_ERR_UNSUPPORTED, "tridiagonal size > 160 is not supported by the GPU eigen-solver");
  for (int c = 0; c < nc; ++c)
    if (n[c] < 0 || n[c] > ld) return fail(FTLM_ERR_INVALID, "chain length outside [0, ld]");
  if (static_cast<long long>(nc) * n_bt > 0x7fffffffLL) return fail(FTLM_ERR_INVALID, "n_chains * n_bt exceeds 2^31 - 1");
  if (nc == 0 || n_bt == 0) return FTLM_OK;
  const size_t mat = static_cast<size_t>(nc) * ld * sizeof(double);
  const size_t outb = static_cast<size_t>(nc) * n_bt * sizeof(double);
  DevBuf da, db, dn, dl, dw, dbt, dq, de, di;
  CU_TRY(da.alloc(mat));
  CU_TRY(db.alloc(mat));
  CU_TRY(dn.alloc(nc * sizeof(int)));
  CU_TRY(dl.alloc(mat));
  CU_TRY(dw.alloc(mat));
  CU_TRY(dbt.alloc(n_bt * sizeof(double)));
  CU_TRY(dq.alloc(outb));
  CU_TRY(de.alloc(outb));
  CU_TRY(di.alloc(nc * sizeof(int)));
  CU_TRY(cudaMemcpy(da.p, alpha, mat, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(db.p, beta, mat, cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(dn.p, n, nc * sizeof(int), cudaMemcpyHostToDevice));
  CU_TRY(cudaMemcpy(dbt.p, bts, n_bt * sizeof(double), cudaMemcpyHostToDevice));
  CU_TRY(symeig_tridiag(da.as<double>(), db.as<double>(), dn.as<int>(), nc, ld, dl.as<double>(), dw.as<double>(),
                        nullptr, di.as<int>(), nullptr));
  CU_TRY(quad_eval(dl.as<double>(), dw.as<double>(), dn.as<int>(), nc, ld, dbt.as<double>(), n_bt, dq.as<double>(),
                   de.as<double>(), nullptr));
  std::vector<int> info(static_cast<size_t>(nc));
  CU_TRY(cudaMemcpy(info.data(), di.p, nc * sizeof(int), cudaMemcpyDeviceToHost));
  for (int c = 0; c < nc; ++c)
    if (n[c] > 0 && info[static_cast<size_t>(c)] != 0) return fail(FTLM_ERR_NUMERIC, "GPU Jacobi eigen-solver did not converge");
  CU_TRY(cudaMemcpy(logq, dq.p, outb, cudaMemcpyDeviceToHost));
  CU_TRY(cudaMemcpy(energy, de.p, outb, cudaMemcpyDeviceToHost));
  return FTLM_OK;
}

// Host-only helper exposed for tests: eigenvalues/eigenvectors of a symmetric tridiagonal.
int ftlm_gpu_tridiag_eigvec(const double* alpha, const double* beta, int n, double* lam, double* Z) {
  if (n < 0 || (n > 0 && (!alpha || !lam || !Z || (n > 1 && !beta)))) return fail(FTLM_ERR_INVALID, "bad arguments");
  const std::string err = tridiag_eigvec(n, alpha, beta, lam, Z);
  if (!err.empty()) return fail(FTLM_ERR_NUMERIC, err);
  return FTLM_OK;
}

// Host-only helper exposed for tests: the Duhamel weight matrix of one tridiagonal.
int ftlm_gpu_duhamel_weights(const double* alpha, const double* beta, int n, double bT, double* K, double* g,
                             double* lam_min) {
  if (n < 0 || (n > 0 && (!alpha || !K || !g || (n > 1 && !beta)))) return fail(FTLM_ERR_INVALID, "bad arguments");
  const std::string err = duhamel_weights(n, alpha, beta, bT, K, g, lam_min);
  if (!err.empty()) return fail(FTLM_ERR_NUMERIC, err);
  return FTLM_OK;
}

}  // extern "C"

