// C ABI of the batched complex64 FTLM (batched.cu): 32 chains per block vector, the M Lanczos steps
// of a block captured once into a CUDA graph and launched without host synchronisation.
#include "capi_internal.hpp"

using namespace ftlm_b200;
using namespace ftlm_b200::capi;

namespace ftlm_b200 {
namespace capi {

BtWs g_bt;
std::mutex g_bt_mu;
GradWs g_grad;

int bt_run_chains(ftlm_sector* s, int R, int M, unsigned seed, std::vector<double>* A, std::vector<double>* B,
                  std::vector<int>* used) {
  cudaStream_t st = s->stream;
  const DevSector& S = s->dev;
  return bt_run_chains_impl(
      s->plan.dim, st,
      [&S, st](const float2* wk, const float2* wkm1, float2* y, int k, double* sd, double* part, double* al, double* be,
               int* us, int* fl) { return bt_step(S, wk, wkm1, y, k, sd, part, al, be, us, fl, st); },
      R, M, seed, A, B, used);
}

}  // namespace capi
}  // namespace ftlm_b200

extern "C" {

int ftlm_gpu_batched_lanczos(ftlm_sector* s, int R, int M, unsigned seed, double* alpha, double* beta, int* used) {
  int rc = need_device(s);
  if (rc) return rc;
  if (s->plan.max_up_deg > 120)
    return fail(FTLM_ERR_UNSUPPORTED, "batched path: more than 120 up-hop sources per string");
  if (R <= 0 || M <= 0 || !alpha || !beta || !used) return fail(FTLM_ERR_INVALID, "bad arguments");
  std::vector<double> A, B;
  std::vector<int> u;
  rc = bt_run_chains(s, R, M, seed, &A, &B, &u);
  if (rc) return rc;
  std::copy(A.begin(), A.end(), alpha);
  std::copy(B.begin(), B.end(), beta);
  std::copy(u.begin(), u.end(), used);
  return FTLM_OK;
}

int ftlm_gpu_batched_ftlm_sector(ftlm_sector* s, const double* bts, int n_bt, int R, int M, unsigned seed, double* lnz,
                                 double* energy) {
  int rc = need_device(s);
  if (rc) return rc;
  if (n_bt < 0 || (n_bt > 0 && (!bts || !lnz || !energy))) return fail(FTLM_ERR_INVALID, "bad arguments");
  R = std::max(1, R);
  M = std::max(1, M);
  if (M > 160) return fail(FTLM_ERR_UNSUPPORTED, "more than 160 Lanczos steps for the on-chip Jacobi");
  const int64_t dim = s->plan.dim;
  // Sectors whose Krylov space the chain can exhaust stay on the complex128 path (same Philox
  // start vectors), where the reference's breakdown test is meaningful.
  if (dim <= 2 * static_cast<int64_t>(M)) return ftlm_gpu_ftlm_sector(s, bts, n_bt, R, M, seed, FTLM_START_PHILOX, lnz, energy);
  if (s->plan.max_up_deg > 120)
    return fail(FTLM_ERR_UNSUPPORTED, "batched path: more than 120 up-hop sources per string");
  std::vector<double> A, B;
  std::vector<int> used;
  rc = bt_run_chains(s, R, M, seed, &A, &B, &used);
  if (rc) return rc;
  std::vector<double> lq(static_cast<size_t>(R) * n_bt), eq(static_cast<size_t>(R) * n_bt);
  rc = ftlm_gpu_tridiag_quadrature(A.data(), B.data(), used.data(), R, M, bts, n_bt, lq.data(), eq.data());
  if (rc) return rc;
  return ftlm_gpu_ftlm_combine(lq.data(), eq.data(), used.data(), R, n_bt, std::log(static_cast<double>(dim)), lnz, energy);
}

int ftlm_gpu_batched_sweep(const ftlm_params* p, int R, int M, unsigned seed, const double* bts, int n_bt,
                           const double* mus, int n_mu, double* lnz_s, double* e_s, double* lnz_gc, double* n_avg,
                           double* e_avg) {
  if (!p || !lnz_s || !e_s) return fail(FTLM_ERR_INVALID, "null argument");
  const int n = p->Lx * p->Ly;
  if (n <= 0 || n > 32) return fail(FTLM_ERR_INVALID, "FockBasis: require 1 <= n_sites <= 32 (bit packing)");
  const int nsec = (n + 1) * (n + 1);
  std::vector<int> N(static_cast<size_t>(nsec));
  // sectors the batched path runs in complex128 (dim <= 2M, Philox starts) go to one fused launch
  std::vector<ftlm_sector*> small;
  std::vector<int> small_idx;
  auto clear_and = [&small](int rc) {
    for (ftlm_sector* x : small) ftlm_gpu_sector_destroy(x);
    small.clear();
    return rc;
  };
  for (int nu = 0; nu <= n; ++nu)
    for (int nd = 0; nd <= n; ++nd) {
      const int idx = nu * (n + 1) + nd;
      N[static_cast<size_t>(idx)] = nu + nd;
      ftlm_sector* s = nullptr;
      int rc = ftlm_gpu_sector_create(p, nu, nd, &s);
      if (rc) return clear_and(rc);
      if (s->plan.dim >= 2 && s->plan.dim <= 2 * static_cast<int64_t>(std::max(1, M)) && M <= 160) {
        small.push_back(s);
        small_idx.push_back(idx);
        continue;
      }
      rc = ftlm_gpu_batched_ftlm_sector(s, bts, n_bt, R, M, seed, lnz_s + static_cast<size_t>(idx) * n_bt,
                                        e_s + static_cast<size_t>(idx) * n_bt);
      ftlm_gpu_sector_destroy(s);
      if (rc) return clear_and(rc);
    }
  const int rcf = fused_sectors_ftlm(small, small_idx, std::max(1, R), std::max(1, M), seed, FTLM_START_PHILOX, bts,
                                     n_bt, lnz_s, e_s);
  clear_and(FTLM_OK);
  if (rcf) return rcf;
  if (lnz_gc && n_avg && e_avg)
    return ftlm_gpu_gc_reduce(lnz_s, e_s, N.data(), nsec, bts, n_bt, mus, n_mu, n, lnz_gc, n_avg, e_avg);
  return FTLM_OK;
}

int ftlm_gpu_batched_release(void) {
  std::lock_guard<std::mutex> lock(g_bt_mu);
  g_bt.release();
  g_grad.release();
  return FTLM_OK;
}

}  // extern "C"

