// Tridiagonal quadrature on the GPU, FP64 (reference src/ftlm_thermo.cpp:17-146, 150-256):
//   quad_jacobi   the reference's classical Jacobi (largest |off-diagonal| first, row-major
//                 first occurrence on ties), one CTA per chain, the dense n x n matrix in shared
//                 memory, only row 0 of the eigenvector matrix carried (rows of V never mix).
//                 Rotation arithmetic uses explicit round-to-nearest operations in the
//                 reference's evaluation order (no contraction), so results follow the
//                 reference's IEEE sequence up to the atan2/cos/sin implementations.
//   quad_eval     log sum_k w_k e^{-b lam_k} (+ the FTLM energy ratio) per chain and temperature.
//   quad_sector   ln(dim) + log mean_r e^{L_r} per temperature (src/ftlm_thermo.cpp:246-256).
//   gc_reduce     grand-canonical mu grid (benchmarks/bench_ftlm_nmu_rect.cpp:186-219).
//   ritz_bisect   exact Ritz values by Sturm-sequence bisection (lowest k).
#include <cfloat>
#include <math_constants.h>

#include "hv.cuh"

namespace ftlm_b200 {

namespace {

constexpr int kJacThreads = 256;

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

__global__ void __launch_bounds__(kJacThreads) jacobi_kernel(const double* __restrict__ alpha,
                                                             const double* __restrict__ beta,
                                                             const int* __restrict__ nv, int ld, int max_rot_in,
                                                             double tol, double* __restrict__ lam,
                                                             double* __restrict__ w0, int* __restrict__ bad) {
  extern __shared__ double sm[];
  __shared__ double red_v[kJacThreads / 32];
  __shared__ int red_i[kJacThreads / 32];
  __shared__ double s_c, s_s, s_app, s_aqq, s_apq;
  __shared__ int s_p, s_q, s_stop;
  const int ch = blockIdx.x;
  int n = nv[ch];
  const int tid = threadIdx.x;
  // A chain length outside [0, ld] would overrun the ld x ld shared matrix and the chain's rows of
  // alpha/beta/lam/w0: such a chain is skipped and reported through *bad (when given).
  if (n < 0 || n > ld) {
    if (tid == 0 && bad) atomicOr(bad, 1);
    n = 0;
  }
  const double* a = alpha + static_cast<int64_t>(ch) * ld;
  const double* b = beta + static_cast<int64_t>(ch) * ld;
  double* lo = lam + static_cast<int64_t>(ch) * ld;
  double* wo = w0 + static_cast<int64_t>(ch) * ld;
  if (n <= 0) return;
  if (n == 1) {
    if (tid == 0) {
      lo[0] = a[0];
      wo[0] = 1.0;
    }
    return;
  }
  double* A = sm;
  double* v0 = sm + n * n;
  for (int i = tid; i < n * n; i += kJacThreads) {
    const int r = i / n, c = i - r * n;
    double v = 0.0;
    if (r == c) v = a[r];
    else if (c == r + 1) v = b[r];
    else if (r == c + 1) v = b[c];
    A[i] = v;
  }
  for (int i = tid; i < n; i += kJacThreads) v0[i] = (i == 0) ? 1.0 : 0.0;
  __syncthreads();
  const int max_rot = max_rot_in > 0 ? max_rot_in : max(3000, 120 * n);
  const int lane = tid & 31, warp = tid >> 5;
  for (int rot = 0; rot < max_rot; ++rot) {
    // Pivot: largest |A_ij| over i<j, first in row-major order (strict > as the reference).
    double best = 0.0;
    int bidx = 0x7fffffff;
    for (int L = tid; L < n * n; L += kJacThreads) {
      const int r = L / n, c = L - r * n;
      if (c <= r) continue;
      const double v = fabs(A[L]);
      if (v > best) {
        best = v;
        bidx = L;
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_down_sync(0xffffffffu, best, off);
      const int oi = __shfl_down_sync(0xffffffffu, bidx, off);
      if (ov > best || (ov == best && oi < bidx)) {
        best = ov;
        bidx = oi;
      }
    }
    if (lane == 0) {
      red_v[warp] = best;
      red_i[warp] = bidx;
    }
    __syncthreads();
    if (tid == 0) {
      double bv = red_v[0];
      int bi = red_i[0];
      for (int w = 1; w < kJacThreads / 32; ++w)
        if (red_v[w] > bv || (red_v[w] == bv && red_i[w] < bi)) {
          bv = red_v[w];
          bi = red_i[w];
        }
      int p = 0, q = 1;
      if (bi != 0x7fffffff) {
        p = bi / n;
        q = bi - p * n;
      }
      s_stop = !(bv >= tol);  // reference: break if max_abs < tol (max_abs starts at 0)
      if (!s_stop) {
        const double app = A[p * n + p], aqq = A[q * n + q], apq = A[p * n + q];
        const double phi = mul(0.5, atan2(mul(2.0, apq), sub(aqq, app)));
        s_c = cos(phi);
        s_s = sin(phi);
        s_app = app;
        s_aqq = aqq;
        s_apq = apq;
        s_p = p;
        s_q = q;
      }
    }
    __syncthreads();
    if (s_stop) break;
    const int p = s_p, q = s_q;
    const double c = s_c, s = s_s;
    for (int k = tid; k < n; k += kJacThreads) {
      if (k == p || k == q) continue;
      const double apk = A[p * n + k], aqk = A[q * n + k];
      const double rpk = sub(mul(c, apk), mul(s, aqk));
      const double rqk = add(mul(c, aqk), mul(s, apk));
      A[p * n + k] = rpk;
      A[k * n + p] = rpk;
      A[q * n + k] = rqk;
      A[k * n + q] = rqk;
    }
    if (tid == 0) {
      const double app = s_app, aqq = s_aqq, apq = s_apq;
      const double cc = mul(c, c), ss = mul(s, s), tsc = mul(mul(2.0, s), c);
      const double npp = add(sub(mul(cc, app), mul(tsc, apq)), mul(ss, aqq));
      const double nqq = add(add(mul(ss, app), mul(tsc, apq)), mul(cc, aqq));
      A[p * n + q] = 0.0;
      A[q * n + p] = 0.0;
      A[p * n + p] = npp;
      A[q * n + q] = nqq;
      const double vip = v0[p], viq = v0[q];
      v0[p] = sub(mul(c, vip), mul(s, viq));
      v0[q] = add(mul(s, vip), mul(c, viq));
    }
    __syncthreads();
  }
  for (int k = tid; k < n; k += kJacThreads) {
    lo[k] = A[k * n + k];
    wo[k] = mul(v0[k], v0[k]);
  }
}

// src/ftlm_thermo.cpp:124-146 (log-sum-exp over Ritz pairs with w > 0) and the energy ratio.
__global__ void eval_kernel(const double* __restrict__ lam, const double* __restrict__ w0, const int* __restrict__ nv,
                            int nc, int ld, const double* __restrict__ bts, int nbt, double* __restrict__ logq,
                            double* __restrict__ energy, int* __restrict__ bad) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= static_cast<int64_t>(nc) * nbt) return;
  const int ch = static_cast<int>(i / nbt), bi = static_cast<int>(i - static_cast<int64_t>(ch) * nbt);
  const int n = nv[ch];
  const double bT = bts[bi];
  const double* l = lam + static_cast<int64_t>(ch) * ld;
  const double* w = w0 + static_cast<int64_t>(ch) * ld;
  double out = -CUDART_INF, e = 0.0;
  if (n < 0 || n > ld) {  // invalid chain length (see jacobi_kernel): NaN outputs, reported
    if (bad) atomicOr(bad, 1);
    out = CUDART_NAN;
    e = CUDART_NAN;
  } else if (n == 1) {
    out = -bT * l[0];
    e = l[0];
  } else if (n > 1) {
    double mx = -CUDART_INF;
    for (int k = 0; k < n; ++k) {
      if (w[k] <= 0.0) continue;
      mx = fmax(mx, add(mul(-bT, l[k]), log(w[k])));
    }
    if (isfinite(mx)) {
      double s = 0.0, se = 0.0;
      for (int k = 0; k < n; ++k) {
        if (w[k] <= 0.0) continue;
        const double t = exp(sub(add(mul(-bT, l[k]), log(w[k])), mx));
        s = add(s, t);
        se = fma(l[k], t, se);
      }
      out = add(mx, log(s));
      e = se / s;
    }
  }
  logq[i] = out;
  energy[i] = e;
}

// src/ftlm_thermo.cpp:246-256: ln(dim) + max_l + log(sum_r e^{L_r - max_l} / count), chains
// with n <= 0 skipped.  Energy: e^{L_r}-weighted mean of the chain energies.
__global__ void sector_kernel(const double* __restrict__ logq, const double* __restrict__ eq,
                              const int* __restrict__ nv, int R, int nbt, double log_dim, double* __restrict__ lnz,
                              double* __restrict__ energy) {
  const int bi = blockIdx.x * blockDim.x + threadIdx.x;
  if (bi >= nbt) return;
  double mx = -CUDART_INF;
  int cnt = 0;
  bool first = true;
  for (int r = 0; r < R; ++r) {
    if (nv[r] <= 0) continue;
    const double x = logq[r * nbt + bi];
    mx = first ? x : fmax(mx, x);
    first = false;
    ++cnt;
  }
  if (cnt == 0) {
    lnz[bi] = -CUDART_INF;
    energy[bi] = 0.0;
    return;
  }
  double s = 0.0, se = 0.0;
  for (int r = 0; r < R; ++r) {
    if (nv[r] <= 0) continue;
    const double t = exp(sub(logq[r * nbt + bi], mx));
    s = add(s, t);
    se = fma(t, eq[r * nbt + bi], se);
  }
  lnz[bi] = add(log_dim, add(mx, log(s / static_cast<double>(cnt))));
  energy[bi] = se / s;
}

__global__ void gc_kernel(const double* __restrict__ lnz_s, const double* __restrict__ e_s,
                          const int* __restrict__ N_s, int n_sec, const double* __restrict__ bts, int n_bt,
                          const double* __restrict__ mus, int n_mu, int n_sites, double* __restrict__ lnz_gc,
                          double* __restrict__ n_avg, double* __restrict__ e_avg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_bt * n_mu) return;
  const int b = i / n_mu, m = i - b * n_mu;
  const double bT = bts[b], mu = mus[m];
  const double bm = mul(bT, mu);
  double mx = -CUDART_INF;
  for (int s = 0; s < n_sec; ++s) {
    const double lz = lnz_s[static_cast<int64_t>(s) * n_bt + b];
    if (!isfinite(lz)) continue;
    mx = fmax(mx, add(lz, mul(bm, static_cast<double>(N_s[s]))));
  }
  if (!isfinite(mx)) {
    lnz_gc[i] = -CUDART_INF;
    n_avg[i] = 0.0;
    e_avg[i] = 0.0;
    return;
  }
  double sw = 0.0, snw = 0.0, sew = 0.0;
  for (int s = 0; s < n_sec; ++s) {
    const double lz = lnz_s[static_cast<int64_t>(s) * n_bt + b];
    if (!isfinite(lz)) continue;
    const double w = exp(sub(add(lz, mul(bm, static_cast<double>(N_s[s]))), mx));
    sw = add(sw, w);
    snw = add(snw, mul(static_cast<double>(N_s[s]), w));
    sew = fma(e_s[static_cast<int64_t>(s) * n_bt + b], w, sew);
  }
  lnz_gc[i] = add(mx, log(sw));
  n_avg[i] = (sw > 0.0) ? (snw / sw) / static_cast<double>(n_sites) : 0.0;
  e_avg[i] = (sw > 0.0) ? sew / sw : 0.0;
}

// Number of eigenvalues of the tridiagonal (a, b) strictly below x (Sturm sequence).
__device__ int sturm_count(const double* a, const double* b, int n, double x) {
  int cnt = 0;
  double d = 1.0;
  for (int i = 0; i < n; ++i) {
    const double bb = (i > 0) ? b[i - 1] * b[i - 1] : 0.0;
    d = (a[i] - x) - ((i > 0) ? bb / d : 0.0);
    if (d == 0.0) d = -DBL_MIN;  // pivot shift: treat an exact zero as a tiny negative
    if (d < 0.0) ++cnt;
  }
  return cnt;
}

__global__ void ritz_kernel(const double* __restrict__ a, const double* __restrict__ b, int n, int k,
                            double* __restrict__ ritz) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= k || j >= n) return;
  double lo = DBL_MAX, hi = -DBL_MAX;
  for (int i = 0; i < n; ++i) {
    const double r = ((i > 0) ? fabs(b[i - 1]) : 0.0) + ((i + 1 < n) ? fabs(b[i]) : 0.0);
    lo = fmin(lo, a[i] - r);
    hi = fmax(hi, a[i] + r);
  }
  const double span = hi - lo;
  lo -= 1e-12 * span + DBL_MIN;
  hi += 1e-12 * span + DBL_MIN;
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    if (sturm_count(a, b, n, mid) > j)
      hi = mid;
    else
      lo = mid;
  }
  ritz[j] = 0.5 * (lo + hi);
}

}  // namespace

cudaError_t quad_jacobi(const double* alpha, const double* beta, const int* n, int nc, int ld, int max_rot,
                        double tol, double* lam, double* w0, cudaStream_t st, int* bad) {
  if (nc <= 0) return cudaSuccess;
  const size_t sm = (static_cast<size_t>(ld) * ld + ld) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(sm));
  if (e != cudaSuccess) return e;
  jacobi_kernel<<<nc, kJacThreads, sm, st>>>(alpha, beta, n, ld, max_rot, tol, lam, w0, bad);
  return cudaGetLastError();
}

cudaError_t quad_eval(const double* lam, const double* w0, const int* n, int nc, int ld, const double* bts, int nbt,
                      double* logq, double* energy, cudaStream_t st, int* bad) {
  const int64_t tot = static_cast<int64_t>(nc) * nbt;
  if (tot <= 0) return cudaSuccess;
  if ((tot + 127) / 128 > 0x7fffffffLL) return cudaErrorInvalidValue;
  eval_kernel<<<static_cast<unsigned>((tot + 127) / 128), 128, 0, st>>>(lam, w0, n, nc, ld, bts, nbt, logq, energy,
                                                                       bad);
  return cudaGetLastError();
}

cudaError_t quad_sector(const double* logq, const double* eq, const int* n, int R, int nbt, double log_dim,
                        double* lnz, double* energy, cudaStream_t st) {
  if (nbt <= 0) return cudaSuccess;
  sector_kernel<<<(nbt + 127) / 128, 128, 0, st>>>(logq, eq, n, R, nbt, log_dim, lnz, energy);
  return cudaGetLastError();
}

cudaError_t gc_reduce_dev(const double* lnz_s, const double* e_s, const int* N_s, int n_sec, const double* bts,
                          int n_bt, const double* mus, int n_mu, int n_sites, double* lnz_gc, double* n_avg,
                          double* e_avg, cudaStream_t st) {
  const int tot = n_bt * n_mu;
  if (tot <= 0) return cudaSuccess;
  gc_kernel<<<(tot + 127) / 128, 128, 0, st>>>(lnz_s, e_s, N_s, n_sec, bts, n_bt, mus, n_mu, n_sites, lnz_gc, n_avg,
                                                e_avg);
  return cudaGetLastError();
}

cudaError_t ritz_bisect(const double* alpha, const double* beta, int n, int k, double* ritz, cudaStream_t st) {
  if (k <= 0 || n <= 0) return cudaSuccess;
  ritz_kernel<<<(k + 63) / 64, 64, 0, st>>>(alpha, beta, n, k, ritz);
  return cudaGetLastError();
}

}  // namespace ftlm_b200
