#include "tridiag.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <vector>

namespace ftlm_b200 {

std::string tridiag_eigvec(int n, const double* alpha, const double* beta, double* lam, double* Z) {
  if (n <= 0) return "";
  std::vector<double> d(alpha, alpha + n), e(static_cast<size_t>(n), 0.0);
  for (int i = 0; i + 1 < n; ++i) e[static_cast<size_t>(i)] = beta[i];
  std::fill(Z, Z + static_cast<size_t>(n) * n, 0.0);
  for (int i = 0; i < n; ++i) Z[static_cast<size_t>(i) * n + i] = 1.0;
  const double eps = std::numeric_limits<double>::epsilon();
  for (int l = 0; l < n; ++l) {
    for (int iter = 0;; ++iter) {
      int m = l;
      for (; m + 1 < n; ++m) {
        const double dd = std::fabs(d[static_cast<size_t>(m)]) + std::fabs(d[static_cast<size_t>(m) + 1]);
        if (std::fabs(e[static_cast<size_t>(m)]) <= eps * dd) break;
      }
      if (m == l) break;
      if (iter >= 64) return "tridiagonal QL did not converge";
      // shift from the leading 2x2 block at l, then chase the bulge from m-1 up to l
      double g = (d[static_cast<size_t>(l) + 1] - d[static_cast<size_t>(l)]) / (2.0 * e[static_cast<size_t>(l)]);
      double r = std::hypot(g, 1.0);
      g = d[static_cast<size_t>(m)] - d[static_cast<size_t>(l)] + e[static_cast<size_t>(l)] / (g + std::copysign(r, g));
      double s = 1.0, c = 1.0, p = 0.0;
      bool split = false;
      for (int i = m - 1; i >= l; --i) {
        const double f = s * e[static_cast<size_t>(i)];
        const double b = c * e[static_cast<size_t>(i)];
        r = std::hypot(f, g);
        e[static_cast<size_t>(i) + 1] = r;
        if (r == 0.0) {  // exact split: undo the partial shift and restart this eigenvalue
          d[static_cast<size_t>(i) + 1] -= p;
          e[static_cast<size_t>(m)] = 0.0;
          split = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[static_cast<size_t>(i) + 1] - p;
        r = (d[static_cast<size_t>(i)] - g) * s + 2.0 * c * b;
        p = s * r;
        d[static_cast<size_t>(i) + 1] = g + p;
        g = c * r - b;
        for (int k = 0; k < n; ++k) {
          double* zk = Z + static_cast<size_t>(k) * n;
          const double zf = zk[i + 1];
          zk[i + 1] = s * zk[i] + c * zf;
          zk[i] = c * zk[i] - s * zf;
        }
      }
      if (split) continue;
      d[static_cast<size_t>(l)] -= p;
      e[static_cast<size_t>(l)] = g;
      e[static_cast<size_t>(m)] = 0.0;
    }
  }
  std::vector<int> ord(static_cast<size_t>(n));
  std::iota(ord.begin(), ord.end(), 0);
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return d[static_cast<size_t>(a)] < d[static_cast<size_t>(b)]; });
  std::vector<double> Zs(static_cast<size_t>(n) * n);
  for (int j = 0; j < n; ++j) {
    lam[j] = d[static_cast<size_t>(ord[static_cast<size_t>(j)])];
    for (int k = 0; k < n; ++k)
      Zs[static_cast<size_t>(k) * n + j] = Z[static_cast<size_t>(k) * n + ord[static_cast<size_t>(j)]];
  }
  std::copy(Zs.begin(), Zs.end(), Z);
  return "";
}

std::string duhamel_weights(int n, const double* alpha, const double* beta, double bT, double* K, double* g,
                            double* lam_min) {
  *g = 0.0;
  if (n <= 0) return "";
  std::vector<double> lam(static_cast<size_t>(n)), Z(static_cast<size_t>(n) * n);
  const std::string err = tridiag_eigvec(n, alpha, beta, lam.data(), Z.data());
  if (!err.empty()) return err;
  const double shift = lam[0];
  if (lam_min) *lam_min = shift;
  std::vector<double> ew(static_cast<size_t>(n));
  double gs = 0.0;
  for (int j = 0; j < n; ++j) {
    ew[static_cast<size_t>(j)] = std::exp(-bT * (lam[static_cast<size_t>(j)] - shift));
    gs += Z[static_cast<size_t>(j)] * Z[static_cast<size_t>(j)] * ew[static_cast<size_t>(j)];
  }
  *g = gs;
  // P_jk = Z_0j Z_0k D_jk (lam ascending: j < k means lam_j <= lam_k)
  std::vector<double> P(static_cast<size_t>(n) * n);
  for (int j = 0; j < n; ++j)
    for (int k = j; k < n; ++k) {
      const double delta = lam[static_cast<size_t>(k)] - lam[static_cast<size_t>(j)];
      const double D = (j == k || delta == 0.0) ? bT * ew[static_cast<size_t>(j)]
                                                : ew[static_cast<size_t>(j)] * (-std::expm1(-bT * delta)) / delta;
      const double v = Z[static_cast<size_t>(j)] * Z[static_cast<size_t>(k)] * D;
      P[static_cast<size_t>(j) * n + k] = v;
      P[static_cast<size_t>(k) * n + j] = v;
    }
  // K = Z P Z^T
  std::vector<double> Y(static_cast<size_t>(n) * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const double zij = Z[static_cast<size_t>(i) * n + j];
      if (zij == 0.0) continue;
      const double* pj = P.data() + static_cast<size_t>(j) * n;
      double* yi = Y.data() + static_cast<size_t>(i) * n;
      for (int k = 0; k < n; ++k) yi[k] += zij * pj[k];
    }
  for (int i = 0; i < n; ++i)
    for (int l = i; l < n; ++l) {
      const double* yi = Y.data() + static_cast<size_t>(i) * n;
      const double* zl = Z.data() + static_cast<size_t>(l) * n;
      double acc = 0.0;
      for (int k = 0; k < n; ++k) acc += yi[k] * zl[k];
      K[static_cast<size_t>(i) * n + l] = acc;
      K[static_cast<size_t>(l) * n + i] = acc;
    }
  return "";
}

std::string sym_eigvals(int m, double* A, double* lam) {
  if (m <= 0) return "";
  auto a = [A, m](int i, int j) -> double& { return A[static_cast<size_t>(i) * m + j]; };
  double fro = 0.0;
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) fro += a(i, j) * a(i, j);
  const double stop = 1e-30 * fro;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < m; ++i)
      for (int j = i + 1; j < m; ++j) off += 2.0 * a(i, j) * a(i, j);
    if (off <= stop) break;
    if (sweep == 99) return "Jacobi eigenvalues did not converge";
    for (int p = 0; p < m; ++p)
      for (int q = p + 1; q < m; ++q) {
        const double apq = a(p, q);
        if (apq == 0.0) continue;
        // rotation zeroing a(p,q): t = sgn(theta) / (|theta| + sqrt(theta^2 + 1)), theta = (a_qq - a_pp) / (2 a_pq)
        const double theta = (a(q, q) - a(p, p)) / (2.0 * apq);
        const double t = std::copysign(1.0, theta) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c, tau = sn / (1.0 + c);
        a(p, p) -= t * apq;
        a(q, q) += t * apq;
        a(p, q) = a(q, p) = 0.0;
        for (int r = 0; r < m; ++r) {
          if (r == p || r == q) continue;
          const double arp = a(r, p), arq = a(r, q);
          const double np = arp - sn * (arq + tau * arp);
          const double nq = arq + sn * (arp - tau * arq);
          a(r, p) = a(p, r) = np;
          a(r, q) = a(q, r) = nq;
        }
      }
  }
  for (int i = 0; i < m; ++i) lam[i] = a(i, i);
  std::sort(lam, lam + m);
  return "";
}

}  // namespace ftlm_b200
