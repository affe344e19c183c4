// Drop-in for the reference header include/ftlm/lanczos.hpp.  The recurrence runs on the GPU
// with device-resident vectors; the caller's operator keeps its host-pointer signature and is
// called once per step on host copies.
#pragma once

#include <complex>
#include <cstddef>
#include <functional>
#include <utility>
#include <vector>

namespace ftlm {

/// Kept for signature compatibility: the three Lanczos vectors live on the GPU, so these host
/// buffers are only sized (ensure) and never used as vectors.
struct LanczosComplexWorkspace {
  std::vector<std::complex<double>> q{};
  std::vector<std::complex<double>> q_prev{};
  std::vector<std::complex<double>> w{};

  void ensure(int dim) {
    (void)dim;
  }
  std::size_t bytes_capacity() const {
    return (q.capacity() + q_prev.capacity() + w.capacity()) * sizeof(std::complex<double>);
  }
  void shrink_to_fit() {
    q.shrink_to_fit();
    q_prev.shrink_to_fit();
    w.shrink_to_fit();
  }
};

struct LanczosExtrema {
  double min_eval = 0.0;
  double max_eval = 0.0;
  int steps_used = 0;
};

/// Smallest / largest eigenvalue estimate: Lanczos tridiagonal, then the reference's
/// 120-rotation Jacobi (tol 1e-15) on it.
LanczosExtrema lanczos_extrema(int dim,
                               const std::function<void(const std::complex<double>* v, std::complex<double>* Hv)>& apply_h,
                               int max_steps, unsigned seed = 1);

/// Hermitian Lanczos without reorthogonalisation from the std::mt19937(seed) complex Gaussian
/// start vector.  alpha gets the steps used; beta keeps one entry per completed step (the last
/// one included) and one fewer after a breakdown (||w||^2 < 1e-24).  Returns steps used.
int lanczos_tridiagonal(int dim,
                        const std::function<void(const std::complex<double>* v, std::complex<double>* Hv)>& apply_h,
                        int max_steps, unsigned seed, std::vector<double>* alpha, std::vector<double>* beta,
                        LanczosComplexWorkspace* ws = nullptr);

/// Extrema of the symmetric tridiagonal (alpha, beta) of size steps.
std::pair<double, double> tridiagonal_extrema(const std::vector<double>& alpha, const std::vector<double>& beta,
                                              int steps);

}  // namespace ftlm
