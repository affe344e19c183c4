// Drop-in for the reference header include/ftlm/ftlm_thermo.hpp.
#pragma once

#include <complex>
#include <functional>
#include <vector>

#include "ftlm/lanczos.hpp"

namespace ftlm {

/// Kept for signature compatibility (the quadrature runs on the GPU, not in these buffers).
struct FtlmTridiagonalQuadratureScratch {
  std::vector<double> T_flat{};
  std::vector<double> V_flat{};
  void shrink_to_fit() {
    T_flat.shrink_to_fit();
    V_flat.shrink_to_fit();
  }
};

struct FtlmParams {
  int n_random = 16;
  int lanczos_steps = 96;
  unsigned seed = 1;
  LanczosComplexWorkspace* lanczos_ws = nullptr;
  FtlmTridiagonalQuadratureScratch* quad_scratch = nullptr;
};

/// ln Tr e^{-beta H} by FTLM for real-symmetric H given as a real operator (applied to the real
/// and imaginary parts of each complex Lanczos vector): R = n_random chains of lanczos_steps steps,
/// seeds seed + r*100003.  dim <= 0 gives -inf; dim == 1 gives -beta * H_00.
double ftlm_log_partition_real(int dim, const std::function<void(const double* x, double* y)>& apply_real,
                               double beta, const FtlmParams& par);

/// Same for a complex Hermitian operator.
double ftlm_log_partition_complex(
    int dim, const std::function<void(const std::complex<double>* x, std::complex<double>* y)>& apply_h, double beta,
    const FtlmParams& par);

}  // namespace ftlm
