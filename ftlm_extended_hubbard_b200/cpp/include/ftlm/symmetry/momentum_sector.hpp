// Drop-in for the part of the reference header include/ftlm/symmetry/momentum_sector.hpp that the
// orbit k-block path uses: the momentum label and the Bloch phase (momentum_sector.hpp:20-63).
// The orbit map / KBasis machinery of that header is not provided.
#pragma once

#include <cmath>
#include <complex>

namespace ftlm {
namespace symmetry {

struct MomentumSector {
  int kx = 0;
  int ky = 0;
  int lx = 4;
  int ly = 4;
  constexpr int flat_index() const noexcept { return ky * lx + kx; }
};

/// exp(-i 2 pi (kx dx / lx + ky dy / ly)) for a translation by (dx, dy).
inline std::complex<double> translation_bloch_phase(MomentumSector K, int dx, int dy) {
  const double pi = std::acos(-1.0);
  const double theta = -2.0 * pi *
                       (static_cast<double>(K.kx * dx) / static_cast<double>(K.lx) +
                        static_cast<double>(K.ky * dy) / static_cast<double>(K.ly));
  return {std::cos(theta), std::sin(theta)};
}

}  // namespace symmetry
}  // namespace ftlm
