// Drop-in for the reference header include/ftlm/lattice.hpp.
#pragma once

#include <complex>
#include <vector>

#include "ftlm/hubbard_params.hpp"

namespace ftlm {

/// One directed kinetic term H += coeff c^dag_{to,spin} c_{from,spin} (spin 0 = up, 1 = down).
struct SpinfulHopping {
  int from = 0;
  int to = 0;
  int spin = 0;
  std::complex<double> coeff{0.0, 0.0};
};

/// Nearest-neighbour pair (i < j) of the V n_i n_j interaction.
struct NearestPair {
  int i = 0;
  int j = 0;
};

/// Periodic rectangle, sites numbered row-major (site = y * Lx + x).
struct RectLattice {
  int Lx = 1;
  int Ly = 1;

  int n_sites() const { return Lx * Ly; }
  int site_index(int x, int y) const { return y * Lx + x; }
  void coords(int site, int* x, int* y) const {
    *x = site % Lx;
    *y = site / Lx;
  }
};

/// Directed hoppings (both directions, both spins) and nn pairs; computed by the native library.
void build_hubbard_geometry(const HubbardParams& p, const RectLattice& lat, std::vector<SpinfulHopping>* hoppings,
                            std::vector<NearestPair>* nn_pairs);

}  // namespace ftlm
