// Drop-in for the reference header include/ftlm/hubbard_params.hpp (same names and fields, so
// code written against the reference compiles unchanged).
#pragma once

namespace ftlm {

/// Extended Hubbard model on an Lx x Ly periodic rectangle: hoppings t (nearest) and tp
/// (diagonal), on-site U, nearest-neighbour V, Peierls phases phi_x / phi_y on the wrap bonds.
struct HubbardParams {
  int Lx = 2;
  int Ly = 2;
  double t = 1.0;
  double tp = 0.0;
  double U = 0.0;
  double V = 0.0;
  double phi_x = 0.0;
  double phi_y = 0.0;
};

int nsites(const HubbardParams& p);

}  // namespace ftlm
