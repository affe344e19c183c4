// Drop-in for the reference header include/ftlm/hubbard_hamiltonian.hpp.
#pragma once

#include <complex>
#include <vector>

#include "ftlm/fock_basis.hpp"
#include "ftlm/hubbard_params.hpp"
#include "ftlm/lattice.hpp"

namespace ftlm {

/// y = H x in one (N_up, N_down) sector on host buffers of length basis.dim(); y is overwritten.
/// Runs on the GPU: x is copied in, y copied out; device tables are built once per
/// (basis, hoppings, pairs, U, V) and cached.
void apply_extended_hubbard(const HubbardParams& p, const FockBasis& basis,
                            const std::vector<SpinfulHopping>& hoppings, const std::vector<NearestPair>& nn_pairs,
                            const std::complex<double>* x, std::complex<double>* y);

}  // namespace ftlm
