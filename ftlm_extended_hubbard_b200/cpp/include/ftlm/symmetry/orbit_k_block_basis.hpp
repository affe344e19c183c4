// Drop-in for the reference header include/ftlm/symmetry/orbit_k_block_basis.hpp.  Same public
// interface; build() canonicalises the sector on the GPU (ftlm_gpu_orbit_create_ex) and
// apply_orbit_k_block runs the GPU H_K v on host buffers (copied in and out; device tables cached
// per (basis, hoppings, pairs, U, V, K)).
#pragma once

#include <complex>
#include <cstddef>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "ftlm/fock_basis.hpp"
#include "ftlm/hubbard_params.hpp"
#include "ftlm/lattice.hpp"
#include "ftlm/symmetry/momentum_sector.hpp"
#include "ftlm/symmetry/packed_raw_state.hpp"
#include "ftlm/symmetry/raw_state.hpp"

namespace ftlm {
namespace symmetry {

struct OrbitKRepEntry {
  RawState rep{};
  std::size_t orbit_index = 0;  // index of the orbit among the sector's orbits (ascending representative)
  std::uint16_t orbit_size = 0;
  std::uint16_t stabilizer_size = 0;
  std::complex<double> A_k{0.0, 0.0};
  double abs_A = 0.0;
};

/// Reduced basis of one momentum block: canonical orbit representatives (smallest packed image
/// under the translations) with |A_alpha(K)| > survive_tol, ascending packed order.
class OrbitKBlockBasis {
 public:
  MomentumSector K{};
  int lx = 0;
  int ly = 0;

  /// Throws std::invalid_argument for more than 16 sites or lx*ly != n_sites.
  bool build(const FockBasis& fb, MomentumSector K, double survive_tol = 1e-12);

  int dim() const noexcept { return static_cast<int>(entries_.size()); }
  const std::vector<OrbitKRepEntry>& entries() const noexcept { return entries_; }
  double survive_tol() const noexcept { return survive_tol_; }

  /// Row of the canonical representative `rep`, or -1.
  int reduced_index_of_rep(RawState rep) const;

  /// Reduced row, translation (first in dx-outer, dy-inner order) with T_R rep = s, and the
  /// fermionic sign of T_R on rep; false if the orbit of s is not in the block.
  bool map_raw_to_rep(RawState s, int* reduced_index, int* dx, int* dy, double* eta) const;

 private:
  std::vector<OrbitKRepEntry> entries_;
  std::unordered_map<std::uint32_t, std::size_t> rep_pack_to_row_;
  double survive_tol_ = 1e-12;
};

/// y = H_K x in the reduced basis (y overwritten), the reference's matrix-free orbit apply.
void apply_orbit_k_block(const HubbardParams& p, const FockBasis& fb, const OrbitKBlockBasis& basis,
                         const std::vector<SpinfulHopping>& hoppings, const std::vector<NearestPair>& nn_pairs,
                         const std::complex<double>* x, std::complex<double>* y);

}  // namespace symmetry
}  // namespace ftlm
