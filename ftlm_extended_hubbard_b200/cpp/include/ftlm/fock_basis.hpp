// Drop-in for the reference header include/ftlm/fock_basis.hpp.  Same public interface; the
// strings are held per spin species (C(n,n_up) + C(n,n_dn) entries instead of dim pairs) and
// index_of ranks them arithmetically instead of probing a hash map.
#pragma once

#include <cstdint>

struct ftlm_sector;

namespace ftlm {

/// Fixed (N_up, N_down) sector: index = rank_up * C(n, N_down) + rank_down, strings of each
/// species in lexicographic order of their site lists.  Throws std::invalid_argument for
/// n_sites outside [1, 32] or particle numbers outside [0, n_sites].
class FockBasis {
 public:
  FockBasis(int n_sites, int n_up, int n_down);
  ~FockBasis();
  FockBasis(const FockBasis&) = delete;
  FockBasis& operator=(const FockBasis&) = delete;

  int n_sites() const { return n_sites_; }
  int n_up() const { return n_up_; }
  int n_down() const { return n_down_; }
  int dim() const { return dim_; }

  /// Throws std::out_of_range for idx outside [0, dim).
  uint64_t up_mask(int idx) const;
  uint64_t down_mask(int idx) const;

  /// Index of (up, down), or -1 if outside this sector.
  int index_of(uint64_t up, uint64_t down) const;

  /// Native host handle (tables of this basis), for the GPU entry points.
  const ftlm_sector* native() const { return h_; }

 private:
  int n_sites_;
  int n_up_;
  int n_down_;
  int dim_ = 0;
  ftlm_sector* h_ = nullptr;
};

}  // namespace ftlm
