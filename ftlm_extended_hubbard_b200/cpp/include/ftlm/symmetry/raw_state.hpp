// Drop-in for the reference header include/ftlm/symmetry/raw_state.hpp: a (up, down) occupation
// pair of at most 16 sites.
#pragma once

#include <cstdint>

namespace ftlm {
namespace symmetry {

struct RawState {
  std::uint16_t up = 0;
  std::uint16_t dn = 0;
};

inline bool operator==(RawState a, RawState b) { return a.up == b.up && a.dn == b.dn; }
inline bool operator!=(RawState a, RawState b) { return !(a == b); }

}  // namespace symmetry
}  // namespace ftlm
