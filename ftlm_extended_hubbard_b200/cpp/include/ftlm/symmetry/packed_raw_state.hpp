// Drop-in for the reference header include/ftlm/symmetry/packed_raw_state.hpp: up << 16 | dn.
#pragma once

#include <cstdint>

#include "ftlm/symmetry/raw_state.hpp"

namespace ftlm {
namespace symmetry {

inline constexpr std::uint32_t pack_raw_state(RawState s) noexcept {
  return (static_cast<std::uint32_t>(s.up) << 16) | static_cast<std::uint32_t>(s.dn);
}
inline constexpr RawState unpack_raw_state(std::uint32_t p) noexcept {
  return RawState{static_cast<std::uint16_t>(p >> 16), static_cast<std::uint16_t>(p & 0xFFFFu)};
}

}  // namespace symmetry
}  // namespace ftlm
