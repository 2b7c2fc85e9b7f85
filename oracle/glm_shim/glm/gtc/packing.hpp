// Test infrastructure (oracle): the two half-float packing functions of glm's
// gtc/packing.hpp that src/splat/gaussian_cloud.cpp names (pack_half_sh), as
// IEEE binary16 conversions rounded to nearest even through the compiler's
// _Float16. Only what that file needs to compile and link.
#pragma once

#include <cstdint>
#include <cstring>

namespace glm {

inline std::uint16_t packHalf1x16(float v) {
  const _Float16 h = static_cast<_Float16>(v);
  std::uint16_t bits;
  std::memcpy(&bits, &h, sizeof bits);
  return bits;
}

inline float unpackHalf1x16(std::uint16_t bits) {
  _Float16 h;
  std::memcpy(&h, &bits, sizeof h);
  return static_cast<float>(h);
}

} // namespace glm
