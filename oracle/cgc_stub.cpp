// Test infrastructure (oracle): src/splat/gaussian_cloud.cpp dispatches to the
// compressed CGC format, whose implementation needs liblzma and is not built
// here. These definitions only satisfy the link; the .ply tests never reach
// them.
#include "splat/cgc.hpp"

#include <stdexcept>

namespace splat {

CgcStats save_cgc(const GaussianCloud &, const std::filesystem::path &, const CgcOptions &) {
  throw std::runtime_error("CGC is not built into the oracle");
}

GaussianCloud load_cgc(const std::filesystem::path &) { throw std::runtime_error("CGC is not built into the oracle"); }

} // namespace splat
