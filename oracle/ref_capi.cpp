// ORACLE (test infrastructure only; never linked into the product).
//
// A plain C interface over the reference trainer's own FP64 CPU twin,
// src/train/reference.cpp (reference_render :238, reference_contributions :242,
// reference_loss :276, reference_gradients :343), which oracle/Makefile
// compiles unmodified from the reference's sources into oracle/_ref/. Python
// tests load the result with ctypes. Arrays are the reference's GaussianCloud
// layout (src/splat/gaussian_cloud.hpp:138-151): positions 3/Gaussian,
// log-scales 3, quaternions (w,x,y,z) 4, opacity logits 1, SH [k][rgb].
// The camera is the reference's Camera (src/render/camera.hpp:84-89): a
// column-major world->camera matrix, the camera centre, fx, fy, cx, cy, size.
#include "splat/cgc.hpp"
#include "splat/lzma.hpp"
#include "train/densify.hpp"
#include "train/reference.hpp"
#include "train/schedule.hpp"

#include <cstdint>
#include <cstring>
#include <exception>
#include <algorithm>
#include <array>
#include <numeric>
#include <random>
#include <vector>

using namespace splat;

namespace {

GaussianCloud make_cloud(int n, int degree, const float *positions, const float *scales, const float *rotations,
                         const float *opacities, const float *sh) {
  GaussianCloud cloud;
  cloud.shDegree = degree;
  const std::size_t count = static_cast<std::size_t>(n);
  const std::size_t floats = count * 3 * static_cast<std::size_t>((degree + 1) * (degree + 1));
  cloud.positions.assign(positions, positions + count * 3);
  cloud.scales.assign(scales, scales + count * 3);
  cloud.rotations.assign(rotations, rotations + count * 4);
  cloud.opacities.assign(opacities, opacities + count);
  cloud.sh.assign(sh, sh + floats);
  return cloud;
}

Camera make_camera(const float *view16, const float *position3, const float *intrinsics4, int width, int height) {
  Camera camera;
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) camera.view[c][r] = view16[c * 4 + r];
  camera.position = glm::vec3(position3[0], position3[1], position3[2]);
  camera.fx = intrinsics4[0];
  camera.fy = intrinsics4[1];
  camera.cx = intrinsics4[2];
  camera.cy = intrinsics4[3];
  camera.width = width;
  camera.height = height;
  return camera;
}

// flags: 1 noCutoffs, 2 mipFilter2d. background 3 floats. filter3d may be null.
ReferenceOptions make_options(const float *background, float nearPlane, int flags, float opacityReg, float scaleReg,
                              const float *filter3d, int n) {
  ReferenceOptions options;
  for (int c = 0; c < 3; ++c) options.background[static_cast<std::size_t>(c)] = background[c];
  options.nearPlane = nearPlane;
  options.noCutoffs = (flags & 1) != 0;
  options.mipFilter2d = (flags & 2) != 0;
  options.opacityReg = opacityReg;
  options.scaleReg = scaleReg;
  if (filter3d != nullptr) options.filter3d.assign(filter3d, filter3d + n);
  return options;
}

} // namespace

extern "C" {

// rgb: 3 doubles per pixel, logT: 1 per pixel, stop: 1 uint64 per pixel.
int ref_render(int n, int degree, const float *positions, const float *scales, const float *rotations, const float *opacities,
               const float *sh, const float *view16, const float *position3, const float *intrinsics4, int width, int height,
               const float *background, float nearPlane, int flags, const float *filter3d, double *rgb, double *logT,
               std::uint64_t *stop) {
  try {
    const GaussianCloud cloud = make_cloud(n, degree, positions, scales, rotations, opacities, sh);
    const Camera camera = make_camera(view16, position3, intrinsics4, width, height);
    const ReferenceImage image =
        reference_render(cloud, camera, make_options(background, nearPlane, flags, 0.f, 0.f, filter3d, n));
    for (std::size_t i = 0; i < image.rgb.size(); ++i) {
      rgb[i * 3] = image.rgb[i].r;
      rgb[i * 3 + 1] = image.rgb[i].g;
      rgb[i * 3 + 2] = image.rgb[i].b;
      logT[i] = image.logTransmittance[i];
      stop[i] = image.stop[i];
    }
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

int ref_contributions(int n, int degree, const float *positions, const float *scales, const float *rotations,
                      const float *opacities, const float *sh, const float *view16, const float *position3,
                      const float *intrinsics4, int width, int height, const float *background, float nearPlane, int flags,
                      double *out) {
  try {
    const GaussianCloud cloud = make_cloud(n, degree, positions, scales, rotations, opacities, sh);
    const Camera camera = make_camera(view16, position3, intrinsics4, width, height);
    const std::vector<double> c =
        reference_contributions(cloud, camera, make_options(background, nearPlane, flags, 0.f, 0.f, nullptr, n));
    std::memcpy(out, c.data(), c.size() * sizeof(double));
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

// remove_largest / remove_least_contributing / remove_least_opaque
// (densify.cpp:95-113): kind 0, 1, 2. source gets, per survivor, the old index
// (count = survivors); contribution is read for kind 1.
int ref_prune(int kind, int n, int degree, const float *positions, const float *scales, const float *rotations,
              const float *opacities, const float *sh, const float *contribution, double share, std::int64_t *source,
              int *count) {
  try {
    const GaussianCloud cloud = make_cloud(n, degree, positions, scales, rotations, opacities, sh);
    DensifyResult r;
    if (kind == 0) r = remove_largest(cloud, share);
    else if (kind == 1) r = remove_least_contributing(cloud, std::vector<float>(contribution, contribution + n), share);
    else r = remove_least_opaque(cloud, share);
    *count = static_cast<int>(r.source.size());
    std::memcpy(source, r.source.data(), r.source.size() * sizeof(std::int64_t));
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

// save_ply (gaussian_cloud.cpp:330-365): the reference's writer.
int ref_save_ply(const char *path, int n, int degree, const float *positions, const float *scales, const float *rotations,
                 const float *opacities, const float *sh) {
  try {
    save_ply(make_cloud(n, degree, positions, scales, rotations, opacities, sh), path);
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

// load_ply (gaussian_cloud.cpp:236-328): the reference's reader. With null
// arrays only the count and degree; then again with arrays sized for them.
int ref_load_ply(const char *path, int *n, int *degree, float *positions, float *scales, float *rotations, float *opacities,
                 float *sh) {
  try {
    const GaussianCloud c = load_ply(path);
    *n = static_cast<int>(c.size());
    *degree = c.shDegree;
    if (positions != nullptr) {
      std::memcpy(positions, c.positions.data(), c.positions.size() * sizeof(float));
      std::memcpy(scales, c.scales.data(), c.scales.size() * sizeof(float));
      std::memcpy(rotations, c.rotations.data(), c.rotations.size() * sizeof(float));
      std::memcpy(opacities, c.opacities.data(), c.opacities.size() * sizeof(float));
      std::memcpy(sh, c.sh.data(), c.sh.size() * sizeof(float));
    }
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

// save_cgc (src/splat/cgc.cpp): the reference's CGC writer; preset 0
// balanced, 1 small. stats: bytes, then the three layer counts.
int ref_save_cgc(const char *path, int n, int degree, const float *positions, const float *scales, const float *rotations,
                 const float *opacities, const float *sh, int preset, int fast, std::uint64_t *stats) {
  try {
    CgcOptions options;
    options.preset = preset == 1 ? CgcPreset::Small : CgcPreset::Balanced;
    options.fast = fast != 0;
    const CgcStats s = save_cgc(make_cloud(n, degree, positions, scales, rotations, opacities, sh), path, options);
    if (stats != nullptr) {
      stats[0] = s.bytes;
      for (int l = 0; l < 3; ++l) stats[1 + l] = s.layerCounts[static_cast<std::size_t>(l)];
    }
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

// load_cgc (src/splat/cgc.cpp): the reference's CGC reader, as ref_load_ply.
int ref_load_cgc(const char *path, int *n, int *degree, float *positions, float *scales, float *rotations, float *opacities,
                 float *sh) {
  try {
    const GaussianCloud c = load_cgc(path);
    *n = static_cast<int>(c.size());
    *degree = c.shDegree;
    if (positions != nullptr) {
      std::memcpy(positions, c.positions.data(), c.positions.size() * sizeof(float));
      std::memcpy(scales, c.scales.data(), c.scales.size() * sizeof(float));
      std::memcpy(rotations, c.rotations.data(), c.rotations.size() * sizeof(float));
      std::memcpy(opacities, c.opacities.data(), c.opacities.size() * sizeof(float));
      std::memcpy(sh, c.sh.data(), c.sh.size() * sizeof(float));
    }
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

// cgc_detail::morton_code and canonicalize_axes (src/splat/cgc.hpp:53-58).
std::uint64_t ref_cgc_morton(std::uint32_t x, std::uint32_t y, std::uint32_t z) { return cgc_detail::morton_code(x, y, z); }
void ref_cgc_canonicalize(float *scales3, float *wxyz) {
  std::array<float, 3> s = {scales3[0], scales3[1], scales3[2]};
  std::array<float, 4> q = {wxyz[0], wxyz[1], wxyz[2], wxyz[3]};
  cgc_detail::canonicalize_axes(s, q);
  std::copy(s.begin(), s.end(), scales3);
  std::copy(q.begin(), q.end(), wxyz);
}

// lzma_compress / lzma_decompress (src/splat/lzma.hpp), through the shim.
// Returns the size written (or needed), or -1.
long long ref_lzma_compress(const std::uint8_t *data, std::size_t size, int level, int extreme, int lc, int lp, int pb,
                            std::uint8_t *out, std::size_t capacity) {
  try {
    const auto packed = lzma_compress(std::as_bytes(std::span(data, size)), level, extreme != 0, lc, lp, pb);
    if (out != nullptr) std::memcpy(out, packed.data(), std::min(capacity, packed.size()));
    return static_cast<long long>(packed.size());
  } catch (const std::exception &) {
    return -1;
  }
}

// reference_marked_pixels (reference.cpp:248-276): per Gaussian, the pixels it
// reaches whose mean error is at least `share` of the image's worst; target RGBA8.
int ref_marked_pixels(int n, int degree, const float *positions, const float *scales, const float *rotations,
                      const float *opacities, const float *sh, const float *view16, const float *position3,
                      const float *intrinsics4, int width, int height, const std::uint8_t *target, double share,
                      const float *background, float nearPlane, double *out) {
  try {
    const GaussianCloud cloud = make_cloud(n, degree, positions, scales, rotations, opacities, sh);
    const Camera camera = make_camera(view16, position3, intrinsics4, width, height);
    const std::vector<std::uint8_t> t(target, target + static_cast<std::size_t>(width) * height * 4);
    const std::vector<double> c =
        reference_marked_pixels(cloud, camera, t, share, make_options(background, nearPlane, 0, 0.f, 0.f, nullptr, n));
    std::memcpy(out, c.data(), c.size() * sizeof(double));
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

// rgb: 3 doubles per pixel; target RGBA8; adjoint out: 3 doubles per pixel; totals out: loss, l1, ssim.
int ref_loss(int width, int height, const double *rgb, const std::uint8_t *target, double lambda, double *adjoint,
             double *totals) {
  try {
    ReferenceImage image;
    image.width = width;
    image.height = height;
    const std::size_t pixels = static_cast<std::size_t>(width) * height;
    image.rgb.resize(pixels);
    for (std::size_t i = 0; i < pixels; ++i) image.rgb[i] = glm::dvec3(rgb[i * 3], rgb[i * 3 + 1], rgb[i * 3 + 2]);
    image.logTransmittance.assign(pixels, 0.0);
    image.stop.assign(pixels, 0);
    const std::vector<std::uint8_t> t(target, target + pixels * 4);
    const ReferenceLoss loss = reference_loss(image, t, lambda);
    for (std::size_t i = 0; i < pixels; ++i) {
      adjoint[i * 3] = loss.adjoint[i].r;
      adjoint[i * 3 + 1] = loss.adjoint[i].g;
      adjoint[i * 3 + 2] = loss.adjoint[i].b;
    }
    totals[0] = loss.loss;
    totals[1] = loss.l1;
    totals[2] = loss.ssim;
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

// adjoint: 3 doubles per pixel. Outputs are the reference's ParameterGradients arrays.
int ref_gradients(int n, int degree, const float *positions, const float *scales, const float *rotations, const float *opacities,
                  const float *sh, const float *view16, const float *position3, const float *intrinsics4, int width, int height,
                  const double *adjoint, const float *background, float nearPlane, int flags, float opacityReg, float scaleReg,
                  const float *filter3d, double *gPositions, double *gScales, double *gRotations, double *gOpacities,
                  double *gSh, double *absoluteCentre) {
  try {
    const GaussianCloud cloud = make_cloud(n, degree, positions, scales, rotations, opacities, sh);
    const Camera camera = make_camera(view16, position3, intrinsics4, width, height);
    const std::size_t pixels = static_cast<std::size_t>(width) * height;
    std::vector<glm::dvec3> a(pixels);
    for (std::size_t i = 0; i < pixels; ++i) a[i] = glm::dvec3(adjoint[i * 3], adjoint[i * 3 + 1], adjoint[i * 3 + 2]);
    const ParameterGradients g = reference_gradients(
        cloud, camera, a, make_options(background, nearPlane, flags, opacityReg, scaleReg, filter3d, n));
    std::memcpy(gPositions, g.positions.data(), g.positions.size() * sizeof(double));
    std::memcpy(gScales, g.scales.data(), g.scales.size() * sizeof(double));
    std::memcpy(gRotations, g.rotations.data(), g.rotations.size() * sizeof(double));
    std::memcpy(gOpacities, g.opacities.data(), g.opacities.size() * sizeof(double));
    std::memcpy(gSh, g.sh.data(), g.sh.size() * sizeof(double));
    std::memcpy(absoluteCentre, g.absoluteCentre.data(), g.absoluteCentre.size() * sizeof(double));
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

// A std::mt19937 that lives across ref_densify calls, as the reference's
// session keeps one (train.hpp:254).
void *ref_rng_create(std::uint32_t seed) { return new std::mt19937(seed); }
void ref_rng_destroy(void *rng) { delete static_cast<std::mt19937 *>(rng); }
// The session's pick of a view to score (train.cpp:690-692).
std::uint64_t ref_rng_pick(void *rng, std::uint64_t count) {
  return std::uniform_int_distribution<std::size_t>(0, count - 1)(*static_cast<std::mt19937 *>(rng));
}

// DensifyOptions (densify.hpp:23-50), in the field order of the product's
// splat_densify_options so that one ctypes structure serves both.
struct RefDensifyOptions {
  float gradientThreshold, denseScale, pruneOpacity;
  std::int32_t pruneLarge;
  float maxScreenRadius, maxWorldScale;
  std::uint64_t maxGaussians;
  float splitThreshold;
  std::int32_t scoredViews;
  float minMarkedPixels;
  double transparentShare;
  std::uint64_t exploreSplits, exploreSeeds;
  std::int32_t edgeSplit;
};

// densify_cloud (densify.cpp:115-326) on the cloud and the trainer's raw
// statistics (8 floats per Gaussian, trainer.cpp:686-708). The new cloud goes
// to the out* arrays (room for 2n + exploreSeeds Gaussians), the source
// table to source, counts = {count, cloned, split, seeded, pruned, heldBack}.
// Returns 0, or 1 if the reference threw.
int ref_densify(int n, int degree, const float *positions, const float *scales, const float *rotations, const float *opacities,
                const float *sh, const float *raw, const RefDensifyOptions *o, void *rng, float *outPositions,
                float *outScales, float *outRotations, float *outOpacities, float *outSh, std::int64_t *source,
                std::uint64_t *counts) {
  try {
    const GaussianCloud cloud = make_cloud(n, degree, positions, scales, rotations, opacities, sh);
    DensifyStats stats;
    std::vector<float> *columns[8] = {&stats.gradientSum, &stats.visits, &stats.maxRadius, &stats.contribution,
                                      &stats.absoluteGradientSum, &stats.markedPixels, &stats.markedLoss, &stats.edgeScore};
    for (int c = 0; c < 8; ++c) {
      columns[c]->resize(static_cast<std::size_t>(n));
      for (int i = 0; i < n; ++i) (*columns[c])[static_cast<std::size_t>(i)] = raw[i * 8 + c];
    }
    DensifyOptions options;
    options.gradientThreshold = o->gradientThreshold;
    options.denseScale = o->denseScale;
    options.pruneOpacity = o->pruneOpacity;
    options.pruneLarge = o->pruneLarge != 0;
    options.maxScreenRadius = o->maxScreenRadius;
    options.maxWorldScale = o->maxWorldScale;
    options.maxGaussians = o->maxGaussians;
    options.splitThreshold = o->splitThreshold;
    options.scoredViews = o->scoredViews;
    options.minMarkedPixels = o->minMarkedPixels;
    options.transparentShare = o->transparentShare;
    options.exploreSplits = o->exploreSplits;
    options.exploreSeeds = o->exploreSeeds;
    options.edgeSplit = o->edgeSplit != 0;
    const DensifyResult r = densify_cloud(cloud, stats, options, *static_cast<std::mt19937 *>(rng));
    const GaussianCloud &c = r.cloud;
    std::memcpy(outPositions, c.positions.data(), c.positions.size() * sizeof(float));
    std::memcpy(outScales, c.scales.data(), c.scales.size() * sizeof(float));
    std::memcpy(outRotations, c.rotations.data(), c.rotations.size() * sizeof(float));
    std::memcpy(outOpacities, c.opacities.data(), c.opacities.size() * sizeof(float));
    std::memcpy(outSh, c.sh.data(), c.sh.size() * sizeof(float));
    std::memcpy(source, r.source.data(), r.source.size() * sizeof(std::int64_t));
    const std::uint64_t out[6] = {c.size(), r.cloned, r.split, r.seeded, r.pruned, r.heldBack};
    std::memcpy(counts, out, sizeof(out));
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

// RelocateOptions (densify.hpp:87-91) in the product's field order.
struct RefRelocateOptions {
  float minOpacity;
  double growth;
  std::uint64_t maxGaussians;
};

// relocate_cloud (densify.cpp:328-420): the out* arrays have room for
// n + growth n + 1 Gaussians; counts as ref_densify.
int ref_relocate(int n, int degree, const float *positions, const float *scales, const float *rotations, const float *opacities,
                 const float *sh, const RefRelocateOptions *o, void *rng, float *outPositions, float *outScales,
                 float *outRotations, float *outOpacities, float *outSh, std::int64_t *source, std::uint64_t *counts) {
  try {
    const GaussianCloud cloud = make_cloud(n, degree, positions, scales, rotations, opacities, sh);
    RelocateOptions options;
    options.minOpacity = o->minOpacity;
    options.growth = o->growth;
    options.maxGaussians = o->maxGaussians;
    const DensifyResult r = relocate_cloud(cloud, options, *static_cast<std::mt19937 *>(rng));
    const GaussianCloud &c = r.cloud;
    std::memcpy(outPositions, c.positions.data(), c.positions.size() * sizeof(float));
    std::memcpy(outScales, c.scales.data(), c.scales.size() * sizeof(float));
    std::memcpy(outRotations, c.rotations.data(), c.rotations.size() * sizeof(float));
    std::memcpy(outOpacities, c.opacities.data(), c.opacities.size() * sizeof(float));
    std::memcpy(outSh, c.sh.data(), c.sh.size() * sizeof(float));
    std::memcpy(source, r.source.data(), r.source.size() * sizeof(std::int64_t));
    const std::uint64_t out[6] = {c.size(), r.cloned, r.split, r.seeded, r.pruned, r.heldBack};
    std::memcpy(counts, out, sizeof(out));
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

// frequency_energy and resolution_switches (schedule.cpp:41-82): the
// reference's own, for the schedule's parity.
int ref_frequency_energy(const std::uint8_t *rgba, int width, int height, const int *factors, int count, double *out) {
  try {
    const std::vector<std::uint8_t> image(rgba, rgba + static_cast<std::size_t>(width) * height * 4);
    const std::vector<double> e = frequency_energy(image, width, height, std::vector<int>(factors, factors + count));
    std::copy(e.begin(), e.end(), out);
    return 0;
  } catch (const std::exception &) {
    return 1;
  }
}

void ref_resolution_switches(double full, double half, double quarter, double *out) {
  const std::array<double, 2> s = resolution_switches(full, half, quarter);
  out[0] = s[0];
  out[1] = s[1];
}

// GrowthBudget (schedule.hpp:26-41) after the observations: limit and final count.
void ref_growth_limit(double initial, double factor, const std::uint64_t *observed, int observations, double imageFactor,
                      double progress, std::uint64_t *limit, double *finalCount) {
  GrowthBudget budget(static_cast<std::size_t>(initial), factor);
  for (int k = 0; k < observations; ++k) budget.observe(observed[k]);
  *limit = budget.limit(imageFactor, progress);
  *finalCount = budget.final_count();
}

// The order TrainSession draws its views in (train.cpp:560-565, 580-586),
// restated over the same generator and std::shuffle: for each of `steps`
// iterations the view it trains on.
void ref_view_order(std::uint32_t seed, int views, int steps, int *out) {
  std::mt19937 rng(seed);
  std::vector<std::size_t> order;
  const auto refill = [&] {
    if (!order.empty()) return;
    order.resize(static_cast<std::size_t>(views));
    std::iota(order.begin(), order.end(), std::size_t{0});
    std::shuffle(order.begin(), order.end(), rng);
  };
  for (int i = 0; i < steps; ++i) {
    refill();
    out[i] = static_cast<int>(order.back());
    order.pop_back();
    refill();
  }
}

} // extern "C"
