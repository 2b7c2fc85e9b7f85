// ORACLE / TEST FIXTURES (test infrastructure only).
//
// The reference's tests use no stored golden files: every input comes from
// std::mt19937 seeds through the helpers of tests/reference_helpers.hpp
// (random_cloud :17-34, train_camera :37-45, smooth_target :48-61) and the
// adjoints of tests/test_train.cpp:86-90. These functions restate those
// helpers with the same standard-library distributions and call order, so the
// same seeds give the same clouds, targets and adjoints as the reference's
// own tests (libstdc++'s mt19937 and distributions are deterministic).
#include <cmath>
#include <cstdint>
#include <random>

extern "C" {

// random_cloud(count, degree, seed): positions x in +-1.4, y in +-1.1, z in
// [3, 6]; log-scales log(0.06 + 0.2 U); raw quaternions U(-1, 1); opacity
// logits +-1.5; DC so that the colour is U(0, 1); higher SH +-0.2.
void fixture_random_cloud(int count, int degree, uint32_t seed, float *positions, float *scales, float *rotations,
                          float *opacities, float *sh) {
  constexpr float kShC0 = 0.28209479177387814f;
  std::mt19937 rng(seed);
  std::uniform_real_distribution<float> u(-1.f, 1.f), unit(0.f, 1.f);
  const int coefficients = (degree + 1) * (degree + 1);
  for (int i = 0; i < count * 3 * coefficients; ++i) sh[i] = 0.f;
  for (int i = 0; i < count; ++i) {
    positions[i * 3] = u(rng) * 1.4f;
    positions[i * 3 + 1] = u(rng) * 1.1f;
    positions[i * 3 + 2] = 3.f + unit(rng) * 3.f;
    for (int a = 0; a < 3; ++a) scales[i * 3 + a] = std::log(0.06f + 0.2f * unit(rng));
    for (int a = 0; a < 4; ++a) rotations[i * 4 + a] = u(rng);
    opacities[i] = u(rng) * 1.5f;
    for (int c = 0; c < 3; ++c) sh[i * coefficients * 3 + c] = (unit(rng) - 0.5f) / kShC0;
    for (int k = 3; k < coefficients * 3; ++k) sh[i * coefficients * 3 + k] = u(rng) * 0.2f;
  }
}

// smooth_target(width, height, seed): RGBA8, a sinusoid plus noise.
void fixture_smooth_target(int width, int height, uint32_t seed, uint8_t *target) {
  std::mt19937 rng(seed);
  for (int y = 0; y < height; ++y) {
    for (int x = 0; x < width; ++x) {
      const size_t at = (static_cast<size_t>(y) * width + x) * 4;
      target[at] = static_cast<uint8_t>(127.f + 100.f * std::sin(0.2f * static_cast<float>(x)) + static_cast<float>(rng() % 16));
      target[at + 1] = static_cast<uint8_t>(127.f + 100.f * std::cos(0.15f * static_cast<float>(y)) + static_cast<float>(rng() % 16));
      target[at + 2] = static_cast<uint8_t>(60 + (x + y) % 120);
      target[at + 3] = 255;
    }
  }
}

// Standard-normal adjoint, 3 doubles per pixel, as test_train.cpp:86-90.
void fixture_normal_adjoint(uint32_t seed, int pixels, double *out) {
  std::mt19937 rng(seed);
  std::normal_distribution<double> n(0.0, 1.0);
  for (int i = 0; i < pixels; ++i) {
    const double a = n(rng), b = n(rng), c = n(rng);
    out[i * 3] = a;
    out[i * 3 + 1] = b;
    out[i * 3 + 2] = c;
  }
}

// Raw 32-bit outputs of std::mt19937(seed), as the sort test draws its keys
// (tests/test_radix_sort.cpp:19-27).
void fixture_mt19937(uint32_t seed, int count, uint32_t *out) {
  std::mt19937 rng(seed);
  for (int i = 0; i < count; ++i) out[i] = static_cast<uint32_t>(rng());
}

} // extern "C"
