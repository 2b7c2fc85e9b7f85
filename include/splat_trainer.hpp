// Header-only C++ face of the C ABI in splat_b200.h with the reference
// trainer's class shape (splat::Trainer, src/train/trainer.hpp:89-270 of the
// reference), so that code written against the reference's trainer can switch
// to this library by changing its include and its construction. Errors become
// the exceptions the reference throws: BudgetExceeded (trainer.hpp:46-49),
// std::runtime_error, std::logic_error (trainer.cpp:853).
//
// Types are this header's own plain structs; a caller with the reference's
// GaussianCloud and Camera converts with the two adapters at the end, which
// compile only where the reference's headers are included first.
#pragma once

#include <array>
#include <cstdint>
#include <cstring>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "splat_b200.h"

namespace splat_b200 {

class BudgetExceeded : public std::runtime_error {
public:
  using std::runtime_error::runtime_error;
};

inline void check(int status) {
  if (status == SPLAT_OK) return;
  const std::string message = splat_last_error();
  if (status == SPLAT_ERR_BUDGET) throw BudgetExceeded(message);
  if (status == SPLAT_ERR_STATE) throw std::logic_error(message);
  if (status == SPLAT_ERR_INVALID) throw std::invalid_argument(message);
  throw std::runtime_error(message);
}

struct Cloud {
  int shDegree = 0;
  std::vector<float> positions, scales, rotations, opacities, sh;
  [[nodiscard]] std::size_t size() const noexcept { return opacities.size(); }
  [[nodiscard]] splat_cloud view() const {
    return splat_cloud{static_cast<int32_t>(size()), shDegree, positions.data(), scales.data(), rotations.data(),
                       opacities.data(), sh.data()};
  }
};

inline splat_trainer_options default_options() {
  splat_trainer_options o;
  splat_trainer_options_default(&o);
  return o;
}

inline splat_learning_rates default_rates() {
  splat_learning_rates r;
  splat_learning_rates_default(&r);
  return r;
}

// The generator densification draws from (std::mt19937 inside), kept by
// the caller across rounds as the reference's session keeps densifyRng_.
class Rng {
public:
  explicit Rng(std::uint32_t seed) { check(splat_rng_create(seed, &handle_)); }
  ~Rng() { splat_rng_destroy(handle_); }
  Rng(const Rng &) = delete;
  Rng &operator=(const Rng &) = delete;
  // std::uniform_int_distribution<std::size_t>(0, count - 1)(rng).
  std::size_t pick(std::size_t count) {
    std::uint64_t out = 0;
    check(splat_rng_pick(handle_, count, &out));
    return static_cast<std::size_t>(out);
  }
  [[nodiscard]] splat_rng *handle() const noexcept { return handle_; }

private:
  splat_rng *handle_ = nullptr;
};

inline splat_densify_options default_densify_options() {
  splat_densify_options o;
  splat_densify_options_default(&o);
  return o;
}

inline splat_relocate_options default_relocate_options() {
  splat_relocate_options o;
  splat_relocate_options_default(&o);
  return o;
}

// DensifyResult (densify.hpp:52-62) without the cloud, which stays on the GPU
// (Trainer::cloud() downloads it).
struct DensifyResult {
  std::vector<std::int64_t> source;
  std::size_t cloned = 0, split = 0, seeded = 0, pruned = 0, heldBack = 0;
};

class Trainer {
public:
  explicit Trainer(const Cloud &initial, const splat_trainer_options &options = default_options())
      : shDegree_(initial.shDegree), count_(initial.size()) {
    const splat_cloud c = initial.view();
    check(splat_trainer_create(&c, &options, &handle_));
  }
  ~Trainer() { splat_trainer_destroy(handle_); }
  Trainer(const Trainer &) = delete;
  Trainer &operator=(const Trainer &) = delete;

  [[nodiscard]] std::vector<float> render(const splat_camera &camera) {
    std::vector<float> out(static_cast<std::size_t>(camera.width) * camera.height * 4);
    check(splat_trainer_render(handle_, &camera, out.data()));
    return out;
  }
  splat_step_stats compute_gradients(const splat_camera &camera, std::span<const std::uint8_t> target) {
    splat_step_stats s{};
    check(splat_trainer_compute_gradients(handle_, &camera, target.data(), target.size(), &s));
    return s;
  }
  splat_step_stats collect_statistics(const splat_camera &camera, std::span<const std::uint8_t> target) {
    splat_step_stats s{};
    check(splat_trainer_collect_statistics(handle_, &camera, target.data(), target.size(), &s));
    return s;
  }
  void apply_gradients(const splat_learning_rates &rates) { check(splat_trainer_apply_gradients(handle_, &rates)); }
  splat_step_stats step(const splat_camera &camera, std::span<const std::uint8_t> target, const splat_learning_rates &rates,
                        std::span<const std::uint8_t> nextTarget = {}) {
    splat_step_stats s{};
    check(splat_trainer_step(handle_, &camera, target.data(), target.size(), &rates,
                             nextTarget.empty() ? nullptr : nextTarget.data(), nextTarget.size(), &s));
    return s;
  }
  void prefetch_target(std::span<const std::uint8_t> target) {
    check(splat_trainer_prefetch_target(handle_, target.data(), target.size()));
  }

  struct Gradients {
    std::vector<float> positions, scales, rotations, opacities, sh;
  };
  [[nodiscard]] Gradients gradients() const {
    Gradients g;
    const std::size_t n = count_, f = 3u * static_cast<std::size_t>((shDegree_ + 1) * (shDegree_ + 1));
    g.positions.resize(n * 3);
    g.scales.resize(n * 3);
    g.rotations.resize(n * 4);
    g.opacities.resize(n);
    g.sh.resize(n * f);
    check(splat_trainer_get_gradients(handle_, g.positions.data(), g.scales.data(), g.rotations.data(), g.opacities.data(),
                                      g.sh.data()));
    return g;
  }
  [[nodiscard]] Cloud cloud() const {
    Cloud c;
    c.shDegree = shDegree_;
    const std::size_t n = count_, f = 3u * static_cast<std::size_t>((shDegree_ + 1) * (shDegree_ + 1));
    c.positions.resize(n * 3);
    c.scales.resize(n * 3);
    c.rotations.resize(n * 4);
    c.opacities.resize(n);
    c.sh.resize(n * f);
    check(splat_trainer_get_cloud(handle_, c.positions.data(), c.scales.data(), c.rotations.data(), c.opacities.data(),
                                  c.sh.data()));
    return c;
  }
  void set_active_sh_degree(int degree) { check(splat_trainer_set_active_sh_degree(handle_, degree)); }
  void reset_densify_stats() { check(splat_trainer_reset_densify_stats(handle_)); }
  void reset_opacity(float maximum) { check(splat_trainer_reset_opacity(handle_, maximum)); }
  // Trainer::apply_changes: source[i] is the old index whose optimiser state
  // Gaussian i keeps, or -1.
  void apply_changes(const Cloud &next, std::span<const std::int32_t> source) {
    const splat_cloud c = next.view();
    check(splat_trainer_apply_changes(handle_, &c, source.data()));
    count_ = next.size();
  }
  // Trainer::score_view: the FastGS scoring pass.
  splat_step_stats score_view(const splat_camera &camera, std::span<const std::uint8_t> target, float errorShare,
                              float pixelWeight = 1.f) {
    splat_step_stats s{};
    check(splat_trainer_score_view(handle_, &camera, target.data(), target.size(), errorShare, pixelWeight, &s));
    return s;
  }
  // Trainer::densify and Trainer::relocate, on the GPU.
  DensifyResult densify(const splat_densify_options &options, Rng &rng) {
    return edit([&](splat_densify_result *r, int64_t *source, uint64_t capacity) {
      return splat_trainer_densify(handle_, &options, rng.handle(), r, source, capacity);
    }, 2 * count_ + options.explore_seeds);
  }
  DensifyResult relocate(const splat_relocate_options &options, Rng &rng) {
    const double growth = options.growth > 0.0 ? options.growth * static_cast<double>(count_) : 0.0;
    return edit([&](splat_densify_result *r, int64_t *source, uint64_t capacity) {
      return splat_trainer_relocate(handle_, &options, rng.handle(), r, source, capacity);
    }, count_ + static_cast<std::size_t>(growth) + 1);
  }
  // Trainer::remove_largest_gaussians and its siblings: how many went.
  std::size_t remove_largest_gaussians(double share) { return prune(splat_trainer_remove_largest, share); }
  std::size_t remove_least_contributing_gaussians(double share) { return prune(splat_trainer_remove_least_contributing, share); }
  std::size_t remove_least_opaque_gaussians(double share) { return prune(splat_trainer_remove_least_opaque, share); }
  [[nodiscard]] std::vector<float> densify_stats() const {
    std::vector<float> out(count_ * 8);
    check(splat_trainer_get_densify_stats(handle_, out.data()));
    return out;
  }
  [[nodiscard]] std::size_t gaussian_count() const noexcept { return count_; }
  [[nodiscard]] int sh_degree() const noexcept { return shDegree_; }
  [[nodiscard]] bool uses_fixed_point() const {
    int32_t fixed = 0;
    check(splat_trainer_info(handle_, nullptr, nullptr, nullptr, &fixed, nullptr, nullptr));
    return fixed != 0;
  }
  [[nodiscard]] std::uint64_t gpu_bytes() const {
    uint64_t bytes = 0;
    check(splat_trainer_info(handle_, nullptr, nullptr, nullptr, nullptr, &bytes, nullptr));
    return bytes;
  }
  [[nodiscard]] splat_trainer *handle() const noexcept { return handle_; }

private:
  template <class F> DensifyResult edit(F call, std::size_t capacity) {
    DensifyResult out;
    out.source.resize(capacity);
    splat_densify_result r{};
    check(call(&r, out.source.data(), capacity));
    count_ = static_cast<std::size_t>(r.count);
    out.source.resize(count_);
    out.cloned = r.cloned;
    out.split = r.split;
    out.seeded = r.seeded;
    out.pruned = r.pruned;
    out.heldBack = r.held_back;
    return out;
  }
  std::size_t prune(int (*call)(splat_trainer *, double, uint64_t *), double share) {
    uint64_t removed = 0;
    check(call(handle_, share, &removed));
    count_ -= static_cast<std::size_t>(removed);
    return static_cast<std::size_t>(removed);
  }

  splat_trainer *handle_ = nullptr;
  int shDegree_ = 0;
  std::size_t count_ = 0;
};

inline splat_session_options default_session_options() {
  splat_session_options o;
  splat_session_options_default(&o);
  return o;
}

// TrainSession (train.hpp:193-270) over the C ABI: the schedule around a
// trainer, one iteration per step(); the views live in device memory.
class Session {
public:
  Session(const splat_session_data &data, const splat_session_options &options = default_session_options(),
          const splat_trainer_options &trainerOptions = default_options())
      : iterations_(options.iterations) {
    check(splat_session_create(&data, &options, &trainerOptions, &handle_));
  }
  ~Session() { splat_session_destroy(handle_); }
  Session(const Session &) = delete;
  Session &operator=(const Session &) = delete;

  splat_step_stats step() {
    splat_step_stats s{};
    check(splat_session_step(handle_, &s));
    return s;
  }
  [[nodiscard]] splat_session_state state() const {
    splat_session_state s{};
    check(splat_session_get_state(handle_, &s));
    return s;
  }
  [[nodiscard]] bool finished() const { return state().iteration >= iterations_; }
  // The session's trainer, borrowed: its handle serves the C calls (render, get_cloud).
  [[nodiscard]] splat_trainer *trainer() const {
    splat_trainer *t = nullptr;
    check(splat_session_trainer(handle_, &t));
    return t;
  }

private:
  splat_session *handle_ = nullptr;
  int iterations_ = 0;
};

} // namespace splat_b200

// Adapters from the reference's own types, available where its headers come first.
#if defined(SPLAT_B200_WITH_REFERENCE_TYPES)
namespace splat_b200 {
inline Cloud from_reference(const splat::GaussianCloud &c) {
  Cloud out;
  out.shDegree = c.shDegree;
  out.positions = c.positions;
  out.scales = c.scales;
  out.rotations = c.rotations;
  out.opacities = c.opacities;
  out.sh = c.sh;
  return out;
}
inline splat_camera from_reference(const splat::Camera &c) {
  splat_camera out{};
  std::memcpy(out.view, &c.view[0][0], sizeof(out.view));
  out.position[0] = c.position.x;
  out.position[1] = c.position.y;
  out.position[2] = c.position.z;
  out.fx = c.fx;
  out.fy = c.fy;
  out.cx = c.cx;
  out.cy = c.cy;
  out.width = c.width;
  out.height = c.height;
  return out;
}
} // namespace splat_b200
#endif
