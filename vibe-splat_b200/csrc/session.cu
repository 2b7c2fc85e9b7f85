// The training session around the trainer (TrainSession, src/train/train.cpp
// :474-760; the schedule of src/train/schedule.cpp): coarse-to-fine views
// kept in HBM at three sizes, the order the views come in, the position rate
// and SH degree schedules, the densification rounds with their scored views,
// growth cap and opacity resets, the pruning rounds, and the starting cloud
// from points. It drives the trainer through its C ABI only, as the
// reference's session drives its Trainer.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "splat_b200.h"

namespace sb {
void set_last_error(const char *message);
}

namespace {

struct SessionFailure {
  int status;
  std::string message;
};

void ok(int status) {
  if (status != SPLAT_OK) throw SessionFailure{status, splat_last_error()};
}

#define SS_CUDA(call)                                                                                        \
  do {                                                                                                       \
    const cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess) throw SessionFailure{SPLAT_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

constexpr int kCoarseLevels = 2;
constexpr float kInitialOpacity = 0.1f;
constexpr float kResetOpacity = 0.01f;
constexpr double kMaxWorldFraction = 1.0;
constexpr double kMaxScreenFraction = 0.25;
constexpr float kScoreErrorShare = 0.1f;
constexpr int kOpacityResetInterval = 3000;
constexpr int kCheckpointRecovery = 1000;
constexpr int kRecoveryDelay = 300;
constexpr int kSpectrumViews = 8;
constexpr float kShC0 = 0.28209479177387814f;
// What a Gaussian's tile entries and a view's pixels cost this library's
// trainer: keys, values and their sort copies per entry; image, stops,
// adjoint, loss fields and target per pixel.
constexpr double kBytesPerTileEntry = 24.0;
constexpr double kBytesPerPixel = 80.0;

// A device buffer owned by the session.
struct Device {
  void *p = nullptr;
  Device() = default;
  Device(const Device &) = delete;
  Device &operator=(const Device &) = delete;
  Device(Device &&o) noexcept : p(o.p) { o.p = nullptr; }
  ~Device() {
    if (p != nullptr) cudaFree(p);
  }
  void make(size_t bytes) {
    if (p != nullptr) cudaFree(p);
    p = nullptr;
    SS_CUDA(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
  }
  template <class T = void> T *get() const { return static_cast<T *>(p); }
};

// resolution_switches (schedule.cpp:77-82).
std::array<double, 2> switches_of(double full, double half, double quarter) {
  const double lowest = full / 4.0;
  const auto at = [&](double energy) { return energy > lowest ? std::log(energy / lowest) / std::log(full / lowest) : 0.0; };
  const double untilFull = std::clamp(at(half), 0.0, 1.0);
  return {untilFull, std::clamp(at(quarter), 0.0, untilFull)};
}

// GrowthBudget (schedule.hpp:26-41, schedule.cpp:84-94).
struct Growth {
  double initial, final;
  Growth(size_t start, double factor)
      : initial((double)start), final(factor > 0.0 ? factor * (double)start : std::numeric_limits<double>::infinity()) {}
  uint64_t limit(double factor, double progress) const {
    if (std::isinf(final)) return std::numeric_limits<uint64_t>::max();
    const double growth = (final - initial) / std::pow(factor, 2.0 - progress);
    return static_cast<uint64_t>(initial + growth);
  }
  void observe(uint64_t wanted) {
    if (std::isinf(final)) return;
    final = std::max(final, 0.98 * final + (double)wanted);
  }
};

// frequency_energy on the device for one host or device RGBA8 image.
std::vector<double> energy_of(const uint8_t *deviceRgba, int width, int height, const std::vector<int> &factors, cudaStream_t stream) {
  if (!sb::spectrum_supported(width, height)) throw SessionFailure{SPLAT_ERR_INVALID, "spectrum: images up to 4096 x 4096"};
  if (factors.empty() || factors.size() > 8) throw SessionFailure{SPLAT_ERR_INVALID, "spectrum: 1 to 8 factors"};
  for (int f : factors)
    if (f < 1) throw SessionFailure{SPLAT_ERR_INVALID, "spectrum: factors must be positive"};
  const int blocks = 592;
  Device scratch, partials, dFactors;
  scratch.make(sb::spectrum_scratch_bytes(width, height));
  partials.make((size_t)blocks * factors.size() * sizeof(double));
  dFactors.make(factors.size() * sizeof(int));
  SS_CUDA(cudaMemcpyAsync(dFactors.p, factors.data(), factors.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
  sb::launch_frequency_energy(deviceRgba, width, height, dFactors.get<int>(), (int)factors.size(), scratch.p, partials.get<double>(), blocks,
                              stream);
  SS_CUDA(cudaGetLastError());
  std::vector<double> h((size_t)blocks * factors.size());
  SS_CUDA(cudaMemcpyAsync(h.data(), partials.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
  SS_CUDA(cudaStreamSynchronize(stream));
  std::vector<double> out(factors.size(), 0.0);
  for (int b = 0; b < blocks; ++b)
    for (size_t k = 0; k < factors.size(); ++k) out[k] += h[(size_t)b * factors.size() + k];
  return out;
}

// neighbour_distances (train.cpp:143-189) on the device: the grid from the
// points' bounds, then the search.
std::vector<float> distances_of(const double *points, size_t count, cudaStream_t stream) {
  if (count == 0) return {};
  if (count > 0xFFFFFFFFull / 2) throw SessionFailure{SPLAT_ERR_INVALID, "too many points"};
  double low[3], high[3];
  for (int a = 0; a < 3; ++a) {
    low[a] = std::numeric_limits<double>::max();
    high[a] = std::numeric_limits<double>::lowest();
  }
  for (size_t i = 0; i < count; ++i)
    for (int a = 0; a < 3; ++a) {
      low[a] = std::min(low[a], points[i * 3 + a]);
      high[a] = std::max(high[a], points[i * 3 + a]);
    }
  const double size[3] = {high[0] - low[0], high[1] - low[1], high[2] - low[2]};
  const double cell = std::max(std::cbrt(std::max(size[0] * size[1] * size[2], 1e-30) / static_cast<double>(count) * 8.0),
                               std::max({size[0], size[1], size[2]}) / 512.0);
  int3 dims;
  dims.x = (int)((high[0] - low[0]) / cell) + 1;
  dims.y = (int)((high[1] - low[1]) / cell) + 1;
  dims.z = (int)((high[2] - low[2]) / cell) + 1;
  if ((uint64_t)dims.x * dims.y * dims.z > 0xFFFFFFFFull) throw SessionFailure{SPLAT_ERR_INVALID, "the points' grid is too large"};
  Device scratch, out, error;
  scratch.make(sb::neighbour_scratch_bytes((uint32_t)count));
  out.make(count * 4);
  error.make(4);
  SS_CUDA(cudaMemsetAsync(error.p, 0, 4, stream));
  if (sb::neighbour_distances(points, (uint32_t)count, make_double3(low[0], low[1], low[2]), cell, dims, scratch.p, out.get<float>(),
                              error.get<uint32_t>(), stream) != 0)
    throw SessionFailure{SPLAT_ERR_DEVICE, "neighbour search: copy failed"};
  SS_CUDA(cudaGetLastError());
  std::vector<float> h(count);
  uint32_t flag = 0;
  SS_CUDA(cudaMemcpyAsync(h.data(), out.p, count * 4, cudaMemcpyDeviceToHost, stream));
  SS_CUDA(cudaMemcpyAsync(&flag, error.p, 4, cudaMemcpyDeviceToHost, stream));
  SS_CUDA(cudaStreamSynchronize(stream));
  if (flag != 0) throw SessionFailure{SPLAT_ERR_DEVICE, "neighbour search: the sort's look-back gave up waiting"};
  return h;
}

// initial_cloud (train.cpp:194-212): a Gaussian per point, as large as its
// neighbours are far, unrotated, opacity 0.1, its colour in the DC term.
struct HostCloud {
  int degree = 0;
  std::vector<float> positions, scales, rotations, opacities, sh;
};

HostCloud initial_cloud(const double *points, const uint8_t *colors, size_t count, int degree, cudaStream_t stream) {
  HostCloud c;
  c.degree = degree;
  const size_t coefficients = (size_t)(degree + 1) * (degree + 1);
  c.positions.resize(count * 3);
  c.scales.resize(count * 3);
  c.rotations.assign(count * 4, 0.f);
  c.opacities.resize(count);
  c.sh.assign(count * coefficients * 3, 0.f);
  const std::vector<float> distances = distances_of(points, count, stream);
  const float logitOpacity = std::log(kInitialOpacity / (1.f - kInitialOpacity));
  for (size_t i = 0; i < count; ++i) {
    for (size_t a = 0; a < 3; ++a) {
      c.positions[i * 3 + a] = static_cast<float>(points[i * 3 + a]);
      c.scales[i * 3 + a] = std::log(distances[i]);
      c.sh[i * coefficients * 3 + a] = (static_cast<float>(colors[i * 3 + a]) / 255.f - 0.5f) / kShC0;
    }
    c.rotations[i * 4] = 1.f;
    c.opacities[i] = logitOpacity;
  }
  return c;
}

// growth_factor (train.cpp:362-366).
double growth_factor_of(double maxGrowth, int iterations) {
  if (maxGrowth >= 0.0) return maxGrowth;
  return 4.0 * std::max(1.0, static_cast<double>(iterations) / 7000.0);
}

// psnr_of (evaluate.cpp:27-32) with the neutral exposure.
double psnr_of(const std::vector<float> &render, const uint8_t *target, size_t pixels) {
  double sum = 0.0;
  for (size_t i = 0; i < pixels; ++i) {
    const float *c = render.data() + i * 4;
    double e = 0.0;
    for (size_t r = 0; r < 3; ++r) {
      const double d = std::clamp(static_cast<double>(c[r]), 0.0, 1.0) - target[i * 4 + r] / 255.0;
      e += d * d;
    }
    sum += e;
  }
  const double mse = sum / (3.0 * static_cast<double>(pixels));
  return mse > 0.0 ? -10.0 * std::log10(mse) : 100.0;
}

} // namespace

struct splat_session {
  splat_session_options options{};
  splat_trainer_options trainerOptions{};
  splat_trainer *trainer = nullptr;
  splat_rng *densifyRng = nullptr;
  cudaStream_t stream = nullptr;
  double extent = 1.0, typicalDepth = 1.0;
  // levels[l][i]: view i at 1 / 2^(l + 1) of its size for l < 2, full size at l = 2.
  std::vector<splat_camera> cameras[kCoarseLevels + 1];
  std::vector<Device> images[kCoarseLevels + 1];
  std::vector<uint8_t> probe; // the first view at full size, on the host, for the reports
  std::array<double, kCoarseLevels> coarseUntil{0.35, 0.15};
  bool haveSmaller = false;
  int densifyFrom = 0, densifyUntil = 0, pruneAgainAt = 0, shInterval = 1;
  std::mt19937 rng;
  std::vector<size_t> order;
  splat_learning_rates rates{};
  double positionStart = 0.0, positionEnd = 0.0;
  Growth growth{1, 0.0};
  double entriesPerVisible = 16.0;
  double lossSum = 0.0;
  int lossCount = 0;
  int lastOpacityReset = -kCheckpointRecovery;
  int iteration = 0;
  size_t lastView = 0;
  splat_session_state state{};

  ~splat_session() {
    if (trainer != nullptr) splat_trainer_destroy(trainer);
    if (densifyRng != nullptr) splat_rng_destroy(densifyRng);
    for (auto &level : images) level.clear();
    if (stream != nullptr) cudaStreamDestroy(stream);
  }

  int views() const { return (int)cameras[kCoarseLevels].size(); }

  size_t coarse_level(int at) const {
    if (!haveSmaller) return kCoarseLevels;
    const double progress = static_cast<double>(at - 1) / std::max(options.iterations - 1, 1);
    for (size_t level = kCoarseLevels; level-- > 0;)
      if (progress < coarseUntil[level]) return level;
    return kCoarseLevels;
  }

  void refill_order() {
    if (!order.empty()) return;
    order.resize((size_t)views());
    std::iota(order.begin(), order.end(), size_t{0});
    std::shuffle(order.begin(), order.end(), rng);
  }

  uint64_t bytes_per_gaussian() const {
    uint64_t b = 0;
    ok(splat_trainer_info(trainer, nullptr, nullptr, nullptr, nullptr, nullptr, &b));
    return b;
  }
  uint64_t gaussians() const {
    int64_t n = 0;
    ok(splat_trainer_info(trainer, &n, nullptr, nullptr, nullptr, nullptr, nullptr));
    return (uint64_t)n;
  }

  // A view that does not fit the budget gives up its largest Gaussians and is
  // tried again (TrainSession::fitting, train.cpp:531-543).
  template <class F> void fitting(F work) {
    for (;;) {
      const int status = work();
      if (status == SPLAT_OK) return;
      if (status != SPLAT_ERR_BUDGET) ok(status);
      uint64_t removed = 0;
      ok(splat_trainer_remove_largest(trainer, 0.05, &removed));
      if (removed == 0) ok(status);
    }
  }

  size_t pixels_of(size_t level, size_t view) const {
    return (size_t)cameras[level][view].width * cameras[level][view].height;
  }
  const uint8_t *image_of(size_t level, size_t view) const { return images[level][view].get<uint8_t>(); }

  void step(splat_step_stats *out);
};

void splat_session::step(splat_step_stats *out) {
  if (iteration >= options.iterations) throw SessionFailure{SPLAT_ERR_STATE, "training has already finished"};
  const int it = ++iteration;
  const size_t level = coarse_level(it);
  // The views of this step, drawn one after another as the reference draws
  // one per iteration (refill, take the back, refill for the next).
  const int batch = std::clamp(options.views_per_step, 1, 8);
  size_t picked[8];
  for (int b = 0; b < batch; ++b) {
    refill_order();
    picked[b] = order.back();
    order.pop_back();
    refill_order(); // the next view's draw, as the reference makes it for its prefetch
  }
  lastView = picked[batch - 1];
  const size_t viewIndex = lastView;

  const double progress = static_cast<double>(it - 1) / std::max(options.iterations - 1, 1);
  const double held = options.adaptive_schedule != 0 && options.full_resolution == 0 ? coarseUntil[0] : 0.0;
  const double decay = std::clamp((progress - held) / std::max(1.0 - held, 1e-9), 0.0, 1.0);
  rates.position = static_cast<float>(positionStart * std::pow(positionEnd / positionStart, decay));
  ok(splat_trainer_set_active_sh_degree(trainer, (it - 1) / shInterval));
  splat_step_stats stats{};
  const splat_camera &camera = cameras[level][viewIndex];
  if (batch == 1) {
    fitting([&] {
      return splat_trainer_step_device_target(trainer, &camera, image_of(level, viewIndex), pixels_of(level, viewIndex) * 4, &rates,
                                              &stats);
    });
  } else {
    splat_camera group[8];
    const uint8_t *targets[8];
    splat_step_stats each[8];
    for (int b = 0; b < batch; ++b) {
      group[b] = cameras[level][picked[b]];
      targets[b] = image_of(level, picked[b]);
    }
    fitting([&] { return splat_trainer_step_batch_device_targets(trainer, group, targets, batch, &rates, each); });
    stats = each[0];
    float loss = 0.f;
    for (int b = 0; b < batch; ++b) loss += each[b].loss;
    stats.loss = loss / (float)batch;
  }
  state.views_in_step = batch;
  if (!std::isfinite(stats.loss))
    throw SessionFailure{SPLAT_ERR_NONFINITE, "the loss became " + std::to_string(stats.loss) + " at iteration " + std::to_string(it)};
  if (it == 1) state.first_loss = stats.loss;
  state.last_loss = stats.loss;
  lossSum += stats.loss;
  ++lossCount;
  if (stats.visible_splats > 0) entriesPerVisible = 0.98 * entriesPerVisible + 0.02 * stats.tile_entries / stats.visible_splats;

  // The probe view's PSNR, before this iteration's pruning and opacity reset.
  const bool reportDue = options.report_every > 0 && (it % options.report_every == 0 || it == options.iterations);
  if (reportDue) {
    const splat_camera &p = cameras[kCoarseLevels][0];
    std::vector<float> render((size_t)p.width * p.height * 4);
    fitting([&] { return splat_trainer_render(trainer, &p, render.data()); });
    state.probe_psnr = psnr_of(render, probe.data(), (size_t)p.width * p.height);
    state.report_iteration = it;
    state.mean_loss = lossSum / std::max(lossCount, 1);
    lossSum = 0.0;
    lossCount = 0;
  }

  // Before densification, which may cap the opacities the ranking depends on.
  if (options.prune_share > 0.0 && (it == densifyUntil || it == pruneAgainAt)) {
    if (it == densifyUntil) {
      ok(splat_trainer_reset_densify_stats(trainer));
      for (int i = 0; i < views(); ++i) {
        splat_step_stats s{};
        fitting([&] {
          return splat_trainer_collect_statistics_device_target(trainer, &cameras[kCoarseLevels][(size_t)i],
                                                                image_of(kCoarseLevels, (size_t)i),
                                                                pixels_of(kCoarseLevels, (size_t)i) * 4, &s);
        });
      }
    }
    uint64_t removed = 0;
    ok(splat_trainer_remove_least_contributing(trainer, options.prune_share, &removed));
    state.pruned_total += removed;
  }

  if (options.densify != 0 && it >= densifyFrom && it <= densifyUntil && it % options.densify_interval == 0) {
    const auto started = std::chrono::steady_clock::now();
    const double perGaussian = static_cast<double>(bytes_per_gaussian()) + 1.5 * kBytesPerTileEntry * entriesPerVisible;
    const uint64_t available = trainerOptions.memory_budget;
    const uint64_t pixelBytes = static_cast<uint64_t>((double)camera.width * camera.height * kBytesPerPixel);
    splat_densify_options d;
    splat_densify_options_default(&d);
    const double densifyProgress = static_cast<double>(it) / std::max(densifyUntil, 1);
    const auto rise = static_cast<float>(std::pow(options.threshold_rise, densifyProgress - 0.5));
    d.gradient_threshold = options.gradient_threshold * rise;
    d.split_threshold = options.split_threshold * rise;
    d.dense_scale = static_cast<float>(options.dense_fraction * extent);
    d.max_world_scale = static_cast<float>(kMaxWorldFraction * extent);
    d.max_screen_radius = static_cast<float>(kMaxScreenFraction * std::max(camera.width, camera.height));
    d.prune_large = it > kOpacityResetInterval && options.significance_prune == 0 ? 1 : 0;
    if (options.significance_prune != 0) d.transparent_share = 0.5;
    d.explore_splits = d.explore_seeds = (uint64_t)std::max(options.explore, 0);
    d.edge_split = options.edge_split;
    d.max_gaussians = available > pixelBytes ? static_cast<uint64_t>(static_cast<double>(available - pixelBytes) / perGaussian) : 0;
    if (options.max_gaussians > 0) d.max_gaussians = std::min<uint64_t>(d.max_gaussians, options.max_gaussians);
    if (options.score_views > 0 && options.densify_mode == 0) {
      d.scored_views = options.score_views;
      d.min_marked_pixels = options.score_min_pixels;
      for (int k = 0; k < options.score_views; ++k) {
        uint64_t i = 0;
        ok(splat_rng_pick(densifyRng, (uint64_t)views(), &i));
        const size_t scoredLevel = coarse_level(it);
        // A pixel of a smaller image stands for several of the full one.
        const float area = static_cast<float>(cameras[kCoarseLevels][i].width) / static_cast<float>(cameras[scoredLevel][i].width);
        splat_step_stats s{};
        fitting([&] {
          return splat_trainer_score_view_device_target(trainer, &cameras[scoredLevel][i], image_of(scoredLevel, i),
                                                        pixels_of(scoredLevel, i) * 4, kScoreErrorShare, area * area, &s);
        });
      }
    }
    if (options.adaptive_schedule != 0) {
      const size_t lv = coarse_level(it);
      const double factor = lv == kCoarseLevels ? 1.0 : std::pow(2.0, static_cast<double>(lv + 1));
      d.max_gaussians = std::min<uint64_t>(d.max_gaussians, growth.limit(factor, progress));
    } else {
      d.max_gaussians = std::min<uint64_t>(d.max_gaussians, growth.limit(1.0, 1.0));
    }
    splat_densify_result r{};
    if (options.densify_mode == 1) {
      splat_relocate_options m;
      splat_relocate_options_default(&m);
      m.max_gaussians = d.max_gaussians;
      ok(splat_trainer_relocate(trainer, &m, densifyRng, &r, nullptr, 0));
    } else {
      ok(splat_trainer_densify(trainer, &d, densifyRng, &r, nullptr, 0));
      if (options.adaptive_schedule != 0) growth.observe(r.cloned + r.split + r.held_back);
      state.held_back_total += r.held_back;
      // Not on the last round: the cloud would have no densification left to recover with.
      if (it % kOpacityResetInterval == 0 && it < densifyUntil) {
        ok(splat_trainer_reset_opacity(trainer, kResetOpacity));
        lastOpacityReset = it;
      }
    }
    state.last_densify = r;
    state.densify_rounds += 1;
    state.densify_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - started).count();
  }

  if (options.recovery_prune > 0.0 && lastOpacityReset > 0 && it == lastOpacityReset + kRecoveryDelay) {
    uint64_t removed = 0;
    ok(splat_trainer_remove_least_opaque(trainer, options.recovery_prune, &removed));
    state.pruned_total += removed;
  }
  state.iteration = it;
  state.level = (int32_t)level;
  state.view = (int32_t)viewIndex;
  state.position_rate = rates.position;
  state.gaussians = gaussians();
  state.coarse_until[0] = coarseUntil[0];
  state.coarse_until[1] = coarseUntil[1];
  if (out != nullptr) *out = stats;
}

namespace {

template <class F> int session_guarded(F &&f) {
  try {
    f();
    return SPLAT_OK;
  } catch (const SessionFailure &e) {
    sb::set_last_error(e.message.c_str());
    return e.status;
  } catch (const std::bad_alloc &) {
    sb::set_last_error("host allocation failed");
    return SPLAT_ERR_NOMEM;
  } catch (const std::exception &e) {
    sb::set_last_error(e.what());
    return SPLAT_ERR_INVALID;
  }
}

} // namespace

extern "C" {

void splat_session_options_default(splat_session_options *o) {
  if (o == nullptr) return;
  *o = splat_session_options{};
  o->iterations = 15000;
  o->sh_degree = 2;
  o->seed = 1;
  o->report_every = 500;
  o->densify = 1;
  o->densify_mode = 0;
  o->full_adam = 0;
  o->full_resolution = 0;
  o->adaptive_schedule = 0;
  o->gradient_threshold = 2e-4f;
  o->split_threshold = 1.2e-3f;
  o->dense_fraction = 0.001;
  o->densify_interval = 100;
  o->score_views = 10;
  o->score_min_pixels = 5.f;
  o->explore = 0;
  o->significance_prune = 0;
  o->edge_split = 0;
  o->threshold_rise = 1.0;
  o->prune_share = 0.0;
  o->recovery_prune = 0.0;
  o->max_growth = -1.0;
  o->max_gaussians = 0;
  o->coarse_until[0] = 0.35;
  o->coarse_until[1] = 0.15;
  o->views_per_step = 1;
}

int splat_session_create(const splat_session_data *data, const splat_session_options *options,
                         const splat_trainer_options *trainer_options, splat_session **out) {
  return session_guarded([&] {
    if (data == nullptr || options == nullptr || out == nullptr) throw SessionFailure{SPLAT_ERR_INVALID, "null argument"};
    if (data->views < 1 || data->cameras == nullptr || data->images == nullptr) throw SessionFailure{SPLAT_ERR_INVALID, "no training views"};
    if (data->point_count == 0 || data->points == nullptr || data->colors == nullptr)
      throw SessionFailure{SPLAT_ERR_INVALID, "no starting points"};
    if (options->iterations < 1 || options->densify_interval < 1) throw SessionFailure{SPLAT_ERR_INVALID, "iterations and interval must be positive"};
    if (options->sh_degree < 0 || options->sh_degree > 3) throw SessionFailure{SPLAT_ERR_INVALID, "SH degree must be 0..3"};
    auto *s = new splat_session();
    try {
      s->options = *options;
      if (trainer_options != nullptr) s->trainerOptions = *trainer_options;
      else splat_trainer_options_default(&s->trainerOptions);
      s->extent = data->extent;
      s->typicalDepth = data->typical_depth;
      SS_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
      // The views in HBM at full size, then halved twice on the device
      // (train.cpp:416-427) unless training at full size throughout.
      const int views = data->views;
      s->haveSmaller = options->full_resolution == 0;
      s->coarseUntil = {options->coarse_until[0], options->coarse_until[1]};
      for (int i = 0; i < views; ++i) {
        const splat_camera &c = data->cameras[i];
        if (c.width < 1 || c.height < 1 || data->images[i] == nullptr) throw SessionFailure{SPLAT_ERR_INVALID, "bad view"};
        Device d;
        d.make((size_t)c.width * c.height * 4);
        SS_CUDA(cudaMemcpyAsync(d.p, data->images[i], (size_t)c.width * c.height * 4, cudaMemcpyHostToDevice, s->stream));
        s->cameras[kCoarseLevels].push_back(c);
        s->images[kCoarseLevels].push_back(std::move(d));
      }
      s->probe.assign(data->images[0], data->images[0] + (size_t)data->cameras[0].width * data->cameras[0].height * 4);
      if (s->haveSmaller) {
        for (int level = 0; level < kCoarseLevels; ++level) {
          const int from = level == 0 ? kCoarseLevels : level - 1;
          for (int i = 0; i < views; ++i) {
            splat_camera c = s->cameras[from][(size_t)i];
            const int width = c.width;
            c.width /= 2;
            c.height /= 2;
            c.fx *= 0.5f;
            c.fy *= 0.5f;
            c.cx *= 0.5f;
            c.cy *= 0.5f;
            if (c.width < 1 || c.height < 1) throw SessionFailure{SPLAT_ERR_INVALID, "views too small for the coarse levels"};
            Device d;
            d.make((size_t)c.width * c.height * 4);
            sb::launch_half_size(s->image_of((size_t)from, (size_t)i), width, c.height * 2, d.get<uint8_t>(), s->stream);
            s->cameras[level].push_back(c);
            s->images[level].push_back(std::move(d));
          }
        }
        SS_CUDA(cudaGetLastError());
        if (options->adaptive_schedule != 0) {
          std::array<double, 3> energy{};
          const size_t step = std::max<size_t>((size_t)views / kSpectrumViews, 1);
          for (size_t i = 0; i < (size_t)views; i += step) {
            const splat_camera &c = s->cameras[kCoarseLevels][i];
            const std::vector<double> x = energy_of(s->image_of(kCoarseLevels, i), c.width, c.height, {1, 2, 4}, s->stream);
            for (size_t k = 0; k < 3; ++k) energy[k] += x[k];
          }
          s->coarseUntil = switches_of(energy[0], energy[1], energy[2]);
        }
      }
      SS_CUDA(cudaStreamSynchronize(s->stream));

      // The trainer (train.cpp:486-506), from the starting points.
      s->trainerOptions.selective_adam = options->full_adam != 0 ? 0 : 1;
      if (options->views_per_step < 1 || options->views_per_step > 8)
        throw SessionFailure{SPLAT_ERR_INVALID, "views_per_step must be 1..8"};
      if (options->views_per_step > 1) s->trainerOptions.sort_form = SPLAT_SORT_TILE_DEPTH_64; // several views share one sort
      s->trainerOptions.near_plane = static_cast<float>(s->typicalDepth * 0.01);
      const HostCloud c = initial_cloud(data->points, data->colors, data->point_count, options->sh_degree, s->stream);
      splat_cloud cloud{(int32_t)data->point_count, options->sh_degree, c.positions.data(), c.scales.data(), c.rotations.data(),
                        c.opacities.data(), c.sh.data()};
      ok(splat_trainer_create(&cloud, &s->trainerOptions, &s->trainer));

      // The paper's schedule for 30000 iterations, proportional when shorter.
      const int iterations = options->iterations;
      s->densifyFrom = std::min(500, iterations / 20 + 1);
      s->densifyUntil = iterations / 2;
      s->pruneAgainAt = (s->densifyUntil + iterations) / 2;
      s->shInterval = std::max(1, std::min(1000, iterations / 10));
      ok(splat_trainer_set_active_sh_degree(s->trainer, 0));
      s->rng.seed(options->seed);
      ok(splat_rng_create(options->seed + 1, &s->densifyRng));
      splat_learning_rates_default(&s->rates);
      s->positionStart = 1.6e-4 * s->extent;
      s->positionEnd = 1.6e-6 * s->extent;
      s->growth = Growth(data->point_count, growth_factor_of(options->max_growth, iterations));
      s->state.coarse_until[0] = s->coarseUntil[0];
      s->state.coarse_until[1] = s->coarseUntil[1];
      s->state.gaussians = data->point_count;
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
  });
}

int splat_session_destroy(splat_session *session) {
  delete session;
  return SPLAT_OK;
}

int splat_session_step(splat_session *session, splat_step_stats *stats) {
  return session_guarded([&] {
    if (session == nullptr) throw SessionFailure{SPLAT_ERR_INVALID, "null session"};
    session->step(stats);
  });
}

int splat_session_get_state(splat_session *session, splat_session_state *out) {
  return session_guarded([&] {
    if (session == nullptr || out == nullptr) throw SessionFailure{SPLAT_ERR_INVALID, "null argument"};
    *out = session->state;
  });
}

int splat_session_trainer(splat_session *session, splat_trainer **out) {
  return session_guarded([&] {
    if (session == nullptr || out == nullptr) throw SessionFailure{SPLAT_ERR_INVALID, "null argument"};
    *out = session->trainer;
  });
}

int splat_frequency_energy(const uint8_t *rgba, int32_t width, int32_t height, const int32_t *factors, int32_t count, double *out) {
  return session_guarded([&] {
    if (rgba == nullptr || factors == nullptr || out == nullptr || count < 1) throw SessionFailure{SPLAT_ERR_INVALID, "null argument"};
    cudaStream_t stream = nullptr;
    SS_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    try {
      Device image;
      image.make((size_t)width * height * 4);
      SS_CUDA(cudaMemcpyAsync(image.p, rgba, (size_t)width * height * 4, cudaMemcpyHostToDevice, stream));
      const std::vector<double> e = energy_of(image.get<uint8_t>(), width, height, std::vector<int>(factors, factors + count), stream);
      std::copy(e.begin(), e.end(), out);
    } catch (...) {
      cudaStreamDestroy(stream);
      throw;
    }
    cudaStreamDestroy(stream);
  });
}

int splat_resolution_switches(double full, double half, double quarter, double out[2]) {
  return session_guarded([&] {
    if (out == nullptr) throw SessionFailure{SPLAT_ERR_INVALID, "null output"};
    const std::array<double, 2> s = switches_of(full, half, quarter);
    out[0] = s[0];
    out[1] = s[1];
  });
}

int splat_growth_limit(double initial_count, double factor, const uint64_t *observed, int32_t observations, double image_factor,
                       double progress, uint64_t *limit, double *final_count) {
  return session_guarded([&] {
    Growth g((size_t)initial_count, factor);
    for (int32_t k = 0; k < observations; ++k) g.observe(observed[k]);
    if (limit != nullptr) *limit = g.limit(image_factor, progress);
    if (final_count != nullptr) *final_count = g.final;
  });
}

int splat_half_size(const uint8_t *rgba, int32_t width, int32_t height, uint8_t *out) {
  return session_guarded([&] {
    if (rgba == nullptr || out == nullptr || width < 2 || height < 2) throw SessionFailure{SPLAT_ERR_INVALID, "bad image"};
    Device in, half;
    in.make((size_t)width * height * 4);
    half.make((size_t)(width / 2) * (height / 2) * 4);
    SS_CUDA(cudaMemcpy(in.p, rgba, (size_t)width * height * 4, cudaMemcpyHostToDevice));
    sb::launch_half_size(in.get<uint8_t>(), width, height, half.get<uint8_t>(), nullptr);
    SS_CUDA(cudaGetLastError());
    SS_CUDA(cudaMemcpy(out, half.p, (size_t)(width / 2) * (height / 2) * 4, cudaMemcpyDeviceToHost));
  });
}

int splat_initial_cloud(const double *points, const uint8_t *colors, uint64_t count, int32_t sh_degree, float *positions, float *scales,
                        float *rotations, float *opacities, float *sh) {
  return session_guarded([&] {
    if (points == nullptr || colors == nullptr || count == 0) throw SessionFailure{SPLAT_ERR_INVALID, "no points"};
    if (sh_degree < 0 || sh_degree > 3) throw SessionFailure{SPLAT_ERR_INVALID, "SH degree must be 0..3"};
    const HostCloud c = initial_cloud(points, colors, count, sh_degree, nullptr);
    std::copy(c.positions.begin(), c.positions.end(), positions);
    std::copy(c.scales.begin(), c.scales.end(), scales);
    std::copy(c.rotations.begin(), c.rotations.end(), rotations);
    std::copy(c.opacities.begin(), c.opacities.end(), opacities);
    std::copy(c.sh.begin(), c.sh.end(), sh);
  });
}

} // extern "C"
