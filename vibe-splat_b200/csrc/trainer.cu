// The trainer behind the C ABI of include/splat_b200.h: device buffers, the
// order of the step's launches, the host reads, and the CUDA-graph form.
//
// Mirrors splat::Trainer (src/train/trainer.cpp). The reference records two
// Vulkan submissions per step with a host wait between them, to read the tile
// entry count and size the entry buffers (trainer.cpp:328-375, 593-602). This
// trainer does the same in its plain form. In its graph form the entry count
// stays on the device: the entry pool is sized from earlier steps, the
// kernels after the emission skip their work when a step would overflow it
// (an error bit, never an out-of-bounds write), and the host grows the pool
// and runs that step again. With no host wait inside, the whole step is one
// CUDA graph.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <new>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include <cuda_fp16.h>

#include "kernels.cuh"
#include "sort.cuh"
#include "splat_b200.h"

namespace sb {

thread_local std::string g_lastError;

// For entry points outside this file. An empty message clears without
// allocating.
void set_last_error(const char *message) {
  if (message == nullptr || message[0] == '\0') g_lastError.clear();
  else g_lastError.assign(message);
}

struct Failure {
  int status;
  std::string message;
};

#define SB_CUDA(call)                                                                                  \
  do {                                                                                                 \
    const cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) throw Failure{SPLAT_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

class DeviceBuffer {
public:
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  ~DeviceBuffer() { release(); }
  void release() {
    if (ptr_ != nullptr) cudaFree(ptr_);
    ptr_ = nullptr;
    bytes_ = 0;
  }
  // Makes the buffer at least `bytes` long; the contents are lost when it grows.
  void ensure(size_t bytes) {
    if (bytes <= bytes_ && ptr_ != nullptr) return;
    release();
    const size_t want = std::max<size_t>(bytes, 256);
    if (cudaMalloc(&ptr_, want) != cudaSuccess) {
      cudaGetLastError();
      ptr_ = nullptr;
      throw Failure{SPLAT_ERR_NOMEM, "device allocation of " + std::to_string(want) + " bytes failed"};
    }
    bytes_ = want;
  }
  template <class T = void> T *get() const { return static_cast<T *>(ptr_); }
  size_t bytes() const { return bytes_; }
  friend void swap(DeviceBuffer &a, DeviceBuffer &b) noexcept {
    std::swap(a.ptr_, b.ptr_);
    std::swap(a.bytes_, b.bytes_);
  }

private:
  void *ptr_ = nullptr;
  size_t bytes_ = 0;
};

// Makes buffer at least `bytes` long, with a quarter to spare when it must
// grow, for buffers that follow a Gaussian count that grows by steps.
void grow(DeviceBuffer &buffer, size_t bytes) {
  if (buffer.get() == nullptr || buffer.bytes() < bytes) buffer.ensure(bytes + bytes / 4);
}

class PinnedBuffer {
public:
  PinnedBuffer() = default;
  PinnedBuffer(const PinnedBuffer &) = delete;
  PinnedBuffer &operator=(const PinnedBuffer &) = delete;
  friend void swap(PinnedBuffer &a, PinnedBuffer &b) noexcept {
    std::swap(a.ptr_, b.ptr_);
    std::swap(a.bytes_, b.bytes_);
  }
  ~PinnedBuffer() {
    if (ptr_ != nullptr) cudaFreeHost(ptr_);
  }
  void ensure(size_t bytes) {
    if (bytes <= bytes_ && ptr_ != nullptr) return;
    if (ptr_ != nullptr) cudaFreeHost(ptr_);
    ptr_ = nullptr;
    bytes_ = 0;
    if (cudaMallocHost(&ptr_, std::max<size_t>(bytes, 64)) != cudaSuccess) {
      cudaGetLastError();
      throw Failure{SPLAT_ERR_NOMEM, "pinned host allocation failed"};
    }
    bytes_ = std::max<size_t>(bytes, 64);
  }
  template <class T = void> T *get() const { return static_cast<T *>(ptr_); }
  size_t bytes() const { return bytes_; }

private:
  void *ptr_ = nullptr;
  size_t bytes_ = 0;
};

// What the host reads back at the end of a step.
struct StepReadback {
  uint32_t counters[4];
  uint32_t error;
  uint32_t pad[3];
  LossTotals totals;
};

// The step's read-back written by a kernel straight into the pinned host
// block (mapped into the device's address space), after the step's last
// kernel: no copy node after the step, and the stream synchronisation that
// follows makes the writes visible to the host.
__global__ void __launch_bounds__(64) k_readback(const uint32_t *__restrict__ src, uint32_t *dst, uint32_t words) {
  chain_enter();
  for (uint32_t i = threadIdx.x; i < words; i += 64u) dst[i] = src[i];
}

constexpr int kStages = 8;
const char *const kStageNames[kStages] = {"project", "depth sort", "count tiles", "tile lists",
                                          "composite", "loss", "backward", "chain rule and step"};

// The entry sort's digit width: no more passes than digitBits would take, the
// key's bits spread evenly over them (12-bit tile ids: two 6-bit passes
// rather than 8 + 4; fewer buckets per pass write longer runs).
int entry_digits(int bits, int digitBits) {
  const int passes = (bits + digitBits - 1) / digitBits;
  const int even = (bits + passes - 1) / passes;
  return even < 6 ? 6 : (even > 8 ? 8 : even);
}

uint32_t bits_for(uint32_t values) {
  uint32_t b = 0;
  while (b < 32 && (1ull << b) < values) ++b;
  return std::max<uint32_t>(b, 1);
}

class Trainer {
public:
  // upload false: only sizes the buffers (the cloud's arrays may be null) and
  // leaves the parameters zero, for a caller that fills them on the device.
  Trainer(const splat_cloud &cloud, const splat_trainer_options &options, bool upload = true);
  ~Trainer();

  splat_trainer_options opt;
  uint32_t n = 0;
  int shDegree = 0, shCoeffs = 1, activeDegree = 0;
  uint32_t planeStride = 0; // elements between SH planes: n rounded up to kPlaneAlign
  ShStore shStore = ShStore::F16;
  StateStore stateStore = StateStore::BF16Pair;
  bool fixedPoint = false, oneSort = false, exactMath = true, useGraph = false;
  bool blendLists = false; // store-everything backward
  int digitBits = 8;
  int forwardPixels = 1, backwardPixels = 2; // pixels per thread of the compositing and float backward kernels
  int tileSize = 16, batchDepth = 128;        // the two-pixel kernels' tile edge and staging batch
  bool persistent = false;                    // the two-pixel kernels as persistent launches
  bool groupedSums = false;                   // the two-pixel float backward's sums by groups
  DeviceBuffer workCounters;                  // their tile counters (2 words), cleared every step
  cudaStream_t stream = nullptr;
  // The step's clears run on a second stream, forked from and joined back to
  // the first (branches of the same graph when captured).
  cudaStream_t side = nullptr;
  cudaEvent_t forkEvent = nullptr, joinEvent = nullptr, countForkEvent = nullptr, countEvent = nullptr;
  // The backward's tile order and the loss totals, made on the second stream
  // beside the loss and the backward.
  cudaEvent_t orderForkEvent = nullptr, orderEvent = nullptr, totalsForkEvent = nullptr, totalsEvent = nullptr;
  bool orderPending = false, orderForked = false, totalsPending = false;
  // Recording a CUDA graph: the forks onto the second stream above cost the
  // one-launch-at-a-time forms more host time than they save, so only a
  // captured step makes them.
  bool capturing = false;
  bool entryScratchClear = false; // the entry sort's scratch was cleared for this step
  // The next step's target on its way to the device: copied to pinned memory
  // and on to targetNext by copyStream while this step runs (copied is
  // recorded after that copy, consumed after the step that used it took it).
  cudaStream_t copyStream = nullptr;
  cudaEvent_t copied = nullptr, consumed = nullptr;
  DeviceBuffer targetNext;
  // A scored view (score_view): above 0, the share of the worst error that
  // marks a pixel; the target's edge weights and the worst error.
  float scoreShare = 0.0f;
  DeviceBuffer scoreEdge, scoreMax;

  DeviceBuffer positions, scales, rotations, opacities, shDc, shRest;
  DeviceBuffer state[5], grads[5], densifyStats;
  // Edits of the cloud (densify, relocate, prune): the next parameter and
  // state buffers, gathered into and swapped with the current ones; and the
  // scratch, tables and host-computed rows of an edit. Kept from one edit to
  // the next, so that a training run's edits allocate little.
  DeviceBuffer spareParams[6], spareState[5], editScratch, editTables, editRows;
  PinnedBuffer editHost;
  // Host scratch of relocation, kept so that later rounds touch no new pages.
  std::vector<int32_t> editOrigin, editState;
  std::vector<int> editTimes;
  std::vector<double> editCumulative, editCoarse;
  bool haveGradients = false, haveRaw = false;

  // Per (view, Gaussian).
  int viewSlots = 0;
  DeviceBuffer splats, reach, depthKeys, values, tmpKeys, tmpValues, offsets, raw, shGrad;
  // Tile entries.
  uint32_t entryCapacity = 0;
  DeviceBuffer entryKeys, entryValues, tmpEntryKeys, tmpEntryValues;
  bool entriesInTmp = false, depthInTmp = false, countOverlap = false;
  // Per pixel and per tile of the views of a step.
  DeviceBuffer image, stops, adjoint, fields, target, ranges, partials;
  // Store-everything variant: per-pixel blend counts, list offsets, the list pool, scan scratch and counters.
  DeviceBuffer listCounts, listOffsets, listPool, listScratch, listCounters;
  // Small things.
  // The step's small device inputs and outputs in one block, the views, the
  // chain rule's arguments, then the read-back, so that one copy from the
  // pinned block of the same layout (whose read-back part stays zero) sets
  // the first two and clears the third at the start of a step.
  DeviceBuffer dStep, sortScratchDepth, sortScratchEntries, scanScratch;
  PinnedBuffer hStep, hReadback, staging, stagingNext;
  void *hReadbackDevice = nullptr;
  static constexpr size_t kArgsAt = (sizeof(ViewSet) + 255) / 256 * 256;
  static constexpr size_t kReadbackAt = kArgsAt + (sizeof(ChainArgs) + 255) / 256 * 256;
  static constexpr size_t kStepBytes = kReadbackAt + sizeof(StepReadback);
  ViewSet *d_views() const { return dStep.get<ViewSet>(); }
  ChainArgs *d_args() const { return reinterpret_cast<ChainArgs *>(dStep.get<unsigned char>() + kArgsAt); }
  StepReadback *d_readback() const { return reinterpret_cast<StepReadback *>(dStep.get<unsigned char>() + kReadbackAt); }
  ViewSet *h_views() const { return hStep.get<ViewSet>(); }
  ChainArgs *h_args() const { return reinterpret_cast<ChainArgs *>(hStep.get<unsigned char>() + kArgsAt); }
  const uint8_t *prefetched = nullptr;
  size_t prefetchedBytes = 0;
  const uint8_t *pendingPrefetch = nullptr; // the next step's target, copied during this step
  size_t pendingPrefetchBytes = 0;

  ViewSet views{};
  uint32_t adamStep = 0;
  ChainArgs lastArgs{};

  // Graph form: one instantiated graph per shape of step.
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
  };
  std::map<std::string, GraphEntry> graphs;

  // Timings.
  bool timing = false;
  cudaEvent_t events[2 * kStages] = {};
  double stageTotals[kStages] = {};
  uint64_t timedIterations = 0;

  void set_views(const splat_camera *cameras, int count);
  void ensure_view_buffers();
  void ensure_entries(uint32_t total);
  uint64_t entry_bytes(uint64_t entries) const;
  uint64_t gpu_bytes() const;
  uint64_t bytes_per_gaussian() const;
  Params params() const;
  OptimState optim_state();
  void upload_targets(const uint8_t *const *targets, const size_t *bytes, int count);
  void stage_prefetch();
  void prefetch(const uint8_t *next, size_t bytes);
  bool take_prefetched(const uint8_t *const *targets, const size_t *bytes, int count);
  void record_prepare(bool backward);
  void record_forward();
  int entry_sort_bits() const;
  int raster_tile() const;
  RasterConfig raster_config();
  void record_backward_and_chain(ChainMode mode, bool statistics);
  void record_readback();
  void begin(int stage);
  void end(int stage);
  void clear_graphs();
  void score_view(const splat_camera *camera, const uint8_t *target, size_t bytes, float share, float pixelWeight,
                  splat_step_stats *stats, bool deviceTarget = false);
  std::string graph_key(ChainMode mode, bool statistics) const;
  void run(const splat_camera *cameras, const uint8_t *const *targets, const size_t *bytes, int count, ChainMode mode,
           const splat_learning_rates *rates, bool statistics, splat_step_stats *stats, bool deviceTargets = false);
  void render(const splat_camera *camera, float *out);
  void finish_stats(splat_step_stats *stats, int count);
  void fill_chain_args(ChainMode mode, bool statistics, const splat_learning_rates *rates);
  void set_sort(bool single, int digits);
  // Replaces the Gaussians, in place, by newN gathered from the current ones
  // (or, with a host cloud, uploaded from it; the state is gathered either way).
  void replace_gaussians(const int32_t *paramSource, const int32_t *stateSource, uint32_t newN, const splat_cloud *host = nullptr);
  void autotune(const splat_camera *camera, const uint8_t *target, size_t bytes, int repeats, splat_autotune_result *out);
};

// ---------------------------------------------------------------- set-up

// The cloud's parameters into device buffers in the trainer's layout, `to`
// = positions, scales, rotations, opacities (rows), SH DC (planes of `stride`
// elements) and SH rest (`stride` rows of sh_rest_stride elements), padding
// zero: DC as FP32, the rest in `store`, rounded to nearest.
void upload_cloud(const splat_cloud &cloud, int shCoeffs, ShStore store, uint32_t stride, DeviceBuffer *to[6]) {
  const size_t nn = (size_t)cloud.count, ps = stride;
  SB_CUDA(cudaMemcpy(to[0]->get(), cloud.positions, nn * 12, cudaMemcpyHostToDevice));
  SB_CUDA(cudaMemcpy(to[1]->get(), cloud.scales, nn * 12, cudaMemcpyHostToDevice));
  SB_CUDA(cudaMemcpy(to[2]->get(), cloud.rotations, nn * 16, cudaMemcpyHostToDevice));
  SB_CUDA(cudaMemcpy(to[3]->get(), cloud.opacities, nn * 4, cudaMemcpyHostToDevice));
  const int floats = 3 * shCoeffs;
  std::vector<float> dc(ps * 3, 0.0f);
  for (size_t i = 0; i < nn; ++i)
    for (int c = 0; c < 3; ++c) dc[c * ps + i] = cloud.sh[i * floats + c];
  SB_CUDA(cudaMemcpy(to[4]->get(), dc.data(), ps * 12, cudaMemcpyHostToDevice));
  const size_t rowStride = sh_rest_stride(shCoeffs, store), rest = ps * rowStride;
  if (rest == 0) return;
  std::vector<float> planes(rest, 0.0f);
  for (size_t i = 0; i < nn; ++i)
    for (int j = 3; j < floats; ++j) planes[i * rowStride + (size_t)(j - 3)] = cloud.sh[i * floats + j];
  if (store == ShStore::F32) {
    SB_CUDA(cudaMemcpy(to[5]->get(), planes.data(), rest * 4, cudaMemcpyHostToDevice));
    return;
  }
  std::vector<uint16_t> half(rest);
  for (size_t k = 0; k < rest; ++k) {
    if (store == ShStore::BF16) {
      uint32_t bits;
      std::memcpy(&bits, &planes[k], 4);
      half[k] = (uint16_t)((bits + 0x7FFFu + ((bits >> 16) & 1u)) >> 16);
    } else {
      half[k] = __half_as_ushort(__float2half_rn(planes[k]));
    }
  }
  SB_CUDA(cudaMemcpy(to[5]->get(), half.data(), rest * 2, cudaMemcpyHostToDevice));
}

Trainer::Trainer(const splat_cloud &cloud, const splat_trainer_options &options, bool upload) : opt(options) {
  if (cloud.count <= 0) throw Failure{SPLAT_ERR_INVALID, "nothing to train: the cloud is empty"};
  if (cloud.sh_degree < 0 || cloud.sh_degree > 3) throw Failure{SPLAT_ERR_INVALID, "GaussianCloud: SH degree must be 0..3"};
  if (upload && (cloud.positions == nullptr || cloud.scales == nullptr || cloud.rotations == nullptr || cloud.opacities == nullptr ||
                 cloud.sh == nullptr)) {
    throw Failure{SPLAT_ERR_INVALID, "GaussianCloud: inconsistent array sizes"};
  }
  if (opt.position_noise != 0.f) throw Failure{SPLAT_ERR_UNSUPPORTED, "position noise has no kernel in this library"};
  if (opt.mip_filter_2d != 0) throw Failure{SPLAT_ERR_UNSUPPORTED, "the Mip 2D filter has no kernel in this library"};
  if (opt.pose_gradients != 0) throw Failure{SPLAT_ERR_UNSUPPORTED, "pose gradients have no kernel in this library"};
  if (opt.sh_storage < 0 || opt.sh_storage > 2 || opt.state_storage < 0 || opt.state_storage > 1 || opt.sort_form < 0 ||
      opt.sort_form > 1) {
    throw Failure{SPLAT_ERR_INVALID, "unknown storage or sort form"};
  }
  n = (uint32_t)cloud.count;
  shDegree = cloud.sh_degree;
  activeDegree = shDegree;
  shCoeffs = (shDegree + 1) * (shDegree + 1);
  shStore = (ShStore)opt.sh_storage;
  stateStore = (StateStore)opt.state_storage;
  // The reference picks fixed point on GPUs without float atomics (trainer.cpp:181); a B200 has them.
  fixedPoint = opt.force_fixed_point != 0;
  blendLists = opt.blend_lists != 0;
  if (blendLists && fixedPoint) throw Failure{SPLAT_ERR_UNSUPPORTED, "blend lists keep float sums: no fixed-point form"};
  oneSort = opt.sort_form == SPLAT_SORT_TILE_DEPTH_64;
  exactMath = opt.exact_math != 0;
  useGraph = opt.use_graph != 0;
  digitBits = opt.digit_bits == 0 ? 8 : opt.digit_bits;
  if (digitBits < 6 || digitBits > 8) throw Failure{SPLAT_ERR_INVALID, "digit_bits must be 6, 7 or 8"};
  forwardPixels = opt.forward_pixels_per_thread == 0 ? 1 : opt.forward_pixels_per_thread;
  backwardPixels = opt.backward_pixels_per_thread == 0 ? 2 : opt.backward_pixels_per_thread;
  if (forwardPixels != 1 && forwardPixels != 2)
    throw Failure{SPLAT_ERR_INVALID, "forward_pixels_per_thread must be 1 or 2"};
  if (backwardPixels != 1 && backwardPixels != 2)
    throw Failure{SPLAT_ERR_INVALID, "backward_pixels_per_thread must be 1 or 2"};
  tileSize = opt.tile_size == 0 ? 16 : opt.tile_size;
  if (tileSize != 16 && tileSize != 32) throw Failure{SPLAT_ERR_INVALID, "tile_size must be 16 or 32"};
  batchDepth = opt.batch_depth == 0 ? 128 : opt.batch_depth;
  if (batchDepth != 128 && batchDepth != 256) throw Failure{SPLAT_ERR_INVALID, "batch_depth must be 128 or 256"};
  persistent = opt.persistent_raster != 0;
  groupedSums = opt.grouped_backward != 0;
  // The step's own stream at the greatest priority, the second stream (the
  // clears and the tile count beside the depth sort) at the least: the sort's
  // passes, one after another, are the longer chain.
  int leastPriority = 0, greatestPriority = 0;
  SB_CUDA(cudaDeviceGetStreamPriorityRange(&leastPriority, &greatestPriority));
  SB_CUDA(cudaStreamCreateWithPriority(&stream, cudaStreamNonBlocking, greatestPriority));
  SB_CUDA(cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, leastPriority));
  SB_CUDA(cudaEventCreateWithFlags(&forkEvent, cudaEventDisableTiming));
  SB_CUDA(cudaEventCreateWithFlags(&joinEvent, cudaEventDisableTiming));
  SB_CUDA(cudaEventCreateWithFlags(&countForkEvent, cudaEventDisableTiming));
  SB_CUDA(cudaEventCreateWithFlags(&countEvent, cudaEventDisableTiming));
  SB_CUDA(cudaEventCreateWithFlags(&orderForkEvent, cudaEventDisableTiming));
  SB_CUDA(cudaEventCreateWithFlags(&orderEvent, cudaEventDisableTiming));
  SB_CUDA(cudaEventCreateWithFlags(&totalsForkEvent, cudaEventDisableTiming));
  SB_CUDA(cudaEventCreateWithFlags(&totalsEvent, cudaEventDisableTiming));
  SB_CUDA(cudaStreamCreateWithFlags(&copyStream, cudaStreamNonBlocking));
  // The persistent launches' tile counters, made here: a step may be recorded
  // into a graph, where nothing may be allocated.
  workCounters.ensure(16);
  SB_CUDA(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
  SB_CUDA(cudaEventCreateWithFlags(&consumed, cudaEventDisableTiming));
  for (auto &e : events) SB_CUDA(cudaEventCreate(&e));

  const size_t nn = n;
  planeStride = (uint32_t)(((nn + kPlaneAlign - 1) / kPlaneAlign) * kPlaneAlign);
  const size_t ps = planeStride;
  positions.ensure(nn * 12);
  scales.ensure(nn * 12);
  rotations.ensure(nn * 16);
  opacities.ensure(nn * 4);
  shDc.ensure(ps * 12);
  const size_t rest = ps * sh_rest_stride(shCoeffs, shStore);
  shRest.ensure(std::max<size_t>(rest * (shStore == ShStore::F32 ? 4 : 2), 4));
  SB_CUDA(cudaMemset(shDc.get(), 0, shDc.bytes()));
  SB_CUDA(cudaMemset(shRest.get(), 0, shRest.bytes()));
  if (!upload) {
    for (DeviceBuffer *b : {&positions, &scales, &rotations, &opacities}) SB_CUDA(cudaMemset(b->get(), 0, b->bytes()));
  } else {
    DeviceBuffer *to[6] = {&positions, &scales, &rotations, &opacities, &shDc, &shRest};
    upload_cloud(cloud, shCoeffs, shStore, planeStride, to);
  }
  const size_t groupCounts[5] = {nn * 3, nn * 3, nn * 4, nn, ps * sh_state_stride(shCoeffs)};
  for (int g = 0; g < 5; ++g) {
    const size_t bytes = groupCounts[g] * (stateStore == StateStore::F32 ? 8 : 4);
    state[g].ensure(bytes);
    SB_CUDA(cudaMemset(state[g].get(), 0, bytes));
  }
  // Geometry gradients pass through these on their way to Adam; the SH ones
  // are made only when compute_gradients() stores them (fill_chain_args).
  for (int g = 0; g < 4; ++g) grads[g].ensure(groupCounts[g] * 4);
  densifyStats.ensure(nn * kStatStride * 4);
  SB_CUDA(cudaMemset(densifyStats.get(), 0, nn * kStatStride * 4));
  dStep.ensure(kStepBytes);
  hStep.ensure(kStepBytes);
  std::memset(hStep.get(), 0, kStepBytes);
  hReadback.ensure(sizeof(StepReadback));
  // The read-back's address on the device side of the pinned block (null
  // where the block is not mapped: the read-back is then copied).
  if (cudaHostGetDevicePointer(&hReadbackDevice, hReadback.get(), 0) != cudaSuccess) {
    cudaGetLastError();
    hReadbackDevice = nullptr;
  }
}

Trainer::~Trainer() {
  if (stream != nullptr) cudaStreamSynchronize(stream);
  clear_graphs();
  for (auto &e : events)
    if (e != nullptr) cudaEventDestroy(e);
  if (forkEvent != nullptr) cudaEventDestroy(forkEvent);
  if (joinEvent != nullptr) cudaEventDestroy(joinEvent);
  if (countForkEvent != nullptr) cudaEventDestroy(countForkEvent);
  if (countEvent != nullptr) cudaEventDestroy(countEvent);
  for (cudaEvent_t e : {orderForkEvent, orderEvent, totalsForkEvent, totalsEvent})
    if (e != nullptr) cudaEventDestroy(e);
  if (side != nullptr) cudaStreamDestroy(side);
  if (copyStream != nullptr) {
    cudaStreamSynchronize(copyStream);
    cudaStreamDestroy(copyStream);
  }
  if (copied != nullptr) cudaEventDestroy(copied);
  if (consumed != nullptr) cudaEventDestroy(consumed);
  if (stream != nullptr) cudaStreamDestroy(stream);
}

void Trainer::clear_graphs() {
  for (auto &g : graphs)
    if (g.second.exec != nullptr) cudaGraphExecDestroy(g.second.exec);
  graphs.clear();
}

Params Trainer::params() const {
  Params p;
  p.positions = positions.get<float>();
  p.scales = scales.get<float>();
  p.rotations = rotations.get<float>();
  p.opacities = opacities.get<float>();
  p.shDc = shDc.get<float>();
  p.shRest = shRest.get();
  p.shStore = shStore;
  p.n = n;
  p.planeStride = planeStride;
  p.restStride = sh_rest_stride(shCoeffs, shStore);
  p.shDegree = shDegree;
  p.shCoeffs = shCoeffs;
  return p;
}

OptimState Trainer::optim_state() {
  OptimState s;
  for (int g = 0; g < 5; ++g) s.state[g] = state[g].get();
  s.store = stateStore;
  return s;
}

uint64_t Trainer::bytes_per_gaussian() const {
  const uint64_t rest = 3ull * (shCoeffs - 1) * (shStore == ShStore::F32 ? 4 : 2);
  const uint64_t floats = 3 + 3 + 4 + 1 + 3ull * shCoeffs;
  const uint64_t params = (3 + 3 + 4 + 1 + 3) * 4 + rest;
  const uint64_t optimiser = floats * (stateStore == StateStore::F32 ? 8 : 4);
  // Per view: splat 48, reach 4, keys/values and their copies 16, offsets,
  // reached-tile masks and counts 12, raw sums 64, colour gradient and
  // direction for the SH step 32.
  const uint64_t perView = sizeof(Splat) + 4 + 16 + 12 + kRawStride * 4 + 32;
  // Geometry gradients between the chain rule and Adam: 11 floats.
  return params + optimiser + 11 * 4 + kStatStride * 4 + perView * (uint64_t)std::max(viewSlots, 1);
}

uint64_t Trainer::entry_bytes(uint64_t entries) const {
  // Keys and values with their copies, plus the sort's look-back words.
  return entries * ((oneSort ? 16 : 8) + 8) + entries / 16;
}

// Trainer::score_view (trainer.cpp:521-532): a statistics pass over the view
// with the high-error pixels marked and the target's edge weights kept, then
// the marked-pixel count, that count times the view's loss and the edge score
// added to each Gaussian's statistics, in pixels times pixelWeight.
void Trainer::score_view(const splat_camera *camera, const uint8_t *targetImage, size_t bytes, float share, float pixelWeight,
                         splat_step_stats *stats, bool deviceTarget) {
  if (!(share > 0.0f) || !std::isfinite(share)) throw Failure{SPLAT_ERR_INVALID, "error_share must be above 0"};
  if (!std::isfinite(pixelWeight)) throw Failure{SPLAT_ERR_INVALID, "pixel_weight must be finite"};
  if (blendLists) throw Failure{SPLAT_ERR_UNSUPPORTED, "scoring a view does not run with blend lists"};
  splat_step_stats own{};
  const uint8_t *targets[1] = {targetImage};
  const size_t sizes[1] = {bytes};
  scoreShare = share;
  try {
    run(camera, targets, sizes, 1, ChainMode::Statistics, nullptr, true, &own, deviceTarget);
  } catch (...) {
    scoreShare = 0.0f;
    throw;
  }
  scoreShare = 0.0f;
  // The raw sums are over 3 pixels of the image, like the derivatives.
  const float toPixels = 3.0f * (float)camera->width * (float)camera->height * pixelWeight;
  launch_score(raw.get(), fixedPoint, views.v[0].fixedScale, n, toPixels, (float)own.loss, densifyStats.get<float>(), stream);
  SB_CUDA(cudaStreamSynchronize(stream));
  if (stats != nullptr) *stats = own;
}

uint64_t Trainer::gpu_bytes() const {
  uint64_t total = bytes_per_gaussian() * n;
  for (const DeviceBuffer *b : {&image, &stops, &adjoint, &fields, &target, &targetNext, &ranges, &partials, &entryKeys, &entryValues,
                                &tmpEntryKeys, &tmpEntryValues, &sortScratchDepth, &sortScratchEntries, &scanScratch,
                                &listCounts, &listOffsets, &listPool, &listScratch, &listCounters})
    total += b->bytes();
  return total;
}

// ---------------------------------------------------------------- views

void Trainer::set_views(const splat_camera *cameras, int count) {
  if (count < 1 || count > kMaxViews) throw Failure{SPLAT_ERR_INVALID, "between 1 and 8 views per step"};
  ViewSet vs{};
  vs.count = count;
  const int tile = raster_tile();
  int tileBase = 0, lossTileBase = 0;
  long long pixelBase = 0;
  for (int k = 0; k < count; ++k) {
    const splat_camera &c = cameras[k];
    if (c.width <= 0 || c.height <= 0) throw Failure{SPLAT_ERR_INVALID, "bad image size"};
    ViewParams &v = vs.v[k];
    for (int r = 0; r < 3; ++r) {
      for (int col = 0; col < 3; ++col) v.R[r * 3 + col] = c.view[col * 4 + r];
      v.T[r] = c.view[12 + r];
    }
    for (int a = 0; a < 3; ++a) v.pos[a] = c.position[a];
    v.nearPlane = opt.near_plane;
    v.fx = c.fx;
    v.fy = c.fy;
    v.cx = c.cx;
    v.cy = c.cy;
    v.widthF = (float)c.width;
    v.heightF = (float)c.height;
    v.tanX = 0.5f * (float)c.width / c.fx;
    v.tanY = 0.5f * (float)c.height / c.fy;
    v.width = c.width;
    v.height = c.height;
    v.gridW = (int)div_up((uint32_t)c.width, (uint32_t)tile);
    v.gridH = (int)div_up((uint32_t)c.height, (uint32_t)tile);
    v.tileBase = tileBase;
    v.tileCount = v.gridW * v.gridH;
    v.lossGridW = (int)div_up((uint32_t)c.width, kLossTileW);
    v.lossGridH = (int)div_up((uint32_t)c.height, kLossTileH);
    v.lossTileBase = lossTileBase;
    v.lossTileCount = v.lossGridW * v.lossGridH;
    lossTileBase += v.lossTileCount;
    v.pixelBase = pixelBase;
    v.perPixel = 1.0f / (3.0f * (float)c.width * (float)c.height);
    v.fixedScale = 3.0f * (float)c.width * (float)c.height * 64.0f;
    v.activeDegree = activeDegree;
    v.activeCoeffs = (activeDegree + 1) * (activeDegree + 1);
    tileBase += v.tileCount;
    pixelBase += (long long)c.width * c.height;
  }
  // The depth-sorted form sorts entries by as many bits as the tile count needs.
  if (!oneSort && tileBase > (1 << 24)) throw Failure{SPLAT_ERR_INVALID, "too many tiles for one step"};
  vs.totalTiles = tileBase;
  vs.totalPixels = pixelBase;
  vs.tileSize = tile;
  vs.totalLossTiles = lossTileBase;
  views = vs;
}

void Trainer::ensure_view_buffers() {
  const int count = views.count;
  if (count > viewSlots) {
    const size_t items = (size_t)n * count;
    splats.ensure(items * sizeof(Splat));
    reach.ensure(items * 4);
    depthKeys.ensure(items * 4);
    values.ensure(items * 4);
    tmpKeys.ensure(items * 4);
    tmpValues.ensure(items * 4);
    offsets.ensure(items * 12); // entry offsets, the reached-tile masks, then (depth-sorted form) the counts per splat
    raw.ensure(items * kRawStride * 4);
    shGrad.ensure(items * 32);
    SB_CUDA(cudaMemset(raw.get(), 0, items * kRawStride * 4));
    viewSlots = count;
    clear_graphs();
  }
  const size_t pixels = (size_t)views.totalPixels, tiles = (size_t)views.totalTiles;
  const size_t before = image.bytes() + target.bytes() + ranges.bytes();
  image.ensure(pixels * 16);
  stops.ensure(pixels * 4);
  adjoint.ensure(pixels * 16);
  fields.ensure(pixels * 36);
  target.ensure(pixels * 4);
  // The tile ranges, then per tile the compositing's work record and the
  // backward's tile order (launch_tile_order).
  ranges.ensure(tiles * 16);
  partials.ensure((size_t)views.totalLossTiles * 8);
  if (image.bytes() + target.bytes() + ranges.bytes() != before) clear_graphs();
  if (blendLists) {
    listCounts.ensure(pixels * 4);
    listOffsets.ensure(pixels * 4);
    listScratch.ensure(bin_scan_scratch_bytes((uint32_t)pixels));
    listCounters.ensure(16);
  }
  const size_t items = (size_t)n * (oneSort ? count : 1);
  if (scanScratch.bytes() < bin_scan_scratch_bytes((uint32_t)items)) {
    scanScratch.ensure(bin_scan_scratch_bytes((uint32_t)items));
    clear_graphs();
  }
  if (!oneSort) {
    const size_t need = sort_scratch_bytes(n, 4, 32, digitBits);
    if (sortScratchDepth.bytes() < need) {
      sortScratchDepth.ensure(need);
      clear_graphs();
    }
  }
}

void Trainer::ensure_entries(uint32_t total) {
  if (total <= entryCapacity && entryKeys.get() != nullptr) return;
  const uint64_t others = gpu_bytes() - (entryKeys.bytes() + entryValues.bytes() + tmpEntryKeys.bytes() +
                                         tmpEntryValues.bytes() + sortScratchEntries.bytes());
  if (others + entry_bytes(total) > opt.memory_budget) {
    throw Failure{SPLAT_ERR_BUDGET, std::to_string(total) + " tile entries do not fit the memory budget"};
  }
  // Room to grow as splats change, as far as the budget lets it (trainer.cpp:361-364).
  const uint64_t wanted = (uint64_t)total + total / 2 + 1024;
  const uint64_t affordable =
      opt.memory_budget == ~0ull ? wanted : (opt.memory_budget - others) / std::max<uint64_t>(entry_bytes(1), 1);
  const uint64_t cap = std::max<uint64_t>(std::min(wanted, affordable), total);
  if (cap > 0xFFFFFFF0ull) throw Failure{SPLAT_ERR_BUDGET, "more tile entries than 32-bit indices hold"};
  const size_t keyBytes = oneSort ? 8 : 4;
  entryKeys.release();
  entryValues.release();
  tmpEntryKeys.release();
  tmpEntryValues.release();
  sortScratchEntries.release();
  entryKeys.ensure(cap * keyBytes);
  entryValues.ensure(cap * 4);
  tmpEntryKeys.ensure(cap * keyBytes);
  tmpEntryValues.ensure(cap * 4);
  const uint32_t bits = oneSort ? 32 + bits_for((uint32_t)views.totalTiles) : bits_for((uint32_t)views.totalTiles);
  size_t scratch = 0;
  for (int d = 6; d <= 8; ++d) scratch = std::max(scratch, sort_scratch_bytes(cap, (int)keyBytes, std::max<uint32_t>(bits, 32 + 24), d));
  sortScratchEntries.ensure(scratch);
  entryCapacity = (uint32_t)cap;
  entryScratchClear = false;
  clear_graphs();
}

// Copies the target named for the next step into the second pinned buffer
// and from there, on copyStream, into targetNext; run() calls it once the
// step's work is queued, so both copies overlap the step.
void Trainer::stage_prefetch() {
  if (pendingPrefetch == nullptr) return;
  prefetch(pendingPrefetch, pendingPrefetchBytes);
  pendingPrefetch = nullptr;
}

void Trainer::prefetch(const uint8_t *next, size_t bytes) {
  // The last copy out of the pinned buffer has ended, and the step that took
  // targetNext has copied it away, before either is written again.
  SB_CUDA(cudaEventSynchronize(copied));
  SB_CUDA(cudaStreamWaitEvent(copyStream, consumed, 0));
  stagingNext.ensure(bytes);
  // The host copy runs while the GPU works on this step; split over four
  // threads it stays inside the step on a slow host.
  uint8_t *dst = stagingNext.get<uint8_t>();
  if (bytes >= (1u << 20)) {
    const size_t quarter = (bytes / 4 + 63) & ~size_t{63};
    std::thread helpers[3];
    for (int k = 1; k < 4; ++k) {
      const size_t from = std::min(bytes, (size_t)k * quarter), to = std::min(bytes, (size_t)(k + 1) * quarter);
      helpers[k - 1] = std::thread([=] { std::memcpy(dst + from, next + from, to - from); });
    }
    std::memcpy(dst, next, std::min(bytes, quarter));
    for (std::thread &h : helpers) h.join();
  } else {
    std::memcpy(dst, next, bytes);
  }
  targetNext.ensure(bytes);
  SB_CUDA(cudaMemcpyAsync(targetNext.get(), stagingNext.get(), bytes, cudaMemcpyHostToDevice, copyStream));
  SB_CUDA(cudaEventRecord(copied, copyStream));
  prefetched = next;
  prefetchedBytes = bytes;
}

// Whether this step's single target is the one prefetched: then it is (or
// soon will be) in targetNext.
bool Trainer::take_prefetched(const uint8_t *const *targets, const size_t *bytes, int count) {
  if (count != 1 || prefetched == nullptr || prefetched != targets[0] || prefetchedBytes != bytes[0]) return false;
  const size_t want = (size_t)views.v[0].width * views.v[0].height * 4;
  if (bytes[0] != want) throw Failure{SPLAT_ERR_INVALID, "the target image does not match the camera"};
  prefetched = nullptr;
  return true;
}

void Trainer::upload_targets(const uint8_t *const *targets, const size_t *bytes, int count) {
  size_t total = 0;
  for (int k = 0; k < count; ++k) {
    const size_t want = (size_t)views.v[k].width * views.v[k].height * 4;
    if (bytes[k] != want || targets[k] == nullptr) throw Failure{SPLAT_ERR_INVALID, "the target image does not match the camera"};
    total += want;
  }
  staging.ensure(total);
  size_t off = 0;
  for (int k = 0; k < count; ++k) {
    std::memcpy(staging.get<uint8_t>() + off, targets[k], bytes[k]);
    off += bytes[k];
  }
}

// ---------------------------------------------------------------- recording

// Per-stage timing: a pair of events around each stage's kernels, so host
// waits and small copies between stages are not counted.
void Trainer::begin(int stage) {
  if (timing) SB_CUDA(cudaEventRecord(events[2 * stage], stream));
}
void Trainer::end(int stage) {
  if (timing) SB_CUDA(cudaEventRecord(events[2 * stage + 1], stream));
}

// The entry sort's key bits and digit width for the current views and form.
int Trainer::entry_sort_bits() const {
  return oneSort ? 32 + (int)bits_for((uint32_t)views.totalTiles) : (int)bits_for((uint32_t)views.totalTiles);
}

// The rasterizer's tile edge: the option's where both kernels take two
// pixels per thread with float sums (the kernels built for other edges),
// else the reference's 16.
int Trainer::raster_tile() const {
  return forwardPixels == 2 && backwardPixels == 2 && !fixedPoint && !blendLists ? tileSize : kTileSize;
}

RasterConfig Trainer::raster_config() {
  RasterConfig cfg;
  cfg.exactMath = exactMath ? 1 : 0;
  cfg.forwardPixels = forwardPixels;
  cfg.backwardPixels = backwardPixels;
  for (int c = 0; c < 3; ++c) cfg.background[c] = opt.background[c];
  cfg.tile = views.tileSize;
  cfg.batch = batchDepth;
  cfg.twoPhase = groupedSums;
  if (persistent) {
    if (forwardPixels == 2) cfg.workForward = workCounters.get<uint32_t>();
    if (backwardPixels == 2 && !fixedPoint) cfg.workBackward = workCounters.get<uint32_t>() + 1;
  }
  return cfg;
}

void Trainer::record_prepare(bool backward) {
  const Params p = params();
  // The views, the chain rule's arguments (here at the start, so that no
  // copy sits between the backward pass and the chain rule) and a cleared
  // read-back, in one copy.
  SB_CUDA(cudaMemcpyAsync(dStep.get(), hStep.get(), kStepBytes, cudaMemcpyHostToDevice, stream));
  StepReadback *rb = d_readback();
  uint32_t *counters = rb->counters, *error = &rb->error;
  // What the step clears, cleared on the second stream while the projection
  // runs: the backward pass's sums (not for a render, which keeps the last
  // ones for apply_gradients), the tile ranges and both sorts' scratch. The
  // kernels between the projection and the chain rule then follow one
  // another with nothing in between.
  SB_CUDA(cudaEventRecord(forkEvent, stream));
  SB_CUDA(cudaStreamWaitEvent(side, forkEvent, 0));
  if (backward) SB_CUDA(cudaMemsetAsync(raw.get(), 0, (size_t)n * views.count * kRawStride * 4, side));
  SB_CUDA(cudaMemsetAsync(ranges.get(), 0, (size_t)views.totalTiles * 8, side));
  if (persistent) SB_CUDA(cudaMemsetAsync(workCounters.get(), 0, 16, side));
  if (!oneSort) SB_CUDA(cudaMemsetAsync(sortScratchDepth.get(), 0, sort_scratch_bytes(n, 4, 32, digitBits), side));
  entryScratchClear = entryKeys.get() != nullptr;
  if (entryScratchClear) {
    const int bits = entry_sort_bits();
    SB_CUDA(cudaMemsetAsync(sortScratchEntries.get(), 0,
                            sort_scratch_bytes(entryCapacity, oneSort ? 8 : 4, bits, entry_digits(bits, digitBits)), side));
  }
  SB_CUDA(cudaEventRecord(joinEvent, side));
  begin(0);
  launch_preprocess(p, views, d_views(), splats.get<Splat>(), reach.get<float>(), depthKeys.get<uint32_t>(),
                    oneSort ? nullptr : values.get<uint32_t>(), stream, error);
  end(0);
  const uint32_t items = oneSort ? n * (uint32_t)views.count : n;
  uint32_t *offs = offsets.get<uint32_t>(), *masks = offs + items, *countsBySplat = offs + 2 * (size_t)items;
  // Depth-sorted form: the tiles of each splat are counted per splat index on
  // the second stream while the depth sort runs, and the scan gathers the
  // counts in depth order; the two latency-bound passes overlap. With stage
  // timing on, they run one after the other so that each is timed alone.
  countOverlap = !oneSort && !timing;
  if (countOverlap) {
    SB_CUDA(cudaEventRecord(countForkEvent, stream));
    SB_CUDA(cudaStreamWaitEvent(side, countForkEvent, 0));
    SB_CUDA(cudaMemsetAsync(scanScratch.get(), 0, bin_scan_scratch_bytes(items), side));
    // No keys: the depth sort permutes them in place meanwhile.
    // Three blocks per SM walk the splats in chunks, leaving the sort's
    // passes (one to two blocks per SM each) room beside them: measured at
    // 1M splats, 1.509 ms a step against 1.519 with one block per chunk of
    // splats and 1.544 with two per SM.
    launch_bin_count(splats.get<Splat>(), reach.get<float>(), nullptr, nullptr, n, n, views, d_views(),
                     countsBySplat, masks, counters, side, 3u);
    SB_CUDA(cudaEventRecord(countEvent, side));
  }
  SB_CUDA(cudaStreamWaitEvent(stream, joinEvent, 0));
  begin(1);
  if (!oneSort) {
    depthInTmp = sort_pairs_u32(depthKeys.get<uint32_t>(), values.get<uint32_t>(), tmpKeys.get<uint32_t>(),
                                tmpValues.get<uint32_t>(), n, n, nullptr, 0, 32, digitBits, sortScratchDepth.get(), error,
                                stream, false) == 1;
  }
  end(1);
  begin(2);
  const uint32_t *itemKeys = oneSort ? depthKeys.get<uint32_t>() : (depthInTmp ? tmpKeys.get<uint32_t>() : depthKeys.get<uint32_t>());
  const uint32_t *itemSplat = oneSort ? nullptr : (depthInTmp ? tmpValues.get<uint32_t>() : values.get<uint32_t>());
  if (countOverlap) {
    SB_CUDA(cudaStreamWaitEvent(stream, countEvent, 0));
    launch_offsets_scan(items, countsBySplat, itemSplat, offs, counters, entryCapacity, scanScratch.get(), error, stream, false);
  } else {
    launch_bin_count_scan(splats.get<Splat>(), reach.get<float>(), itemKeys, itemSplat, items, n, views, d_views(), offs,
                          masks, counters, entryCapacity, scanScratch.get(), error, stream);
  }
  end(2);
}

void Trainer::record_forward() {
  StepReadback *rb = d_readback();
  uint32_t *counters = rb->counters, *error = &rb->error;
  const uint32_t *itemKeys = oneSort ? depthKeys.get<uint32_t>() : (depthInTmp ? tmpKeys.get<uint32_t>() : depthKeys.get<uint32_t>());
  const uint32_t *itemSplat = oneSort ? nullptr : (depthInTmp ? tmpValues.get<uint32_t>() : values.get<uint32_t>());
  const uint32_t items = oneSort ? n * (uint32_t)views.count : n;
  begin(3);
  launch_bin_emit(splats.get<Splat>(), reach.get<float>(), itemKeys, itemSplat, items, n, views, d_views(),
                  offsets.get<uint32_t>(), offsets.get<uint32_t>() + items, countOverlap, entryCapacity,
                  oneSort ? nullptr : entryKeys.get<uint32_t>(),
                  oneSort ? entryKeys.get<unsigned long long>() : nullptr, entryValues.get<uint32_t>(), error, stream);
  // The scratch was cleared with the step's other clears unless the entry
  // buffers were (re)made after them.
  const int bits = entry_sort_bits();
  if (oneSort) {
    entriesInTmp = sort_pairs_u64(entryKeys.get<unsigned long long>(), entryValues.get<uint32_t>(),
                                  tmpEntryKeys.get<unsigned long long>(), tmpEntryValues.get<uint32_t>(), entryCapacity, 0,
                                  &counters[2], 0, bits, entry_digits(bits, digitBits), sortScratchEntries.get(), error,
                                  stream, !entryScratchClear) == 1;
  } else {
    entriesInTmp = sort_pairs_u32(entryKeys.get<uint32_t>(), entryValues.get<uint32_t>(), tmpEntryKeys.get<uint32_t>(),
                                  tmpEntryValues.get<uint32_t>(), entryCapacity, 0, &counters[2], 0, bits,
                                  entry_digits(bits, digitBits), sortScratchEntries.get(), error, stream,
                                  !entryScratchClear) == 1;
  }
  const void *keys = entriesInTmp ? tmpEntryKeys.get() : entryKeys.get();
  launch_tile_ranges(oneSort ? nullptr : static_cast<const uint32_t *>(keys),
                     oneSort ? static_cast<const unsigned long long *>(keys) : nullptr, &counters[2], entryCapacity,
                     (uint32_t)views.totalTiles, ranges.get<uint2>(), error, stream);
  end(3);
  const RasterConfig cfg = raster_config();
  const uint32_t *vals = entriesInTmp ? tmpEntryValues.get<uint32_t>() : entryValues.get<uint32_t>();
  begin(4);
  if (blendLists) {
    // Store everything: count each pixel's blended splats, scan the counts
    // into list offsets, read the total back, then composite again recording
    // the lists.
    BlendLists lists;
    lists.counts = listCounts.get<uint32_t>();
    launch_forward(splats.get<Splat>(), vals, ranges.get<uint2>(), views, d_views(), cfg, image.get<float4>(),
                   stops.get<uint32_t>(), n * (uint32_t)views.count, error, stream, 1, lists);
    const size_t pixels = (size_t)views.totalPixels;
    SB_CUDA(cudaMemcpyAsync(listOffsets.get(), listCounts.get(), pixels * 4, cudaMemcpyDeviceToDevice, stream));
    launch_exclusive_scan((uint32_t)pixels, listOffsets.get<uint32_t>(), listCounters.get<uint32_t>(), listScratch.get(), error,
                          stream);
    uint32_t counters[4] = {0, 0, 0, 0};
    SB_CUDA(cudaMemcpyAsync(counters, listCounters.get(), sizeof(counters), cudaMemcpyDeviceToHost, stream));
    SB_CUDA(cudaStreamSynchronize(stream));
    const size_t pool = (size_t)counters[1] * sizeof(uint2);
    if (listPool.bytes() < pool) {
      listPool.release();
      listPool.ensure(pool + pool / 2 + 4096);
    }
    lists.offsets = listOffsets.get<uint32_t>();
    lists.pool = listPool.get<uint2>();
    launch_forward(splats.get<Splat>(), vals, ranges.get<uint2>(), views, d_views(), cfg, image.get<float4>(),
                   stops.get<uint32_t>(), n * (uint32_t)views.count, error, stream, 2, lists);
  } else {
    RasterConfig c = cfg;
    // The two-pixel compositing records what the backward pass will walk in
    // each tile, for the backward's tile order. (Its own tiles stay in raster
    // order: measured, ordering them by the length of their entry ranges
    // made the compositing no faster; how far a tile's pixels walk before
    // they stop is not known before it runs.)
    if (forwardPixels == 2 && backwardPixels == 2 && !fixedPoint)
      c.tileWork = reinterpret_cast<uint32_t *>(ranges.get<uint2>() + views.totalTiles);
    launch_forward(splats.get<Splat>(), vals, ranges.get<uint2>(), views, d_views(), c, image.get<float4>(),
                   stops.get<uint32_t>(), n * (uint32_t)views.count, error, stream);
    if (backwardPixels == 2 && !fixedPoint) {
      // The backward's tiles, heaviest first (by the entries each walks, as
      // the two-pixel compositing recorded them, else by the length of their
      // entry ranges), ordered on the second stream while the loss runs.
      const uint32_t tiles = (uint32_t)views.totalTiles;
      uint32_t *extra = reinterpret_cast<uint32_t *>(ranges.get<uint2>() + tiles);
      cudaStream_t where = stream;
      if (capturing) {
        SB_CUDA(cudaEventRecord(orderForkEvent, stream));
        SB_CUDA(cudaStreamWaitEvent(side, orderForkEvent, 0));
        where = side;
      }
      launch_tile_order(ranges.get<uint2>(), forwardPixels == 2 ? extra : nullptr, tiles, extra + tiles, where);
      if (capturing) SB_CUDA(cudaEventRecord(orderEvent, side));
      orderPending = true;
      orderForked = capturing;
    }
  }
  end(4);
}

void Trainer::record_backward_and_chain(ChainMode mode, bool statistics) {
  StepReadback *rb = d_readback();
  uint32_t *error = &rb->error;
  begin(5);
  launch_ssim(image.get<float4>(), target.get<uint32_t>(), views, d_views(), fields.get<float4>(),
              partials.get<float2>(), stream);
  LossScoring scoring;
  if (scoreShare > 0.0f) {
    scoreEdge.ensure((size_t)views.totalPixels * 4);
    scoreMax.ensure(4);
    SB_CUDA(cudaMemsetAsync(scoreMax.get(), 0, 4, stream));
    scoring.edge = scoreEdge.get<float>();
    scoring.errorMax = scoreMax.get<uint32_t>();
  }
  launch_loss(image.get<float4>(), target.get<uint32_t>(), fields.get<float4>(), views, d_views(), opt.lambda_ssim,
              adjoint.get<float4>(), partials.get<float2>(), stream, scoring);
  if (scoreShare > 0.0f)
    launch_error_mask(adjoint.get<float4>(), (uint32_t)views.totalPixels, scoreMax.get<uint32_t>(), scoreShare, stream);
  // The FP64 totals; in a captured step on the second stream beside the
  // backward pass (only the step's read-back needs them).
  totalsPending = capturing;
  if (totalsPending) {
    SB_CUDA(cudaEventRecord(totalsForkEvent, stream));
    SB_CUDA(cudaStreamWaitEvent(side, totalsForkEvent, 0));
  }
  launch_loss_totals(partials.get<float2>(), views, d_views(), &rb->totals, totalsPending ? side : stream);
  if (totalsPending) SB_CUDA(cudaEventRecord(totalsEvent, side));
  end(5);
  const RasterConfig cfg = raster_config();
  const uint32_t *vals = entriesInTmp ? tmpEntryValues.get<uint32_t>() : entryValues.get<uint32_t>();
  begin(6);
  if (blendLists) {
    BlendLists lists;
    lists.counts = listCounts.get<uint32_t>();
    lists.offsets = listOffsets.get<uint32_t>();
    lists.pool = listPool.get<uint2>();
    launch_backward_lists(splats.get<Splat>(), vals, ranges.get<uint2>(), views, d_views(), cfg, image.get<float4>(),
                          adjoint.get<float4>(), stops.get<uint32_t>(), lists, raw.get<float>(), n * (uint32_t)views.count,
                          error, stream);
  } else {
    RasterConfig c = cfg;
    if (orderPending) {
      if (orderForked) SB_CUDA(cudaStreamWaitEvent(stream, orderEvent, 0));
      c.orderBackward = reinterpret_cast<uint32_t *>(ranges.get<uint2>() + views.totalTiles) + views.totalTiles;
      orderPending = orderForked = false;
    }
    launch_backward(splats.get<Splat>(), vals, ranges.get<uint2>(), views, d_views(), c, image.get<float4>(),
                    adjoint.get<float4>(), stops.get<uint32_t>(), fixedPoint, raw.get(), n * (uint32_t)views.count, error,
                    stream, scoreShare > 0.0f ? scoreEdge.get<float>() : nullptr);
  }
  end(6);
  ChainArgs args{};
  std::memcpy(&args, h_args(), sizeof(ChainArgs));
  (void)mode;
  (void)statistics;
  OptimState st = optim_state();
  // The geometry gradients always pass through these buffers on their way to
  // Adam; compute_gradients() also keeps the SH ones there.
  GradientsOut g{};
  for (int k = 0; k < 5; ++k) g.g[k] = grads[k].get<float>();
  const GradientsOut *gp = &g;
  begin(7);
  launch_chain(params(), views, d_views(), raw.get(), splats.get<Splat>(), args, d_args(), st, gp,
               shGrad.get<float4>(), densifyStats.get<float>(), error, stream);
  end(7);
  if (totalsPending) {
    SB_CUDA(cudaStreamWaitEvent(stream, totalsEvent, 0));
    totalsPending = false;
  }
}

void Trainer::record_readback() {
  static_assert(sizeof(StepReadback) % 4 == 0, "the read-back goes as words");
  if (hReadbackDevice == nullptr) {
    SB_CUDA(cudaMemcpyAsync(hReadback.get(), d_readback(), sizeof(StepReadback), cudaMemcpyDeviceToHost, stream));
    return;
  }
  launch_chained(k_readback, dim3(1), dim3(64), 0, stream, reinterpret_cast<const uint32_t *>(d_readback()),
                 static_cast<uint32_t *>(hReadbackDevice), (uint32_t)(sizeof(StepReadback) / 4));
  SB_CUDA(cudaGetLastError());
}

void Trainer::fill_chain_args(ChainMode mode, bool statistics, const splat_learning_rates *rates) {
  ChainArgs a{};
  a.mode = mode;
  a.statistics = statistics;
  a.selective = opt.selective_adam != 0;
  a.fixedPoint = fixedPoint;
  a.splitStep = opt.split_step != 0;
  a.beta1 = 0.9f;
  a.beta2 = 0.999f;
  a.epsilon = 1e-15f;
  a.opacityReg = opt.opacity_reg / (float)n;
  a.scaleReg = opt.scale_reg / (float)n;
  if (mode == ChainMode::Step) {
    ++adamStep;
    a.rates[0] = rates->position;
    a.rates[1] = rates->scale;
    a.rates[2] = rates->rotation;
    a.rates[3] = rates->opacity;
    a.rates[4] = rates->sh;
    a.restScale = rates->sh_rest_scale;
    a.correction1 = 1.f - std::pow(0.9f, (float)adamStep);
    a.correction2 = 1.f - std::pow(0.999f, (float)adamStep);
    a.seed = adamStep;
  } else if (mode == ChainMode::Gradients) {
    for (int g = 0; g < 5; ++g) {
      const size_t counts[5] = {(size_t)n * 3, (size_t)n * 3, (size_t)n * 4, n, (size_t)n * 3 * shCoeffs};
      if (grads[g].bytes() < counts[g] * 4) {
        grads[g].ensure(counts[g] * 4);
        clear_graphs();
      }
    }
  }
  std::memcpy(h_args(), &a, sizeof(ChainArgs));
  lastArgs = a;
}

std::string Trainer::graph_key(ChainMode mode, bool statistics) const {
  // The active SH degree sets the projection's staging (its shared memory), so
  // a graph serves one degree only.
  std::string key = std::to_string((int)mode) + (statistics ? "s" : "-") + std::to_string(views.count) + "d" +
                    std::to_string(activeDegree);
  for (int k = 0; k < views.count; ++k) key += ":" + std::to_string(views.v[k].width) + "x" + std::to_string(views.v[k].height);
  return key;
}

void Trainer::finish_stats(splat_step_stats *stats, int count) {
  const StepReadback *rb = hReadback.get<StepReadback>();
  for (int k = 0; k < count; ++k) {
    splat_step_stats s{};
    const double perValue = 1.0 / (3.0 * (double)views.v[k].width * views.v[k].height);
    s.l1 = (float)(rb->totals.l1Sum[k] * perValue);
    s.ssim = (float)(rb->totals.ssimSum[k] * perValue);
    s.loss = (1.f - opt.lambda_ssim) * s.l1 + opt.lambda_ssim * (1.f - s.ssim);
    s.visible_splats = rb->counters[0];
    s.tile_entries = rb->counters[1];
    if (stats != nullptr) stats[k] = s;
  }
}

void Trainer::run(const splat_camera *cameras, const uint8_t *const *targets, const size_t *bytes, int count, ChainMode mode,
                  const splat_learning_rates *rates, bool statistics, splat_step_stats *stats, bool deviceTargets) {
  set_views(cameras, count);
  if (count > 1 && !oneSort) throw Failure{SPLAT_ERR_UNSUPPORTED, "several views per step need sort_form SPLAT_SORT_TILE_DEPTH_64"};
  if (count > 1 && blendLists) throw Failure{SPLAT_ERR_UNSUPPORTED, "blend lists are for one view per step"};
  ensure_view_buffers();
  // One view on a device target: the loss reads it where it is, no copy.
  const bool targetInPlace = deviceTargets && count == 1 && targets[0] != nullptr &&
                             bytes[0] == (size_t)views.v[0].width * views.v[0].height * 4 &&
                             reinterpret_cast<uintptr_t>(targets[0]) % 4 == 0;
  views.target = targetInPlace ? reinterpret_cast<const uint32_t *>(targets[0]) : nullptr;
  std::memcpy(h_views(), &views, sizeof(ViewSet));
  fill_chain_args(mode, statistics, rates);
  // The targets reach the device before the step's launches (and outside the graph).
  if (targetInPlace) {
    // Nothing to copy: the loss reads views.target.
  } else if (deviceTargets) {
    size_t off = 0;
    for (int k = 0; k < count; ++k) {
      const size_t want = (size_t)views.v[k].width * views.v[k].height * 4;
      if (bytes[k] != want || targets[k] == nullptr) throw Failure{SPLAT_ERR_INVALID, "the target image does not match the camera"};
      SB_CUDA(cudaMemcpyAsync(target.get<uint8_t>() + off, targets[k], want, cudaMemcpyDeviceToDevice, stream));
      off += want;
    }
  } else if (take_prefetched(targets, bytes, count)) {
    SB_CUDA(cudaStreamWaitEvent(stream, copied, 0));
    SB_CUDA(cudaMemcpyAsync(target.get(), targetNext.get(), bytes[0], cudaMemcpyDeviceToDevice, stream));
    SB_CUDA(cudaEventRecord(consumed, stream));
  } else {
    upload_targets(targets, bytes, count);
    SB_CUDA(cudaMemcpyAsync(target.get(), staging.get(), (size_t)views.totalPixels * 4, cudaMemcpyHostToDevice, stream));
  }

  bool graphDone = false;
  // A scored view runs the plain form (it is rare, and its loss and backward differ).
  if (useGraph && !blendLists && entryKeys.get() != nullptr && !timing && scoreShare <= 0.0f) {
    for (int attempt = 0; attempt < 3 && !graphDone; ++attempt) {
      const std::string key = graph_key(mode, statistics);
      auto it = graphs.find(key);
      if (it == graphs.end()) {
        cudaGraph_t graph = nullptr;
        SB_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        capturing = true;
        try {
          record_prepare(true);
          record_forward();
          record_backward_and_chain(mode, statistics);
          record_readback();
          capturing = false;
        } catch (...) {
          capturing = false;
          cudaStreamEndCapture(stream, &graph);
          if (graph != nullptr) cudaGraphDestroy(graph);
          throw;
        }
        SB_CUDA(cudaStreamEndCapture(stream, &graph));
        GraphEntry e;
        const cudaError_t ie = cudaGraphInstantiate(&e.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) throw Failure{SPLAT_ERR_DEVICE, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie)};
        it = graphs.emplace(key, e).first;
      }
      SB_CUDA(cudaGraphLaunch(it->second.exec, stream));
      stage_prefetch(); // host copy of the next target while the GPU runs the step
      SB_CUDA(cudaStreamSynchronize(stream));
      const StepReadback *rb = hReadback.get<StepReadback>();
      if ((rb->error & kErrEntryOverflow) != 0u) {
        // The kernels after the emission skipped their work: grow and run again.
        ensure_entries(rb->counters[1]);
        continue;
      }
      graphDone = true;
    }
    if (!graphDone) throw Failure{SPLAT_ERR_DEVICE, "the entry pool kept overflowing"};
  } else {
    record_prepare(true);
    // The reference's host wait: read the entry count and size the entry buffers.
    SB_CUDA(cudaMemcpyAsync(hReadback.get(), d_readback(), sizeof(StepReadback), cudaMemcpyDeviceToHost, stream));
    SB_CUDA(cudaStreamSynchronize(stream));
    const uint32_t total = hReadback.get<StepReadback>()->counters[1];
    if (total > entryCapacity || entryKeys.get() == nullptr) {
      ensure_entries(total);
      // The count-and-scan pass wrote the clipped count for the old capacity.
      const uint32_t fix[2] = {total, total};
      SB_CUDA(cudaMemcpyAsync(&d_readback()->counters[1], fix, sizeof(fix), cudaMemcpyHostToDevice, stream));
      uint32_t *err = &d_readback()->error;
      SB_CUDA(cudaMemsetAsync(err, 0, 4, stream));
      SB_CUDA(cudaStreamSynchronize(stream));
    }
    record_forward();
    record_backward_and_chain(mode, statistics);
    record_readback();
    stage_prefetch();
    SB_CUDA(cudaStreamSynchronize(stream));
  }
  const StepReadback *rb = hReadback.get<StepReadback>();
  if (rb->error != 0u) {
    char msg[96];
    std::snprintf(msg, sizeof msg, "device check failed (error bits 0x%x)", rb->error);
    throw Failure{SPLAT_ERR_DEVICE, msg};
  }
  if (timing) {
    for (int s = 0; s < kStages; ++s) {
      float ms = 0.f;
      SB_CUDA(cudaEventElapsedTime(&ms, events[2 * s], events[2 * s + 1]));
      stageTotals[s] += ms;
    }
    ++timedIterations;
  }
  haveRaw = true;
  if (mode == ChainMode::Gradients) haveGradients = true;
  finish_stats(stats, count);
  for (int k = 0; k < count; ++k) {
    if (stats != nullptr && !std::isfinite(stats[k].loss)) throw Failure{SPLAT_ERR_NONFINITE, "the loss is not finite"};
  }
}

// Switches the tile sort's form and digit width; the entry buffers (whose key
// width may change) and the captured graphs are rebuilt on the next step.
// Trainer::apply_changes (trainer.cpp:749-787): the parameters are gathered
// through paramSource (or uploaded from a host cloud), the optimiser state
// through stateSource (-1: fresh, zero), into the spare buffers, which
// then take the current ones' place; the densification statistics start at
// zero and the buffers sized by the count follow it at the next step. The
// views' buffers, the tile entries and the targets stay. With a memory
// budget the old buffers are freed at once; without one they are kept as the
// next edit's spares.
void Trainer::replace_gaussians(const int32_t *paramSource, const int32_t *stateSource, uint32_t newN, const splat_cloud *host) {
  SB_CUDA(cudaStreamSynchronize(stream));
  SB_CUDA(cudaStreamSynchronize(copyStream));
  const uint32_t oldN = n, oldStride = planeStride;
  const size_t nn = newN;
  const uint32_t newStride = (uint32_t)(((nn + kPlaneAlign - 1) / kPlaneAlign) * kPlaneAlign);
  const size_t copies = stateStore == StateStore::F32 ? 2 : 1;
  const uint32_t rowStride = sh_rest_stride(shCoeffs, shStore), rowWords = rowStride * (shStore == ShStore::F32 ? 4u : 2u) / 4u;
  const size_t paramBytes[6] = {nn * 12, nn * 12, nn * 16, nn * 4, (size_t)newStride * 12,
                                std::max<size_t>((size_t)newStride * rowWords * 4, 4)};
  const size_t stateBytes[5] = {nn * 12 * copies, nn * 12 * copies, nn * 16 * copies, nn * 4 * copies,
                                (size_t)newStride * sh_state_stride(shCoeffs) * 4 * copies};
  for (int g = 0; g < 6; ++g) grow(spareParams[g], paramBytes[g]);
  for (int g = 0; g < 5; ++g) grow(spareState[g], stateBytes[g]);
  const uint32_t strides[4] = {3, 3, 4, 1};
  DeviceBuffer *params[4] = {&positions, &scales, &rotations, &opacities};
  if (host != nullptr) {
    DeviceBuffer *to[6] = {&spareParams[0], &spareParams[1], &spareParams[2], &spareParams[3], &spareParams[4], &spareParams[5]};
    upload_cloud(*host, shCoeffs, shStore, newStride, to);
  } else {
    for (int g = 0; g < 4; ++g)
      launch_gather_rows(paramSource, params[g]->get<uint32_t>(), spareParams[g].get<uint32_t>(), newN, oldN, strides[g], 1u, stream);
    launch_gather_planes(paramSource, shDc.get<uint32_t>(), spareParams[4].get<uint32_t>(), newN, newStride, oldStride, 3u, stream);
    // The rows of higher coefficients, as words (a row is a whole number of 16-byte units).
    launch_gather_rows(paramSource, shRest.get<uint32_t>(), spareParams[5].get<uint32_t>(), newStride, oldStride, rowWords, 1u,
                       stream, newN);
  }
  for (int g = 0; g < 4; ++g)
    launch_gather_rows(stateSource, state[g].get<uint32_t>(), spareState[g].get<uint32_t>(), newN, oldN, strides[g],
                       (uint32_t)copies, stream);
  // The SH state rows: the row counts are the plane strides, the rows from
  // newN on padding.
  launch_gather_rows(stateSource, state[4].get<uint32_t>(), spareState[4].get<uint32_t>(), newStride, oldStride,
                     sh_state_stride(shCoeffs), (uint32_t)copies, stream, newN);
  SB_CUDA(cudaGetLastError());
  SB_CUDA(cudaStreamSynchronize(stream));
  for (int g = 0; g < 4; ++g) swap(*params[g], spareParams[g]);
  swap(shDc, spareParams[4]);
  swap(shRest, spareParams[5]);
  for (int g = 0; g < 5; ++g) swap(state[g], spareState[g]);
  if (opt.memory_budget != UINT64_MAX) {
    for (DeviceBuffer &b : spareParams) b.release();
    for (DeviceBuffer &b : spareState) b.release();
  }
  n = newN;
  planeStride = newStride;
  clear_graphs();
  viewSlots = 0; // the per-view buffers follow the count, and the raw sums are cleared, at the next step
  haveGradients = false;
  haveRaw = false;
  const size_t groupCounts[4] = {nn * 3, nn * 3, nn * 4, nn};
  for (int g = 0; g < 4; ++g) grow(grads[g], groupCounts[g] * 4);
  grow(densifyStats, nn * kStatStride * 4);
  SB_CUDA(cudaMemsetAsync(densifyStats.get(), 0, nn * kStatStride * 4, stream));
  SB_CUDA(cudaStreamSynchronize(stream));
}


void Trainer::set_sort(bool single, int digits) {
  if (single == oneSort && digits == digitBits) return;
  SB_CUDA(cudaStreamSynchronize(stream));
  oneSort = single;
  digitBits = digits;
  entryKeys.release();
  entryValues.release();
  tmpEntryKeys.release();
  tmpEntryValues.release();
  sortScratchEntries.release();
  sortScratchDepth.release();
  entryCapacity = 0;
  clear_graphs();
}

// The autotuner: times every sort form and digit width on one view with
// gradient passes, which change neither the parameters, the optimiser state
// nor the densification statistics, and keeps the fastest; then the
// rasterizer's pixel layouts; then, for the two-pixel float kernels, their
// tile edge (16 or 32), batch depth (128 or 256) and launch form (a block per
// tile or persistent). The one-pixel kernels keep the reference's 16 x 16
// tiles and 256-splat batches, one staged splat per pixel thread.
void Trainer::autotune(const splat_camera *camera, const uint8_t *target, size_t bytes, int repeats,
                       splat_autotune_result *out) {
  if (repeats < 1) repeats = 1;
  // A candidate replaces the configured setting of a stage only when it is
  // more than kKeep faster: differences inside the timing noise do not flip
  // the form from one run to the next.
  constexpr double kKeep = 1.01;
  const int oldForm = oneSort ? 1 : 0, oldDigits = digitBits;
  double best = 1e30, configuredMs = -1.0;
  int bestForm = oldForm, bestDigits = digitBits;
  const uint8_t *targets[1] = {target};
  const size_t sizes[1] = {bytes};
  splat_autotune_result result{};
  for (int form = 0; form < 2; ++form) {
    for (int digits = 6; digits <= 8; ++digits) {
      set_sort(form == 1, digits);
      splat_step_stats s{};
      // The first runs size the entry pool and capture the graph.
      run(camera, targets, sizes, 1, ChainMode::Gradients, nullptr, false, &s);
      run(camera, targets, sizes, 1, ChainMode::Gradients, nullptr, false, &s);
      const auto t0 = std::chrono::steady_clock::now();
      for (int r = 0; r < repeats; ++r) run(camera, targets, sizes, 1, ChainMode::Gradients, nullptr, false, &s);
      const double ms =
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / repeats;
      result.ms[form][digits - 6] = ms;
      if (form == oldForm && digits == oldDigits) configuredMs = ms;
      if (ms < best) {
        best = ms;
        bestForm = form;
        bestDigits = digits;
      }
    }
  }
  if (configuredMs > 0.0 && configuredMs <= best * kKeep) {
    bestForm = oldForm;
    bestDigits = oldDigits;
  }
  set_sort(bestForm == 1, bestDigits);
  result.sort_form = bestForm;
  result.digit_bits = bestDigits;
  // Then the rasterizer's layouts with that sort (the graphs are keyed by
  // shape only, so they are dropped before each change).
  const int oldForward = forwardPixels, oldBackward = backwardPixels;
  int bestForward = forwardPixels, bestBackward = backwardPixels;
  double bestLayoutMs = 1e30;
  configuredMs = -1.0;
  for (int fwd = 1; fwd <= 2; ++fwd) {
    for (int bwd = 1; bwd <= 2; ++bwd) {
      forwardPixels = fwd;
      backwardPixels = bwd;
      clear_graphs();
      splat_step_stats s{};
      run(camera, targets, sizes, 1, ChainMode::Gradients, nullptr, false, &s);
      const auto t0 = std::chrono::steady_clock::now();
      for (int r = 0; r < repeats; ++r) run(camera, targets, sizes, 1, ChainMode::Gradients, nullptr, false, &s);
      const double ms =
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / repeats;
      result.layout_ms[fwd - 1][bwd - 1] = ms;
      if (fwd == oldForward && bwd == oldBackward) configuredMs = ms;
      if (ms < bestLayoutMs) {
        bestLayoutMs = ms;
        bestForward = fwd;
        bestBackward = bwd;
      }
    }
  }
  if (configuredMs > 0.0 && configuredMs <= bestLayoutMs * kKeep) {
    bestForward = oldForward;
    bestBackward = oldBackward;
  }
  forwardPixels = bestForward;
  backwardPixels = bestBackward;
  clear_graphs();
  result.forward_pixels_per_thread = bestForward;
  result.backward_pixels_per_thread = bestBackward;
  // Then, where both layouts take two pixels per thread with float sums, the
  // tile edge, the staging batch and the launch form of those kernels.
  if (forwardPixels == 2 && backwardPixels == 2 && !fixedPoint && !blendLists) {
    const int oldTile = tileSize, oldBatch = batchDepth;
    const bool oldPersistent = persistent, oldGrouped = groupedSums;
    int bestTile = tileSize, bestBatch = batchDepth;
    bool bestPersistent = persistent, bestGrouped = groupedSums;
    double bestMs = 1e30;
    configuredMs = -1.0;
    for (int gi = 0; gi < 2; ++gi)
    for (int ti = 0; ti < 2; ++ti) {
      for (int bi = 0; bi < 2; ++bi) {
        for (int pi = 0; pi < 2; ++pi) {
          tileSize = 16 << ti;
          batchDepth = 128 << bi;
          persistent = pi == 1;
          groupedSums = gi == 1;
          clear_graphs();
          splat_step_stats s{};
          run(camera, targets, sizes, 1, ChainMode::Gradients, nullptr, false, &s);
          run(camera, targets, sizes, 1, ChainMode::Gradients, nullptr, false, &s);
          const auto t0 = std::chrono::steady_clock::now();
          for (int r = 0; r < repeats; ++r) run(camera, targets, sizes, 1, ChainMode::Gradients, nullptr, false, &s);
          const double ms =
              std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / repeats;
          (gi == 1 ? result.grouped_ms : result.tile_ms)[ti][bi][pi] = ms;
          if (tileSize == oldTile && batchDepth == oldBatch && persistent == oldPersistent && groupedSums == oldGrouped)
            configuredMs = ms;
          if (ms < bestMs) {
            bestMs = ms;
            bestTile = tileSize;
            bestBatch = batchDepth;
            bestPersistent = persistent;
            bestGrouped = groupedSums;
          }
        }
      }
    }
    if (configuredMs > 0.0 && configuredMs <= bestMs * kKeep) {
      bestTile = oldTile;
      bestBatch = oldBatch;
      bestPersistent = oldPersistent;
      bestGrouped = oldGrouped;
    }
    tileSize = bestTile;
    batchDepth = bestBatch;
    persistent = bestPersistent;
    groupedSums = bestGrouped;
    clear_graphs();
  }
  result.tile_size = raster_tile();
  result.batch_depth = batchDepth;
  result.persistent_raster = persistent ? 1 : 0;
  result.grouped_backward = groupedSums ? 1 : 0;
  if (out != nullptr) *out = result;
}

void Trainer::render(const splat_camera *camera, float *out) {
  set_views(camera, 1);
  ensure_view_buffers();
  std::memcpy(h_views(), &views, sizeof(ViewSet));
  record_prepare(false);
  SB_CUDA(cudaMemcpyAsync(hReadback.get(), d_readback(), sizeof(StepReadback), cudaMemcpyDeviceToHost, stream));
  SB_CUDA(cudaStreamSynchronize(stream));
  const uint32_t total = hReadback.get<StepReadback>()->counters[1];
  if (total > entryCapacity || entryKeys.get() == nullptr) {
    ensure_entries(total);
    const uint32_t fix[2] = {total, total};
    SB_CUDA(cudaMemcpyAsync(&d_readback()->counters[1], fix, sizeof(fix), cudaMemcpyHostToDevice, stream));
    SB_CUDA(cudaMemsetAsync(&d_readback()->error, 0, 4, stream));
  }
  const bool wasTiming = timing;
  timing = false;
  record_forward();
  timing = wasTiming;
  if (orderPending) {
    // No backward pass follows a render: take the order's stream back.
    if (orderForked) SB_CUDA(cudaStreamWaitEvent(stream, orderEvent, 0));
    orderPending = orderForked = false;
  }
  record_readback();
  SB_CUDA(cudaStreamSynchronize(stream));
  if (hReadback.get<StepReadback>()->error != 0u) throw Failure{SPLAT_ERR_DEVICE, "device check failed during render"};
  const size_t pixels = (size_t)camera->width * camera->height;
  SB_CUDA(cudaMemcpy(out, image.get(), pixels * 16, cudaMemcpyDeviceToHost));
  // The SFU form keeps log T in base 2 on the device; the caller gets natural logs.
  if (!exactMath)
    for (size_t p = 0; p < pixels; ++p) out[p * 4 + 3] *= 0.6931471805599453f;
}

// ---------------------------------------------------------------- small kernels

__global__ void k_detmath(const float *in, float *outExp, float *outLog, uint32_t count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  outExp[i] = splat_expf(in[i]);
  outLog[i] = in[i] > 0.0f ? splat_logf(in[i]) : 0.0f;
}

} // namespace sb

// ---------------------------------------------------------------- C ABI

using sb::Failure;
using sb::Trainer;

struct splat_trainer {
  Trainer *impl;
};

namespace {

int fail(int status, const std::string &message) {
  sb::g_lastError = message;
  return status;
}

template <class F> int guarded(F &&f) {
  try {
    f();
    sb::g_lastError.clear();
    return SPLAT_OK;
  } catch (const Failure &e) {
    return fail(e.status, e.message);
  } catch (const std::bad_alloc &) {
    return fail(SPLAT_ERR_NOMEM, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(SPLAT_ERR_INVALID, e.what());
  }
}

Trainer *impl_of(splat_trainer *t) {
  if (t == nullptr || t->impl == nullptr) throw Failure{SPLAT_ERR_INVALID, "null trainer"};
  return t->impl;
}

// A part of a device buffer.
struct Slice {
  void *p = nullptr;
  template <class T = void> T *get() const { return static_cast<T *>(p); }
};

// An edit's scratch: 256-byte aligned slices of a device buffer the trainer
// keeps, made large enough up front for everything the edit takes.
class Arena {
public:
  Arena(sb::DeviceBuffer &buffer, size_t bytes) : buffer_(buffer), limit_(bytes) { sb::grow(buffer, bytes); }
  Slice take(size_t bytes) {
    const size_t size = (std::max<size_t>(bytes, 1) + 255) & ~size_t{255};
    if (used_ + size > limit_) throw Failure{SPLAT_ERR_DEVICE, "an edit's scratch was sized too small"};
    Slice s{buffer_.get<uint8_t>() + used_};
    used_ += size;
    return s;
  }
  static size_t room(size_t bytes) { return (std::max<size_t>(bytes, 1) + 255) & ~size_t{255}; }

private:
  sb::DeviceBuffer &buffer_;
  size_t limit_, used_ = 0;
};

} // namespace

extern "C" {

const char *splat_last_error(void) { return sb::g_lastError.c_str(); }

void splat_trainer_options_default(splat_trainer_options *o) {
  if (o == nullptr) return;
  std::memset(o, 0, sizeof(*o));
  o->lambda_ssim = 0.2f;
  o->near_plane = 0.01f;
  o->selective_adam = 1;
  o->memory_budget = ~0ull;
  o->sh_storage = SPLAT_SH_F16;
  o->state_storage = SPLAT_STATE_BF16_PAIR;
  o->sort_form = SPLAT_SORT_DEPTH_THEN_TILE;
  o->exact_math = 1;
  o->use_graph = 0;
  o->digit_bits = 8;
  o->forward_pixels_per_thread = 1;
  o->backward_pixels_per_thread = 2;
  o->tile_size = 16;
  o->batch_depth = 128;
  o->persistent_raster = 0;
  o->grouped_backward = 0;
}

void splat_learning_rates_default(splat_learning_rates *r) {
  if (r == nullptr) return;
  r->position = 1.6e-4f;
  r->scale = 0.005f;
  r->rotation = 0.001f;
  r->opacity = 0.05f;
  r->sh = 0.025f;
  r->sh_rest_scale = 0.05f;
  r->trust_region = 0.f;
}

int splat_trainer_create(const splat_cloud *cloud, const splat_trainer_options *options, splat_trainer **out) {
  return guarded([&] {
    if (cloud == nullptr || out == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    splat_trainer_options o;
    if (options != nullptr) o = *options;
    else splat_trainer_options_default(&o);
    *out = nullptr;
    Trainer *t = new Trainer(*cloud, o);
    *out = new splat_trainer{t};
  });
}

int splat_trainer_destroy(splat_trainer *trainer) {
  return guarded([&] {
    if (trainer == nullptr) return;
    delete trainer->impl;
    delete trainer;
  });
}

int splat_trainer_render(splat_trainer *trainer, const splat_camera *camera, float *out_pixels) {
  return guarded([&] {
    if (camera == nullptr || out_pixels == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    impl_of(trainer)->render(camera, out_pixels);
  });
}

static int run_one(splat_trainer *trainer, const splat_camera *camera, const uint8_t *target, size_t bytes,
                   sb::ChainMode mode, const splat_learning_rates *rates, bool statistics, splat_step_stats *stats) {
  return guarded([&] {
    if (camera == nullptr) throw Failure{SPLAT_ERR_INVALID, "null camera"};
    if (mode == sb::ChainMode::Step && (rates == nullptr || rates->trust_region != 0.f))
      throw Failure{rates == nullptr ? SPLAT_ERR_INVALID : SPLAT_ERR_UNSUPPORTED, "rates missing, or a trust region (second order)"};
    const uint8_t *targets[1] = {target};
    const size_t sizes[1] = {bytes};
    impl_of(trainer)->run(camera, targets, sizes, 1, mode, rates, statistics, stats);
  });
}

int splat_trainer_compute_gradients(splat_trainer *trainer, const splat_camera *camera, const uint8_t *target,
                                    size_t target_bytes, splat_step_stats *stats) {
  return run_one(trainer, camera, target, target_bytes, sb::ChainMode::Gradients, nullptr, true, stats);
}

int splat_trainer_collect_statistics(splat_trainer *trainer, const splat_camera *camera, const uint8_t *target,
                                     size_t target_bytes, splat_step_stats *stats) {
  return run_one(trainer, camera, target, target_bytes, sb::ChainMode::Statistics, nullptr, true, stats);
}

int splat_trainer_score_view(splat_trainer *trainer, const splat_camera *camera, const uint8_t *target, size_t target_bytes,
                             float error_share, float pixel_weight, splat_step_stats *stats) {
  return guarded([&] {
    if (camera == nullptr || target == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    impl_of(trainer)->score_view(camera, target, target_bytes, error_share, pixel_weight, stats);
  });
}

int splat_trainer_collect_statistics_device_target(splat_trainer *trainer, const splat_camera *camera, const uint8_t *device_target,
                                                   size_t target_bytes, splat_step_stats *stats) {
  return guarded([&] {
    if (camera == nullptr || device_target == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    const uint8_t *targets[1] = {device_target};
    const size_t sizes[1] = {target_bytes};
    impl_of(trainer)->run(camera, targets, sizes, 1, sb::ChainMode::Statistics, nullptr, true, stats, true);
  });
}

int splat_trainer_score_view_device_target(splat_trainer *trainer, const splat_camera *camera, const uint8_t *device_target,
                                           size_t target_bytes, float error_share, float pixel_weight, splat_step_stats *stats) {
  return guarded([&] {
    if (camera == nullptr || device_target == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    impl_of(trainer)->score_view(camera, device_target, target_bytes, error_share, pixel_weight, stats, true);
  });
}

int splat_trainer_apply_gradients(splat_trainer *trainer, const splat_learning_rates *rates) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    if (rates == nullptr) throw Failure{SPLAT_ERR_INVALID, "null rates"};
    if (rates->trust_region != 0.f) throw Failure{SPLAT_ERR_UNSUPPORTED, "second-order steps have no kernel in this library"};
    if (!t->haveRaw) throw Failure{SPLAT_ERR_STATE, "no gradients: compute_gradients() leaves the sums apply_gradients() uses"};
    t->fill_chain_args(sb::ChainMode::Step, false, rates);
    SB_CUDA(cudaMemcpyAsync(t->d_args(), t->h_args(), sizeof(sb::ChainArgs), cudaMemcpyHostToDevice, t->stream));
    sb::OptimState st = t->optim_state();
    sb::GradientsOut g{};
    for (int k = 0; k < 5; ++k) g.g[k] = t->grads[k].get<float>();
    sb::launch_chain(t->params(), t->views, t->d_views(), t->raw.get(), t->splats.get<sb::Splat>(), t->lastArgs,
                     t->d_args(), st, &g, t->shGrad.get<float4>(), t->densifyStats.get<float>(), nullptr,
                     t->stream);
    SB_CUDA(cudaStreamSynchronize(t->stream));
  });
}

int splat_trainer_step(splat_trainer *trainer, const splat_camera *camera, const uint8_t *target, size_t target_bytes,
                       const splat_learning_rates *rates, const uint8_t *next_target, size_t next_target_bytes,
                       splat_step_stats *stats) {
  // The next target is copied to pinned memory while this step runs on the GPU.
  if (trainer != nullptr && trainer->impl != nullptr && next_target != nullptr) {
    impl_of(trainer)->pendingPrefetch = next_target;
    impl_of(trainer)->pendingPrefetchBytes = next_target_bytes;
  }
  const int status = run_one(trainer, camera, target, target_bytes, sb::ChainMode::Step, rates, true, stats);
  if (trainer != nullptr && trainer->impl != nullptr) impl_of(trainer)->pendingPrefetch = nullptr;
  return status;
}

int splat_trainer_step_device_target(splat_trainer *trainer, const splat_camera *camera, const uint8_t *device_target,
                                     size_t target_bytes, const splat_learning_rates *rates, splat_step_stats *stats) {
  return guarded([&] {
    if (camera == nullptr || rates == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    if (rates->trust_region != 0.f) throw Failure{SPLAT_ERR_UNSUPPORTED, "second-order steps have no kernel in this library"};
    const uint8_t *targets[1] = {device_target};
    const size_t sizes[1] = {target_bytes};
    impl_of(trainer)->run(camera, targets, sizes, 1, sb::ChainMode::Step, rates, true, stats, true);
  });
}

int splat_trainer_stream(splat_trainer *trainer, void **stream) {
  return guarded([&] {
    if (stream == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    *stream = impl_of(trainer)->stream;
  });
}

int splat_trainer_step_batch(splat_trainer *trainer, const splat_camera *cameras, const uint8_t *const *targets,
                             int32_t views, const splat_learning_rates *rates, splat_step_stats *stats) {
  return guarded([&] {
    if (cameras == nullptr || targets == nullptr || rates == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    if (rates->trust_region != 0.f) throw Failure{SPLAT_ERR_UNSUPPORTED, "second-order steps have no kernel in this library"};
    if (views < 1 || views > sb::kMaxViews) throw Failure{SPLAT_ERR_INVALID, "between 1 and 8 views per step"};
    size_t sizes[sb::kMaxViews];
    for (int k = 0; k < views; ++k) sizes[k] = (size_t)cameras[k].width * cameras[k].height * 4;
    impl_of(trainer)->run(cameras, targets, sizes, views, sb::ChainMode::Step, rates, true, stats);
  });
}

int splat_trainer_step_batch_device_targets(splat_trainer *trainer, const splat_camera *cameras, const uint8_t *const *device_targets,
                                            int32_t views, const splat_learning_rates *rates, splat_step_stats *stats) {
  return guarded([&] {
    if (cameras == nullptr || device_targets == nullptr || rates == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    if (rates->trust_region != 0.f) throw Failure{SPLAT_ERR_UNSUPPORTED, "second-order steps have no kernel in this library"};
    if (views < 1 || views > sb::kMaxViews) throw Failure{SPLAT_ERR_INVALID, "between 1 and 8 views per step"};
    size_t sizes[sb::kMaxViews];
    for (int k = 0; k < views; ++k) sizes[k] = (size_t)cameras[k].width * cameras[k].height * 4;
    impl_of(trainer)->run(cameras, device_targets, sizes, views, sb::ChainMode::Step, rates, true, stats, true);
  });
}

int splat_trainer_prefetch_target(splat_trainer *trainer, const uint8_t *target, size_t target_bytes) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    if (target == nullptr) throw Failure{SPLAT_ERR_INVALID, "null target"};
    t->prefetch(target, target_bytes);
  });
}

int splat_trainer_get_gradients(splat_trainer *trainer, float *positions, float *scales, float *rotations, float *opacities,
                                float *sh) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    if (!t->haveGradients) throw Failure{SPLAT_ERR_STATE, "no gradients: compute_gradients() stores them"};
    const size_t n = t->n;
    float *outs[5] = {positions, scales, rotations, opacities, sh};
    const size_t counts[5] = {n * 3, n * 3, n * 4, n, n * 3 * t->shCoeffs};
    for (int g = 0; g < 5; ++g)
      if (outs[g] != nullptr) SB_CUDA(cudaMemcpy(outs[g], t->grads[g].get(), counts[g] * 4, cudaMemcpyDeviceToHost));
  });
}

int splat_trainer_get_cloud(splat_trainer *trainer, float *positions, float *scales, float *rotations, float *opacities,
                            float *sh) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    SB_CUDA(cudaStreamSynchronize(t->stream));
    const size_t n = t->n;
    if (positions) SB_CUDA(cudaMemcpy(positions, t->positions.get(), n * 12, cudaMemcpyDeviceToHost));
    if (scales) SB_CUDA(cudaMemcpy(scales, t->scales.get(), n * 12, cudaMemcpyDeviceToHost));
    if (rotations) SB_CUDA(cudaMemcpy(rotations, t->rotations.get(), n * 16, cudaMemcpyDeviceToHost));
    if (opacities) SB_CUDA(cudaMemcpy(opacities, t->opacities.get(), n * 4, cudaMemcpyDeviceToHost));
    if (sh) {
      const int floats = 3 * t->shCoeffs;
      const size_t ps = t->planeStride;
      std::vector<float> dc(ps * 3);
      SB_CUDA(cudaMemcpy(dc.data(), t->shDc.get(), ps * 12, cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) sh[i * floats + c] = dc[c * ps + i];
      const size_t rowStride = sh_rest_stride(t->shCoeffs, t->shStore), rest = ps * rowStride;
      if (rest > 0) {
        std::vector<float> planes(rest);
        if (t->shStore == sb::ShStore::F32) {
          SB_CUDA(cudaMemcpy(planes.data(), t->shRest.get(), rest * 4, cudaMemcpyDeviceToHost));
        } else {
          std::vector<uint16_t> half(rest);
          SB_CUDA(cudaMemcpy(half.data(), t->shRest.get(), rest * 2, cudaMemcpyDeviceToHost));
          for (size_t k = 0; k < rest; ++k) {
            if (t->shStore == sb::ShStore::BF16) {
              const uint32_t bits = (uint32_t)half[k] << 16;
              std::memcpy(&planes[k], &bits, 4);
            } else {
              planes[k] = __half2float(__ushort_as_half(half[k]));
            }
          }
        }
        for (size_t i = 0; i < n; ++i)
          for (int j = 3; j < floats; ++j) sh[i * floats + j] = planes[i * rowStride + (size_t)(j - 3)];
      }
    }
  });
}

int splat_trainer_set_active_sh_degree(splat_trainer *trainer, int32_t degree) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    t->activeDegree = std::clamp<int>(degree, 0, t->shDegree);
  });
}

int splat_trainer_get_densify_stats(splat_trainer *trainer, float *out) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    if (out == nullptr) throw Failure{SPLAT_ERR_INVALID, "null output"};
    SB_CUDA(cudaStreamSynchronize(t->stream));
    SB_CUDA(cudaMemcpy(out, t->densifyStats.get(), (size_t)t->n * sb::kStatStride * 4, cudaMemcpyDeviceToHost));
  });
}

int splat_trainer_set_densify_stats(splat_trainer *trainer, const float *raw) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    if (raw == nullptr) throw Failure{SPLAT_ERR_INVALID, "null input"};
    SB_CUDA(cudaStreamSynchronize(t->stream));
    SB_CUDA(cudaMemcpy(t->densifyStats.get(), raw, (size_t)t->n * sb::kStatStride * 4, cudaMemcpyHostToDevice));
  });
}

int splat_trainer_reset_densify_stats(splat_trainer *trainer) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    SB_CUDA(cudaMemsetAsync(t->densifyStats.get(), 0, (size_t)t->n * sb::kStatStride * 4, t->stream));
    SB_CUDA(cudaStreamSynchronize(t->stream));
  });
}

int splat_trainer_reset_opacity(splat_trainer *trainer, float maximum) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    const float limit = std::log(maximum / (1.f - maximum));
    std::vector<float> values(t->n);
    SB_CUDA(cudaStreamSynchronize(t->stream));
    SB_CUDA(cudaMemcpy(values.data(), t->opacities.get(), (size_t)t->n * 4, cudaMemcpyDeviceToHost));
    for (float &v : values) v = std::min(v, limit);
    SB_CUDA(cudaMemcpy(t->opacities.get(), values.data(), (size_t)t->n * 4, cudaMemcpyHostToDevice));
    SB_CUDA(cudaMemset(t->state[3].get(), 0, t->state[3].bytes()));
  });
}

int splat_trainer_apply_changes(splat_trainer *trainer, const splat_cloud *cloud, const int32_t *source) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    if (cloud == nullptr || source == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    if (cloud->count <= 0) throw Failure{SPLAT_ERR_INVALID, "densification removed every Gaussian"};
    if (cloud->sh_degree != t->shDegree) throw Failure{SPLAT_ERR_INVALID, "the SH degree cannot change"};
    if (cloud->positions == nullptr || cloud->scales == nullptr || cloud->rotations == nullptr || cloud->opacities == nullptr ||
        cloud->sh == nullptr)
      throw Failure{SPLAT_ERR_INVALID, "GaussianCloud: inconsistent array sizes"};
    const size_t oldN = t->n, newN = (size_t)cloud->count;
    for (size_t i = 0; i < newN; ++i)
      if (source[i] >= (int64_t)oldN) throw Failure{SPLAT_ERR_INVALID, "a source index is past the old Gaussians"};
    // The new cloud is uploaded into the spare buffers and the survivors'
    // optimiser state gathered on the GPU through the source table
    // (train_gather.comp), so that the moments never cross to the host; the
    // densification statistics start anew.
    sb::DeviceBuffer table;
    table.ensure(newN * sizeof(int32_t));
    SB_CUDA(cudaMemcpy(table.get(), source, newN * sizeof(int32_t), cudaMemcpyHostToDevice));
    t->replace_gaussians(nullptr, table.get<int32_t>(), (uint32_t)newN, cloud);
  });
}

namespace {

// The trainer's Gaussians replaced by newN gathered on the device
// (Trainer::apply_changes, trainer.cpp:749-787): parameters through
// paramSource, optimiser state through stateSource (-1: fresh, zero).
Trainer *regather(splat_trainer *handle, const int32_t *paramSource, const int32_t *stateSource, uint32_t newN) {
  Trainer *t = impl_of(handle);
  t->replace_gaussians(paramSource, stateSource, newN);
  return t;
}

// remove_highest on the GPU (densify.cpp:70-90, Trainer::apply_changes,
// trainer.cpp:749-787): removes ceil(share n) Gaussians (at most n - 1) by the
// key of `kind`, highest first, ties in index order; the survivors keep
// their order, parameters and optimiser state, gathered on the device through
// the source table; the densification statistics start anew. Returns how
// many were removed.
uint64_t prune_gaussians(splat_trainer *handle, int kind, double share) {
  Trainer *t = impl_of(handle);
  if (!(share >= 0.0 && share <= 1.0)) throw Failure{SPLAT_ERR_INVALID, "share must be in [0, 1]"};
  const uint32_t oldN = t->n;
  const uint32_t removed = (uint32_t)std::min<double>((double)oldN - 1.0, std::ceil((double)oldN * share));
  if (removed == 0) return 0;
  const uint32_t newN = oldN - removed;
  cudaStream_t s = t->stream;
  SB_CUDA(cudaStreamSynchronize(s));
  const size_t words = Arena::room((size_t)oldN * 4);
  Arena arena(t->editScratch, 7 * words + Arena::room(sb::sort_scratch_bytes(oldN, 4, 32, 8)) +
                                  Arena::room(sb::bin_scan_scratch_bytes(oldN)) + Arena::room(16));
  Slice keys = arena.take(words), values = arena.take(words), tmpKeys = arena.take(words), tmpValues = arena.take(words);
  Slice keep = arena.take(words), place = arena.take(words), table = arena.take(words);
  Slice scratch = arena.take(sb::sort_scratch_bytes(oldN, 4, 32, 8)), scanScratch = arena.take(sb::bin_scan_scratch_bytes(oldN));
  Slice counters = arena.take(16);
  SB_CUDA(cudaMemsetAsync(counters.get(), 0, 16, s));
  uint32_t *error = counters.get<uint32_t>() + 3;
  const float *stats = kind == 1 ? t->densifyStats.get<float>() : nullptr;
  if (kind == 1 && stats == nullptr) throw Failure{SPLAT_ERR_STATE, "no densification statistics to prune by"};
  sb::launch_prune_keys(kind, t->scales.get<float>(), t->opacities.get<float>(), stats, oldN, keys.get<uint32_t>(),
                        values.get<uint32_t>(), s);
  const int where = sb::sort_pairs_u32(keys.get<uint32_t>(), values.get<uint32_t>(), tmpKeys.get<uint32_t>(), tmpValues.get<uint32_t>(),
                                       oldN, oldN, nullptr, 0, 32, 8, scratch.get(), error, s);
  const uint32_t *order = where == 1 ? tmpValues.get<uint32_t>() : values.get<uint32_t>();
  sb::launch_prune_keep(order, removed, oldN, keep.get<uint32_t>(), s);
  SB_CUDA(cudaMemcpyAsync(place.get(), keep.get(), (size_t)oldN * 4, cudaMemcpyDeviceToDevice, s));
  sb::launch_exclusive_scan(oldN, place.get<uint32_t>(), counters.get<uint32_t>(), scanScratch.get(), error, s);
  sb::launch_survivor_sources(keep.get<uint32_t>(), place.get<uint32_t>(), oldN, table.get<int32_t>(), s);
  uint32_t status[4] = {0, 0, 0, 0};
  SB_CUDA(cudaMemcpyAsync(status, counters.get(), 16, cudaMemcpyDeviceToHost, s));
  SB_CUDA(cudaStreamSynchronize(s));
  if (status[3] != 0u) throw Failure{SPLAT_ERR_DEVICE, "the pruning sort's look-back gave up waiting"};
  if (status[1] != newN) throw Failure{SPLAT_ERR_DEVICE, "the pruning kept an unexpected number of Gaussians"};
  regather(handle, table.get<int32_t>(), table.get<int32_t>(), newN);
  return removed;
}


} // namespace
} // extern "C"

namespace {

// ------------------------------------------------------------ densification

// The smallest float x, in the order -inf .. +inf, for which holds(x), when
// holds is false below some point and true from it on; NaN if it holds
// nowhere. A bisection over the floats' bit patterns.
template <class F> float first_holding(F holds) {
  const auto from_key = [](uint32_t k) {
    const uint32_t bits = (k & 0x80000000u) != 0u ? (k ^ 0x80000000u) : ~k;
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
  };
  uint32_t lo = 0x007FFFFFu, hi = 0xFF800000u; // -inf, +inf
  if (!holds(from_key(hi))) return std::numeric_limits<float>::quiet_NaN();
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (holds(from_key(mid))) hi = mid;
    else lo = mid + 1;
  }
  return from_key(lo);
}

// Thresholds on the device's side of the comparisons densify_cloud makes
// through the host's exp (densify.cpp:17,130,135,138): a Gaussian is larger
// than s exactly when its largest log-scale is at least the first x with
// exp(x) > s, and too transparent exactly when its logit is below the first
// x whose sigmoid is not below the limit. The device then compares floats
// only, and decides as the reference does bit for bit.
float log_threshold(float scale) {
  return first_holding([&](float x) { return std::exp(x) > scale; });
}
float logit_threshold(float limit) {
  const float x = first_holding([&](float o) { return !(1.f / (1.f + std::exp(-o)) < limit); });
  return std::isnan(x) ? std::numeric_limits<float>::infinity() : x;
}
// The same for "at or below the limit" (relocation's dead, densify.cpp:336).
float logit_threshold_inclusive(float limit) {
  const float x = first_holding([&](float o) { return !(1.f / (1.f + std::exp(-o)) <= limit); });
  return std::isnan(x) ? std::numeric_limits<float>::infinity() : x;
}

// The Gaussian's rotation as a matrix, identity for a degenerate quaternion:
// the same float arithmetic as densify.cpp:42-59, since the children's
// positions are compared bit for bit.
void rotation_matrix(const float q[4], float R[3][3]) {
  float w = q[0], x = q[1], y = q[2], z = q[3];
  const float length = std::sqrt(w * w + x * x + y * y + z * z);
  if (length > 0.f) {
    w /= length;
    x /= length;
    y /= length;
    z /= length;
  } else {
    w = 1.f;
    x = y = z = 0.f;
  }
  R[0][0] = 1.f - 2.f * (y * y + z * z);
  R[0][1] = 2.f * (x * y - w * z);
  R[0][2] = 2.f * (x * z + w * y);
  R[1][0] = 2.f * (x * y + w * z);
  R[1][1] = 1.f - 2.f * (x * x + z * z);
  R[1][2] = 2.f * (y * z - w * x);
  R[2][0] = 2.f * (x * z - w * y);
  R[2][1] = 2.f * (y * z + w * x);
  R[2][2] = 1.f - 2.f * (x * x + y * y);
}

// Rows of the old cloud gathered to the host for a list of indices.
struct HostRows {
  std::vector<float> positions, scales, rotations, opacities;
  std::vector<uint32_t> actions;
};

} // namespace

struct splat_rng {
  std::mt19937 engine;
};

namespace {

struct DensifyRun {
  Trainer *t;
  cudaStream_t s;
  uint32_t n;
  Arena arena;
  Slice counters, scanScratch, sortScratch, tmpKeys, tmpValues, rows;

  // arrays: how many further n-word arrays the edit takes (take()).
  static size_t bytes(uint32_t n, int arrays) {
    return Arena::room(64 * 4) + Arena::room(sb::bin_scan_scratch_bytes(n)) + Arena::room(sb::sort_scratch_bytes(n, 4, 32, 8)) +
           (2 + 8 + (size_t)arrays) * Arena::room((size_t)n * 4 + 4);
  }
  DensifyRun(Trainer *trainer, int arrays)
      : t(trainer), s(trainer->stream), n(trainer->n), arena(trainer->editScratch, bytes(trainer->n, arrays)) {
    counters = arena.take(64 * 4);
    SB_CUDA(cudaMemsetAsync(counters.get(), 0, 64 * 4, s));
    scanScratch = arena.take(sb::bin_scan_scratch_bytes(n));
    sortScratch = arena.take(sb::sort_scratch_bytes(n, 4, 32, 8));
    tmpKeys = take();
    tmpValues = take();
    rows = arena.take(8 * ((size_t)n * 4 + 4));
  }
  // An array of n + 1 words.
  Slice take() { return arena.take((size_t)n * 4 + 4); }
  uint32_t *error() { return counters.get<uint32_t>() + 63; }
  // Exclusive scan of flags into place (both n words); the total lands in
  // counter block `block` (word 1).
  void scan(const Slice &flags, const Slice &place, int block) {
    SB_CUDA(cudaMemcpyAsync(place.get(), flags.get(), (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    sb::launch_exclusive_scan(n, place.get<uint32_t>(), counters.get<uint32_t>() + 4 * block, scanScratch.get(), error(), s);
  }
  // The counters, after the stream's work so far.
  std::vector<uint32_t> read() {
    std::vector<uint32_t> h(64);
    SB_CUDA(cudaMemcpyAsync(h.data(), counters.get(), 64 * 4, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    if (h[63] != 0u) throw Failure{SPLAT_ERR_DEVICE, "a densification scan or sort gave up waiting"};
    return h;
  }
  // Stable ascending sort of count (key, index) pairs; returns the indices.
  const uint32_t *sort(const Slice &keys, const Slice &indices, uint32_t count) {
    if (count <= 1) return indices.get<uint32_t>();
    const int where = sb::sort_pairs_u32(keys.get<uint32_t>(), indices.get<uint32_t>(), tmpKeys.get<uint32_t>(),
                                         tmpValues.get<uint32_t>(), n, count, nullptr, 0, 32, 8, sortScratch.get(), error(), s);
    return where == 1 ? tmpValues.get<uint32_t>() : indices.get<uint32_t>();
  }
  // Downloads a device list of count indices.
  std::vector<uint32_t> download(const uint32_t *list, uint32_t count) {
    std::vector<uint32_t> h(count);
    if (count > 0) SB_CUDA(cudaMemcpyAsync(h.data(), list, (size_t)count * 4, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    return h;
  }
  // The rows of `stride` (at most 8) words of `in` (n rows) for the count
  // listed indices.
  std::vector<float> gather(const int32_t *list, const void *in, uint32_t count, uint32_t stride) {
    std::vector<float> h((size_t)count * stride);
    if (count == 0) return h;
    sb::launch_gather_rows(list, static_cast<const uint32_t *>(in), rows.get<uint32_t>(), count, n, stride, 1u, s);
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaMemcpyAsync(h.data(), rows.get(), h.size() * 4, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    return h;
  }
};

// Trainer::densify on the GPU (trainer.cpp:710-715; densify_cloud,
// densify.cpp:115-326; apply_changes). Every per-Gaussian decision, both
// global selections and the tables run on the device; the host draws from
// rng in the reference's order (edge splits, the exploration shuffle, the
// split children in index order, the seeds) over lists the device compacted.
void densify_gaussians(splat_trainer *handle, const splat_densify_options &o, std::mt19937 &rng, splat_densify_result *result,
                       int64_t *source, uint64_t sourceCapacity) {
  Trainer *t = impl_of(handle);
  if (o.transparent_share < 0.0) throw Failure{SPLAT_ERR_INVALID, "transparent_share must not be negative"};
  SB_CUDA(cudaStreamSynchronize(t->stream));
  if (t->densifyStats.get() == nullptr) throw Failure{SPLAT_ERR_STATE, "no densification statistics"};
  DensifyRun run(t, 14);
  cudaStream_t s = run.s;
  const uint32_t n = run.n;
  const float *stats = t->densifyStats.get<float>();
  const float *scales = t->scales.get<float>();

  sb::DensifyArgs a{};
  a.gradientThreshold = o.gradient_threshold;
  a.splitThreshold = o.split_threshold;
  a.maxScreenRadius = o.max_screen_radius;
  a.minMarkedPixels = o.min_marked_pixels;
  a.worldLog = log_threshold(o.max_world_scale);
  a.denseLog = log_threshold(o.dense_scale);
  a.opacityLogit = logit_threshold(o.prune_opacity);
  a.pruneLarge = o.prune_large != 0 ? 1 : 0;
  a.scoredViews = o.scored_views;
  a.allTransparent = o.transparent_share < 1.0 ? 0 : 1;
  a.edgeSplit = o.edge_split != 0 ? 1 : 0;

  Slice action = run.take(), flags = run.take(), keys = run.take(), place = run.take(), list = run.take(), keyList = run.take();
  Slice kept = run.take(), keptPlace = run.take(), candidate = run.take(), candidatePlace = run.take(), priority = run.take();
  Slice chosen = run.take(), parents = run.take(), childSlot = run.take();

  // The oversized, the non-finite and the too transparent.
  sb::launch_densify_classify(t->params(), stats, a, action.get<uint32_t>(), flags.get<uint32_t>(), keys.get<uint32_t>(), s);
  if (!a.allTransparent) {
    run.scan(flags, place, 0);
    const uint32_t clear = run.read()[1];
    sb::launch_compact(flags.get<uint32_t>(), place.get<uint32_t>(), keys.get<uint32_t>(), n, list.get<uint32_t>(),
                       keyList.get<uint32_t>(), s);
    const uint32_t *order = run.sort(keyList, list, clear);
    const auto removed = (uint32_t)std::ceil((double)clear * o.transparent_share);
    sb::launch_set_first(order, std::min(removed, clear), sb::kDensifyPrune, action.get<uint32_t>(), s);
  }

  // Candidates, and the count limit.
  sb::launch_densify_candidates(scales, stats, a, n, action.get<uint32_t>(), kept.get<uint32_t>(), candidate.get<uint32_t>(),
                                priority.get<uint32_t>(), s);
  run.scan(kept, keptPlace, 1);
  run.scan(candidate, candidatePlace, 2);
  std::vector<uint32_t> c = run.read();
  const uint64_t keptCount = c[5], candidates = c[9];
  const uint64_t room = o.max_gaussians > keptCount ? o.max_gaussians - keptCount : 0;
  uint64_t chosenCount = candidates, heldBack = 0;
  if (candidates > room) {
    sb::launch_compact(candidate.get<uint32_t>(), candidatePlace.get<uint32_t>(), priority.get<uint32_t>(), n, list.get<uint32_t>(),
                       keyList.get<uint32_t>(), s);
    const uint32_t *order = run.sort(keyList, list, (uint32_t)candidates);
    SB_CUDA(cudaMemsetAsync(chosen.get(), 0, (size_t)n * 4, s));
    sb::launch_set_first(order, (uint32_t)room, 1u, chosen.get<uint32_t>(), s);
    heldBack = candidates - room;
    chosenCount = room;
  } else {
    SB_CUDA(cudaMemcpyAsync(chosen.get(), candidate.get(), (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
  }

  // Edge splits (densify.cpp:181-190): each chosen candidate stays with
  // probability score / best, drawn in index order.
  if (a.edgeSplit && chosenCount > 0) {
    run.scan(chosen, place, 3);
    sb::launch_compact(chosen.get<uint32_t>(), place.get<uint32_t>(), nullptr, n, list.get<uint32_t>(), nullptr, s);
    const std::vector<uint32_t> listed = run.download(list.get<uint32_t>(), (uint32_t)chosenCount);
    const std::vector<float> rowsOf = run.gather(list.get<int32_t>(), stats, (uint32_t)chosenCount, sb::kStatStride);
    float best = 0.f;
    for (size_t k = 0; k < listed.size(); ++k) best = std::max(best, rowsOf[k * sb::kStatStride + 7]);
    if (best > 0.f) {
      std::uniform_real_distribution<float> draw(0.f, 1.f);
      std::vector<uint32_t> stay;
      for (size_t k = 0; k < listed.size(); ++k)
        if (!(draw(rng) > rowsOf[k * sb::kStatStride + 7] / best)) stay.push_back(listed[k]);
      SB_CUDA(cudaMemsetAsync(chosen.get(), 0, (size_t)n * 4, s));
      if (!stay.empty()) {
        SB_CUDA(cudaMemcpyAsync(list.get(), stay.data(), stay.size() * 4, cudaMemcpyHostToDevice, s));
        sb::launch_set_first(list.get<uint32_t>(), (uint32_t)stay.size(), 1u, chosen.get<uint32_t>(), s);
      }
      SB_CUDA(cudaStreamSynchronize(s));
      chosenCount = stay.size();
    }
  }
  sb::launch_densify_choose(scales, a, n, chosen.get<uint32_t>(), action.get<uint32_t>(), s);

  // Exploration (densify.cpp:207-224): of the large Gaussians left alone,
  // the larger half by summed log-scale, shuffled, and the first few split.
  uint64_t left = room - chosenCount, exploreSplits = 0;
  if (o.explore_splits > 0 && left > 0) {
    sb::launch_densify_large(scales, a, n, action.get<uint32_t>(), flags.get<uint32_t>(), s);
    run.scan(flags, place, 4);
    const uint32_t count = run.read()[17];
    sb::launch_compact(flags.get<uint32_t>(), place.get<uint32_t>(), nullptr, n, list.get<uint32_t>(), nullptr, s);
    const std::vector<uint32_t> listed = run.download(list.get<uint32_t>(), count);
    const std::vector<float> rowsOf = run.gather(list.get<int32_t>(), scales, count, 3);
    std::vector<float> sums(n);
    for (size_t k = 0; k < listed.size(); ++k) sums[listed[k]] = rowsOf[k * 3] + rowsOf[k * 3 + 1] + rowsOf[k * 3 + 2];
    std::vector<size_t> large(listed.begin(), listed.end());
    const auto middle = large.begin() + static_cast<std::ptrdiff_t>(large.size() / 2);
    std::nth_element(large.begin(), middle, large.end(), [&](size_t x, size_t y) { return sums[x] > sums[y]; });
    large.resize((large.size() + 1) / 2);
    std::shuffle(large.begin(), large.end(), rng);
    exploreSplits = std::min<uint64_t>({o.explore_splits, (uint64_t)large.size(), left});
    if (exploreSplits > 0) {
      std::vector<uint32_t> picked(large.begin(), large.begin() + static_cast<std::ptrdiff_t>(exploreSplits));
      SB_CUDA(cudaMemcpyAsync(list.get(), picked.data(), picked.size() * 4, cudaMemcpyHostToDevice, s));
      sb::launch_set_first(list.get<uint32_t>(), (uint32_t)picked.size(), sb::kDensifySplit, action.get<uint32_t>(), s);
      SB_CUDA(cudaStreamSynchronize(s));
    }
    left -= exploreSplits;
  }

  // Seeds (densify.cpp:226-251): the survivors' box and median mean
  // log-scale, from their rows.
  uint64_t seeded = std::min<uint64_t>(o.explore_seeds, left);
  std::vector<uint32_t> survivors;
  float low[3], high[3], seedScale = 0.f;
  if (seeded > 0) {
    if (keptCount == 0) {
      seeded = 0;
    } else {
      sb::launch_compact(kept.get<uint32_t>(), keptPlace.get<uint32_t>(), nullptr, n, list.get<uint32_t>(), nullptr, s);
      survivors = run.download(list.get<uint32_t>(), (uint32_t)keptCount);
      const std::vector<float> at = run.gather(list.get<int32_t>(), t->positions.get(), (uint32_t)keptCount, 3);
      const std::vector<float> sc = run.gather(list.get<int32_t>(), scales, (uint32_t)keptCount, 3);
      std::fill(low, low + 3, std::numeric_limits<float>::max());
      std::fill(high, high + 3, std::numeric_limits<float>::lowest());
      std::vector<float> means;
      means.reserve(survivors.size());
      for (size_t k = 0; k < survivors.size(); ++k) {
        for (size_t d = 0; d < 3; ++d) {
          low[d] = std::min(low[d], at[k * 3 + d]);
          high[d] = std::max(high[d], at[k * 3 + d]);
        }
        means.push_back((sc[k * 3] + sc[k * 3 + 1] + sc[k * 3 + 2]) / 3.f);
      }
      std::nth_element(means.begin(), means.begin() + static_cast<std::ptrdiff_t>(means.size() / 2), means.end());
      seedScale = means[means.size() / 2];
    }
  }

  // The new cloud's layout.
  const Slice &survivor = kept, &survivorPlace = keptPlace, &added = candidate, &addedPlace = candidatePlace;
  const Slice &patched = flags, &patchedPlace = place;
  sb::launch_densify_flags(n, action.get<uint32_t>(), survivor.get<uint32_t>(), added.get<uint32_t>(), patched.get<uint32_t>(), s);
  run.scan(survivor, survivorPlace, 5);
  run.scan(added, addedPlace, 6);
  run.scan(patched, patchedPlace, 7);
  c = run.read();
  const uint64_t survivorCount = c[21], addedCount = c[25], parentsCount = c[29];
  const uint64_t newCount = survivorCount + addedCount + seeded;
  if (newCount == 0) throw Failure{SPLAT_ERR_INVALID, "densification removed every Gaussian"};
  if (newCount > 0x7FFFFFFFull) throw Failure{SPLAT_ERR_INVALID, "densification would exceed 2^31 - 1 Gaussians"};
  const auto newN = (uint32_t)newCount;
  Arena tables(t->editTables, 2 * Arena::room((size_t)newN * 4));
  const Slice paramSource = tables.take((size_t)newN * 4), stateSource = tables.take((size_t)newN * 4);
  sb::launch_densify_tables(n, (uint32_t)survivorCount, action.get<uint32_t>(), survivorPlace.get<uint32_t>(),
                            addedPlace.get<uint32_t>(), patchedPlace.get<uint32_t>(), paramSource.get<int32_t>(),
                            stateSource.get<int32_t>(), parents.get<uint32_t>(), childSlot.get<uint32_t>(), s);

  // Split children (densify.cpp:264-299), in index order: samples of the
  // parent shrunk by 1.6, or two halves along the longest axis.
  std::vector<sb::DensifyPatch> rowsOut;
  const std::vector<uint32_t> parentList = run.download(parents.get<uint32_t>(), (uint32_t)parentsCount);
  const std::vector<uint32_t> slots = run.download(childSlot.get<uint32_t>(), (uint32_t)parentsCount);
  uint64_t splits = 0, longAxis = 0;
  if (parentsCount > 0) {
    const auto *listed = parents.get<int32_t>();
    const std::vector<float> at = run.gather(listed, t->positions.get(), (uint32_t)parentsCount, 3);
    const std::vector<float> sc = run.gather(listed, scales, (uint32_t)parentsCount, 3);
    const std::vector<float> rot = run.gather(listed, t->rotations.get(), (uint32_t)parentsCount, 4);
    const std::vector<float> op = run.gather(listed, t->opacities.get(), (uint32_t)parentsCount, 1);
    const std::vector<float> acts = run.gather(listed, action.get(), (uint32_t)parentsCount, 1);
    const float shrink = std::log(1.6f);
    for (size_t k = 0; k < parentList.size(); ++k) {
      uint32_t act;
      std::memcpy(&act, &acts[k], 4);
      float R[3][3];
      if (act == sb::kDensifySplit) {
        ++splits;
        for (uint32_t child = 0; child < 2; ++child) {
          sb::DensifyPatch q{};
          q.slot = slots[k] + child;
          std::normal_distribution<float> normal(0.f, 1.f);
          const float local[3] = {normal(rng) * std::exp(sc[k * 3]), normal(rng) * std::exp(sc[k * 3 + 1]),
                                  normal(rng) * std::exp(sc[k * 3 + 2])};
          rotation_matrix(&rot[k * 4], R);
          for (int r = 0; r < 3; ++r) {
            q.position[r] = at[k * 3 + r] + R[r][0] * local[0] + R[r][1] * local[1] + R[r][2] * local[2];
            q.scale[r] = sc[k * 3 + r] - shrink;
          }
          rowsOut.push_back(q);
        }
      } else {
        ++longAxis;
        // Tangent to the parent at its ends: 0.45 of the semi-axis out, 0.55
        // of it long, the other axes shrunk to stay inside, 0.6 of the opacity.
        constexpr float kOffset = 0.45f;
        const float *own = &sc[k * 3];
        const int axis = (int)(std::max_element(own, own + 3) - own);
        rotation_matrix(&rot[k * 4], R);
        const float length = std::exp(own[axis]);
        const double opacity = 0.6 * (1.f / (1.f + std::exp(-op[k])));
        const float sides[2] = {-1.f, 1.f};
        for (uint32_t child = 0; child < 2; ++child) {
          sb::DensifyPatch q{};
          q.slot = slots[k] + child;
          q.what = sb::kPatchOpacity;
          for (int d = 0; d < 3; ++d) {
            q.position[d] = at[k * 3 + d] + sides[child] * kOffset * length * R[d][axis];
            q.scale[d] = own[d] + (d == axis ? std::log(1.f - kOffset) : 0.5f * std::log(1.f - kOffset * kOffset));
          }
          q.opacity = static_cast<float>(std::log(opacity / (1.0 - opacity)));
          rowsOut.push_back(q);
        }
      }
    }
  }

  // Seeds: a random survivor's colour at a random place in the box, of the
  // median size, unrotated, opacity 0.1, the same colour from all sides.
  std::vector<int32_t> seedSources;
  for (uint64_t k = 0; k < seeded; ++k) {
    const size_t pick = std::uniform_int_distribution<size_t>(0, survivors.size() - 1)(rng);
    seedSources.push_back((int32_t)survivors[pick]);
    sb::DensifyPatch q{};
    q.slot = (uint32_t)(survivorCount + addedCount + k);
    q.what = sb::kPatchRotation | sb::kPatchOpacity | sb::kPatchShRest;
    for (int d = 0; d < 3; ++d) {
      q.position[d] = std::uniform_real_distribution<float>(low[d], high[d])(rng);
      q.scale[d] = seedScale;
    }
    q.rotation[0] = 1.f;
    q.opacity = std::log(0.1f / 0.9f);
    rowsOut.push_back(q);
  }
  if (!seedSources.empty()) {
    const std::vector<int32_t> fresh(seedSources.size(), -1);
    const size_t offset = (size_t)(survivorCount + addedCount) * 4;
    SB_CUDA(cudaMemcpyAsync(paramSource.get<uint8_t>() + offset, seedSources.data(), seedSources.size() * 4, cudaMemcpyHostToDevice, s));
    SB_CUDA(cudaMemcpyAsync(stateSource.get<uint8_t>() + offset, fresh.data(), fresh.size() * 4, cudaMemcpyHostToDevice, s));
  }
  if (!rowsOut.empty()) {
    sb::grow(t->editRows, rowsOut.size() * sizeof(sb::DensifyPatch));
    SB_CUDA(cudaMemcpyAsync(t->editRows.get(), rowsOut.data(), rowsOut.size() * sizeof(sb::DensifyPatch), cudaMemcpyHostToDevice, s));
  }
  std::vector<int32_t> table;
  if (source != nullptr && sourceCapacity >= newCount) {
    table.resize(newN);
    SB_CUDA(cudaMemcpyAsync(table.data(), stateSource.get(), (size_t)newN * 4, cudaMemcpyDeviceToHost, s));
  }
  SB_CUDA(cudaGetLastError());
  SB_CUDA(cudaStreamSynchronize(s));

  Trainer *fresh = regather(handle, paramSource.get<int32_t>(), stateSource.get<int32_t>(), newN);
  if (!rowsOut.empty()) {
    const uint32_t restPlanes = 3u * (uint32_t)(fresh->shCoeffs - 1);
    sb::launch_densify_patch(fresh->editRows.get<sb::DensifyPatch>(), (uint32_t)rowsOut.size(), fresh->positions.get<float>(),
                             fresh->scales.get<float>(), fresh->rotations.get<float>(), fresh->opacities.get<float>(),
                             fresh->shRest.get(), restPlanes, sb::sh_rest_stride(fresh->shCoeffs, fresh->shStore),
                             fresh->shStore == sb::ShStore::F32 ? 4u : 2u,
                             fresh->stream);
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaStreamSynchronize(fresh->stream));
  }
  for (size_t i = 0; i < table.size(); ++i) source[i] = table[i];
  if (result != nullptr) {
    result->count = newCount;
    result->cloned = addedCount - 2 * parentsCount;
    result->split = splits + longAxis;
    result->seeded = seeded;
    result->pruned = n - keptCount;
    result->held_back = heldBack;
  }
}


// f(begin, end) over [0, count), split across up to 16 host threads, each
// given at least `grain` items.
template <class F> void parallel_ranges(size_t count, F f, size_t grain = 32768) {
  const size_t cores = std::max(1u, std::thread::hardware_concurrency());
  const size_t threads = std::min<size_t>({cores, 16, std::max<size_t>(count / grain, 1)});
  if (threads <= 1) {
    f(size_t{0}, count);
    return;
  }
  const size_t chunk = (count + threads - 1) / threads;
  std::vector<std::thread> pool;
  for (size_t k = 0; k < threads && k * chunk < count; ++k) pool.emplace_back(f, k * chunk, std::min(count, (k + 1) * chunk));
  for (std::thread &t : pool) t.join();
}

// Draws of std::discrete_distribution<std::size_t> over `weights` (m of
// them, filled in by weight(k)), restated so that its parts that do not
// depend on each other run in parallel: the weights normalised by their sum,
// their running sum with the last entry set to 1, and per draw the first
// entry not below std::generate_canonical<double, 53> of the generator, the
// draws taken from it in order. With fewer than two weights every draw is 0
// and takes nothing from the generator. The search goes through the last
// entry of every block of 64 first, which finds the same entry with a few
// cache misses instead of twenty.
template <class W>
std::vector<size_t> discrete_draws(size_t m, W weight, size_t count, std::mt19937 &rng, std::vector<double> &cumulative,
                                   std::vector<double> &coarse) {
  std::vector<size_t> picks(count, 0);
  if (m < 2) return picks;
  cumulative.resize(m);
  parallel_ranges(m, [&](size_t b, size_t e) {
    for (size_t k = b; k < e; ++k) cumulative[k] = weight(k);
  });
  double sum = 0.0;
  for (size_t k = 0; k < m; ++k) sum += cumulative[k];
  parallel_ranges(m, [&](size_t b, size_t e) {
    for (size_t k = b; k < e; ++k) cumulative[k] = cumulative[k] / sum;
  });
  for (size_t k = 1; k < m; ++k) cumulative[k] = cumulative[k - 1] + cumulative[k];
  cumulative[m - 1] = 1.0;
  constexpr size_t kBlock = 64;
  const size_t blocks = (m + kBlock - 1) / kBlock;
  coarse.resize(blocks);
  for (size_t b = 0; b < blocks; ++b) coarse[b] = cumulative[std::min(m, (b + 1) * kBlock) - 1];
  std::vector<double> p(count);
  for (double &v : p) v = std::generate_canonical<double, std::numeric_limits<double>::digits>(rng);
  parallel_ranges(count, [&](size_t b, size_t e) {
    for (size_t j = b; j < e; ++j) {
      const size_t block = (size_t)(std::lower_bound(coarse.begin(), coarse.end(), p[j]) - coarse.begin());
      const auto from = cumulative.begin() + (ptrdiff_t)(block * kBlock);
      const auto to = cumulative.begin() + (ptrdiff_t)std::min(m, (block + 1) * kBlock);
      picks[j] = (size_t)(std::lower_bound(from, to, p[j]) - cumulative.begin());
    }
  }, 1024);
  return picks;
}

// Trainer::relocate on the GPU and the host (trainer.cpp:717-722;
// relocate_cloud, densify.cpp:328-420; apply_changes). The device splits the
// Gaussians into dead and alive and gathers the new cloud and its optimiser
// state; the draws (from rng in the reference's order) and the opacity and
// scale updates of the drawn targets run on the host, in parallel where
// they do not depend on each other, over the opacities and log-scales, the
// only values relocation changes, kept in pinned memory.
void relocate_gaussians(splat_trainer *handle, const splat_relocate_options &o, std::mt19937 &rng, splat_densify_result *result,
                        int64_t *source, uint64_t sourceCapacity) {
  Trainer *t = impl_of(handle);
  if (!(o.growth >= 0.0)) throw Failure{SPLAT_ERR_INVALID, "growth must not be negative"};
  SB_CUDA(cudaStreamSynchronize(t->stream));
  DensifyRun run(t, 5);
  cudaStream_t s = run.s;
  const uint32_t n = run.n;
  Slice dead = run.take(), alive = run.take(), deadPlace = run.take(), alivePlace = run.take(), list = run.take();
  sb::launch_relocate_flags(t->params(), logit_threshold_inclusive(o.min_opacity), dead.get<uint32_t>(), alive.get<uint32_t>(), s);
  run.scan(dead, deadPlace, 0);
  run.scan(alive, alivePlace, 1);
  const std::vector<uint32_t> c = run.read();
  const uint32_t deadCount = c[1], aliveCount = c[5];
  // Growth, fixed by the count alone (densify.cpp:389-390).
  const uint64_t room = o.max_gaussians > n ? o.max_gaussians - n : 0;
  const double share = o.growth * static_cast<double>(n);
  const uint64_t wanted = share >= static_cast<double>(room) ? room : std::min<uint64_t>(static_cast<size_t>(share), room);
  if (wanted + n > 0x7FFFFFFFull) throw Failure{SPLAT_ERR_INVALID, "relocation would exceed 2^31 - 1 Gaussians"};
  splat_densify_result counts{};
  counts.count = n;
  if (aliveCount == 0) {
    // Nothing to draw from: the cloud stays; its statistics start anew, as
    // apply_changes leaves them.
    SB_CUDA(cudaMemsetAsync(t->densifyStats.get(), 0, (size_t)n * sb::kStatStride * 4, s));
    SB_CUDA(cudaStreamSynchronize(s));
    if (source != nullptr && sourceCapacity >= n)
      for (uint32_t i = 0; i < n; ++i) source[i] = i;
    if (result != nullptr) *result = counts;
    return;
  }
  const size_t capacity = (size_t)n + wanted;
  const size_t hostBytes = capacity * 16 + (size_t)n * 8;
  if (t->editHost.bytes() < hostBytes) t->editHost.ensure(hostBytes + hostBytes / 4);
  float *opacity = t->editHost.get<float>();
  float *logScale = opacity + capacity;
  uint32_t *deadList = reinterpret_cast<uint32_t *>(logScale + capacity * 3);
  uint32_t *aliveList = deadList + n;
  sb::launch_compact(dead.get<uint32_t>(), deadPlace.get<uint32_t>(), nullptr, n, list.get<uint32_t>(), nullptr, s);
  if (deadCount > 0) SB_CUDA(cudaMemcpyAsync(deadList, list.get(), (size_t)deadCount * 4, cudaMemcpyDeviceToHost, s));
  sb::launch_compact(alive.get<uint32_t>(), alivePlace.get<uint32_t>(), nullptr, n, deadPlace.get<uint32_t>(), nullptr, s);
  SB_CUDA(cudaMemcpyAsync(aliveList, deadPlace.get(), (size_t)aliveCount * 4, cudaMemcpyDeviceToHost, s));
  SB_CUDA(cudaMemcpyAsync(opacity, t->opacities.get(), (size_t)n * 4, cudaMemcpyDeviceToHost, s));
  SB_CUDA(cudaMemcpyAsync(logScale, t->scales.get(), (size_t)n * 12, cudaMemcpyDeviceToHost, s));
  SB_CUDA(cudaGetLastError());
  SB_CUDA(cudaStreamSynchronize(s));

  // origin[k]: the old Gaussian whose position, rotation and SH slot k holds.
  std::vector<int32_t> &origin = t->editOrigin, &stateSource = t->editState;
  origin.resize(capacity);
  stateSource.resize(capacity);
  std::vector<int> &times = t->editTimes;
  times.resize(n);
  parallel_ranges(capacity, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      origin[i] = (int32_t)i;
      stateSource[i] = i < n ? (int32_t)i : -1;
    }
  });
  const auto sigmoid = [](float x) { return 1.f / (1.f + std::exp(-x)); };
  // A target drawn m times becomes m + 1 equal copies (at most 51): opacity
  // 1 - (1 - o)^(1/N) and scale times o / D, D the alternating binomial sum
  // of 3DGS-MCMC (densify.cpp:342-364). Each target's update is its own.
  const auto update_targets = [&](const std::vector<size_t> &targets) {
    std::fill(times.begin(), times.end(), 0);
    for (const size_t k : targets) ++times[k];
    parallel_ranges(n, [&](size_t b, size_t e) {
      for (size_t k = b; k < e; ++k) {
        if (times[k] == 0) continue;
        const int copies = std::min(times[k] + 1, 51);
        const double was = sigmoid(opacity[k]);
        const double fresh = 1.0 - std::pow(1.0 - was, 1.0 / copies);
        double divisor = 0.0;
        for (int i = 1; i <= copies; ++i) {
          double binom = 1.0;
          for (int j = 0; j < i; ++j) {
            if (j > 0) binom = binom * static_cast<double>(i - j) / j;
            divisor += binom * (j % 2 == 0 ? 1.0 : -1.0) * std::pow(fresh, j + 1) / std::sqrt(static_cast<double>(j + 1));
          }
        }
        const double clamped = std::clamp(fresh, static_cast<double>(o.min_opacity), 1.0 - 1e-6);
        opacity[k] = static_cast<float>(std::log(clamped / (1.0 - clamped)));
        const double factor = divisor > 0.0 ? was / divisor : 1.0;
        for (size_t a = 0; a < 3; ++a) logScale[k * 3 + a] += static_cast<float>(std::log(factor));
        stateSource[k] = -1;
      }
    });
  };
  const auto copy_into = [&](size_t from, size_t to) {
    origin[to] = origin[from];
    opacity[to] = opacity[from];
    for (size_t a = 0; a < 3; ++a) logScale[to * 3 + a] = logScale[from * 3 + a];
  };
  if (deadCount > 0) {
    std::vector<size_t> targets = discrete_draws(
        aliveCount, [&](size_t k) { return (double)sigmoid(opacity[aliveList[k]]); }, deadCount, rng, t->editCumulative,
        t->editCoarse);
    for (size_t &k : targets) k = aliveList[k];
    update_targets(targets);
    for (size_t j = 0; j < deadCount; ++j) {
      copy_into(targets[j], deadList[j]);
      stateSource[deadList[j]] = -1;
    }
    counts.cloned = deadCount;
  }
  if (wanted > 0) {
    const std::vector<size_t> targets = discrete_draws(n, [&](size_t k) { return (double)sigmoid(opacity[k]); }, wanted, rng,
                                                       t->editCumulative, t->editCoarse);
    update_targets(targets);
    for (size_t k = 0; k < targets.size(); ++k) copy_into(targets[k], n + k);
    counts.seeded = wanted;
  }
  const auto newN = (uint32_t)capacity;
  counts.count = newN;
  Arena tables(t->editTables, 2 * Arena::room((size_t)newN * 4));
  const Slice paramTable = tables.take((size_t)newN * 4), stateTable = tables.take((size_t)newN * 4);
  SB_CUDA(cudaMemcpyAsync(paramTable.get(), origin.data(), (size_t)newN * 4, cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaMemcpyAsync(stateTable.get(), stateSource.data(), (size_t)newN * 4, cudaMemcpyHostToDevice, s));
  SB_CUDA(cudaStreamSynchronize(s));
  Trainer *fresh = regather(handle, paramTable.get<int32_t>(), stateTable.get<int32_t>(), newN);
  SB_CUDA(cudaMemcpyAsync(fresh->opacities.get(), opacity, (size_t)newN * 4, cudaMemcpyHostToDevice, fresh->stream));
  SB_CUDA(cudaMemcpyAsync(fresh->scales.get(), logScale, (size_t)newN * 12, cudaMemcpyHostToDevice, fresh->stream));
  SB_CUDA(cudaStreamSynchronize(fresh->stream));
  if (source != nullptr && sourceCapacity >= newN)
    for (uint32_t k = 0; k < newN; ++k) source[k] = stateSource[k];
  if (result != nullptr) *result = counts;
}
} // namespace

extern "C" {

int splat_rng_create(uint32_t seed, splat_rng **out) {
  return guarded([&] {
    if (out == nullptr) throw Failure{SPLAT_ERR_INVALID, "null output"};
    *out = new splat_rng{std::mt19937(seed)};
  });
}

int splat_rng_destroy(splat_rng *rng) {
  delete rng;
  return SPLAT_OK;
}

int splat_rng_pick(splat_rng *rng, uint64_t count, uint64_t *out) {
  return guarded([&] {
    if (rng == nullptr || out == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    if (count == 0) throw Failure{SPLAT_ERR_INVALID, "nothing to pick from"};
    *out = std::uniform_int_distribution<size_t>(0, (size_t)count - 1)(rng->engine);
  });
}

void splat_densify_options_default(splat_densify_options *options) {
  if (options == nullptr) return;
  *options = splat_densify_options{};
  options->gradient_threshold = 2e-4f;
  options->dense_scale = 0.f;
  options->prune_opacity = 0.005f;
  options->prune_large = 0;
  options->max_screen_radius = 20.f;
  options->max_world_scale = 0.f;
  options->max_gaussians = UINT64_MAX;
  options->split_threshold = 0.f;
  options->scored_views = 0;
  options->min_marked_pixels = 5.f;
  options->transparent_share = 1.0;
  options->explore_splits = 0;
  options->explore_seeds = 0;
  options->edge_split = 0;
}

int splat_trainer_densify(splat_trainer *trainer, const splat_densify_options *options, splat_rng *rng,
                          splat_densify_result *result, int64_t *source, uint64_t source_capacity) {
  return guarded([&] {
    if (options == nullptr || rng == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    densify_gaussians(trainer, *options, rng->engine, result, source, source_capacity);
  });
}

void splat_relocate_options_default(splat_relocate_options *options) {
  if (options == nullptr) return;
  *options = splat_relocate_options{};
  options->min_opacity = 0.005f;
  options->growth = 0.05;
  options->max_gaussians = UINT64_MAX;
}

int splat_trainer_relocate(splat_trainer *trainer, const splat_relocate_options *options, splat_rng *rng,
                           splat_densify_result *result, int64_t *source, uint64_t source_capacity) {
  return guarded([&] {
    if (options == nullptr || rng == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    relocate_gaussians(trainer, *options, rng->engine, result, source, source_capacity);
  });
}

int splat_trainer_remove_largest(splat_trainer *trainer, double share, uint64_t *removed) {
  return guarded([&] {
    const uint64_t r = prune_gaussians(trainer, 0, share);
    if (removed != nullptr) *removed = r;
  });
}

int splat_trainer_remove_least_contributing(splat_trainer *trainer, double share, uint64_t *removed) {
  return guarded([&] {
    const uint64_t r = prune_gaussians(trainer, 1, share);
    if (removed != nullptr) *removed = r;
  });
}

int splat_trainer_remove_least_opaque(splat_trainer *trainer, double share, uint64_t *removed) {
  return guarded([&] {
    const uint64_t r = prune_gaussians(trainer, 2, share);
    if (removed != nullptr) *removed = r;
  });
}

int splat_trainer_set_exposure(splat_trainer *trainer, const float exposure[12]) {
  return guarded([&] {
    (void)impl_of(trainer);
    if (exposure == nullptr) throw Failure{SPLAT_ERR_INVALID, "null exposure"};
    static const float neutral[12] = {1.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f};
    for (int k = 0; k < 12; ++k)
      if (exposure[k] != neutral[k]) throw Failure{SPLAT_ERR_UNSUPPORTED, "exposure has no kernel in this library"};
  });
}

int splat_trainer_set_sh_dropout(splat_trainer *trainer, float probability, int32_t retained_degree, uint32_t seed) {
  return guarded([&] {
    (void)impl_of(trainer);
    (void)retained_degree;
    (void)seed;
    if (probability > 0.f) throw Failure{SPLAT_ERR_UNSUPPORTED, "SH dropout has no kernel in this library"};
  });
}

int splat_trainer_set_filter3d(splat_trainer *trainer, const float *filter, size_t count) {
  return guarded([&] {
    (void)impl_of(trainer);
    (void)filter;
    if (count != 0) throw Failure{SPLAT_ERR_UNSUPPORTED, "the 3D filter has no kernel in this library"};
  });
}

int splat_trainer_add_position_noise(splat_trainer *trainer, float scaler, uint32_t iteration) {
  return guarded([&] {
    (void)impl_of(trainer);
    (void)iteration;
    if (scaler != 0.f) throw Failure{SPLAT_ERR_UNSUPPORTED, "position noise has no kernel in this library"};
  });
}

int splat_trainer_enable_second_order(splat_trainer *trainer) {
  return guarded([&] {
    (void)impl_of(trainer);
    throw Failure{SPLAT_ERR_UNSUPPORTED, "second-order steps have no kernel in this library"};
  });
}

int splat_trainer_update_curvature(splat_trainer *trainer) {
  return guarded([&] {
    (void)impl_of(trainer);
    throw Failure{SPLAT_ERR_UNSUPPORTED, "second-order steps have no kernel in this library"};
  });
}

int splat_trainer_info(splat_trainer *trainer, int64_t *gaussians, int32_t *sh_degree, int32_t *active_sh_degree,
                       int32_t *uses_fixed_point, uint64_t *gpu_bytes, uint64_t *bytes_per_gaussian) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    if (gaussians) *gaussians = t->n;
    if (sh_degree) *sh_degree = t->shDegree;
    if (active_sh_degree) *active_sh_degree = t->activeDegree;
    if (uses_fixed_point) *uses_fixed_point = t->fixedPoint ? 1 : 0;
    if (gpu_bytes) *gpu_bytes = t->gpu_bytes();
    if (bytes_per_gaussian) *bytes_per_gaussian = t->bytes_per_gaussian();
  });
}

int splat_trainer_timings(splat_trainer *trainer, const char **names, double *ms, int32_t capacity, int32_t *count) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    if (count) *count = t->timedIterations > 0 ? sb::kStages : 0;
    if (t->timedIterations == 0) return;
    for (int s = 0; s < sb::kStages && s < capacity; ++s) {
      if (names) names[s] = sb::kStageNames[s];
      if (ms) ms[s] = t->stageTotals[s] / (double)t->timedIterations;
    }
  });
}

int splat_trainer_autotune(splat_trainer *trainer, const splat_camera *camera, const uint8_t *target, size_t target_bytes,
                           int32_t repeats, splat_autotune_result *result) {
  return guarded([&] {
    if (camera == nullptr || target == nullptr) throw Failure{SPLAT_ERR_INVALID, "null argument"};
    impl_of(trainer)->autotune(camera, target, target_bytes, repeats, result);
  });
}

int splat_trainer_set_timing(splat_trainer *trainer, int32_t enabled) {
  return guarded([&] { impl_of(trainer)->timing = enabled != 0; });
}

int splat_trainer_device_parameters(splat_trainer *trainer, int32_t group, uint64_t *device_address, uint64_t *bytes) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    const sb::DeviceBuffer *b[6] = {&t->positions, &t->scales, &t->rotations, &t->opacities, &t->shDc, &t->shRest};
    if (group < 0 || group > 5) throw Failure{SPLAT_ERR_INVALID, "group must be 0..5"};
    if (device_address) *device_address = (uint64_t)(uintptr_t)b[group]->get();
    if (bytes) *bytes = b[group]->bytes();
  });
}

int splat_trainer_debug_download(splat_trainer *trainer, int32_t which, void *out, size_t bytes, size_t *size) {
  return guarded([&] {
    Trainer *t = impl_of(trainer);
    SB_CUDA(cudaStreamSynchronize(t->stream));
    const size_t items = (size_t)t->n * std::max(t->views.count, 1);
    const void *src = nullptr;
    size_t have = 0;
    sb::StepReadback *rb = t->d_readback();
    switch (which) {
    case 0: src = t->splats.get(); have = items * sizeof(sb::Splat); break;
    case 1: src = t->reach.get(); have = items * 4; break;
    case 2:
      if (!t->oneSort) {
        // The depth sort permuted the keys in place: put them back in Gaussian order.
        const size_t n = t->n;
        std::vector<uint32_t> k(n), v(n), g(n);
        const uint32_t *sk = t->depthInTmp ? t->tmpKeys.get<uint32_t>() : t->depthKeys.get<uint32_t>();
        const uint32_t *sv = t->depthInTmp ? t->tmpValues.get<uint32_t>() : t->values.get<uint32_t>();
        SB_CUDA(cudaMemcpy(k.data(), sk, n * 4, cudaMemcpyDeviceToHost));
        SB_CUDA(cudaMemcpy(v.data(), sv, n * 4, cudaMemcpyDeviceToHost));
        for (size_t r = 0; r < n; ++r)
          if (v[r] < n) g[v[r]] = k[r];
        if (size) *size = n * 4;
        if (out != nullptr) std::memcpy(out, g.data(), std::min(bytes, n * 4));
        return;
      }
      src = t->depthKeys.get();
      have = items * 4;
      break;
    case 3: src = t->entriesInTmp ? t->tmpEntryKeys.get() : t->entryKeys.get(); have = (size_t)t->hReadback.get<sb::StepReadback>()->counters[2] * (t->oneSort ? 8 : 4); break;
    case 4: src = t->entriesInTmp ? t->tmpEntryValues.get() : t->entryValues.get(); have = (size_t)t->hReadback.get<sb::StepReadback>()->counters[2] * 4; break;
    case 5: src = t->ranges.get(); have = (size_t)t->views.totalTiles * 8; break;
    case 6: src = t->image.get(); have = (size_t)t->views.totalPixels * 16; break;
    case 7: src = t->stops.get(); have = (size_t)t->views.totalPixels * 4; break;
    case 8: src = t->adjoint.get(); have = (size_t)t->views.totalPixels * 16; break;
    case 9: src = t->raw.get(); have = items * sb::kRawStride * 4; break;
    case 10: src = rb->counters; have = 16; break;
    case 11: src = t->partials.get(); have = (size_t)t->views.totalLossTiles * 8; break;
    case 12: src = &rb->error; have = 4; break;
    case 13: src = t->listCounts.get(); have = t->blendLists ? (size_t)t->views.totalPixels * 4 : 0; break;
    case 19:
      src = t->ranges.get<uint2>() + t->views.totalTiles;
      have = (size_t)t->views.totalTiles * 8;
      break;
    case 14: case 15: case 16: case 17: case 18: {
      const size_t g = t->n;
      const size_t counts[5] = {g * 3, g * 3, g * 4, g, (size_t)t->planeStride * sb::sh_state_stride(t->shCoeffs)};
      src = t->state[which - 14].get();
      have = counts[which - 14] * (t->stateStore == sb::StateStore::F32 ? 8 : 4);
      break;
    }
    default: throw Failure{SPLAT_ERR_INVALID, "unknown buffer"};
    }
    if (size) *size = have;
    if (out != nullptr && bytes > 0 && src != nullptr) SB_CUDA(cudaMemcpy(out, src, std::min(bytes, have), cudaMemcpyDeviceToHost));
  });
}

int splat_radix_sort_u32(uint32_t *keys, uint32_t *values, uint32_t *tmp_keys, uint32_t *tmp_values, uint32_t count,
                         int32_t key_bits, int32_t digit_bits, void *stream) {
  return guarded([&] {
    if (key_bits < 1 || key_bits > 32) throw Failure{SPLAT_ERR_INVALID, "key_bits must be 1..32"};
    const int digits = digit_bits == 0 ? 8 : digit_bits;
    if (digits < 6 || digits > 8) throw Failure{SPLAT_ERR_INVALID, "digit_bits must be 6, 7 or 8"};
    if (!sb::sort_aligned(keys, values, tmp_keys, tmp_values))
      throw Failure{SPLAT_ERR_INVALID, "keys, values and temporaries must be 16-byte aligned"};
    if (count <= 1) return;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    sb::DeviceBuffer scratch, error;
    scratch.ensure(sb::sort_scratch_bytes(count, 4, key_bits, digits));
    error.ensure(4);
    SB_CUDA(cudaMemsetAsync(error.get(), 0, 4, s));
    const int where = sb::sort_pairs_u32(keys, values, tmp_keys, tmp_values, count, count, nullptr, 0, key_bits, digits,
                                         scratch.get(), error.get<uint32_t>(), s);
    SB_CUDA(cudaGetLastError());
    if (where == 1) {
      SB_CUDA(cudaMemcpyAsync(keys, tmp_keys, (size_t)count * 4, cudaMemcpyDeviceToDevice, s));
      SB_CUDA(cudaMemcpyAsync(values, tmp_values, (size_t)count * 4, cudaMemcpyDeviceToDevice, s));
    }
    uint32_t err = 0;
    SB_CUDA(cudaMemcpyAsync(&err, error.get(), 4, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    if (err != 0) throw Failure{SPLAT_ERR_DEVICE, "the sort's look-back gave up waiting"};
  });
}

int splat_radix_sort_u64(uint64_t *keys, uint32_t *values, uint64_t *tmp_keys, uint32_t *tmp_values, uint32_t count,
                         int32_t key_bits, int32_t digit_bits, void *stream) {
  return guarded([&] {
    if (key_bits < 1 || key_bits > 64) throw Failure{SPLAT_ERR_INVALID, "key_bits must be 1..64"};
    const int digits = digit_bits == 0 ? 8 : digit_bits;
    if (digits < 6 || digits > 8) throw Failure{SPLAT_ERR_INVALID, "digit_bits must be 6, 7 or 8"};
    if (!sb::sort_aligned(keys, values, tmp_keys, tmp_values))
      throw Failure{SPLAT_ERR_INVALID, "keys, values and temporaries must be 16-byte aligned"};
    if (count <= 1) return;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    sb::DeviceBuffer scratch, error;
    scratch.ensure(sb::sort_scratch_bytes(count, 8, key_bits, digits));
    error.ensure(4);
    SB_CUDA(cudaMemsetAsync(error.get(), 0, 4, s));
    auto *k = reinterpret_cast<unsigned long long *>(keys);
    auto *tk = reinterpret_cast<unsigned long long *>(tmp_keys);
    const int where = sb::sort_pairs_u64(k, values, tk, tmp_values, count, count, nullptr, 0, key_bits, digits, scratch.get(),
                                         error.get<uint32_t>(), s);
    SB_CUDA(cudaGetLastError());
    if (where == 1) {
      SB_CUDA(cudaMemcpyAsync(keys, tmp_keys, (size_t)count * 8, cudaMemcpyDeviceToDevice, s));
      SB_CUDA(cudaMemcpyAsync(values, tmp_values, (size_t)count * 4, cudaMemcpyDeviceToDevice, s));
    }
    uint32_t err = 0;
    SB_CUDA(cudaMemcpyAsync(&err, error.get(), 4, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    if (err != 0) throw Failure{SPLAT_ERR_DEVICE, "the sort's look-back gave up waiting"};
  });
}

int splat_debug_set_wait_limit(int32_t polls) {
  return guarded([&] { sb::set_lookback_limit(polls); });
}

int splat_debug_detmath(const float *in, float *out_exp, float *out_log, uint32_t count) {
  return guarded([&] {
    if (count == 0) return;
    sb::k_detmath<<<sb::div_up(count, 256), 256>>>(in, out_exp, out_log, count);
    SB_CUDA(cudaGetLastError());
    SB_CUDA(cudaDeviceSynchronize());
  });
}

} // extern "C"
