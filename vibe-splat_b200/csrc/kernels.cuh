// Launch wrappers of the training kernels (host side). Each names the
// reference shader it replaces.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace sb {

constexpr int kMaxViews = 8;
// Several views of one step. The rasterizer's tiles are tileSize x tileSize
// pixels (16, the reference's, or 32), numbered view by view from each view's
// tileBase; the loss works on its own grid of 16 x 16 tiles (lossTileBase,
// totalLossTiles), whatever the rasterizer's tile.
struct ViewSet {
  ViewParams v[kMaxViews];
  int count;
  int totalTiles;
  long long totalPixels;
  int tileSize;
  int totalLossTiles;
  // A one-view step on a target already in device memory reads it where the
  // caller keeps it (RGBA8, the view's width x height); null: the trainer's
  // own target buffer.
  const uint32_t *target;
};

// SH storage of the coefficients above degree 0 (the DC term is always FP32).
enum class ShStore : int { F32 = 0, BF16 = 1, F16 = 2 };
// Adam's moments: two FP32 words per parameter, or the reference's word of two
// bfloat16 (first moment rounded to nearest, second stochastically).
enum class StateStore : int { F32 = 0, BF16Pair = 1 };

// Trainable parameters, in this library's HBM layout: positions, log-scales and
// quaternions per Gaussian (12, 12, 16 bytes), opacity logits (4 bytes), SH DC
// planar: shDc[c * planeStride + i]; the higher SH coefficients in rows:
// shRest[i * restStride + (k - 1) * 3 + c], restStride = 3 (coeffs - 1)
// elements rounded up to 16 bytes (sh_rest_stride). planeStride is n rounded
// up to kPlaneAlign, and the rows count as many, so that a block of
// kPlaneAlign Gaussians starts every plane and its rows 16-byte aligned (bulk
// copies). The SH Adam state is in rows too (sh_state_at).
constexpr uint32_t kPlaneAlign = 128;

// Words in a Gaussian's row of SH Adam state: 3 coeffs, rounded up to 16 bytes.
__host__ __device__ inline uint32_t sh_state_stride(int shCoeffs) { return (3u * (uint32_t)shCoeffs + 3u) & ~3u; }

// Elements in a Gaussian's row of higher SH coefficients.
inline uint32_t sh_rest_stride(int shCoeffs, ShStore store) {
  const uint32_t elements = 3u * (uint32_t)(shCoeffs - 1), bytes = store == ShStore::F32 ? 4u : 2u;
  return elements == 0u ? 0u : (elements * bytes + 15u) / 16u * 16u / bytes;
}
struct Params {
  float *positions;
  float *scales;
  float *rotations;
  float *opacities;
  float *shDc;
  void *shRest;
  ShStore shStore;
  uint32_t n;
  uint32_t planeStride;
  uint32_t restStride; // elements per row of shRest
  int shDegree;
  int shCoeffs;
};

// train_preprocess.comp: projects every Gaussian into every view. Writes
// splats[v n + i], reach[v n + i], depthKeys[v n + i] (kInvisible, and a
// reach of minus infinity, when culled) and, if values is not null,
// values[v n + i] = i.
void launch_preprocess(const Params &p, const ViewSet &views, const ViewSet *dViews, Splat *splats, float *reach, uint32_t *depthKeys,
                       uint32_t *values, cudaStream_t stream, uint32_t *error = nullptr);

// train_bin_count.comp + record_scan(coverage): for every item r (a sorted
// splat in the depth-sorted form, v n + i in the single-sort form) counts the
// tiles the splat reaches and writes their exclusive scan to offsets[r].
// counters[0] += visible items, counters[1] = total entries, counters[2] =
// min(total, capacity). itemSplat: if not null, the splat of item r is
// itemSplat[r] (sorted values); itemKeys: kInvisible marks culled items
// (without keys, a reach of minus infinity does).
// masks[r]: the reached tiles of a rectangle of at most 32 tiles, bit
// (y - y0) * width + (x - x0), for the emission to replay (0 for larger ones).
void launch_bin_count_scan(const Splat *splats, const float *reach, const uint32_t *itemKeys, const uint32_t *itemSplat,
                           uint32_t items, uint32_t n, const ViewSet &views, const ViewSet *dViews, uint32_t *offsets, uint32_t *masks,
                           uint32_t *counters, uint32_t capacity, void *scratch, uint32_t *error, cudaStream_t stream);
size_t bin_scan_scratch_bytes(uint32_t items);
// The two halves of launch_bin_count_scan, for the depth-sorted form, whose
// counting runs per splat while the depth sort runs on another stream:
// counts[r] and masks[r] of item r; then offsets[r] = the exclusive scan of
// counts[gather[r]] (gather null: of counts[r]; counts may be offsets), with
// counters[1], counters[2] and the overflow bit as above.
void launch_bin_count(const Splat *splats, const float *reach, const uint32_t *itemKeys, const uint32_t *itemSplat, uint32_t items,
                      uint32_t n, const ViewSet &views, const ViewSet *dViews, uint32_t *counts, uint32_t *masks, uint32_t *counters,
                      cudaStream_t stream,
                      uint32_t blocksPerSm = 0);
// clearScratch false: the caller cleared scratch (bin_scan_scratch_bytes) already.
void launch_offsets_scan(uint32_t items, const uint32_t *counts, const uint32_t *gather, uint32_t *offsets, uint32_t *counters,
                         uint32_t capacity, void *scratch, uint32_t *error, cudaStream_t stream, bool clearScratch = true);

// train_bin_emit.comp. Depth-sorted form: tileKeys32[slot] = tile, entryValues[slot]
// = splat. Single-sort form (tileKeys64 not null): tileKeys64[slot] = (global
// tile << 32) | depth key. masks are indexed by item, or by splat with
// masksBySplat (a count that ran per splat).
void launch_bin_emit(const Splat *splats, const float *reach, const uint32_t *itemKeys, const uint32_t *itemSplat,
                     uint32_t items, uint32_t n, const ViewSet &views, const ViewSet *dViews, const uint32_t *offsets,
                     const uint32_t *masks, bool masksBySplat, uint32_t capacity, uint32_t *tileKeys32, unsigned long long *tileKeys64,
                     uint32_t *entryValues, uint32_t *error, cudaStream_t stream);

// train_tile_ranges.comp over the sorted keys; ranges (2 u32 per global tile)
// must be cleared first. count is read from deviceCount.
void launch_tile_ranges(const uint32_t *tileKeys32, const unsigned long long *tileKeys64, const uint32_t *deviceCount,
                        uint32_t capacity, uint32_t tileLimit, uint2 *ranges, uint32_t *error, cudaStream_t stream);

// The tiles of a launch, heaviest first, into order (tiles entries): the work
// of tile i is tileWork[i], or, without tileWork, the length of ranges[i].
void launch_tile_order(const uint2 *ranges, const uint32_t *tileWork, uint32_t tiles, uint32_t *order, cudaStream_t stream);

// Per-pixel blend lists of the store-everything variant: counts[p] splats
// blended at pixel p, recorded front to back at pool[offsets[p] ...] as
// (entry index, alpha bits).
struct BlendLists {
  uint32_t *counts = nullptr;
  const uint32_t *offsets = nullptr;
  uint2 *pool = nullptr;
};

struct RasterConfig {
  int exactMath = 1;   // deterministic exp/log (bit-reproducible by the CPU restatement)
  // Pixels per thread. 1: the reference's 2x16-pixel warps; 2: 8x8-pixel warps, two pixels per lane.
  int forwardPixels = 1;
  int backwardPixels = 2; // float backward only; the fixed-point sums keep 1
  float background[3] = {0.f, 0.f, 0.f};
  // The two-pixel kernels' tile edge (16 or 32; views.tileSize must agree)
  // and batch depth (splats staged per round: 128 or 256), and, for a
  // persistent launch, each kernel's tile counter (zeroed before the launch;
  // null: one block per tile).
  int tile = 16;
  int batch = 256;
  uint32_t *workForward = nullptr;
  uint32_t *workBackward = nullptr;
  // The two-pixel kernels' tile orders, heaviest first (launch_tile_order;
  // null: raster order), and where the two-pixel compositing records each
  // tile's work for the backward's order (null: not recorded).
  const uint32_t *orderForward = nullptr;
  const uint32_t *orderBackward = nullptr;
  uint32_t *tileWork = nullptr;
  // The two-pixel float backward's sums: a butterfly per (splat, warp), or,
  // twoPhase, splat-parallel per group of splats (not for scored views).
  bool twoPhase = false;
};

// train_forward.comp: one block per tile of 16x16 pixels. image: 4 floats per
// pixel (rgb, log transmittance), stops: 1 u32 per pixel, both indexed by
// view pixelBase + y W + x.
// listMode 1 also counts each pixel's blended splats into lists.counts, 2
// also records them (store-everything variant; one pixel per thread).
void launch_forward(const Splat *splats, const uint32_t *entryValues, const uint2 *ranges, const ViewSet &views, const ViewSet *dViews,
                    const RasterConfig &cfg, float4 *image, uint32_t *stops, uint32_t splatLimit, uint32_t *error,
                    cudaStream_t stream, int listMode = 0, BlendLists lists = BlendLists{});

// train_ssim.comp + train_loss.comp: SSIM fields, then the adjoint and L1.
// partials: 2 floats per global loss tile (SSIM sum, L1 sum).
void launch_ssim(const float4 *image, const uint32_t *target, const ViewSet &views, const ViewSet *dViews, float4 *fields, float2 *partials,
                 cudaStream_t stream);
// A scored view (Trainer::score_view): with edge not null the loss also leaves
// each pixel's mean absolute error in the adjoint's alpha, the view's worst
// error (in 1/65535) in *errorMax (cleared by the caller) and the target's
// edge weight in edge (one float per pixel).
struct LossScoring {
  float *edge = nullptr;
  uint32_t *errorMax = nullptr;
};
void launch_loss(const float4 *image, const uint32_t *target, const float4 *fields, const ViewSet &views, const ViewSet *dViews, float lambda,
                 float4 *adjoint, float2 *partials, cudaStream_t stream, LossScoring scoring = LossScoring{});
// train_error_mask.comp over one view's pixels: the adjoint's alpha becomes 1
// where the error is at least `share` of the worst, else 0.
void launch_error_mask(float4 *adjoint, uint32_t pixels, const uint32_t *errorMax, float share, cudaStream_t stream);
// FP64 sums of the per-tile partials into stats (see LossTotals).
struct LossTotals {
  double ssimSum[kMaxViews];
  double l1Sum[kMaxViews];
};
void launch_loss_totals(const float2 *partials, const ViewSet &views, const ViewSet *dViews, LossTotals *totals, cudaStream_t stream);

// train_backward_{fixed,float}.comp: raw sums, kRawStride per splat per view
// (int32 fixed point with each view's fixedScale, or float).
// With edge not null (a scored view, Trainer::score_view) also values 12 and
// 13: the pixels marked in the adjoint's alpha, and the edge weight (one
// float per pixel) times the blending weight, each over 3 pixels.
void launch_backward(const Splat *splats, const uint32_t *entryValues, const uint2 *ranges, const ViewSet &views, const ViewSet *dViews,
                     const RasterConfig &cfg, const float4 *image, const float4 *adjoint, const uint32_t *stops,
                     bool fixedPoint, void *raw, uint32_t splatLimit, uint32_t *error, cudaStream_t stream,
                     const float *edge = nullptr);
// The store-everything backward: float sums from the recorded blend lists.
void launch_backward_lists(const Splat *splats, const uint32_t *entryValues, const uint2 *ranges, const ViewSet &views,
                           const ViewSet *dViews, const RasterConfig &cfg, const float4 *image, const float4 *adjoint,
                           const uint32_t *stops, BlendLists lists, float *raw, uint32_t splatLimit, uint32_t *error,
                           cudaStream_t stream);
// Exclusive scan of `items` u32 values in place; *total gets their sum.
// scratch: bin_scan_scratch_bytes(items) bytes.
void launch_exclusive_scan(uint32_t items, uint32_t *values, uint32_t *counters, void *scratch, uint32_t *error,
                           cudaStream_t stream);

// train_gradient.comp + train_sh_step.comp: the chain rule from the raw sums of
// every view, then (mode) gradients stored, or Adam's step. shGrad holds 2
// float4 per (view, Gaussian) between the two kernels.
enum class ChainMode : int { Statistics = 0, Gradients = 1, Step = 2 };
struct ChainArgs {
  ChainMode mode;
  bool statistics;     // add to the densification statistics
  bool selective;      // Adam leaves parameters without a gradient alone
  bool fixedPoint;
  float rates[5];      // position, scale, rotation, opacity, SH
  float restScale;
  float beta1, beta2, epsilon, correction1, correction2;
  uint32_t seed;
  float opacityReg, scaleReg; // per Gaussian: the option over the count
  bool splitStep;      // host side: three kernels even for one view
};
struct OptimState {
  void *state[5];      // per group: F32 {m, v} pairs or BF16 pair words
  StateStore store;
};
struct GradientsOut {
  float *g[5];         // positions, scales, rotations, opacities, sh (GaussianCloud layout)
};
// train_score.comp after a scored view: densifyStats[i * 8 + 5..7] += marked
// pixels, marked pixels times the loss, edge score (raw values 12 and 13 of n
// Gaussians, int32 fixed point with fixedScale or float, times toPixels).
void launch_score(const void *raw, bool fixedPoint, float fixedScale, uint32_t n, float toPixels, float loss, float *densifyStats,
                  cudaStream_t stream);
void launch_chain(const Params &p, const ViewSet &views, const ViewSet *dViews, const void *raw, const Splat *splats, const ChainArgs &args,
                  const ChainArgs *dArgs, OptimState &state, const GradientsOut *grads, float4 *shGrad,
                  float *densifyStats, uint32_t *error, cudaStream_t stream);
// Blocks of `threads` threads of `kernel` resident on the whole GPU at once.
uint32_t resident_blocks(const void *kernel, int threads);

// train_gather.comp: optimiser state of the new Gaussians from the old ones
// through a source table (negative: fresh, zero state). Rows: `stride` words
// per Gaussian, `copies` consecutive copies of the layout (2 for F32 m and v).
// Planes: `planes` planes of one word per Gaussian, newStride / oldStride apart.
void launch_gather_rows(const int32_t *source, const uint32_t *in, uint32_t *out, uint32_t newCount, uint32_t oldCount,
                        uint32_t stride, uint32_t copies, cudaStream_t stream,
                        uint32_t valid = 0xFFFFFFFFu);
void launch_gather_planes(const int32_t *source, const uint32_t *in, uint32_t *out, uint32_t newCount, uint32_t newStride,
                          uint32_t oldStride, uint32_t planes, cudaStream_t stream);
void launch_gather_planes16(const int32_t *source, const uint16_t *in, uint16_t *out, uint32_t newCount, uint32_t newStride,
                            uint32_t oldStride, uint32_t planes, cudaStream_t stream);

// Pruning on the GPU (remove_highest, src/train/densify.cpp:70-90): keys whose
// ascending stable sort puts first the Gaussians to remove (kind 0 largest
// log-scale, 1 least contribution, 2 least opacity), values = indices; then
// keep flags from the sorted order, and the survivors' source table from the
// exclusive scan of the flags.
void launch_prune_keys(int kind, const float *scales, const float *opacities, const float *densifyStats, uint32_t n, uint32_t *keys,
                       uint32_t *values, cudaStream_t stream);
void launch_prune_keep(const uint32_t *order, uint32_t removed, uint32_t n, uint32_t *keep, cudaStream_t stream);
void launch_survivor_sources(const uint32_t *keep, const uint32_t *place, uint32_t n, int32_t *source, cudaStream_t stream);

// Adaptive density control (densify_cloud, densify.cpp:115-326). Actions
// per Gaussian, and the options the kernels read. worldLog and denseLog are
// the smallest largest-log-scales whose exp exceeds max_world_scale and the
// dense scale (NaN: none does); opacityLogit the smallest logit whose
// sigmoid is not below the opacity limit.
enum : uint32_t { kDensifyKeep = 0, kDensifyPrune = 1, kDensifyClone = 2, kDensifySplit = 3, kDensifyLongAxis = 4 };
struct DensifyArgs {
  float gradientThreshold, splitThreshold, maxScreenRadius, minMarkedPixels;
  float worldLog, denseLog, opacityLogit;
  int pruneLarge, scoredViews, allTransparent, edgeSplit;
};
// A row computed on the host for a new Gaussian's slot.
enum : uint32_t { kPatchRotation = 1, kPatchOpacity = 2, kPatchShRest = 4 };
struct DensifyPatch {
  uint32_t slot, what;
  float position[3], scale[3], rotation[4], opacity;
};
// action = prune (oversized, non-finite, or too transparent when all such go)
// or keep; transparent flags the too transparent otherwise, with the
// ascending sort key of their share.
void launch_densify_classify(const Params &p, const float *stats, const DensifyArgs &a, uint32_t *action, uint32_t *transparent,
                             uint32_t *transparentKey, cudaStream_t stream);
// kept, candidate flags and the ascending sort key of the candidates' priority.
void launch_densify_candidates(const float *scales, const float *stats, const DensifyArgs &a, uint32_t n, const uint32_t *action,
                               uint32_t *kept, uint32_t *candidate, uint32_t *priorityKey, cudaStream_t stream);
// flag[order[r]] = value for r < count.
void launch_set_first(const uint32_t *order, uint32_t count, uint32_t value, uint32_t *flag, cudaStream_t stream);
// out[place[i]] = i, keysOut[place[i]] = keys[i] (if keysOut) where flag[i].
void launch_compact(const uint32_t *flag, const uint32_t *place, const uint32_t *keys, uint32_t n, uint32_t *out, uint32_t *keysOut,
                    cudaStream_t stream);
// The chosen candidates' actions: long-axis split, split or clone.
void launch_densify_choose(const float *scales, const DensifyArgs &a, uint32_t n, const uint32_t *chosen, uint32_t *action,
                           cudaStream_t stream);
// Flags the kept Gaussians larger than the dense scale.
void launch_densify_large(const float *scales, const DensifyArgs &a, uint32_t n, const uint32_t *action, uint32_t *large,
                          cudaStream_t stream);
// Survivor, added-slot and patched-children flags from the actions.
void launch_densify_flags(uint32_t n, const uint32_t *action, uint32_t *survivor, uint32_t *added, uint32_t *patched,
                          cudaStream_t stream);
// The new cloud's parameter and state source tables, the split parents in
// index order and their first child's slot.
void launch_densify_tables(uint32_t n, uint32_t survivors, const uint32_t *action, const uint32_t *survivorPlace,
                           const uint32_t *addedPlace, const uint32_t *patchedPlace, int32_t *paramSource, int32_t *stateSource,
                           uint32_t *parents, uint32_t *childSlot, cudaStream_t stream);
// Relocation (relocate_cloud, densify.cpp:328-420): dead and alive flags,
// dead where the logit is below deadLogit or a value is not finite.
void launch_relocate_flags(const Params &p, float deadLogit, uint32_t *dead, uint32_t *alive, cudaStream_t stream);
// Writes host-computed rows into their slots (shRest: rows of restStride
// elements of shBytes bytes, the first restElements in use).
void launch_densify_patch(const DensifyPatch *patches, uint32_t count, float *positions, float *scales, float *rotations,
                          float *opacities, void *shRest, uint32_t restElements, uint32_t restStride, uint32_t shBytes,
                          cudaStream_t stream);

// The coarse-to-fine schedule's device work (csrc/schedule.cu).
// half_size (train.cpp:232-255): out is (width / 2) x (height / 2) RGBA8.
void launch_half_size(const uint8_t *in, int width, int height, uint8_t *out, cudaStream_t stream);
// frequency_energy (schedule.cpp:41-75) of an RGBA8 image on the device:
// partials gets blocks x count sums (summed by the caller) for count <= 8
// factors; scratch: spectrum_scratch_bytes; sizes up to 4096.
size_t spectrum_scratch_bytes(int width, int height);
bool spectrum_supported(int width, int height);
void launch_frequency_energy(const uint8_t *rgba, int width, int height, const int *factors, int count, void *scratch, double *partials,
                             int blocks, cudaStream_t stream);
// neighbour_distances (train.cpp:143-189) of n host points (3 doubles each)
// on the grid of `cell` from `low` with `dims` cells per axis; out (device)
// gets the float distances. scratch: neighbour_scratch_bytes(n).
size_t neighbour_scratch_bytes(uint32_t n);
int neighbour_distances(const double *points, uint32_t n, double3 low, double cell, int3 dims, void *scratch, float *out, uint32_t *error,
                        cudaStream_t stream);

} // namespace sb

