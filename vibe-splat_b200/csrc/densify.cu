// Adaptive density control on the GPU (densify_cloud, src/train/densify.cpp
// :115-326): the per-Gaussian decisions, the two global selections (which of
// the too transparent go when only a share of them does, which candidates
// stay when the count limit holds some back) as stable radix sorts over
// compacted lists, and the tables the new cloud and its optimiser state are
// gathered through. The comparisons against exp(largest log-scale) and
// sigmoid(opacity logit) are made against thresholds the host derives from
// the host's own exp, so that they decide as the reference's CPU code does
// bit for bit (densify_thresholds in trainer.cu). The random draws (split
// children, edge splits, exploration) stay on the host in the reference's
// order; only their few rows are patched in here.
#include "kernels.cuh"
#include "shmath.cuh"

namespace sb {

namespace {

// The float's order as unsigned order; both zeros count as one.
__device__ __forceinline__ uint32_t ordered(float f) {
  if (f == 0.0f) f = 0.0f;
  const uint32_t bits = __float_as_uint(f);
  return bits ^ ((bits >> 31) != 0u ? 0xFFFFFFFFu : 0x80000000u);
}

__device__ __forceinline__ float largest_log(const float *scales, uint32_t i) {
  return fmaxf(fmaxf(scales[(size_t)i * 3], scales[(size_t)i * 3 + 1]), scales[(size_t)i * 3 + 2]);
}

// Every value finite; all loads issued before any test, so that they overlap.
template <ShStore S> __device__ bool finite_gaussian(const Params &p, uint32_t i) {
  bool ok = isfinite(p.opacities[i]);
#pragma unroll
  for (int a = 0; a < 3; ++a) ok &= isfinite(p.positions[(size_t)i * 3 + a]) & isfinite(p.scales[(size_t)i * 3 + a]);
#pragma unroll
  for (int a = 0; a < 4; ++a) ok &= isfinite(p.rotations[(size_t)i * 4 + a]);
#pragma unroll
  for (int c = 0; c < 3; ++c) ok &= isfinite(p.shDc[(size_t)c * p.planeStride + i]);
  for (int k = 1; k < p.shCoeffs; ++k) {
#pragma unroll
    for (int c = 0; c < 3; ++c) ok &= isfinite(sh_coefficient<S>(p, i, k, c));
  }
  return ok;
}

// First pass (densify.cpp:132-141): oversized or non-finite Gaussians are
// pruned; of the rest, those below the opacity limit are too transparent:
// pruned at once when all of them go, else flagged with the key their share
// is chosen by (worst first: the most marked loss when views were scored,
// else the least contribution).
template <ShStore S>
__global__ void __launch_bounds__(256) k_densify_classify(Params p, const float *__restrict__ stats, DensifyArgs a,
                                                          uint32_t *__restrict__ action, uint32_t *__restrict__ transparent,
                                                          uint32_t *__restrict__ transparentKey) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  const float *st = stats + (size_t)i * kStatStride;
  const bool oversized = a.pruneLarge != 0 && (st[2] > a.maxScreenRadius || largest_log(p.scales, i) >= a.worldLog);
  bool clear = false;
  uint32_t act = kDensifyKeep;
  if (oversized || !finite_gaussian<S>(p, i)) {
    act = kDensifyPrune;
  } else if (p.opacities[i] < a.opacityLogit) {
    if (a.allTransparent != 0) act = kDensifyPrune;
    else clear = true;
  }
  action[i] = act;
  transparent[i] = clear ? 1u : 0u;
  transparentKey[i] = a.scoredViews > 0 ? ~ordered(st[6]) : ordered(st[3]);
}

// Candidates (densify.cpp:151-168) among the Gaussians not pruned: the
// gradient (for a large one when the split threshold is set, the gradient
// that does not cancel) per visit at or above its limit, with the key of the
// priority the count limit ranks them by (highest first). kept flags the
// unpruned.
__global__ void __launch_bounds__(256) k_densify_candidates(const float *__restrict__ scales, const float *__restrict__ stats,
                                                            DensifyArgs a, uint32_t n, const uint32_t *__restrict__ action,
                                                            uint32_t *__restrict__ kept, uint32_t *__restrict__ candidate,
                                                            uint32_t *__restrict__ priorityKey) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float *st = stats + (size_t)i * kStatStride;
  const bool live = action[i] != kDensifyPrune;
  bool chosen = false;
  float priority = 0.0f;
  if (live && !(st[1] <= 0.0f) && !(a.scoredViews > 0 && st[5] / (float)a.scoredViews <= a.minMarkedPixels)) {
    const bool splitsAlone = a.splitThreshold > 0.0f && largest_log(scales, i) >= a.denseLog;
    const float value = (splitsAlone ? st[4] : st[0]) / st[1];
    const float limit = splitsAlone ? a.splitThreshold : a.gradientThreshold;
    if (value >= limit) {
      chosen = true;
      priority = limit > 0.0f ? value / limit : value;
    }
  }
  kept[i] = live ? 1u : 0u;
  candidate[i] = chosen ? 1u : 0u;
  priorityKey[i] = ~ordered(priority);
}

// flag[order[r]] = value for r < count.
__global__ void __launch_bounds__(256) k_set_first(const uint32_t *__restrict__ order, uint32_t count, uint32_t value,
                                                   uint32_t *__restrict__ flag) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < count) flag[order[r]] = value;
}

// out[place[i]] = i (and keysOut[place[i]] = keys[i]) where flag[i] is set.
__global__ void __launch_bounds__(256) k_compact(const uint32_t *__restrict__ flag, const uint32_t *__restrict__ place,
                                                 const uint32_t *__restrict__ keys, uint32_t n, uint32_t *__restrict__ out,
                                                 uint32_t *__restrict__ keysOut) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || flag[i] == 0u) return;
  out[place[i]] = i;
  if (keysOut != nullptr) keysOut[place[i]] = keys[i];
}

// The chosen candidates' actions (densify.cpp:191-205): with edge splits a
// split along the longest axis, else a split where the Gaussian is larger
// than the dense scale and a clone where not.
__global__ void __launch_bounds__(256) k_densify_choose(const float *__restrict__ scales, DensifyArgs a, uint32_t n,
                                                        const uint32_t *__restrict__ chosen, uint32_t *__restrict__ action) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || chosen[i] == 0u) return;
  action[i] = a.edgeSplit != 0 ? kDensifyLongAxis : largest_log(scales, i) >= a.denseLog ? kDensifySplit : kDensifyClone;
}

// Exploration's pool (densify.cpp:210-213): the Gaussians left alone that
// are larger than the dense scale.
__global__ void __launch_bounds__(256) k_densify_large(const float *__restrict__ scales, DensifyArgs a, uint32_t n,
                                                       const uint32_t *__restrict__ action, uint32_t *__restrict__ large) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  large[i] = action[i] == kDensifyKeep && largest_log(scales, i) >= a.denseLog ? 1u : 0u;
}

// What each Gaussian adds to the new cloud: a survivor slot (kept or
// cloned), new slots (1 for a clone, 2 for either split) and whether its
// children are patched (both splits).
__global__ void __launch_bounds__(256) k_densify_flags(uint32_t n, const uint32_t *__restrict__ action,
                                                       uint32_t *__restrict__ survivor, uint32_t *__restrict__ added,
                                                       uint32_t *__restrict__ patched) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t act = action[i];
  const bool splits = act == kDensifySplit || act == kDensifyLongAxis;
  survivor[i] = act == kDensifyKeep || act == kDensifyClone ? 1u : 0u;
  added[i] = act == kDensifyClone ? 1u : splits ? 2u : 0u;
  patched[i] = splits ? 1u : 0u;
}

// The new cloud (densify.cpp:262-300): survivors first in their order, then,
// in index order, a copy per clone and two children per split. paramSource
// gives each new Gaussian the old one its parameters come from; stateSource
// the old one whose optimiser state it keeps (-1 for new ones). The split
// parents are listed in index order with their first child's slot.
__global__ void __launch_bounds__(256) k_densify_tables(uint32_t n, uint32_t survivors, const uint32_t *__restrict__ action,
                                                        const uint32_t *__restrict__ survivorPlace,
                                                        const uint32_t *__restrict__ addedPlace,
                                                        const uint32_t *__restrict__ patchedPlace, int32_t *__restrict__ paramSource,
                                                        int32_t *__restrict__ stateSource, uint32_t *__restrict__ parents,
                                                        uint32_t *__restrict__ childSlot) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t act = action[i];
  if (act == kDensifyKeep || act == kDensifyClone) {
    paramSource[survivorPlace[i]] = (int32_t)i;
    stateSource[survivorPlace[i]] = (int32_t)i;
  }
  const uint32_t at = survivors + addedPlace[i];
  if (act == kDensifyClone) {
    paramSource[at] = (int32_t)i;
    stateSource[at] = -1;
  } else if (act == kDensifySplit || act == kDensifyLongAxis) {
    for (uint32_t c = 0; c < 2; ++c) {
      paramSource[at + c] = (int32_t)i;
      stateSource[at + c] = -1;
    }
    parents[patchedPlace[i]] = i;
    childSlot[patchedPlace[i]] = at;
  }
}

// Rows the host computed (split children, seeds) into their slots of the
// new cloud: position and log-scales always, the rotation and opacity logit
// and a zero SH rest where asked.
__global__ void __launch_bounds__(128) k_densify_patch(const DensifyPatch *__restrict__ patches, uint32_t count, float *positions,
                                                       float *scales, float *rotations, float *opacities, void *shRest,
                                                       uint32_t restElements, uint32_t restStride, uint32_t shBytes) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const DensifyPatch q = patches[k];
  const size_t at = q.slot;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    positions[at * 3 + a] = q.position[a];
    scales[at * 3 + a] = q.scale[a];
  }
  if ((q.what & kPatchRotation) != 0u) {
#pragma unroll
    for (int a = 0; a < 4; ++a) rotations[at * 4 + a] = q.rotation[a];
  }
  if ((q.what & kPatchOpacity) != 0u) opacities[at] = q.opacity;
  if ((q.what & kPatchShRest) != 0u) {
    for (uint32_t element = 0; element < restElements; ++element) {
      const size_t e = at * restStride + element;
      if (shBytes == 4) static_cast<float *>(shRest)[e] = 0.0f;
      else static_cast<uint16_t *>(shRest)[e] = 0;
    }
  }
}


// Relocation's split (relocate_cloud, densify.cpp:335-337): dead where the
// opacity is at or below the limit (the logit below deadLogit) or a value is
// not finite; alive otherwise.
template <ShStore S>
__global__ void __launch_bounds__(256) k_relocate_flags(Params p, float deadLogit, uint32_t *__restrict__ dead,
                                                        uint32_t *__restrict__ alive) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  const bool gone = !finite_gaussian<S>(p, i) || p.opacities[i] < deadLogit;
  dead[i] = gone ? 1u : 0u;
  alive[i] = gone ? 0u : 1u;
}

} // namespace

void launch_densify_classify(const Params &p, const float *stats, const DensifyArgs &a, uint32_t *action, uint32_t *transparent,
                             uint32_t *transparentKey, cudaStream_t stream) {
  if (p.n == 0) return;
  const uint32_t blocks = div_up(p.n, 256);
  switch (p.shStore) {
  case ShStore::BF16: k_densify_classify<ShStore::BF16><<<blocks, 256, 0, stream>>>(p, stats, a, action, transparent, transparentKey); break;
  case ShStore::F16: k_densify_classify<ShStore::F16><<<blocks, 256, 0, stream>>>(p, stats, a, action, transparent, transparentKey); break;
  default: k_densify_classify<ShStore::F32><<<blocks, 256, 0, stream>>>(p, stats, a, action, transparent, transparentKey); break;
  }
}

void launch_relocate_flags(const Params &p, float deadLogit, uint32_t *dead, uint32_t *alive, cudaStream_t stream) {
  if (p.n == 0) return;
  const uint32_t blocks = div_up(p.n, 256);
  switch (p.shStore) {
  case ShStore::BF16: k_relocate_flags<ShStore::BF16><<<blocks, 256, 0, stream>>>(p, deadLogit, dead, alive); break;
  case ShStore::F16: k_relocate_flags<ShStore::F16><<<blocks, 256, 0, stream>>>(p, deadLogit, dead, alive); break;
  default: k_relocate_flags<ShStore::F32><<<blocks, 256, 0, stream>>>(p, deadLogit, dead, alive); break;
  }
}

void launch_densify_candidates(const float *scales, const float *stats, const DensifyArgs &a, uint32_t n, const uint32_t *action,
                               uint32_t *kept, uint32_t *candidate, uint32_t *priorityKey, cudaStream_t stream) {
  if (n == 0) return;
  k_densify_candidates<<<div_up(n, 256), 256, 0, stream>>>(scales, stats, a, n, action, kept, candidate, priorityKey);
}

void launch_set_first(const uint32_t *order, uint32_t count, uint32_t value, uint32_t *flag, cudaStream_t stream) {
  if (count == 0) return;
  k_set_first<<<div_up(count, 256), 256, 0, stream>>>(order, count, value, flag);
}

void launch_compact(const uint32_t *flag, const uint32_t *place, const uint32_t *keys, uint32_t n, uint32_t *out, uint32_t *keysOut,
                    cudaStream_t stream) {
  if (n == 0) return;
  k_compact<<<div_up(n, 256), 256, 0, stream>>>(flag, place, keys, n, out, keysOut);
}

void launch_densify_choose(const float *scales, const DensifyArgs &a, uint32_t n, const uint32_t *chosen, uint32_t *action,
                           cudaStream_t stream) {
  if (n == 0) return;
  k_densify_choose<<<div_up(n, 256), 256, 0, stream>>>(scales, a, n, chosen, action);
}

void launch_densify_large(const float *scales, const DensifyArgs &a, uint32_t n, const uint32_t *action, uint32_t *large,
                          cudaStream_t stream) {
  if (n == 0) return;
  k_densify_large<<<div_up(n, 256), 256, 0, stream>>>(scales, a, n, action, large);
}

void launch_densify_flags(uint32_t n, const uint32_t *action, uint32_t *survivor, uint32_t *added, uint32_t *patched,
                          cudaStream_t stream) {
  if (n == 0) return;
  k_densify_flags<<<div_up(n, 256), 256, 0, stream>>>(n, action, survivor, added, patched);
}

void launch_densify_tables(uint32_t n, uint32_t survivors, const uint32_t *action, const uint32_t *survivorPlace,
                           const uint32_t *addedPlace, const uint32_t *patchedPlace, int32_t *paramSource, int32_t *stateSource,
                           uint32_t *parents, uint32_t *childSlot, cudaStream_t stream) {
  if (n == 0) return;
  k_densify_tables<<<div_up(n, 256), 256, 0, stream>>>(n, survivors, action, survivorPlace, addedPlace, patchedPlace, paramSource,
                                                       stateSource, parents, childSlot);
}

void launch_densify_patch(const DensifyPatch *patches, uint32_t count, float *positions, float *scales, float *rotations,
                          float *opacities, void *shRest, uint32_t restElements, uint32_t restStride, uint32_t shBytes,
                          cudaStream_t stream) {
  if (count == 0) return;
  k_densify_patch<<<div_up(count, 128), 128, 0, stream>>>(patches, count, positions, scales, rotations, opacities, shRest,
                                                          restElements, restStride, shBytes);
}

} // namespace sb
