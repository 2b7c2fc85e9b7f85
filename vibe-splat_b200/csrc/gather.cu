// Optimiser state across densification (shaders/train_gather.comp:1-24,
// Trainer::apply_changes, src/train/trainer.cpp:749-787): element k of new
// Gaussian g takes old element k of Gaussian source[g], or zero when source[g]
// is negative (a new Gaussian starts with fresh moments). Two layouts: rows of
// `stride` words per Gaussian (positions, scales, rotations, opacities, and
// the SH state, whose row count is rounded up to a multiple of 128: rows from
// `valid` on are padding, zeroed) and planes of one word per Gaussian (the SH
// coefficients, planeStride apart). F32 state keeps its v words as a second
// copy of the layout after the m words.
#include <algorithm>

#include "kernels.cuh"

namespace sb {

namespace {

// A thread per (new Gaussian, copy): the source index read once, the row's
// `stride` words copied (STRIDE 0: any stride).
template <uint32_t STRIDE>
__global__ void __launch_bounds__(256) k_gather_rows(const int32_t *__restrict__ source, const uint32_t *__restrict__ in,
                                                     uint32_t *__restrict__ out, uint32_t newCount, uint32_t oldCount,
                                                     uint32_t runtimeStride, uint32_t valid) {
  const uint32_t stride = STRIDE != 0 ? STRIDE : runtimeStride;
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x, copy = blockIdx.y;
  if (g >= newCount) return;
  const int32_t from = g < valid ? source[g] : -1;
  uint32_t *dst = out + ((size_t)copy * newCount + g) * stride;
  if (from < 0) {
    for (uint32_t k = 0; k < stride; ++k) dst[k] = 0u;
    return;
  }
  const uint32_t *src = in + ((size_t)copy * oldCount + (uint32_t)from) * stride;
  if constexpr (STRIDE == 4) {
    *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<const uint4 *>(src);
  } else {
#pragma unroll
    for (uint32_t k = 0; k < (STRIDE != 0 ? STRIDE : 1u); ++k) dst[k] = src[k];
    if constexpr (STRIDE == 0)
      for (uint32_t k = 1; k < stride; ++k) dst[k] = src[k];
  }
}

// A thread per new Gaussian (padding included, zeroed): the source index read
// once, then every plane's element for it, planes in groups of 8 loads in
// flight.
template <class T>
__global__ void __launch_bounds__(256) k_gather_planes(const int32_t *__restrict__ source, const T *__restrict__ in, T *__restrict__ out,
                                                       uint32_t newCount, uint32_t newStride, uint32_t oldStride, uint32_t planes) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= newStride) return;
  const int32_t from = g < newCount ? source[g] : -1;
  T *dst = out + g;
  if (from < 0) {
    for (uint32_t q = 0; q < planes; ++q) dst[(size_t)q * newStride] = T(0);
    return;
  }
  const T *src = in + (uint32_t)from;
  uint32_t q = 0;
  for (; q + 8 <= planes; q += 8) {
    T v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = src[(size_t)(q + j) * oldStride];
#pragma unroll
    for (int j = 0; j < 8; ++j) dst[(size_t)(q + j) * newStride] = v[j];
  }
  for (; q < planes; ++q) dst[(size_t)q * newStride] = src[(size_t)q * oldStride];
}

// Pruning (remove_highest, src/train/densify.cpp:70-90): a key per Gaussian
// whose ascending stable sort puts first the Gaussians to remove, those with
// the highest value: kind 0 the largest log-scale (remove_largest), 1 minus
// the contribution (remove_least_contributing), 2 minus the opacity logit
// (remove_least_opaque). The float's order is flipped into unsigned order and
// then reversed; both zeros count as one, as the reference's comparison has it.
__global__ void __launch_bounds__(256) k_prune_keys(int kind, const float *__restrict__ scales, const float *__restrict__ opacities,
                                                    const float *__restrict__ densifyStats, uint32_t n, uint32_t *__restrict__ keys,
                                                    uint32_t *__restrict__ values) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float f;
  if (kind == 0) f = fmaxf(fmaxf(scales[(size_t)i * 3], scales[(size_t)i * 3 + 1]), scales[(size_t)i * 3 + 2]);
  else if (kind == 1) f = -densifyStats[(size_t)i * kStatStride + 3];
  else f = -opacities[i];
  if (f == 0.0f) f = 0.0f;
  const uint32_t bits = __float_as_uint(f);
  const uint32_t ordered = bits ^ ((bits >> 31) != 0u ? 0xFFFFFFFFu : 0x80000000u);
  keys[i] = ~ordered;
  values[i] = i;
}

// keep[i] = 0 for the first `removed` Gaussians of the sorted order, else 1.
__global__ void __launch_bounds__(256) k_prune_keep(const uint32_t *__restrict__ order, uint32_t removed, uint32_t n,
                                                    uint32_t *__restrict__ keep) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const uint32_t g = order[r];
  if (g < n) keep[g] = r < removed ? 0u : 1u;
}

// source[place[i]] = i for every kept Gaussian (place: the exclusive scan of keep).
__global__ void __launch_bounds__(256) k_survivor_sources(const uint32_t *__restrict__ keep, const uint32_t *__restrict__ place,
                                                          uint32_t n, int32_t *__restrict__ source) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && keep[i] != 0u) source[place[i]] = (int32_t)i;
}

} // namespace

void launch_gather_rows(const int32_t *source, const uint32_t *in, uint32_t *out, uint32_t newCount, uint32_t oldCount,
                        uint32_t stride, uint32_t copies, cudaStream_t stream, uint32_t valid) {
  if (newCount == 0 || stride == 0 || copies == 0) return;
  valid = std::min(valid, newCount);
  const dim3 grid(div_up(newCount, 256), copies);
  // Rows of 4 words move as one 16-byte access when both arrays keep 16-byte rows.
  const bool aligned = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u) == 0u;
  switch (stride) {
  case 1: k_gather_rows<1><<<grid, 256, 0, stream>>>(source, in, out, newCount, oldCount, 1, valid); break;
  case 3: k_gather_rows<3><<<grid, 256, 0, stream>>>(source, in, out, newCount, oldCount, 3, valid); break;
  case 4:
    if (aligned) k_gather_rows<4><<<grid, 256, 0, stream>>>(source, in, out, newCount, oldCount, 4, valid);
    else k_gather_rows<0><<<grid, 256, 0, stream>>>(source, in, out, newCount, oldCount, 4, valid);
    break;
  default: k_gather_rows<0><<<grid, 256, 0, stream>>>(source, in, out, newCount, oldCount, stride, valid); break;
  }
}

void launch_gather_planes(const int32_t *source, const uint32_t *in, uint32_t *out, uint32_t newCount, uint32_t newStride,
                          uint32_t oldStride, uint32_t planes, cudaStream_t stream) {
  if (newStride == 0 || planes == 0) return;
  k_gather_planes<uint32_t><<<div_up(newStride, 256), 256, 0, stream>>>(source, in, out, newCount, newStride, oldStride, planes);
}

void launch_gather_planes16(const int32_t *source, const uint16_t *in, uint16_t *out, uint32_t newCount, uint32_t newStride,
                            uint32_t oldStride, uint32_t planes, cudaStream_t stream) {
  if (newStride == 0 || planes == 0) return;
  k_gather_planes<uint16_t><<<div_up(newStride, 256), 256, 0, stream>>>(source, in, out, newCount, newStride, oldStride, planes);
}

void launch_prune_keys(int kind, const float *scales, const float *opacities, const float *densifyStats, uint32_t n, uint32_t *keys,
                       uint32_t *values, cudaStream_t stream) {
  if (n == 0) return;
  k_prune_keys<<<div_up(n, 256), 256, 0, stream>>>(kind, scales, opacities, densifyStats, n, keys, values);
}

void launch_prune_keep(const uint32_t *order, uint32_t removed, uint32_t n, uint32_t *keep, cudaStream_t stream) {
  if (n == 0) return;
  k_prune_keep<<<div_up(n, 256), 256, 0, stream>>>(order, removed, n, keep);
}

void launch_survivor_sources(const uint32_t *keep, const uint32_t *place, uint32_t n, int32_t *source, cudaStream_t stream) {
  if (n == 0) return;
  k_survivor_sources<<<div_up(n, 256), 256, 0, stream>>>(keep, place, n, source);
}

} // namespace sb
