// Optimiser state across densification (shaders/train_gather.comp:1-24,
// Trainer::apply_changes, src/train/trainer.cpp:749-787): element k of new
// Gaussian g takes old element k of Gaussian source[g], or zero when source[g]
// is negative (a new Gaussian starts with fresh moments). Two layouts: rows of
// `stride` words per Gaussian (positions, scales, rotations, opacities) and
// planes of one word per Gaussian (the SH state, planeStride apart). F32
// state keeps its v words as a second copy of the layout after the m words.
#include "kernels.cuh"

namespace sb {

namespace {

__global__ void __launch_bounds__(256) k_gather_rows(const int32_t *__restrict__ source, const uint32_t *__restrict__ in,
                                                     uint32_t *__restrict__ out, uint32_t newCount, uint32_t oldCount,
                                                     uint32_t stride, uint32_t copies) {
  const size_t total = (size_t)newCount * stride;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total * copies; e += (size_t)gridDim.x * blockDim.x) {
    const size_t copy = e / total, i = e - copy * total;
    const size_t g = i / stride, k = i - g * stride;
    const int32_t from = source[g];
    out[e] = from < 0 ? 0u : in[copy * (size_t)oldCount * stride + (size_t)from * stride + k];
  }
}

__global__ void __launch_bounds__(256) k_gather_planes(const int32_t *__restrict__ source, const uint32_t *__restrict__ in,
                                                       uint32_t *__restrict__ out, uint32_t newCount, uint32_t newStride,
                                                       uint32_t oldStride, uint32_t planes) {
  const size_t total = (size_t)planes * newStride;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const size_t q = e / newStride, g = e - q * newStride;
    const int32_t from = g < newCount ? source[g] : -1;
    out[e] = from < 0 ? 0u : in[q * oldStride + (size_t)from];
  }
}

// The same for planes of 16-bit elements (SH above degree 0 in BF16 or FP16).
__global__ void __launch_bounds__(256) k_gather_planes16(const int32_t *__restrict__ source, const uint16_t *__restrict__ in,
                                                         uint16_t *__restrict__ out, uint32_t newCount, uint32_t newStride,
                                                         uint32_t oldStride, uint32_t planes) {
  const size_t total = (size_t)planes * newStride;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const size_t q = e / newStride, g = e - q * newStride;
    const int32_t from = g < newCount ? source[g] : -1;
    out[e] = from < 0 ? (uint16_t)0 : in[q * oldStride + (size_t)from];
  }
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

uint32_t gather_blocks(size_t elements) {
  const size_t blocks = (elements + 255) / 256;
  return (uint32_t)(blocks < 148 * 16 ? (blocks > 0 ? blocks : 1) : 148 * 16);
}

} // namespace

void launch_gather_rows(const int32_t *source, const uint32_t *in, uint32_t *out, uint32_t newCount, uint32_t oldCount,
                        uint32_t stride, uint32_t copies, cudaStream_t stream) {
  if (newCount == 0) return;
  k_gather_rows<<<gather_blocks((size_t)newCount * stride * copies), 256, 0, stream>>>(source, in, out, newCount, oldCount,
                                                                                       stride, copies);
}

void launch_gather_planes(const int32_t *source, const uint32_t *in, uint32_t *out, uint32_t newCount, uint32_t newStride,
                          uint32_t oldStride, uint32_t planes, cudaStream_t stream) {
  if (newCount == 0) return;
  k_gather_planes<<<gather_blocks((size_t)planes * newStride), 256, 0, stream>>>(source, in, out, newCount, newStride, oldStride,
                                                                                 planes);
}

void launch_gather_planes16(const int32_t *source, const uint16_t *in, uint16_t *out, uint32_t newCount, uint32_t newStride,
                            uint32_t oldStride, uint32_t planes, cudaStream_t stream) {
  if (newCount == 0 || planes == 0) return;
  k_gather_planes16<<<gather_blocks((size_t)planes * newStride), 256, 0, stream>>>(source, in, out, newCount, newStride, oldStride,
                                                                                   planes);
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
