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

} // namespace sb
