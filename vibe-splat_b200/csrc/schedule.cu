// The coarse-to-fine schedule's device work (src/train/schedule.cpp and the
// image and point preparation of src/train/train.cpp): half-size views, the
// spectrum energy that sets the image sizes, and the starting Gaussians'
// sizes from their nearest neighbours.
#include <cfloat>
#include <cstdint>

#include "kernels.cuh"
#include "sort.cuh"

namespace sb {

namespace {

// half_size (train.cpp:232-255): each output pixel the rounded mean of the
// 2x2 pixels it covers, channel by channel (alpha included).
__global__ void __launch_bounds__(256) k_half_size(const uint8_t *__restrict__ in, int width, uint8_t *__restrict__ out, int w, int h) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= w || y >= h) return;
  const size_t stride = (size_t)width * 4;
  const uchar4 *row0 = reinterpret_cast<const uchar4 *>(in + 2 * (size_t)y * stride) + 2 * x;
  const uchar4 *row1 = reinterpret_cast<const uchar4 *>(in + (2 * (size_t)y + 1) * stride) + 2 * x;
  const uchar4 a = row0[0], b = row0[1], c = row1[0], d = row1[1];
  uchar4 m;
  m.x = (uint8_t)((a.x + b.x + c.x + d.x + 2) / 4);
  m.y = (uint8_t)((a.y + b.y + c.y + d.y + 2) / 4);
  m.z = (uint8_t)((a.z + b.z + c.z + d.z + 2) / 4);
  m.w = (uint8_t)((a.w + b.w + c.w + d.w + 2) / 4);
  reinterpret_cast<uchar4 *>(out)[(size_t)y * w + x] = m;
}

// frequency_energy (schedule.cpp:41-75), first part: the image's brightness
// (BT.601 weights) mirrored out to the power-of-two size W x H.
__global__ void __launch_bounds__(256) k_spectrum_load(const uint8_t *__restrict__ rgba, int width, int height, double2 *values, int W,
                                                       int H) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W || y >= H) return;
  const auto mirrored = [](int at, int size) { return at < size ? at : 2 * size - 1 - min(at, 2 * size - 1); };
  const uint8_t *p = rgba + ((size_t)mirrored(y, height) * width + mirrored(x, width)) * 4;
  const double v = (0.299 * p[0] + 0.587 * p[1] + 0.114 * p[2]) / 255.0;
  values[(size_t)y * W + x] = make_double2(v, 0.0);
}

// One radix-2 FFT of `size` (a power of two, at most 4096) complex values per
// block, `stride` apart, starting at block * step: loaded into shared memory
// in bit-reversed order, then the butterfly stages.
__global__ void __launch_bounds__(512) k_fft(double2 *values, int size, int logSize, size_t stride, size_t step) {
  extern __shared__ double2 s_values[];
  double2 *base = values + (size_t)blockIdx.x * step;
  for (int i = threadIdx.x; i < size; i += blockDim.x) {
    const int j = (int)(__brev((unsigned)i) >> (32 - logSize));
    s_values[j] = base[(size_t)i * stride];
  }
  __syncthreads();
  for (int length = 2; length <= size; length <<= 1) {
    const int half = length >> 1;
    for (int b = threadIdx.x; b < size / 2; b += blockDim.x) {
      const int k = b % half, start = (b / half) * length;
      double s, c;
      sincospi(-2.0 * (double)k / (double)length, &s, &c);
      const double2 u = s_values[start + k], v = s_values[start + k + half];
      const double2 t = make_double2(v.x * c - v.y * s, v.x * s + v.y * c);
      s_values[start + k] = make_double2(u.x + t.x, u.y + t.y);
      s_values[start + k + half] = make_double2(u.x - t.x, u.y - t.y);
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < size; i += blockDim.x) base[(size_t)i * stride] = s_values[i];
}

// The spectrum's magnitude summed within the frequencies an image smaller by
// each factor can hold (|fx|, |fy| <= 0.5 / factor), one partial sum per
// block and factor.
__global__ void __launch_bounds__(256) k_spectrum_sum(const double2 *__restrict__ values, int W, int H, const int *__restrict__ factors,
                                                      int count, double *__restrict__ partials) {
  __shared__ double s_sum[8][8];
  double sums[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const size_t total = (size_t)W * H;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(e / W), x = (int)(e % W);
    const double fy = (double)min(y, H - y) / (double)H, fx = (double)min(x, W - x) / (double)W;
    const double magnitude = hypot(values[e].x, values[e].y);
    for (int k = 0; k < count; ++k) {
      const double limit = 0.5 / factors[k];
      if (fx <= limit && fy <= limit) sums[k] += magnitude;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < count; ++k) {
    double v = sums[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if (lane == 0) s_sum[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < count) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += s_sum[threadIdx.x][w];
    partials[(size_t)blockIdx.x * count + threadIdx.x] = v;
  }
}

// neighbour_distances (train.cpp:143-189): a point's cell on the grid.
__device__ __forceinline__ int3 cell_of(double3 p, double3 low, double cell) {
  return make_int3((int)((p.x - low.x) / cell), (int)((p.y - low.y) / cell), (int)((p.z - low.z) / cell));
}

__global__ void __launch_bounds__(256) k_point_cells(const double3 *__restrict__ points, uint32_t n, double3 low, double cell,
                                                     int3 dims, uint32_t *__restrict__ keys, uint32_t *__restrict__ values) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int3 c = cell_of(points[i], low, cell);
  keys[i] = ((uint32_t)c.x * (uint32_t)dims.y + (uint32_t)c.y) * (uint32_t)dims.z + (uint32_t)c.z;
  values[i] = i;
}

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *keys, uint32_t n, uint32_t key) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (keys[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// The mean distance to the 3 nearest other points within the cube of cells
// of radius r around the point's, for the first r of 1..4 that holds 3; the
// cell size if none does. The cells are found in the points sorted by cell.
__global__ void __launch_bounds__(128) k_neighbours(const double3 *__restrict__ points, uint32_t n, double3 low, double cell, int3 dims,
                                                    const uint32_t *__restrict__ sortedKeys, const uint32_t *__restrict__ sortedIndex,
                                                    float *__restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double3 p = points[i];
  const int3 c = cell_of(p, low, cell);
  double best[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
  for (int r = 1; r <= 4 && best[2] == DBL_MAX; ++r) {
    best[0] = best[1] = best[2] = DBL_MAX;
    for (int dx = -r; dx <= r; ++dx) {
      const int x = c.x + dx;
      if (x < 0 || x >= dims.x) continue;
      for (int dy = -r; dy <= r; ++dy) {
        const int y = c.y + dy;
        if (y < 0 || y >= dims.y) continue;
        // The cells of one (x, y) column are consecutive keys: one search for
        // the run of z in [c.z - r, c.z + r].
        const int z0 = max(c.z - r, 0), z1 = min(c.z + r, dims.z - 1);
        if (z0 > z1) continue;
        const uint32_t column = ((uint32_t)x * (uint32_t)dims.y + (uint32_t)y) * (uint32_t)dims.z;
        const uint32_t from = lower_bound_u32(sortedKeys, n, column + (uint32_t)z0);
        for (uint32_t k = from; k < n && sortedKeys[k] <= column + (uint32_t)z1; ++k) {
          const uint32_t j = sortedIndex[k];
          if (j == i) continue;
          const double3 q = points[j];
          const double ex = q.x - p.x, ey = q.y - p.y, ez = q.z - p.z;
          const double dist = ex * ex + ey * ey + ez * ez;
          if (dist < best[2]) {
            best[2] = dist;
            if (best[2] < best[1]) {
              const double t = best[1];
              best[1] = best[2];
              best[2] = t;
            }
            if (best[1] < best[0]) {
              const double t = best[0];
              best[0] = best[1];
              best[1] = t;
            }
          }
        }
      }
    }
  }
  const double mean = best[2] == DBL_MAX ? cell : (sqrt(best[0]) + sqrt(best[1]) + sqrt(best[2])) / 3.0;
  out[i] = (float)fmax(mean, 1e-7);
}

} // namespace

void launch_half_size(const uint8_t *in, int width, int height, uint8_t *out, cudaStream_t stream) {
  const int w = width / 2, h = height / 2;
  if (w <= 0 || h <= 0) return;
  k_half_size<<<dim3(div_up((uint32_t)w, 256), (uint32_t)h), 256, 0, stream>>>(in, width, out, w, h);
}

size_t spectrum_scratch_bytes(int width, int height) {
  size_t W = 1, H = 1;
  while (W < (size_t)width) W <<= 1;
  while (H < (size_t)height) H <<= 1;
  return W * H * sizeof(double2) + 1024 * 8 * sizeof(double);
}

bool spectrum_supported(int width, int height) { return width >= 1 && height >= 1 && width <= 4096 && height <= 4096; }

void launch_frequency_energy(const uint8_t *rgba, int width, int height, const int *factors, int count, void *scratch, double *partials,
                             int blocks, cudaStream_t stream) {
  int W = 1, H = 1, logW = 0, logH = 0;
  while (W < width) W <<= 1, ++logW;
  while (H < height) H <<= 1, ++logH;
  double2 *values = static_cast<double2 *>(scratch);
  k_spectrum_load<<<dim3(div_up((uint32_t)W, 256), (uint32_t)H), 256, 0, stream>>>(rgba, width, height, values, W, H);
  if (W > 1) {
    cudaFuncSetAttribute(k_fft, cudaFuncAttributeMaxDynamicSharedMemorySize, 4096 * (int)sizeof(double2));
    k_fft<<<H, 512, W * sizeof(double2), stream>>>(values, W, logW, 1, (size_t)W);
  }
  if (H > 1) {
    cudaFuncSetAttribute(k_fft, cudaFuncAttributeMaxDynamicSharedMemorySize, 4096 * (int)sizeof(double2));
    k_fft<<<W, 512, H * sizeof(double2), stream>>>(values, H, logH, (size_t)W, 1);
  }
  k_spectrum_sum<<<blocks, 256, 0, stream>>>(values, W, H, factors, count, partials);
}

int neighbour_distances(const double *points, uint32_t n, double3 low, double cell, int3 dims, void *scratch, float *out, uint32_t *error,
                        cudaStream_t stream) {
  // scratch: points (24 n), keys, values and their sort copies (16 n), sort scratch.
  uint8_t *at = static_cast<uint8_t *>(scratch);
  const auto take = [&](size_t bytes) {
    uint8_t *p = at;
    at += (bytes + 255) & ~size_t{255};
    return p;
  };
  double3 *dev = reinterpret_cast<double3 *>(take((size_t)n * 24));
  uint32_t *keys = reinterpret_cast<uint32_t *>(take((size_t)n * 4));
  uint32_t *values = reinterpret_cast<uint32_t *>(take((size_t)n * 4));
  uint32_t *tmpKeys = reinterpret_cast<uint32_t *>(take((size_t)n * 4));
  uint32_t *tmpValues = reinterpret_cast<uint32_t *>(take((size_t)n * 4));
  void *sortScratch = take(sort_scratch_bytes(n, 4, 32, 8));
  if (cudaMemcpyAsync(dev, points, (size_t)n * 24, cudaMemcpyHostToDevice, stream) != cudaSuccess) return 1;
  k_point_cells<<<div_up(n, 256), 256, 0, stream>>>(dev, n, low, cell, dims, keys, values);
  const uint64_t cells = (uint64_t)dims.x * dims.y * dims.z;
  int bits = 8;
  while (bits < 32 && (1ull << bits) < cells) ++bits;
  const uint32_t *sk = keys, *sv = values;
  if (n > 1) {
    const int where = sort_pairs_u32(keys, values, tmpKeys, tmpValues, n, n, nullptr, 0, bits, 8, sortScratch, error, stream);
    if (where == 1) sk = tmpKeys, sv = tmpValues;
  }
  k_neighbours<<<div_up(n, 128), 128, 0, stream>>>(dev, n, low, cell, dims, sk, sv, out);
  return 0;
}

size_t neighbour_scratch_bytes(uint32_t n) {
  const auto room = [](size_t b) { return (b + 255) & ~size_t{255}; };
  return room((size_t)n * 24) + 4 * room((size_t)n * 4) + room(sort_scratch_bytes(n, 4, 32, 8));
}

} // namespace sb
