// Loss: SSIM fields (shaders/train_ssim.comp:42-123), then the adjoint
// dL/dImage and L1 (shaders/train_loss.comp:52-113), for
//   L = (1 - lambda) mean|image - target| + lambda (1 - mean SSIM)
// over pixels and channels, 11x11 Gaussian window (sigma 1.5) cut off and
// renormalised at the image border. Both kernels run one block of 512 threads
// per loss tile of 16 x 32 pixels (the reference's passes run per pixel): the
// tile and a 5-pixel halo are staged into shared memory once, a horizontal
// pass over the tile plus 5 rows above and below goes into shared memory,
// then a vertical pass out of it. The tall tile spends fewer of its
// horizontal sums on halo rows (42 rows for 32 against 26 for 16), and its
// horizontal items fill the block's threads in one round. Normalisations are multiplications
// by reciprocals (the reference's GLSL division is not correctly rounded
// either). The fields are stored as 9
// FP32 planes (P, Q, R per channel; 36 bytes per pixel instead of the
// reference's 48). Per-tile partial sums are added in FP64 on the GPU.
#include <mutex>
#include <set>

#include "kernels.cuh"

namespace sb {

namespace {

constexpr int kHalo = 5;
constexpr int kLossW = kLossTileW, kLossH = kLossTileH;
constexpr int kLossThreads = kLossW * kLossH;
constexpr int kRows = kLossH + 2 * kHalo;
constexpr int kSpan = kRows * kLossW;
constexpr float kC1 = 0.0001f, kC2 = 0.0009f;

__constant__ float c_weights[11] = {0.00102838f, 0.00759876f, 0.03600077f, 0.10936069f, 0.21300554f, 0.26601172f,
                                    0.21300554f, 0.10936069f, 0.03600077f, 0.00759876f, 0.00102838f};

// The norm of a window that lies inside the image: the eleven weights added in
// window_norm's order.
__device__ __forceinline__ float c_weights_total() {
  float norm = 0.0f;
#pragma unroll
  for (int i = 0; i < 11; ++i) norm += c_weights[i];
  return norm;
}

__device__ __forceinline__ float window_norm(int at, int size) {
  float norm = 0.0f;
  for (int i = max(at - 5, 0); i <= min(at + 5, size - 1); ++i) norm += c_weights[i - at + 5];
  return norm;
}

__device__ __forceinline__ float3 unpack_unorm(uint32_t v) {
  return make_float3((float)(v & 0xFFu) / 255.0f, (float)((v >> 8) & 0xFFu) / 255.0f, (float)((v >> 16) & 0xFFu) / 255.0f);
}

__device__ __forceinline__ int view_of_tile(const ViewSet &views, int tile) {
  int v = 0;
  while (v + 1 < views.count && tile >= views.v[v + 1].lossTileBase) ++v;
  return v;
}

// Sum over the block's threads; valid in thread 0.
__device__ __forceinline__ float block_sum(float v, float *s_warp) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  if ((threadIdx.x & 31u) == 0) s_warp[threadIdx.x >> 5] = v;
  __syncthreads();
  float total = 0.0f;
  if (threadIdx.x == 0)
    for (int w = 0; w < kLossThreads / 32; ++w) total += s_warp[w];
  return total;
}

// The tile with a 5-pixel halo on every side, one float per pixel and
// plane, zero outside the image: a tap there adds an exact zero, as if the
// window had been cut at the border, so every pass runs all 11 taps.
//
// The horizontal pass leaves unnormalised window sums: the horizontal norm
// depends on the column only, so it leaves the double sum as a factor and is
// applied, with the vertical one, in the epilogue. Both passes are register
// blocked: a thread takes kGroup neighbouring outputs of one channel, which
// share kGroup + 10 staged values per plane.
constexpr int kSpanCols = kLossW + 2 * kHalo;
constexpr int kStage = kRows * kSpanCols;
constexpr int kGroup = 4;
constexpr int kGroupsX = kLossW / kGroup;               // horizontal items per row
constexpr int kGroupsY = kLossH / kGroup;               // vertical items per column
constexpr int kHorizontalItems = kRows * kGroupsX;      // per channel
constexpr int kVerticalItems = kLossW * kGroupsY;       // per channel
static_assert(3 * kHorizontalItems <= kLossThreads, "one horizontal item per thread");
static_assert(3 * kVerticalItems <= kLossThreads, "one vertical item per thread");
static_assert(kLossW == 16 && kGroup == 4 && kRows % 2 == 0, "h_index's swizzle assumes 16-wide rows and 4-row groups");

// Where the horizontal sum of (row, column) lives in its plane: rows in pairs
// of 32 words, a pair's two 16-word halves swapped where bit 2 of the row is
// set, so that the two half-warps of the vertical pass, four rows apart, read
// opposite halves of the banks.
__device__ __forceinline__ int h_index(int row, int col) {
  return (row >> 1) * 32 + ((((row & 1) << 4) | col) ^ (((row >> 2) & 1) << 4));
}

// The window norms of a row or column (the sum of the taps inside the image).
__device__ __forceinline__ float norm_of(int at, int size) {
  return (at >= kHalo && at + kHalo < size) ? c_weights_total() : window_norm(at, size);
}

// Horizontal window sums x, y, x^2, y^2, xy of the staged image and target
// planes into s_h, kGroup outputs per item.
__device__ __forceinline__ void horizontal_pass(const float (*s_in)[kStage], float (*s_h)[kSpan]) {
  for (int item = threadIdx.x; item < 3 * kHorizontalItems; item += kLossThreads) {
    const int k = item / kHorizontalItems, rem = item % kHorizontalItems;
    const int r = rem / kGroupsX, c = (rem % kGroupsX) * kGroup;
    const int row = r * kSpanCols + c;
    float m[kGroup][5];
#pragma unroll
    for (int o = 0; o < kGroup; ++o)
#pragma unroll
      for (int q = 0; q < 5; ++q) m[o][q] = 0.0f;
#pragma unroll
    for (int u = 0; u < kGroup + 10; ++u) {
      const float a = s_in[k][row + u], b = s_in[3 + k][row + u];
#pragma unroll
      for (int o = 0; o < kGroup; ++o) {
        const int tap = u - o; // output c + o takes staged column c + o + tap
        if (tap < 0 || tap > 10) continue;
        const float w = c_weights[tap];
        const float wa = w * a, wb = w * b;
        m[o][0] = fmaf(w, a, m[o][0]);
        m[o][1] = fmaf(w, b, m[o][1]);
        m[o][2] = fmaf(wa, a, m[o][2]);
        m[o][3] = fmaf(wb, b, m[o][3]);
        m[o][4] = fmaf(wa, b, m[o][4]);
      }
    }
#pragma unroll
    for (int o = 0; o < kGroup; ++o)
#pragma unroll
      for (int q = 0; q < 5; ++q) s_h[q * 3 + k][h_index(r, c + o)] = m[o][q];
  }
}

// Vertical window sums of kOut planes of channel k for kGroup rows of column
// c, from the horizontal sums.
template <int kOut>
__device__ __forceinline__ void vertical_sums(const float (*s_h)[kSpan], int k, int c, int row0, float m[kGroup][kOut]) {
#pragma unroll
  for (int o = 0; o < kGroup; ++o)
#pragma unroll
    for (int q = 0; q < kOut; ++q) m[o][q] = 0.0f;
#pragma unroll
  for (int v = 0; v < kGroup + 10; ++v) {
    float h[kOut];
#pragma unroll
    for (int q = 0; q < kOut; ++q) h[q] = s_h[q * 3 + k][h_index(row0 + v, c)];
#pragma unroll
    for (int o = 0; o < kGroup; ++o) {
      const int tap = v - o;
      if (tap < 0 || tap > 10) continue;
#pragma unroll
      for (int q = 0; q < kOut; ++q) m[o][q] = fmaf(c_weights[tap], h[q], m[o][q]);
    }
  }
}

struct TileOrigin {
  const ViewParams *cam;
  int x0, y0;
};

__device__ __forceinline__ TileOrigin tile_origin(const ViewSet &views, int tile) {
  const ViewParams &cam = views.v[view_of_tile(views, tile)];
  const int local = tile - cam.lossTileBase;
  return TileOrigin{&cam, (local % cam.lossGridW) * kLossW, (local / cam.lossGridW) * kLossH};
}

// Dynamic shared memory of k_ssim: image r, g, b, then target r, g, b staged;
// the horizontal sums x, y, x^2, y^2, xy, three channels each.
constexpr size_t kSsimShared = sizeof(float) * (6 * kStage + 15 * kSpan);

__global__ void __launch_bounds__(kLossThreads, 3) k_ssim(const float4 *__restrict__ image, const uint32_t *__restrict__ targetBuffer,
                                                       const ViewSet *__restrict__ viewsPtr, float *__restrict__ fields,
                                                       float2 *__restrict__ partials) {
  chain_enter();
  const ViewSet &views = *viewsPtr;
  const uint32_t *__restrict__ target = views.target != nullptr ? views.target : targetBuffer;
  extern __shared__ __align__(16) float s_dynamic[];
  float(*s_in)[kStage] = reinterpret_cast<float(*)[kStage]>(s_dynamic);
  float(*s_h)[kSpan] = reinterpret_cast<float(*)[kSpan]>(s_dynamic + 6 * kStage);
  __shared__ float s_warp[kLossThreads / 32];
  const int tile = blockIdx.x;
  const TileOrigin origin = tile_origin(views, tile);
  const ViewParams &cam = *origin.cam;
  const int W = cam.width, H = cam.height, x0 = origin.x0, y0 = origin.y0;
  const size_t base = (size_t)cam.pixelBase;
  const size_t plane = (size_t)views.totalPixels;

#pragma unroll
  for (int round = 0; round < (kStage + kLossThreads - 1) / kLossThreads; ++round) {
    const int i = round * kLossThreads + threadIdx.x;
    if (i >= kStage) break;
    const int r = i / kSpanCols, c = i % kSpanCols;
    const int y = y0 + r - kHalo, x = x0 + c - kHalo;
    float4 a4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float3 b3 = make_float3(0.f, 0.f, 0.f);
    if (y >= 0 && y < H && x >= 0 && x < W) {
      const size_t at = base + (size_t)y * W + x;
      a4 = image[at];
      b3 = unpack_unorm(target[at]);
    }
    s_in[0][i] = a4.x;
    s_in[1][i] = a4.y;
    s_in[2][i] = a4.z;
    s_in[3][i] = b3.x;
    s_in[4][i] = b3.y;
    s_in[5][i] = b3.z;
  }
  __syncthreads();
  horizontal_pass(s_in, s_h);
  __syncthreads();

  float own = 0.0f;
  if (threadIdx.x < 3 * kVerticalItems) {
    const int c = threadIdx.x % kLossW, g = (threadIdx.x / kLossW) % kGroupsY, k = threadIdx.x / kVerticalItems;
    const int px = x0 + c, row0 = g * kGroup;
    float m[kGroup][5];
    vertical_sums<5>(s_h, k, c, row0, m);
    if (px < W) {
      const float invCol = 1.0f / norm_of(px, W);
#pragma unroll
      for (int o = 0; o < kGroup; ++o) {
        const int py = y0 + row0 + o;
        if (py >= H) continue;
        const float inv = invCol / norm_of(py, H);
        const float mx = m[o][0] * inv, my = m[o][1] * inv;
        const float vx = fmaf(m[o][2], inv, -mx * mx), vy = fmaf(m[o][3], inv, -my * my), cxy = fmaf(m[o][4], inv, -mx * my);
        const float n1 = fmaf(2.0f * mx, my, kC1), n2 = fmaf(2.0f, cxy, kC2);
        const float d1 = fmaf(mx, mx, fmaf(my, my, kC1)), d2 = vx + vy + kC2;
        const float invD = 1.0f / (d1 * d2), invD1 = d2 * invD, invD2 = d1 * invD;
        const float ssim = (n1 * n2) * invD;
        own += ssim;
        // n1 and n2 cancelled by hand, as the reference does: n2 can be zero.
        const float dMu = 2.0f * my * n2 * invD - ssim * 2.0f * mx * invD1;
        const float dVar = -ssim * invD2;
        const float dCov = 2.0f * n1 * invD;
        const size_t pixel = base + (size_t)py * W + px;
        fields[(0 * 3 + k) * plane + pixel] = (dMu - 2.0f * mx * dVar - my * dCov) * inv;
        fields[(1 * 3 + k) * plane + pixel] = dVar * inv;
        fields[(2 * 3 + k) * plane + pixel] = dCov * inv;
      }
    }
  }
  const float total = block_sum(own, s_warp);
  if (threadIdx.x == 0) partials[tile].x = total;
}

// The target's luminance at (x, y), clamped to the image (train_loss.comp:34-39).
__device__ __forceinline__ float target_luminance(const uint32_t *target, size_t base, int W, int H, int x, int y) {
  x = min(max(x, 0), W - 1);
  y = min(max(y, 0), H - 1);
  const float3 t = unpack_unorm(target[base + (size_t)y * W + x]);
  return t.x * 0.299f + t.y * 0.587f + t.z * 0.114f;
}

// The edge weight of the edge-aware score: a Laplacian of the target's
// luminance, as differences so that a flat patch gives exactly zero, clamped
// to [0, 0.999] (train_loss.comp:41-50).
__device__ __forceinline__ float target_edge(const uint32_t *target, size_t base, int W, int H, int x, int y) {
  const float centre = target_luminance(target, base, W, H, x, y);
  const float laplacian = (target_luminance(target, base, W, H, x - 1, y) - centre) +
                          (target_luminance(target, base, W, H, x + 1, y) - centre) +
                          (target_luminance(target, base, W, H, x, y - 1) - centre) +
                          (target_luminance(target, base, W, H, x, y + 1) - centre);
  return fminf(fmaxf(fabsf(laplacian) / 4.0f, 0.0f), 0.999f);
}

// Dynamic shared memory of k_loss: the nine field planes staged, their
// horizontal sums, the adjoint's three channels.
constexpr size_t kLossShared = sizeof(float) * (9 * kStage + 9 * kSpan + 3 * kLossThreads);

// Horizontal window sums of the nine staged field planes into s_h, kGroup
// outputs per item.
__device__ __forceinline__ void horizontal_fields(const float (*s_in)[kStage], float (*s_h)[kSpan]) {
  for (int item = threadIdx.x; item < 3 * kHorizontalItems; item += kLossThreads) {
    const int k = item / kHorizontalItems, rem = item % kHorizontalItems;
    const int r = rem / kGroupsX, c = (rem % kGroupsX) * kGroup;
    const int row = r * kSpanCols + c;
    float m[kGroup][3];
#pragma unroll
    for (int o = 0; o < kGroup; ++o)
#pragma unroll
      for (int q = 0; q < 3; ++q) m[o][q] = 0.0f;
#pragma unroll
    for (int u = 0; u < kGroup + 10; ++u) {
      const float v[3] = {s_in[k][row + u], s_in[3 + k][row + u], s_in[6 + k][row + u]};
#pragma unroll
      for (int o = 0; o < kGroup; ++o) {
        const int tap = u - o;
        if (tap < 0 || tap > 10) continue;
#pragma unroll
        for (int q = 0; q < 3; ++q) m[o][q] = fmaf(c_weights[tap], v[q], m[o][q]);
      }
    }
#pragma unroll
    for (int o = 0; o < kGroup; ++o)
#pragma unroll
      for (int q = 0; q < 3; ++q) s_h[q * 3 + k][h_index(r, c + o)] = m[o][q];
  }
}

// SCORE (a scored view, train_loss.comp:101-107): the adjoint's alpha gets the
// pixel's mean absolute error over its three channels, errorMax the view's
// worst (in 1/65535), edge the target's edge weight.
template <bool SCORE>
__global__ void __launch_bounds__(kLossThreads, 3) k_loss(const float4 *__restrict__ image, const uint32_t *__restrict__ targetBuffer,
                                                       const float *__restrict__ fields, const ViewSet *__restrict__ viewsPtr,
                                                       float lambda, float4 *__restrict__ adjoint, float2 *__restrict__ partials,
                                                       LossScoring scoring) {
  chain_enter();
  const ViewSet &views = *viewsPtr;
  const uint32_t *__restrict__ target = views.target != nullptr ? views.target : targetBuffer;
  extern __shared__ __align__(16) float s_dynamic[];
  float(*s_in)[kStage] = reinterpret_cast<float(*)[kStage]>(s_dynamic);
  float(*s_h)[kSpan] = reinterpret_cast<float(*)[kSpan]>(s_dynamic + 9 * kStage);
  float(*s_result)[kLossThreads] = reinterpret_cast<float(*)[kLossThreads]>(s_dynamic + 9 * kStage + 9 * kSpan);
  __shared__ float s_warp[kLossThreads / 32];
  const int tile = blockIdx.x;
  const TileOrigin origin = tile_origin(views, tile);
  const ViewParams &cam = *origin.cam;
  const int W = cam.width, H = cam.height, x0 = origin.x0, y0 = origin.y0;
  const size_t base = (size_t)cam.pixelBase;
  const size_t plane = (size_t)views.totalPixels;
  // This thread's epilogue pixels (kGroup rows of one column, one channel):
  // their image and target values are asked for first, so that they arrive
  // while the fields are staged and filtered.
  const bool epilogue = threadIdx.x < 3 * kVerticalItems;
  const int ec = threadIdx.x % kLossW, eg = (threadIdx.x / kLossW) % kGroupsY, ek = threadIdx.x / kVerticalItems;
  float xs[kGroup], ys[kGroup];
#pragma unroll
  for (int o = 0; o < kGroup; ++o) {
    const int px = x0 + ec, py = y0 + eg * kGroup + o;
    xs[o] = 0.0f;
    ys[o] = 0.0f;
    if (epilogue && px < W && py < H) {
      const size_t pixel = base + (size_t)py * W + px;
      xs[o] = reinterpret_cast<const float *>(image)[pixel * 4 + ek];
      ys[o] = (float)((target[pixel] >> (8 * ek)) & 0xFFu) / 255.0f;
    }
  }

#pragma unroll
  for (int round = 0; round < (kStage + kLossThreads - 1) / kLossThreads; ++round) {
    const int i = round * kLossThreads + threadIdx.x;
    if (i >= kStage) break;
    const int r = i / kSpanCols, c = i % kSpanCols;
    const int y = y0 + r - kHalo, x = x0 + c - kHalo;
    const bool in = y >= 0 && y < H && x >= 0 && x < W;
    const size_t at = in ? base + (size_t)y * W + x : 0;
#pragma unroll
    for (int f = 0; f < 9; ++f) s_in[f][i] = in ? fields[f * plane + at] : 0.0f;
  }
  __syncthreads();
  horizontal_fields(s_in, s_h);
  __syncthreads();

  float own = 0.0f;
  if (epilogue) {
    const int c = ec, k = ek;
    const int px = x0 + c, row0 = eg * kGroup;
    float m[kGroup][3];
    vertical_sums<3>(s_h, k, c, row0, m);
    const float perValue = cam.perPixel;
#pragma unroll
    for (int o = 0; o < kGroup; ++o) {
      const int py = y0 + row0 + o;
      float result = 0.0f;
      if (px < W && py < H) {
        const float xv = xs[o], yv = ys[o];
        const float d = xv - yv;
        own += fabsf(d);
        const float sgn = d > 0.0f ? 1.0f : (d < 0.0f ? -1.0f : 0.0f);
        const float ssimPart = m[o][0] + 2.0f * xv * m[o][1] + yv * m[o][2];
        result = ((1.0f - lambda) * sgn - lambda * ssimPart) * perValue;
      }
      s_result[k][(row0 + o) * kLossW + c] = result;
    }
  }
  __syncthreads();
  {
    const int px = x0 + (int)(threadIdx.x % kLossW), py = y0 + (int)(threadIdx.x / kLossW);
    if (px < W && py < H) {
      const size_t pixel = base + (size_t)py * W + px;
      float alpha = 0.0f;
      if constexpr (SCORE) {
        const float4 x4 = image[pixel];
        const float3 y3 = unpack_unorm(target[pixel]);
        const float own3 = fabsf(x4.x - y3.x) + fabsf(x4.y - y3.y) + fabsf(x4.z - y3.z);
        alpha = own3 / 3.0f;
        atomicMax(scoring.errorMax, (uint32_t)(fminf(fmaxf(alpha, 0.0f), 1.0f) * 65535.0f));
        scoring.edge[pixel] = target_edge(target, base, W, H, px, py);
      }
      adjoint[pixel] = make_float4(s_result[0][threadIdx.x], s_result[1][threadIdx.x], s_result[2][threadIdx.x], alpha);
    }
  }
  const float total = block_sum(own, s_warp);
  if (threadIdx.x == 0) partials[tile].y = total;
}

// train_error_mask.comp: the adjoint's alpha becomes 1 where the pixel's
// error is at least `share` of the view's worst, else 0.
__global__ void __launch_bounds__(256) k_error_mask(float4 *__restrict__ adjoint, uint32_t pixels, const uint32_t *__restrict__ errorMax,
                                                    float share) {
  chain_enter();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= pixels) return;
  const uint32_t worst = *errorMax;
  const float error = adjoint[i].w;
  adjoint[i].w = worst > 0u && error >= share * (float)worst / 65535.0f ? 1.0f : 0.0f;
}

__global__ void __launch_bounds__(256) k_loss_totals(const float2 *__restrict__ partials, const ViewSet *__restrict__ viewsPtr,
                                                     LossTotals *totals) {
  chain_enter();
  const ViewSet &views = *viewsPtr;
  __shared__ double s_ssim[256], s_l1[256];
  const int v = blockIdx.x;
  const ViewParams &cam = views.v[v];
  double ssim = 0.0, l1 = 0.0;
  for (int i = threadIdx.x; i < cam.lossTileCount; i += 256) {
    const float2 p = partials[cam.lossTileBase + i];
    ssim += (double)p.x;
    l1 += (double)p.y;
  }
  s_ssim[threadIdx.x] = ssim;
  s_l1[threadIdx.x] = l1;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < (unsigned)o) {
      s_ssim[threadIdx.x] += s_ssim[threadIdx.x + o];
      s_l1[threadIdx.x] += s_l1[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    totals->ssimSum[v] = s_ssim[0];
    totals->l1Sum[v] = s_l1[0];
  }
}

} // namespace

// The loss kernels' shared memory is above the static 48 KB: allowed once per
// process and device.
void allow_loss_shared() {
  static std::mutex lock;
  static std::set<int> done;
  int device = 0;
  cudaGetDevice(&device);
  std::lock_guard<std::mutex> guard(lock);
  if (done.count(device) != 0) return;
  cudaFuncSetAttribute(k_ssim, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSsimShared);
  cudaFuncSetAttribute(k_loss<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLossShared);
  cudaFuncSetAttribute(k_loss<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLossShared);
  done.insert(device);
}

void launch_ssim(const float4 *image, const uint32_t *target, const ViewSet &views, const ViewSet *dViews, float4 *fields, float2 *partials,
                 cudaStream_t stream) {
  if (views.totalLossTiles == 0) return;
  allow_loss_shared();
  launch_chained(k_ssim, dim3(views.totalLossTiles), dim3(kLossThreads), kSsimShared, stream, image, target, dViews,
                 reinterpret_cast<float *>(fields), partials);
}

void launch_loss(const float4 *image, const uint32_t *target, const float4 *fields, const ViewSet &views, const ViewSet *dViews, float lambda,
                 float4 *adjoint, float2 *partials, cudaStream_t stream, LossScoring scoring) {
  if (views.totalLossTiles == 0) return;
  const float *f = reinterpret_cast<const float *>(fields);
  allow_loss_shared();
  if (scoring.edge != nullptr)
    launch_chained(k_loss<true>, dim3(views.totalLossTiles), dim3(kLossThreads), kLossShared, stream, image, target, f, dViews, lambda,
                   adjoint, partials, scoring);
  else
    launch_chained(k_loss<false>, dim3(views.totalLossTiles), dim3(kLossThreads), kLossShared, stream, image, target, f, dViews, lambda,
                   adjoint, partials, scoring);
}

void launch_error_mask(float4 *adjoint, uint32_t pixels, const uint32_t *errorMax, float share, cudaStream_t stream) {
  if (pixels == 0) return;
  launch_chained(k_error_mask, dim3(div_up(pixels, 256)), dim3(256), 0, stream, adjoint, pixels, errorMax, share);
}

void launch_loss_totals(const float2 *partials, const ViewSet &views, const ViewSet *dViews, LossTotals *totals, cudaStream_t stream) {
  launch_chained(k_loss_totals, dim3(views.count), dim3(256), 0, stream, partials, dViews, totals);
}

} // namespace sb
