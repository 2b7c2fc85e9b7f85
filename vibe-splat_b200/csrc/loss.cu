// Loss: SSIM fields (shaders/train_ssim.comp:42-123), then the adjoint
// dL/dImage and L1 (shaders/train_loss.comp:52-113), for
//   L = (1 - lambda) mean|image - target| + lambda (1 - mean SSIM)
// over pixels and channels, 11x11 Gaussian window (sigma 1.5) cut off and
// renormalised at the image border. Both kernels run one block per 16x16
// tile: the tile and a 5-pixel halo are staged into shared memory once, a
// horizontal pass over the tile plus 5 rows above and below goes into shared
// memory, then a vertical pass out of it. Normalisations are multiplications
// by reciprocals (the reference's GLSL division is not correctly rounded
// either). The fields are stored as 9
// FP32 planes (P, Q, R per channel; 36 bytes per pixel instead of the
// reference's 48). Per-tile partial sums are added in FP64 on the GPU.
#include "kernels.cuh"

namespace sb {

namespace {

constexpr int kHalo = 5;
constexpr int kRows = kTileSize + 2 * kHalo;
constexpr int kSpan = kRows * kTileSize;
constexpr float kC1 = 0.0001f, kC2 = 0.0009f;

__constant__ float c_weights[11] = {0.00102838f, 0.00759876f, 0.03600077f, 0.10936069f, 0.21300554f, 0.26601172f,
                                    0.21300554f, 0.10936069f, 0.03600077f, 0.00759876f, 0.00102838f};

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
  while (v + 1 < views.count && tile >= views.v[v + 1].tileBase) ++v;
  return v;
}

// Sum over the block of 256 threads; valid in thread 0.
__device__ __forceinline__ float block_sum(float v, float *s_warp) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  if ((threadIdx.x & 31u) == 0) s_warp[threadIdx.x >> 5] = v;
  __syncthreads();
  float total = 0.0f;
  if (threadIdx.x == 0)
    for (int w = 0; w < kTilePixels / 32; ++w) total += s_warp[w];
  return total;
}

// The tile with a 5-pixel halo on every side, one float per pixel and
// plane, zero outside the image: a tap there adds an exact zero, as if the
// window had been cut at the border. The horizontal pass gives each thread
// two neighbouring outputs of a row, which share 10 of their 11 taps.
constexpr int kSpanCols = kTileSize + 2 * kHalo;
constexpr int kStage = kRows * kSpanCols;
constexpr int kStagePlane = kStage;
constexpr int kPairs = kRows * kTileSize / 2; // horizontal work items
__device__ __forceinline__ int stage_row(int r) { return r * kSpanCols; }

__global__ void __launch_bounds__(kTilePixels) k_ssim(const float4 *__restrict__ image, const uint32_t *__restrict__ target,
                                                      const ViewSet *__restrict__ viewsPtr, float *__restrict__ fields,
                                                      float2 *__restrict__ partials) {
  const ViewSet &views = *viewsPtr;
  __shared__ float s_in[6][kStagePlane]; // image r, g, b, then target r, g, b
  __shared__ float s_h[5][3][kSpan];
  __shared__ float s_warp[kTilePixels / 32];
  const int tile = blockIdx.x;
  const ViewParams &cam = views.v[view_of_tile(views, tile)];
  const int local = tile - cam.tileBase;
  const int W = cam.width, H = cam.height;
  const int x0 = (local % cam.gridW) * kTileSize, y0 = (local / cam.gridW) * kTileSize;
  const size_t base = (size_t)cam.pixelBase;
  const size_t plane = (size_t)views.totalPixels;

  for (int i = threadIdx.x; i < kStage; i += kTilePixels) {
    const int r = i / kSpanCols, c = i % kSpanCols;
    const int y = y0 + r - kHalo, x = x0 + c - kHalo;
    float4 a4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float3 b3 = make_float3(0.f, 0.f, 0.f);
    if (y >= 0 && y < H && x >= 0 && x < W) {
      const size_t at = base + (size_t)y * W + x;
      a4 = image[at];
      b3 = unpack_unorm(target[at]);
    }
    const int o = stage_row(r) + c;
    s_in[0][o] = a4.x;
    s_in[1][o] = a4.y;
    s_in[2][o] = a4.z;
    s_in[3][o] = b3.x;
    s_in[4][o] = b3.y;
    s_in[5][o] = b3.z;
  }
  __syncthreads();

  // Horizontal pass: tile columns, tile rows plus the halo rows, two
  // neighbouring columns per thread.
  for (int i = threadIdx.x; i < kPairs; i += kTilePixels) {
    const int r = i / (kTileSize / 2), c = 2 * (i % (kTileSize / 2));
    const int y = y0 + r - kHalo, x = x0 + c;
    float m[2][5][3] = {};
    if (y >= 0 && y < H && x < W) {
      const int row = stage_row(r) + c;
#pragma unroll
      for (int u = 0; u < 12; ++u) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float a = s_in[k][row + u], b = s_in[3 + k][row + u];
#pragma unroll
          for (int o = 0; o < 2; ++o) {
            const int tap = u - o; // output c + o takes staged column c + o + tap
            if (tap < 0 || tap > 10) continue;
            const float w = c_weights[tap];
            const float wa = w * a;
            m[o][0][k] = fmaf(w, a, m[o][0][k]);
            m[o][1][k] = fmaf(w, b, m[o][1][k]);
            m[o][2][k] = fmaf(wa, a, m[o][2][k]);
            m[o][3][k] = fmaf(w * b, b, m[o][3][k]);
            m[o][4][k] = fmaf(wa, b, m[o][4][k]);
          }
        }
      }
#pragma unroll
      for (int o = 0; o < 2; ++o) {
        const float inv = x + o < W ? 1.0f / window_norm(x + o, W) : 0.0f;
#pragma unroll
        for (int q = 0; q < 5; ++q)
#pragma unroll
          for (int k = 0; k < 3; ++k) m[o][q][k] *= inv;
      }
    }
#pragma unroll
    for (int o = 0; o < 2; ++o)
#pragma unroll
      for (int q = 0; q < 5; ++q)
#pragma unroll
        for (int k = 0; k < 3; ++k) s_h[q][k][r * kTileSize + c + o] = m[o][q][k];
  }
  __syncthreads();

  const int px = x0 + (threadIdx.x & 15), py = y0 + (threadIdx.x >> 4);
  float own = 0.0f;
  if (px < W && py < H) {
    const float rowNorm = window_norm(py, H);
    float m[5][3] = {};
    const int v0 = max(py - 5, 0), v1 = min(py + 5, H - 1);
    for (int v = v0; v <= v1; ++v) {
      const float w = c_weights[v - py + 5];
      const int at = (v - y0 + kHalo) * kTileSize + (threadIdx.x & 15);
#pragma unroll
      for (int q = 0; q < 5; ++q)
#pragma unroll
        for (int k = 0; k < 3; ++k) m[q][k] = fmaf(w, s_h[q][k][at], m[q][k]);
    }
    const float invRow = 1.0f / rowNorm;
    const float invNorm = 1.0f / (rowNorm * window_norm(px, W));
    const size_t pixel = base + (size_t)py * W + px;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float mx = m[0][k] * invRow, my = m[1][k] * invRow;
      const float vx = m[2][k] * invRow - mx * mx, vy = m[3][k] * invRow - my * my, cxy = m[4][k] * invRow - mx * my;
      const float n1 = 2.0f * mx * my + kC1, n2 = 2.0f * cxy + kC2;
      const float d1 = mx * mx + my * my + kC1, d2 = vx + vy + kC2;
      const float invD = 1.0f / (d1 * d2), invD1 = 1.0f / d1, invD2 = 1.0f / d2;
      const float s = (n1 * n2) * invD;
      own += s;
      // n1 and n2 cancelled by hand, as the reference does: n2 can be zero.
      const float dMu = 2.0f * my * n2 * invD - s * 2.0f * mx * invD1;
      const float dVar = -s * invD2;
      const float dCov = 2.0f * n1 * invD;
      fields[(0 * 3 + k) * plane + pixel] = (dMu - 2.0f * mx * dVar - my * dCov) * invNorm;
      fields[(1 * 3 + k) * plane + pixel] = dVar * invNorm;
      fields[(2 * 3 + k) * plane + pixel] = dCov * invNorm;
    }
  }
  const float total = block_sum(own, s_warp);
  if (threadIdx.x == 0) partials[tile].x = total;
}

__global__ void __launch_bounds__(kTilePixels) k_loss(const float4 *__restrict__ image, const uint32_t *__restrict__ target,
                                                      const float *__restrict__ fields, const ViewSet *__restrict__ viewsPtr,
                                                      float lambda, float4 *__restrict__ adjoint, float2 *__restrict__ partials) {
  const ViewSet &views = *viewsPtr;
  __shared__ float s_in[9][kStagePlane]; // the nine field planes
  __shared__ float s_h[3][3][kSpan];
  __shared__ float s_warp[kTilePixels / 32];
  const int tile = blockIdx.x;
  const ViewParams &cam = views.v[view_of_tile(views, tile)];
  const int local = tile - cam.tileBase;
  const int W = cam.width, H = cam.height;
  const int x0 = (local % cam.gridW) * kTileSize, y0 = (local / cam.gridW) * kTileSize;
  const size_t base = (size_t)cam.pixelBase;
  const size_t plane = (size_t)views.totalPixels;

  for (int i = threadIdx.x; i < kStage; i += kTilePixels) {
    const int r = i / kSpanCols, c = i % kSpanCols;
    const int y = y0 + r - kHalo, x = x0 + c - kHalo;
    const bool in = y >= 0 && y < H && x >= 0 && x < W;
    const size_t at = in ? base + (size_t)y * W + x : 0;
    const int o = stage_row(r) + c;
#pragma unroll
    for (int f = 0; f < 9; ++f) s_in[f][o] = in ? fields[f * plane + at] : 0.0f;
  }
  __syncthreads();

  for (int i = threadIdx.x; i < kPairs; i += kTilePixels) {
    const int r = i / (kTileSize / 2), c = 2 * (i % (kTileSize / 2));
    const int y = y0 + r - kHalo, x = x0 + c;
    float m[2][3][3] = {};
    if (y >= 0 && y < H && x < W) {
      const int row = stage_row(r) + c;
#pragma unroll
      for (int u = 0; u < 12; ++u) {
#pragma unroll
        for (int f = 0; f < 9; ++f) {
          const float v = s_in[f][row + u];
#pragma unroll
          for (int o = 0; o < 2; ++o) {
            const int tap = u - o;
            if (tap < 0 || tap > 10) continue;
            m[o][f / 3][f % 3] = fmaf(c_weights[tap], v, m[o][f / 3][f % 3]);
          }
        }
      }
      if (x + 1 >= W) {
#pragma unroll
        for (int q = 0; q < 3; ++q)
#pragma unroll
          for (int k = 0; k < 3; ++k) m[1][q][k] = 0.0f;
      }
    }
#pragma unroll
    for (int o = 0; o < 2; ++o)
#pragma unroll
      for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int k = 0; k < 3; ++k) s_h[q][k][r * kTileSize + c + o] = m[o][q][k];
  }
  __syncthreads();

  const int px = x0 + (threadIdx.x & 15), py = y0 + (threadIdx.x >> 4);
  float own = 0.0f;
  if (px < W && py < H) {
    const float perValue = cam.perPixel;
    const size_t pixel = base + (size_t)py * W + px;
    const float4 x4 = image[pixel];
    const float3 y3 = unpack_unorm(target[pixel]);
    const float xv[3] = {x4.x, x4.y, x4.z}, yv[3] = {y3.x, y3.y, y3.z};
    float m[3][3] = {};
    const int v0 = max(py - 5, 0), v1 = min(py + 5, H - 1);
    for (int v = v0; v <= v1; ++v) {
      const float w = c_weights[v - py + 5];
      const int at = (v - y0 + kHalo) * kTileSize + (threadIdx.x & 15);
#pragma unroll
      for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int k = 0; k < 3; ++k) m[q][k] = fmaf(w, s_h[q][k][at], m[q][k]);
    }
    float result[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const float d = xv[k] - yv[k];
      own += fabsf(d);
      const float sgn = d > 0.0f ? 1.0f : (d < 0.0f ? -1.0f : 0.0f);
      const float ssimPart = m[0][k] + 2.0f * xv[k] * m[1][k] + yv[k] * m[2][k];
      result[k] = ((1.0f - lambda) * sgn - lambda * ssimPart) * perValue;
    }
    adjoint[pixel] = make_float4(result[0], result[1], result[2], 0.0f);
  }
  const float total = block_sum(own, s_warp);
  if (threadIdx.x == 0) partials[tile].y = total;
}

__global__ void __launch_bounds__(256) k_loss_totals(const float2 *__restrict__ partials, const ViewSet *__restrict__ viewsPtr,
                                                     LossTotals *totals) {
  const ViewSet &views = *viewsPtr;
  __shared__ double s_ssim[256], s_l1[256];
  const int v = blockIdx.x;
  const ViewParams &cam = views.v[v];
  double ssim = 0.0, l1 = 0.0;
  for (int i = threadIdx.x; i < cam.tileCount; i += 256) {
    const float2 p = partials[cam.tileBase + i];
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

void launch_ssim(const float4 *image, const uint32_t *target, const ViewSet &views, const ViewSet *dViews, float4 *fields, float2 *partials,
                 cudaStream_t stream) {
  if (views.totalTiles == 0) return;
  k_ssim<<<views.totalTiles, kTilePixels, 0, stream>>>(image, target, dViews, reinterpret_cast<float *>(fields), partials);
}

void launch_loss(const float4 *image, const uint32_t *target, const float4 *fields, const ViewSet &views, const ViewSet *dViews, float lambda,
                 float4 *adjoint, float2 *partials, cudaStream_t stream) {
  if (views.totalTiles == 0) return;
  k_loss<<<views.totalTiles, kTilePixels, 0, stream>>>(image, target, reinterpret_cast<const float *>(fields), dViews, lambda,
                                                       adjoint, partials);
}

void launch_loss_totals(const float2 *partials, const ViewSet &views, const ViewSet *dViews, LossTotals *totals, cudaStream_t stream) {
  k_loss_totals<<<views.count, 256, 0, stream>>>(partials, dViews, totals);
}

} // namespace sb
