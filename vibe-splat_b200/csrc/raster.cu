// Forward compositing and its hand-written adjoint, one block of 16x16 threads
// per tile, one thread per pixel (shaders/train_forward.comp:38-100,
// shaders/train_backward.glsl:78-157).
//
// What differs from the reference, and why it changes no result:
//   * When a batch of splats is staged into shared memory, the staging thread
//     folds splat_pixels() and the radius test of splat_at()
//     (train_types.glsl:43-48,82-86) into two 16-bit masks, one bit per column
//     and per row of the tile, evaluated with the very expressions a pixel
//     would use. The per-pixel test becomes one AND; a warp whose two rows the
//     splat misses skips it without divergence.
//   * The backward pass reduces each splat's 14 sums over a warp with the
//     reference's transposed butterfly (reduce_and_add, train_backward.glsl
//     :51-76), lanes grouped exactly as the reference's 32-wide subgroups (two
//     rows of 16). Fixed point: each warp total is quantised as the reference
//     quantises it, then the warps of the tile add their integers in shared
//     memory and one global atomic per (tile, splat, value) adds the result.
//     Integer addition is associative, so the sums are bit-identical to the
//     reference's per-warp global atomics, with up to 8 times fewer of them.
//     Float: the same shared-memory pre-aggregation (float atomics are not
//     order-deterministic in the reference either).
#include <algorithm>
#include <mutex>
#include <unordered_map>
#include <type_traits>

#include "kernels.cuh"

namespace sb {

namespace {

constexpr int kBatch = kTilePixels; // splats staged per round, one per thread
constexpr int kGradValues = 12;     // sums per splat without scoring (values 12, 13 need the scoring pass)
constexpr int kAccStride = 13;      // shared accumulator words per staged splat (odd: no bank conflicts)

// A staged splat, 64 bytes in four 16-byte words so that a pixel reads only
// what it needs: first the tile's column (bits 0-15) and row (bits 16-31)
// masks with the centre and opacity, then -qxx/2, -qxy, -qyy/2 (exact
// rescalings of the conic) and the colour, then the conic itself for the
// backward pass.
struct __align__(16) Staged {
  uint32_t mask;
  float cx, cy, opacity;
  float hqx, nqy, hqz, r;
  float g, b, qx, qy;
  float qz;
  uint32_t index;
  uint32_t maskHi; // 32 x 32 tiles: the row bits (the column bits are in mask)
  float pad1;
};

__device__ __forceinline__ uint32_t to_u32_clamped(float v) { return (uint32_t)fminf(v, 4294967040.0f); }

// The global tile's view.
__device__ __forceinline__ int view_of_tile(const ViewSet &views, int tile) {
  int v = 0;
  while (v + 1 < views.count && tile >= views.v[v + 1].tileBase) ++v;
  return v;
}

// splat_pixels() and the radius test of splat_at(), per column and per row.
__device__ __forceinline__ uint32_t pixel_masks(const Splat &s, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1) {
  const float cx = s.centerExtent.x, cy = s.centerExtent.y, ex = s.centerExtent.z, ey = s.centerExtent.w;
  const float r = s.colorRadius.w;
  const uint32_t ax0 = max(to_u32_clamped(fmaxf(cx - ex - 0.5f, 0.0f)), x0);
  const uint32_t ay0 = max(to_u32_clamped(fmaxf(cy - ey - 0.5f, 0.0f)), y0);
  const uint32_t ax1 = min(to_u32_clamped(fmaxf(cx + ex + 0.5f, 0.0f)) + 1u, x1);
  const uint32_t ay1 = min(to_u32_clamped(fmaxf(cy + ey + 0.5f, 0.0f)) + 1u, y1);
  uint32_t mask = 0;
#pragma unroll
  for (int l = 0; l < kTileSize; ++l) {
    const uint32_t x = x0 + l, y = y0 + l;
    const float dx = ((float)x + 0.5f) - cx, dy = ((float)y + 0.5f) - cy;
    if (x >= ax0 && x < ax1 && !(fabsf(dx) > r)) mask |= 1u << l;
    if (y >= ay0 && y < ay1 && !(fabsf(dy) > r)) mask |= 1u << (16 + l);
  }
  return mask;
}

// Every field of a staged splat but its pixel masks.
template <class M> __device__ __forceinline__ Staged stage_fields(const Splat &s, uint32_t index) {
  Staged out;
  out.cx = s.centerExtent.x;
  out.cy = s.centerExtent.y;
  // The exponent's coefficients in the form's log base (a factor of 1 for the exact form).
  out.hqx = (-0.5f * s.conicOpacity.x) * M::kLogScale;
  out.nqy = (-s.conicOpacity.y) * M::kLogScale;
  out.hqz = (-0.5f * s.conicOpacity.z) * M::kLogScale;
  out.opacity = s.conicOpacity.w;
  out.r = s.colorRadius.x;
  out.g = s.colorRadius.y;
  out.b = s.colorRadius.z;
  out.qx = s.conicOpacity.x;
  out.qy = s.conicOpacity.y;
  out.qz = s.conicOpacity.z;
  out.mask = 0u;
  out.index = index;
  out.maskHi = 0u;
  out.pad1 = 0.0f;
  return out;
}

template <class M>
__device__ __forceinline__ Staged stage(const Splat &s, uint32_t index, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1) {
  Staged out = stage_fields<M>(s, index);
  out.mask = pixel_masks(s, x0, y0, x1, y1);
  return out;
}

// The tiles of the float two-pixel rasterizer: T x T pixels, T * T / 2
// threads, one warp per 8 x 8 block of pixels (two pixels per lane). A
// staged splat's pixel mask has T column bits then T row bits: 32 bits for
// the reference's 16 x 16 tiles, 64 for 32 x 32 ones.
template <int T> struct TileShape {
  static constexpr int kThreads = T * T / 2;
  static constexpr int kWarps = kThreads / 32;
  static constexpr int kBlocksX = T / 8;
  using Mask = typename std::conditional<(T > 16), unsigned long long, uint32_t>::type;
};

// splat_pixels() and the radius test of splat_at() per column and per row of
// a tile of T pixels (pixel_masks for any T).
template <int T>
__device__ __forceinline__ typename TileShape<T>::Mask pixel_masks_t(const Splat &s, uint32_t x0, uint32_t y0, uint32_t x1,
                                                                     uint32_t y1) {
  using Mask = typename TileShape<T>::Mask;
  const float cx = s.centerExtent.x, cy = s.centerExtent.y, ex = s.centerExtent.z, ey = s.centerExtent.w;
  const float r = s.colorRadius.w;
  const uint32_t ax0 = max(to_u32_clamped(fmaxf(cx - ex - 0.5f, 0.0f)), x0);
  const uint32_t ay0 = max(to_u32_clamped(fmaxf(cy - ey - 0.5f, 0.0f)), y0);
  const uint32_t ax1 = min(to_u32_clamped(fmaxf(cx + ex + 0.5f, 0.0f)) + 1u, x1);
  const uint32_t ay1 = min(to_u32_clamped(fmaxf(cy + ey + 0.5f, 0.0f)) + 1u, y1);
  Mask mask = 0;
#pragma unroll
  for (int l = 0; l < T; ++l) {
    const uint32_t x = x0 + l, y = y0 + l;
    const float dx = ((float)x + 0.5f) - cx, dy = ((float)y + 0.5f) - cy;
    if (x >= ax0 && x < ax1 && !(fabsf(dx) > r)) mask |= (Mask)1 << l;
    if (y >= ay0 && y < ay1 && !(fabsf(dy) > r)) mask |= (Mask)1 << (T + l);
  }
  return mask;
}

template <int T> __device__ __forceinline__ typename TileShape<T>::Mask staged_mask(const Staged &s) {
  if constexpr (T > 16) return (unsigned long long)s.mask | ((unsigned long long)s.maskHi << 32);
  else return s.mask;
}

// -0.5 (qxx dx^2 + qyy dy^2) - qxy dx dy, in this rounding order.
__device__ __forceinline__ float splat_power(const Staged &s, float dx, float dy) {
  const float pxy = fmaf(s.nqy, dy, s.hqx * dx);
  return fmaf(s.hqz * dy, dy, pxy * dx);
}

struct TileGeometry {
  int view;
  uint32_t x0, y0, x1, y1; // pixels of the tile, upper bounds exclusive
};

__device__ __forceinline__ TileGeometry tile_geometry(const ViewSet &views, int tile, uint32_t T = kTileSize) {
  TileGeometry g;
  g.view = view_of_tile(views, tile);
  const ViewParams &cam = views.v[g.view];
  const int local = tile - cam.tileBase;
  const uint32_t tx = local % cam.gridW, ty = local / cam.gridW;
  g.x0 = tx * T;
  g.y0 = ty * T;
  g.x1 = min(g.x0 + T, (uint32_t)cam.width);
  g.y1 = min(g.y0 + T, (uint32_t)cam.height);
  return g;
}

// An index outside the splat array can only come from a broken earlier stage:
// record it and stage a splat that covers no pixel.
template <class M>
__device__ __forceinline__ Staged stage_checked(const Splat *__restrict__ splats, uint32_t s, uint32_t splatLimit,
                                                const TileGeometry &geo, uint32_t *error) {
  if (s >= splatLimit) {
    atomicOr(error, kErrBadIndex);
    Staged empty{};
    empty.mask = 0u;
    empty.index = 0u;
    return empty;
  }
  return stage<M>(splats[s], s, geo.x0, geo.y0, geo.x1, geo.y1);
}

// Per-warp lists of the staged splats, as bitmaps: word w of warp v has bit b
// set when splat 32 w + b reaches a pixel of warp v's block. The warps then
// walk only their own splats; a splat that no pixel of the warp can take is
// one no lane would have taken, so nothing else changes. Every lane of the
// staging warp calls this (mask 0 for lanes without a splat); warps of the
// 1-pixel layout cover two rows of 16, those of the 2-pixel layout 8x8.
// Warp shapes: kStrips, 8 warps of two rows of 16 (the reference's groups);
// kBlocks8x4, 8 warps of 8 columns by 4 rows; kBlocks8x8, 4 warps of 8x8.
enum WarpShape { kStrips = 0, kBlocks8x4 = 1, kBlocks8x8 = 2 };

template <int SHAPE>
__device__ __forceinline__ void publish_cover(uint32_t mask, uint32_t word, uint32_t lane, uint32_t (*cover)[kBatch / 32],
                                              uint32_t warpsMet = 0xFFFFFFFFu) {
  constexpr int WARPS = SHAPE == kBlocks8x8 ? 4 : 8;
  uint32_t mine = 0;
#pragma unroll
  for (int w = 0; w < WARPS; ++w) {
    uint32_t cols, rows;
    if (SHAPE == kStrips) {
      cols = 0xFFFFu;
      rows = 3u << (16 + 2 * w);
    } else if (SHAPE == kBlocks8x4) {
      cols = 0xFFu << (8 * (w & 1));
      rows = 0xFu << (16 + 4 * (w >> 1));
    } else {
      cols = 0xFFu << (8 * (w & 1));
      rows = 0xFFu << (16 + 8 * (w >> 1));
    }
    const uint32_t b = __ballot_sync(0xFFFFFFFFu, (mask & cols) != 0u && (mask & rows) != 0u && ((warpsMet >> w) & 1u) != 0u);
    if (lane == (uint32_t)w) mine = b;
  }
  if (lane < (uint32_t)WARPS) cover[lane][word] = mine;
}

// LISTS: 0 plain; 1 also counts each pixel's blended splats into
// lists.counts; 2 also records them, front to back, as (entry index, alpha)
// at lists.pool[lists.offsets[pixel] ...] (the store-everything variant).
template <class M, int LISTS>
__global__ void __launch_bounds__(kTilePixels) k_forward(const Splat *__restrict__ splats, const uint32_t *__restrict__ entryValues,
                                                         const uint2 *__restrict__ ranges, const ViewSet *__restrict__ viewsPtr,
                                                         float bgR, float bgG, float bgB, float4 *__restrict__ image,
                                                         uint32_t *__restrict__ stops, BlendLists lists, uint32_t splatLimit,
                                                         uint32_t *error) {
  chain_enter();
  const ViewSet &views = *viewsPtr;
  __shared__ Staged s_batch[kBatch];
  __shared__ uint32_t s_cover[kTilePixels / 32][kBatch / 32];
  if (error != nullptr && (*error & kErrEntryOverflow) != 0u) return;
  const int tile = blockIdx.x;
  const TileGeometry geo = tile_geometry(views, tile);
  const ViewParams &cam = views.v[geo.view];
  // Compositing needs no particular grouping of pixels into warps: warp w
  // takes the 8x4 block (w & 1, w >> 1), lane l its pixel (l & 7, l >> 3), a
  // shape that meets fewer splats than a strip of two rows.
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const uint32_t lx = (warp & 1u) * 8u + (lane & 7u), ly = (warp >> 1) * 4u + (lane >> 3);
  const uint32_t x = geo.x0 + lx, y = geo.y0 + ly;
  const bool inside = x < (uint32_t)cam.width && y < (uint32_t)cam.height;
  const uint32_t myBits = (1u << lx) | (1u << (16 + ly));
  const float pxf = (float)x + 0.5f, pyf = (float)y + 0.5f;

  const uint2 range = ranges[tile];
  float cr = 0.0f, cg = 0.0f, cb = 0.0f, T = 1.0f, logT = 0.0f;
  uint32_t stop = range.x;
  bool done = !inside;
  const size_t pixel = inside ? (size_t)cam.pixelBase + (size_t)y * cam.width + x : 0;
  uint32_t blended = 0;
  uint2 *list = nullptr;
  if (LISTS == 2 && inside) list = lists.pool + lists.offsets[pixel];
  for (uint32_t end = range.y; end > range.x;) {
    const uint32_t count = min((uint32_t)kBatch, end - range.x);
    end -= count;
    if (__syncthreads_count(done) == kTilePixels) break;
    uint32_t stagedMask = 0u;
    if (t < count) {
      const Staged st = stage_checked<M>(splats, entryValues[end + t], splatLimit, geo, error);
      s_batch[t] = st;
      stagedMask = st.mask;
    }
    publish_cover<kBlocks8x4>(stagedMask, warp, lane, s_cover);
    __syncthreads();
    // Back to front within the batch: the highest index first.
    for (int word = (int)((count - 1u) >> 5); word >= 0 && !done; --word) {
      for (uint32_t bits = s_cover[warp][word]; bits != 0u;) {
        const int bit = 31 - __clz(bits);
        bits ^= 1u << bit;
        const uint32_t k = (uint32_t)word * 32u + (uint32_t)bit;
        const Staged &s = s_batch[k];
        if ((s.mask & myBits) != myBits) continue;
        const float dx = pxf - s.cx, dy = pyf - s.cy;
        const float power = splat_power(s, dx, dy);
        if (power > 0.0f) continue;
        const float alpha = fminf(kAlphaMax, s.opacity * M::exp(power));
        if (!(alpha >= kAlphaMin)) continue;
        const float oneMinus = 1.0f - alpha;
        const float logRest = M::log(oneMinus);
        if (logT + logRest < kLogMinTransmittance * M::kLogScale) {
          stop = end + k + 1u;
          done = true;
          break;
        }
        const float w = T * alpha;
        cr = fmaf(w, s.r, cr);
        cg = fmaf(w, s.g, cg);
        cb = fmaf(w, s.b, cb);
        T = T * oneMinus;
        logT = logT + logRest;
        if (LISTS == 2) list[blended] = make_uint2(end + k, __float_as_uint(alpha));
        if (LISTS != 0) ++blended;
      }
    }
  }
  if (inside) {
    image[pixel] = make_float4(fmaf(T, bgR, cr), fmaf(T, bgG, cg), fmaf(T, bgB, cb), logT);
    stops[pixel] = stop;
    if (LISTS == 1) lists.counts[pixel] = blended;
  }
}

// The reference's transposed butterfly (reduce_and_add) over the 12 values the
// backward pass produces without scoring; lane l (< 16) ends up with the warp
// total of value bitreverse4(l). The reference pads to 16 values with zeros.
// In its first level the partners of values 4-7 are pads (12-15): a lower lane
// adds the same two numbers as the reference without selecting, and an upper
// lane's sum there stands for a pad total that no lane ever reads. Every total
// that is read is made of the same additions in the same order.
__device__ __forceinline__ float butterfly12(float v[12]) {
  const uint32_t lane = threadIdx.x & 31u;
  {
    const bool upper = (lane & 1u) != 0u;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float send = upper ? v[i] : v[i + 8];
      const float keep = upper ? v[i + 8] : v[i];
      v[i] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, 1);
    }
#pragma unroll
    for (int i = 4; i < 8; ++i) v[i] = v[i] + __shfl_xor_sync(0xFFFFFFFFu, v[i], 1);
  }
#define SB_HALVE(offset, count)                                           \
  {                                                                       \
    const bool upper = (lane & (offset)) != 0u;                           \
    _Pragma("unroll") for (int i = 0; i < (count) / 2; ++i) {             \
      const float send = upper ? v[i] : v[i + (count) / 2];               \
      const float keep = upper ? v[i + (count) / 2] : v[i];               \
      v[i] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, (offset));         \
    }                                                                     \
  }
  SB_HALVE(2, 8)
  SB_HALVE(4, 4)
  SB_HALVE(8, 2)
  return v[0] + __shfl_xor_sync(0xFFFFFFFFu, v[0], 16);
}

// The same over all 16 values (a scored view's 14, padded with zeros as the
// reference pads them): lane l (< 16) ends up with the warp total of value
// bitreverse4(l); the totals of values 0-11 are those of butterfly12.
__device__ __forceinline__ float butterfly16(float v[16]) {
  const uint32_t lane = threadIdx.x & 31u;
  SB_HALVE(1, 16)
  SB_HALVE(2, 8)
  SB_HALVE(4, 4)
  SB_HALVE(8, 2)
  return v[0] + __shfl_xor_sync(0xFFFFFFFFu, v[0], 16);
}
#undef SB_HALVE

// SCORE (a scored view): also values 12 and 13, the pixels marked as high
// error in the adjoint's alpha and the edge weight times the blending weight,
// each over 3 pixels of the image (train_backward.glsl:125-126).
template <bool SCORE> __host__ __device__ constexpr int score_values() { return SCORE ? kGradValues + 2 : kGradValues; }
template <bool SCORE> __host__ __device__ constexpr int score_stride() { return SCORE ? kGradValues + 3 : kAccStride; }

template <class M, bool FIXED, bool SCORE>
__global__ void __launch_bounds__(kTilePixels, 4)
    k_backward(const Splat *__restrict__ splats, const uint32_t *__restrict__ entryValues, const uint2 *__restrict__ ranges,
               const ViewSet *__restrict__ viewsPtr, float bgR, float bgG, float bgB, const float4 *__restrict__ image,
               const float4 *__restrict__ adjoint, const uint32_t *__restrict__ stops, void *__restrict__ rawOut,
               uint32_t splatLimit, uint32_t *error, const float *__restrict__ edge) {
  chain_enter();
  constexpr int kValues = score_values<SCORE>(), kStride = score_stride<SCORE>();
  const ViewSet &views = *viewsPtr;
  __shared__ Staged s_batch[kBatch];
  __shared__ uint32_t s_acc[kBatch * kStride];
  __shared__ uint32_t s_min[kTilePixels / 32];
  __shared__ uint32_t s_cover[kTilePixels / 32][kBatch / 32];
  if (error != nullptr && (*error & kErrEntryOverflow) != 0u) return;
  const int tile = blockIdx.x;
  const TileGeometry geo = tile_geometry(views, tile);
  const ViewParams &cam = views.v[geo.view];
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5, lx = t & 15u, ly = t >> 4;
  const uint32_t x = geo.x0 + lx, y = geo.y0 + ly;
  const bool inside = x < (uint32_t)cam.width && y < (uint32_t)cam.height;
  const uint32_t myBits = (1u << lx) | (1u << (16 + ly));
  const float pxf = (float)x + 0.5f, pyf = (float)y + 0.5f;
  const size_t at = inside ? (size_t)cam.pixelBase + (size_t)y * cam.width + x : 0;
  const float logTotal = inside ? image[at].w : 0.0f;
  float4 A = inside ? adjoint[at] : make_float4(0.f, 0.f, 0.f, 0.f);
  const float edgeWeight = SCORE && inside ? edge[at] : 0.0f;
  const float perPixel = cam.perPixel;
  const float scale = cam.fixedScale;
  const uint2 range = ranges[tile];
  const uint32_t stop = inside ? stops[at] : range.y;
  const uint32_t warpMin = __reduce_min_sync(0xFFFFFFFFu, stop);
  if (lane == 0) s_min[t >> 5] = warpMin;
  for (int i = t; i < kBatch * kStride; i += kTilePixels) s_acc[i] = 0u;
  __syncthreads();
  uint32_t tileStop = s_min[0];
#pragma unroll
  for (int w = 1; w < kTilePixels / 32; ++w) tileStop = min(tileStop, s_min[w]);

  // The composite behind the current splat, and its log transmittance.
  float Br = bgR, Bg = bgG, Bb = bgB, logBehind = 0.0f;
  // Index of value bitreverse4(lane) held by this lane after the butterfly.
  const uint32_t held = __brev(lane) >> 28;
  uint32_t *raw32 = static_cast<uint32_t *>(rawOut);

  for (uint32_t start = tileStop; start < range.y; start += kBatch) {
    const uint32_t count = min((uint32_t)kBatch, range.y - start);
    __syncthreads();
    uint32_t stagedMask = 0u;
    if (t < count) {
      const Staged st = stage_checked<M>(splats, entryValues[start + t], splatLimit, geo, error);
      s_batch[t] = st;
      stagedMask = st.mask;
    }
    publish_cover<kStrips>(stagedMask, warp, lane, s_cover);
    __syncthreads();
    // Front to back: the lowest index first. The walk is warp-uniform.
    for (uint32_t word = 0; word <= ((count - 1u) >> 5); ++word)
    for (uint32_t bits = s_cover[warp][word]; bits != 0u; bits &= bits - 1u) {
      const uint32_t k = word * 32u + (uint32_t)(__ffs(bits) - 1);
      const Staged &s = s_batch[k];
      const uint32_t mask = s.mask;
      // The tests of splat_at() first; one vote decides whether the warp has work.
      const float dx = pxf - s.cx, dy = pyf - s.cy;
      const float power = splat_power(s, dx, dy);
      // exp of a clamped power: an inactive lane may have power > 0, and its
      // exp must stay finite because it is multiplied by zero below.
      const float ep = M::exp(fminf(power, 0.0f));
      const float oe = s.opacity * ep;
      const float alpha = fminf(kAlphaMax, oe);
      const bool act = start + k >= stop && (mask & myBits) == myBits && !(power > 0.0f) && alpha >= kAlphaMin;
      if (!__any_sync(0xFFFFFFFFu, act)) continue;
      // The warp's arithmetic without branches: an inactive lane takes alpha
      // and the weights as exact zeros, which leaves its B and log T behind as
      // they were and adds zeros to the sums.
      const float aAct = act ? alpha : 0.0f;
      const float logRest = M::log(1.0f - aAct);
      const float T = M::exp((logTotal - logBehind) - logRest);
      const float wA = act ? T * alpha : 0.0f;
      float g[SCORE ? 16 : 12];
      if constexpr (SCORE) {
        g[12] = act ? A.w * perPixel : 0.0f;
        g[13] = edgeWeight * wA * perPixel;
        g[14] = g[15] = 0.0f;
      }
      g[6] = wA * A.x;
      g[7] = wA * A.y;
      g[8] = wA * A.z;
      g[9] = wA * perPixel;
      // At the 0.99 clamp alpha no longer depends on the parameters.
      const float dAlpha = (act && oe < kAlphaMax) ? T * fmaf(A.z, s.b - Bb, fmaf(A.y, s.g - Bg, A.x * (s.r - Br))) : 0.0f;
      g[0] = dAlpha * ep;
      const float dPower = dAlpha * alpha;
      const float vx = fmaf(s.qy, dy, s.qx * dx), vy = fmaf(s.qz, dy, s.qy * dx);
      g[1] = dPower * vx;
      g[2] = dPower * vy;
      g[10] = fabsf(g[1]);
      g[11] = fabsf(g[2]);
      const float h = dPower * 0.5f;
      g[3] = h * vx * vx;
      g[4] = h * vx * vy;
      g[5] = h * vy * vy;
      Br = fmaf(aAct, s.r - Br, Br);
      Bg = fmaf(aAct, s.g - Bg, Bg);
      Bb = fmaf(aAct, s.b - Bb, Bb);
      logBehind = logBehind + logRest;
      float total;
      if constexpr (SCORE) total = butterfly16(g);
      else total = butterfly12(g);
      if (lane < 16 && held < (uint32_t)kValues && total != 0.0f) {
        uint32_t *slot = &s_acc[k * kStride + held];
        if (FIXED) {
          atomicAdd(reinterpret_cast<int *>(slot), __float2int_rn(fminf(fmaxf(total * scale, -1.0e9f), 1.0e9f)));
        } else {
          atomicAdd(reinterpret_cast<float *>(slot), total);
        }
      }
    }
    __syncthreads();
    // One global atomic per (splat, value) for the whole tile.
    if (t < count && s_batch[t].mask != 0u) {
      const size_t base = ((size_t)s_batch[t].index) * kRawStride;
#pragma unroll
      for (int j = 0; j < kValues; ++j) {
        const uint32_t v = s_acc[t * kStride + j];
        if (v != 0u) {
          if (FIXED) {
            atomicAdd(reinterpret_cast<int *>(raw32 + base + j), (int)v);
          } else {
            atomicAdd(reinterpret_cast<float *>(raw32 + base + j), __uint_as_float(v));
          }
          s_acc[t * kStride + j] = 0u;
        }
      }
    }
  }
}

// The store-everything backward (float sums): each pixel walks the list of
// (entry index, alpha) its forward recorded, from the back, instead of
// recomputing alpha and the transmittance: T in front of a splat is the
// transmittance behind it divided by (1 - alpha). One pixel per thread, the
// reference's 16x2 warps and butterfly; the per-splat arithmetic of the
// gradients is that of k_backward.
template <class M>
__global__ void __launch_bounds__(kTilePixels, 4)
    k_backward_lists(const Splat *__restrict__ splats, const uint32_t *__restrict__ entryValues, const uint2 *__restrict__ ranges,
                     const ViewSet *__restrict__ viewsPtr, float bgR, float bgG, float bgB, const float4 *__restrict__ image,
                     const float4 *__restrict__ adjoint, const uint32_t *__restrict__ stops, BlendLists lists,
                     float *__restrict__ raw, uint32_t splatLimit, uint32_t *error) {
  chain_enter();
  const ViewSet &views = *viewsPtr;
  __shared__ Staged s_batch[kBatch];
  __shared__ float s_acc[kBatch * kAccStride];
  __shared__ uint32_t s_min[kTilePixels / 32];
  __shared__ uint32_t s_cover[kTilePixels / 32][kBatch / 32];
  if (error != nullptr && (*error & kErrEntryOverflow) != 0u) return;
  const int tile = blockIdx.x;
  const TileGeometry geo = tile_geometry(views, tile);
  const ViewParams &cam = views.v[geo.view];
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5, lx = t & 15u, ly = t >> 4;
  const uint32_t x = geo.x0 + lx, y = geo.y0 + ly;
  const bool inside = x < (uint32_t)cam.width && y < (uint32_t)cam.height;
  const uint32_t myBits = (1u << lx) | (1u << (16 + ly));
  const float pxf = (float)x + 0.5f, pyf = (float)y + 0.5f;
  const size_t at = inside ? (size_t)cam.pixelBase + (size_t)y * cam.width + x : 0;
  // Transmittance behind everything the pixel blended.
  float Tcur = inside ? M::exp(image[at].w) : 1.0f;
  const float4 A = inside ? adjoint[at] : make_float4(0.f, 0.f, 0.f, 0.f);
  const float perPixel = cam.perPixel;
  const uint2 range = ranges[tile];
  const uint32_t stop = inside ? stops[at] : range.y;
  // The list, walked from its end (the farthest blended splat).
  const uint2 *list = lists.pool + (inside ? lists.offsets[at] : 0u);
  int cursor = inside ? (int)lists.counts[at] - 1 : -1;
  uint2 next = cursor >= 0 ? list[cursor] : make_uint2(0xFFFFFFFFu, 0u);
  const uint32_t warpMin = __reduce_min_sync(0xFFFFFFFFu, stop);
  if (lane == 0) s_min[warp] = warpMin;
  for (int i = t; i < kBatch * kAccStride; i += kTilePixels) s_acc[i] = 0.0f;
  __syncthreads();
  uint32_t tileStop = s_min[0];
#pragma unroll
  for (int w = 1; w < kTilePixels / 32; ++w) tileStop = min(tileStop, s_min[w]);

  float Br = bgR, Bg = bgG, Bb = bgB;
  const uint32_t held = __brev(lane) >> 28;

  for (uint32_t start = tileStop; start < range.y; start += kBatch) {
    const uint32_t count = min((uint32_t)kBatch, range.y - start);
    __syncthreads();
    uint32_t stagedMask = 0u;
    if (t < count) {
      const Staged st = stage_checked<M>(splats, entryValues[start + t], splatLimit, geo, error);
      s_batch[t] = st;
      stagedMask = st.mask;
    }
    publish_cover<kStrips>(stagedMask, warp, lane, s_cover);
    __syncthreads();
    for (uint32_t word = 0; word <= ((count - 1u) >> 5); ++word)
    for (uint32_t bits = s_cover[warp][word]; bits != 0u; bits &= bits - 1u) {
      const uint32_t k = word * 32u + (uint32_t)(__ffs(bits) - 1);
      const bool act = next.x == start + k;
      if (!__any_sync(0xFFFFFFFFu, act)) continue;
      const Staged &s = s_batch[k];
      const float alpha = act ? __uint_as_float(next.y) : 0.0f;
      const float Tf = Tcur * __frcp_rn(1.0f - alpha);
      const float wA = Tf * alpha;
      const float dx = pxf - s.cx, dy = pyf - s.cy;
      float g[12];
      g[6] = wA * A.x;
      g[7] = wA * A.y;
      g[8] = wA * A.z;
      g[9] = wA * perPixel;
      // At the 0.99 clamp alpha no longer depends on the parameters; below it
      // alpha = opacity * exp(power).
      const float dAlpha = (act && alpha < kAlphaMax) ? Tf * fmaf(A.z, s.b - Bb, fmaf(A.y, s.g - Bg, A.x * (s.r - Br))) : 0.0f;
      g[0] = dAlpha * (alpha / s.opacity);
      const float dPower = dAlpha * alpha;
      const float vx = fmaf(s.qy, dy, s.qx * dx), vy = fmaf(s.qz, dy, s.qy * dx);
      g[1] = dPower * vx;
      g[2] = dPower * vy;
      g[10] = fabsf(g[1]);
      g[11] = fabsf(g[2]);
      const float h = dPower * 0.5f;
      g[3] = h * vx * vx;
      g[4] = h * vx * vy;
      g[5] = h * vy * vy;
      Br = fmaf(alpha, s.r - Br, Br);
      Bg = fmaf(alpha, s.g - Bg, Bg);
      Bb = fmaf(alpha, s.b - Bb, Bb);
      if (act) {
        Tcur = Tf;
        --cursor;
        next = cursor >= 0 ? list[cursor] : make_uint2(0xFFFFFFFFu, 0u);
      }
      const float total = butterfly12(g);
      if (lane < 16 && held < (uint32_t)kGradValues && total != 0.0f) atomicAdd(&s_acc[k * kAccStride + held], total);
    }
    __syncthreads();
    // One global atomic per (splat, value) for the whole tile.
    if (t < count && s_batch[t].mask != 0u) {
      float *dst = raw + (size_t)s_batch[t].index * kRawStride;
#pragma unroll
      for (int j = 0; j < kGradValues; ++j) {
        const float v = s_acc[t * kAccStride + j];
        if (v != 0.0f) {
          atomicAdd(dst + j, v);
          s_acc[t * kAccStride + j] = 0.0f;
        }
      }
    }
  }
}

// Two pixels per thread, for the forms whose sums need not follow the
// reference's 32-lane groups: T * T / 2 threads per tile of T x T pixels,
// warp w covering the 8x8 block (w % (T / 8), w / (T / 8)), lane l its pixels
// (l & 7, l >> 3) and (l & 7, (l >> 3) + 4). The per-pixel arithmetic is that
// of k_forward and k_backward; what changes is that a warp skips a splat that
// misses its 8x8 block, and that a staged splat's record and (backward) its
// reduction serve two pixels per lane.
constexpr int kHalfTile = kTilePixels / 2;

template <int T> struct PixelPair {
  uint32_t x[2], y[2];
  typename TileShape<T>::Mask bits[2];
  float px[2], py[2];
  bool inside[2];
};

template <int T>
__device__ __forceinline__ PixelPair<T> pixel_pair(const TileGeometry &geo, const ViewParams &cam, uint32_t t) {
  using Mask = typename TileShape<T>::Mask;
  PixelPair<T> pp;
  const uint32_t warp = t >> 5, lane = t & 31u;
  const uint32_t bx = (warp % TileShape<T>::kBlocksX) * 8u, by = (warp / TileShape<T>::kBlocksX) * 8u;
  const uint32_t lx = bx + (lane & 7u), ly = by + (lane >> 3);
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const uint32_t yy = ly + 4u * q;
    pp.x[q] = geo.x0 + lx;
    pp.y[q] = geo.y0 + yy;
    pp.bits[q] = ((Mask)1 << lx) | ((Mask)1 << (T + yy));
    pp.px[q] = (float)pp.x[q] + 0.5f;
    pp.py[q] = (float)pp.y[q] + 0.5f;
    pp.inside[q] = pp.x[q] < (uint32_t)cam.width && pp.y[q] < (uint32_t)cam.height;
  }
  return pp;
}

// Whether the cutoff ellipse {d : d' Q d <= reach} (Q = [qx qy; qy qz], the
// splat's conic) may reach a pixel centre of [lowX, highX] x [lowY, highY]
// (offsets from the splat's centre): the least of the quadratic over the
// rectangle lies on an edge, at the ellipse's tangent point clamped to it; the
// binning's margin covers the rounding of these SFU divisions. A warp whose
// pixel block fails it has no pixel with alpha >= 1/255 for that splat.
__device__ __forceinline__ bool ellipse_meets_rect(float qx, float qy, float qz, float reach, float lowX, float highX, float lowY,
                                                   float highY) {
  if (lowX <= 0.0f && lowY <= 0.0f && highX >= 0.0f && highY >= 0.0f) return true;
  float least = 1e30f;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const float x = side == 0 ? lowX : highX;
    const float y = fminf(fmaxf(__fdividef(-qy * x, qz), lowY), highY);
    least = fminf(least, qx * x * x + 2.0f * qy * x * y + qz * y * y);
    const float v = side == 0 ? lowY : highY;
    const float u = fminf(fmaxf(__fdividef(-qy * v, qx), lowX), highX);
    least = fminf(least, qx * u * u + 2.0f * qy * u * v + qz * v * v);
  }
  return least <= reach * 1.001f + 1e-3f;
}

// The 8x8-block bitmaps of a T x T tile (publish_cover's kBlocks8x8 for any
// T): word `word` of block w has bit b set when the staging warp's splat b
// reaches a pixel row and column of block w and `met` (the caller's finer test)
// has bit w. Every lane of the staging warp calls this.
template <int T, int B>
__device__ __forceinline__ void publish_blocks(typename TileShape<T>::Mask mask, uint32_t met, uint32_t word, uint32_t lane,
                                               uint32_t (*cover)[B / 32]) {
  using Mask = typename TileShape<T>::Mask;
  constexpr int W = TileShape<T>::kWarps;
  uint32_t mine = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) {
    const Mask cols = (Mask)0xFFu << (8 * (w % TileShape<T>::kBlocksX));
    const Mask rows = (Mask)0xFFu << (T + 8 * (w / TileShape<T>::kBlocksX));
    const uint32_t b = __ballot_sync(0xFFFFFFFFu, (mask & cols) != 0 && (mask & rows) != 0 && ((met >> w) & 1u) != 0u);
    if (lane == (uint32_t)w) mine = b;
  }
  if (lane < (uint32_t)W) cover[lane][word] = mine;
}

// Stages `count` (at most B) splats with the tile's T * T / 2 threads and
// publishes the 8x8-block bitmaps: a block is listed when the splat's masks
// reach it and its cutoff ellipse meets the block's pixel centres. With
// minStops (the backward pass), also only when the splat's entry (first + j)
// is at or after the least stop of the block's pixels: before it, every pixel
// there has stopped.
template <class M, int T, int B>
__device__ __forceinline__ void stage_pairs(const Splat *__restrict__ splats, const uint32_t *__restrict__ values, uint32_t count,
                                            uint32_t splatLimit, const TileGeometry &geo, uint32_t *error, Staged *batch,
                                            uint32_t (*cover)[B / 32], const uint32_t *minStops = nullptr,
                                            uint32_t first = 0u) {
  using Mask = typename TileShape<T>::Mask;
  constexpr int kThreads = TileShape<T>::kThreads, W = TileShape<T>::kWarps;
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
#pragma unroll
  for (uint32_t round = 0; round < (uint32_t)((B + kThreads - 1) / kThreads); ++round) {
    const uint32_t j = round * kThreads + t;
    Mask mask = 0;
    uint32_t met = 0u;
    if (j < count) {
      const uint32_t s = values[j];
      Staged st{};
      if (s >= splatLimit) {
        atomicOr(error, kErrBadIndex);
      } else {
        const Splat sp = splats[s];
        st = stage_fields<M>(sp, s);
        const Mask full = pixel_masks_t<T>(sp, geo.x0, geo.y0, geo.x1, geo.y1);
        st.mask = (uint32_t)full;
        st.maskHi = (uint32_t)((unsigned long long)full >> 32);
      }
      batch[j] = st;
      mask = staged_mask<T>(st);
      if (mask != 0) {
        // 2 ln(255 opacity): alpha >= 1/255 exactly where d' Q d <= reach.
        const float reach = 2.0f * __logf(255.0f * st.opacity);
#pragma unroll
        for (uint32_t w = 0; w < (uint32_t)W; ++w) {
          if (minStops != nullptr && first + j < minStops[w]) continue;
          const float lowX = ((float)(geo.x0 + (w % TileShape<T>::kBlocksX) * 8u) + 0.5f) - st.cx;
          const float lowY = ((float)(geo.y0 + (w / TileShape<T>::kBlocksX) * 8u) + 0.5f) - st.cy;
          if (ellipse_meets_rect(st.qx, st.qy, st.qz, reach, lowX, lowX + 7.0f, lowY, lowY + 7.0f)) met |= 1u << w;
        }
      }
    }
    // Only the warps whose 32 splats fall inside the batch publish.
    const uint32_t word = round * (kThreads / 32) + warp;
    if (word < (uint32_t)(B / 32)) publish_blocks<T, B>(mask, met, word, lane, cover);
  }
}

// Packed two-lane FP32 arithmetic (sm_100a): each lane of fma2/mul2/add2 is
// rounded once, exactly as fmaf / * / + on that lane alone, so a pixel pair
// computed this way gets the bits each pixel would get on its own.
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// c - a, lane by lane. Written as a packed fused multiply-add by the constant
// -1, it gave wrong sums inside k_backward2 with nvcc 12.9 for sm_100a (a
// stand-alone kernel computed the same form correctly), so it stays scalar.
__device__ __forceinline__ float2 rsub2(float2 a, float2 c) { return make_float2(c.x - a.x, c.y - a.y); }

// The exponent of a staged splat at a lane's two pixels, which share their
// column (dx) and sit 4 rows apart: splat_power() of each, in its rounding
// order, with the column's products computed once.
__device__ __forceinline__ float2 splat_power2(const Staged &s, float dx, float2 dy) {
  const float hx = s.hqx * dx;
  const float2 pxy = fma2(f2(s.nqy), dy, f2(hx));
  return fma2(mul2(f2(s.hqz), dy), dy, mul2(pxy, f2(dx)));
}

// Blocks per SM the two-pixel kernels are compiled for, by tile edge. The
// backward's eight (62 registers, no spills) were measured against six, seven,
// nine and ten at 1M Gaussians, 1237x822: 0.565 ms a pass against 0.586,
// 0.577, 0.579 and 0.58, with batches of 128 (whose shared memory lets eight
// blocks in).
template <int T> constexpr int forward2_blocks() { return T > 16 ? 2 : 8; }
template <int T> constexpr int backward2_blocks() { return T > 16 ? 1 : 8; }

// The next tile of a launch: blockIdx.x the first time, then, for a
// persistent launch (work not null: a grid of resident blocks), tiles of every
// view claimed from the launch's counter until they run out. Every thread of
// the block gets the same answer; -1 when the block is done.
// With an order (not null), the i-th tile taken is order[i] (heaviest first,
// k_tile_order) instead of tile i.
__device__ __forceinline__ int next_tile(uint32_t *work, uint32_t total, bool first, uint32_t *s_next,
                                         const uint32_t *order = nullptr) {
  if (work == nullptr) {
    if (!first) return -1;
    return order != nullptr ? (int)order[blockIdx.x] : (int)blockIdx.x;
  }
  __syncthreads(); // the previous tile is finished with shared memory
  if (threadIdx.x == 0) *s_next = atomicAdd(work, 1u);
  __syncthreads();
  const uint32_t tile = *s_next;
  if (tile >= total) return -1;
  return order != nullptr ? (int)order[tile] : (int)tile;
}

// The rasterizer's tiles, heaviest first (new here; the reference launches its
// tiles in raster order): tiles cost what they walk, from a few entries to
// thousands, and a launch whose heavy tiles start last ends with most SMs idle
// while those finish. Each tile's work (tileWork, or without it the length of
// its entry range) is put into one of 32 half-octave classes, and the tiles are
// listed class by class, heaviest class first; the order inside a class is
// the order in which the block's threads claim places (it changes which block
// takes which tile, not what any tile computes). One block.
constexpr int kOrderThreads = 1024, kOrderClasses = 32;

__device__ __forceinline__ uint32_t work_class(uint32_t work) {
  return work == 0u ? 0u : min((uint32_t)kOrderClasses - 1u, 1u + (uint32_t)(2.0f * __log2f((float)work)));
}

__global__ void __launch_bounds__(kOrderThreads) k_tile_order(const uint2 *__restrict__ ranges, const uint32_t *__restrict__ tileWork,
                                                              uint32_t tiles, uint32_t *__restrict__ order) {
  chain_enter();
  __shared__ uint32_t s_count[kOrderClasses];
  const uint32_t t = threadIdx.x, lane = t & 31u;
  if (t < (uint32_t)kOrderClasses) s_count[t] = 0u;
  __syncthreads();
  const uint32_t rounds = div_up(tiles, kOrderThreads);
  for (uint32_t r = 0; r < rounds; ++r) {
    const uint32_t i = r * kOrderThreads + t;
    const bool in = i < tiles;
    const uint32_t c = in ? work_class(tileWork != nullptr ? tileWork[i] : ranges[i].y - ranges[i].x) : kOrderClasses;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, c);
    if (in && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&s_count[c], (uint32_t)__popc(peers));
  }
  __syncthreads();
  if (t == 0) {
    uint32_t run = 0;
    for (int c = kOrderClasses - 1; c >= 0; --c) {
      const uint32_t k = s_count[c];
      s_count[c] = run;
      run += k;
    }
  }
  __syncthreads();
  for (uint32_t r = 0; r < rounds; ++r) {
    const uint32_t i = r * kOrderThreads + t;
    const bool in = i < tiles;
    const uint32_t c = in ? work_class(tileWork != nullptr ? tileWork[i] : ranges[i].y - ranges[i].x) : kOrderClasses;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, c);
    const uint32_t leader = (uint32_t)(__ffs(peers) - 1);
    uint32_t base = 0u;
    if (in && lane == leader) base = atomicAdd(&s_count[c], (uint32_t)__popc(peers));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (in) order[base + (uint32_t)__popc(peers & ((1u << lane) - 1u))] = i;
  }
}

template <class M, int T, int B>
__device__ __forceinline__ void forward2_tile(int tile, const Splat *__restrict__ splats, const uint32_t *__restrict__ entryValues,
                                              const uint2 *__restrict__ ranges, const ViewSet &views, float bgR, float bgG,
                                              float bgB, float4 *__restrict__ image, uint32_t *__restrict__ stops,
                                              uint32_t splatLimit, uint32_t *error, Staged *s_batch, uint32_t (*s_cover)[B / 32],
                                              uint32_t *tileWork, uint32_t *s_least) {
  constexpr int kThreads = TileShape<T>::kThreads;
  const TileGeometry geo = tile_geometry(views, tile, T);
  const ViewParams &cam = views.v[geo.view];
  const uint32_t t = threadIdx.x, warp = t >> 5;
  const PixelPair<T> pp = pixel_pair<T>(geo, cam, t);
  const uint2 range = ranges[tile];
  const float px = pp.px[0];
  const float2 py = make_float2(pp.py[0], pp.py[1]);
  const float logMin = kLogMinTransmittance * M::kLogScale;
  float2 cr = f2(0.0f), cg = f2(0.0f), cb = f2(0.0f), Tr = f2(1.0f), logT = f2(0.0f);
  uint32_t stop0 = range.x, stop1 = range.x;
  bool done0 = !pp.inside[0], done1 = !pp.inside[1];
  for (uint32_t end = range.y; end > range.x;) {
    const uint32_t count = min((uint32_t)B, end - range.x);
    end -= count;
    if (__syncthreads_count(done0 && done1) == kThreads) break;
    stage_pairs<M, T, B>(splats, entryValues + end, count, splatLimit, geo, error, s_batch, s_cover);
    __syncthreads();
    for (int word = (int)((count - 1u) >> 5); word >= 0 && !(done0 && done1); --word) {
    for (uint32_t bits = s_cover[warp][word]; bits != 0u;) {
      const int bit = 31 - __clz(bits);
      bits ^= 1u << bit;
      const uint32_t k = (uint32_t)word * 32u + (uint32_t)bit;
      const Staged &s = s_batch[k];
      const auto mask = staged_mask<T>(s);
      // Both pixels' tests of k_forward, the exponent and alpha packed.
      const float dx = px - s.cx;
      const float2 dy = add2(py, f2(-s.cy));
      const float2 power = splat_power2(s, dx, dy);
      const float2 oe = mul2(f2(s.opacity), make_float2(M::exp(power.x), M::exp(power.y)));
      const float a0 = fminf(kAlphaMax, oe.x), a1 = fminf(kAlphaMax, oe.y);
      const bool v0 = !done0 && (mask & pp.bits[0]) == pp.bits[0] && !(power.x > 0.0f) && a0 >= kAlphaMin;
      const bool v1 = !done1 && (mask & pp.bits[1]) == pp.bits[1] && !(power.y > 0.0f) && a1 >= kAlphaMin;
      if (!(v0 || v1)) continue;
      // A pixel that does not blend takes alpha 0: weight 0, factor 1 - 0 = 1
      // and log 1 = 0 (exact in both forms), so its update is an exact no-op
      // that needs no select. Its log T stays at or above the floor, so only
      // a blending pixel can stop.
      float2 alpha = make_float2(v0 ? a0 : 0.0f, v1 ? a1 : 0.0f);
      float2 oneMinus = rsub2(alpha, f2(1.0f));
      float2 next = add2(logT, make_float2(M::log(oneMinus.x), M::log(oneMinus.y)));
      if (next.x < logMin || next.y < logMin) {
        // A pixel whose transmittance would fall below the floor stops here,
        // and this splat changes nothing in it.
        if (next.x < logMin) {
          stop0 = end + k + 1u;
          done0 = true;
          alpha.x = 0.0f;
          oneMinus.x = 1.0f;
          next.x = logT.x;
        }
        if (next.y < logMin) {
          stop1 = end + k + 1u;
          done1 = true;
          alpha.y = 0.0f;
          oneMinus.y = 1.0f;
          next.y = logT.y;
        }
        const float2 w = mul2(Tr, alpha);
        cr = fma2(w, f2(s.r), cr);
        cg = fma2(w, f2(s.g), cg);
        cb = fma2(w, f2(s.b), cb);
        Tr = mul2(Tr, oneMinus);
        logT = next;
        if (done0 && done1) break;
        continue;
      }
      const float2 w = mul2(Tr, alpha);
      cr = fma2(w, f2(s.r), cr);
      cg = fma2(w, f2(s.g), cg);
      cb = fma2(w, f2(s.b), cb);
      Tr = mul2(Tr, oneMinus);
      logT = next;
    }
    }
  }
  if (pp.inside[0]) {
    const size_t at = (size_t)cam.pixelBase + (size_t)pp.y[0] * cam.width + pp.x[0];
    image[at] = make_float4(fmaf(Tr.x, bgR, cr.x), fmaf(Tr.x, bgG, cg.x), fmaf(Tr.x, bgB, cb.x), logT.x);
    stops[at] = stop0;
  }
  if (pp.inside[1]) {
    const size_t at = (size_t)cam.pixelBase + (size_t)pp.y[1] * cam.width + pp.x[1];
    image[at] = make_float4(fmaf(Tr.y, bgR, cr.y), fmaf(Tr.y, bgG, cg.y), fmaf(Tr.y, bgB, cb.y), logT.y);
    stops[at] = stop1;
  }
  if (tileWork != nullptr) {
    // The entries the backward pass walks here: from the least stop of the
    // tile's pixels to the end of its range.
    const uint32_t least = __reduce_min_sync(0xFFFFFFFFu, min(pp.inside[0] ? stop0 : range.y, pp.inside[1] ? stop1 : range.y));
    if ((t & 31u) == 0u) s_least[warp] = least;
    __syncthreads();
    if (t == 0) {
      uint32_t m = s_least[0];
#pragma unroll
      for (int w = 1; w < TileShape<T>::kWarps; ++w) m = min(m, s_least[w]);
      tileWork[tile] = range.y - m;
    }
  }
}

// Compositing, two pixels per thread, tiles of T x T pixels, batches of B
// staged splats; work: a persistent launch's tile counter (or null: one
// block per tile).
template <class M, int T, int B>
__global__ void __launch_bounds__(TileShape<T>::kThreads, forward2_blocks<T>())
    k_forward2(const Splat *__restrict__ splats, const uint32_t *__restrict__ entryValues, const uint2 *__restrict__ ranges,
               const ViewSet *__restrict__ viewsPtr, float bgR, float bgG, float bgB, float4 *__restrict__ image,
               uint32_t *__restrict__ stops, uint32_t splatLimit, uint32_t *error, uint32_t *work, const uint32_t *order,
               uint32_t *tileWork) {
  chain_enter();
  const ViewSet &views = *viewsPtr;
  __shared__ Staged s_batch[B];
  __shared__ uint32_t s_cover[TileShape<T>::kWarps][B / 32];
  __shared__ uint32_t s_least[TileShape<T>::kWarps];
  __shared__ uint32_t s_next;
  if (error != nullptr && (*error & kErrEntryOverflow) != 0u) return;
  for (int tile = next_tile(work, (uint32_t)views.totalTiles, true, &s_next, order); tile >= 0;
       tile = next_tile(work, (uint32_t)views.totalTiles, false, &s_next, order))
    forward2_tile<M, T, B>(tile, splats, entryValues, ranges, views, bgR, bgG, bgB, image, stops, splatLimit, error, s_batch,
                           s_cover, tileWork, s_least);
}

// Float sums only: each lane adds its two pixels' values before one
// butterfly. The per-pixel arithmetic runs on both pixels at once in packed
// FP32. One tile of T x T pixels, batches of B staged splats.
template <class M, bool SCORE, int T, int B>
__device__ __forceinline__ void backward2_tile(int tile, const Splat *__restrict__ splats, const uint32_t *__restrict__ entryValues,
                                               const uint2 *__restrict__ ranges, const ViewSet &views, float bgR, float bgG,
                                               float bgB, const float4 *__restrict__ image, const float4 *__restrict__ adjoint,
                                               const uint32_t *__restrict__ stops, float *__restrict__ raw, uint32_t splatLimit,
                                               uint32_t *error, const float *__restrict__ edge, Staged *s_batch, float *s_acc,
                                               uint32_t *s_min, uint32_t (*s_cover)[B / 32]) {
  constexpr int kValues = score_values<SCORE>(), kStride = score_stride<SCORE>();
  constexpr int kThreads = TileShape<T>::kThreads, W = TileShape<T>::kWarps;
  const TileGeometry geo = tile_geometry(views, tile, T);
  const ViewParams &cam = views.v[geo.view];
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const PixelPair<T> pp = pixel_pair<T>(geo, cam, t);
  const uint2 range = ranges[tile];
  // front: log T total minus the log transmittance of the splats already
  // walked (those behind), kept as one running value. behind: the adjoint
  // dotted with the colour the splats behind (and the background) give, the
  // one thing of that colour the alpha gradient needs. One lane per pixel.
  float fr[2], ax[2], ay[2], az[2], bh[2], mk[2], ew[2];
  uint32_t stop[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const size_t at = pp.inside[q] ? (size_t)cam.pixelBase + (size_t)pp.y[q] * cam.width + pp.x[q] : 0;
    fr[q] = pp.inside[q] ? image[at].w : 0.0f;
    const float4 a = pp.inside[q] ? adjoint[at] : make_float4(0.f, 0.f, 0.f, 0.f);
    ax[q] = a.x;
    ay[q] = a.y;
    az[q] = a.z;
    stop[q] = pp.inside[q] ? stops[at] : range.y;
    bh[q] = fmaf(a.z, bgB, fmaf(a.y, bgG, a.x * bgR));
    mk[q] = a.w;
    ew[q] = SCORE && pp.inside[q] ? edge[at] : 0.0f;
  }
  float2 front = make_float2(fr[0], fr[1]), behind = make_float2(bh[0], bh[1]);
  const float2 Ax = make_float2(ax[0], ax[1]), Ay = make_float2(ay[0], ay[1]), Az = make_float2(az[0], az[1]);
  const float2 marked = make_float2(mk[0], mk[1]), edgeWeight = make_float2(ew[0], ew[1]);
  const float px = pp.px[0];
  const float2 py = make_float2(pp.py[0], pp.py[1]);
  const float perPixel = cam.perPixel;
  const uint32_t warpMin = __reduce_min_sync(0xFFFFFFFFu, min(stop[0], stop[1]));
  if (lane == 0) s_min[t >> 5] = warpMin;
  for (int i = t; i < B * kStride; i += kThreads) s_acc[i] = 0.0f;
  __syncthreads();
  uint32_t tileStop = s_min[0];
#pragma unroll
  for (int w = 1; w < W; ++w) tileStop = min(tileStop, s_min[w]);
  const uint32_t held = __brev(lane) >> 28;

  for (uint32_t start = tileStop; start < range.y; start += B) {
    const uint32_t count = min((uint32_t)B, range.y - start);
    __syncthreads();
    stage_pairs<M, T, B>(splats, entryValues + start, count, splatLimit, geo, error, s_batch, s_cover, s_min, start);
    __syncthreads();
    for (uint32_t word = 0; word <= ((count - 1u) >> 5); ++word)
    for (uint32_t bits = s_cover[warp][word]; bits != 0u; bits &= bits - 1u) {
      const uint32_t k = word * 32u + (uint32_t)(__ffs(bits) - 1);
      const Staged &s = s_batch[k];
      const auto mask = staged_mask<T>(s);
      const float dx = px - s.cx;
      const float2 dy = add2(py, f2(-s.cy));
      const float2 power = splat_power2(s, dx, dy);
      const float2 ep = make_float2(M::exp(fminf(power.x, 0.0f)), M::exp(fminf(power.y, 0.0f)));
      const float2 oe = mul2(f2(s.opacity), ep);
      const float2 alpha = make_float2(fminf(kAlphaMax, oe.x), fminf(kAlphaMax, oe.y));
      const uint32_t entry = start + k;
      const bool act0 = entry >= stop[0] && (mask & pp.bits[0]) == pp.bits[0] && !(power.x > 0.0f) && alpha.x >= kAlphaMin;
      const bool act1 = entry >= stop[1] && (mask & pp.bits[1]) == pp.bits[1] && !(power.y > 0.0f) && alpha.y >= kAlphaMin;
      if (!__any_sync(0xFFFFFFFFu, act0 || act1)) continue;
      // An inactive pixel takes alpha 0: its front and behind stay as they
      // were and it adds zeros to the sums.
      const float2 aAct = make_float2(act0 ? alpha.x : 0.0f, act1 ? alpha.y : 0.0f);
      const float2 oneMinus = rsub2(aAct, f2(1.0f));
      const float2 logRest = make_float2(M::log(oneMinus.x), M::log(oneMinus.y));
      const float2 nextFront = rsub2(logRest, front);
      const float2 Tf = make_float2(M::exp(nextFront.x), M::exp(nextFront.y));
      const float2 wA = mul2(Tf, aAct);
      float g[SCORE ? 16 : 12];
      const float2 c6 = mul2(wA, Ax), c7 = mul2(wA, Ay), c8 = mul2(wA, Az);
      g[6] = c6.x + c6.y;
      g[7] = c7.x + c7.y;
      g[8] = c8.x + c8.y;
      g[9] = (wA.x + wA.y) * perPixel;
      if constexpr (SCORE) {
        g[12] = ((act0 ? marked.x : 0.0f) + (act1 ? marked.y : 0.0f)) * perPixel;
        const float2 e = mul2(edgeWeight, wA);
        g[13] = (e.x + e.y) * perPixel;
        g[14] = g[15] = 0.0f;
      }
      const float2 ahead = rsub2(behind, fma2(Az, f2(s.b), fma2(Ay, f2(s.g), mul2(Ax, f2(s.r)))));
      // At the 0.99 clamp alpha no longer depends on the parameters.
      const float2 dT = mul2(Tf, ahead);
      const float2 dAlpha = make_float2(act0 && oe.x < kAlphaMax ? dT.x : 0.0f, act1 && oe.y < kAlphaMax ? dT.y : 0.0f);
      const float2 c0 = mul2(dAlpha, ep);
      g[0] = c0.x + c0.y;
      const float2 dPower = mul2(dAlpha, alpha);
      const float2 vx = fma2(f2(s.qy), dy, f2(s.qx * dx)), vy = fma2(f2(s.qz), dy, f2(s.qy * dx));
      const float2 g1 = mul2(dPower, vx), g2 = mul2(dPower, vy);
      g[1] = g1.x + g1.y;
      g[2] = g2.x + g2.y;
      g[10] = fabsf(g1.x) + fabsf(g1.y);
      g[11] = fabsf(g2.x) + fabsf(g2.y);
      // Twice the conic sums; the flush halves them (exactly).
      const float2 c3 = mul2(g1, vx), c4 = mul2(g1, vy), c5 = mul2(g2, vy);
      g[3] = c3.x + c3.y;
      g[4] = c4.x + c4.y;
      g[5] = c5.x + c5.y;
      behind = fma2(aAct, ahead, behind);
      front = nextFront;
      float total;
      if constexpr (SCORE) total = butterfly16(g);
      else total = butterfly12(g);
      if (lane < 16 && held < (uint32_t)kValues && total != 0.0f) atomicAdd(&s_acc[k * kStride + held], total);
    }
    __syncthreads();
    // One global atomic per (splat, value) for the whole tile.
    for (uint32_t j = t; j < count; j += kThreads) {
      if (s_batch[j].mask == 0u) continue;
      float *dst = raw + (size_t)s_batch[j].index * kRawStride;
#pragma unroll
      for (int v = 0; v < kValues; ++v) {
        const float x = s_acc[j * kStride + v];
        if (x != 0.0f) {
          atomicAdd(dst + v, v >= 3 && v <= 5 ? 0.5f * x : x);
          s_acc[j * kStride + v] = 0.0f;
        }
      }
    }
  }
}

template <class M, bool SCORE, int T, int B>
__global__ void __launch_bounds__(TileShape<T>::kThreads, backward2_blocks<T>())
    k_backward2(const Splat *__restrict__ splats, const uint32_t *__restrict__ entryValues, const uint2 *__restrict__ ranges,
                const ViewSet *__restrict__ viewsPtr, float bgR, float bgG, float bgB, const float4 *__restrict__ image,
                const float4 *__restrict__ adjoint, const uint32_t *__restrict__ stops, float *__restrict__ raw,
                uint32_t splatLimit, uint32_t *error, const float *__restrict__ edge, uint32_t *work, const uint32_t *order) {
  chain_enter();
  const ViewSet &views = *viewsPtr;
  __shared__ Staged s_batch[B];
  __shared__ float s_acc[B * score_stride<SCORE>()];
  __shared__ uint32_t s_min[TileShape<T>::kWarps];
  __shared__ uint32_t s_cover[TileShape<T>::kWarps][B / 32];
  __shared__ uint32_t s_next;
  if (error != nullptr && (*error & kErrEntryOverflow) != 0u) return;
  for (int tile = next_tile(work, (uint32_t)views.totalTiles, true, &s_next, order); tile >= 0;
       tile = next_tile(work, (uint32_t)views.totalTiles, false, &s_next, order))
    backward2_tile<M, SCORE, T, B>(tile, splats, entryValues, ranges, views, bgR, bgG, bgB, image, adjoint, stops, raw, splatLimit,
                                   error, edge, s_batch, s_acc, s_min, s_cover);
}

// The float backward in two phases (new here; the reference sums each splat
// over a 32-lane group, train_backward.glsl:51-76). A warp walks its 8x8
// block's listed splats pixel-parallel exactly as k_backward2 does, but
// keeps, instead of the splat's twelve sums, two numbers per pixel (dPower and
// the blending weight wA) in shared memory, for a group of up to G splats
// that reach any of its pixels. Then the group's sums are made splat-parallel:
// lane i % G takes splat i, lane / G a share of the block's 64 pixels, and
// walks only the pixels the splat reached, adding the twelve sums in
// registers; the shares meet by shuffles, and one shared atomic per (splat,
// value) adds the group's totals. The per-(splat, block) reduction of twelve
// values over 32 lanes is gone; what remains per reached pixel is a dozen
// fused multiply-adds. Float sums in another order than k_backward2's.
// g0 = sum dAlpha e^power is taken as sum dPower / opacity (alpha = opacity
// e^power wherever dAlpha is not zero).
template <int T> __host__ __device__ constexpr int group_size() { return T > 16 ? 8 : 16; }

template <int T> struct PairStore {
  float2 v[group_size<T>()][64]; // per group splat, per pixel of the block: (dPower, wA)
};

template <int G, int T, int B>
__device__ __forceinline__ void backward3_sums(int count, uint32_t myK, uint32_t myLo, uint32_t myHi, const Staged *s_batch,
                                               const PairStore<T> &pairs, const float4 *pix, const float *pixAz, float perPixel,
                                               float *s_acc) {
  constexpr uint32_t P = 64u / (32u / G); // pixels of a lane's share
  const uint32_t lane = threadIdx.x & 31u, i = lane % G, h = lane / G;
  const uint32_t k = __shfl_sync(0xFFFFFFFFu, myK, i);
  const uint32_t lo = __shfl_sync(0xFFFFFFFFu, myLo, i), hi = __shfl_sync(0xFFFFFFFFu, myHi, i);
  float acc[12];
#pragma unroll
  for (int v = 0; v < 12; ++v) acc[v] = 0.0f;
  if ((int)i < count) {
    const Staged &s = s_batch[k];
    const float cx = s.cx, cy = s.cy, qx = s.qx, qy = s.qy, qz = s.qz, invOp = 1.0f / s.opacity;
    const uint32_t first = h * P;
    uint32_t mask;
    if constexpr (P == 32u) {
      mask = h == 0u ? lo : hi;
    } else {
      const uint32_t word = first < 32u ? lo : hi;
      mask = (word >> (first & 31u)) & ((1u << P) - 1u);
    }
    for (; mask != 0u; mask &= mask - 1u) {
      const uint32_t p = first + (uint32_t)(__ffs(mask) - 1);
      const float4 px = pix[p];
      const float2 pd = pairs.v[i][p];
      const float dx = px.x - cx, dy = px.y - cy;
      const float vx = fmaf(qy, dy, qx * dx), vy = fmaf(qz, dy, qy * dx);
      const float g1 = pd.x * vx, g2 = pd.x * vy;
      acc[0] = fmaf(pd.x, invOp, acc[0]);
      acc[1] += g1;
      acc[2] += g2;
      // Twice the conic sums; the flush halves them (exactly).
      acc[3] = fmaf(g1, vx, acc[3]);
      acc[4] = fmaf(g1, vy, acc[4]);
      acc[5] = fmaf(g2, vy, acc[5]);
      acc[6] = fmaf(pd.y, px.z, acc[6]);
      acc[7] = fmaf(pd.y, px.w, acc[7]);
      acc[8] = fmaf(pd.y, pixAz[p], acc[8]);
      acc[9] += pd.y;
      acc[10] += fabsf(g1);
      acc[11] += fabsf(g2);
    }
  }
#pragma unroll
  for (uint32_t o = G; o < 32u; o <<= 1)
#pragma unroll
    for (int v = 0; v < 12; ++v) acc[v] += __shfl_xor_sync(0xFFFFFFFFu, acc[v], o);
  if (h == 0u && (int)i < count) {
    acc[9] *= perPixel;
#pragma unroll
    for (int v = 0; v < 12; ++v)
      if (acc[v] != 0.0f) atomicAdd(&s_acc[k * kAccStride + v], acc[v]);
  }
}

template <class M, int T, int B>
__device__ __forceinline__ void backward3_tile(int tile, const Splat *__restrict__ splats, const uint32_t *__restrict__ entryValues,
                                               const uint2 *__restrict__ ranges, const ViewSet &views, float bgR, float bgG,
                                               float bgB, const float4 *__restrict__ image, const float4 *__restrict__ adjoint,
                                               const uint32_t *__restrict__ stops, float *__restrict__ raw, uint32_t splatLimit,
                                               uint32_t *error, Staged *s_batch, float *s_acc, uint32_t *s_min,
                                               uint32_t (*s_cover)[B / 32], PairStore<T> *s_pairs, float4 (*s_pix)[64],
                                               float (*s_az)[64]) {
  constexpr int kThreads = TileShape<T>::kThreads, W = TileShape<T>::kWarps, G = group_size<T>();
  const TileGeometry geo = tile_geometry(views, tile, T);
  const ViewParams &cam = views.v[geo.view];
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const PixelPair<T> pp = pixel_pair<T>(geo, cam, t);
  const uint2 range = ranges[tile];
  float fr[2], ax[2], ay[2], az[2], bh[2];
  uint32_t stop[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const size_t at = pp.inside[q] ? (size_t)cam.pixelBase + (size_t)pp.y[q] * cam.width + pp.x[q] : 0;
    fr[q] = pp.inside[q] ? image[at].w : 0.0f;
    const float4 a = pp.inside[q] ? adjoint[at] : make_float4(0.f, 0.f, 0.f, 0.f);
    ax[q] = a.x;
    ay[q] = a.y;
    az[q] = a.z;
    stop[q] = pp.inside[q] ? stops[at] : range.y;
    bh[q] = fmaf(a.z, bgB, fmaf(a.y, bgG, a.x * bgR));
    // The block's pixel table for the splat-parallel sums: pixel q * 32 + lane.
    s_pix[warp][q * 32 + lane] = make_float4(pp.px[q], pp.py[q], a.x, a.y);
    s_az[warp][q * 32 + lane] = a.z;
  }
  float2 front = make_float2(fr[0], fr[1]), behind = make_float2(bh[0], bh[1]);
  const float2 Ax = make_float2(ax[0], ax[1]), Ay = make_float2(ay[0], ay[1]), Az = make_float2(az[0], az[1]);
  const float px = pp.px[0];
  const float2 py = make_float2(pp.py[0], pp.py[1]);
  const float perPixel = cam.perPixel;
  const uint32_t warpMin = __reduce_min_sync(0xFFFFFFFFu, min(stop[0], stop[1]));
  if (lane == 0) s_min[warp] = warpMin;
  for (int i = t; i < B * kAccStride; i += kThreads) s_acc[i] = 0.0f;
  __syncthreads();
  uint32_t tileStop = s_min[0];
#pragma unroll
  for (int w = 1; w < W; ++w) tileStop = min(tileStop, s_min[w]);
  PairStore<T> &pairs = s_pairs[warp];

  for (uint32_t start = tileStop; start < range.y; start += B) {
    const uint32_t count = min((uint32_t)B, range.y - start);
    __syncthreads();
    stage_pairs<M, T, B>(splats, entryValues + start, count, splatLimit, geo, error, s_batch, s_cover, s_min, start);
    __syncthreads();
    int group = 0;
    uint32_t myK = 0u, myLo = 0u, myHi = 0u; // lane i < group: the group's i-th splat and the pixels it reached
    for (uint32_t word = 0; word <= ((count - 1u) >> 5); ++word)
    for (uint32_t bits = s_cover[warp][word]; bits != 0u; bits &= bits - 1u) {
      const uint32_t k = word * 32u + (uint32_t)(__ffs(bits) - 1);
      const Staged &s = s_batch[k];
      const auto mask = staged_mask<T>(s);
      const float dx = px - s.cx;
      const float2 dy = add2(py, f2(-s.cy));
      const float2 power = splat_power2(s, dx, dy);
      const float2 ep = make_float2(M::exp(fminf(power.x, 0.0f)), M::exp(fminf(power.y, 0.0f)));
      const float2 oe = mul2(f2(s.opacity), ep);
      const float2 alpha = make_float2(fminf(kAlphaMax, oe.x), fminf(kAlphaMax, oe.y));
      const uint32_t entry = start + k;
      const bool act0 = entry >= stop[0] && (mask & pp.bits[0]) == pp.bits[0] && !(power.x > 0.0f) && alpha.x >= kAlphaMin;
      const bool act1 = entry >= stop[1] && (mask & pp.bits[1]) == pp.bits[1] && !(power.y > 0.0f) && alpha.y >= kAlphaMin;
      const uint32_t lo = __ballot_sync(0xFFFFFFFFu, act0), hi = __ballot_sync(0xFFFFFFFFu, act1);
      if ((lo | hi) == 0u) continue;
      const float2 aAct = make_float2(act0 ? alpha.x : 0.0f, act1 ? alpha.y : 0.0f);
      const float2 oneMinus = rsub2(aAct, f2(1.0f));
      const float2 logRest = make_float2(M::log(oneMinus.x), M::log(oneMinus.y));
      const float2 nextFront = rsub2(logRest, front);
      const float2 Tf = make_float2(M::exp(nextFront.x), M::exp(nextFront.y));
      const float2 wA = mul2(Tf, aAct);
      const float2 ahead = rsub2(behind, fma2(Az, f2(s.b), fma2(Ay, f2(s.g), mul2(Ax, f2(s.r)))));
      // At the 0.99 clamp alpha no longer depends on the parameters.
      const float2 dT = mul2(Tf, ahead);
      const float2 dAlpha = make_float2(act0 && oe.x < kAlphaMax ? dT.x : 0.0f, act1 && oe.y < kAlphaMax ? dT.y : 0.0f);
      const float2 dPower = mul2(dAlpha, alpha);
      behind = fma2(aAct, ahead, behind);
      front = nextFront;
      pairs.v[group][lane] = make_float2(dPower.x, wA.x);
      pairs.v[group][32 + lane] = make_float2(dPower.y, wA.y);
      if (lane == (uint32_t)group) {
        myK = k;
        myLo = lo;
        myHi = hi;
      }
      if (++group == G) {
        __syncwarp();
        backward3_sums<G, T, B>(group, myK, myLo, myHi, s_batch, pairs, s_pix[warp], s_az[warp], perPixel, s_acc);
        __syncwarp();
        group = 0;
      }
    }
    if (group > 0) {
      __syncwarp();
      backward3_sums<G, T, B>(group, myK, myLo, myHi, s_batch, pairs, s_pix[warp], s_az[warp], perPixel, s_acc);
      __syncwarp();
    }
    __syncthreads();
    // One global atomic per (splat, value) for the whole tile.
    for (uint32_t j = t; j < count; j += kThreads) {
      if (s_batch[j].mask == 0u && s_batch[j].maskHi == 0u) continue;
      float *dst = raw + (size_t)s_batch[j].index * kRawStride;
#pragma unroll
      for (int v = 0; v < kGradValues; ++v) {
        const float x = s_acc[j * kAccStride + v];
        if (x != 0.0f) {
          atomicAdd(dst + v, v >= 3 && v <= 5 ? 0.5f * x : x);
          s_acc[j * kAccStride + v] = 0.0f;
        }
      }
    }
  }
}

template <class M, int T, int B>
__global__ void __launch_bounds__(TileShape<T>::kThreads, T > 16 ? 1 : 4)
    k_backward3(const Splat *__restrict__ splats, const uint32_t *__restrict__ entryValues, const uint2 *__restrict__ ranges,
                const ViewSet *__restrict__ viewsPtr, float bgR, float bgG, float bgB, const float4 *__restrict__ image,
                const float4 *__restrict__ adjoint, const uint32_t *__restrict__ stops, float *__restrict__ raw,
                uint32_t splatLimit, uint32_t *error, uint32_t *work, const uint32_t *order) {
  chain_enter();
  constexpr int W = TileShape<T>::kWarps;
  const ViewSet &views = *viewsPtr;
  // Dynamic shared memory: each warp's pair store, then its pixel tables.
  extern __shared__ __align__(16) unsigned char s_dynamic[];
  PairStore<T> *s_pairs = reinterpret_cast<PairStore<T> *>(s_dynamic);
  float4(*s_pix)[64] = reinterpret_cast<float4(*)[64]>(s_dynamic + W * sizeof(PairStore<T>));
  float(*s_az)[64] = reinterpret_cast<float(*)[64]>(s_dynamic + W * (sizeof(PairStore<T>) + 64 * sizeof(float4)));
  __shared__ Staged s_batch[B];
  __shared__ float s_acc[B * kAccStride];
  __shared__ uint32_t s_min[W];
  __shared__ uint32_t s_cover[W][B / 32];
  __shared__ uint32_t s_next;
  if (error != nullptr && (*error & kErrEntryOverflow) != 0u) return;
  for (int tile = next_tile(work, (uint32_t)views.totalTiles, true, &s_next, order); tile >= 0;
       tile = next_tile(work, (uint32_t)views.totalTiles, false, &s_next, order))
    backward3_tile<M, T, B>(tile, splats, entryValues, ranges, views, bgR, bgG, bgB, image, adjoint, stops, raw, splatLimit, error,
                            s_batch, s_acc, s_min, s_cover, s_pairs, s_pix, s_az);
}

} // namespace

// Blocks of a kernel that fit on the GPU at once (its occupancy times the
// SMs): the grid of a persistent launch. Asked once per kernel.
uint32_t resident_blocks(const void *kernel, int threads) {
  static std::mutex lock;
  static std::unordered_map<const void *, uint32_t> known;
  std::lock_guard<std::mutex> guard(lock);
  const auto hit = known.find(kernel);
  if (hit != known.end()) return hit->second;
  int device = 0, sms = 0, perSm = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, threads, 0);
  const uint32_t blocks = (uint32_t)std::max(1, sms * std::max(perSm, 1));
  known.emplace(kernel, blocks);
  return blocks;
}

namespace {

template <class M, int T, int B>
void launch_forward2(const Splat *splats, const uint32_t *entryValues, const uint2 *ranges, const ViewSet &views, const ViewSet *dViews,
                     const RasterConfig &cfg, float4 *image, uint32_t *stops, uint32_t splatLimit, uint32_t *error,
                     cudaStream_t stream) {
  constexpr int kThreads = TileShape<T>::kThreads;
  uint32_t grid = (uint32_t)views.totalTiles;
  if (cfg.workForward != nullptr) grid = std::min(grid, resident_blocks((const void *)k_forward2<M, T, B>, kThreads));
  launch_chained(k_forward2<M, T, B>, dim3(grid), dim3(kThreads), 0, stream, splats, entryValues, ranges, dViews, cfg.background[0],
                 cfg.background[1], cfg.background[2], image, stops, splatLimit, error, cfg.workForward, cfg.orderForward,
                 cfg.tileWork);
}

template <class M, bool SCORE, int T, int B>
void launch_backward2(const Splat *splats, const uint32_t *entryValues, const uint2 *ranges, const ViewSet &views,
                      const ViewSet *dViews, const RasterConfig &cfg, const float4 *image, const float4 *adjoint,
                      const uint32_t *stops, float *raw, uint32_t splatLimit, uint32_t *error, cudaStream_t stream,
                      const float *edge) {
  constexpr int kThreads = TileShape<T>::kThreads;
  uint32_t grid = (uint32_t)views.totalTiles;
  if (cfg.workBackward != nullptr) grid = std::min(grid, resident_blocks((const void *)k_backward2<M, SCORE, T, B>, kThreads));
  launch_chained(k_backward2<M, SCORE, T, B>, dim3(grid), dim3(kThreads), 0, stream, splats, entryValues, ranges, dViews,
                 cfg.background[0], cfg.background[1], cfg.background[2], image, adjoint, stops, raw, splatLimit, error, edge,
                 cfg.workBackward, cfg.orderBackward);
}

template <int T> constexpr size_t backward3_dynamic_bytes() {
  return (size_t)TileShape<T>::kWarps * (sizeof(PairStore<T>) + 64 * sizeof(float4) + 64 * sizeof(float));
}

template <class M, int T, int B>
void launch_backward3(const Splat *splats, const uint32_t *entryValues, const uint2 *ranges, const ViewSet &views,
                      const ViewSet *dViews, const RasterConfig &cfg, const float4 *image, const float4 *adjoint,
                      const uint32_t *stops, float *raw, uint32_t splatLimit, uint32_t *error, cudaStream_t stream) {
  constexpr int kThreads = TileShape<T>::kThreads;
  constexpr size_t kDynamic = backward3_dynamic_bytes<T>();
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_backward3<M, T, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDynamic);
    configured = true;
  }
  uint32_t grid = (uint32_t)views.totalTiles;
  if (cfg.workBackward != nullptr) {
    int perSm = 0, device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_backward3<M, T, B>, kThreads, kDynamic);
    grid = std::min(grid, (uint32_t)std::max(1, sms * std::max(perSm, 1)));
  }
  launch_chained(k_backward3<M, T, B>, dim3(grid), dim3(kThreads), kDynamic, stream, splats, entryValues, ranges, dViews,
                 cfg.background[0], cfg.background[1], cfg.background[2], image, adjoint, stops, raw, splatLimit, error,
                 cfg.workBackward, cfg.orderBackward);
}

// Calls f(tile edge, batch depth) with the two-pixel kernels' settings as
// compile-time constants.
template <class F> void dispatch_tile_batch(const RasterConfig &cfg, F &&f) {
  using I = std::integral_constant<int, 16>;
  if (cfg.tile == 32) {
    if (cfg.batch == 128) f(std::integral_constant<int, 32>{}, std::integral_constant<int, 128>{});
    else f(std::integral_constant<int, 32>{}, std::integral_constant<int, 256>{});
  } else {
    if (cfg.batch == 128) f(I{}, std::integral_constant<int, 128>{});
    else f(I{}, std::integral_constant<int, 256>{});
  }
}

} // namespace

void launch_forward(const Splat *splats, const uint32_t *entryValues, const uint2 *ranges, const ViewSet &views, const ViewSet *dViews,
                    const RasterConfig &cfg, float4 *image, uint32_t *stops, uint32_t splatLimit, uint32_t *error,
                    cudaStream_t stream, int listMode, BlendLists lists) {
  if (views.totalTiles == 0) return;
  const float r = cfg.background[0], g = cfg.background[1], b = cfg.background[2];
  if (listMode != 0) {
#define SB_FORWARD_LISTS(MATH, MODE)                                                                                         \
  launch_chained(k_forward<MATH, MODE>, dim3(views.totalTiles), dim3(kTilePixels), 0, stream, splats, entryValues, ranges, dViews, r, g, b, image, stops, \
                                                                     lists, splatLimit, error)
    if (cfg.exactMath) {
      if (listMode == 1) SB_FORWARD_LISTS(ExactMath, 1);
      else SB_FORWARD_LISTS(ExactMath, 2);
    } else {
      if (listMode == 1) SB_FORWARD_LISTS(FastMath, 1);
      else SB_FORWARD_LISTS(FastMath, 2);
    }
#undef SB_FORWARD_LISTS
    return;
  }
  if (cfg.forwardPixels == 2) {
    dispatch_tile_batch(cfg, [&](auto T, auto B) {
      if (cfg.exactMath)
        launch_forward2<ExactMath, decltype(T)::value, decltype(B)::value>(splats, entryValues, ranges, views, dViews, cfg, image,
                                                                           stops, splatLimit, error, stream);
      else
        launch_forward2<FastMath, decltype(T)::value, decltype(B)::value>(splats, entryValues, ranges, views, dViews, cfg, image,
                                                                          stops, splatLimit, error, stream);
    });
  } else {
    if (cfg.exactMath)
      launch_chained(k_forward<ExactMath, 0>, dim3(views.totalTiles), dim3(kTilePixels), 0, stream, splats, entryValues, ranges, dViews, r, g, b, image,
                                                                           stops, BlendLists{}, splatLimit, error);
    else
      launch_chained(k_forward<FastMath, 0>, dim3(views.totalTiles), dim3(kTilePixels), 0, stream, splats, entryValues, ranges, dViews, r, g, b, image,
                                                                          stops, BlendLists{}, splatLimit, error);
  }
}

void launch_backward(const Splat *splats, const uint32_t *entryValues, const uint2 *ranges, const ViewSet &views, const ViewSet *dViews,
                     const RasterConfig &cfg, const float4 *image, const float4 *adjoint, const uint32_t *stops,
                     bool fixedPoint, void *raw, uint32_t splatLimit, uint32_t *error, cudaStream_t stream, const float *edge) {
  if (views.totalTiles == 0) return;
  const float r = cfg.background[0], g = cfg.background[1], b = cfg.background[2];
  const uint32_t tiles = views.totalTiles;
  const bool score = edge != nullptr;
  // The fixed-point sums keep the reference's 32-lane groups: one pixel per thread.
  if (!fixedPoint && cfg.backwardPixels == 2 && cfg.twoPhase && !score) {
    float *rawF = static_cast<float *>(raw);
    dispatch_tile_batch(cfg, [&](auto T, auto B) {
      constexpr int kT = decltype(T)::value, kB = decltype(B)::value;
      if (cfg.exactMath)
        launch_backward3<ExactMath, kT, kB>(splats, entryValues, ranges, views, dViews, cfg, image, adjoint, stops, rawF, splatLimit,
                                            error, stream);
      else
        launch_backward3<FastMath, kT, kB>(splats, entryValues, ranges, views, dViews, cfg, image, adjoint, stops, rawF, splatLimit,
                                           error, stream);
    });
    return;
  }
  if (!fixedPoint && cfg.backwardPixels == 2) {
    float *rawF = static_cast<float *>(raw);
    dispatch_tile_batch(cfg, [&](auto T, auto B) {
      constexpr int kT = decltype(T)::value, kB = decltype(B)::value;
      if (cfg.exactMath) {
        if (score) launch_backward2<ExactMath, true, kT, kB>(splats, entryValues, ranges, views, dViews, cfg, image, adjoint, stops, rawF, splatLimit, error, stream, edge);
        else launch_backward2<ExactMath, false, kT, kB>(splats, entryValues, ranges, views, dViews, cfg, image, adjoint, stops, rawF, splatLimit, error, stream, edge);
      } else {
        if (score) launch_backward2<FastMath, true, kT, kB>(splats, entryValues, ranges, views, dViews, cfg, image, adjoint, stops, rawF, splatLimit, error, stream, edge);
        else launch_backward2<FastMath, false, kT, kB>(splats, entryValues, ranges, views, dViews, cfg, image, adjoint, stops, rawF, splatLimit, error, stream, edge);
      }
    });
    return;
  }
#define SB_BACKWARD(MATH, FIX, SCORE)                                                                                   \
  launch_chained(k_backward<MATH, FIX, SCORE>, dim3(tiles), dim3(kTilePixels), 0, stream, splats, entryValues, ranges, dViews, r, g, \
                 b, image, adjoint, stops, raw, splatLimit, error, edge)
#define SB_BACKWARD_FIX(MATH, FIX)           \
  {                                          \
    if (score) SB_BACKWARD(MATH, FIX, true);  \
    else SB_BACKWARD(MATH, FIX, false);       \
  }
  if (cfg.exactMath) {
    if (fixedPoint) SB_BACKWARD_FIX(ExactMath, true) else SB_BACKWARD_FIX(ExactMath, false)
  } else {
    if (fixedPoint) SB_BACKWARD_FIX(FastMath, true) else SB_BACKWARD_FIX(FastMath, false)
  }
#undef SB_BACKWARD_FIX
#undef SB_BACKWARD
}

void launch_tile_order(const uint2 *ranges, const uint32_t *tileWork, uint32_t tiles, uint32_t *order, cudaStream_t stream) {
  if (tiles == 0) return;
  launch_chained(k_tile_order, dim3(1), dim3(kOrderThreads), 0, stream, ranges, tileWork, tiles, order);
}

void launch_backward_lists(const Splat *splats, const uint32_t *entryValues, const uint2 *ranges, const ViewSet &views,
                           const ViewSet *dViews, const RasterConfig &cfg, const float4 *image, const float4 *adjoint,
                           const uint32_t *stops, BlendLists lists, float *raw, uint32_t splatLimit, uint32_t *error,
                           cudaStream_t stream) {
  if (views.totalTiles == 0) return;
  const float r = cfg.background[0], g = cfg.background[1], b = cfg.background[2];
  if (cfg.exactMath)
    launch_chained(k_backward_lists<ExactMath>, dim3(views.totalTiles), dim3(kTilePixels), 0, stream, splats, entryValues, ranges, dViews, r, g, b, image,
                                                                             adjoint, stops, lists, raw, splatLimit, error);
  else
    launch_chained(k_backward_lists<FastMath>, dim3(views.totalTiles), dim3(kTilePixels), 0, stream, splats, entryValues, ranges, dViews, r, g, b, image,
                                                                            adjoint, stops, lists, raw, splatLimit, error);
}

} // namespace sb
