// Tile binning: coverage count with a fused single-pass exclusive scan, entry
// emission, and tile ranges. Restates shaders/train_bin_count.comp:18-38,
// shaders/train_bin_emit.comp:18-38, shaders/train_tile_ranges.comp:11-23 and
// the tile tests of shaders/train_types.glsl:34-77 (splat_tiles,
// splat_reaches_tile). The reach 2 log(255 opacity) comes from the preprocess
// pass, so the test here is exact IEEE arithmetic only.
#include <algorithm>

#include "kernels.cuh"

namespace sb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;
constexpr unsigned long long kScanAggregate = 1ull << 32;
constexpr unsigned long long kScanInclusive = 2ull << 32;
constexpr int kScanSpinLimit = 1 << 20;

struct TileRect {
  uint32_t x0, y0, x1, y1; // inclusive
};

// Covered tiles of a splat, inclusive (splat_tiles), for tiles of T x T
// pixels (the reference's 16, or 32; a power of two, so the divisions are
// exact scalings and T = 16 gives the reference's expressions' bits).
__device__ __forceinline__ TileRect splat_tiles(const float4 ce, int gridW, int gridH, float T) {
  const float lastX = (float)(gridW - 1), lastY = (float)(gridH - 1);
  const float lx = fminf(fmaxf(floorf((ce.x - ce.z - 1.0f) / T), 0.0f), lastX);
  const float ly = fminf(fmaxf(floorf((ce.y - ce.w - 1.0f) / T), 0.0f), lastY);
  const float hx = fminf(fmaxf(floorf((ce.x + ce.z + 1.0f) / T), 0.0f), lastX);
  const float hy = fminf(fmaxf(floorf((ce.y + ce.w + 1.0f) / T), 0.0f), lastY);
  return {(uint32_t)lx, (uint32_t)ly, (uint32_t)hx, (uint32_t)hy};
}

// Whether the splat reaches any pixel centre of tile (tx, ty)
// (splat_reaches_tile): the closest point of each tile edge to the centre is
// found by clamping the ellipse's tangent point to the edge. The tangent
// points on the two vertical edges depend on the column only, those on the
// two horizontal edges on the row only, so they are computed per column and
// per row (col_tangents, row_tangents) and the test combines them: the same
// operations in the same order as evaluating everything per tile.
struct ColTangents {
  float lowX, highX, yLow, yHigh; // edge offsets from the centre and their unclamped tangent y
};
struct RowTangents {
  float lowY, highY, uLow, uHigh; // edge offsets from the centre and their unclamped tangent x
};

// The conic's diagonal reciprocals, correctly rounded: the tangent points are
// products by them (the reference's GLSL division is not correctly rounded
// either), one reciprocal per splat instead of four divisions per tile.
struct TangentScales {
  float invX, invZ;
};
__device__ __forceinline__ TangentScales tangent_scales(const float4 q) { return {__frcp_rn(q.x), __frcp_rn(q.z)}; }

__device__ __forceinline__ ColTangents col_tangents(const float4 q, const TangentScales k, const float4 ce, uint32_t tx, float T) {
  ColTangents c;
  c.lowX = ((float)tx * T + 0.5f) - ce.x;
  c.highX = c.lowX + (T - 1.0f);
  c.yLow = (-q.y * c.lowX) * k.invZ;
  c.yHigh = (-q.y * c.highX) * k.invZ;
  return c;
}

__device__ __forceinline__ RowTangents row_tangents(const float4 q, const TangentScales k, const float4 ce, uint32_t ty, float T) {
  RowTangents r;
  r.lowY = ((float)ty * T + 0.5f) - ce.y;
  r.highY = r.lowY + (T - 1.0f);
  r.uLow = (-q.y * r.lowY) * k.invX;
  r.uHigh = (-q.y * r.highY) * k.invX;
  return r;
}

__device__ __forceinline__ bool reaches_tile(const float4 q, float reach, const ColTangents &col, const RowTangents &row) {
  const float lowX = col.lowX, highX = col.highX, lowY = row.lowY, highY = row.highY;
  if (lowX <= 0.0f && lowY <= 0.0f && highX >= 0.0f && highY >= 0.0f) return true;
  float least = 1e30f;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const float x = side == 0 ? lowX : highX;
    const float y = fminf(fmaxf(side == 0 ? col.yLow : col.yHigh, lowY), highY);
    least = fminf(least, q.x * x * x + 2.0f * q.y * x * y + q.z * y * y);
    const float v = side == 0 ? lowY : highY;
    const float u = fminf(fmaxf(side == 0 ? row.uLow : row.uHigh, lowX), highX);
    least = fminf(least, q.x * u * u + 2.0f * q.y * u * v + q.z * v * v);
  }
  return least <= reach * 1.001f + 1e-3f;
}

// Splats whose tile rectangle holds more than this many tiles are tested by a
// whole warp, one tile per lane, so that no thread walks a large splat's
// rectangle alone while its block (and, through the scan, every later block)
// waits for it.
constexpr uint32_t kWarpTiles = 16;
// Columns and rows of the per-warp tangent tables for those rectangles; a
// larger rectangle computes its tangents tile by tile.
constexpr uint32_t kTableMax = 64;

__device__ __forceinline__ uint32_t rect_area(const TileRect &t) { return (t.x1 - t.x0 + 1u) * (t.y1 - t.y0 + 1u); }

// A large rectangle's tangent tables, filled by the whole warp. False (and
// nothing filled) when the rectangle is wider or taller than the tables.
__device__ __forceinline__ bool fill_tables(const float4 q, const float4 ce, const TileRect &t, uint32_t lane, ColTangents *cols,
                                            RowTangents *rows, float T) {
  const uint32_t width = t.x1 - t.x0 + 1u, height = t.y1 - t.y0 + 1u;
  if (width > kTableMax || height > kTableMax) return false;
  const TangentScales k = tangent_scales(q);
  for (uint32_t c = lane; c < width; c += 32u) cols[c] = col_tangents(q, k, ce, t.x0 + c, T);
  for (uint32_t r = lane; r < height; r += 32u) rows[r] = row_tangents(q, k, ce, t.y0 + r, T);
  __syncwarp();
  return true;
}

// The tiles base .. base + 31 of the rectangle in row-major order: lane l
// tests tile base + l. Returns the lanes whose tile the splat reaches. The
// row is found with a float reciprocal: (i + 1/2) / width lies at least
// 1/(2 width) from an integer, far more than the rounding error.
__device__ __forceinline__ uint32_t warp_reach(const float4 q, const float4 ce, float reach, const TileRect &t, uint32_t width,
                                               float invWidth, uint32_t area, uint32_t base, uint32_t lane,
                                               const ColTangents *cols, const RowTangents *rows, uint32_t &x, uint32_t &y,
                                               float T) {
  const uint32_t li = base + lane;
  bool hit = false;
  if (li < area) {
    const uint32_t r = (uint32_t)(((float)li + 0.5f) * invWidth);
    const uint32_t c = li - r * width;
    x = t.x0 + c;
    y = t.y0 + r;
    const TangentScales k = tangent_scales(q);
    hit = cols != nullptr ? reaches_tile(q, reach, cols[c], rows[r])
                          : reaches_tile(q, reach, col_tangents(q, k, ce, x, T), row_tangents(q, k, ce, y, T));
  }
  return __ballot_sync(0xFFFFFFFFu, hit);
}

__device__ __forceinline__ unsigned long long load_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void store_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ int item_view(uint32_t splatIndex, uint32_t n, int views) {
  return views == 1 ? 0 : (int)(splatIndex / n);
}

// Coverage count, one thread per item, no block-wide waits: counts[r] (in
// the offsets array, scanned in place afterwards) and masks[r].
constexpr int kCountThreads = 256;

__global__ void __launch_bounds__(kCountThreads)
    k_bin_count(const Splat *__restrict__ splats, const float *__restrict__ reach, const uint32_t *__restrict__ itemKeys,
                const uint32_t *__restrict__ itemSplat, uint32_t items, uint32_t n, const ViewSet *__restrict__ viewsPtr,
                uint32_t *__restrict__ counts, uint32_t *__restrict__ masks, uint32_t *counters) {
  chain_enter();
  const ViewSet &views = *viewsPtr;
  const float T = (float)views.tileSize;
  __shared__ ColTangents s_cols[kCountThreads / 32][kTableMax];
  __shared__ RowTangents s_rows[kCountThreads / 32][kTableMax];
  __shared__ uint32_t s_mask[kCountThreads / 32][32];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  // A grid smaller than the items (the count beside the depth sort) walks
  // them in chunks of a block's width, leaving SM slots to the sort's passes.
  for (uint32_t chunk = blockIdx.x; chunk * kCountThreads < items; chunk += gridDim.x) {
  const uint32_t r = chunk * kCountThreads + threadIdx.x;
  // Whole warps stay to the end: the loops below are warp-wide. Without item
  // keys (the count beside the depth sort, which permutes them), a culled
  // splat is the one whose reach the projection left at minus infinity.
  const uint32_t item = r < items ? (itemSplat != nullptr ? itemSplat[r] : r) : 0u;
  const bool valid = r < items && (itemKeys != nullptr ? itemKeys[r] != kInvisible : reach[item] != -INFINITY);
  const uint32_t s = valid ? item : 0u;
  float4 ce = make_float4(0.f, 0.f, 0.f, 0.f), cq = ce;
  float rc = 0.0f;
  TileRect rect{0u, 0u, 0u, 0u};
  uint32_t area = 0;
  if (valid) {
    ce = splats[s].centerExtent;
    cq = splats[s].conicOpacity;
    rc = reach[s];
    const ViewParams &cam = views.v[item_view(s, n, views.count)];
    rect = splat_tiles(ce, cam.gridW, cam.gridH, T);
    area = rect_area(rect);
  }
  const uint32_t visibleLanes = __ballot_sync(0xFFFFFFFFu, valid);
  if (lane == 0 && visibleLanes != 0u) atomicAdd(&counters[0], (uint32_t)__popc(visibleLanes));
  const bool big = area > kWarpTiles;
  uint32_t count = 0, mask = 0;

  // Small rectangles: the warp's (splat, tile) pairs laid out flat, 32 tests
  // per trip with every lane busy; each splat's mask (bit = row-major index in
  // its rectangle) is assembled in shared memory.
  {
    const uint32_t own = big ? 0u : area;
    uint32_t incl = own;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= (uint32_t)o) incl += x;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31), excl = incl - own;
    const uint32_t width = rect.x1 - rect.x0 + 1u;
    const float invWidth = 1.0f / (float)width;
    const TangentScales ks = valid ? tangent_scales(cq) : TangentScales{0.f, 0.f};
    s_mask[warp][lane] = 0u;
    __syncwarp();
    for (uint32_t base = 0; base < total; base += 32u) {
      const uint32_t f = base + lane;
      uint32_t owner = 0;
#pragma unroll
      for (uint32_t step = 16; step > 0; step >>= 1)
        if (__shfl_sync(0xFFFFFFFFu, incl, owner + step - 1u) <= f) owner += step;
      const uint32_t li = f - __shfl_sync(0xFFFFFFFFu, excl, owner);
      const float4 oce = make_float4(__shfl_sync(0xFFFFFFFFu, ce.x, owner), __shfl_sync(0xFFFFFFFFu, ce.y, owner), 0.f, 0.f);
      const float4 oq = make_float4(__shfl_sync(0xFFFFFFFFu, cq.x, owner), __shfl_sync(0xFFFFFFFFu, cq.y, owner),
                                    __shfl_sync(0xFFFFFFFFu, cq.z, owner), 0.f);
      const float orc = __shfl_sync(0xFFFFFFFFu, rc, owner);
      const uint32_t ox0 = __shfl_sync(0xFFFFFFFFu, rect.x0, owner), oy0 = __shfl_sync(0xFFFFFFFFu, rect.y0, owner);
      const uint32_t ow = __shfl_sync(0xFFFFFFFFu, width, owner);
      const float oinv = __shfl_sync(0xFFFFFFFFu, invWidth, owner);
      const TangentScales ok = {__shfl_sync(0xFFFFFFFFu, ks.invX, owner), __shfl_sync(0xFFFFFFFFu, ks.invZ, owner)};
      if (f < total) {
        const uint32_t row = (uint32_t)(((float)li + 0.5f) * oinv), col = li - row * ow;
        if (reaches_tile(oq, orc, col_tangents(oq, ok, oce, ox0 + col, T), row_tangents(oq, ok, oce, oy0 + row, T)))
          atomicOr(&s_mask[warp][owner], 1u << li);
      }
    }
    __syncwarp();
    if (!big) {
      mask = s_mask[warp][lane];
      count = (uint32_t)__popc(mask);
    }
  }
  // Large rectangles: the whole warp, one after another.
  for (uint32_t bigLanes = __ballot_sync(0xFFFFFFFFu, big); bigLanes != 0u; bigLanes &= bigLanes - 1u) {
    const uint32_t src = (uint32_t)__ffs(bigLanes) - 1u;
    const uint32_t bs = __shfl_sync(0xFFFFFFFFu, s, src);
    const ViewParams &cam = views.v[item_view(bs, n, views.count)];
    const Splat sp = splats[bs];
    const float rcb = reach[bs];
    const TileRect bt = splat_tiles(sp.centerExtent, cam.gridW, cam.gridH, T);
    const uint32_t width = bt.x1 - bt.x0 + 1u, barea = rect_area(bt);
    const bool tables = fill_tables(sp.conicOpacity, sp.centerExtent, bt, lane, s_cols[warp], s_rows[warp], T);
    const float invWidth = 1.0f / (float)width;
    uint32_t total = 0, hits = 0, x = 0, y = 0;
    for (uint32_t base = 0; base < barea; base += 32u) {
      hits = warp_reach(sp.conicOpacity, sp.centerExtent, rcb, bt, width, invWidth, barea, base, lane,
                        tables ? s_cols[warp] : nullptr, s_rows[warp], x, y, T);
      total += (uint32_t)__popc(hits);
    }
    __syncwarp(); // the tables are read before the next rectangle fills them
    if (lane == src) {
      count = total;
      mask = barea <= 32u ? hits : 0u; // the emission replays masks of one word only
    }
  }
  if (r < items) {
    counts[r] = count;
    masks[r] = mask;
  }
  __syncwarp(); // the warp's tables and masks are reused by its next chunk
  }
}

// Exclusive scan of the coverage counts into offsets:
// a block of kScanThreads threads takes kScanTile consecutive items, claimed
// in launch order through a ticket, and finds what precedes it by a
// decoupled look-back. counters[1] gets the total, counters[2] the entries
// that fit the capacity; a total above it sets kErrEntryOverflow.
// With gather, item r's count is counts[gather[r]] (counts indexed by splat,
// the items in depth order); otherwise counts[r], and counts may be offsets.
__global__ void __launch_bounds__(kScanThreads)
    k_offsets_scan(uint32_t items, const uint32_t *counts, const uint32_t *__restrict__ gather, uint32_t *offsets,
                   uint32_t *counters, uint32_t capacity, unsigned long long *status, uint32_t *ticket, uint32_t *error) {
  chain_enter();
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ unsigned long long s_exclusive;
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  if (t == 0) s_tile = atomicAdd(ticket, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t numTiles = div_up(items, kScanTile);
  if (tile >= numTiles) return;
  uint32_t counts_[kScanItems];
  uint32_t threadSum = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    const uint32_t r = tile * kScanTile + t * kScanItems + j;
    counts_[j] = r < items ? counts[gather != nullptr ? gather[r] : r] : 0u;
    threadSum += counts_[j];
  }
  // Block scan of the thread sums.
  uint32_t inclusive = threadSum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t x = __shfl_up_sync(0xFFFFFFFFu, inclusive, o);
    if (lane >= (uint32_t)o) inclusive += x;
  }
  if (lane == 31) s_warp[warp] = inclusive;
  __syncthreads();
  uint32_t before = 0, tileSum = 0;
#pragma unroll
  for (int w = 0; w < kScanThreads / 32; ++w) {
    before += (uint32_t)w < warp ? s_warp[w] : 0u;
    tileSum += s_warp[w];
  }
  // Decoupled look-back over the tiles before this one, by warp 0: each poll
  // reads the 32 nearest predecessors at once (lane j the tile j + 1 back),
  // takes the nearest inclusive prefix, and adds the aggregates in between.
  if (warp == 0) {
    unsigned long long exclusive = 0;
    if (tile == 0) {
      if (lane == 0) store_u64(&status[0], kScanInclusive | tileSum);
    } else {
      if (lane == 0) store_u64(&status[tile], kScanAggregate | tileSum);
      int64_t window = (int64_t)tile - 1;
      int spins = 0;
      for (;;) {
        const int64_t pred = window - (int64_t)lane;
        // Before the first tile there is nothing: an inclusive prefix of zero.
        const unsigned long long v = pred >= 0 ? load_u64(&status[pred]) : kScanInclusive;
        const unsigned long long flag = v & 0xFFFFFFFF00000000ull;
        const uint32_t inclusiveLanes = __ballot_sync(0xFFFFFFFFu, flag == kScanInclusive);
        const uint32_t pendingLanes = __ballot_sync(0xFFFFFFFFu, flag == 0);
        const int nearest = inclusiveLanes != 0u ? __ffs(inclusiveLanes) - 1 : 32;
        const uint32_t needed = nearest >= 31 ? 0xFFFFFFFFu : ((2u << nearest) - 1u);
        if ((pendingLanes & needed) != 0u) {
          if (++spins > kScanSpinLimit) {
            if (lane == 0) atomicOr(error, kErrLookbackTimeout);
            break;
          }
          continue;
        }
        const unsigned long long mine = (int)lane <= nearest ? (v & 0xFFFFFFFFull) : 0ull;
        unsigned long long sum = mine;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
        exclusive += sum;
        if (nearest < 32) break;
        window -= 32;
      }
      if (lane == 0) store_u64(&status[tile], kScanInclusive | ((exclusive + tileSum) & 0xFFFFFFFFull));
    }
    if (lane == 0) s_exclusive = exclusive;
    if (lane == 0 && tile == numTiles - 1) {
      const unsigned long long total = exclusive + tileSum;
      const uint32_t clipped = total > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)total;
      counters[1] = clipped;
      counters[2] = clipped < capacity ? clipped : capacity;
      if (clipped > capacity) atomicOr(error, kErrEntryOverflow);
    }
  }
  __syncthreads();
  uint32_t running = (uint32_t)s_exclusive + before + inclusive - threadSum;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    const uint32_t r = tile * kScanTile + t * kScanItems + j;
    if (r < items) offsets[r] = running;
    running += counts_[j];
  }
}

// Emission. Rectangles of up to 32 tiles replay the counting pass's masks
// with the warp's entries laid out flat: lane l writes entries l, l + 32, ...
// of the warp's run, so consecutive lanes write consecutive slots. Larger
// rectangles are tested again by the whole warp.
__global__ void __launch_bounds__(256)
    k_bin_emit(const Splat *__restrict__ splats, const float *__restrict__ reach, const uint32_t *__restrict__ itemKeys,
               const uint32_t *__restrict__ itemSplat, uint32_t items, uint32_t n, const ViewSet *__restrict__ viewsPtr,
               const uint32_t *__restrict__ offsets, const uint32_t *__restrict__ masks, bool masksBySplat, uint32_t capacity,
               uint32_t *__restrict__ tileKeys32, unsigned long long *__restrict__ tileKeys64, uint32_t *__restrict__ entryValues,
               uint32_t *error) {
  chain_enter();
  const ViewSet &views = *viewsPtr;
  const float T = (float)views.tileSize;
  __shared__ ColTangents s_cols[8][kTableMax];
  __shared__ RowTangents s_rows[8][kTableMax];
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x, lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  // Whole warps stay to the end: every loop below is warp-wide.
  const bool valid = r < items && itemKeys[r] != kInvisible;
  const uint32_t depthKey = valid ? itemKeys[r] : 0u;
  const uint32_t s = valid ? (itemSplat != nullptr ? itemSplat[r] : r) : 0u;
  const int view = valid ? item_view(s, n, views.count) : 0;
  TileRect t{0u, 0u, 0u, 0u};
  if (valid) t = splat_tiles(splats[s].centerExtent, views.v[view].gridW, views.v[view].gridH, T);
  const uint32_t width = t.x1 - t.x0 + 1u, area = valid ? rect_area(t) : 0u;
  const bool big = area > 32u;
  const uint32_t mask = valid && !big ? masks[masksBySplat ? s : r] : 0u;
  const uint32_t first = valid ? offsets[r] : 0u;
  bool overflow = false;
  auto put = [&](uint32_t slot, int v, uint32_t x, uint32_t y, uint32_t key, uint32_t splat) {
    if (slot < capacity) {
      const ViewParams &cam = views.v[v];
      const uint32_t tileId = y * (uint32_t)cam.gridW + x;
      if (tileKeys64 != nullptr) {
        tileKeys64[slot] = ((unsigned long long)((uint32_t)cam.tileBase + tileId) << 32) | key;
      } else {
        tileKeys32[slot] = tileId;
      }
      entryValues[slot] = splat;
    } else {
      overflow = true;
    }
  };

  // The small rectangles' entries, flat: an inclusive scan of their counts
  // over the warp, then entry j belongs to the first lane whose prefix passes j.
  const uint32_t count = (uint32_t)__popc(mask);
  uint32_t inclusive = count;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, inclusive, o);
    if (lane >= (uint32_t)o) inclusive += v;
  }
  const uint32_t total = __shfl_sync(0xFFFFFFFFu, inclusive, 31);
  const uint32_t exclusive = inclusive - count;
  for (uint32_t base = 0; base < total; base += 32u) {
    const uint32_t j = base + lane;
    uint32_t owner = 0;
#pragma unroll
    for (uint32_t step = 16; step > 0; step >>= 1) {
      const uint32_t v = __shfl_sync(0xFFFFFFFFu, inclusive, owner + step - 1u);
      if (v <= j) owner += step;
    }
    const uint32_t oExclusive = __shfl_sync(0xFFFFFFFFu, exclusive, owner);
    const uint32_t oMask = __shfl_sync(0xFFFFFFFFu, mask, owner);
    const uint32_t oFirst = __shfl_sync(0xFFFFFFFFu, first, owner);
    const uint32_t oX0 = __shfl_sync(0xFFFFFFFFu, t.x0, owner), oY0 = __shfl_sync(0xFFFFFFFFu, t.y0, owner);
    const uint32_t oWidth = __shfl_sync(0xFFFFFFFFu, width, owner);
    const uint32_t oSplat = __shfl_sync(0xFFFFFFFFu, s, owner), oKey = __shfl_sync(0xFFFFFFFFu, depthKey, owner);
    const int oView = __shfl_sync(0xFFFFFFFFu, view, owner);
    if (j < total) {
      // The rank-th set bit of the owner's mask: the largest p with rank set bits below it.
      const uint32_t rank = j - oExclusive;
      uint32_t bit = 0;
#pragma unroll
      for (uint32_t step = 16; step > 0; step >>= 1) {
        const uint32_t p = bit + step;
        if ((uint32_t)__popc(oMask & ((1u << p) - 1u)) <= rank) bit = p;
      }
      const uint32_t row = bit / oWidth;
      put(oFirst + rank, oView, oX0 + (bit - row * oWidth), oY0 + row, oKey, oSplat);
    }
  }

  // Rectangles of more than 32 tiles are tested again, by the whole warp;
  // row-major order kept by counting the lower lanes' hits.
  for (uint32_t bigLanes = __ballot_sync(0xFFFFFFFFu, big); bigLanes != 0u; bigLanes &= bigLanes - 1u) {
    const uint32_t src = (uint32_t)__ffs(bigLanes) - 1u;
    const uint32_t bs = __shfl_sync(0xFFFFFFFFu, s, src);
    const uint32_t key = __shfl_sync(0xFFFFFFFFu, depthKey, src);
    const uint32_t bFirst = __shfl_sync(0xFFFFFFFFu, first, src);
    const int bView = __shfl_sync(0xFFFFFFFFu, view, src);
    const ViewParams &cam = views.v[bView];
    const Splat sp = splats[bs];
    const float rc = reach[bs];
    const TileRect bt = splat_tiles(sp.centerExtent, cam.gridW, cam.gridH, T);
    const uint32_t bWidth = bt.x1 - bt.x0 + 1u, bArea = rect_area(bt);
    const bool tables = fill_tables(sp.conicOpacity, sp.centerExtent, bt, lane, s_cols[warp], s_rows[warp], T);
    const float invWidth = 1.0f / (float)bWidth;
    uint32_t slot = bFirst;
    for (uint32_t base = 0; base < bArea; base += 32u) {
      uint32_t x = 0, y = 0;
      const uint32_t hits = warp_reach(sp.conicOpacity, sp.centerExtent, rc, bt, bWidth, invWidth, bArea, base, lane,
                                       tables ? s_cols[warp] : nullptr, s_rows[warp], x, y, T);
      if ((hits >> lane) & 1u) put(slot + (uint32_t)__popc(hits & ((1u << lane) - 1u)), bView, x, y, key, bs);
      slot += (uint32_t)__popc(hits);
    }
    __syncwarp(); // the tables are read before the next rectangle fills them
  }
  if (overflow) atomicOr(error, kErrEntryOverflow);
}

// Tile ranges over the sorted keys: a grid of a few blocks per SM walks the
// entries (the count lives on the device, so a grid sized by the capacity
// would be mostly blocks with nothing to do), each thread four consecutive
// entries and their right neighbour.
constexpr uint32_t kRangesPerThread = 4;

__global__ void __launch_bounds__(256) k_tile_ranges(const uint32_t *__restrict__ keys32, const unsigned long long *__restrict__ keys64,
                                                     const uint32_t *deviceCount, uint32_t tileLimit, uint2 *__restrict__ ranges,
                                                     uint32_t *error) {
  chain_enter();
  const uint32_t count = *deviceCount;
  auto tile_of = [&](uint32_t i) { return keys64 != nullptr ? (uint32_t)(keys64[i] >> 32) : keys32[i]; };
  const uint32_t stride = gridDim.x * blockDim.x * kRangesPerThread;
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) * kRangesPerThread; base < count; base += stride) {
    uint32_t tiles[kRangesPerThread + 1];
#pragma unroll
    for (uint32_t j = 0; j <= kRangesPerThread; ++j) tiles[j] = base + j < count ? tile_of(base + j) : 0xFFFFFFFFu;
    const uint32_t before = base > 0 ? tile_of(base - 1) : 0xFFFFFFFFu;
#pragma unroll
    for (uint32_t j = 0; j < kRangesPerThread; ++j) {
      const uint32_t k = base + j;
      if (k >= count) break;
      const uint32_t tile = tiles[j];
      if (tile >= tileLimit) {
        atomicOr(error, kErrBadIndex);
        continue;
      }
      const uint32_t prev = j == 0 ? before : tiles[j - 1];
      if (k == 0 || prev != tile) ranges[tile].x = k;
      if (k + 1 == count || tiles[j + 1] != tile) ranges[tile].y = k + 1;
    }
  }
}

} // namespace

size_t bin_scan_scratch_bytes(uint32_t items) {
  return (size_t)(div_up(items, kScanTile) + 1) * sizeof(unsigned long long) + 256;
}

void launch_bin_count(const Splat *splats, const float *reach, const uint32_t *itemKeys, const uint32_t *itemSplat, uint32_t items,
                      uint32_t n, const ViewSet &views, const ViewSet *dViews, uint32_t *counts, uint32_t *masks, uint32_t *counters,
                      cudaStream_t stream, uint32_t blocksPerSm) {
  if (items == 0) return;
  uint32_t grid = div_up(items, kCountThreads);
  if (blocksPerSm > 0) {
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    grid = std::min(grid, (uint32_t)std::max(sms, 1) * blocksPerSm);
  }
  launch_chained(k_bin_count, dim3(grid), dim3(kCountThreads), 0, stream, splats, reach, itemKeys, itemSplat, items, n, dViews,
                 counts, masks, counters);
}

void launch_offsets_scan(uint32_t items, const uint32_t *counts, const uint32_t *gather, uint32_t *offsets, uint32_t *counters,
                         uint32_t capacity, void *scratch, uint32_t *error, cudaStream_t stream, bool clearScratch) {
  if (items == 0) return;
  const uint32_t tiles = div_up(items, kScanTile);
  unsigned long long *status = static_cast<unsigned long long *>(scratch);
  uint32_t *ticket = reinterpret_cast<uint32_t *>(status + tiles);
  if (clearScratch) cudaMemsetAsync(scratch, 0, bin_scan_scratch_bytes(items), stream);
  launch_chained(k_offsets_scan, dim3(tiles), dim3(kScanThreads), 0, stream, items, counts, gather, offsets, counters, capacity, status,
                 ticket, error);
}

void launch_bin_count_scan(const Splat *splats, const float *reach, const uint32_t *itemKeys, const uint32_t *itemSplat,
                           uint32_t items, uint32_t n, const ViewSet &views, const ViewSet *dViews, uint32_t *offsets, uint32_t *masks,
                           uint32_t *counters, uint32_t capacity, void *scratch, uint32_t *error, cudaStream_t stream) {
  if (items == 0) return;
  launch_bin_count(splats, reach, itemKeys, itemSplat, items, n, views, dViews, offsets, masks, counters, stream);
  launch_offsets_scan(items, offsets, nullptr, offsets, counters, capacity, scratch, error, stream);
}

void launch_bin_emit(const Splat *splats, const float *reach, const uint32_t *itemKeys, const uint32_t *itemSplat,
                     uint32_t items, uint32_t n, const ViewSet &views, const ViewSet *dViews, const uint32_t *offsets,
                     const uint32_t *masks, bool masksBySplat, uint32_t capacity, uint32_t *tileKeys32, unsigned long long *tileKeys64,
                     uint32_t *entryValues, uint32_t *error, cudaStream_t stream) {
  if (items == 0) return;
  launch_chained(k_bin_emit, dim3(div_up(items, 256)), dim3(256), 0, stream, splats, reach, itemKeys, itemSplat, items, n, dViews, offsets, masks,
                 masksBySplat, capacity, tileKeys32, tileKeys64, entryValues, error);
}

void launch_tile_ranges(const uint32_t *tileKeys32, const unsigned long long *tileKeys64, const uint32_t *deviceCount,
                        uint32_t capacity, uint32_t tileLimit, uint2 *ranges, uint32_t *error, cudaStream_t stream) {
  if (capacity == 0) return;
  const uint32_t blocks = std::min<uint32_t>(div_up(div_up(capacity, kRangesPerThread), 256), 148u * 8u);
  launch_chained(k_tile_ranges, dim3(blocks), dim3(256), 0, stream, tileKeys32, tileKeys64, deviceCount, tileLimit, ranges, error);
}

void launch_exclusive_scan(uint32_t items, uint32_t *values, uint32_t *counters, void *scratch, uint32_t *error,
                           cudaStream_t stream) {
  if (items == 0) return;
  const uint32_t tiles = div_up(items, kScanTile);
  unsigned long long *status = static_cast<unsigned long long *>(scratch);
  uint32_t *ticket = reinterpret_cast<uint32_t *>(status + tiles);
  cudaMemsetAsync(scratch, 0, bin_scan_scratch_bytes(items), stream);
  launch_chained(k_offsets_scan, dim3(tiles), dim3(kScanThreads), 0, stream, items, values, nullptr, values, counters, 0xFFFFFFFFu, status,
                 ticket, error);
}

} // namespace sb
