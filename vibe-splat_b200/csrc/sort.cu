// Onesweep radix sort: see sort.cuh.
#include "sort.cuh"

#include <algorithm>
#include <atomic>

#include "bulk.cuh"
#include "common.cuh"

namespace sb {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;                        // keys per thread
constexpr int kSortTileKeys = kSortThreads * kSortItems; // 4096 keys per tile
constexpr int kMaxPasses = 11;                        // 64 bits at 6-bit digits
constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagInclusive = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1u;
constexpr int kLookbackSpinLimit = 1 << 20;
// The limit the passes are launched with: kLookbackSpinLimit unless a caller
// lowered it (set_lookback_limit, for the tests that make a wait run out).
std::atomic<int> g_lookbackLimit{kLookbackSpinLimit};
constexpr int kLookbackWindow = 8;

struct ScratchLayout {
  size_t hist;      // [passes][bins] u32 digit totals
  size_t counters;  // [passes] u32 tile tickets
  size_t lookback;  // [passes][tiles][bins] u32 flagged partial sums
  size_t total;
};

ScratchLayout sort_scratch_layout(size_t capacity, int bits, int digitBits) {
  const int passes = (bits + digitBits - 1) / digitBits;
  const size_t bins = size_t{1} << digitBits;
  const size_t tiles = (capacity + kSortTileKeys - 1) / kSortTileKeys;
  ScratchLayout l{};
  l.hist = 0;
  l.counters = l.hist + passes * bins * 4;
  l.lookback = (l.counters + passes * 4 + 255) / 256 * 256;
  l.total = l.lookback + passes * (tiles > 0 ? tiles : 1) * bins * 4;
  return l;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ uint32_t load_volatile(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void store_volatile(uint32_t *p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <typename K> __device__ __forceinline__ uint32_t digit_of(K key, int shift, uint32_t mask) {
  return (uint32_t)(key >> shift) & mask;
}

// Counts the digits of every pass in one read of the keys: 16-byte vector
// loads, kHistogramVecs per thread, and shared-memory atomics on one
// histogram copy per pair of warps (kHistogramCopies), added up and sent to
// the global histogram once per block.
constexpr int kHistogramVecs = 4;
constexpr int kHistogramCopies = kSortWarps / 2;

template <typename K, int BITS>
__global__ void __launch_bounds__(kSortThreads) k_histogram(const K *__restrict__ keys, const uint32_t *deviceCount,
                                                            uint32_t hostCount, int firstBit, int passes,
                                                            uint32_t *__restrict__ hist) {
  chain_enter();
  constexpr int kBins = 1 << BITS;
  constexpr uint32_t kMask = kBins - 1;
  constexpr int kPerVec = 16 / sizeof(K);
  extern __shared__ uint32_t s_hist[]; // [kHistogramCopies][passes][kBins]
  const int words = passes * kBins;
  for (int i = threadIdx.x; i < kHistogramCopies * words; i += kSortThreads) s_hist[i] = 0u;
  __syncthreads();
  const uint32_t count = deviceCount != nullptr ? *deviceCount : hostCount;
  uint32_t *mine = s_hist + ((threadIdx.x >> 5) % kHistogramCopies) * words;
  const size_t vecs = div_up(count, kPerVec);
  const size_t stride = (size_t)gridDim.x * kSortThreads * kHistogramVecs;
  for (size_t base = (size_t)blockIdx.x * kSortThreads * kHistogramVecs; base < vecs; base += stride) {
    // All loads first; the last, ragged vector element by element.
    K items[kHistogramVecs][kPerVec];
#pragma unroll
    for (int q = 0; q < kHistogramVecs; ++q) {
      const size_t v = base + (size_t)q * kSortThreads + threadIdx.x;
      if ((v + 1) * kPerVec <= count) {
        const uint4 raw = reinterpret_cast<const uint4 *>(keys)[v];
        const K *k = reinterpret_cast<const K *>(&raw);
#pragma unroll
        for (int e = 0; e < kPerVec; ++e) items[q][e] = k[e];
      } else {
#pragma unroll
        for (int e = 0; e < kPerVec; ++e) items[q][e] = v * kPerVec + e < count ? keys[v * kPerVec + e] : K(0);
      }
    }
#pragma unroll
    for (int q = 0; q < kHistogramVecs; ++q) {
      const size_t v = base + (size_t)q * kSortThreads + threadIdx.x;
#pragma unroll
      for (int e = 0; e < kPerVec; ++e) {
        if (v * kPerVec + e >= count) continue;
        for (int p = 0; p < passes; ++p) atomicAdd(&mine[p * kBins + digit_of(items[q][e], firstBit + p * BITS, kMask)], 1u);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < words; i += kSortThreads) {
    uint32_t total = 0;
#pragma unroll
    for (int c = 0; c < kHistogramCopies; ++c) total += s_hist[c * words + i];
    if (total != 0u) atomicAdd(&hist[i], total);
  }
}

// Polls of a tile's bulk-copy barrier before the kernel gives up on it.
constexpr int kBulkSpinLimit = 1 << 22;

// Named barrier 1 over the block's first `threads` threads (a multiple of
// 32): the threads that own a digit wait for one another while the other
// warps go on to the block barrier.
__device__ __forceinline__ void digit_barrier(uint32_t threads) {
  asm volatile("bar.sync 1, %0;" ::"r"(threads) : "memory");
}

// Two exclusive prefix sums at once over the first kBins threads (one digit
// each), of a into exA and of b into exB. s_warp needs 2 x kBins / 32 words.
// One named barrier.
template <int kBins>
__device__ __forceinline__ void digit_exclusive_scan2(uint32_t a, uint32_t b, uint32_t *s_warp, uint32_t &exA, uint32_t &exB) {
  constexpr int kWarps = kBins / 32;
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t inA = a, inB = b;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t na = __shfl_up_sync(0xFFFFFFFFu, inA, o), nb = __shfl_up_sync(0xFFFFFFFFu, inB, o);
    if (lane >= (uint32_t)o) {
      inA += na;
      inB += nb;
    }
  }
  uint32_t beforeA = 0, beforeB = 0;
  if constexpr (kWarps > 1) {
    if (lane == 31) {
      s_warp[warp] = inA;
      s_warp[kWarps + warp] = inB;
    }
    digit_barrier(kBins);
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      beforeA += (uint32_t)w < warp ? s_warp[w] : 0u;
      beforeB += (uint32_t)w < warp ? s_warp[kWarps + w] : 0u;
    }
  }
  exA = beforeA + inA - a;
  exB = beforeB + inB - b;
}

// One pass: rank, look back, scatter. Dynamic shared memory holds the tile's
// keys (later the keys in digit order), its values as read, the values in
// digit order (in the keys' place, after them, where kApart is false), and
// one digit byte per key. A full tile's keys and values arrive by bulk copy,
// issued as soon as the ticket names the tile; each thread's wait on the
// copy's barrier makes the data visible to it, so a full tile needs no block
// barrier there. The digit-owning threads (the first kBins) combine the
// warps' counts, scan and look back among themselves (named barrier 1); the
// block meets four times in all for a full tile (six where the values take
// the keys' place).
template <typename K, int BITS>
__global__ void __launch_bounds__(kSortThreads, 3) k_onesweep(const K *__restrict__ keysIn, const uint32_t *__restrict__ valsIn,
                                                              K *__restrict__ keysOut, uint32_t *__restrict__ valsOut,
                                                              const uint32_t *deviceCount, uint32_t hostCount,
                                                              const uint32_t *__restrict__ passHist, uint32_t *lookback,
                                                              uint32_t *tileCounter, int shift, int spinLimit, uint32_t *error) {
  chain_enter();
  constexpr int kBins = 1 << BITS;
  constexpr uint32_t kMask = kBins - 1;
  static_assert(kBins % 32 == 0 && kBins <= kSortThreads, "one thread per digit, whole warps");
  // 32-bit keys with digits of up to 7 bits: the values in digit order get
  // their own array, and keys and values go out together. Otherwise they take
  // the keys' place once the keys are out: 64-bit keys would fit two blocks
  // per SM instead of three, and the 8-bit passes measured slower with it.
  constexpr bool kApart = sizeof(K) == 4 && BITS <= 7;
  extern __shared__ __align__(128) unsigned char s_dynamic[];
  K *s_keys = reinterpret_cast<K *>(s_dynamic);
  uint32_t *s_vals = reinterpret_cast<uint32_t *>(s_dynamic + kSortTileKeys * sizeof(K));
  uint32_t *s_out = kApart ? s_vals + kSortTileKeys : reinterpret_cast<uint32_t *>(s_dynamic);
  uint8_t *s_digit = s_dynamic + kSortTileKeys * (sizeof(K) + (kApart ? 8 : 4));
  __shared__ uint32_t s_warpHist[kSortWarps][kBins];
  __shared__ uint32_t s_digitBase[kBins];
  __shared__ uint32_t s_globalBase[kBins];
  __shared__ uint32_t s_scan[2 * (kBins / 32)];
  __shared__ uint32_t s_tile;
  __shared__ __align__(8) uint64_t s_bar;

  const uint32_t t = threadIdx.x, lane = lane_id(), warp = t >> 5;
  if (t == 0) {
    s_tile = atomicAdd(tileCounter, 1u);
    bulk_barrier_init(&s_bar, 1);
  }
  for (int i = t; i < kSortWarps * kBins; i += kSortThreads) (&s_warpHist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t count = deviceCount != nullptr ? *deviceCount : hostCount;
  const size_t tileStart = (size_t)tile * kSortTileKeys;
  if (tileStart >= count) return; // the whole block leaves; no copy was issued
  const uint32_t tileKeys = count - tileStart < (size_t)kSortTileKeys ? (uint32_t)(count - tileStart) : (uint32_t)kSortTileKeys;
  const bool bulk = tileKeys == kSortTileKeys;
  // The pass's digit total, asked for now so that it has arrived by the scan.
  const uint32_t passTotal = t < (uint32_t)kBins ? passHist[t] : 0u;
  if (bulk) {
    if (t == 0) {
      bulk_expect(&s_bar, kSortTileKeys * (uint32_t)(sizeof(K) + 4));
      bulk_load(s_keys, keysIn + tileStart, kSortTileKeys * sizeof(K), &s_bar);
      bulk_load(s_vals, valsIn + tileStart, kSortTileKeys * 4, &s_bar);
    }
    if (!bulk_wait(&s_bar, 0, kBulkSpinLimit)) {
      // Never leave with a copy still landing in this block's shared memory.
      if (t == 0) atomicOr(error, kErrLookbackTimeout);
      bulk_wait(&s_bar, 0, kBulkSpinLimit);
    }
  } else {
    for (uint32_t i = t; i < tileKeys; i += kSortThreads) {
      s_keys[i] = keysIn[tileStart + i];
      s_vals[i] = valsIn[tileStart + i];
    }
    __syncthreads();
  }
  // Warp w owns keys [w*kSortItems*32, (w+1)*kSortItems*32); item j of lane l
  // is at j*32 + l inside that chunk, so (warp, item, lane) is the input order.
  K key[kSortItems];
  uint32_t slot[kSortItems];
  const uint32_t chunk = warp * kSortItems * 32;
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const uint32_t i = chunk + j * 32 + lane;
    key[j] = i < tileKeys ? s_keys[i] : K(0);
  }

  // Multi-split by ballots, item by item in input order: the peers of a
  // digit are the AND of the warp's ballots of its bits (match.any measured
  // slower); the warp's running count of each digit lives in shared memory,
  // read by every peer and advanced by the highest one. (Running counts in
  // registers, lane b % 32 holding digit b, measured slower for 6-bit digits.)
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const uint32_t i = chunk + j * 32 + lane;
    const bool valid = i < tileKeys;
    const uint32_t d = valid ? digit_of(key[j], shift, kMask) : 0u;
    uint32_t peers = __ballot_sync(0xFFFFFFFFu, valid);
    // x ^ (flag - 1): x where the flag is 1, ~x where it is 0.
#pragma unroll
    for (int b = 0; b < BITS; ++b) peers &= __ballot_sync(0xFFFFFFFFu, (d >> b) & 1u) ^ (((d >> b) & 1u) - 1u);
    const uint32_t before = __popc(peers & ((1u << lane) - 1u));
    const uint32_t prior = valid ? s_warpHist[warp][d] : 0u;
    __syncwarp();
    if (valid && lane == (uint32_t)(31 - __clz(peers))) s_warpHist[warp][d] = prior + __popc(peers);
    __syncwarp();
    slot[j] = prior + before;
  }
  __syncthreads();

  if (t < (uint32_t)kBins) {
    // Per digit: exclusive offsets across warps, and the tile's total.
    uint32_t digitTotal = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = s_warpHist[w][t];
      s_warpHist[w][t] = digitTotal;
      digitTotal += c;
    }
    // Publish this tile's aggregate (or, for tile 0, its inclusive prefix) early.
    store_volatile(&lookback[(size_t)tile * kBins + t], (tile == 0 ? kFlagInclusive : kFlagAggregate) | digitTotal);
    // The pass's global digit offsets (an exclusive scan of its histogram) and
    // the digits' offsets inside the tile.
    uint32_t passOffset, digitBase;
    digit_exclusive_scan2<kBins>(passTotal, digitTotal, s_scan, passOffset, digitBase);

    // Decoupled look-back, kLookbackWindow predecessors per poll: the
    // aggregates up to the nearest inclusive prefix are added; a predecessor
    // that has published nothing yet stops the walk there, and the next poll
    // starts from it.
    uint32_t exclusive = 0;
    if (tile > 0) {
      int64_t pred = (int64_t)tile - 1;
      int spins = 0;
      for (;;) {
        uint32_t v[kLookbackWindow];
#pragma unroll
        for (int k = 0; k < kLookbackWindow; ++k)
          v[k] = pred - k >= 0 ? load_volatile(&lookback[(size_t)(pred - k) * kBins + t]) : kFlagInclusive;
        int used = 0;
        bool done = false;
#pragma unroll
        for (int k = 0; k < kLookbackWindow; ++k) {
          if (done || used < k) continue; // stopped before k
          const uint32_t flag = v[k] & ~kValueMask;
          if (flag == 0u) continue;       // pending: the walk resumes here
          exclusive += v[k] & kValueMask;
          used = k + 1;
          done = flag == kFlagInclusive;
        }
        if (done) break;
        pred -= used;
        if (used < kLookbackWindow && ++spins > spinLimit) {
          atomicOr(error, kErrLookbackTimeout);
          break;
        }
      }
      store_volatile(&lookback[(size_t)tile * kBins + t], kFlagInclusive | ((exclusive + digitTotal) & kValueMask));
    }
    s_digitBase[t] = digitBase;
    s_globalBase[t] = passOffset + exclusive - digitBase;
  }
  __syncthreads();

  // Keys (and, kApart, values) into shared memory in digit order, then out:
  // the threads of a warp write consecutive addresses within each digit's run.
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const uint32_t i = chunk + j * 32 + lane;
    if (i < tileKeys) {
      const uint32_t d = digit_of(key[j], shift, kMask);
      slot[j] += s_digitBase[d] + s_warpHist[warp][d];
      s_keys[slot[j]] = key[j];
      if constexpr (kApart) s_out[slot[j]] = s_vals[i];
      s_digit[slot[j]] = (uint8_t)d;
    }
  }
  __syncthreads();
  // A position outside [0, count) can only come from a look-back that gave up
  // (kErrLookbackTimeout is set then): skip the write rather than fault.
  const bool full = tileKeys == kSortTileKeys;
  auto write_out = [&](bool keys, bool values) {
    if (full) {
#pragma unroll
      for (int j = 0; j < kSortItems; ++j) {
        const uint32_t i = j * kSortThreads + t;
        const uint32_t dst = s_globalBase[s_digit[i]] + i;
        if (dst < count) {
          if (keys) keysOut[dst] = s_keys[i];
          if (values) valsOut[dst] = s_out[i];
        }
      }
    } else {
      for (uint32_t i = t; i < tileKeys; i += kSortThreads) {
        const uint32_t dst = s_globalBase[s_digit[i]] + i;
        if (dst < count) {
          if (keys) keysOut[dst] = s_keys[i];
          if (values) valsOut[dst] = s_out[i];
        }
      }
    }
  };
  if constexpr (kApart) {
    write_out(true, true);
  } else {
    write_out(true, false);
    __syncthreads();
    // The same permutation for the values, straight from where they landed.
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
      const uint32_t i = chunk + j * 32 + lane;
      if (i < tileKeys) s_out[slot[j]] = s_vals[i];
    }
    __syncthreads();
    write_out(false, true);
  }
}

template <typename K, int BITS> size_t onesweep_smem() {
  return kSortTileKeys * (sizeof(K) + (sizeof(K) == 4 && BITS <= 7 ? 8 : 4)) + kSortTileKeys;
}

template <typename K, int BITS>
int sort_pairs_impl(K *keys, uint32_t *values, K *tmpKeys, uint32_t *tmpValues, size_t capacity, uint32_t hostCount,
                    const uint32_t *deviceCount, int firstBit, int bits, void *scratch, uint32_t *error,
                    cudaStream_t stream, bool clearScratch) {
  constexpr int kBins = 1 << BITS;
  const int passes = (bits + BITS - 1) / BITS;
  if (capacity == 0 || passes == 0) return 0;
  if (deviceCount == nullptr && hostCount <= 1) return 0;
  const ScratchLayout l = sort_scratch_layout(capacity, bits, BITS);
  unsigned char *base = static_cast<unsigned char *>(scratch);
  uint32_t *hist = reinterpret_cast<uint32_t *>(base + l.hist);
  uint32_t *counters = reinterpret_cast<uint32_t *>(base + l.counters);
  uint32_t *lookback = reinterpret_cast<uint32_t *>(base + l.lookback);
  if (clearScratch) cudaMemsetAsync(scratch, 0, l.total, stream);

  const uint32_t launchKeys = deviceCount != nullptr ? (uint32_t)capacity : hostCount;
  const uint32_t tiles = div_up(launchKeys, kSortTileKeys);
  constexpr uint32_t kPerVec = 16 / sizeof(K);
  const uint32_t histBlocks =
      std::min<uint32_t>(div_up(div_up(launchKeys, kPerVec), (uint32_t)(kSortThreads * kHistogramVecs)), 148u * 8u);
  const size_t histSmem = (size_t)kHistogramCopies * passes * kBins * 4;
  static bool configured = false;
  const size_t smem = onesweep_smem<K, BITS>();
  if (!configured) {
    cudaFuncSetAttribute(k_onesweep<K, BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_histogram<K, BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kHistogramCopies * kMaxPasses * kBins * 4));
    configured = true;
  }
  launch_chained(k_histogram<K, BITS>, dim3(std::max(histBlocks, 1u)), dim3(kSortThreads), histSmem, stream, keys, deviceCount, hostCount, firstBit,
                                                                                     passes, hist);
  K *srcK = keys, *dstK = tmpKeys;
  uint32_t *srcV = values, *dstV = tmpValues;
  for (int p = 0; p < passes; ++p) {
    launch_chained(k_onesweep<K, BITS>, dim3(tiles), dim3(kSortThreads), smem, stream, srcK, srcV, dstK, dstV, deviceCount, hostCount,
                                                               hist + p * kBins, lookback + (size_t)p * tiles * kBins,
                                                               counters + p, firstBit + p * BITS,
                                                               g_lookbackLimit.load(std::memory_order_relaxed), error);
    K *tk = srcK;
    srcK = dstK;
    dstK = tk;
    uint32_t *tv = srcV;
    srcV = dstV;
    dstV = tv;
  }
  return srcK == keys ? 0 : 1;
}

} // namespace

size_t sort_scratch_bytes(size_t capacity, int /*keyBytes*/, int bits, int digitBits) {
  return sort_scratch_layout(capacity, bits, digitBits).total;
}

int sort_pairs_u32(uint32_t *keys, uint32_t *values, uint32_t *tmpKeys, uint32_t *tmpValues, size_t capacity,
                   uint32_t hostCount, const uint32_t *deviceCount, int firstBit, int bits, int digitBits, void *scratch,
                   uint32_t *error, cudaStream_t stream, bool clearScratch) {
  switch (digitBits) {
  case 6:
    return sort_pairs_impl<uint32_t, 6>(keys, values, tmpKeys, tmpValues, capacity, hostCount, deviceCount, firstBit, bits,
                                        scratch, error, stream, clearScratch);
  case 7:
    return sort_pairs_impl<uint32_t, 7>(keys, values, tmpKeys, tmpValues, capacity, hostCount, deviceCount, firstBit, bits,
                                        scratch, error, stream, clearScratch);
  default:
    return sort_pairs_impl<uint32_t, 8>(keys, values, tmpKeys, tmpValues, capacity, hostCount, deviceCount, firstBit, bits,
                                        scratch, error, stream, clearScratch);
  }
}

int sort_pairs_u64(unsigned long long *keys, uint32_t *values, unsigned long long *tmpKeys, uint32_t *tmpValues,
                   size_t capacity, uint32_t hostCount, const uint32_t *deviceCount, int firstBit, int bits, int digitBits,
                   void *scratch, uint32_t *error, cudaStream_t stream, bool clearScratch) {
  switch (digitBits) {
  case 6:
    return sort_pairs_impl<unsigned long long, 6>(keys, values, tmpKeys, tmpValues, capacity, hostCount, deviceCount,
                                                  firstBit, bits, scratch, error, stream, clearScratch);
  case 7:
    return sort_pairs_impl<unsigned long long, 7>(keys, values, tmpKeys, tmpValues, capacity, hostCount, deviceCount,
                                                  firstBit, bits, scratch, error, stream, clearScratch);
  default:
    return sort_pairs_impl<unsigned long long, 8>(keys, values, tmpKeys, tmpValues, capacity, hostCount, deviceCount,
                                                  firstBit, bits, scratch, error, stream, clearScratch);
  }
}

void set_lookback_limit(int polls) { g_lookbackLimit.store(polls < 0 ? kLookbackSpinLimit : polls, std::memory_order_relaxed); }

} // namespace sb
