// Onesweep-style stable LSD radix sort of (key, u32 value) pairs.
//
// Replaces the reference's three-kernel-per-pass sort (RadixSorter::record,
// src/core/radix_sort.cpp:70-97, with shaders/radix_histogram.comp,
// scan_blocks/scan_add.comp and radix_scatter.comp) with the single-pass
// scheme of Adinets and Merrill ("Onesweep", 2022):
//   1. one histogram kernel counts the digits of every pass at once;
//   2. one kernel per pass brings a tile of 4096 keys and their values into
//      shared memory by bulk asynchronous copy (cp.async.bulk, completed on an
//      mbarrier), ranks the keys warp by warp (ballots of the digit bits for
//      6- and 7-bit digits, match.any for 8-bit ones), finds its global
//      offsets through a decoupled look-back over the tiles before it, and
//      scatters through shared memory so that each warp writes contiguous
//      runs. Keys, values and their temporaries must be 16-byte aligned.
// Keys are read once per pass and written once; the reference reads them
// twice per pass (histogram and scatter) and runs a recursive scan between.
// Stability matches std::stable_sort (tests/test_radix_sort.cpp:48-59 in the
// reference): keys of equal digit keep their input order inside a tile (ranks
// follow warp, then item, then lane order over a warp-contiguous chunk), and
// tiles are ordered by their id, which is claimed in launch order through an
// atomic counter, so a tile only ever waits on tiles that already run.
//
// Every look-back wait is bounded: after 2^20 polls the kernel sets
// kErrLookbackTimeout in the error word, takes what it has and finishes; every
// scattered position is then still checked against the count, so no write
// leaves the arrays (a partial prefix only moves a key to a lower slot).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace sb {

// Whether all four arrays start on a 16-byte boundary (vector loads and bulk
// copies need it).
inline bool sort_aligned(const void *a, const void *b, const void *c, const void *d) {
  return ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) | reinterpret_cast<uintptr_t>(c) |
           reinterpret_cast<uintptr_t>(d)) &
          15u) == 0u;
}

// Scratch one sort needs, in bytes, for `capacity` keys of `keyBytes` bytes,
// sorted over `bits` significant bits (from bit `firstBit`) with `digitBits`-bit
// digits. The layout is fixed by sort_scratch_layout() in sort.cu.
size_t sort_scratch_bytes(size_t capacity, int keyBytes, int bits, int digitBits);

// Sorts count pairs, ascending by bits [firstBit, firstBit + bits) of the keys.
// keys/values hold the input; tmpKeys/tmpValues are the same size. Returns 0 if
// the sorted pairs ended in keys/values, 1 if in tmpKeys/tmpValues. The count is
// read from *deviceCount when it is not null (CUDA-graph friendly; capacity
// bounds the launch), else hostCount is used. scratch must hold
// sort_scratch_bytes(capacity, ...) bytes, cleared by the sort itself unless
// clearScratch is false, when the caller has already set those bytes to zero;
// error is a device word that gets kErrLookbackTimeout if a wait ran out.
// Supported digitBits: 6, 7, 8.
int sort_pairs_u32(uint32_t *keys, uint32_t *values, uint32_t *tmpKeys, uint32_t *tmpValues, size_t capacity,
                   uint32_t hostCount, const uint32_t *deviceCount, int firstBit, int bits, int digitBits,
                   void *scratch, uint32_t *error, cudaStream_t stream, bool clearScratch = true);
int sort_pairs_u64(unsigned long long *keys, uint32_t *values, unsigned long long *tmpKeys, uint32_t *tmpValues,
                   size_t capacity, uint32_t hostCount, const uint32_t *deviceCount, int firstBit, int bits, int digitBits,
                   void *scratch, uint32_t *error, cudaStream_t stream, bool clearScratch = true);

// The look-back poll limit of later sort launches; a negative value restores
// the default. For the tests that make a wait run out on purpose.
void set_lookback_limit(int polls);

} // namespace sb
