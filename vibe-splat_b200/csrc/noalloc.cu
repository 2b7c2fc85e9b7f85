// The radix sort of splat_radix_sort_u32 for callers that must not allocate
// device memory: an application that owns a fixed device-memory budget (as
// the reference trainer's memoryBudget option, trainer.hpp:41, does for its
// own buffers) and cannot let a helper take more, or a latency-critical loop
// in which cudaMalloc and cudaFree would synchronise the device. Its scratch
// (digit histograms, tile tickets, look-back words and an error word) is one
// file-scope __device__ array of a fixed size, which every GPU that loads this
// library holds until the process exits.
#include <cstring>

#include "common.cuh"
#include "sort.cuh"
#include "splat_b200.h"

namespace sb {
namespace {

// Largest sort this entry point takes: 4,194,304 keys of up to 32 bits. With
// 8-bit digits that is 4 passes x 1024 tiles x 256 look-back words, 4 MiB,
// the largest of the 6/7/8-bit digit layouts.
constexpr uint32_t kNoAllocMaxKeys = 1u << 22;
constexpr size_t kNoAllocSortBytes = (size_t{4} << 20) + (size_t{8} << 10);
constexpr size_t kNoAllocErrorOffset = kNoAllocSortBytes;
constexpr size_t kNoAllocBytes = kNoAllocSortBytes + 256;

static __device__ __align__(256) unsigned char g_noAllocScratch[kNoAllocBytes];

// The device address of g_noAllocScratch in the current context. In host code
// the array's name stands for a host-side shadow, not device memory, so the
// address is asked for with the device current, on every call: a cache keyed
// by device index would go stale after cudaDeviceReset (the module is loaded
// again, possibly elsewhere) or under another context on the same device, and
// the lookup costs little next to the sort and its wait.
int scratch_address(void **out, const char **message) {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    *message = "no current CUDA device";
    return SPLAT_ERR_DEVICE;
  }
  void *address = nullptr;
  if (cudaGetSymbolAddress(&address, g_noAllocScratch) != cudaSuccess || address == nullptr) {
    cudaGetLastError();
    *message = "cudaGetSymbolAddress of the no-allocation sort's scratch failed";
    return SPLAT_ERR_DEVICE;
  }
  *out = address;
  return SPLAT_OK;
}

} // namespace

// Defined with the other entry points; records the message of a failed call.
void set_last_error(const char *message);

} // namespace sb

extern "C" int splat_radix_sort_u32_noalloc(uint32_t *keys, uint32_t *values, uint32_t *tmp_keys, uint32_t *tmp_values,
                                            uint32_t count, int32_t key_bits, int32_t digit_bits, void *stream) {
  const auto fail = [](int status, const char *message) {
    sb::set_last_error(message);
    return status;
  };
  if (key_bits < 1 || key_bits > 32) return fail(SPLAT_ERR_INVALID, "key_bits must be 1..32");
  const int digits = digit_bits == 0 ? 8 : digit_bits;
  if (digits < 6 || digits > 8) return fail(SPLAT_ERR_INVALID, "digit_bits must be 6, 7 or 8");
  if (!sb::sort_aligned(keys, values, tmp_keys, tmp_values)) {
    return fail(SPLAT_ERR_INVALID, "keys, values and temporaries must be 16-byte aligned");
  }
  if (count > sb::kNoAllocMaxKeys) {
    return fail(SPLAT_ERR_INVALID, "count exceeds the no-allocation sort's maximum of 4194304 keys");
  }
  if (count <= 1) {
    sb::set_last_error("");
    return SPLAT_OK;
  }
  if (sb::sort_scratch_bytes(count, 4, key_bits, digits) > sb::kNoAllocSortBytes) {
    return fail(SPLAT_ERR_INVALID, "the sort needs more scratch than the no-allocation sort holds");
  }
  void *base = nullptr;
  const char *message = nullptr;
  const int status = sb::scratch_address(&base, &message);
  if (status != SPLAT_OK) return fail(status, message);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint32_t *error = reinterpret_cast<uint32_t *>(static_cast<unsigned char *>(base) + sb::kNoAllocErrorOffset);
  // The array keeps the last call's contents: the error word is cleared here,
  // the histograms, tickets and look-back words by sort_pairs_u32 itself.
  if (cudaMemsetAsync(error, 0, sizeof(uint32_t), s) != cudaSuccess) {
    cudaGetLastError();
    return fail(SPLAT_ERR_DEVICE, "cudaMemsetAsync of the error word failed");
  }
  const int where = sb::sort_pairs_u32(keys, values, tmp_keys, tmp_values, count, count, nullptr, 0, key_bits, digits, base,
                                       error, s);
  if (cudaGetLastError() != cudaSuccess) return fail(SPLAT_ERR_DEVICE, "a launch of the sort's kernels failed");
  if (where == 1) {
    if (cudaMemcpyAsync(keys, tmp_keys, (size_t)count * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(values, tmp_values, (size_t)count * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
      cudaGetLastError();
      return fail(SPLAT_ERR_DEVICE, "copying the sorted pairs back failed");
    }
  }
  uint32_t err = 0;
  if (cudaMemcpyAsync(&err, error, sizeof(uint32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    cudaGetLastError();
    return fail(SPLAT_ERR_DEVICE, "the sort failed on the device");
  }
  if (err != 0) return fail(SPLAT_ERR_DEVICE, "the sort's look-back gave up waiting");
  sb::set_last_error("");
  return SPLAT_OK;
}
