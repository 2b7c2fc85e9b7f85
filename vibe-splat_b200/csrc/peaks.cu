// Microbenchmarks of the SM pipes that bound the rasterizer kernels (which
// are bound by instruction issue, not by HBM): FP32 fused multiply-adds, the
// SFU's ex2, conflict-free 16-byte shared-memory loads, and the warp
// instructions the FMA benchmark issues per second. Each kernel fills every SM
// with as many 256-thread blocks as fit and runs a few milliseconds; the best
// of three timed runs (after one untimed) is kept.
#include <algorithm>

#include "common.cuh"
#include "splat_b200.h"

namespace sb {
namespace {

constexpr int kPeakThreads = 256;
constexpr int kChains = 8;   // independent dependency chains per thread
constexpr int kUnroll = 16;  // operations per chain per loop trip

// The sums decide a store that never happens in practice but that the
// compiler cannot rule out, so no chain is optimised away.
__device__ __forceinline__ void keep(float s, float *sink) {
  if (s == 1.2345678e-30f) sink[0] = s;
}

__global__ void __launch_bounds__(kPeakThreads) k_peak_fma(int trips, float *sink) {
  float a[kChains];
#pragma unroll
  for (int j = 0; j < kChains; ++j) a[j] = (float)threadIdx.x * 1e-3f + (float)j;
  for (int t = 0; t < trips; ++t) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
#pragma unroll
      for (int j = 0; j < kChains; ++j) a[j] = fmaf(a[j], 0.999f, 1e-3f);
  }
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < kChains; ++j) s += a[j];
  keep(s, sink);
}

__global__ void __launch_bounds__(kPeakThreads) k_peak_ex2(int trips, float *sink) {
  float a[kChains];
#pragma unroll
  for (int j = 0; j < kChains; ++j) a[j] = -0.01f * (float)(threadIdx.x & 31u) - 0.1f * (float)j;
  for (int t = 0; t < trips; ++t) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
#pragma unroll
      for (int j = 0; j < kChains; ++j) {
        float r;
        asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a[j]));
        a[j] = r - 1.0f; // stays in (-0.5, 0]
      }
  }
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < kChains; ++j) s += a[j];
  keep(s, sink);
}

__global__ void __launch_bounds__(kPeakThreads) k_peak_shared(int trips, float *sink) {
  __shared__ float4 s_data[4 * kPeakThreads];
  for (int i = threadIdx.x; i < 4 * kPeakThreads; i += kPeakThreads)
    s_data[i] = make_float4((float)i, 1.0f, 2.0f, 3.0f);
  __syncthreads();
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  // A warp reads 32 consecutive float4 (512 bytes, four wavefronts, no
  // conflict); volatile loads, so that none is hoisted out of the loop.
  const uint32_t base = static_cast<uint32_t>(__cvta_generic_to_shared(s_data + threadIdx.x));
  for (int t = 0; t < trips; ++t) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      float4 v;
      asm volatile("ld.volatile.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                   : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                   : "r"(base + (uint32_t)(u * kPeakThreads * 16)));
      acc.x += v.x;
      acc.y += v.y;
      acc.z += v.z;
      acc.w += v.w;
    }
  }
  keep(acc.x + acc.y + acc.z + acc.w, sink);
}

template <typename Kernel> double best_ms(Kernel kernel, int blocks, int trips, float *sink) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int r = 0; r < 4; ++r) {
    cudaEventRecord(e0);
    kernel<<<blocks, kPeakThreads>>>(trips, sink);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0) best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

template <typename Kernel> int resident_blocks(Kernel kernel) {
  int device = 0, sms = 0, perSm = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kPeakThreads, 0);
  return std::max(1, sms * std::max(1, perSm));
}

} // namespace

// Defined with the other entry points; records the message of a failed call.
void set_last_error(const char *message);

} // namespace sb

extern "C" int splat_measure_sm_peaks(splat_sm_peaks *out) {
  if (out == nullptr) {
    sb::set_last_error("null output");
    return SPLAT_ERR_INVALID;
  }
  float *sink = nullptr;
  if (cudaMalloc(&sink, 16) != cudaSuccess) {
    cudaGetLastError();
    sb::set_last_error("no CUDA device for the SM microbenchmarks");
    return SPLAT_ERR_DEVICE;
  }
  const int fmaBlocks = sb::resident_blocks(sb::k_peak_fma), ex2Blocks = sb::resident_blocks(sb::k_peak_ex2),
            smemBlocks = sb::resident_blocks(sb::k_peak_shared);
  const int fmaTrips = 2048, ex2Trips = 256, smemTrips = 2048;
  const double fmaMs = sb::best_ms(sb::k_peak_fma, fmaBlocks, fmaTrips, sink);
  const double ex2Ms = sb::best_ms(sb::k_peak_ex2, ex2Blocks, ex2Trips, sink);
  const double smemMs = sb::best_ms(sb::k_peak_shared, smemBlocks, smemTrips, sink);
  const cudaError_t status = cudaDeviceSynchronize();
  cudaFree(sink);
  if (status != cudaSuccess) {
    cudaGetLastError();
    sb::set_last_error("the SM microbenchmarks failed on the device");
    return SPLAT_ERR_DEVICE;
  }
  const double threadsFma = (double)fmaBlocks * sb::kPeakThreads, threadsEx2 = (double)ex2Blocks * sb::kPeakThreads,
               threadsSmem = (double)smemBlocks * sb::kPeakThreads;
  const double fmas = threadsFma * fmaTrips * sb::kUnroll * sb::kChains;
  out->fp32_flops = 2.0 * fmas / (fmaMs * 1e-3);
  out->warp_instructions = fmas / 32.0 / (fmaMs * 1e-3);
  out->sfu_ops = threadsEx2 * ex2Trips * sb::kUnroll * sb::kChains / (ex2Ms * 1e-3);
  out->shared_bytes = threadsSmem * smemTrips * 4.0 * 16.0 / (smemMs * 1e-3);
  sb::set_last_error("");
  return SPLAT_OK;
}
