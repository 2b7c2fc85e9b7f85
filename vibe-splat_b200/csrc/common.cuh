// Shared device-side definitions of the B200 training path: constants, the
// per-view camera record, the projected-splat record and the two math
// policies. Everything here is sm_100a CUDA C++; the file is compiled with
// --fmad=false so that every fused multiply-add is an explicit fmaf and every
// rounding is the same on the GPU and in the CPU restatement.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "chain.cuh"
#include "splat_detmath.h"

namespace sb {

// Reference constants (shaders/train_types.glsl:6-15, src/train/trainer.cpp:22-24).
// The reference's tile (16 x 16 pixels): the binning and rasterizer's default
// and the loss's tile. The float two-pixel rasterizer also runs 32 x 32 tiles.
constexpr int kTileSize = 16;
constexpr int kTilePixels = kTileSize * kTileSize;
// The loss kernels' own tiles: 16 pixels wide, 32 tall.
constexpr int kLossTileW = 16, kLossTileH = 32;
constexpr uint32_t kInvisible = 0xFFFFFFFFu;
constexpr float kLogMinTransmittance = -9.210340372f;
constexpr float kMinQuaternionLength = 1e-4f;
constexpr float kMinConicDeterminant = 1e-6f;
constexpr int kRawPerSplat = 14;   // sums per splat from the backward pass
constexpr int kRawStride = 16;     // padded to 64 bytes per splat in HBM
constexpr int kStatStride = 8;     // densification statistics per splat
constexpr float kAlphaMin = 1.0f / 255.0f;
constexpr float kAlphaMax = 0.99f;

// Status bits a kernel may set in the device error word. No kernel traps:
// it records what went wrong and skips the access.
enum DeviceError : uint32_t {
  kErrLookbackTimeout = 1u,   // a decoupled look-back gave up waiting on a predecessor
  kErrEntryOverflow = 2u,     // more tile entries than the entry pool holds
  kErrBadIndex = 4u,          // an index read from memory was out of range
  kErrShStage = 8u,           // a view's SH coefficients in use exceed the staging its launch was given
};

// One view, as the kernels need it (src/train/trainer.cpp:29-36 GpuCamera,
// shaders/splat_types.glsl:134-140 CameraParams). R and T are the world->camera
// rotation rows and translation: t = R p + T.
struct ViewParams {
  float R[9];          // row-major: R[r*3+c] = view[c][r]
  float T[3];
  float pos[3];        // camera centre in world space
  float nearPlane;
  float fx, fy, cx, cy;
  float widthF, heightF;
  float tanX, tanY;    // 0.5 W / fx, 0.5 H / fy
  int width, height;
  int gridW, gridH;
  int tileBase;        // first global tile id of this view
  int tileCount;
  long long pixelBase; // first pixel of this view in the batched image planes
  float perPixel;      // 1 / (3 W H)
  float fixedScale;    // 3 W H 64, the fixed-point resolution
  int activeDegree;    // SH degree in use
  int activeCoeffs;    // (degree + 1)^2
  // The loss's own grid of kLossTileW x kLossTileH tiles.
  int lossGridW, lossGridH;
  int lossTileBase;    // first global loss tile of this view
  int lossTileCount;
};

// A projected splat, 48 bytes (shaders/train_types.glsl:26-31 TrainSplat):
// conic (inverse 2D covariance xx, xy, yy) and opacity, colour and radius,
// centre and extent (half size of the area it reaches). The binning test's
// reach, 2 log(255 opacity), is kept beside it in its own array.
struct __align__(16) Splat {
  float4 conicOpacity;
  float4 colorRadius;
  float4 centerExtent;
};

// exp and log inside the rasterizer loops. Exact: the deterministic
// functions of splat_detmath.h, bit-reproducible by the CPU restatement.
// Fast: the SFU approximations (ex2.approx / lg2.approx), for the forms that
// trade bit-reproducibility on the CPU for speed; the GPU results are still
// deterministic run to run.
// The rasterizer's exp/log and the base of its log transmittance. The exact
// form works in natural logs with the deterministic exp/log; the SFU form in
// base 2, so that ex2/lg2 need no change of base: the staged conic is scaled
// by kLogScale = log2(e) instead, and log T (image.w) is in bits.
struct ExactMath {
  static constexpr float kLogScale = 1.0f;
  static __device__ __forceinline__ float exp(float x) { return splat_expf(x); }
  static __device__ __forceinline__ float log(float x) { return splat_logf(x); }
};
struct FastMath {
  static constexpr float kLogScale = 1.4426950408889634f;
  static __device__ __forceinline__ float exp(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  }
  static __device__ __forceinline__ float log(float x) {
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  }
};

__host__ __device__ __forceinline__ uint32_t div_up(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// PCG's output permutation as a hash (shaders/train_types.glsl:156-160).
__device__ __forceinline__ uint32_t pcg_word(uint32_t index, uint32_t seed) {
  const uint32_t state = (index ^ (seed * 0x9E3779B9u)) * 747796405u + 2891336453u;
  return ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
}
__device__ __forceinline__ float pcg_uniform(uint32_t index, uint32_t seed) {
  const uint32_t word = pcg_word(index, seed);
  return (float)((word >> 22u) ^ word) * (1.0f / 4294967296.0f);
}

} // namespace sb
