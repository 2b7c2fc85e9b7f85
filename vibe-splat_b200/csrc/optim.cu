// The chain rule from the backward pass's screen-space sums to the raw
// parameters, and what becomes of the result: densification statistics only,
// gradients stored, or Adam's step. Restates shaders/train_gradient.comp
// :105-315 (chain), :94-101 (add_statistics), :57-76 (EMITTER),
// shaders/train_step.glsl:119-130 (step_parameter), shaders/bf16.glsl:6-27 and
// shaders/train_sh_step.comp:19-70 (the SH step, with half_stochastic,
// train_step.glsl:140-150).
//
// SH lives in planes (coefficient-major), so neighbouring threads touch
// neighbouring words for every coefficient, which is what the reference's
// separate one-thread-per-word SH pass was for. A one-view Adam step is one
// kernel, one thread per Gaussian (k_chain_step). The other cases run the
// chain rule (k_chain), then Adam on the geometry (k_adam_geometry) and the
// SH step (k_sh_step); with several views in a batch the chain rule runs per
// view and the gradients are summed before one step.
// Out of scope and rejected by the host: the Mip 2D filter, the 3D filter,
// SH dropout, second-order steps, pose gradients, position noise.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "bulk.cuh"
#include "kernels.cuh"
#include "shmath.cuh"

namespace sb {

namespace {

constexpr int kMaxCoeffs = 16;

__device__ __forceinline__ float bf16_load(uint32_t word, int slot) {
  return __uint_as_float(slot == 0 ? word << 16 : word & 0xFFFF0000u);
}
__device__ __forceinline__ uint32_t bf16_stochastic(float x, uint32_t index, uint32_t seed) {
  const uint32_t word = pcg_word(index, seed);
  return (__float_as_uint(x) + (((word >> 22u) ^ word) & 0xFFFFu)) >> 16;
}
// The state word of a BF16 pair: m rounded to nearest even in the low half,
// v rounded at random (as bf16_stochastic) in the high half. The random
// rounding is done on v's bits first, which leaves a value the conversion
// keeps exactly; one conversion then rounds m and packs both.
__device__ __forceinline__ uint32_t bf16_pair(float m, float v, uint32_t index, uint32_t seed) {
  const uint32_t word = pcg_word(index, seed);
  const float vRounded = __uint_as_float((__float_as_uint(v) + (((word >> 22u) ^ word) & 0xFFFFu)) & 0xFFFF0000u);
  uint32_t packed;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(packed) : "f"(vRounded), "f"(m));
  return packed;
}

// Half floats rounded at random, in proportion to the distance to each neighbour.
__device__ __forceinline__ __half half_stochastic(float x, uint32_t index, uint32_t seed) {
  const __half nearest = __float2half_rn(x);
  const float rounded = __half2float(nearest);
  if (rounded == x || isinf(rounded)) return nearest;
  const unsigned short nb = __half_as_ushort(nearest);
  const unsigned short ob = fabsf(x) > fabsf(rounded) ? (unsigned short)(nb + 1u) : (unsigned short)(nb - 1u);
  const __half other = __ushort_as_half(ob);
  const float gap = __half2float(other) - rounded;
  return pcg_uniform(index, seed) < (x - rounded) / gap ? other : nearest;
}

struct AdamArgs {
  float beta1, beta2, epsilon, invCorrection1, invCorrection2;
  uint32_t seed;
};

__device__ __forceinline__ AdamArgs adam_args(const ChainArgs &c) {
  return AdamArgs{c.beta1, c.beta2, c.epsilon, 1.0f / c.correction1, 1.0f / c.correction2, c.seed};
}

__device__ __forceinline__ float sqrt_sfu(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// The SH Adam state lies in rows: element e (= 3 k + c) of Gaussian i at word
// i S + e, S = sh_state_stride (3 (degree + 1)^2 words rounded up to 16
// bytes), the row count rounded up to a multiple of 128 (kPlaneAlign); F32
// state keeps its v rows after the m rows, planeStride S words later. A
// Gaussian's state is one contiguous, 16-byte aligned run, which a step
// touching a few Gaussians here and there reads and writes in whole sectors.
__host__ __device__ __forceinline__ size_t sh_state_at(uint32_t i, uint32_t e, uint32_t S) { return (size_t)i * S + e; }

// Adam on one parameter (step_parameter with radius < 0): the bias
// corrections as multiplications by their reciprocals, the square root and
// the step's division on the SFU (the reference's GLSL sqrt and division are
// not correctly rounded either); the square root flushes subnormal inputs to
// zero, where the step's denominator is the epsilon either way.
__device__ __forceinline__ void adam(float &value, float &m, float &v, float g, float rate, const AdamArgs &a) {
  m = a.beta1 * m + (1.0f - a.beta1) * g;
  v = a.beta2 * v + (1.0f - a.beta2) * g * g;
  value -= __fdividef(rate * (m * a.invCorrection1), sqrt_sfu(v * a.invCorrection2) + a.epsilon);
}

// Steps parameter `at` of a group whose state is `state` (F32: m then v planes
// of `count` floats each; BF16Pair: one word per parameter).
__device__ __forceinline__ void step_state(float &value, void *state, StateStore store, size_t count, size_t at, float g,
                                           float rate, const AdamArgs &a, uint32_t hashIndex) {
  if (store == StateStore::F32) {
    float *s = static_cast<float *>(state);
    float m = s[at], v = s[count + at];
    adam(value, m, v, g, rate, a);
    s[at] = m;
    s[count + at] = v;
  } else {
    uint32_t *s = static_cast<uint32_t *>(state);
    const uint32_t word = s[at];
    float m = bf16_load(word, 0), v = bf16_load(word, 1);
    adam(value, m, v, g, rate, a);
    s[at] = bf16_pair(m, v, hashIndex, a.seed);
  }
}

// tr(G (A X J^T)) for symmetric 2x2 G, 2x3 A and J, 3x3 X (trace_term).
__device__ __forceinline__ float trace_term(const float G[2][2], const float A[2][3], const float X[3][3], const float J[2][3]) {
  float AX[2][3];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) AX[r][c] = fmaf(A[r][2], X[2][c], fmaf(A[r][1], X[1][c], A[r][0] * X[0][c]));
  float Mx[2][2];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int s = 0; s < 2; ++s) Mx[r][s] = fmaf(AX[r][2], J[s][2], fmaf(AX[r][1], J[s][1], AX[r][0] * J[s][0]));
  return fmaf(G[0][0], Mx[0][0], G[0][1] * Mx[1][0]) + fmaf(G[1][0], Mx[0][1], G[1][1] * Mx[1][1]);
}

template <ShStore S>
__device__ __forceinline__ void store_sh_rest(void *p, size_t idx, float value, uint32_t hashIndex, uint32_t seed) {
  if constexpr (S == ShStore::F32) {
    static_cast<float *>(p)[idx] = value;
  } else if constexpr (S == ShStore::BF16) {
    static_cast<uint16_t *>(p)[idx] = (uint16_t)bf16_stochastic(value, hashIndex, seed ^ 0x5DEECE66u);
  } else {
    static_cast<__half *>(p)[idx] = half_stochastic(value, hashIndex, seed ^ 0x5DEECE66u);
  }
}

// One SH basis function and its gradient, for a coefficient index the caller
// unrolls (so the switch folds away). Formulas as sh_basis / sh_basis_gradient.
__device__ __forceinline__ float basis_one(int k, float x, float y, float z) {
  switch (k) {
  case 0: return 0.28209479177387814f;
  case 1: return -0.4886025119029199f * y;
  case 2: return 0.4886025119029199f * z;
  case 3: return -0.4886025119029199f * x;
  case 4: return 1.0925484305920792f * x * y;
  case 5: return -1.0925484305920792f * y * z;
  case 6: return 0.31539156525252005f * (2.0f * (z * z) - x * x - y * y);
  case 7: return -1.0925484305920792f * x * z;
  case 8: return 0.5462742152960396f * (x * x - y * y);
  case 9: return -0.5900435899266435f * y * (3.0f * (x * x) - y * y);
  case 10: return 2.890611442640554f * x * y * z;
  case 11: return -0.4570457994644658f * y * (4.0f * (z * z) - x * x - y * y);
  case 12: return 0.3731763325901154f * z * (2.0f * (z * z) - 3.0f * (x * x) - 3.0f * (y * y));
  case 13: return -0.4570457994644658f * x * (4.0f * (z * z) - x * x - y * y);
  case 14: return 1.445305721320277f * z * (x * x - y * y);
  default: return -0.5900435899266435f * x * (x * x - 3.0f * (y * y));
  }
}

__device__ __forceinline__ void basis_gradient_one(int k, float x, float y, float z, float g[3]) {
  const float C1 = 0.4886025119029199f, A = 1.0925484305920792f, K = 0.31539156525252005f, L = 0.5462742152960396f;
  const float C = -0.5900435899266435f, E = 2.890611442640554f, F = -0.4570457994644658f, G = 0.3731763325901154f,
              H = 1.445305721320277f;
  const float xx = x * x, yy = y * y, zz = z * z;
  switch (k) {
  case 1: g[0] = 0.f; g[1] = -C1; g[2] = 0.f; break;
  case 2: g[0] = 0.f; g[1] = 0.f; g[2] = C1; break;
  case 3: g[0] = -C1; g[1] = 0.f; g[2] = 0.f; break;
  case 4: g[0] = A * y; g[1] = A * x; g[2] = 0.f; break;
  case 5: g[0] = -A * 0.f; g[1] = -A * z; g[2] = -A * y; break;
  case 6: g[0] = K * (-2.0f * x); g[1] = K * (-2.0f * y); g[2] = K * (4.0f * z); break;
  case 7: g[0] = -A * z; g[1] = -A * 0.f; g[2] = -A * x; break;
  case 8: g[0] = L * (2.0f * x); g[1] = L * (-2.0f * y); g[2] = 0.f; break;
  case 9: g[0] = C * (6.0f * x * y); g[1] = C * (3.0f * xx - 3.0f * yy); g[2] = 0.f; break;
  case 10: g[0] = E * (y * z); g[1] = E * (x * z); g[2] = E * (x * y); break;
  case 11: g[0] = F * (-2.0f * x * y); g[1] = F * (4.0f * zz - xx - 3.0f * yy); g[2] = F * (8.0f * y * z); break;
  case 12: g[0] = G * (-6.0f * x * z); g[1] = G * (-6.0f * y * z); g[2] = G * (6.0f * zz - 3.0f * xx - 3.0f * yy); break;
  case 13: g[0] = F * (4.0f * zz - 3.0f * xx - yy); g[1] = F * (-2.0f * x * y); g[2] = F * (8.0f * x * z); break;
  case 14: g[0] = H * (2.0f * x * z); g[1] = H * (-2.0f * y * z); g[2] = H * (xx - yy); break;
  case 15: g[0] = C * (3.0f * xx - 3.0f * yy); g[1] = C * (-6.0f * x * y); g[2] = 0.f; break;
  default: g[0] = g[1] = g[2] = 0.f; break;
  }
}

// The chain rule of one view for Gaussian i (train_gradient.comp:165-275):
// adds its scale, rotation and opacity gradients, and returns the position
// gradient of this view without the view-direction term (gPv), the colour
// gradient where the colour was not clamped, the view direction and the
// distance. The direction term needs the SH coefficients: add_direction_term
// finishes gPv with it.
__device__ __forceinline__ void chain_view(const ViewParams &cam, const float raw[kRawPerSplat], const float4 col,
                                           const float pos[3], const float logScale[3], float opacity, float4 rq,
                                           float gPv[3], float gScale[3], float gRot[4], float &gOpacity, float gColour[3],
                                           float dir[3], float &distance) {
  const float px = pos[0], py = pos[1], pz = pos[2];
  const float quatLength = sqrtf(fmaf(rq.w, rq.w, fmaf(rq.z, rq.z, fmaf(rq.y, rq.y, rq.x * rq.x))));
  float q[4] = {1.f, 0.f, 0.f, 0.f};
  if (quatLength > 0.0f) {
    q[0] = rq.x / quatLength;
    q[1] = rq.y / quatLength;
    q[2] = rq.z / quatLength;
    q[3] = rq.w / quatLength;
  }
  const float t[3] = {fmaf(cam.R[2], pz, fmaf(cam.R[1], py, fmaf(cam.R[0], px, cam.T[0]))),
                      fmaf(cam.R[5], pz, fmaf(cam.R[4], py, fmaf(cam.R[3], px, cam.T[1]))),
                      fmaf(cam.R[8], pz, fmaf(cam.R[7], py, fmaf(cam.R[6], px, cam.T[2])))};
  const float fx = cam.fx, fy = cam.fy;
  const float z = t[2], iz = 1.0f / z, iz2 = iz * iz;
  const float G[2][2] = {{raw[3], raw[4]}, {raw[4], raw[5]}};
  float Rv[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) Rv[r][c] = cam.R[r * 3 + c];
  float R[3][3];
  quat_to_matrix(q[0], q[1], q[2], q[3], R);
  const float s2[3] = {splat_expf(2.0f * logScale[0]), splat_expf(2.0f * logScale[1]), splat_expf(2.0f * logScale[2])};
  float sigma[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c)
      sigma[r][c] = fmaf(R[r][2] * s2[2], R[c][2], fmaf(R[r][1] * s2[1], R[c][1], R[r][0] * s2[0] * R[c][0]));
  float X[3][3];
  {
    float RS[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) RS[r][c] = fmaf(Rv[r][2], sigma[2][c], fmaf(Rv[r][1], sigma[1][c], Rv[r][0] * sigma[0][c]));
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) X[r][c] = fmaf(RS[r][2], Rv[c][2], fmaf(RS[r][1], Rv[c][1], RS[r][0] * Rv[c][0]));
  }
  const float limX = 1.3f * cam.tanX, limY = 1.3f * cam.tanY;
  const float rx = t[0] * iz, ry = t[1] * iz;
  const bool clampedX = fabsf(rx) > limX, clampedY = fabsf(ry) > limY;
  const float tx = fminf(fmaxf(rx, -limX), limX) * z, ty = fminf(fmaxf(ry, -limY), limY) * z;
  const float J[2][3] = {{fx * iz, 0.f, -fx * tx * iz2}, {0.f, fy * iz, -fy * ty * iz2}};
  const float Jc[2][3] = {{fx * iz, 0.f, -fx * t[0] * iz2}, {0.f, fy * iz, -fy * t[1] * iz2}};
  float gT[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) gT[k] = fmaf(Jc[1][k], raw[2], Jc[0][k] * raw[1]);
  const float dJx[2][3] = {{0.f, 0.f, clampedX ? 0.0f : -fx * iz2}, {0.f, 0.f, 0.f}};
  const float dJy[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, clampedY ? 0.0f : -fy * iz2}};
  const float dJz[2][3] = {{-fx * iz2, 0.f, clampedX ? fx * tx * iz2 * iz : 2.0f * fx * tx * iz2 * iz},
                           {0.f, -fy * iz2, clampedY ? fy * ty * iz2 * iz : 2.0f * fy * ty * iz2 * iz}};
  gT[0] += 2.0f * trace_term(G, dJx, X, J);
  gT[1] += 2.0f * trace_term(G, dJy, X, J);
  gT[2] += 2.0f * trace_term(G, dJz, X, J);
#pragma unroll
  for (int c = 0; c < 3; ++c) gPv[c] = fmaf(Rv[2][c], gT[2], fmaf(Rv[1][c], gT[1], Rv[0][c] * gT[0]));

  // T2 = J Rv (2x3), G3 = T2^T G T2.
  float T2[2][3];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) T2[r][c] = fmaf(J[r][2], Rv[2][c], fmaf(J[r][1], Rv[1][c], J[r][0] * Rv[0][c]));
  float G3[3][3];
  {
    float GT[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) GT[r][c] = fmaf(G[r][1], T2[1][c], G[r][0] * T2[0][c]);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) G3[a][b] = fmaf(T2[1][a], GT[1][b], T2[0][a] * GT[0][b]);
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float ax[3] = {R[0][a], R[1][a], R[2][a]};
    float Ga[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) Ga[r] = fmaf(G3[r][2], ax[2], fmaf(G3[r][1], ax[1], G3[r][0] * ax[0]));
    gScale[a] += 2.0f * s2[a] * fmaf(ax[2], Ga[2], fmaf(ax[1], Ga[1], ax[0] * Ga[0]));
  }
  // Rotation: P = 2 G3 R D, gq_k = <P, dR/dq_k> (the GLSL column constructors, transposed to rows).
  float P[3][3];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) P[r][c] = 2.0f * fmaf(G3[r][2], R[2][c], fmaf(G3[r][1], R[1][c], G3[r][0] * R[0][c])) * s2[c];
  const float w = q[0], x = q[1], y = q[2], zq = q[3];
  const float gq[4] = {
      2.0f * (-P[0][1] * zq + P[0][2] * y + P[1][0] * zq - P[1][2] * x - P[2][0] * y + P[2][1] * x),
      2.0f * (P[0][1] * y + P[0][2] * zq + P[1][0] * y - 2.0f * P[1][1] * x - P[1][2] * w + P[2][0] * zq + P[2][1] * w -
              2.0f * P[2][2] * x),
      2.0f * (-2.0f * P[0][0] * y + P[0][1] * x + P[0][2] * w + P[1][0] * x + P[1][2] * zq - P[2][0] * w + P[2][1] * zq -
              2.0f * P[2][2] * y),
      2.0f * (-2.0f * P[0][0] * zq - P[0][1] * w + P[0][2] * x + P[1][0] * w - 2.0f * P[1][1] * zq + P[1][2] * y +
              P[2][0] * x + P[2][1] * y)};
  const float qg = fmaf(q[3], gq[3], fmaf(q[2], gq[2], fmaf(q[1], gq[1], q[0] * gq[0])));
  const float inv = fmaxf(quatLength, 1e-12f);
#pragma unroll
  for (int k = 0; k < 4; ++k) gRot[k] += (gq[k] - q[k] * qg) / inv;
  gOpacity += raw[0] * opacity * (1.0f - opacity);

  // Colour: the gradient reaches the coefficients in use where the colour was
  // not clamped at zero (the splat keeps the clamped colour).
  gColour[0] = col.x > 0.0f ? raw[6] : 0.0f;
  gColour[1] = col.y > 0.0f ? raw[7] : 0.0f;
  gColour[2] = col.z > 0.0f ? raw[8] : 0.0f;
  const float ddx = px - cam.pos[0], ddy = py - cam.pos[1], ddz = pz - cam.pos[2];
  distance = sqrtf(fmaf(ddz, ddz, fmaf(ddy, ddy, ddx * ddx)));
  dir[0] = ddx / distance;
  dir[1] = ddy / distance;
  dir[2] = ddz / distance;
}

// Position also changes the view direction, and with it the colour: the
// gradient through the coefficients 1..active-1 of each channel, in order.
// c[3] are coefficient k's values before any step.
__device__ __forceinline__ void direction_term(int k, const float c[3], const float gColour[3], const float dir[3], float gDir[3]) {
  const float d = fmaf(gColour[2], c[2], fmaf(gColour[1], c[1], gColour[0] * c[0]));
  float bg[3];
  basis_gradient_one(k, dir[0], dir[1], dir[2], bg);
#pragma unroll
  for (int a = 0; a < 3; ++a) gDir[a] = fmaf(d, bg[a], gDir[a]);
}

__device__ __forceinline__ void add_direction_term(const float gDir[3], const float dir[3], float distance, float gPv[3]) {
  const float dd = fmaf(dir[2], gDir[2], fmaf(dir[1], gDir[1], dir[0] * gDir[0]));
#pragma unroll
  for (int c = 0; c < 3; ++c) gPv[c] += (gDir[c] - dir[c] * dd) / distance;
}

// Geometry part of the chain rule and Adam for positions, scales, rotations
// and opacities (train_gradient.comp:105-315), one thread per Gaussian. For the
// SH step that follows it leaves, per view, the colour gradient where the colour
// was not clamped and the number of coefficients in use (0: the view did not
// reach the Gaussian), then the view direction: shGrad[(v n + i) * 2 + {0, 1}],
// as the reference leaves them in its sums for train_sh_step.comp.
template <ShStore S, bool FIXED, bool MULTI>
__global__ void __launch_bounds__(128, 4) k_chain(Params p, const ViewSet *__restrict__ viewsPtr, const void *__restrict__ rawIn,
                                                  const Splat *__restrict__ splats, const ChainArgs *__restrict__ argsPtr,
                                                  OptimState state, GradientsOut grads, bool storeGradients,
                                                  float4 *__restrict__ shGrad, float *__restrict__ densifyStats,
                                                  const uint32_t *error) {
  chain_enter();
  const ViewSet &views = *viewsPtr;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  const ChainArgs args = *argsPtr;
  if (error != nullptr && (*error & kErrEntryOverflow) != 0u) return;
  const size_t n = p.n;
  const bool zeros = args.mode == ChainMode::Gradients || (args.mode == ChainMode::Step && !args.selective);
  const bool penalties = args.opacityReg > 0.0f || args.scaleReg > 0.0f;

  float gP[3] = {0.f, 0.f, 0.f}, gScale[3] = {0.f, 0.f, 0.f}, gRot[4] = {0.f, 0.f, 0.f, 0.f}, gOpacity = 0.f;
  bool anyTouched = false;
  const float pos[3] = {p.positions[i * 3], p.positions[i * 3 + 1], p.positions[i * 3 + 2]};
  const float logScale[3] = {p.scales[i * 3], p.scales[i * 3 + 1], p.scales[i * 3 + 2]};
  const float opacity = 1.0f / (1.0f + splat_expf(-p.opacities[i]));
  const float4 rq = reinterpret_cast<const float4 *>(p.rotations)[i];

  const int viewCount = MULTI ? views.count : 1;
  for (int v = 0; v < viewCount; ++v) {
    const ViewParams &cam = views.v[v];
    const uint4 *r4 = reinterpret_cast<const uint4 *>(rawIn) + ((size_t)v * n + i) * (kRawStride / 4);
    uint32_t words[16];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint4 w4 = r4[q];
      words[q * 4] = w4.x;
      words[q * 4 + 1] = w4.y;
      words[q * 4 + 2] = w4.z;
      words[q * 4 + 3] = w4.w;
    }
    float raw[kRawPerSplat];
    bool touched = false;
#pragma unroll
    for (int k = 0; k < kRawPerSplat; ++k) {
      raw[k] = FIXED ? (float)(int)words[k] / cam.fixedScale : __uint_as_float(words[k]);
      touched = touched || raw[k] != 0.0f;
    }
    float4 *sg = shGrad + ((size_t)v * n + i) * 2;
    if (!touched || args.mode == ChainMode::Statistics) {
      if (args.mode != ChainMode::Statistics) sg[0] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (!touched) continue;
    }
    anyTouched = true;
    const float4 col = splats[(size_t)v * n + i].colorRadius;
    if (args.statistics) {
      float4 *st = reinterpret_cast<float4 *>(densifyStats + (size_t)i * kStatStride);
      float4 a = st[0], b = st[1];
      const float hx = 0.5f * cam.widthF, hy = 0.5f * cam.heightF;
      const float ax = raw[1] * hx, ay = raw[2] * hy;
      a.x += sqrtf(fmaf(ay, ay, ax * ax));
      a.y += 1.0f;
      a.z = fmaxf(a.z, col.w);
      a.w += raw[9] * 3.0f * cam.widthF * cam.heightF;
      const float bx = raw[10] * hx, by = raw[11] * hy;
      b.x += sqrtf(fmaf(by, by, bx * bx));
      st[0] = a;
      st[1] = b;
    }
    if (args.mode == ChainMode::Statistics) continue;
    float gColour[3], dir[3], gPv[3], distance;
    chain_view(cam, raw, col, pos, logScale, opacity, rq, gPv, gScale, gRot, gOpacity, gColour, dir, distance);
    if (cam.activeDegree > 0) {
      float gDir[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int k = 1; k < kMaxCoeffs; ++k) {
        if (k < cam.activeCoeffs) {
          const float c[3] = {sh_coefficient<S>(p, i, k, 0), sh_coefficient<S>(p, i, k, 1), sh_coefficient<S>(p, i, k, 2)};
          direction_term(k, c, gColour, dir, gDir);
        }
      }
      add_direction_term(gDir, dir, distance, gPv);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) gP[c] += gPv[c];
    sg[0] = make_float4(gColour[0], gColour[1], gColour[2], __uint_as_float((uint32_t)cam.activeCoeffs));
    sg[1] = make_float4(dir[0], dir[1], dir[2], 0.0f);
  }

  if (args.mode == ChainMode::Statistics) return;
  // The penalties (3DGS-MCMC) apply to every Gaussian, seen or not.
  if (penalties) {
#pragma unroll
    for (int a = 0; a < 3; ++a) gScale[a] += args.scaleReg * splat_expf(logScale[a]);
    gOpacity += args.opacityReg * opacity * (1.0f - opacity);
  }
  (void)zeros;
  (void)anyTouched;
  (void)state;
  (void)storeGradients;
  // The geometry gradients, zeros for a Gaussian no view reached; the Adam
  // kernel steps them (or they are the stored gradients).
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    grads.g[0][i * 3 + a] = gP[a];
    grads.g[1][i * 3 + a] = gScale[a];
  }
  reinterpret_cast<float4 *>(grads.g[2])[i] = make_float4(gRot[0], gRot[1], gRot[2], gRot[3]);
  grads.g[3][i] = gOpacity;
}

// Adam on positions, scales, rotations and opacities (EMITTER,
// train_gradient.comp:57-76), one thread per element of the four arrays taken
// as one: [positions 3n | scales 3n | rotations 4n | opacities n].
__global__ void __launch_bounds__(256) k_adam_geometry(Params p, const ChainArgs *__restrict__ argsPtr, OptimState state,
                                                       GradientsOut grads, const uint32_t *error) {
  chain_enter();
  const size_t n = p.n;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 11 * n) return;
  if (error != nullptr && (*error & kErrEntryOverflow) != 0u) return;
  const ChainArgs args = *argsPtr;
  uint32_t group;
  size_t idx, count;
  float *values;
  const float *gradient;
  void *st;
  float rate;
  if (t < 3 * n) {
    group = 0, idx = t, count = 3 * n, values = p.positions, gradient = grads.g[0], st = state.state[0], rate = args.rates[0];
  } else if (t < 6 * n) {
    group = 1, idx = t - 3 * n, count = 3 * n, values = p.scales, gradient = grads.g[1], st = state.state[1], rate = args.rates[1];
  } else if (t < 10 * n) {
    group = 2, idx = t - 6 * n, count = 4 * n, values = p.rotations, gradient = grads.g[2], st = state.state[2], rate = args.rates[2];
  } else {
    group = 3, idx = t - 10 * n, count = n, values = p.opacities, gradient = grads.g[3], st = state.state[3], rate = args.rates[3];
  }
  const float g = gradient[idx];
  // A parameter with a zero gradient is left alone when selective.
  if (g == 0.0f && args.selective) return;
  const AdamArgs a = adam_args(args);
  float value = values[idx];
  step_state(value, st, state.store, count, idx, g, rate, a, (uint32_t)idx * 5u + group);
  values[idx] = value;
}

// The SH step (train_sh_step.comp:19-70): blocks along y are groups of four
// coefficients, along x the Gaussians; a thread steps the 12 elements (4
// coefficients x 3 channels) of one Gaussian, so it reads the colour gradient
// and direction the chain-rule kernel left once per group rather than once
// per element, and each warp's accesses to an SH plane cover 32 neighbouring
// Gaussians. The gradient of coefficient k is basis_k(direction) times the
// colour gradient, summed over the views.
constexpr int kShGroup = 4;

template <ShStore S, bool MULTI>
__global__ void __launch_bounds__(256) k_sh_step(Params p, const ViewSet *__restrict__ viewsPtr, const float4 *__restrict__ shGrad,
                                                 const ChainArgs *__restrict__ argsPtr, OptimState state, GradientsOut grads,
                                                 bool storeGradients, const uint32_t *error) {
  chain_enter();
  const ViewSet &views = *viewsPtr;
  const uint32_t n = p.n;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (error != nullptr && (*error & kErrEntryOverflow) != 0u) return;
  const int k0 = (int)blockIdx.y * kShGroup;
  const int shFloats = 3 * p.shCoeffs;
  float g[kShGroup][3];
#pragma unroll
  for (int kk = 0; kk < kShGroup; ++kk) g[kk][0] = g[kk][1] = g[kk][2] = 0.0f;
  bool touched = false;
  const int viewCount = MULTI ? views.count : 1;
  for (int v = 0; v < viewCount; ++v) {
    const float4 a = shGrad[((size_t)v * n + i) * 2];
    const uint32_t coeffs = __float_as_uint(a.w);
    if (coeffs == 0u) continue;
    touched = true;
    const float4 d = shGrad[((size_t)v * n + i) * 2 + 1];
#pragma unroll
    for (int kk = 0; kk < kShGroup; ++kk) {
      const int k = k0 + kk;
      if ((uint32_t)k < coeffs) {
        const float b = basis_one(k, d.x, d.y, d.z);
        g[kk][0] = fmaf(b, a.x, g[kk][0]);
        g[kk][1] = fmaf(b, a.y, g[kk][1]);
        g[kk][2] = fmaf(b, a.z, g[kk][2]);
      }
    }
  }
  if (storeGradients) {
#pragma unroll
    for (int kk = 0; kk < kShGroup; ++kk) {
      if (k0 + kk < p.shCoeffs) {
#pragma unroll
        for (int c = 0; c < 3; ++c) grads.g[4][(size_t)i * shFloats + (k0 + kk) * 3 + c] = g[kk][c];
      }
    }
    return;
  }
  const ChainArgs args = *argsPtr;
  // Only Adam, when not selective, steps parameters without a gradient.
  const bool stepZeros = !args.selective;
  if (!touched && !stepZeros) return;
  const AdamArgs a = adam_args(args);
  const uint32_t stateStride = sh_state_stride(p.shCoeffs);
  const size_t ps = p.planeStride, count = ps * stateStride;
  // Every load first, then the arithmetic, then the stores: the values and the
  // state are reached through plain pointers, so a load placed after a store
  // could not be moved before it, and the 12 updates would run one by one.
  float value[kShGroup][3], m[kShGroup][3], vv[kShGroup][3];
  uint32_t word[kShGroup][3];
#pragma unroll
  for (int kk = 0; kk < kShGroup; ++kk) {
    const int k = k0 + kk;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      value[kk][c] = m[kk][c] = vv[kk][c] = 0.0f;
      word[kk][c] = 0u;
      if (k >= p.shCoeffs) continue;
      const size_t t = (size_t)(k * 3 + c) * ps + i, ts = sh_state_at(i, (uint32_t)(k * 3 + c), stateStride);
      value[kk][c] = k == 0 ? p.shDc[t] : load_sh_rest<S>(p.shRest, sh_rest_at(i, (uint32_t)((k - 1) * 3 + c), p.restStride));
      if (state.store == StateStore::F32) {
        m[kk][c] = static_cast<const float *>(state.state[4])[ts];
        vv[kk][c] = static_cast<const float *>(state.state[4])[count + ts];
      } else {
        word[kk][c] = static_cast<const uint32_t *>(state.state[4])[ts];
        m[kk][c] = bf16_load(word[kk][c], 0);
        vv[kk][c] = bf16_load(word[kk][c], 1);
      }
    }
  }
#pragma unroll
  for (int kk = 0; kk < kShGroup; ++kk) {
    const int k = k0 + kk;
    if (k >= p.shCoeffs) continue;
    const float rate = k == 0 ? args.rates[4] : args.rates[4] * args.restScale;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (g[kk][c] == 0.0f && !stepZeros) continue;
      const uint32_t plane = (uint32_t)(k * 3 + c);
      const size_t t = (size_t)plane * ps + i, ts = sh_state_at(i, plane, stateStride);
      const uint32_t hashIndex = (i * (uint32_t)shFloats + plane) * 5u + 4u;
      adam(value[kk][c], m[kk][c], vv[kk][c], g[kk][c], rate, a);
      if (state.store == StateStore::F32) {
        static_cast<float *>(state.state[4])[ts] = m[kk][c];
        static_cast<float *>(state.state[4])[count + ts] = vv[kk][c];
      } else {
        static_cast<uint32_t *>(state.state[4])[ts] = bf16_pair(m[kk][c], vv[kk][c], hashIndex, a.seed);
      }
      if (k == 0) {
        p.shDc[t] = value[kk][c];
      } else {
        store_sh_rest<S>(p.shRest, sh_rest_at(i, plane - 3u, p.restStride), value[kk][c], hashIndex, args.seed);
      }
    }
  }
}

// One view, Adam step: the chain rule, Adam on the geometry and the SH step
// in one pass, one thread per Gaussian. The SH coefficients are read once,
// for the direction term and for their own step, and no gradient leaves
// registers. Element by element the arithmetic, the hash indices and the
// order of the sums are those of k_chain, k_adam_geometry and k_sh_step, so
// the results are the same bits.
//
// A block's SH planes and SH Adam state (one 16-byte aligned segment of
// kStepThreads elements per plane) are brought into shared memory by bulk
// asynchronous copies issued first thing, so they land while the chain rule
// runs; the SH step then reads them from shared memory.
constexpr int kStepThreads = kPlaneAlign;
// Polls of the staging barrier before the kernel gives up on it.
constexpr int kStageSpinLimit = 1 << 22;

__device__ __forceinline__ void load_state(const void *st, StateStore store, uint32_t count, uint32_t at, float &m, float &v,
                                           uint32_t &word) {
  if (store == StateStore::F32) {
    m = static_cast<const float *>(st)[at];
    v = static_cast<const float *>(st)[count + at];
    word = 0u;
  } else {
    word = static_cast<const uint32_t *>(st)[at];
    m = bf16_load(word, 0);
    v = bf16_load(word, 1);
  }
}

__device__ __forceinline__ void store_state(void *st, StateStore store, uint32_t count, uint32_t at, float m, float v,
                                            uint32_t word, uint32_t hashIndex, uint32_t seed) {
  if (store == StateStore::F32) {
    static_cast<float *>(st)[at] = m;
    static_cast<float *>(st)[count + at] = v;
  } else {
    static_cast<uint32_t *>(st)[at] = bf16_pair(m, v, hashIndex, seed);
  }
}

// Shared-memory bytes of a block's staged SH: the DC planes, the rows of
// higher coefficients (restStride elements each) and the state rows.
__host__ __device__ inline uint32_t step_stage_bytes(int coeffs, int shBytes, bool stateF32, uint32_t restStride) {
  return 3u * kStepThreads * 4u + restStride * kStepThreads * (uint32_t)shBytes +
         (stateF32 ? 2u : 1u) * sh_state_stride(coeffs) * kStepThreads * 4u;
}

template <ShStore S> __device__ __forceinline__ float staged_sh_rest(const unsigned char *rest, uint32_t at) {
  if constexpr (S == ShStore::F32) {
    return reinterpret_cast<const float *>(rest)[at];
  } else if constexpr (S == ShStore::BF16) {
    return __uint_as_float((uint32_t)reinterpret_cast<const uint16_t *>(rest)[at] << 16);
  } else {
    return __half2float(reinterpret_cast<const __half *>(rest)[at]);
  }
}

template <ShStore S, StateStore ST, bool FIXED>
__global__ void __launch_bounds__(kStepThreads, 6) k_chain_step(Params p, const ViewSet *__restrict__ viewsPtr,
                                                                const void *__restrict__ rawIn, const Splat *__restrict__ splats,
                                                                const ChainArgs *__restrict__ argsPtr, OptimState state,
                                                                float *__restrict__ densifyStats, uint32_t *error) {
  chain_enter();
  constexpr uint32_t kShBytes = S == ShStore::F32 ? 4u : 2u;
  extern __shared__ __align__(128) unsigned char s_stage[];
  __shared__ __align__(8) uint64_t s_bar;
  const ViewParams &cam = viewsPtr->v[0];
  if (error != nullptr && (*error & kErrEntryOverflow) != 0u) return; // the whole block, before any copy
  const uint32_t n = p.n, ps = p.planeStride, tid = threadIdx.x;
  const uint32_t i0 = blockIdx.x * kStepThreads, i = i0 + tid;
  const uint32_t planes = 3u * (uint32_t)p.shCoeffs, restPlanes = planes - 3u;
  constexpr bool stateF32 = ST == StateStore::F32;
  float *s_dc = reinterpret_cast<float *>(s_stage);
  unsigned char *s_rest = s_stage + 3u * kStepThreads * 4u;
  unsigned char *s_state = s_rest + p.restStride * kStepThreads * kShBytes;
  if (tid == 0) bulk_barrier_init(&s_bar, 1);
  __syncthreads();
  if (tid < 32u) {
    // Warp 0 issues the copies: DC planes, rest planes, state planes (F32: m then v).
    if (tid == 0) bulk_expect(&s_bar, step_stage_bytes(p.shCoeffs, (int)kShBytes, stateF32, p.restStride));
    __syncwarp();
    // The DC planes, the block's rows of higher coefficients, its state rows.
    const uint32_t rest = restPlanes > 0u ? 1u : 0u, copies = 3u + rest + (stateF32 ? 2u : 1u);
    for (uint32_t c = tid; c < copies; c += 32u) {
      if (c < 3u) {
        bulk_load(s_dc + c * kStepThreads, p.shDc + (size_t)c * ps + i0, kStepThreads * 4u, &s_bar);
      } else if (c < 3u + rest) {
        bulk_load(s_rest, static_cast<const unsigned char *>(p.shRest) + (size_t)i0 * p.restStride * kShBytes,
                  kStepThreads * p.restStride * kShBytes, &s_bar);
      } else {
        // The block's state rows, one copy (F32: the m rows, then the v rows).
        const uint32_t q = c - 3u - rest;
        const uint32_t stride = sh_state_stride(p.shCoeffs);
        bulk_load(s_state + q * kStepThreads * stride * 4u,
                  static_cast<const unsigned char *>(state.state[4]) + ((size_t)q * ps + i0) * stride * 4u,
                  kStepThreads * stride * 4u, &s_bar);
      }
    }
  }
  // From here on a block's threads leave only after waiting for the copies,
  // or when they have no Gaussian (the issuing thread always has one).
  if (i >= n) return;
  const ChainArgs args = *argsPtr;
  const AdamArgs a = adam_args(args);

  const float pos[3] = {p.positions[i * 3], p.positions[i * 3 + 1], p.positions[i * 3 + 2]};
  const float logScale[3] = {p.scales[i * 3], p.scales[i * 3 + 1], p.scales[i * 3 + 2]};
  const float rawOpacity = p.opacities[i];
  const float4 rq = reinterpret_cast<const float4 *>(p.rotations)[i];
  float raw[kRawPerSplat];
  bool touched = false;
  {
    const uint4 *r4 = reinterpret_cast<const uint4 *>(rawIn) + (size_t)i * (kRawStride / 4);
    uint32_t words[16];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint4 w4 = r4[q];
      words[q * 4] = w4.x;
      words[q * 4 + 1] = w4.y;
      words[q * 4 + 2] = w4.z;
      words[q * 4 + 3] = w4.w;
    }
#pragma unroll
    for (int k = 0; k < kRawPerSplat; ++k) {
      raw[k] = FIXED ? (float)(int)words[k] / cam.fixedScale : __uint_as_float(words[k]);
      touched = touched || raw[k] != 0.0f;
    }
  }
  const float opacity = 1.0f / (1.0f + splat_expf(-rawOpacity));

  float gP[3] = {0.f, 0.f, 0.f}, gScale[3] = {0.f, 0.f, 0.f}, gRot[4] = {0.f, 0.f, 0.f, 0.f}, gOpacity = 0.f;
  float gColour[3] = {0.f, 0.f, 0.f}, dir[3] = {0.f, 0.f, 0.f}, gPv[3] = {0.f, 0.f, 0.f}, distance = 1.0f;
  if (touched) {
    const float4 col = splats[i].colorRadius;
    if (args.statistics) {
      float4 *st = reinterpret_cast<float4 *>(densifyStats + (size_t)i * kStatStride);
      float4 sa = st[0], sb = st[1];
      const float hx = 0.5f * cam.widthF, hy = 0.5f * cam.heightF;
      const float ax = raw[1] * hx, ay = raw[2] * hy;
      sa.x += sqrtf(fmaf(ay, ay, ax * ax));
      sa.y += 1.0f;
      sa.z = fmaxf(sa.z, col.w);
      sa.w += raw[9] * 3.0f * cam.widthF * cam.heightF;
      const float bx = raw[10] * hx, by = raw[11] * hy;
      sb.x += sqrtf(fmaf(by, by, bx * bx));
      st[0] = sa;
      st[1] = sb;
    }
    chain_view(cam, raw, col, pos, logScale, opacity, rq, gPv, gScale, gRot, gOpacity, gColour, dir, distance);
  }

  if (!bulk_wait(&s_bar, 0, kStageSpinLimit)) {
    // Never leave with a copy still landing in this block's shared memory.
    atomicOr(error, kErrLookbackTimeout);
    bulk_wait(&s_bar, 0, kStageSpinLimit);
  }
  const bool stepZeros = !args.selective;
  const int active = touched ? cam.activeCoeffs : 0;
  // The direction term, unrolled (its basis gradients fold per coefficient),
  // from the staged coefficients before any step.
  if (touched && cam.activeDegree > 0) {
    float gDir[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 1; k < kMaxCoeffs; ++k) {
      if (k >= active) break;
      const uint32_t r = (uint32_t)(k - 1) * 3u;
      const float value[3] = {staged_sh_rest<S>(s_rest, tid * p.restStride + r),
                              staged_sh_rest<S>(s_rest, tid * p.restStride + r + 1u),
                              staged_sh_rest<S>(s_rest, tid * p.restStride + r + 2u)};
      direction_term(k, value, gColour, dir, gDir);
    }
    add_direction_term(gDir, dir, distance, gPv);
  }
  if (touched) {
#pragma unroll
    for (int c = 0; c < 3; ++c) gP[c] += gPv[c];
  }
  // The penalties (3DGS-MCMC) apply to every Gaussian, seen or not.
  if (args.opacityReg > 0.0f || args.scaleReg > 0.0f) {
#pragma unroll
    for (int c = 0; c < 3; ++c) gScale[c] += args.scaleReg * splat_expf(logScale[c]);
    gOpacity += args.opacityReg * opacity * (1.0f - opacity);
  }

  // Adam on the 11 geometry elements: [positions 3 | scales 3 | rotations 4 |
  // opacity 1], before the SH step so that none of it stays live through the
  // SH loop.
  {
    float gv[11], value[11], m[11], vv[11];
    uint32_t word[11];
#pragma unroll
    for (int e = 0; e < 11; ++e) {
      const int group = e < 3 ? 0 : e < 6 ? 1 : e < 10 ? 2 : 3;
      const int a0 = e < 3 ? e : e < 6 ? e - 3 : e < 10 ? e - 6 : 0;
      const uint32_t per = group == 2 ? 4u : group == 3 ? 1u : 3u;
      const uint32_t idx = i * per + (uint32_t)a0;
      gv[e] = group == 0 ? gP[a0] : group == 1 ? gScale[a0] : group == 2 ? gRot[a0] : gOpacity;
      value[e] = group == 0 ? pos[a0] : group == 1 ? logScale[a0] : group == 3 ? rawOpacity
               : a0 == 0 ? rq.x : a0 == 1 ? rq.y : a0 == 2 ? rq.z : rq.w;
      m[e] = vv[e] = 0.0f;
      word[e] = 0u;
      if (gv[e] == 0.0f && args.selective) continue;
      load_state(state.state[group], ST, per * n, idx, m[e], vv[e], word[e]);
    }
#pragma unroll
    for (int e = 0; e < 11; ++e) {
      const int group = e < 3 ? 0 : e < 6 ? 1 : e < 10 ? 2 : 3;
      const int a0 = e < 3 ? e : e < 6 ? e - 3 : e < 10 ? e - 6 : 0;
      const uint32_t per = group == 2 ? 4u : group == 3 ? 1u : 3u;
      const uint32_t idx = i * per + (uint32_t)a0;
      // A parameter with a zero gradient is left alone when selective.
      if (gv[e] == 0.0f && args.selective) continue;
      adam(value[e], m[e], vv[e], gv[e], args.rates[group], a);
      store_state(state.state[group], ST, per * n, idx, m[e], vv[e], word[e], idx * 5u + (uint32_t)group, a.seed);
      float *values = group == 0 ? p.positions : group == 1 ? p.scales : group == 2 ? p.rotations : p.opacities;
      values[idx] = value[e];
    }
  }

  // The SH step from the staged planes: the DC planes, then one coefficient of
  // the rest per trip of a rolled loop (unrolled, the step's code overflows
  // the instruction cache).
  if (!(touched || stepZeros)) return;
  const uint32_t shFloats = 3u * (uint32_t)p.shCoeffs;
  const uint32_t hashBase = i * shFloats * 5u + 4u;
  // The staged rows: this thread's row at tid * stateStride (F32: the v rows
  // after the block's m rows).
  const uint32_t stateStride = sh_state_stride(p.shCoeffs);
  const float *s_statef = reinterpret_cast<const float *>(s_state) + (size_t)tid * stateStride;
  const uint32_t *s_statew = reinterpret_cast<const uint32_t *>(s_statef);
  uint32_t *stateOut = static_cast<uint32_t *>(state.state[4]) + sh_state_at(i, 0u, stateStride);
  const size_t stateCount = (size_t)ps * stateStride; // F32: the v rows follow the m rows
  // One element: Adam from the staged state, the new state and value returned.
  auto element = [&](uint32_t plane, float &val, float g, float rate) {
    if constexpr (ST == StateStore::F32) {
      float m = s_statef[plane], v = s_statef[(size_t)kStepThreads * stateStride + plane];
      adam(val, m, v, g, rate, a);
      reinterpret_cast<float *>(stateOut)[plane] = m;
      reinterpret_cast<float *>(stateOut)[stateCount + plane] = v;
    } else {
      const uint32_t word = s_statew[plane];
      float m = bf16_load(word, 0), v = bf16_load(word, 1);
      adam(val, m, v, g, rate, a);
      stateOut[plane] = bf16_pair(m, v, hashBase + plane * 5u, a.seed);
    }
  };
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float g = active > 0 ? fmaf(basis_one(0, dir[0], dir[1], dir[2]), gColour[c], 0.0f) : 0.0f;
    if (g == 0.0f && !stepZeros) continue;
    float val = s_dc[c * kStepThreads + tid];
    element((uint32_t)c, val, g, args.rates[4]);
    p.shDc[(size_t)c * ps + i] = val;
  }
  const float restRate = args.rates[4] * args.restScale;
#pragma unroll 1
  for (int k = 1; k < p.shCoeffs; ++k) {
    const float b = k < active ? basis_one(k, dir[0], dir[1], dir[2]) : 0.0f;
    const uint32_t r = (uint32_t)(k - 1) * 3u;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float g = k < active ? fmaf(b, gColour[c], 0.0f) : 0.0f;
      if (g == 0.0f && !stepZeros) continue;
      const uint32_t plane = r + 3u + (uint32_t)c;
      float val = staged_sh_rest<S>(s_rest, tid * p.restStride + r + (uint32_t)c);
      element(plane, val, g, restRate);
      store_sh_rest<S>(p.shRest, sh_rest_at(i, r + (uint32_t)c, p.restStride), val, hashBase + plane * 5u, args.seed);
    }
  }
}

// Selective Adam with no penalty leaves a Gaussian the view did not reach
// (every backward sum zero) exactly as it was, and behind the front layers of
// a scene most Gaussians are not reached: one thread per Gaussian would run
// the chain rule and the step with a few lanes of each warp. So each block of
// k_chain_reached first lists the reached Gaussians of its chunk of
// kReachChunk in shared memory, then its threads step that list, full warps.
// The list's order (warp-aggregated appends) varies from run to run and does
// not matter: a Gaussian's step reads and writes its own values only, with
// its own hash indices, so the results are those of k_chain_step, bit for bit.
constexpr uint32_t kTouchedThreads = 128;
constexpr uint32_t kReachChunk = 2048;

// Whether Gaussian i's backward sums hold anything, as k_chain_step's test
// raw[k] != 0.0f: an integer sum is non-zero exactly when its value is; a
// float sum of -0 (only its sign bit set) counts as zero.
template <bool FIXED> __device__ __forceinline__ uint32_t reached_bits(const void *rawIn, uint32_t i) {
  const uint4 *r4 = reinterpret_cast<const uint4 *>(rawIn) + (size_t)i * (kRawStride / 4);
  const uint4 a = r4[0], b = r4[1], c = r4[2], d = r4[3];
  const uint32_t keep = FIXED ? 0xFFFFFFFFu : 0x7FFFFFFFu;
  static_assert(kRawPerSplat == 14, "the last word read is sum 13");
  return ((a.x | a.y | a.z | a.w | b.x | b.y | b.z | b.w) & keep) | ((c.x | c.y | c.z | c.w) & keep) | ((d.x | d.y) & keep);
}

// A Gaussian's row of higher SH coefficients in registers: up to 48 elements
// (degree 3) in 16-byte pieces. get() reads element e; set() writes it as
// the store of the SH step does (stochastic rounding to 16-bit types, the
// reference's rule, with the element's hash index).
template <ShStore S> struct ShRow {
  static constexpr uint32_t kBytes = S == ShStore::F32 ? 4u : 2u;
  static constexpr int kPieces = (int)(48u * kBytes / 16u);
  uint4 piece[kPieces];
  __device__ __forceinline__ uint32_t &word(int w) { return reinterpret_cast<uint32_t *>(piece)[w]; }
  __device__ __forceinline__ float get(int e) {
    if constexpr (S == ShStore::F32) {
      return __uint_as_float(word(e));
    } else {
      const uint32_t half = (e & 1) != 0 ? word(e >> 1) >> 16 : word(e >> 1) & 0xFFFFu;
      if constexpr (S == ShStore::BF16) return __uint_as_float(half << 16);
      else return __half2float(__ushort_as_half((unsigned short)half));
    }
  }
  __device__ __forceinline__ void set(int e, float value, uint32_t hashIndex, uint32_t seed) {
    if constexpr (S == ShStore::F32) {
      word(e) = __float_as_uint(value);
    } else {
      uint32_t bits;
      if constexpr (S == ShStore::BF16) bits = bf16_stochastic(value, hashIndex, seed ^ 0x5DEECE66u) & 0xFFFFu;
      else bits = __half_as_ushort(half_stochastic(value, hashIndex, seed ^ 0x5DEECE66u));
      uint32_t &w = word(e >> 1);
      w = (e & 1) != 0 ? (w & 0x0000FFFFu) | (bits << 16) : (w & 0xFFFF0000u) | bits;
    }
  }
};

// The one-view selective step of a reached Gaussian. Its loads are issued up
// front: the row of backward sums, the DC coefficients (three planes) and the
// row of higher coefficients (16-byte pieces, predicated on the degree in
// use, no branch between them); the SH Adam state row goes in batches of 16
// words. A handful of memory latencies per Gaussian instead of one per
// coefficient. Element by element the arithmetic, hash indices and order of
// sums are k_chain_step's.
template <ShStore S, StateStore ST, bool FIXED>
__device__ __forceinline__ void step_reached(uint32_t i, const Params &p, const ViewParams &cam, const ChainArgs &args,
                                             const AdamArgs &a, int active, const void *__restrict__ rawIn,
                                             const Splat *__restrict__ splats, const OptimState &state,
                                             float *__restrict__ densifyStats) {
  const uint32_t n = p.n, ps = p.planeStride;
  const float pos[3] = {p.positions[i * 3], p.positions[i * 3 + 1], p.positions[i * 3 + 2]};
  const float logScale[3] = {p.scales[i * 3], p.scales[i * 3 + 1], p.scales[i * 3 + 2]};
  const float rawOpacity = p.opacities[i];
  const float4 rq = reinterpret_cast<const float4 *>(p.rotations)[i];
  const float4 col = splats[i].colorRadius;
  uint32_t words[16];
  {
    const uint4 *r4 = reinterpret_cast<const uint4 *>(rawIn) + (size_t)i * (kRawStride / 4);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint4 w4 = r4[q];
      words[q * 4] = w4.x;
      words[q * 4 + 1] = w4.y;
      words[q * 4 + 2] = w4.z;
      words[q * 4 + 3] = w4.w;
    }
  }
  // The coefficients: the DC planes and the Gaussian's row of the rest, the
  // row moved in 16-byte pieces (kept in registers for the step, written back
  // whole).
  float dc[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) dc[c] = active > 0 ? p.shDc[(size_t)c * ps + i] : 0.0f;
  ShRow<S> row;
  uint4 *rowAt = reinterpret_cast<uint4 *>(static_cast<unsigned char *>(p.shRest) + (size_t)i * p.restStride * ShRow<S>::kBytes);
  const uint32_t pieces = active > 1 ? p.restStride * ShRow<S>::kBytes / 16u : 0u;
#pragma unroll
  for (int q = 0; q < ShRow<S>::kPieces; ++q) row.piece[q] = (uint32_t)q < pieces ? rowAt[q] : make_uint4(0u, 0u, 0u, 0u);
  float raw[kRawPerSplat];
#pragma unroll
  for (int k = 0; k < kRawPerSplat; ++k) raw[k] = FIXED ? (float)(int)words[k] / cam.fixedScale : __uint_as_float(words[k]);
  const float opacity = 1.0f / (1.0f + splat_expf(-rawOpacity));
  float gP[3] = {0.f, 0.f, 0.f}, gScale[3] = {0.f, 0.f, 0.f}, gRot[4] = {0.f, 0.f, 0.f, 0.f}, gOpacity = 0.f;
  float gColour[3] = {0.f, 0.f, 0.f}, dir[3] = {0.f, 0.f, 0.f}, gPv[3] = {0.f, 0.f, 0.f}, distance = 1.0f;
  if (args.statistics) {
    float4 *stats = reinterpret_cast<float4 *>(densifyStats + (size_t)i * kStatStride);
    float4 sa = stats[0], sb = stats[1];
    const float hx = 0.5f * cam.widthF, hy = 0.5f * cam.heightF;
    const float ax = raw[1] * hx, ay = raw[2] * hy;
    sa.x += sqrtf(fmaf(ay, ay, ax * ax));
    sa.y += 1.0f;
    sa.z = fmaxf(sa.z, col.w);
    sa.w += raw[9] * 3.0f * cam.widthF * cam.heightF;
    const float bx = raw[10] * hx, by = raw[11] * hy;
    sb.x += sqrtf(fmaf(by, by, bx * bx));
    stats[0] = sa;
    stats[1] = sb;
  }
  chain_view(cam, raw, col, pos, logScale, opacity, rq, gPv, gScale, gRot, gOpacity, gColour, dir, distance);
  if (cam.activeDegree > 0) {
    float gDir[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int k = 1; k < kMaxCoeffs; ++k) {
      if (k < active) {
        const float value[3] = {row.get((k - 1) * 3), row.get((k - 1) * 3 + 1), row.get((k - 1) * 3 + 2)};
        direction_term(k, value, gColour, dir, gDir);
      }
    }
    add_direction_term(gDir, dir, distance, gPv);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) gP[c] += gPv[c];

  // Adam on the 11 geometry elements, as k_chain_step (selective: an
  // element with a zero gradient is left alone).
  {
    float gv[11], value[11], m[11], vv[11];
    uint32_t word[11];
#pragma unroll
    for (int e = 0; e < 11; ++e) {
      const int group = e < 3 ? 0 : e < 6 ? 1 : e < 10 ? 2 : 3;
      const int a0 = e < 3 ? e : e < 6 ? e - 3 : e < 10 ? e - 6 : 0;
      const uint32_t per = group == 2 ? 4u : group == 3 ? 1u : 3u;
      const uint32_t idx = i * per + (uint32_t)a0;
      gv[e] = group == 0 ? gP[a0] : group == 1 ? gScale[a0] : group == 2 ? gRot[a0] : gOpacity;
      value[e] = group == 0 ? pos[a0] : group == 1 ? logScale[a0] : group == 3 ? rawOpacity
               : a0 == 0 ? rq.x : a0 == 1 ? rq.y : a0 == 2 ? rq.z : rq.w;
      m[e] = vv[e] = 0.0f;
      word[e] = 0u;
      if (gv[e] == 0.0f) continue;
      load_state(state.state[group], ST, per * n, idx, m[e], vv[e], word[e]);
    }
#pragma unroll
    for (int e = 0; e < 11; ++e) {
      const int group = e < 3 ? 0 : e < 6 ? 1 : e < 10 ? 2 : 3;
      const int a0 = e < 3 ? e : e < 6 ? e - 3 : e < 10 ? e - 6 : 0;
      const uint32_t per = group == 2 ? 4u : group == 3 ? 1u : 3u;
      const uint32_t idx = i * per + (uint32_t)a0;
      if (gv[e] == 0.0f) continue;
      adam(value[e], m[e], vv[e], gv[e], args.rates[group], a);
      store_state(state.state[group], ST, per * n, idx, m[e], vv[e], word[e], idx * 5u + (uint32_t)group, a.seed);
      float *values = group == 0 ? p.positions : group == 1 ? p.scales : group == 2 ? p.rotations : p.opacities;
      values[idx] = value[e];
    }
  }

  // The SH step: only the coefficients in use have a gradient. The state row
  // goes in batches of 16 words (16-byte loads and stores); each element in
  // use is stepped in the reference's order, the values in the row kept in
  // registers, and the batch and then the row are written back whole.
  const uint32_t shFloats = 3u * (uint32_t)p.shCoeffs;
  const uint32_t hashBase = i * shFloats * 5u + 4u;
  const uint32_t stateStride = sh_state_stride(p.shCoeffs);
  uint4 *stateRow = reinterpret_cast<uint4 *>(static_cast<uint32_t *>(state.state[4]) + sh_state_at(i, 0u, stateStride));
  const size_t vRows = (size_t)ps * stateStride / 4u; // F32: the v rows, in 16-byte pieces, after the m rows
  const float restRate = args.rates[4] * args.restScale;
  float basis[kMaxCoeffs];
#pragma unroll
  for (int k = 0; k < kMaxCoeffs; ++k) basis[k] = k < active ? basis_one(k, dir[0], dir[1], dir[2]) : 0.0f;
  const uint32_t inUse = 3u * (uint32_t)active;
  bool dcChanged[3] = {false, false, false};
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    if ((uint32_t)b * 16u >= inUse) break;
    // Pieces past the row's end (a lower degree) are not touched.
    const uint32_t rowPieces = stateStride / 4u;
    uint4 m4[4], v4[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t at = (uint32_t)b * 4u + (uint32_t)q;
      m4[q] = at < rowPieces ? stateRow[at] : make_uint4(0u, 0u, 0u, 0u);
      if constexpr (ST == StateStore::F32) v4[q] = at < rowPieces ? stateRow[vRows + at] : make_uint4(0u, 0u, 0u, 0u);
    }
    uint32_t *mw = reinterpret_cast<uint32_t *>(m4), *vw = reinterpret_cast<uint32_t *>(v4);
#pragma unroll
    for (int w = 0; w < 16; ++w) {
      const int e = b * 16 + w, k = e / 3, c = e % 3;
      if (k >= kMaxCoeffs || (uint32_t)e >= inUse) continue;
      const float g = fmaf(basis[k], gColour[c], 0.0f);
      if (g == 0.0f) continue;
      float val = k == 0 ? dc[c] : row.get(e - 3);
      float m, v;
      if constexpr (ST == StateStore::F32) {
        m = __uint_as_float(mw[w]);
        v = __uint_as_float(vw[w]);
      } else {
        m = bf16_load(mw[w], 0);
        v = bf16_load(mw[w], 1);
      }
      adam(val, m, v, g, k == 0 ? args.rates[4] : restRate, a);
      if constexpr (ST == StateStore::F32) {
        mw[w] = __float_as_uint(m);
        vw[w] = __float_as_uint(v);
      } else {
        mw[w] = bf16_pair(m, v, hashBase + (uint32_t)e * 5u, a.seed);
      }
      if (k == 0) {
        dc[c] = val;
        dcChanged[c] = true;
      } else {
        row.set(e - 3, val, hashBase + (uint32_t)e * 5u, args.seed);
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t at = (uint32_t)b * 4u + (uint32_t)q;
      if (at < rowPieces) {
        stateRow[at] = m4[q];
        if constexpr (ST == StateStore::F32) stateRow[vRows + at] = v4[q];
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
    if (dcChanged[c]) p.shDc[(size_t)c * ps + i] = dc[c];
#pragma unroll
  for (int q = 0; q < ShRow<S>::kPieces; ++q)
    if ((uint32_t)q < pieces) rowAt[q] = row.piece[q];
}

template <ShStore S, StateStore ST, bool FIXED>
__global__ void __launch_bounds__(kTouchedThreads, 4) k_chain_reached(Params p, const ViewSet *__restrict__ viewsPtr,
                                                                      const void *__restrict__ rawIn,
                                                                      const Splat *__restrict__ splats,
                                                                      const ChainArgs *__restrict__ argsPtr, OptimState state,
                                                                      float *__restrict__ densifyStats, const uint32_t *error) {
  chain_enter();
  __shared__ uint32_t s_list[kReachChunk];
  __shared__ uint32_t s_count;
  if (error != nullptr && (*error & kErrEntryOverflow) != 0u) return;
  const uint32_t tid = threadIdx.x, lane = tid & 31u;
  const uint32_t first = blockIdx.x * kReachChunk, n = p.n;
  if (tid == 0) s_count = 0u;
  __syncthreads();
  // The chunk's reached Gaussians, four loads of sums in flight per thread.
  for (uint32_t r = 0; r < kReachChunk; r += 4 * kTouchedThreads) {
    uint32_t bits[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t g = first + r + (uint32_t)q * kTouchedThreads + tid;
      bits[q] = g < n ? reached_bits<FIXED>(rawIn, g) : 0u;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t g = first + r + (uint32_t)q * kTouchedThreads + tid;
      const uint32_t mask = __ballot_sync(0xFFFFFFFFu, bits[q] != 0u);
      if (mask == 0u) continue;
      uint32_t base = 0;
      if (lane == (uint32_t)(__ffs(mask) - 1)) base = atomicAdd(&s_count, (uint32_t)__popc(mask));
      base = __shfl_sync(0xFFFFFFFFu, base, __ffs(mask) - 1);
      if (bits[q] != 0u) s_list[base + __popc(mask & ((1u << lane) - 1u))] = g;
    }
  }
  __syncthreads();
  const uint32_t count = s_count;
  const ViewParams &cam = viewsPtr->v[0];
  const ChainArgs args = *argsPtr;
  const AdamArgs a = adam_args(args);
  const int active = min(cam.activeCoeffs, p.shCoeffs);
  for (uint32_t j = tid; j < count; j += kTouchedThreads)
    step_reached<S, ST, FIXED>(s_list[j], p, cam, args, a, active, rawIn, splats, state, densifyStats);
}

// train_score.comp: to each Gaussian's statistics, the marked pixels it
// reached (raw value 12, in pixels), that count times the view's loss, and its
// edge score (raw value 13, in pixels).
__global__ void __launch_bounds__(256) k_score(const void *__restrict__ rawIn, bool fixedPoint, float fixedScale, uint32_t n,
                                               float toPixels, float loss, float *__restrict__ densifyStats) {
  chain_enter();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t *words = static_cast<const uint32_t *>(rawIn) + (size_t)i * kRawStride;
  const float marked = fixedPoint ? (float)(int)words[12] / fixedScale : __uint_as_float(words[12]);
  const float edge = fixedPoint ? (float)(int)words[13] / fixedScale : __uint_as_float(words[13]);
  float *st = densifyStats + (size_t)i * kStatStride;
  const float pixels = marked * toPixels;
  st[5] += pixels;
  st[6] += pixels * loss;
  st[7] += edge * toPixels;
}

template <ShStore S>
void launch_chain_s(const Params &p, const ViewSet &views, const ViewSet *dViews, const void *raw, const Splat *splats, const ChainArgs &args,
                    const ChainArgs *dArgs, OptimState &state, const GradientsOut *grads, float4 *shGrad, float *densifyStats,
                    uint32_t *error, cudaStream_t stream) {
  const GradientsOut g = *grads;
  const bool store = args.mode == ChainMode::Gradients;
  const uint32_t blocks = div_up(p.n, 128);
  const bool multi = views.count > 1;
  // The fused form indexes the F32 SH state (m and v rows of 48 floats a Gaussian) in 32 bits.
  if (!multi && !args.splitStep && args.mode == ChainMode::Step && (size_t)p.planeStride * 3 * kMaxCoeffs * 2 < (size_t{1} << 32)) {
    if (args.selective && args.opacityReg == 0.0f && args.scaleReg == 0.0f) {
      // Only the reached Gaussians change: each block lists its chunk's, then steps them.
#define SB_REACHED(ST, FIX)                                                                                           \
  launch_chained(k_chain_reached<S, ST, FIX>, dim3(div_up(p.n, kReachChunk)), dim3(kTouchedThreads), 0, stream, p,    \
                 dViews, raw, splats, dArgs, state, densifyStats, (const uint32_t *)error)
      const bool f32 = state.store == StateStore::F32;
      if (args.fixedPoint) {
        if (f32) SB_REACHED(StateStore::F32, true);
        else SB_REACHED(StateStore::BF16Pair, true);
      } else {
        if (f32) SB_REACHED(StateStore::F32, false);
        else SB_REACHED(StateStore::BF16Pair, false);
      }
#undef SB_REACHED
      return;
    }
    const uint32_t smem = step_stage_bytes(p.shCoeffs, S == ShStore::F32 ? 4 : 2, state.store == StateStore::F32, p.restStride);
    const uint32_t stepBlocks = div_up(p.n, kStepThreads);
#define SB_STEP(ST, FIX)                                                                                           \
  {                                                                                                                  \
    cudaFuncSetAttribute(k_chain_step<S, ST, FIX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);           \
    launch_chained(k_chain_step<S, ST, FIX>, dim3(stepBlocks), dim3(kStepThreads), smem, stream, p, dViews, raw, splats, dArgs, state, densifyStats, \
                                                                        error);                                      \
  }
    const bool f32 = state.store == StateStore::F32;
    if (args.fixedPoint) {
      if (f32) SB_STEP(StateStore::F32, true) else SB_STEP(StateStore::BF16Pair, true)
    } else {
      if (f32) SB_STEP(StateStore::F32, false) else SB_STEP(StateStore::BF16Pair, false)
    }
#undef SB_STEP
    return;
  }
#define SB_CHAIN(F, M) \
  launch_chained(k_chain<S, F, M>, dim3(blocks), dim3(128), 0, stream, p, dViews, raw, splats, dArgs, state, g, store, shGrad, densifyStats, error)
  if (args.fixedPoint) {
    if (multi) SB_CHAIN(true, true);
    else SB_CHAIN(true, false);
  } else {
    if (multi) SB_CHAIN(false, true);
    else SB_CHAIN(false, false);
  }
#undef SB_CHAIN
  if (args.mode == ChainMode::Statistics) return;
  if (!store) launch_chained(k_adam_geometry, dim3((uint32_t)((11 * (size_t)p.n + 255) / 256)), dim3(256), 0, stream, p, dArgs, state, g, error);
  const dim3 shGrid(div_up(p.n, 256), div_up(p.shCoeffs, kShGroup));
  if (multi) launch_chained(k_sh_step<S, true>, dim3(shGrid), dim3(256), 0, stream, p, dViews, shGrad, dArgs, state, g, store, error);
  else launch_chained(k_sh_step<S, false>, dim3(shGrid), dim3(256), 0, stream, p, dViews, shGrad, dArgs, state, g, store, error);
}

} // namespace

void launch_score(const void *raw, bool fixedPoint, float fixedScale, uint32_t n, float toPixels, float loss, float *densifyStats,
                  cudaStream_t stream) {
  if (n == 0) return;
  launch_chained(k_score, dim3(div_up(n, 256)), dim3(256), 0, stream, raw, fixedPoint, fixedScale, n, toPixels, loss, densifyStats);
}

void launch_chain(const Params &p, const ViewSet &views, const ViewSet *dViews, const void *raw, const Splat *splats, const ChainArgs &args,
                  const ChainArgs *dArgs, OptimState &state, const GradientsOut *grads, float4 *shGrad, float *densifyStats,
                  uint32_t *error, cudaStream_t stream) {
  if (p.n == 0) return;
  switch (p.shStore) {
  case ShStore::BF16:
    launch_chain_s<ShStore::BF16>(p, views, dViews, raw, splats, args, dArgs, state, grads, shGrad, densifyStats, error, stream);
    break;
  case ShStore::F16:
    launch_chain_s<ShStore::F16>(p, views, dViews, raw, splats, args, dArgs, state, grads, shGrad, densifyStats, error, stream);
    break;
  default:
    launch_chain_s<ShStore::F32>(p, views, dViews, raw, splats, args, dArgs, state, grads, shGrad, densifyStats, error, stream);
    break;
  }
}

} // namespace sb
