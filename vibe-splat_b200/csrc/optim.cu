// The chain rule from the backward pass's screen-space sums to the raw
// parameters, and what becomes of the result: densification statistics only,
// gradients stored, or Adam's step. Restates shaders/train_gradient.comp
// :105-315 (chain), :94-101 (add_statistics), :57-76 (EMITTER),
// shaders/train_step.glsl:119-130 (step_parameter), shaders/bf16.glsl:6-27 and
// shaders/train_sh_step.comp:19-70 (the SH step, with half_stochastic,
// train_step.glsl:140-150).
//
// One thread per Gaussian does all of it, the SH step included: SH lives in
// planes (coefficient-major), so neighbouring threads touch neighbouring words
// for every coefficient, which is what the reference's separate one-thread-
// per-word SH pass was for. With several views in a batch, the chain rule runs
// per view and the gradients are summed before one step.
// Out of scope and rejected by the host: the Mip 2D filter, the 3D filter,
// SH dropout, second-order steps, pose gradients, position noise.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "kernels.cuh"
#include "shmath.cuh"

namespace sb {

namespace {

constexpr int kMaxCoeffs = 16;

__device__ __forceinline__ float bf16_load(uint32_t word, int slot) {
  return __uint_as_float(slot == 0 ? word << 16 : word & 0xFFFF0000u);
}
__device__ __forceinline__ uint32_t bf16_round(float x) {
  const uint32_t bits = __float_as_uint(x);
  return (bits + 0x7FFFu + ((bits >> 16) & 1u)) >> 16;
}
__device__ __forceinline__ uint32_t bf16_stochastic(float x, uint32_t index, uint32_t seed) {
  const uint32_t word = pcg_word(index, seed);
  return (__float_as_uint(x) + (((word >> 22u) ^ word) & 0xFFFFu)) >> 16;
}
__device__ __forceinline__ uint32_t bf16_store(uint32_t word, int slot, uint32_t bits) {
  return slot == 0 ? (word & 0xFFFF0000u) | bits : (word & 0xFFFFu) | (bits << 16);
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
  float beta1, beta2, epsilon, correction1, correction2;
  uint32_t seed;
};

// Adam on one parameter (step_parameter with radius < 0).
__device__ __forceinline__ void adam(float &value, float &m, float &v, float g, float rate, const AdamArgs &a) {
  m = a.beta1 * m + (1.0f - a.beta1) * g;
  v = a.beta2 * v + (1.0f - a.beta2) * g * g;
  value -= rate * (m / a.correction1) / (sqrtf(v / a.correction2) + a.epsilon);
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
    s[at] = bf16_store(bf16_store(word, 0, bf16_round(m)), 1, bf16_stochastic(v, hashIndex, a.seed));
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

template <ShStore S, bool FIXED>
__global__ void __launch_bounds__(128) k_chain(Params p, const ViewSet *__restrict__ viewsPtr, const void *__restrict__ rawIn,
                                               const Splat *__restrict__ splats, const ChainArgs *__restrict__ argsPtr, OptimState state,
                                               GradientsOut grads, bool storeGradients, float *__restrict__ densifyStats,
                                               const uint32_t *error) {
  const ViewSet &views = *viewsPtr;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  const ChainArgs args = *argsPtr;
  if (error != nullptr && (*error & kErrEntryOverflow) != 0u) return;
  const size_t n = p.n;
  const int shFloats = 3 * p.shCoeffs;
  const bool zeros = args.mode == ChainMode::Gradients || (args.mode == ChainMode::Step && !args.selective);
  const bool penalties = args.opacityReg > 0.0f || args.scaleReg > 0.0f;

  // Accumulated over views.
  float gP[3] = {0.f, 0.f, 0.f}, gScale[3] = {0.f, 0.f, 0.f}, gRot[4] = {0.f, 0.f, 0.f, 0.f}, gOpacity = 0.f;
  float gSh[kMaxCoeffs][3];
#pragma unroll
  for (int k = 0; k < kMaxCoeffs; ++k) gSh[k][0] = gSh[k][1] = gSh[k][2] = 0.f;
  bool anyTouched = false;
  int activeCoeffs = 0;

  const float logScale[3] = {p.scales[i * 3], p.scales[i * 3 + 1], p.scales[i * 3 + 2]};
  const float opacity = 1.0f / (1.0f + splat_expf(-p.opacities[i]));

  for (int v = 0; v < views.count; ++v) {
    const ViewParams &cam = views.v[v];
    const size_t at = ((size_t)v * n + i) * kRawStride;
    float raw[kRawPerSplat];
    bool touched = false;
#pragma unroll
    for (int k = 0; k < kRawPerSplat; ++k) {
      if (FIXED) {
        const int q = static_cast<const int *>(rawIn)[at + k];
        raw[k] = (float)q / cam.fixedScale;
        touched = touched || q != 0;
      } else {
        raw[k] = static_cast<const float *>(rawIn)[at + k];
        touched = touched || raw[k] != 0.0f;
      }
    }
    if (!touched) continue;
    anyTouched = true;
    if (args.statistics) {
      float *st = densifyStats + (size_t)i * kStatStride;
      const float hx = 0.5f * cam.widthF, hy = 0.5f * cam.heightF;
      const float ax = raw[1] * hx, ay = raw[2] * hy;
      st[0] += sqrtf(fmaf(ay, ay, ax * ax));
      st[1] += 1.0f;
      st[2] = fmaxf(st[2], splats[(size_t)v * n + i].colorRadius.w);
      st[3] += raw[9] * 3.0f * cam.widthF * cam.heightF;
      const float bx = raw[10] * hx, by = raw[11] * hy;
      st[4] += sqrtf(fmaf(by, by, bx * bx));
    }
    if (args.mode == ChainMode::Statistics) continue;

    const float px = p.positions[i * 3], py = p.positions[i * 3 + 1], pz = p.positions[i * 3 + 2];
    const float4 rq = reinterpret_cast<const float4 *>(p.rotations)[i];
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
    const float gCentre[2] = {raw[1], raw[2]};
    const float G[2][2] = {{raw[3], raw[4]}, {raw[4], raw[5]}};

    float Rv[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) Rv[r][c] = cam.R[r * 3 + c];
    float R[3][3];
    quat_to_matrix(q[0], q[1], q[2], q[3], R);
    const float s2[3] = {splat_expf(2.0f * logScale[0]), splat_expf(2.0f * logScale[1]), splat_expf(2.0f * logScale[2])};
    // sigma = R D R^T, X = Rv sigma Rv^T.
    float sigma[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        sigma[r][c] = fmaf(R[r][2] * s2[2], R[c][2], fmaf(R[r][1] * s2[1], R[c][1], R[r][0] * s2[0] * R[c][0]));
    float RS[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) RS[r][c] = fmaf(Rv[r][2], sigma[2][c], fmaf(Rv[r][1], sigma[1][c], Rv[r][0] * sigma[0][c]));
    float X[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) X[r][c] = fmaf(RS[r][2], Rv[c][2], fmaf(RS[r][1], Rv[c][1], RS[r][0] * Rv[c][0]));

    const float limX = 1.3f * cam.tanX, limY = 1.3f * cam.tanY;
    const float rx = t[0] * iz, ry = t[1] * iz;
    const bool clampedX = fabsf(rx) > limX, clampedY = fabsf(ry) > limY;
    const float tx = fminf(fmaxf(rx, -limX), limX) * z, ty = fminf(fmaxf(ry, -limY), limY) * z;
    const float J[2][3] = {{fx * iz, 0.f, -fx * tx * iz2}, {0.f, fy * iz, -fy * ty * iz2}};
    const float Jc[2][3] = {{fx * iz, 0.f, -fx * t[0] * iz2}, {0.f, fy * iz, -fy * t[1] * iz2}};
    float gT[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) gT[k] = fmaf(Jc[1][k], gCentre[1], Jc[0][k] * gCentre[0]);
    const float dJx[2][3] = {{0.f, 0.f, clampedX ? 0.0f : -fx * iz2}, {0.f, 0.f, 0.f}};
    const float dJy[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, clampedY ? 0.0f : -fy * iz2}};
    const float dJz[2][3] = {{-fx * iz2, 0.f, clampedX ? fx * tx * iz2 * iz : 2.0f * fx * tx * iz2 * iz},
                             {0.f, -fy * iz2, clampedY ? fy * ty * iz2 * iz : 2.0f * fy * ty * iz2 * iz}};
    gT[0] += 2.0f * trace_term(G, dJx, X, J);
    gT[1] += 2.0f * trace_term(G, dJy, X, J);
    gT[2] += 2.0f * trace_term(G, dJz, X, J);
    float gPv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) gPv[c] = fmaf(Rv[2][c], gT[2], fmaf(Rv[1][c], gT[1], Rv[0][c] * gT[0]));

    // T2 = J Rv (2x3), G3 = T2^T G T2.
    float T2[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) T2[r][c] = fmaf(J[r][2], Rv[2][c], fmaf(J[r][1], Rv[1][c], J[r][0] * Rv[0][c]));
    float GT[2][3];
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) GT[r][c] = fmaf(G[r][1], T2[1][c], G[r][0] * T2[0][c]);
    float G3[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) G3[a][b] = fmaf(T2[1][a], GT[1][b], T2[0][a] * GT[0][b]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float ax[3] = {R[0][a], R[1][a], R[2][a]};
      float Ga[3];
#pragma unroll
      for (int r = 0; r < 3; ++r) Ga[r] = fmaf(G3[r][2], ax[2], fmaf(G3[r][1], ax[1], G3[r][0] * ax[0]));
      gScale[a] += 2.0f * s2[a] * fmaf(ax[2], Ga[2], fmaf(ax[1], Ga[1], ax[0] * Ga[0]));
    }
    // Rotation: P = 2 G3 R D, gq_k = <P, dR/dq_k>.
    float P[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) P[r][c] = 2.0f * fmaf(G3[r][2], R[2][c], fmaf(G3[r][1], R[1][c], G3[r][0] * R[0][c])) * s2[c];
    const float w = q[0], x = q[1], y = q[2], zq = q[3];
    // dR/dq as rows (transposed from the GLSL column constructors).
    const float dR[4][3][3] = {
        {{0.f, -2.0f * zq, 2.0f * y}, {2.0f * zq, 0.f, -2.0f * x}, {-2.0f * y, 2.0f * x, 0.f}},
        {{0.f, 2.0f * y, 2.0f * zq}, {2.0f * y, -4.0f * x, -2.0f * w}, {2.0f * zq, 2.0f * w, -4.0f * x}},
        {{-4.0f * y, 2.0f * x, 2.0f * w}, {2.0f * x, 0.f, 2.0f * zq}, {-2.0f * w, 2.0f * zq, -4.0f * y}},
        {{-4.0f * zq, -2.0f * w, 2.0f * x}, {2.0f * w, -4.0f * zq, 2.0f * y}, {2.0f * x, 2.0f * y, 0.f}}};
    float gq[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float acc = 0.0f;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r) acc = fmaf(P[r][c], dR[k][r][c], acc);
      gq[k] = acc;
    }
    const float qg = fmaf(q[3], gq[3], fmaf(q[2], gq[2], fmaf(q[1], gq[1], q[0] * gq[0])));
    const float inv = fmaxf(quatLength, 1e-12f);
#pragma unroll
    for (int k = 0; k < 4; ++k) gRot[k] += (gq[k] - q[k] * qg) / inv;
    gOpacity += raw[0] * opacity * (1.0f - opacity);

    // Colour: the gradient reaches the coefficients in use where the colour
    // was not clamped at zero (the splat keeps the clamped colour).
    const float4 col = splats[(size_t)v * n + i].colorRadius;
    const float gColour[3] = {col.x > 0.0f ? raw[6] : 0.0f, col.y > 0.0f ? raw[7] : 0.0f, col.z > 0.0f ? raw[8] : 0.0f};
    const float ddx = px - cam.pos[0], ddy = py - cam.pos[1], ddz = pz - cam.pos[2];
    const float distance = sqrtf(fmaf(ddz, ddz, fmaf(ddy, ddy, ddx * ddx)));
    const float dir[3] = {ddx / distance, ddy / distance, ddz / distance};
    float basis[16];
    sh_basis(dir[0], dir[1], dir[2], cam.activeDegree, basis);
    activeCoeffs = max(activeCoeffs, cam.activeCoeffs);
#pragma unroll
    for (int k = 0; k < kMaxCoeffs; ++k) {
      if (k < cam.activeCoeffs) {
#pragma unroll
        for (int c = 0; c < 3; ++c) gSh[k][c] += basis[k] * gColour[c];
      }
    }
    // Position also changes the view direction, and with it the colour.
    if (cam.activeDegree > 0) {
      float bg[16][3];
      sh_basis_gradient(dir[0], dir[1], dir[2], cam.activeDegree, bg);
      float gDir[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int k = 1; k < kMaxCoeffs; ++k) {
        if (k < cam.activeCoeffs) {
          const float c0 = sh_coefficient<S>(p, i, k, 0), c1 = sh_coefficient<S>(p, i, k, 1), c2 = sh_coefficient<S>(p, i, k, 2);
          const float d = fmaf(gColour[2], c2, fmaf(gColour[1], c1, gColour[0] * c0));
#pragma unroll
          for (int c = 0; c < 3; ++c) gDir[c] = fmaf(d, bg[k][c], gDir[c]);
        }
      }
      const float dd = fmaf(dir[2], gDir[2], fmaf(dir[1], gDir[1], dir[0] * gDir[0]));
#pragma unroll
      for (int c = 0; c < 3; ++c) gPv[c] += (gDir[c] - dir[c] * dd) / distance;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) gP[c] += gPv[c];
  }

  if (args.mode == ChainMode::Statistics) return;
  if (!anyTouched && !zeros && !penalties) return;
  // The penalties (3DGS-MCMC) apply to every Gaussian, seen or not.
  if (penalties) {
#pragma unroll
    for (int a = 0; a < 3; ++a) gScale[a] += args.scaleReg * splat_expf(logScale[a]);
    gOpacity += args.opacityReg * opacity * (1.0f - opacity);
  }

  if (storeGradients) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      grads.g[0][i * 3 + a] = gP[a];
      grads.g[1][i * 3 + a] = gScale[a];
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) grads.g[2][i * 4 + a] = gRot[a];
    grads.g[3][i] = gOpacity;
    for (int k = 0; k < p.shCoeffs; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) grads.g[4][(size_t)i * shFloats + k * 3 + c] = k < kMaxCoeffs ? gSh[k][c] : 0.0f;
    return;
  }

  // Adam. A parameter with a zero gradient is left alone when selective.
  const AdamArgs a{args.beta1, args.beta2, args.epsilon, args.correction1, args.correction2, args.seed};
  const bool stepZeros = !args.selective;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (gP[c] != 0.0f || stepZeros) {
      float value = p.positions[i * 3 + c];
      step_state(value, state.state[0], state.store, n * 3, i * 3 + c, gP[c], args.rates[0], a, (i * 3 + c) * 5u + 0u);
      p.positions[i * 3 + c] = value;
    }
    if (gScale[c] != 0.0f || stepZeros) {
      float value = p.scales[i * 3 + c];
      step_state(value, state.state[1], state.store, n * 3, i * 3 + c, gScale[c], args.rates[1], a, (i * 3 + c) * 5u + 1u);
      p.scales[i * 3 + c] = value;
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    if (gRot[c] != 0.0f || stepZeros) {
      float value = p.rotations[i * 4 + c];
      step_state(value, state.state[2], state.store, n * 4, i * 4 + c, gRot[c], args.rates[2], a, (i * 4 + c) * 5u + 2u);
      p.rotations[i * 4 + c] = value;
    }
  }
  if (gOpacity != 0.0f || stepZeros) {
    float value = p.opacities[i];
    step_state(value, state.state[3], state.store, n, i, gOpacity, args.rates[3], a, i * 5u + 3u);
    p.opacities[i] = value;
  }
  // SH: planar element (k, c) of Gaussian i; GaussianCloud index i*shFloats + 3k + c.
  if (!anyTouched && !stepZeros) return;
  for (int k = 0; k < p.shCoeffs; ++k) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float g = (k < activeCoeffs && k < kMaxCoeffs) ? gSh[k][c] : 0.0f;
      if (g == 0.0f && !stepZeros) continue;
      const size_t plane = (size_t)(k * 3 + c) * n + i;
      const uint32_t hashIndex = ((uint32_t)(i * shFloats + k * 3 + c)) * 5u + 4u;
      const float rate = k == 0 ? args.rates[4] : args.rates[4] * args.restScale;
      if (k == 0) {
        float value = p.shDc[(size_t)c * n + i];
        step_state(value, state.state[4], state.store, n * shFloats, plane, g, rate, a, hashIndex);
        p.shDc[(size_t)c * n + i] = value;
      } else {
        const size_t idx = ((size_t)(k - 1) * 3 + c) * n + i;
        float value = load_sh_rest<S>(p.shRest, idx);
        step_state(value, state.state[4], state.store, n * shFloats, plane, g, rate, a, hashIndex);
        store_sh_rest<S>(p.shRest, idx, value, hashIndex, args.seed);
      }
    }
  }
}

template <ShStore S>
void launch_chain_s(const Params &p, const ViewSet &views, const ViewSet *dViews, const void *raw, const Splat *splats, const ChainArgs &args,
                    const ChainArgs *dArgs, OptimState &state, const GradientsOut *grads, float *densifyStats, const uint32_t *error,
                    cudaStream_t stream) {
  const GradientsOut g = grads != nullptr ? *grads : GradientsOut{};
  const bool store = grads != nullptr && args.mode == ChainMode::Gradients;
  const uint32_t blocks = div_up(p.n, 128);
  if (args.fixedPoint)
    k_chain<S, true><<<blocks, 128, 0, stream>>>(p, dViews, raw, splats, dArgs, state, g, store, densifyStats, error);
  else
    k_chain<S, false><<<blocks, 128, 0, stream>>>(p, dViews, raw, splats, dArgs, state, g, store, densifyStats, error);
}

} // namespace

void launch_chain(const Params &p, const ViewSet &views, const ViewSet *dViews, const void *raw, const Splat *splats, const ChainArgs &args,
                  const ChainArgs *dArgs, OptimState &state, const GradientsOut *grads, float *densifyStats, const uint32_t *error,
                  cudaStream_t stream) {
  if (p.n == 0) return;
  switch (p.shStore) {
  case ShStore::BF16:
    launch_chain_s<ShStore::BF16>(p, views, dViews, raw, splats, args, dArgs, state, grads, densifyStats, error, stream);
    break;
  case ShStore::F16:
    launch_chain_s<ShStore::F16>(p, views, dViews, raw, splats, args, dArgs, state, grads, densifyStats, error, stream);
    break;
  default:
    launch_chain_s<ShStore::F32>(p, views, dViews, raw, splats, args, dArgs, state, grads, densifyStats, error, stream);
    break;
  }
}

} // namespace sb
