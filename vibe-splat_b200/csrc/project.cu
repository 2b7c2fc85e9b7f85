// Preprocess: from raw trainable parameters to screen-space splats and depth
// keys, one thread per (Gaussian, view). Restates shaders/train_preprocess.comp
// :31-134 (the culling order, the EWA Jacobian with its 1.3 tan(fov/2) clamp,
// the 0.3 px dilation, the conic, the 3-sigma radius, the SH colour, the
// extent from 2 log(255 opacity) and the key 0xFFFFFFFF - bits(z)).
// FP32 rounding order: every product and sum is written out; fmaf is used only
// where it appears below, so the CPU restatement can reproduce each value.
#include <algorithm>

#include "bulk.cuh"
#include "kernels.cuh"
#include "shmath.cuh"

namespace sb {

namespace {

constexpr int kMaxShCoeffs = 16;
constexpr uint32_t kProjectThreads = 256;
// Polls of the SH staging barrier before the kernel gives up on it.
constexpr int kShSpinLimit = 1 << 22;

template <ShStore S> __host__ __device__ constexpr uint32_t sh_bytes() { return S == ShStore::F32 ? 4u : 2u; }

// Shared-memory bytes of a block's staged SH: 3 DC planes (FP32) and, when
// the view uses higher coefficients, the block's rows of them (restStride
// elements each), kProjectThreads Gaussians.
template <ShStore S> inline uint32_t project_stage_bytes(int coeffs, uint32_t restStride) {
  return kProjectThreads * (3u * 4u + (coeffs > 1 ? restStride * sh_bytes<S>() : 0u));
}

// A thread's staged row of higher coefficients, read from shared memory in
// 16-byte pieces (a row is a whole number of them); element e of it.
constexpr int kMaxRowPieces = 12; // 48 FP32 elements
template <ShStore S> struct StagedRow {
  uint4 piece[kMaxRowPieces];
  __device__ __forceinline__ float element(int e) const {
    const uint32_t *w = reinterpret_cast<const uint32_t *>(piece);
    if constexpr (S == ShStore::F32) return __uint_as_float(w[e]);
    const uint32_t half = (e & 1) != 0 ? w[e >> 1] >> 16 : w[e >> 1] & 0xFFFFu;
    if constexpr (S == ShStore::BF16) return __uint_as_float(half << 16);
    else return __half2float(__ushort_as_half((unsigned short)half));
  }
};

// The block's SH planes (those of the view's coefficients in use) arrive by
// bulk copies that thread 0 issues first, so they land while the projection
// and the culling tests run. Thread 0 waits for them before it leaves, culled
// or not, so no copy lands in a block that has gone.
template <ShStore S>
__global__ void __launch_bounds__(kProjectThreads, 3) k_preprocess(Params p, const ViewSet *__restrict__ viewsPtr,
                                                                Splat *__restrict__ splats, float *__restrict__ reachOut,
                                                                uint32_t *__restrict__ depthKeys, uint32_t *__restrict__ values,
                                                                uint32_t *error, int stageCoeffs) {
  chain_enter();
  extern __shared__ __align__(128) unsigned char s_stage[];
  __shared__ __align__(8) uint64_t s_bar;
  const ViewSet &views = *viewsPtr;
  const uint32_t tid = threadIdx.x, i0 = blockIdx.x * kProjectThreads, i = i0 + tid;
  const int v = blockIdx.y;
  const ViewParams &cam = views.v[v];
  // The stage holds stageCoeffs coefficients (the launch's shared memory); a
  // view using more is refused rather than staged past its end: its
  // Gaussians are written as culled, and the error word tells the host.
  if (cam.activeCoeffs > stageCoeffs) {
    if (tid == 0 && error != nullptr) atomicOr(error, kErrShStage);
    if (i < p.n) {
      depthKeys[(size_t)v * p.n + i] = kInvisible;
      reachOut[(size_t)v * p.n + i] = -INFINITY;
      if (values != nullptr) values[(size_t)v * p.n + i] = i;
    }
    return;
  }
  const int coeffs = cam.activeCoeffs;
  const uint32_t rowBytes = p.restStride * sh_bytes<S>();
  unsigned char *s_rest = s_stage + 3u * kProjectThreads * 4u;
  if (tid == 0) {
    bulk_barrier_init(&s_bar, 1);
    // The last block's planes and rows end at the plane stride (a multiple of 128).
    const uint32_t count = min(kProjectThreads, p.planeStride - i0);
    const uint32_t restBytes = coeffs > 1 ? count * rowBytes : 0u;
    bulk_expect(&s_bar, count * 3u * 4u + restBytes);
    for (uint32_t c = 0; c < 3u; ++c)
      bulk_load(s_stage + c * kProjectThreads * 4u, p.shDc + (size_t)c * p.planeStride + i0, count * 4u, &s_bar);
    if (restBytes > 0u)
      bulk_load(s_rest, static_cast<const unsigned char *>(p.shRest) + (size_t)i0 * rowBytes, restBytes, &s_bar);
  }
  __syncthreads();
  bool staged = false;
  const auto wait_stage = [&] {
    if (!bulk_wait(&s_bar, 0, kShSpinLimit)) {
      if (error != nullptr) atomicOr(error, kErrLookbackTimeout);
      bulk_wait(&s_bar, 0, kShSpinLimit);
    }
    staged = true;
  };
  if (i < p.n) [&] {
    const size_t at = (size_t)v * p.n + i;
    // Culled until shown otherwise: the key, and the reach (which the tile
    // count may read while the depth sort permutes the keys).
    depthKeys[at] = kInvisible;
    reachOut[at] = -INFINITY;
    if (values != nullptr) values[at] = i;

    // Every parameter load first, so that they are in flight together.
    const float px = p.positions[i * 3], py = p.positions[i * 3 + 1], pz = p.positions[i * 3 + 2];
    const float rawOpacity = p.opacities[i];
    const float4 rq = reinterpret_cast<const float4 *>(p.rotations)[i];
    const float rawScale[3] = {p.scales[i * 3], p.scales[i * 3 + 1], p.scales[i * 3 + 2]};
    const float tx = fmaf(cam.R[2], pz, fmaf(cam.R[1], py, fmaf(cam.R[0], px, cam.T[0])));
    const float ty = fmaf(cam.R[5], pz, fmaf(cam.R[4], py, fmaf(cam.R[3], px, cam.T[1])));
    const float tz = fmaf(cam.R[8], pz, fmaf(cam.R[7], py, fmaf(cam.R[6], px, cam.T[2])));
    // Written so that NaN fails, as in the reference.
    if (!(tz >= cam.nearPlane)) return;
    const float opacity = 1.0f / (1.0f + splat_expf(-rawOpacity));
    if (!(opacity >= kAlphaMin)) return;

    const float len = sqrtf(fmaf(rq.w, rq.w, fmaf(rq.z, rq.z, fmaf(rq.y, rq.y, rq.x * rq.x))));
    if (!(len >= kMinQuaternionLength)) return;
    const float qw = rq.x / len, qx = rq.y / len, qy = rq.z / len, qz = rq.w / len;
    const float s[3] = {splat_expf(rawScale[0]), splat_expf(rawScale[1]), splat_expf(rawScale[2])};
    float Rq[3][3];
    quat_to_matrix(qw, qx, qy, qz, Rq);
    // M = Rq diag(s); sigma = M M^T (no 3D filter).
    float M[3][3];
  #pragma unroll
    for (int r = 0; r < 3; ++r)
  #pragma unroll
      for (int c = 0; c < 3; ++c) M[r][c] = Rq[r][c] * s[c];
    float sigma[3][3];
  #pragma unroll
    for (int r = 0; r < 3; ++r)
  #pragma unroll
      for (int c = 0; c < 3; ++c) sigma[r][c] = fmaf(M[r][2], M[c][2], fmaf(M[r][1], M[c][1], M[r][0] * M[c][0]));
    // The 3D filter's opacity factor with no filter: 1, or NaN for a degenerate
    // scale (0/0, inf/inf), which culls it as the reference does.
    const float s2[3] = {s[0] * s[0], s[1] * s[1], s[2] * s[2]};
    const float k3 = sqrtf(s2[0] / (s2[0] + 0.0f) * (s2[1] / (s2[1] + 0.0f)) * (s2[2] / (s2[2] + 0.0f)));
    const float opacity3 = opacity * k3;
    if (!(opacity3 >= kAlphaMin)) return;

    const float limX = 1.3f * cam.tanX, limY = 1.3f * cam.tanY;
    const float txc = fminf(fmaxf(tx / tz, -limX), limX) * tz;
    const float tyc = fminf(fmaxf(ty / tz, -limY), limY) * tz;
    const float tz2 = tz * tz;
    const float j00 = cam.fx / tz, j11 = cam.fy / tz;
    const float j02 = (-cam.fx * txc) / tz2, j12 = (-cam.fy * tyc) / tz2;
    // Tm = J Rview (2x3).
    float Tm[2][3];
  #pragma unroll
    for (int c = 0; c < 3; ++c) {
      Tm[0][c] = fmaf(j02, cam.R[6 + c], j00 * cam.R[c]);
      Tm[1][c] = fmaf(j12, cam.R[6 + c], j11 * cam.R[3 + c]);
    }
    // cov = Tm sigma Tm^T.
    float U[3][2];
  #pragma unroll
    for (int k = 0; k < 3; ++k)
  #pragma unroll
      for (int r = 0; r < 2; ++r) U[k][r] = fmaf(sigma[k][2], Tm[r][2], fmaf(sigma[k][1], Tm[r][1], sigma[k][0] * Tm[r][0]));
    const float cov00 = fmaf(Tm[0][2], U[2][0], fmaf(Tm[0][1], U[1][0], Tm[0][0] * U[0][0]));
    const float cov01 = fmaf(Tm[0][2], U[2][1], fmaf(Tm[0][1], U[1][1], Tm[0][0] * U[0][1]));
    const float cov11 = fmaf(Tm[1][2], U[2][1], fmaf(Tm[1][1], U[1][1], Tm[1][0] * U[0][1]));

    const float a = cov00 + 0.3f, b = cov01, c = cov11 + 0.3f;
    const float det = a * c - b * b;
    if (!(det > kMinConicDeterminant)) return;
    const float mid = 0.5f * (a + c);
    const float lambda = mid + sqrtf(fmaxf(0.1f, mid * mid - det));
    const float radius = ceilf(3.0f * sqrtf(lambda));
    const float centerX = cam.fx * tx / tz + cam.cx, centerY = cam.fy * ty / tz + cam.cy;
    if (centerX + radius < 0.0f || centerY + radius < 0.0f || centerX - radius > cam.widthF || centerY - radius > cam.heightF) {
      return;
    }

    // SH colour (no dropout).
    const float dx = px - cam.pos[0], dy = py - cam.pos[1], dz = pz - cam.pos[2];
    const float dlen = sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
    float basis[16];
    sh_basis(dx / dlen, dy / dlen, dz / dlen, cam.activeDegree, basis);
    // Unrolled to the largest count so that the coefficients' loads are issued
    // together; the sums run in coefficient order as before.
    wait_stage();
    StagedRow<S> row;
    const uint4 *mine = reinterpret_cast<const uint4 *>(s_rest + (size_t)tid * rowBytes);
  #pragma unroll
    for (int q = 0; q < kMaxRowPieces; ++q) row.piece[q] = coeffs > 1 && (uint32_t)q * 16u < rowBytes ? mine[q] : make_uint4(0u, 0u, 0u, 0u);
    float coef[kMaxShCoeffs][3];
  #pragma unroll
    for (int ch = 0; ch < 3; ++ch) coef[0][ch] = reinterpret_cast<const float *>(s_stage)[ch * kProjectThreads + tid];
  #pragma unroll
    for (int k = 1; k < kMaxShCoeffs; ++k)
  #pragma unroll
      for (int ch = 0; ch < 3; ++ch) coef[k][ch] = k < coeffs ? row.element((k - 1) * 3 + ch) : 0.0f;
    float col[3] = {0.5f, 0.5f, 0.5f};
  #pragma unroll
    for (int k = 0; k < kMaxShCoeffs; ++k) {
      if (k >= cam.activeCoeffs) break;
  #pragma unroll
      for (int ch = 0; ch < 3; ++ch) col[ch] = fmaf(basis[k], coef[k][ch], col[ch]);
    }
    if (!(fabsf(col[0]) < 1e30f && fabsf(col[1]) < 1e30f && fabsf(col[2]) < 1e30f)) return;

    const float reach = 2.0f * splat_logf(255.0f * opacity3);
    Splat out;
    out.conicOpacity = make_float4(c / det, -b / det, a / det, opacity3);
    out.colorRadius = make_float4(fmaxf(col[0], 0.0f), fmaxf(col[1], 0.0f), fmaxf(col[2], 0.0f), radius);
    out.centerExtent = make_float4(centerX, centerY, fminf(sqrtf(reach * a), radius), fminf(sqrtf(reach * c), radius));
    splats[at] = out;
    reachOut[at] = reach;
    depthKeys[at] = 0xFFFFFFFFu - __float_as_uint(tz);
  }();
  if (tid == 0 && !staged) wait_stage();
}

template <ShStore S>
void launch_preprocess_s(const Params &p, const ViewSet &views, const ViewSet *dViews, Splat *splats, float *reach,
                         uint32_t *depthKeys, uint32_t *values, uint32_t *error, cudaStream_t stream) {
  int coeffs = 1;
  for (int k = 0; k < views.count; ++k) coeffs = std::max(coeffs, views.v[k].activeCoeffs);
  const uint32_t smem = project_stage_bytes<S>(coeffs, p.restStride);
  static uint32_t configured = 0;
  const uint32_t most = project_stage_bytes<S>(kMaxShCoeffs, sh_rest_stride(kMaxShCoeffs, S));
  if (smem > configured) {
    cudaFuncSetAttribute(k_preprocess<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)most);
    configured = most;
  }
  const dim3 grid(div_up(p.n, kProjectThreads), views.count);
  launch_chained(k_preprocess<S>, grid, dim3(kProjectThreads), smem, stream, p, dViews, splats, reach, depthKeys, values, error,
                 coeffs);
}

} // namespace

void launch_preprocess(const Params &p, const ViewSet &views, const ViewSet *dViews, Splat *splats, float *reach, uint32_t *depthKeys,
                       uint32_t *values, cudaStream_t stream, uint32_t *error) {
  if (p.n == 0) return;
  switch (p.shStore) {
  case ShStore::BF16: launch_preprocess_s<ShStore::BF16>(p, views, dViews, splats, reach, depthKeys, values, error, stream); break;
  case ShStore::F16: launch_preprocess_s<ShStore::F16>(p, views, dViews, splats, reach, depthKeys, values, error, stream); break;
  default: launch_preprocess_s<ShStore::F32>(p, views, dViews, splats, reach, depthKeys, values, error, stream); break;
  }
}

} // namespace sb
