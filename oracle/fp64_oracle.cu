// ORACLE (test infrastructure only; nothing here is linked into the product
// library). A double-precision CUDA restatement of the reference's FP64 CPU
// twin, src/train/reference.cpp, for sizes the twin is too slow for (the
// central differences over hundreds of renders of a 100k-Gaussian scene):
//   k_prepare    prepare()          reference.cpp:117-185 (projection, culling,
//                                    SH colour), one thread per Gaussian;
//   k_composite  composite()        reference.cpp:193-232 (front-to-back
//                                    blending with splat_at() :188-196 and the
//                                    transmittance floor), one thread per pixel
//                                    over its 16x16 tile's list; the lists are
//                                    built by oracle/fp64.py in the twin's walk
//                                    order (depth ascending, ties by index
//                                    descending: the reverse of a stable
//                                    descending-depth sort);
//   k_loss_fields, k_loss_adjoint   reference_loss() reference.cpp:276-341
//                                    (L1 + SSIM with the clipped, renormalised
//                                    11x11 window, its P/Q/R fields and the
//                                    adjoint), per pixel with the twin's
//                                    direct window sums;
//   k_backward   the per-pixel part of reference_gradients() :359-405 (the
//                                    reverse walk, back to front, with the
//                                    composite behind and its log
//                                    transmittance), a warp's sums added to the
//                                    splat's 9 raw values by double atomics;
//   k_chain      its per-Gaussian part :407-520 (the chain rule to positions,
//                                    log-scales, quaternions, opacity logits
//                                    and SH, the view-direction term of the
//                                    position included).
// Every expression keeps the twin's order of operations in double; exp, log
// and sqrt are CUDA's double-precision functions (within an ulp or two of the
// host's), so results agree with the twin to rounding, not bit for bit.
#include <cstdint>
#include <cuda_runtime.h>

namespace {

constexpr double kLogMinTransmittance = -9.210340372;
constexpr double kC1 = 0.0001, kC2 = 0.0009;
__constant__ double c_weights[11] = {0.00102838, 0.00759876, 0.03600077, 0.10936069, 0.21300554, 0.26601172,
                                     0.21300554, 0.10936069, 0.03600077, 0.00759876, 0.00102838};

// The reference's Camera (src/render/camera.hpp) as the twin reads it: the
// float view matrix widened to double, column-major (view[c * 4 + r]).
struct Cam {
  double view[16];
  double position[3];
  double fx, fy, cx, cy;
  int width, height;
  double nearPlane;
};

// A projected splat (the twin's Splat, reference.cpp:25-32) and whether the
// Gaussian survived culling.
struct Rec {
  double cx, cy, radius, depth;
  double qx, qy, qz, opacity; // conic xx, xy, yy
  double r, g, b;
  double valid;
};

struct M3 {
  double m[3][3]; // m[column][row], as glm
};

__device__ M3 mul(const M3 &a, const M3 &b) {
  M3 o;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) o.m[c][r] = a.m[0][r] * b.m[c][0] + a.m[1][r] * b.m[c][1] + a.m[2][r] * b.m[c][2];
  return o;
}

__device__ M3 transpose(const M3 &a) {
  M3 o;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) o.m[c][r] = a.m[r][c];
  return o;
}

__device__ void sh_basis(double x, double y, double z, int degree, double b[16]) {
  const double xx = x * x, yy = y * y, zz = z * z;
  const double C1 = 0.4886025119029199;
  for (int k = 0; k < 16; ++k) b[k] = 0.0;
  b[0] = 0.28209479177387814;
  if (degree > 0) {
    b[1] = -C1 * y;
    b[2] = C1 * z;
    b[3] = -C1 * x;
  }
  if (degree > 1) {
    b[4] = 1.0925484305920792 * x * y;
    b[5] = -1.0925484305920792 * y * z;
    b[6] = 0.31539156525252005 * (2.0 * zz - xx - yy);
    b[7] = -1.0925484305920792 * x * z;
    b[8] = 0.5462742152960396 * (xx - yy);
  }
  if (degree > 2) {
    b[9] = -0.5900435899266435 * y * (3.0 * xx - yy);
    b[10] = 2.890611442640554 * x * y * z;
    b[11] = -0.4570457994644658 * y * (4.0 * zz - xx - yy);
    b[12] = 0.3731763325901154 * z * (2.0 * zz - 3.0 * xx - 3.0 * yy);
    b[13] = -0.4570457994644658 * x * (4.0 * zz - xx - yy);
    b[14] = 1.445305721320277 * z * (xx - yy);
    b[15] = -0.5900435899266435 * x * (xx - 3.0 * yy);
  }
}

// cull 0 (the frozen renders of the central differences): every record is
// computed and marked valid, whatever the culling tests say, so that a
// Gaussian the base render kept is never dropped by a parameter's nudge.
__global__ void k_prepare(int n, int degree, const float *__restrict__ positions, const float *__restrict__ scales,
                          const float *__restrict__ rotations, const float *__restrict__ opacities, const float *__restrict__ sh,
                          Cam cam, int cull, Rec *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Rec rec{};
  rec.valid = 0.0;
  out[i] = rec;
  const double *V = cam.view;
  const double px = positions[i * 3], py = positions[i * 3 + 1], pz = positions[i * 3 + 2];
  // t = view * (p, 1)
  const double tx0 = V[0] * px + V[4] * py + V[8] * pz + V[12];
  const double ty0 = V[1] * px + V[5] * py + V[9] * pz + V[13];
  const double tz = V[2] * px + V[6] * py + V[10] * pz + V[14];
  if (!(tz >= cam.nearPlane) && cull) return;
  const double opacity = 1.0 / (1.0 + exp(-(double)opacities[i]));
  if (!(opacity >= 1.0 / 255.0) && cull) return;
  const double qw = rotations[i * 4], qx = rotations[i * 4 + 1], qy = rotations[i * 4 + 2], qz = rotations[i * 4 + 3];
  const double len = sqrt(qw * qw + qx * qx + qy * qy + qz * qz);
  if (!(len >= 1e-4) && cull) return;
  const double w = qw / len, x = qx / len, y = qy / len, z = qz / len;
  const double s[3] = {exp((double)scales[i * 3]), exp((double)scales[i * 3 + 1]), exp((double)scales[i * 3 + 2])};
  // quat_to_mat (columns as constructed there) times diag(s).
  M3 R;
  R.m[0][0] = 1.0 - 2.0 * (y * y + z * z);
  R.m[0][1] = 2.0 * (x * y + w * z);
  R.m[0][2] = 2.0 * (x * z - w * y);
  R.m[1][0] = 2.0 * (x * y - w * z);
  R.m[1][1] = 1.0 - 2.0 * (x * x + z * z);
  R.m[1][2] = 2.0 * (y * z + w * x);
  R.m[2][0] = 2.0 * (x * z + w * y);
  R.m[2][1] = 2.0 * (y * z - w * x);
  R.m[2][2] = 1.0 - 2.0 * (x * x + y * y);
  M3 S{};
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) S.m[c][r] = c == r ? s[c] : 0.0;
  const M3 M = mul(R, S);
  const M3 sigma = mul(M, transpose(M)); // no 3D filter: + dmat3(0)
  // opacity3 = opacity * prod sqrt(s^2 / (s^2 + 0)) = opacity.
  double opacity3 = opacity;
  for (int a = 0; a < 3; ++a) opacity3 *= sqrt(s[a] * s[a] / (s[a] * s[a] + 0.0));
  if (!(opacity3 >= 1.0 / 255.0) && cull) return;
  const double limX = 1.3 * 0.5 * cam.width / cam.fx, limY = 1.3 * 0.5 * cam.height / cam.fy;
  const double tx = fmin(fmax(tx0 / tz, -limX), limX) * tz, ty = fmin(fmax(ty0 / tz, -limY), limY) * tz;
  M3 J{};
  J.m[0][0] = cam.fx / tz;
  J.m[1][1] = cam.fy / tz;
  J.m[2][0] = -cam.fx * tx / (tz * tz);
  J.m[2][1] = -cam.fy * ty / (tz * tz);
  M3 Rv;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) Rv.m[c][r] = V[c * 4 + r];
  const M3 T = mul(J, Rv);
  const M3 cov = mul(mul(T, sigma), transpose(T));
  const double a = cov.m[0][0] + 0.3, b = cov.m[0][1], c = cov.m[1][1] + 0.3;
  const double det = a * c - b * b;
  if (!(det > 1e-6) && cull) return;
  const double mid = 0.5 * (a + c);
  const double lambda = mid + sqrt(fmax(0.1, mid * mid - det));
  rec.radius = ceil(3.0 * sqrt(lambda));
  rec.cx = cam.fx * tx0 / tz + cam.cx;
  rec.cy = cam.fy * ty0 / tz + cam.cy;
  if ((rec.cx + rec.radius < 0.0 || rec.cy + rec.radius < 0.0 || rec.cx - rec.radius > cam.width ||
       rec.cy - rec.radius > cam.height) &&
      cull)
    return;
  rec.depth = tz;
  rec.qx = c / det;
  rec.qy = -b / det;
  rec.qz = a / det;
  rec.opacity = opacity3;
  // Colour from the view direction, the cloud's full degree (as the twin).
  double dx = px - cam.position[0], dy = py - cam.position[1], dz = pz - cam.position[2];
  const double dl = sqrt(dx * dx + dy * dy + dz * dz);
  dx /= dl;
  dy /= dl;
  dz /= dl;
  double basis[16];
  sh_basis(dx, dy, dz, degree, basis);
  const int coeffs = (degree + 1) * (degree + 1);
  double col[3] = {0.5, 0.5, 0.5};
  for (int k = 0; k < coeffs; ++k)
    for (int ch = 0; ch < 3; ++ch) col[ch] += basis[k] * (double)sh[((size_t)i * coeffs + k) * 3 + ch];
  if (!(fabs(col[0]) < 1e30 && fabs(col[1]) < 1e30 && fabs(col[2]) < 1e30) && cull) return;
  rec.r = fmax(col[0], 0.0);
  rec.g = fmax(col[1], 0.0);
  rec.b = fmax(col[2], 0.0);
  rec.valid = 1.0;
  out[i] = rec;
}

// One thread per pixel over its tile's splats, front to back.
// stopRank: the walk rank of the splat at which the pixel's transmittance
// would have fallen below the floor (the twin's stop), or -1 without one.
// mode 0 renders; mode 1 also sets bit (e * 256 + pixel of the tile) of bits
// (cleared by the caller) for every pair the pixel blends; mode 2 blends
// exactly the pairs whose bits are set, with no cutoff test and no stop: the
// render with the base point's contributing pairs and order held fixed, a
// function of the parameters without the cutoffs' jumps, which is what the
// adjoint differentiates.
__global__ void k_composite(const Rec *__restrict__ recs, const int64_t *__restrict__ entries, const int64_t *__restrict__ tileStart,
                            const int64_t *__restrict__ rank, int gridW, int width, int height, double bgR, double bgG, double bgB,
                            double *__restrict__ rgb, double *__restrict__ logT, int64_t *__restrict__ stopRank,
                            uint32_t *__restrict__ bits, int mode) {
  const int tile = blockIdx.x;
  const int x = (tile % gridW) * 16 + (int)(threadIdx.x & 15u), y = (tile / gridW) * 16 + (int)(threadIdx.x >> 4);
  if (x >= width || y >= height) return;
  double r = 0.0, g = 0.0, b = 0.0, lt = 0.0;
  int64_t stopped = -1;
  const double pxc = x + 0.5, pyc = y + 0.5;
  const uint32_t word = threadIdx.x >> 5, bit = 1u << (threadIdx.x & 31u);
  for (int64_t e = tileStart[tile]; e < tileStart[tile + 1]; ++e) {
    if (mode == 2 && (bits[e * 8 + word] & bit) == 0u) continue;
    const Rec &s = recs[entries[e]];
    const double dx = pxc - s.cx, dy = pyc - s.cy;
    if (mode != 2 && (fabs(dx) > s.radius || fabs(dy) > s.radius)) continue;
    const double power = -0.5 * (s.qx * dx * dx + s.qz * dy * dy) - s.qy * dx * dy;
    if (mode != 2 && power > 0.0) continue;
    const double alpha = fmin(0.99, s.opacity * exp(power));
    if (mode != 2 && !(alpha >= 1.0 / 255.0)) continue;
    const double logRest = log(1.0 - alpha);
    if (mode != 2 && lt + logRest < kLogMinTransmittance) {
      stopped = rank[entries[e]];
      break;
    }
    if (mode == 1) atomicOr(&bits[e * 8 + word], bit);
    const double weight = exp(lt) * alpha;
    r += weight * s.r;
    g += weight * s.g;
    b += weight * s.b;
    lt += logRest;
  }
  const double T = exp(lt);
  const size_t at = (size_t)y * width + x;
  rgb[at * 3] = r + T * bgR;
  rgb[at * 3 + 1] = g + T * bgG;
  rgb[at * 3 + 2] = b + T * bgB;
  logT[at] = lt;
  stopRank[at] = stopped;
}

// First pass of reference_loss: P, Q, R per pixel (9 doubles) and the
// per-pixel SSIM sum over channels into a per-block partial.
__global__ void k_loss_fields(const double *__restrict__ rgb, const uint8_t *__restrict__ target, int w, int h,
                              double *__restrict__ fields, double *__restrict__ partials) {
  __shared__ double s_sum[256];
  const int px = blockIdx.x * 16 + (int)(threadIdx.x & 15u), row = blockIdx.y * 16 + (int)(threadIdx.x >> 4);
  double ssim = 0.0;
  if (px < w && row < h) {
    double mx[3] = {0, 0, 0}, my[3] = {0, 0, 0}, xx[3] = {0, 0, 0}, yy[3] = {0, 0, 0}, xy[3] = {0, 0, 0};
    double norm = 0.0;
    for (int v = max(row - 5, 0); v <= min(row + 5, h - 1); ++v) {
      for (int u = max(px - 5, 0); u <= min(px + 5, w - 1); ++u) {
        const double weight = c_weights[v - row + 5] * c_weights[u - px + 5];
        const size_t at = (size_t)v * w + u;
        for (int c = 0; c < 3; ++c) {
          const double a = rgb[at * 3 + c], bt = target[at * 4 + c] / 255.0;
          mx[c] += weight * a;
          my[c] += weight * bt;
          xx[c] += weight * a * a;
          yy[c] += weight * bt * bt;
          xy[c] += weight * a * bt;
        }
        norm += weight;
      }
    }
    const size_t at = (size_t)row * w + px;
    for (int c = 0; c < 3; ++c) {
      const double m_x = mx[c] / norm, m_y = my[c] / norm;
      const double vx = xx[c] / norm - m_x * m_x, vy = yy[c] / norm - m_y * m_y, cxy = xy[c] / norm - m_x * m_y;
      const double n1 = 2.0 * m_x * m_y + kC1, n2 = 2.0 * cxy + kC2, d1 = m_x * m_x + m_y * m_y + kC1, d2 = vx + vy + kC2;
      const double s = (n1 * n2) / (d1 * d2);
      ssim += s;
      const double dMu = 2.0 * m_y * n2 / (d1 * d2) - s * 2.0 * m_x / d1, dVar = -s / d2, dCov = 2.0 * n1 / (d1 * d2);
      fields[at * 9 + c] = (dMu - 2.0 * m_x * dVar - m_y * dCov) / norm;
      fields[at * 9 + 3 + c] = dVar / norm;
      fields[at * 9 + 6 + c] = dCov / norm;
    }
  }
  s_sum[threadIdx.x] = ssim;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) s_sum[threadIdx.x] += s_sum[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = s_sum[0];
}

// Second pass: the adjoint and the per-block L1 partial.
__global__ void k_loss_adjoint(const double *__restrict__ rgb, const uint8_t *__restrict__ target, int w, int h, double lambda,
                               const double *__restrict__ fields, double *__restrict__ adjoint, double *__restrict__ partials) {
  __shared__ double s_sum[256];
  const int px = blockIdx.x * 16 + (int)(threadIdx.x & 15u), row = blockIdx.y * 16 + (int)(threadIdx.x >> 4);
  double l1 = 0.0;
  if (px < w && row < h) {
    const size_t at = (size_t)row * w + px;
    const double perValue = 1.0 / (3.0 * (double)((size_t)w * h));
    double p[3] = {0, 0, 0}, q[3] = {0, 0, 0}, r[3] = {0, 0, 0};
    for (int v = max(row - 5, 0); v <= min(row + 5, h - 1); ++v) {
      for (int u = max(px - 5, 0); u <= min(px + 5, w - 1); ++u) {
        const double weight = c_weights[v - row + 5] * c_weights[u - px + 5];
        const size_t other = (size_t)v * w + u;
        for (int c = 0; c < 3; ++c) {
          p[c] += weight * fields[other * 9 + c];
          q[c] += weight * fields[other * 9 + 3 + c];
          r[c] += weight * fields[other * 9 + 6 + c];
        }
      }
    }
    for (int c = 0; c < 3; ++c) {
      const double x = rgb[at * 3 + c], y = target[at * 4 + c] / 255.0, d = x - y;
      l1 += fabs(d);
      const double sign = d > 0.0 ? 1.0 : (d < 0.0 ? -1.0 : 0.0);
      adjoint[at * 3 + c] = ((1.0 - lambda) * sign - lambda * (p[c] + 2.0 * x * q[c] + y * r[c])) * perValue;
    }
  }
  s_sum[threadIdx.x] = l1;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) s_sum[threadIdx.x] += s_sum[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = s_sum[0];
}

// The twin's backward pass, one warp per two rows of a 16x16 tile walking the
// tile's list back to front (reverse walk order) in lockstep; a pixel takes
// a splat in front of its stopping splat only (the twin's j >= stop). The
// warp's 9 sums (and the two absolute centre sums) go to raw[index * 11 + v].
__global__ void k_backward(const Rec *__restrict__ recs, const int64_t *__restrict__ entries, const int64_t *__restrict__ tileStart,
                           const int64_t *__restrict__ rank, int gridW, int width, int height, double bgR, double bgG, double bgB,
                           const double *__restrict__ logTotal, const int64_t *__restrict__ stopRank,
                           const double *__restrict__ adjoint, double *__restrict__ raw) {
  const int tile = blockIdx.x;
  const int x = (tile % gridW) * 16 + (int)(threadIdx.x & 15u), y = (tile / gridW) * 16 + (int)(threadIdx.x >> 4);
  const bool inside = x < width && y < height;
  const size_t at = inside ? (size_t)y * width + x : 0;
  const double pxc = x + 0.5, pyc = y + 0.5;
  const double total = inside ? logTotal[at] : 0.0;
  const int64_t stop = inside ? stopRank[at] : -1;
  const double Ax = inside ? adjoint[at * 3] : 0.0, Ay = inside ? adjoint[at * 3 + 1] : 0.0, Az = inside ? adjoint[at * 3 + 2] : 0.0;
  double Br = bgR, Bg = bgG, Bb = bgB, logBehind = 0.0;
  for (int64_t e = tileStart[tile + 1] - 1; e >= tileStart[tile]; --e) {
    const int64_t index = entries[e];
    const Rec &s = recs[index];
    double v[11];
    for (int k = 0; k < 11; ++k) v[k] = 0.0;
    bool act = inside && (stop < 0 || rank[index] < stop);
    double dx = 0.0, dy = 0.0, power = 0.0, alpha = 0.0;
    if (act) {
      dx = pxc - s.cx;
      dy = pyc - s.cy;
      if (fabs(dx) > s.radius || fabs(dy) > s.radius) act = false;
    }
    if (act) {
      power = -0.5 * (s.qx * dx * dx + s.qz * dy * dy) - s.qy * dx * dy;
      if (power > 0.0) act = false;
    }
    if (act) {
      alpha = fmin(0.99, s.opacity * exp(power));
      if (!(alpha >= 1.0 / 255.0)) act = false;
    }
    if (act) {
      const double logRest = log(1.0 - alpha);
      const double T = exp(total - logBehind - logRest);
      const double wA = T * alpha;
      v[6] = wA * Ax;
      v[7] = wA * Ay;
      v[8] = wA * Az;
      if (s.opacity * exp(power) < 0.99) {
        const double dAlpha = T * (Ax * (s.r - Br) + Ay * (s.g - Bg) + Az * (s.b - Bb));
        v[0] = dAlpha * exp(power);
        const double dPower = dAlpha * alpha;
        const double vx = s.qx * dx + s.qy * dy, vy = s.qy * dx + s.qz * dy;
        v[1] = dPower * vx;
        v[2] = dPower * vy;
        v[9] = fabs(dPower * vx);
        v[10] = fabs(dPower * vy);
        v[3] = dPower * 0.5 * vx * vx;
        v[4] = dPower * 0.5 * vx * vy;
        v[5] = dPower * 0.5 * vy * vy;
      }
      // glm::mix(B, colour, alpha)
      Br = Br * (1.0 - alpha) + s.r * alpha;
      Bg = Bg * (1.0 - alpha) + s.g * alpha;
      Bb = Bb * (1.0 - alpha) + s.b * alpha;
      logBehind += logRest;
    }
    if (!__any_sync(0xFFFFFFFFu, act)) continue;
    for (int k = 0; k < 11; ++k)
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xFFFFFFFFu, v[k], o);
    if ((threadIdx.x & 31u) == 0u)
      for (int k = 0; k < 11; ++k)
        if (v[k] != 0.0) atomicAdd(&raw[index * 11 + k], v[k]);
  }
}

__device__ void sh_basis_gradient(double x, double y, double z, int degree, double g[16][3]) {
  const double C1 = 0.4886025119029199, A = 1.0925484305920792, K = 0.31539156525252005, L = 0.5462742152960396;
  const double C = -0.5900435899266435, E = 2.890611442640554, F = -0.4570457994644658, G = 0.3731763325901154,
               H = 1.445305721320277;
  const double xx = x * x, yy = y * y, zz = z * z;
  for (int k = 0; k < 16; ++k) g[k][0] = g[k][1] = g[k][2] = 0.0;
  auto set = [&](int k, double a, double b, double c) {
    g[k][0] = a;
    g[k][1] = b;
    g[k][2] = c;
  };
  if (degree > 0) {
    set(1, 0.0, -C1, 0.0);
    set(2, 0.0, 0.0, C1);
    set(3, -C1, 0.0, 0.0);
  }
  if (degree > 1) {
    set(4, A * y, A * x, A * 0.0);
    set(5, -A * 0.0, -A * z, -A * y);
    set(6, K * (-2.0 * x), K * (-2.0 * y), K * (4.0 * z));
    set(7, -A * z, -A * 0.0, -A * x);
    set(8, L * (2.0 * x), L * (-2.0 * y), L * 0.0);
  }
  if (degree > 2) {
    set(9, C * (6.0 * x * y), C * (3.0 * xx - 3.0 * yy), C * 0.0);
    set(10, E * (y * z), E * (x * z), E * (x * y));
    set(11, F * (-2.0 * x * y), F * (4.0 * zz - xx - 3.0 * yy), F * (8.0 * y * z));
    set(12, G * (-6.0 * x * z), G * (-6.0 * y * z), G * (6.0 * zz - 3.0 * xx - 3.0 * yy));
    set(13, F * (4.0 * zz - 3.0 * xx - yy), F * (-2.0 * x * y), F * (8.0 * x * z));
    set(14, H * (2.0 * x * z), H * (-2.0 * y * z), H * (xx - yy));
    set(15, C * (3.0 * xx - 3.0 * yy), C * (-6.0 * x * y), C * 0.0);
  }
}

// A 3x2 matrix as glm's dmat3x2: three columns of two rows, m[column][row].
struct M32 {
  double m[3][2];
};

// trace(G (A X J^T)), G 2x2 (g[column][row]), A and J 3x2, X 3x3.
__device__ double trace_term(const double G[2][2], const M32 &A, const M3 &X, const M32 &J) {
  double AX[3][2]; // A * X: column c = sum_k A[k] X[c][k]
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 2; ++r) AX[c][r] = A.m[0][r] * X.m[c][0] + A.m[1][r] * X.m[c][1] + A.m[2][r] * X.m[c][2];
  double AXJt[2][2]; // (A X) J^T: column c = sum_k AX[k] * J^T[c][k] = sum_k AX[k] J[k][c]
  for (int c = 0; c < 2; ++c)
    for (int r = 0; r < 2; ++r) AXJt[c][r] = AX[0][r] * J.m[0][c] + AX[1][r] * J.m[1][c] + AX[2][r] * J.m[2][c];
  double P[2][2];
  for (int c = 0; c < 2; ++c)
    for (int r = 0; r < 2; ++r) P[c][r] = G[0][r] * AXJt[c][0] + G[1][r] * AXJt[c][1];
  return P[0][0] + P[1][1];
}

__global__ void k_chain(int n, int degree, const float *__restrict__ positions, const float *__restrict__ scales,
                        const float *__restrict__ rotations, const float *__restrict__ opacities, const float *__restrict__ sh,
                        Cam cam, const double *__restrict__ raw, double *__restrict__ gPositions, double *__restrict__ gScales,
                        double *__restrict__ gRotations, double *__restrict__ gOpacities, double *__restrict__ gSh) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int coeffs = (degree + 1) * (degree + 1);
  const double *g = raw + (size_t)i * 11;
  bool any = false;
  for (int k = 0; k < 9; ++k) any = any || g[k] != 0.0;
  if (!any) {
    for (int a = 0; a < 3; ++a) gPositions[i * 3 + a] = gScales[i * 3 + a] = 0.0;
    for (int k = 0; k < 4; ++k) gRotations[i * 4 + k] = 0.0;
    gOpacities[i] = 0.0;
    for (int k = 0; k < coeffs * 3; ++k) gSh[(size_t)i * coeffs * 3 + k] = 0.0;
    return;
  }
  const double *V = cam.view;
  const double px = positions[i * 3], py = positions[i * 3 + 1], pz = positions[i * 3 + 2];
  const double qw0 = rotations[i * 4], qx0 = rotations[i * 4 + 1], qy0 = rotations[i * 4 + 2], qz0 = rotations[i * 4 + 3];
  const double quatLength = sqrt(qw0 * qw0 + qx0 * qx0 + qy0 * qy0 + qz0 * qz0);
  const double qw = quatLength > 0.0 ? qw0 / quatLength : 1.0, qx = quatLength > 0.0 ? qx0 / quatLength : 0.0;
  const double qy = quatLength > 0.0 ? qy0 / quatLength : 0.0, qz = quatLength > 0.0 ? qz0 / quatLength : 0.0;
  const double tX = V[0] * px + V[4] * py + V[8] * pz + V[12];
  const double tY = V[1] * px + V[5] * py + V[9] * pz + V[13];
  const double z = V[2] * px + V[6] * py + V[10] * pz + V[14];
  const double iz = 1.0 / z, iz2 = iz * iz;
  const double G[2][2] = {{g[3], g[4]}, {g[4], g[5]}};
  const double opacity = 1.0 / (1.0 + exp(-(double)opacities[i]));
  M3 R;
  {
    const double w = qw, x = qx, y = qy, zz = qz;
    R.m[0][0] = 1.0 - 2.0 * (y * y + zz * zz);
    R.m[0][1] = 2.0 * (x * y + w * zz);
    R.m[0][2] = 2.0 * (x * zz - w * y);
    R.m[1][0] = 2.0 * (x * y - w * zz);
    R.m[1][1] = 1.0 - 2.0 * (x * x + zz * zz);
    R.m[1][2] = 2.0 * (y * zz + w * x);
    R.m[2][0] = 2.0 * (x * zz + w * y);
    R.m[2][1] = 2.0 * (y * zz - w * x);
    R.m[2][2] = 1.0 - 2.0 * (x * x + y * y);
  }
  const double s2[3] = {exp(2.0 * (double)scales[i * 3]), exp(2.0 * (double)scales[i * 3 + 1]), exp(2.0 * (double)scales[i * 3 + 2])};
  M3 D{};
  for (int a = 0; a < 3; ++a) D.m[a][a] = s2[a];
  M3 Rv;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) Rv.m[c][r] = V[c * 4 + r];
  const M3 X = mul(mul(Rv, mul(mul(R, D), transpose(R))), transpose(Rv));
  const double limX = 1.3 * 0.5 * cam.width / cam.fx, limY = 1.3 * 0.5 * cam.height / cam.fy;
  const double rx = tX * iz, ry = tY * iz;
  const bool clampedX = fabs(rx) > limX, clampedY = fabs(ry) > limY;
  const double tx = fmin(fmax(rx, -limX), limX) * z, ty = fmin(fmax(ry, -limY), limY) * z;
  const double fx = cam.fx, fy = cam.fy;
  M32 J{};
  J.m[0][0] = fx * iz;
  J.m[1][1] = fy * iz;
  J.m[2][0] = -fx * tx * iz2;
  J.m[2][1] = -fy * ty * iz2;
  M32 Jc = J;
  Jc.m[2][0] = -fx * tX * iz2;
  Jc.m[2][1] = -fy * tY * iz2;
  double gT[3];
  for (int c = 0; c < 3; ++c) gT[c] = Jc.m[c][0] * g[1] + Jc.m[c][1] * g[2];
  M32 dJx{}, dJy{}, dJz{};
  dJx.m[2][0] = clampedX ? 0.0 : -fx * iz2;
  dJy.m[2][1] = clampedY ? 0.0 : -fy * iz2;
  dJz.m[0][0] = -fx * iz2;
  dJz.m[1][1] = -fy * iz2;
  dJz.m[2][0] = clampedX ? fx * tx * iz2 * iz : 2.0 * fx * tx * iz2 * iz;
  dJz.m[2][1] = clampedY ? fy * ty * iz2 * iz : 2.0 * fy * ty * iz2 * iz;
  gT[0] += 2.0 * trace_term(G, dJx, X, J);
  gT[1] += 2.0 * trace_term(G, dJy, X, J);
  gT[2] += 2.0 * trace_term(G, dJz, X, J);
  double gP[3];
  for (int c = 0; c < 3; ++c) gP[c] = Rv.m[c][0] * gT[0] + Rv.m[c][1] * gT[1] + Rv.m[c][2] * gT[2]; // Rv^T gT
  // T = J Rv (3x2): column c = sum_k J[k] Rv[c][k]; G3 = T^T G T.
  M32 T;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 2; ++r) T.m[c][r] = J.m[0][r] * Rv.m[c][0] + J.m[1][r] * Rv.m[c][1] + J.m[2][r] * Rv.m[c][2];
  M3 G3;
  for (int c = 0; c < 3; ++c) {
    double GT[2]; // G * T[c]
    for (int r = 0; r < 2; ++r) GT[r] = G[0][r] * T.m[c][0] + G[1][r] * T.m[c][1];
    for (int r = 0; r < 3; ++r) G3.m[c][r] = T.m[r][0] * GT[0] + T.m[r][1] * GT[1];
  }
  for (int a = 0; a < 3; ++a) {
    double GR[3];
    for (int r = 0; r < 3; ++r) GR[r] = G3.m[0][r] * R.m[a][0] + G3.m[1][r] * R.m[a][1] + G3.m[2][r] * R.m[a][2];
    gScales[i * 3 + a] = 2.0 * s2[a] * (R.m[a][0] * GR[0] + R.m[a][1] * GR[1] + R.m[a][2] * GR[2]);
  }
  M3 P = mul(mul(G3, R), D);
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) P.m[c][r] *= 2.0;
  const double w = qw, x = qx, y = qy, zq = qz;
  const double dRv[4][9] = {{0.0, 2.0 * zq, -2.0 * y, -2.0 * zq, 0.0, 2.0 * x, 2.0 * y, -2.0 * x, 0.0},
                            {0.0, 2.0 * y, 2.0 * zq, 2.0 * y, -4.0 * x, 2.0 * w, 2.0 * zq, -2.0 * w, -4.0 * x},
                            {-4.0 * y, 2.0 * x, -2.0 * w, 2.0 * x, 0.0, 2.0 * zq, 2.0 * w, 2.0 * zq, -4.0 * y},
                            {-4.0 * zq, 2.0 * w, 2.0 * x, -2.0 * w, -4.0 * zq, 2.0 * y, 2.0 * x, 2.0 * y, 0.0}};
  double gq[4];
  for (int k = 0; k < 4; ++k) {
    gq[k] = 0.0;
    for (int c = 0; c < 3; ++c) gq[k] += P.m[c][0] * dRv[k][c * 3] + P.m[c][1] * dRv[k][c * 3 + 1] + P.m[c][2] * dRv[k][c * 3 + 2];
  }
  const double quat[4] = {qw, qx, qy, qz};
  const double qdot = quat[0] * gq[0] + quat[1] * gq[1] + quat[2] * gq[2] + quat[3] * gq[3];
  for (int k = 0; k < 4; ++k) gRotations[i * 4 + k] = (gq[k] - quat[k] * qdot) / fmax(quatLength, 1e-12);
  gOpacities[i] = g[0] * 1.0 * 1.0 * opacity * (1.0 - opacity);
  // Colour and its view direction.
  double dx = px - cam.position[0], dy = py - cam.position[1], dz = pz - cam.position[2];
  const double distance = sqrt(dx * dx + dy * dy + dz * dz);
  const double dir[3] = {dx / distance, dy / distance, dz / distance};
  double basis[16];
  sh_basis(dir[0], dir[1], dir[2], degree, basis);
  double colour[3] = {0.5, 0.5, 0.5};
  for (int k = 0; k < coeffs; ++k)
    for (int c = 0; c < 3; ++c) colour[c] += basis[k] * (double)sh[((size_t)i * coeffs + k) * 3 + c];
  const double gColour[3] = {g[6], g[7], g[8]};
  if (degree > 0) {
    double bg[16][3];
    sh_basis_gradient(dir[0], dir[1], dir[2], degree, bg);
    double gDir[3] = {0.0, 0.0, 0.0};
    for (int k = 1; k < coeffs; ++k) {
      double d = 0.0;
      for (int c = 0; c < 3; ++c) d += gColour[c] * (colour[c] > 0.0 ? 1.0 : 0.0) * (double)sh[((size_t)i * coeffs + k) * 3 + c];
      for (int a = 0; a < 3; ++a) gDir[a] += d * bg[k][a];
    }
    const double dd = dir[0] * gDir[0] + dir[1] * gDir[1] + dir[2] * gDir[2];
    for (int a = 0; a < 3; ++a) gP[a] += (gDir[a] - dir[a] * dd) / distance;
  }
  for (int a = 0; a < 3; ++a) gPositions[i * 3 + a] = gP[a];
  for (int k = 0; k < coeffs; ++k)
    for (int c = 0; c < 3; ++c) gSh[((size_t)i * coeffs + k) * 3 + c] = colour[c] > 0.0 ? basis[k] * gColour[c] : 0.0;
}

int status(cudaError_t e) { return e == cudaSuccess ? 0 : (int)e; }

Cam make_cam(const float *view16, const float *position3, const float *intrinsics4, int width, int height, float nearPlane) {
  Cam cam{};
  for (int k = 0; k < 16; ++k) cam.view[k] = view16[k];
  for (int k = 0; k < 3; ++k) cam.position[k] = position3[k];
  cam.fx = intrinsics4[0];
  cam.fy = intrinsics4[1];
  cam.cx = intrinsics4[2];
  cam.cy = intrinsics4[3];
  cam.width = width;
  cam.height = height;
  cam.nearPlane = nearPlane;
  return cam;
}

} // namespace

extern "C" {

// Doubles per projected splat record: cx cy radius depth qx qy qz opacity r g b valid.
int fp64_record_words() { return (int)(sizeof(Rec) / sizeof(double)); }

// All pointers are device memory except view16/position3/intrinsics4 (host).
int fp64_prepare(int n, int degree, const float *positions, const float *scales, const float *rotations, const float *opacities,
                 const float *sh, const float *view16, const float *position3, const float *intrinsics4, int width, int height,
                 float nearPlane, int cull, double *records, void *stream) {
  if (n <= 0) return 0;
  const Cam cam = make_cam(view16, position3, intrinsics4, width, height, nearPlane);
  k_prepare<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(n, degree, positions, scales, rotations, opacities, sh,
                                                                             cam, cull, reinterpret_cast<Rec *>(records));
  return status(cudaGetLastError());
}

// entries: splat indices grouped by tile, each tile's in the twin's walk order;
// tileStart: gridW * gridH + 1 offsets; rank: each splat's walk rank. rgb: 3
// doubles per pixel; logT: 1; stopRank: 1 int64 per pixel. bits: 8 words per
// entry for modes 1 and 2 (k_composite), else null.
int fp64_composite(const double *records, const int64_t *entries, const int64_t *tileStart, const int64_t *rank, int gridW,
                   int gridH, int width, int height, double bgR, double bgG, double bgB, double *rgb, double *logT,
                   int64_t *stopRank, uint32_t *bits, int mode, void *stream) {
  if (gridW * gridH == 0) return 0;
  k_composite<<<gridW * gridH, 256, 0, static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<const Rec *>(records), entries,
                                                                            tileStart, rank, gridW, width, height, bgR, bgG, bgB,
                                                                            rgb, logT, stopRank, bits, mode);
  return status(cudaGetLastError());
}

// reference_gradients from a render's lists, log T and stops and a per-pixel
// adjoint (3 doubles): raw (11 doubles per Gaussian, cleared here), then the
// gradients in the reference's ParameterGradients layout (device doubles).
int fp64_gradients(int n, int degree, const float *positions, const float *scales, const float *rotations, const float *opacities,
                   const float *sh, const float *view16, const float *position3, const float *intrinsics4, int width, int height,
                   const double *records, const int64_t *entries, const int64_t *tileStart, const int64_t *rank, int gridW,
                   int gridH, double bgR, double bgG, double bgB, const double *logT, const int64_t *stopRank,
                   const double *adjoint, double *raw, double *gPositions, double *gScales, double *gRotations,
                   double *gOpacities, double *gSh, void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (n <= 0) return 0;
  cudaMemsetAsync(raw, 0, (size_t)n * 11 * sizeof(double), s);
  if (gridW * gridH > 0)
    k_backward<<<gridW * gridH, 256, 0, s>>>(reinterpret_cast<const Rec *>(records), entries, tileStart, rank, gridW, width, height,
                                             bgR, bgG, bgB, logT, stopRank, adjoint, raw);
  const Cam cam = make_cam(view16, position3, intrinsics4, width, height, 0.0f);
  k_chain<<<(n + 127) / 128, 128, 0, s>>>(n, degree, positions, scales, rotations, opacities, sh, cam, raw, gPositions, gScales,
                                          gRotations, gOpacities, gSh);
  return status(cudaGetLastError());
}

// fields: 9 doubles per pixel of scratch; adjoint: 3 per pixel; partials: 2
// arrays of ceil(w/16) * ceil(h/16) doubles (SSIM sums, then L1 sums).
int fp64_loss(const double *rgb, const uint8_t *target, int width, int height, double lambda, double *fields, double *adjoint,
              double *partials, void *stream) {
  const dim3 grid((width + 15) / 16, (height + 15) / 16);
  const size_t blocks = (size_t)grid.x * grid.y;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_loss_fields<<<grid, 256, 0, s>>>(rgb, target, width, height, fields, partials);
  k_loss_adjoint<<<grid, 256, 0, s>>>(rgb, target, width, height, lambda, fields, adjoint, partials + blocks);
  return status(cudaGetLastError());
}

} // extern "C"
