/*
 * ORACLE (test infrastructure only; the product never links or calls this).
 *
 * A single-threaded FP32 CPU restatement of the reference's training shaders,
 * for bit-level checks of the CUDA kernels "given identical projected inputs":
 *   preprocess      shaders/train_preprocess.comp:31-134
 *   tile tests      shaders/train_types.glsl:34-77 (splat_tiles, splat_reaches_tile)
 *   bin count/emit  shaders/train_bin_count.comp:18-38, train_bin_emit.comp:18-38
 *   tile ranges     shaders/train_tile_ranges.comp:11-23
 *   forward         shaders/train_forward.comp:38-100 with splat_pixels/splat_at
 *                   (train_types.glsl:43-94)
 *   SSIM and loss   shaders/train_ssim.comp:42-123, train_loss.comp:52-113
 *   backward        shaders/train_backward.glsl:78-157 with the 32-lane
 *                   transposed butterfly reduce_and_add (:51-76) and the
 *                   fixed-point add_gradient of train_backward_fixed.comp:16-21
 * Each function evaluates the GLSL expressions in the rounding order this
 * repository's CUDA kernels state (left to right, one rounding per operation,
 * fmaf only where written), and calls the deterministic exp/log of
 * include/splat_detmath.h, so an integer result (tile entries, their order,
 * ranges, stop indices, fixed-point sums) must match the GPU bit for bit.
 * It does not share the kernels' shortcuts: pixel areas and radius tests are
 * evaluated per pixel as the GLSL does, warps are simulated lane by lane, and
 * fixed-point sums are added one warp total at a time as the reference does.
 * Its float results are checked against the reference's own FP64 twin
 * (src/train/reference.cpp) with the reference's tolerances.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "splat_detmath.h"

#define TILE 16
#define INVISIBLE 0xFFFFFFFFu
#define RAW_PER_SPLAT 14
#define RAW_STRIDE 16
static const float kLogMinTransmittance = -9.210340372f;

/* One view, as ViewParams of the CUDA kernels. */
typedef struct {
  float R[9], T[3], pos[3], nearPlane, fx, fy, cx, cy, widthF, heightF, tanX, tanY;
  int width, height, gridW, gridH, activeDegree, activeCoeffs;
  float perPixel, fixedScale;
} OView;

static float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

/* ------------------------------------------------------------ preprocess */

static void sh_basis(float x, float y, float z, int degree, float b[16]) {
  const float C1 = 0.4886025119029199f;
  const float xx = x * x, yy = y * y, zz = z * z;
  b[0] = 0.28209479177387814f;
  if (degree > 0) {
    b[1] = -C1 * y;
    b[2] = C1 * z;
    b[3] = -C1 * x;
  }
  if (degree > 1) {
    b[4] = 1.0925484305920792f * x * y;
    b[5] = -1.0925484305920792f * y * z;
    b[6] = 0.31539156525252005f * (2.0f * zz - xx - yy);
    b[7] = -1.0925484305920792f * x * z;
    b[8] = 0.5462742152960396f * (xx - yy);
  }
  if (degree > 2) {
    b[9] = -0.5900435899266435f * y * (3.0f * xx - yy);
    b[10] = 2.890611442640554f * x * y * z;
    b[11] = -0.4570457994644658f * y * (4.0f * zz - xx - yy);
    b[12] = 0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
    b[13] = -0.4570457994644658f * x * (4.0f * zz - xx - yy);
    b[14] = 1.445305721320277f * z * (xx - yy);
    b[15] = -0.5900435899266435f * x * (xx - 3.0f * yy);
  }
}

/* train_quat_to_mat, as rows. */
static void quat_rows(float w, float x, float y, float z, float m[3][3]) {
  const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z, wx = w * x, wy = w * y, wz = w * z;
  m[0][0] = 1.0f - 2.0f * (yy + zz);
  m[1][0] = 2.0f * (xy + wz);
  m[2][0] = 2.0f * (xz - wy);
  m[0][1] = 2.0f * (xy - wz);
  m[1][1] = 1.0f - 2.0f * (xx + zz);
  m[2][1] = 2.0f * (yz + wx);
  m[0][2] = 2.0f * (xz + wy);
  m[1][2] = 2.0f * (yz - wx);
  m[2][2] = 1.0f - 2.0f * (xx + yy);
}

static uint32_t float_bits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}

/* sh: GaussianCloud layout [i][k][c], as the device holds it (already rounded
 * to the device's storage). splats: 12 floats per Gaussian (conic xyz,
 * opacity, colour rgb, radius, centre xy, extent xy), written only when visible. */
void oracle_preprocess(int n, int shCoeffs, const float *pos, const float *scales, const float *rot, const float *opac,
                       const float *sh, const OView *v, float *splats, float *reach, uint32_t *keys) {
  for (int i = 0; i < n; ++i) {
    keys[i] = INVISIBLE;
    const float px = pos[i * 3], py = pos[i * 3 + 1], pz = pos[i * 3 + 2];
    const float tx = fmaf(v->R[2], pz, fmaf(v->R[1], py, fmaf(v->R[0], px, v->T[0])));
    const float ty = fmaf(v->R[5], pz, fmaf(v->R[4], py, fmaf(v->R[3], px, v->T[1])));
    const float tz = fmaf(v->R[8], pz, fmaf(v->R[7], py, fmaf(v->R[6], px, v->T[2])));
    if (!(tz >= v->nearPlane)) continue;
    const float opacity = 1.0f / (1.0f + splat_expf(-opac[i]));
    if (!(opacity >= 1.0f / 255.0f)) continue;
    const float qw0 = rot[i * 4], qx0 = rot[i * 4 + 1], qy0 = rot[i * 4 + 2], qz0 = rot[i * 4 + 3];
    const float len = sqrtf(fmaf(qz0, qz0, fmaf(qy0, qy0, fmaf(qx0, qx0, qw0 * qw0))));
    if (!(len >= 1e-4f)) continue;
    const float qw = qw0 / len, qx = qx0 / len, qy = qy0 / len, qz = qz0 / len;
    const float s[3] = {splat_expf(scales[i * 3]), splat_expf(scales[i * 3 + 1]), splat_expf(scales[i * 3 + 2])};
    float Rq[3][3], M[3][3], sigma[3][3];
    quat_rows(qw, qx, qy, qz, Rq);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) M[r][c] = Rq[r][c] * s[c];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) sigma[r][c] = fmaf(M[r][2], M[c][2], fmaf(M[r][1], M[c][1], M[r][0] * M[c][0]));
    const float s2[3] = {s[0] * s[0], s[1] * s[1], s[2] * s[2]};
    const float k3 = sqrtf(s2[0] / (s2[0] + 0.0f) * (s2[1] / (s2[1] + 0.0f)) * (s2[2] / (s2[2] + 0.0f)));
    const float opacity3 = opacity * k3;
    if (!(opacity3 >= 1.0f / 255.0f)) continue;
    const float limX = 1.3f * v->tanX, limY = 1.3f * v->tanY;
    const float txc = clampf(tx / tz, -limX, limX) * tz, tyc = clampf(ty / tz, -limY, limY) * tz;
    const float tz2 = tz * tz;
    const float j00 = v->fx / tz, j11 = v->fy / tz, j02 = (-v->fx * txc) / tz2, j12 = (-v->fy * tyc) / tz2;
    float Tm[2][3], U[3][2];
    for (int c = 0; c < 3; ++c) {
      Tm[0][c] = fmaf(j02, v->R[6 + c], j00 * v->R[c]);
      Tm[1][c] = fmaf(j12, v->R[6 + c], j11 * v->R[3 + c]);
    }
    for (int k = 0; k < 3; ++k)
      for (int r = 0; r < 2; ++r) U[k][r] = fmaf(sigma[k][2], Tm[r][2], fmaf(sigma[k][1], Tm[r][1], sigma[k][0] * Tm[r][0]));
    const float cov00 = fmaf(Tm[0][2], U[2][0], fmaf(Tm[0][1], U[1][0], Tm[0][0] * U[0][0]));
    const float cov01 = fmaf(Tm[0][2], U[2][1], fmaf(Tm[0][1], U[1][1], Tm[0][0] * U[0][1]));
    const float cov11 = fmaf(Tm[1][2], U[2][1], fmaf(Tm[1][1], U[1][1], Tm[1][0] * U[0][1]));
    const float a = cov00 + 0.3f, b = cov01, c = cov11 + 0.3f;
    const float det = a * c - b * b;
    if (!(det > 1e-6f)) continue;
    const float mid = 0.5f * (a + c);
    const float lambda = mid + sqrtf(fmaxf(0.1f, mid * mid - det));
    const float radius = ceilf(3.0f * sqrtf(lambda));
    const float centerX = v->fx * tx / tz + v->cx, centerY = v->fy * ty / tz + v->cy;
    if (centerX + radius < 0.0f || centerY + radius < 0.0f || centerX - radius > v->widthF || centerY - radius > v->heightF)
      continue;
    const float dx = px - v->pos[0], dy = py - v->pos[1], dz = pz - v->pos[2];
    const float dlen = sqrtf(fmaf(dz, dz, fmaf(dy, dy, dx * dx)));
    float basis[16];
    sh_basis(dx / dlen, dy / dlen, dz / dlen, v->activeDegree, basis);
    float col[3] = {0.5f, 0.5f, 0.5f};
    for (int k = 0; k < v->activeCoeffs; ++k)
      for (int ch = 0; ch < 3; ++ch) col[ch] = fmaf(basis[k], sh[((size_t)i * shCoeffs + k) * 3 + ch], col[ch]);
    if (!(fabsf(col[0]) < 1e30f && fabsf(col[1]) < 1e30f && fabsf(col[2]) < 1e30f)) continue;
    const float rc = 2.0f * splat_logf(255.0f * opacity3);
    float *o = splats + (size_t)i * 12;
    o[0] = c / det;
    o[1] = -b / det;
    o[2] = a / det;
    o[3] = opacity3;
    o[4] = fmaxf(col[0], 0.0f);
    o[5] = fmaxf(col[1], 0.0f);
    o[6] = fmaxf(col[2], 0.0f);
    o[7] = radius;
    o[8] = centerX;
    o[9] = centerY;
    o[10] = fminf(sqrtf(rc * a), radius);
    o[11] = fminf(sqrtf(rc * c), radius);
    reach[i] = rc;
    keys[i] = 0xFFFFFFFFu - float_bits(tz);
  }
}

/* ------------------------------------------------------------ binning */

static void splat_tiles(const float *s, int gridW, int gridH, uint32_t t[4]) {
  const float lastX = (float)(gridW - 1), lastY = (float)(gridH - 1);
  t[0] = (uint32_t)clampf(floorf((s[8] - s[10] - 1.0f) / 16.0f), 0.0f, lastX);
  t[1] = (uint32_t)clampf(floorf((s[9] - s[11] - 1.0f) / 16.0f), 0.0f, lastY);
  t[2] = (uint32_t)clampf(floorf((s[8] + s[10] + 1.0f) / 16.0f), 0.0f, lastX);
  t[3] = (uint32_t)clampf(floorf((s[9] + s[11] + 1.0f) / 16.0f), 0.0f, lastY);
}

static int splat_reaches_tile(const float *s, float reach, uint32_t tx, uint32_t ty) {
  const float qx = s[0], qy = s[1], qz = s[2];
  /* The tangent points as products by the conic's diagonal reciprocals (the
   * GLSL division is not correctly rounded either; the kernels take one
   * correctly rounded reciprocal per splat). */
  const float iqx = 1.0f / qx, iqz = 1.0f / qz;
  const float lowX = ((float)tx * 16.0f + 0.5f) - s[8], lowY = ((float)ty * 16.0f + 0.5f) - s[9];
  const float highX = lowX + 15.0f, highY = lowY + 15.0f;
  if (lowX <= 0.0f && lowY <= 0.0f && highX >= 0.0f && highY >= 0.0f) return 1;
  float least = 1e30f;
  for (int side = 0; side < 2; ++side) {
    const float x = side == 0 ? lowX : highX;
    const float y = clampf((-qy * x) * iqz, lowY, highY);
    least = fminf(least, qx * x * x + 2.0f * qy * x * y + qz * y * y);
    const float vv = side == 0 ? lowY : highY;
    const float u = clampf((-qy * vv) * iqx, lowX, highX);
    least = fminf(least, qx * u * u + 2.0f * qy * u * vv + qz * vv * vv);
  }
  return least <= reach * 1.001f + 1e-3f;
}

/* Emits (tile, splat) for the splats in `order` (splat indices; items with
 * key INVISIBLE skipped), tile by tile in row order per splat. Writes at most
 * cap entries; returns the total. */
int64_t oracle_bin(int items, const uint32_t *order, const uint32_t *itemKeys, const float *splats, const float *reach,
                   const OView *v, uint32_t *entryTiles, uint32_t *entryValues, int64_t cap) {
  int64_t slot = 0;
  for (int r = 0; r < items; ++r) {
    if (itemKeys[r] == INVISIBLE) continue;
    const uint32_t s = order != NULL ? order[r] : (uint32_t)r;
    const float *sp = splats + (size_t)s * 12;
    uint32_t t[4];
    splat_tiles(sp, v->gridW, v->gridH, t);
    for (uint32_t y = t[1]; y <= t[3]; ++y) {
      for (uint32_t x = t[0]; x <= t[2]; ++x) {
        if (!splat_reaches_tile(sp, reach[s], x, y)) continue;
        if (slot < cap && entryTiles != NULL) {
          entryTiles[slot] = y * (uint32_t)v->gridW + x;
          entryValues[slot] = s;
        }
        ++slot;
      }
    }
  }
  return slot;
}

/* ranges: 2 u32 per tile, zeroed first. */
void oracle_ranges(int64_t count, const uint32_t *tiles, uint32_t *ranges) {
  for (int64_t k = 0; k < count; ++k) {
    const uint32_t tile = tiles[k];
    if (k == 0 || tiles[k - 1] != tile) ranges[tile * 2] = (uint32_t)k;
    if (k + 1 == count || tiles[k + 1] != tile) ranges[tile * 2 + 1] = (uint32_t)(k + 1);
  }
}

/* ------------------------------------------------------------ forward */

/* splat_pixels() and splat_at() for pixel (x, y); returns whether the pixel
 * takes the splat, with d, power, alpha and exp(power). */
static int splat_at(const float *s, uint32_t x, uint32_t y, const uint32_t tile[4], float *dx, float *dy, float *power,
                    float *alpha, float *ep) {
  const float lowX = fmaxf(s[8] - s[10] - 0.5f, 0.0f), lowY = fmaxf(s[9] - s[11] - 0.5f, 0.0f);
  const float highX = fmaxf(s[8] + s[10] + 0.5f, 0.0f), highY = fmaxf(s[9] + s[11] + 0.5f, 0.0f);
  const uint32_t ax0 = (uint32_t)fminf(lowX, 4294967040.0f), ay0 = (uint32_t)fminf(lowY, 4294967040.0f);
  const uint32_t ax1 = (uint32_t)fminf(highX, 4294967040.0f) + 1u, ay1 = (uint32_t)fminf(highY, 4294967040.0f) + 1u;
  const uint32_t x0 = ax0 > tile[0] ? ax0 : tile[0], y0 = ay0 > tile[1] ? ay0 : tile[1];
  const uint32_t x1 = ax1 < tile[2] ? ax1 : tile[2], y1 = ay1 < tile[3] ? ay1 : tile[3];
  if (x < x0 || x >= x1 || y < y0 || y >= y1) return 0;
  *dx = ((float)x + 0.5f) - s[8];
  *dy = ((float)y + 0.5f) - s[9];
  const float r = s[7];
  if (fabsf(*dx) > r || fabsf(*dy) > r) return 0;
  /* -0.5 (qxx dx^2 + qyy dy^2) - qxy dx dy, in the kernels' rounding order. */
  const float hqx = -0.5f * s[0], nqy = -s[1], hqz = -0.5f * s[2];
  const float pxy = fmaf(nqy, *dy, hqx * *dx);
  *power = fmaf(hqz * *dy, *dy, pxy * *dx);
  if (*power > 0.0f) return 0;
  *ep = splat_expf(*power);
  *alpha = fminf(0.99f, s[3] * *ep);
  return *alpha >= 1.0f / 255.0f;
}

static void tile_pixels(const OView *v, int tile, uint32_t out[4]) {
  const uint32_t tx = (uint32_t)(tile % v->gridW), ty = (uint32_t)(tile / v->gridW);
  out[0] = tx * TILE;
  out[1] = ty * TILE;
  out[2] = tx * TILE + TILE < (uint32_t)v->width ? tx * TILE + TILE : (uint32_t)v->width;
  out[3] = ty * TILE + TILE < (uint32_t)v->height ? ty * TILE + TILE : (uint32_t)v->height;
}

/* image: 4 floats per pixel (rgb, log T); stops: 1 per pixel. */
void oracle_forward(const float *splats, const uint32_t *entryValues, const uint32_t *ranges, const OView *v,
                    const float bg[3], float *image, uint32_t *stops) {
  const int tiles = v->gridW * v->gridH;
  for (int tile = 0; tile < tiles; ++tile) {
    uint32_t tp[4];
    tile_pixels(v, tile, tp);
    const uint32_t first = ranges[tile * 2], end = ranges[tile * 2 + 1];
    for (uint32_t y = tp[1]; y < tp[3]; ++y) {
      for (uint32_t x = tp[0]; x < tp[2]; ++x) {
        float cr = 0.0f, cg = 0.0f, cb = 0.0f, T = 1.0f, logT = 0.0f;
        uint32_t stop = first;
        for (uint32_t k = end; k-- > first;) {
          const float *s = splats + (size_t)entryValues[k] * 12;
          float dx, dy, power, alpha, ep;
          if (!splat_at(s, x, y, tp, &dx, &dy, &power, &alpha, &ep)) continue;
          const float oneMinus = 1.0f - alpha;
          const float logRest = splat_logf(oneMinus);
          if (logT + logRest < kLogMinTransmittance) {
            stop = k + 1;
            break;
          }
          const float w = T * alpha;
          cr = fmaf(w, s[4], cr);
          cg = fmaf(w, s[5], cg);
          cb = fmaf(w, s[6], cb);
          T = T * oneMinus;
          logT = logT + logRest;
        }
        const size_t at = (size_t)y * v->width + x;
        image[at * 4] = fmaf(T, bg[0], cr);
        image[at * 4 + 1] = fmaf(T, bg[1], cg);
        image[at * 4 + 2] = fmaf(T, bg[2], cb);
        image[at * 4 + 3] = logT;
        stops[at] = stop;
      }
    }
  }
}

/* ------------------------------------------------------------ loss */

static const float kWeights[11] = {0.00102838f, 0.00759876f, 0.03600077f, 0.10936069f, 0.21300554f, 0.26601172f,
                                   0.21300554f, 0.10936069f, 0.03600077f, 0.00759876f, 0.00102838f};

static float window_norm(int at, int size) {
  float norm = 0.0f;
  for (int i = at - 5 > 0 ? at - 5 : 0; i <= (at + 5 < size - 1 ? at + 5 : size - 1); ++i) norm += kWeights[i - at + 5];
  return norm;
}

static float unorm(uint8_t b) { return (float)b / 255.0f; }

/* image 4 floats per pixel, target RGBA8; adjoint out 4 floats per pixel;
 * ssimSum and l1Sum in double over the whole image. */
void oracle_loss(const float *image, const uint8_t *target, const OView *v, float lambda, float *adjoint, double *ssimSum,
                 double *l1Sum) {
  const int W = v->width, H = v->height;
  const size_t P = (size_t)W * H;
  float *h = (float *)malloc(P * 15 * sizeof(float));
  float *fields = (float *)malloc(P * 9 * sizeof(float));
  float *h2 = (float *)malloc(P * 9 * sizeof(float));
  /* Horizontal means of x, y, x^2, y^2, xy, normalised. */
  for (int y = 0; y < H; ++y) {
    for (int x = 0; x < W; ++x) {
      float m[5][3] = {{0}};
      float norm = 0.0f;
      for (int u = (x - 5 > 0 ? x - 5 : 0); u <= (x + 5 < W - 1 ? x + 5 : W - 1); ++u) {
        const float w = kWeights[u - x + 5];
        const size_t at = (size_t)y * W + u;
        for (int k = 0; k < 3; ++k) {
          const float a = image[at * 4 + k], b = unorm(target[at * 4 + k]);
          m[0][k] = fmaf(w, a, m[0][k]);
          m[1][k] = fmaf(w, b, m[1][k]);
          m[2][k] = fmaf(w * a, a, m[2][k]);
          m[3][k] = fmaf(w * b, b, m[3][k]);
          m[4][k] = fmaf(w * a, b, m[4][k]);
        }
        norm += w;
      }
      for (int q = 0; q < 5; ++q)
        for (int k = 0; k < 3; ++k) h[((size_t)y * W + x) * 15 + q * 3 + k] = m[q][k] / norm;
    }
  }
  double ssim = 0.0, l1 = 0.0;
  for (int py = 0; py < H; ++py) {
    for (int px = 0; px < W; ++px) {
      const float rowNorm = window_norm(py, H);
      float m[5][3] = {{0}};
      for (int vv = (py - 5 > 0 ? py - 5 : 0); vv <= (py + 5 < H - 1 ? py + 5 : H - 1); ++vv) {
        const float w = kWeights[vv - py + 5];
        for (int q = 0; q < 5; ++q)
          for (int k = 0; k < 3; ++k) m[q][k] = fmaf(w, h[((size_t)vv * W + px) * 15 + q * 3 + k], m[q][k]);
      }
      const float norm = rowNorm * window_norm(px, W);
      const size_t pixel = (size_t)py * W + px;
      float own = 0.0f;
      for (int k = 0; k < 3; ++k) {
        const float mx = m[0][k] / rowNorm, my = m[1][k] / rowNorm;
        const float vx = m[2][k] / rowNorm - mx * mx, vy = m[3][k] / rowNorm - my * my, cxy = m[4][k] / rowNorm - mx * my;
        const float n1 = 2.0f * mx * my + 0.0001f, n2 = 2.0f * cxy + 0.0009f;
        const float d1 = mx * mx + my * my + 0.0001f, d2 = vx + vy + 0.0009f;
        const float s = (n1 * n2) / (d1 * d2);
        own += s;
        const float dMu = 2.0f * my * n2 / (d1 * d2) - s * 2.0f * mx / d1;
        const float dVar = -s / d2;
        const float dCov = 2.0f * n1 / (d1 * d2);
        fields[pixel * 9 + 0 + k] = (dMu - 2.0f * mx * dVar - my * dCov) / norm;
        fields[pixel * 9 + 3 + k] = dVar / norm;
        fields[pixel * 9 + 6 + k] = dCov / norm;
      }
      ssim += own;
    }
  }
  for (int y = 0; y < H; ++y) {
    for (int x = 0; x < W; ++x) {
      float m[9] = {0};
      for (int u = (x - 5 > 0 ? x - 5 : 0); u <= (x + 5 < W - 1 ? x + 5 : W - 1); ++u) {
        const float w = kWeights[u - x + 5];
        for (int j = 0; j < 9; ++j) m[j] = fmaf(w, fields[((size_t)y * W + u) * 9 + j], m[j]);
      }
      memcpy(&h2[((size_t)y * W + x) * 9], m, sizeof m);
    }
  }
  for (int py = 0; py < H; ++py) {
    for (int px = 0; px < W; ++px) {
      float m[9] = {0};
      for (int vv = (py - 5 > 0 ? py - 5 : 0); vv <= (py + 5 < H - 1 ? py + 5 : H - 1); ++vv) {
        const float w = kWeights[vv - py + 5];
        for (int j = 0; j < 9; ++j) m[j] = fmaf(w, h2[((size_t)vv * W + px) * 9 + j], m[j]);
      }
      const size_t pixel = (size_t)py * W + px;
      float own = 0.0f;
      for (int k = 0; k < 3; ++k) {
        const float xv = image[pixel * 4 + k], yv = unorm(target[pixel * 4 + k]);
        const float d = xv - yv;
        own += fabsf(d);
        const float sgn = d > 0.0f ? 1.0f : (d < 0.0f ? -1.0f : 0.0f);
        const float ssimPart = m[0 + k] + 2.0f * xv * m[3 + k] + yv * m[6 + k];
        adjoint[pixel * 4 + k] = ((1.0f - lambda) * sgn - lambda * ssimPart) * v->perPixel;
      }
      adjoint[pixel * 4 + 3] = 0.0f;
      l1 += own;
    }
  }
  *ssimSum = ssim;
  *l1Sum = l1;
  free(h);
  free(fields);
  free(h2);
}

/* ------------------------------------------------------------ backward */

static uint32_t reverse4(uint32_t lane) {
  return ((lane & 1u) << 3) | ((lane & 2u) << 1) | ((lane & 4u) >> 1) | ((lane & 8u) >> 3);
}

/* The reference's reduce_and_add over 32 lanes: 16 shuffles that leave lane l
 * (< 16) with the total of value reverse4(l). g[lane][16] is overwritten. */
static void butterfly(float g[32][16], float total[32]) {
  for (int offset = 1, count = 16; offset <= 8; offset <<= 1, count >>= 1) {
    float next[32][16];
    memcpy(next, g, sizeof next);
    for (int lane = 0; lane < 32; ++lane) {
      const int partner = lane ^ offset;
      const int upper = (lane & offset) != 0, partnerUpper = (partner & offset) != 0;
      for (int i = 0; i < count / 2; ++i) {
        const float keep = upper ? g[lane][i + count / 2] : g[lane][i];
        const float send = partnerUpper ? g[partner][i] : g[partner][i + count / 2];
        next[lane][i] = keep + send;
      }
    }
    memcpy(g, next, sizeof next);
  }
  for (int lane = 0; lane < 32; ++lane) total[lane] = g[lane][0] + g[lane ^ 16][0];
}

/* raw: RAW_STRIDE words per splat, int32 (fixed) or float, zeroed first. Adds
 * each warp's totals in warp order, as one lane per value would. */
void oracle_backward(const float *splats, const uint32_t *entryValues, const uint32_t *ranges, const OView *v,
                     const float bg[3], const float *image, const float *adjoint, const uint32_t *stops, int fixed,
                     void *raw) {
  const int tiles = v->gridW * v->gridH;
  int32_t *rawInt = (int32_t *)raw;
  float *rawFloat = (float *)raw;
  for (int tile = 0; tile < tiles; ++tile) {
    uint32_t tp[4];
    tile_pixels(v, tile, tp);
    const uint32_t first = ranges[tile * 2], end = ranges[tile * 2 + 1];
    (void)first;
    /* Per thread (pixel) state, 256 threads in reference invocation order. */
    float B[256][3], logBehind[256], logTotal[256], A[256][3];
    uint32_t stop[256];
    int inside[256];
    uint32_t tileStop = end;
    for (int t = 0; t < 256; ++t) {
      const uint32_t x = tp[0] + (t & 15), y = tp[1] + (t >> 4);
      inside[t] = x < (uint32_t)v->width && y < (uint32_t)v->height;
      const size_t at = inside[t] ? (size_t)y * v->width + x : 0;
      logTotal[t] = inside[t] ? image[at * 4 + 3] : 0.0f;
      for (int c = 0; c < 3; ++c) {
        A[t][c] = inside[t] ? adjoint[at * 4 + c] : 0.0f;
        B[t][c] = bg[c];
      }
      logBehind[t] = 0.0f;
      stop[t] = inside[t] ? stops[at] : end;
      if (stop[t] < tileStop) tileStop = stop[t];
    }
    for (uint32_t k = tileStop; k < end; ++k) {
      const uint32_t index = entryValues[k];
      const float *s = splats + (size_t)index * 12;
      for (int warp = 0; warp < 8; ++warp) {
        float g[32][16];
        int any = 0;
        memset(g, 0, sizeof g);
        for (int lane = 0; lane < 32; ++lane) {
          const int t = warp * 32 + lane;
          const uint32_t x = tp[0] + (t & 15), y = tp[1] + (t >> 4);
          float dx, dy, power, alpha, ep;
          if (!(k >= stop[t] && splat_at(s, x, y, tp, &dx, &dy, &power, &alpha, &ep))) continue;
          const float logRest = splat_logf(1.0f - alpha);
          const float T = splat_expf((logTotal[t] - logBehind[t]) - logRest);
          const float wA = T * alpha;
          g[lane][6] = wA * A[t][0];
          g[lane][7] = wA * A[t][1];
          g[lane][8] = wA * A[t][2];
          g[lane][9] = wA * v->perPixel;
          const float oe = s[3] * ep;
          if (oe < 0.99f) {
            const float dAlpha = T * fmaf(A[t][2], s[6] - B[t][2], fmaf(A[t][1], s[5] - B[t][1], A[t][0] * (s[4] - B[t][0])));
            g[lane][0] = dAlpha * ep;
            const float dPower = dAlpha * alpha;
            const float qx = s[0], qy = s[1], qz = s[2];
            const float vx = fmaf(qy, dy, qx * dx), vy = fmaf(qz, dy, qy * dx);
            g[lane][1] = dPower * vx;
            g[lane][2] = dPower * vy;
            g[lane][10] = fabsf(g[lane][1]);
            g[lane][11] = fabsf(g[lane][2]);
            const float h = dPower * 0.5f;
            g[lane][3] = h * vx * vx;
            g[lane][4] = h * vx * vy;
            g[lane][5] = h * vy * vy;
          }
          any = 1;
          for (int c = 0; c < 3; ++c) B[t][c] = fmaf(alpha, s[4 + c] - B[t][c], B[t][c]);
          logBehind[t] = logBehind[t] + logRest;
        }
        if (!any) continue;
        float total[32];
        butterfly(g, total);
        for (int lane = 0; lane < 16; ++lane) {
          const uint32_t value = reverse4((uint32_t)lane);
          if (value >= RAW_PER_SPLAT || total[lane] == 0.0f) continue;
          const size_t at = (size_t)index * RAW_STRIDE + value;
          if (fixed) {
            rawInt[at] += (int32_t)lrintf(clampf(total[lane] * v->fixedScale, -1.0e9f, 1.0e9f));
          } else {
            rawFloat[at] += total[lane];
          }
        }
      }
    }
  }
}

/* ------------------------------------------------------------ deterministic math */

/* splat_expf and splat_logf on the host, for the GPU bit-for-bit check. */
void oracle_detmath(const float *in, float *outExp, float *outLog, int n) {
  for (int i = 0; i < n; ++i) {
    outExp[i] = splat_expf(in[i]);
    outLog[i] = in[i] > 0.0f ? splat_logf(in[i]) : 0.0f;
  }
}
