// CGC files: the reference's compressed splat format for viewing over the
// network (save_cgc / load_cgc, src/splat/cgc.hpp:41-50, cgc.cpp), version 2
// written and versions 1 and 2 read. A file holds three importance layers,
// each with its own precision: positions on a symlog grid around the scene's
// median, stored as gaps between Morton codes in byte planes; canonical axes
// (log scales descending, quaternion with the largest component first and
// left out); YCoCg DC colour over a robust range; opacity; the higher SH
// bands as labels into one k-means codebook per layer. Every byte column is
// its own LZMA "alone" stream (lc = lp = pb = 0).
//
// Writing: the per-splat work runs on the GPU. Validation, importance and the
// canonical axes are one kernel over the cloud; the scene centre and radius,
// the importance cuts and the colour ranges are order statistics taken from
// this library's radix sort of order-preserving float keys; each layer's
// Morton order is a 64-bit radix sort; all byte columns of a layer come out of
// one kernel. The codebook is Lloyd's k-means on the GPU: one thread per
// point against shared-memory tiles of centres, then the weighted means per
// centre summed in FP64 in a fixed order over the points sorted by label, so
// that a cloud always gives the same file. Column compression runs on host
// threads. Reading is host code: parsing, LZMA and the dequantisation, in the
// reference's arithmetic, so a file decodes to the same values with either
// reader.
//
// The format's constants, layer parameters, header layout and quantisation
// rules are the reference's (they are the file format); the encoder's search
// for the codebook is this library's own, so the label and codebook columns
// differ from the reference writer's while every file stays readable by both.
#include <dlfcn.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iterator>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "sort.cuh"
#include "splat_b200.h"

namespace sb {

void set_last_error(const char *message);

namespace cgc {

constexpr char kMagic[4] = {'C', 'G', 'C', '\0'};
constexpr uint32_t kVersion = 2;
constexpr float kShC0 = 0.28209479177387814f;
constexpr float kRotationRange = 0.70710678f; // the three smaller quaternion components lie within 1/sqrt(2)
constexpr float kMinLogScale = -9.f;          // thinner axes are stored at this log scale
constexpr float kCodebookStep = 0.02f;
constexpr uint32_t kMaxCodebook = 65536;
constexpr int kLayers = 3;

// Layer precision (src/splat/cgc.cpp layer_params): importance percentile the
// layer starts at, bits of position, rotation, opacity and colour, scale steps,
// and splats per codebook entry.
struct LayerParams {
  double fromPercentile;
  uint32_t posBits, rotBits, alphaBits, colorBits[3];
  float scaleStep, gap1Step, gap2Step;
  uint32_t splatsPerCode;
};

inline std::array<LayerParams, kLayers> layer_params(int preset) {
  const bool small = preset == SPLAT_CGC_SMALL;
  return {{{small ? 95.0 : 80.0, 15, 8, 7, {7, 7, 7}, 0.05f, 0.05f, 0.1f, 16},
           {small ? 70.0 : 40.0, 14, 6, 6, {6, 6, 6}, 0.1f, 0.1f, 0.2f, 120},
           {0.0, 13, 5, 5, {6, 5, 5}, 0.15f, 0.15f, 0.3f, 500}}};
}

// A layer's header in the file: 23 little-endian 4-byte fields.
struct LayerHeader {
  uint32_t count = 0, posBits = 0, rotBits = 0, alphaBits = 0;
  uint32_t colorBits[3] = {0, 0, 0};
  uint32_t codebookSize = 0;
  float posLo[3] = {0.f, 0.f, 0.f};
  float posStep = 1.f, scaleLo = kMinLogScale, scaleStep = 1.f, gap1Step = 1.f, gap2Step = 1.f;
  float colorLo[3] = {0.f, 0.f, 0.f}, colorStep[3] = {0.f, 0.f, 0.f};
  float codebookStep = kCodebookStep;
};
static_assert(sizeof(LayerHeader) == 23 * 4, "the layer header is 23 words");

// Bit i of v to bit 3i, for the low 21 bits, and back.
__host__ __device__ inline uint64_t spread3(uint32_t v) {
  uint64_t x = v & 0x1FFFFFu;
  x = (x | x << 32) & 0x1F00000000FFFFull;
  x = (x | x << 16) & 0x1F0000FF0000FFull;
  x = (x | x << 8) & 0x100F00F00F00F00Full;
  x = (x | x << 4) & 0x10C30C30C30C30C3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}
inline uint32_t compact3(uint64_t x) {
  x &= 0x1249249249249249ull;
  x = (x ^ (x >> 2)) & 0x10C30C30C30C30C3ull;
  x = (x ^ (x >> 4)) & 0x100F00F00F00F00Full;
  x = (x ^ (x >> 8)) & 0x1F0000FF0000FFull;
  x = (x ^ (x >> 16)) & 0x1F00000000FFFFull;
  x = (x ^ (x >> 32)) & 0x1FFFFFull;
  return (uint32_t)x;
}
__host__ __device__ inline uint64_t morton(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | spread3(y) << 1 | spread3(z) << 2;
}

__host__ __device__ inline uint32_t zigzag(int v) { return v >= 0 ? (uint32_t)v * 2u : (uint32_t)(-v) * 2u - 1u; }
inline int unzigzag(uint32_t z) { return (z & 1u) != 0u ? -(int)((z + 1u) / 2u) : (int)(z / 2u); }

// YCoCg with the format's simple inverse.
__host__ __device__ inline void to_ycocg(float r, float g, float b, float out[3]) {
  out[0] = 0.25f * r + 0.5f * g + 0.25f * b;
  out[1] = r - b;
  out[2] = g - 0.5f * (r + b);
}
inline void from_ycocg(float y, float co, float cg, float out[3]) {
  const float t = y - 0.5f * cg;
  out[0] = t + 0.5f * co;
  out[1] = y + 0.5f * cg;
  out[2] = t - 0.5f * co;
}

// The canonical axes of a splat (cgc_detail::canonicalize_axes,
// src/splat/cgc.cpp): log scales in descending order (ties keep their order),
// the rotation's columns permuted with them and the third negated if that
// made a reflection; back to a quaternion by Shepperd's method; then, since
// flipping two axes leaves the ellipsoid unchanged and multiplies the
// quaternion by i, j or k, the largest component is moved into w, made
// non-negative. A zero quaternion is the identity. Every operation is a single
// IEEE operation in a fixed order (no fused multiply-adds), so host and device
// give the same bits.
__host__ __device__ inline void canonicalize(float s[3], float q[4]) {
  const float norm = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  if (!(norm > 0.f)) {
    q[0] = 1.f;
    q[1] = q[2] = q[3] = 0.f;
  } else {
    for (int a = 0; a < 4; ++a) q[a] = q[a] / norm;
  }
  const float w = q[0], x = q[1], y = q[2], z = q[3];
  // Rows are the rotation's columns: the ellipsoid's axes.
  float r[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y)},
                   {2 * (x * y - w * z), 1 - 2 * (x * x + z * z), 2 * (y * z + w * x)},
                   {2 * (x * z + w * y), 2 * (y * z - w * x), 1 - 2 * (x * x + y * y)}};
  // A stable three-element sort by descending scale.
  int o[3] = {0, 1, 2};
  for (int i = 1; i < 3; ++i) {
    const int v = o[i];
    int j = i - 1;
    while (j >= 0 && s[o[j]] < s[v]) {
      o[j + 1] = o[j];
      --j;
    }
    o[j + 1] = v;
  }
  const float sorted[3] = {s[o[0]], s[o[1]], s[o[2]]};
  float m[3][3];
  for (int i = 0; i < 3; ++i)
    for (int c = 0; c < 3; ++c) m[i][c] = r[o[i]][c];
  for (int i = 0; i < 3; ++i) s[i] = sorted[i];
  const float det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[1][0] * (m[0][1] * m[2][2] - m[0][2] * m[2][1]) +
                    m[2][0] * (m[0][1] * m[1][2] - m[0][2] * m[1][1]);
  if (det < 0.f)
    for (int c = 0; c < 3; ++c) m[2][c] = -m[2][c];
  const float trace = m[0][0] + m[1][1] + m[2][2];
  float t[4];
  if (trace > 0.f) {
    const float k = sqrtf(trace + 1.f) * 2.f;
    t[0] = k / 4.f;
    t[1] = (m[1][2] - m[2][1]) / k;
    t[2] = (m[2][0] - m[0][2]) / k;
    t[3] = (m[0][1] - m[1][0]) / k;
  } else if (m[0][0] > m[1][1] && m[0][0] > m[2][2]) {
    const float k = sqrtf(1.f + m[0][0] - m[1][1] - m[2][2]) * 2.f;
    t[0] = (m[1][2] - m[2][1]) / k;
    t[1] = k / 4.f;
    t[2] = (m[1][0] + m[0][1]) / k;
    t[3] = (m[2][0] + m[0][2]) / k;
  } else if (m[1][1] > m[2][2]) {
    const float k = sqrtf(1.f + m[1][1] - m[0][0] - m[2][2]) * 2.f;
    t[0] = (m[2][0] - m[0][2]) / k;
    t[1] = (m[1][0] + m[0][1]) / k;
    t[2] = k / 4.f;
    t[3] = (m[2][1] + m[1][2]) / k;
  } else {
    const float k = sqrtf(1.f + m[2][2] - m[0][0] - m[1][1]) * 2.f;
    t[0] = (m[0][1] - m[1][0]) / k;
    t[1] = (m[2][0] + m[0][2]) / k;
    t[2] = (m[2][1] + m[1][2]) / k;
    t[3] = k / 4.f;
  }
  int largest = 0;
  for (int a = 1; a < 4; ++a)
    if (fabsf(t[a]) > fabsf(t[largest])) largest = a;
  switch (largest) {
  case 0: q[0] = t[0]; q[1] = t[1]; q[2] = t[2]; q[3] = t[3]; break;
  case 1: q[0] = -t[1]; q[1] = t[0]; q[2] = t[3]; q[3] = -t[2]; break;
  case 2: q[0] = -t[2]; q[1] = -t[3]; q[2] = t[0]; q[3] = t[1]; break;
  default: q[0] = -t[3]; q[1] = t[2]; q[2] = -t[1]; q[3] = t[0]; break;
  }
  if (q[0] < 0.f)
    for (int a = 0; a < 4; ++a) q[a] = -q[a];
}

// ------------------------------------------------------------------- LZMA

// liblzma, loaded at run time (the library is part of the system; its
// headers are not needed): the "alone" encoder from a preset with lc, lp, pb
// set, and the decoder. Only the leading fields of liblzma's stream and
// option structures are used; the option offsets are checked against what
// the preset call writes before the first use.
struct Lzma {
  unsigned char (*preset)(void *, uint32_t) = nullptr;
  int (*encoder)(void *, const void *) = nullptr;
  int (*decoder)(void *, uint64_t) = nullptr;
  int (*code)(void *, int) = nullptr;
  void (*end)(void *) = nullptr;
};

const Lzma &lzma() {
  static std::once_flag once;
  static Lzma api;
  static std::string failure;
  std::call_once(once, [] {
    void *h = dlopen("liblzma.so.5", RTLD_NOW | RTLD_LOCAL);
    if (h == nullptr) {
      failure = "liblzma.so.5 cannot be loaded";
      return;
    }
    api.preset = reinterpret_cast<unsigned char (*)(void *, uint32_t)>(dlsym(h, "lzma_lzma_preset"));
    api.encoder = reinterpret_cast<int (*)(void *, const void *)>(dlsym(h, "lzma_alone_encoder"));
    api.decoder = reinterpret_cast<int (*)(void *, uint64_t)>(dlsym(h, "lzma_alone_decoder"));
    api.code = reinterpret_cast<int (*)(void *, int)>(dlsym(h, "lzma_code"));
    api.end = reinterpret_cast<void (*)(void *)>(dlsym(h, "lzma_end"));
    if (!api.preset || !api.encoder || !api.decoder || !api.code || !api.end) failure = "liblzma.so.5 lacks an entry point";
  });
  if (!failure.empty()) throw std::runtime_error(failure);
  return api;
}

struct alignas(16) LzmaStream {
  const uint8_t *nextIn = nullptr;
  size_t availIn = 0;
  uint64_t totalIn = 0;
  uint8_t *nextOut = nullptr;
  size_t availOut = 0;
  uint64_t totalOut = 0;
  unsigned char opaque[464] = {}; // the rest of liblzma's structure
};

constexpr int kLzmaOk = 0, kLzmaStreamEnd = 1, kLzmaBufError = 10, kLzmaFinish = 3;

// Runs the stream to its end over `input`, output growing up to `limit` bytes.
void lzma_run(LzmaStream &s, const uint8_t *input, size_t size, std::vector<uint8_t> &out, size_t limit) {
  s.nextIn = input;
  s.availIn = size;
  for (;;) {
    if (s.availOut == 0) {
      const size_t used = out.size();
      if (used >= limit) throw std::runtime_error("LZMA data is longer than expected");
      out.resize(std::min(limit, std::max<size_t>(used * 2, size_t{1} << 16)));
      s.nextOut = out.data() + used;
      s.availOut = out.size() - used;
    }
    const int r = lzma().code(&s, kLzmaFinish);
    if (r == kLzmaStreamEnd) break;
    if (r == kLzmaBufError) throw std::runtime_error("LZMA data is truncated");
    if (r != kLzmaOk) throw std::runtime_error("LZMA error " + std::to_string(r));
  }
  out.resize(out.size() - s.availOut);
}

std::vector<uint8_t> lzma_pack(const uint8_t *data, size_t size, int level, bool extreme, int lc, int lp, int pb) {
  alignas(16) unsigned char options[256] = {};
  if (lzma().preset(options, (uint32_t)level | (extreme ? 0x80000000u : 0u)) != 0)
    throw std::invalid_argument("invalid LZMA preset " + std::to_string(level));
  uint32_t word[3];
  std::memcpy(word, options + 20, 12);
  if (word[0] != 3u || word[1] != 0u || word[2] != 2u) throw std::runtime_error("liblzma's option layout is not the expected one");
  const uint32_t lcs[3] = {(uint32_t)lc, (uint32_t)lp, (uint32_t)pb};
  std::memcpy(options + 20, lcs, 12);
  LzmaStream s;
  if (lzma().encoder(&s, options) != kLzmaOk) throw std::runtime_error("cannot start the LZMA encoder");
  std::vector<uint8_t> out;
  try {
    lzma_run(s, data, size, out, SIZE_MAX);
  } catch (...) {
    lzma().end(&s);
    throw;
  }
  lzma().end(&s);
  return out;
}

std::vector<uint8_t> lzma_unpack(const uint8_t *stream, size_t size, size_t expected) {
  LzmaStream s;
  if (lzma().decoder(&s, UINT64_MAX) != kLzmaOk) throw std::runtime_error("cannot start the LZMA decoder");
  std::vector<uint8_t> out;
  try {
    lzma_run(s, stream, size, out, expected + 1); // one byte over: longer data is caught
  } catch (...) {
    lzma().end(&s);
    throw;
  }
  lzma().end(&s);
  if (out.size() != expected)
    throw std::runtime_error("LZMA data has " + std::to_string(out.size()) + " bytes, expected " + std::to_string(expected));
  return out;
}

// Runs body(i) for i < count on the host's threads.
template <class F> void on_threads(size_t count, F &&body) {
  const unsigned threads = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), (unsigned)std::max<size_t>(count, 1)));
  std::atomic<size_t> next{0};
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; ++t)
    pool.emplace_back([&] {
      for (size_t i; (i = next.fetch_add(1)) < count;) body(i);
    });
  for (auto &t : pool) t.join();
}


// ----------------------------------------------------------------- reading

struct Cloud {
  uint32_t count = 0;
  int degree = 0;
  std::vector<float> positions, scales, rotations, opacities, sh;
  void resize(uint32_t n, int d) {
    count = n;
    degree = d;
    const size_t coeffs = (size_t)(d + 1) * (d + 1);
    positions.assign((size_t)n * 3, 0.f);
    scales.assign((size_t)n * 3, 0.f);
    rotations.assign((size_t)n * 4, 0.f);
    opacities.assign(n, 0.f);
    sh.assign((size_t)n * 3 * coeffs, 0.f);
  }
};

// Bounds-checked reads from a byte span.
class Reader {
public:
  Reader(const uint8_t *data, size_t size) : data_(data), size_(size) {}
  const uint8_t *take(size_t n) {
    if (n > size_ - pos_) throw std::runtime_error("file is shorter than its header says");
    const uint8_t *p = data_ + pos_;
    pos_ += n;
    return p;
  }
  template <class T> T get() {
    T v;
    std::memcpy(&v, take(sizeof(T)), sizeof(T));
    return v;
  }
  size_t remaining() const { return size_ - pos_; }

private:
  const uint8_t *data_;
  size_t size_, pos_ = 0;
};

inline float symexp(float y) { return std::copysign(std::expm1(std::fabs(y)), y); }

// Column sizes of a layer, in file order: position planes, 3 rotation, 3
// scale, 3 colour, opacity; then, with higher SH bands, 2 label bytes per
// splat and 2 bytes per codebook value.
std::vector<size_t> column_sizes(const LayerHeader &h, size_t dims) {
  std::vector<size_t> sizes;
  if (h.count == 0) return sizes;
  sizes.assign((h.posBits * 3 + 7) / 8 + 10, h.count);
  if (dims > 0) {
    sizes.push_back(h.count);
    sizes.push_back(h.count);
    sizes.push_back((size_t)h.codebookSize * dims);
    sizes.push_back((size_t)h.codebookSize * dims);
  }
  return sizes;
}

void decode_layer(const LayerHeader &h, const std::vector<std::vector<uint8_t>> &col, const float center[3], float radius,
                  size_t first, Cloud &cloud) {
  const size_t n = h.count;
  if (n == 0) return;
  const size_t coeffs = (size_t)(cloud.degree + 1) * (cloud.degree + 1);
  const size_t planes = (h.posBits * 3 + 7) / 8;
  uint64_t code = 0;
  for (size_t j = 0; j < n; ++j) {
    uint64_t gap = 0;
    for (size_t p = 0; p < planes; ++p) gap |= (uint64_t)col[p][j] << (8 * p);
    code += gap;
    const uint32_t q[3] = {compact3(code), compact3(code >> 1), compact3(code >> 2)};
    for (int a = 0; a < 3; ++a)
      cloud.positions[(first + j) * 3 + a] = symexp(h.posLo[a] + (float)q[a] * h.posStep) * radius + center[a];
  }
  const size_t rot = planes, sca = planes + 3, colr = planes + 6, alp = planes + 9;
  const float rotationStep = kRotationRange / (float)((1 << (h.rotBits - 1)) - 1);
  const float levels = (float)(1u << h.alphaBits);
  for (size_t j = 0; j < n; ++j) {
    const size_t out = first + j;
    float sum = 0.f;
    for (int a = 0; a < 3; ++a) {
      const float v = (float)unzigzag(col[rot + a][j]) * rotationStep;
      cloud.rotations[out * 4 + a + 1] = v;
      sum += v * v;
    }
    cloud.rotations[out * 4] = std::sqrt(std::max(0.f, 1.f - sum));
    const float s0 = h.scaleLo + (float)col[sca][j] * h.scaleStep;
    const float s1 = s0 - (float)col[sca + 1][j] * h.gap1Step;
    const float s2 = s1 - (float)col[sca + 2][j] * h.gap2Step;
    cloud.scales[out * 3] = s0;
    cloud.scales[out * 3 + 1] = s1;
    cloud.scales[out * 3 + 2] = s2;
    float y[3], rgb[3];
    for (int a = 0; a < 3; ++a) y[a] = h.colorLo[a] + (float)col[colr + a][j] * h.colorStep[a];
    from_ycocg(y[0], y[1], y[2], rgb);
    for (int a = 0; a < 3; ++a) cloud.sh[out * coeffs * 3 + a] = (rgb[a] - 0.5f) / kShC0;
    const float alpha = ((float)col[alp][j] + 0.5f) / levels;
    cloud.opacities[out] = std::log(alpha / (1.f - alpha));
  }
  const size_t dims = (coeffs - 1) * 3;
  if (dims == 0) return;
  const size_t lab = alp + 1, book = h.codebookSize;
  std::vector<float> rgbBook(book * dims);
  for (size_t t = 0; t < book; ++t) {
    for (size_t a = 0; a < dims; a += 3) {
      float e[3], rgb[3];
      for (int k = 0; k < 3; ++k) {
        const uint32_t z = (uint32_t)col[lab + 2][(a + k) * book + t] | (uint32_t)col[lab + 3][(a + k) * book + t] << 8;
        e[k] = (float)unzigzag(z) * h.codebookStep;
      }
      from_ycocg(e[0], e[1], e[2], rgb);
      std::copy(rgb, rgb + 3, &rgbBook[t * dims + a]);
    }
  }
  for (size_t j = 0; j < n; ++j) {
    const size_t label = (size_t)col[lab][j] | (size_t)col[lab + 1][j] << 8;
    if (label >= book) throw std::runtime_error("SH label outside the codebook");
    std::copy_n(&rgbBook[label * dims], dims, &cloud.sh[((first + j) * coeffs + 1) * 3]);
  }
}

// Version 1 (one LZMA stream of byte planes with per-256-splat boxes; the
// reference still reads it).
Cloud load_v1(const uint8_t *bytes, size_t size) {
  constexpr size_t kHeader = 16, kChunk = 256;
  constexpr int kShBits[4] = {0, 5, 4, 4};
  if (size < kHeader) throw std::runtime_error("file is shorter than its header says");
  uint64_t payloadSize;
  std::memcpy(&payloadSize, bytes + 8, 8);
  const std::vector<uint8_t> payload = lzma_unpack(bytes + kHeader, size - kHeader, (size_t)payloadSize);
  Reader r(payload.data(), payload.size());
  const uint32_t n = r.get<uint32_t>();
  float colorMin[3], colorMax[3], shRange[3];
  for (float &v : colorMin) v = r.get<float>();
  for (float &v : colorMax) v = r.get<float>();
  for (float &v : shRange) v = r.get<float>();
  const auto planes = [&](size_t count) {
    const uint8_t *p = r.take(count * 4);
    std::vector<uint32_t> v(count, 0u);
    for (size_t b = 0; b < 4; ++b)
      for (size_t i = 0; i < count; ++i) v[i] |= (uint32_t)p[b * count + i] << (8 * b);
    return v;
  };
  const auto unsigned_value = [](uint32_t q, float lo, float hi, int bits) {
    if (!(hi > lo)) return lo;
    return lo + (float)q / (float)((1u << bits) - 1) * (hi - lo);
  };
  const auto symmetric_value = [](uint32_t q, float range, int bits) {
    const int h = (1 << (bits - 1)) - 1;
    return (float)((int)q - h) / (float)h * range;
  };
  const size_t chunks = (n + kChunk - 1) / kChunk;
  const std::vector<uint32_t> table = planes(chunks * 12);
  const auto bound = [&](size_t j, size_t field) {
    float f;
    std::memcpy(&f, &table[j / kChunk * 12 + field], 4);
    return f;
  };
  const std::vector<uint32_t> pos = planes(n), rots = planes(n);
  const uint8_t *scaleCols[3], *rgba[4];
  for (auto &c : scaleCols) c = r.take(n);
  for (auto &c : rgba) c = r.take(n);
  const uint8_t *degrees = r.take(n);
  int maxDegree = 0;
  for (uint32_t j = 0; j < n; ++j) {
    if (degrees[j] > 3) throw std::runtime_error("SH degree above 3");
    maxDegree = std::max(maxDegree, (int)degrees[j]);
  }
  Cloud cloud;
  cloud.resize(n, maxDegree);
  const size_t coeffs = (size_t)(maxDegree + 1) * (maxDegree + 1);
  for (size_t j = 0; j < n; ++j) {
    cloud.positions[j * 3] = unsigned_value(pos[j] & 0x7FFu, bound(j, 0), bound(j, 3), 11);
    cloud.positions[j * 3 + 1] = unsigned_value(pos[j] >> 11 & 0x3FFu, bound(j, 1), bound(j, 4), 10);
    cloud.positions[j * 3 + 2] = unsigned_value(pos[j] >> 21, bound(j, 2), bound(j, 5), 11);
    // The quaternion: the three smaller components in 10 bits each, the
    // largest's index in the top two bits and its value from the unit norm.
    const uint32_t packed = rots[j];
    const int largest = (int)(packed >> 30);
    float q[4] = {0.f, 0.f, 0.f, 0.f}, sum = 0.f;
    int shift = 0;
    for (int i = 0; i < 4; ++i) {
      if (i == largest) continue;
      q[i] = symmetric_value((packed >> shift) & 0x3FFu, kRotationRange, 10);
      sum += q[i] * q[i];
      shift += 10;
    }
    q[largest] = std::sqrt(std::max(0.f, 1.f - sum));
    const float norm = std::sqrt(sum + q[largest] * q[largest]);
    for (int i = 0; i < 4; ++i) cloud.rotations[j * 4 + i] = q[i] / norm;
    for (int a = 0; a < 3; ++a) cloud.scales[j * 3 + a] = unsigned_value(scaleCols[a][j], bound(j, 6 + a), bound(j, 9 + a), 8);
    for (int c = 0; c < 3; ++c)
      cloud.sh[j * coeffs * 3 + c] = (unsigned_value(rgba[c][j], colorMin[c], colorMax[c], 8) - 0.5f) / kShC0;
    const float alpha = ((float)rgba[3][j] + 0.5f) / 256.f;
    cloud.opacities[j] = std::log(alpha / (1.f - alpha));
  }
  for (int band = 1; band <= maxDegree; ++band) {
    std::vector<size_t> members;
    for (size_t j = 0; j < n; ++j)
      if ((int)degrees[j] >= band) members.push_back(j);
    for (int k = band * band; k < (band + 1) * (band + 1); ++k)
      for (int c = 0; c < 3; ++c) {
        const uint8_t *column = r.take(members.size());
        for (size_t m = 0; m < members.size(); ++m)
          cloud.sh[(members[m] * coeffs + (size_t)k) * 3 + c] = symmetric_value(column[m], shRange[band - 1], kShBits[band]);
      }
  }
  if (r.remaining() != 0) throw std::runtime_error("payload has unexpected trailing data");
  return cloud;
}

Cloud load(const std::string &path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw std::runtime_error("Cannot open '" + path + "'");
  const std::vector<uint8_t> file{std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>()};
  if (file.size() < 8 || std::memcmp(file.data(), kMagic, 4) != 0) throw std::runtime_error(path + ": not a CGC file");
  try {
    Reader r(file.data(), file.size());
    r.take(4);
    const uint32_t version = r.get<uint32_t>();
    if (version == 1) return load_v1(file.data(), file.size());
    if (version != kVersion) throw std::runtime_error("unsupported CGC version " + std::to_string(version));
    const uint32_t n = r.get<uint32_t>(), degree = r.get<uint32_t>(), layers = r.get<uint32_t>();
    if (degree > 3) throw std::runtime_error("SH degree above 3");
    if (layers > 16) throw std::runtime_error("too many layers");
    float center[3];
    for (float &v : center) v = r.get<float>();
    const float radius = r.get<float>();
    const size_t dims = 3 * (((size_t)degree + 1) * (degree + 1) - 1);
    std::vector<LayerHeader> headers(layers);
    uint64_t total = 0;
    for (LayerHeader &h : headers) {
      h = r.get<LayerHeader>();
      total += h.count;
      if (h.count == 0) continue;
      bool colourOk = true;
      for (uint32_t b : h.colorBits) colourOk = colourOk && b >= 1 && b <= 8;
      if (h.posBits < 1 || h.posBits > 21 || h.rotBits < 2 || h.rotBits > 8 || h.alphaBits < 1 || h.alphaBits > 8 || !colourOk ||
          h.codebookSize > kMaxCodebook || (dims > 0 && h.codebookSize == 0))
        throw std::runtime_error("invalid layer header");
    }
    if (total != n) throw std::runtime_error("layer sizes do not add up");
    struct Job {
      const uint8_t *stream;
      size_t streamBytes, size;
      std::vector<uint8_t> *out;
    };
    std::vector<std::vector<std::vector<uint8_t>>> columns(layers);
    std::vector<Job> jobs;
    for (uint32_t l = 0; l < layers; ++l) {
      const std::vector<size_t> sizes = column_sizes(headers[l], dims);
      columns[l].resize(sizes.size());
      for (size_t c = 0; c < sizes.size(); ++c) {
        const uint32_t packed = r.get<uint32_t>();
        jobs.push_back({r.take(packed), packed, sizes[c], &columns[l][c]});
      }
    }
    if (r.remaining() != 0) throw std::runtime_error("file has unexpected trailing data");
    std::mutex failureLock;
    std::string failure;
    on_threads(jobs.size(), [&](size_t i) {
      try {
        *jobs[i].out = lzma_unpack(jobs[i].stream, jobs[i].streamBytes, jobs[i].size);
      } catch (const std::exception &e) {
        std::lock_guard<std::mutex> g(failureLock);
        failure = e.what();
      }
    });
    if (!failure.empty()) throw std::runtime_error(failure);
    Cloud cloud;
    cloud.resize(n, (int)degree);
    size_t first = 0;
    for (uint32_t l = 0; l < layers; ++l) {
      decode_layer(headers[l], columns[l], center, radius, first, cloud);
      first += headers[l].count;
    }
    return cloud;
  } catch (const std::exception &e) {
    throw std::runtime_error(path + ": " + e.what());
  }
}

// ----------------------------------------------------------------- writing

#define CGC_CUDA(call)                                                                                \
  do {                                                                                                \
    const cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string("CUDA: ") + cudaGetErrorString(e_)); \
  } while (0)

// A device allocation that frees itself.
class Dev {
public:
  Dev() = default;
  explicit Dev(size_t bytes) { resize(bytes); }
  Dev(const Dev &) = delete;
  Dev &operator=(const Dev &) = delete;
  ~Dev() {
    if (p_ != nullptr) cudaFree(p_);
  }
  // Grows only (a sort's temporaries are reused by the next sort on the
  // same stream without being freed under its kernels).
  void resize(size_t bytes) {
    if (p_ != nullptr && bytes <= bytes_) return;
    if (p_ != nullptr) cudaFree(p_);
    p_ = nullptr;
    CGC_CUDA(cudaMalloc(&p_, std::max<size_t>(bytes, 16)));
    bytes_ = std::max<size_t>(bytes, 16);
  }
  template <class T = void> T *get() const { return static_cast<T *>(p_); }

private:
  void *p_ = nullptr;
  size_t bytes_ = 0;
};

// Order-preserving unsigned keys of floats (negative values reversed).
__host__ __device__ inline uint32_t float_key(float f) {
#ifdef __CUDA_ARCH__
  const uint32_t u = __float_as_uint(f);
#else
  uint32_t u;
  std::memcpy(&u, &f, 4);
#endif
  return (u & 0x80000000u) != 0u ? ~u : u | 0x80000000u;
}
inline float key_float(uint32_t k) {
  const uint32_t u = (k & 0x80000000u) != 0u ? k & 0x7FFFFFFFu : ~k;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

__device__ inline float sigmoid_d(float x) { return 1.f / (1.f + expf(-x)); }
__device__ inline float symlog_d(float t) { return copysignf(log1pf(fabsf(t)), t); }

// Per splat: the finite check, the position keys (for the median), the
// importance (log opacity plus the two largest log scales) and its key, the
// canonical axes, the YCoCg DC colour, the opacity and the codebook weight
// (opacity times the two largest axes' area).
__global__ void k_splats(uint32_t n, uint32_t coeffs, const float *__restrict__ pos, const float *__restrict__ scales,
                         const float *__restrict__ rot, const float *__restrict__ op, const float *__restrict__ sh,
                         uint32_t *bad, uint32_t *axisKeys, float *importance, uint32_t *importanceKeys, float *canon,
                         float *ycocg, float *sig, float *weight) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bool finite = true;
  float p[3], s[3], q[4];
  for (int a = 0; a < 3; ++a) {
    p[a] = pos[(size_t)i * 3 + a];
    s[a] = scales[(size_t)i * 3 + a];
    finite = finite && isfinite(p[a]) && isfinite(s[a]);
  }
  for (int a = 0; a < 4; ++a) {
    q[a] = rot[(size_t)i * 4 + a];
    finite = finite && isfinite(q[a]);
  }
  const float o = op[i];
  finite = finite && isfinite(o);
  const float *c = sh + (size_t)i * coeffs * 3;
  for (uint32_t k = 0; k < coeffs * 3; ++k) finite = finite && isfinite(c[k]);
  if (!finite) atomicOr(bad, 1u);
  for (int a = 0; a < 3; ++a) axisKeys[(size_t)a * n + i] = float_key(p[a]);
  // The scales ascending: a[2] the largest, a[1] the middle one.
  float lo = fminf(s[0], s[1]), hi = fmaxf(s[0], s[1]);
  const float top = fmaxf(hi, s[2]), mid = fmaxf(lo, fminf(hi, s[2]));
  const float g = sigmoid_d(o);
  const float imp = logf(fmaxf(g, 1e-30f)) + top + mid;
  importance[i] = imp;
  importanceKeys[i] = float_key(imp);
  sig[i] = g;
  weight[i] = g * expf(fminf(fmaxf(top + mid, -30.f), 30.f)) + 1e-12f;
  canonicalize(s, q);
  for (int a = 0; a < 3; ++a) canon[(size_t)i * 7 + a] = s[a];
  for (int a = 0; a < 4; ++a) canon[(size_t)i * 7 + 3 + a] = q[a];
  float y[3];
  to_ycocg(kShC0 * c[0] + 0.5f, kShC0 * c[1] + 0.5f, kShC0 * c[2] + 0.5f, y);
  for (int a = 0; a < 3; ++a) ycocg[(size_t)i * 3 + a] = y[a];
}

__global__ void k_distance_keys(uint32_t n, const float *__restrict__ pos, float cx, float cy, float cz, uint32_t *keys,
                                uint32_t *values) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float dx = pos[(size_t)i * 3] - cx, dy = pos[(size_t)i * 3 + 1] - cy, dz = pos[(size_t)i * 3 + 2] - cz;
  keys[i] = float_key(sqrtf(dx * dx + dy * dy + dz * dz));
  values[i] = i;
}

__global__ void k_iota(uint32_t n, uint32_t *values) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) values[i] = i;
}

// The layer of each splat: the first whose cut its importance reaches.
__global__ void k_layer_keys(uint32_t n, const float *__restrict__ importance, float cut0, float cut1, uint32_t *keys,
                             uint32_t *values, uint32_t *counts) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float v = importance[i];
  const uint32_t l = v < cut0 ? (v < cut1 ? 2u : 1u) : 0u;
  keys[i] = l;
  values[i] = i;
  atomicAdd(&counts[l], 1u);
}

// A layer's members (splat indices, in index order): their symlog positions,
// the order-preserving keys of the per-axis extremes and of the largest log
// scale, and their colour keys (for the robust ranges).
__global__ void k_layer_prepare(uint32_t m, const uint32_t *__restrict__ members, const float *__restrict__ pos,
                                const float *__restrict__ scales, const float *__restrict__ ycocg, float cx, float cy, float cz,
                                float radius, float *warped, uint32_t *extremes, uint32_t *colourKeys, uint32_t *colourValues) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const uint32_t i = members[j];
  const float centre[3] = {cx, cy, cz};
  for (int a = 0; a < 3; ++a) {
    const float w = symlog_d((pos[(size_t)i * 3 + a] - centre[a]) / radius);
    warped[(size_t)j * 3 + a] = w;
    atomicMin(&extremes[a], float_key(w));
    atomicMax(&extremes[3 + a], float_key(w));
  }
  float big = scales[(size_t)i * 3];
  big = fmaxf(big, scales[(size_t)i * 3 + 1]);
  big = fmaxf(big, scales[(size_t)i * 3 + 2]);
  atomicMax(&extremes[6], float_key(big));
  for (int a = 0; a < 3; ++a) {
    colourKeys[(size_t)a * m + j] = float_key(ycocg[(size_t)i * 3 + a]);
    colourValues[(size_t)a * m + j] = j;
  }
}

__global__ void k_morton(uint32_t m, const float *__restrict__ warped, float lo0, float lo1, float lo2, float step,
                         unsigned long long *codes, uint32_t *values) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const float lo[3] = {lo0, lo1, lo2};
  uint32_t q[3];
  for (int a = 0; a < 3; ++a) q[a] = (uint32_t)roundf((warped[(size_t)j * 3 + a] - lo[a]) / step);
  codes[j] = morton(q[0], q[1], q[2]);
  values[j] = j;
}

struct ColumnArgs {
  uint32_t planes, rotationTop, colourTop[3];
  float scaleLo, scaleStep, gap1Step, gap2Step, colourLo[3], colourStep[3], levels;
};

// Every byte column of a layer, in Morton order: position gaps in byte
// planes, rotation, scales, colour and opacity; column c at out + c * m.
__global__ void k_columns(uint32_t m, const unsigned long long *__restrict__ codes, const uint32_t *__restrict__ order,
                          const uint32_t *__restrict__ members, const float *__restrict__ canon, const float *__restrict__ ycocg,
                          const float *__restrict__ sig, ColumnArgs c, uint8_t *out) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const uint64_t gap = codes[j] - (j > 0 ? codes[j - 1] : 0ull);
  for (uint32_t p = 0; p < c.planes; ++p) out[(size_t)p * m + j] = (uint8_t)(gap >> (8 * p));
  const uint32_t i = members[order[j]];
  const float *k = canon + (size_t)i * 7;
  size_t col = c.planes;
  for (int a = 0; a < 3; ++a) {
    const float r = fminf(fmaxf(k[4 + a] / kRotationRange, -1.f), 1.f) * (float)c.rotationTop;
    out[(col + a) * m + j] = (uint8_t)zigzag((int)roundf(r));
  }
  col += 3;
  const float s0 = fmaxf(k[0], kMinLogScale), s1 = fmaxf(k[1], kMinLogScale), s2 = fmaxf(k[2], kMinLogScale);
  const auto level = [](float x) { return (int)fminf(fmaxf(roundf(x), 0.f), 255.f); };
  const int q0 = level((s0 - c.scaleLo) / c.scaleStep);
  const float r0 = c.scaleLo + (float)q0 * c.scaleStep;
  const int q1 = level((r0 - s1) / c.gap1Step);
  const float r1 = r0 - (float)q1 * c.gap1Step;
  const int q2 = level((r1 - s2) / c.gap2Step);
  out[col * m + j] = (uint8_t)q0;
  out[(col + 1) * m + j] = (uint8_t)q1;
  out[(col + 2) * m + j] = (uint8_t)q2;
  col += 3;
  for (int a = 0; a < 3; ++a) {
    const float top = (float)c.colourTop[a];
    const float v = fminf(fmaxf(roundf((ycocg[(size_t)i * 3 + a] - c.colourLo[a]) / c.colourStep[a]), 0.f), top);
    out[(col + a) * m + j] = (uint8_t)(int)v;
  }
  col += 3;
  out[col * m + j] = (uint8_t)(int)fminf(fmaxf(floorf(sig[i] * c.levels), 0.f), c.levels - 1.f);
}

// The codebook's points: the higher SH coefficients of each member in
// Morton order, YCoCg, dims = 3 (coeffs - 1) floats each, and their weights.
__global__ void k_sh_points(uint32_t m, uint32_t coeffs, const uint32_t *__restrict__ order, const uint32_t *__restrict__ members,
                            const float *__restrict__ sh, const float *__restrict__ weight, float *x, float *w) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  const uint32_t i = members[order[j]];
  const uint32_t dims = (coeffs - 1) * 3;
  for (uint32_t k = 1; k < coeffs; ++k) {
    const float *c = sh + ((size_t)i * coeffs + k) * 3;
    float y[3];
    to_ycocg(c[0], c[1], c[2], y);
    for (int a = 0; a < 3; ++a) x[(size_t)j * dims + (k - 1) * 3 + a] = y[a];
  }
  w[j] = weight[i];
}

// Lloyd's assignment: each point's nearest centre (squared distance, ties to
// the lower index), the centres staged in shared memory 64 at a time.
template <int D>
__global__ void __launch_bounds__(256) k_assign(uint32_t m, uint32_t k, const float *__restrict__ x, const float *__restrict__ centres,
                                                uint32_t *labels, uint32_t *labelValues) {
  constexpr int kTile = 64;
  __shared__ float s_c[kTile * D];
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  float p[D];
  for (int a = 0; a < D; ++a) p[a] = j < m ? x[(size_t)j * D + a] : 0.f;
  float best = INFINITY;
  uint32_t label = 0;
  for (uint32_t base = 0; base < k; base += kTile) {
    const uint32_t count = min((uint32_t)kTile, k - base);
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < count * D; t += blockDim.x) s_c[t] = centres[(size_t)base * D + t];
    __syncthreads();
    for (uint32_t t = 0; t < count; ++t) {
      float e = 0.f;
#pragma unroll
      for (int a = 0; a < D; ++a) {
        const float d = p[a] - s_c[t * D + a];
        e = fmaf(d, d, e);
      }
      if (e < best) {
        best = e;
        label = base + t;
      }
    }
  }
  if (j < m) {
    labels[j] = label;
    labelValues[j] = j;
  }
}

// Where each label's run starts and ends in the points sorted by label.
__global__ void k_runs(uint32_t m, const uint32_t *__restrict__ sortedLabels, uint32_t *first, uint32_t *last) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  const uint32_t l = sortedLabels[p];
  if (p == 0 || sortedLabels[p - 1] != l) first[l] = p;
  if (p + 1 == m || sortedLabels[p + 1] != l) last[l] = p + 1;
}

// The weighted mean of each centre's points, one thread per (centre, value),
// summed in FP64 in the sorted order; a centre with no point keeps its place.
__global__ void k_means(uint32_t k, uint32_t dims, const uint32_t *__restrict__ first, const uint32_t *__restrict__ last,
                        const uint32_t *__restrict__ sortedPoints, const float *__restrict__ x, const float *__restrict__ w,
                        float *centres) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= k * dims) return;
  const uint32_t c = t / dims, a = t % dims;
  double sum = 0.0, total = 0.0;
  for (uint32_t p = first[c]; p < last[c]; ++p) {
    const uint32_t j = sortedPoints[p];
    sum += (double)w[j] * (double)x[(size_t)j * dims + a];
    total += (double)w[j];
  }
  if (total > 0.0) centres[t] = (float)(sum / total);
}

// Picks k distinct points by sorting them on a hash of their index.
__global__ void k_seed_keys(uint32_t m, uint32_t seed, uint32_t *keys, uint32_t *values) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m) return;
  uint32_t h = j * 747796405u + seed;
  h = ((h >> ((h >> 28u) + 4u)) ^ h) * 277803737u;
  keys[j] = (h >> 22u) ^ h;
  values[j] = j;
}

__global__ void k_gather_centres(uint32_t k, uint32_t dims, const uint32_t *__restrict__ picks, const float *__restrict__ x,
                                 float *centres) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= k * dims) return;
  centres[t] = x[(size_t)picks[t / dims] * dims + t % dims];
}

struct Stream {
  cudaStream_t s = nullptr;
  Stream() { CGC_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
  ~Stream() { cudaStreamDestroy(s); }
};

inline uint32_t blocks_for(size_t n, uint32_t threads = 256) { return (uint32_t)std::max<size_t>((n + threads - 1) / threads, 1); }

// A radix sort of `count` pairs over `bits` key bits with fresh temporaries;
// returns the arrays that hold the result.
template <class K> std::pair<K *, uint32_t *> sort_pairs(K *keys, uint32_t *values, Dev &tmpKeys, Dev &tmpValues, uint32_t count,
                                                        int bits, cudaStream_t s) {
  if (count <= 1) return {keys, values};
  tmpKeys.resize((size_t)count * sizeof(K));
  tmpValues.resize((size_t)count * 4);
  Dev scratch(sort_scratch_bytes(count, (int)sizeof(K), bits, 8)), error(4);
  CGC_CUDA(cudaMemsetAsync(error.get(), 0, 4, s));
  int where;
  if constexpr (sizeof(K) == 8) {
    where = sort_pairs_u64(reinterpret_cast<unsigned long long *>(keys), values, tmpKeys.get<unsigned long long>(),
                           tmpValues.get<uint32_t>(), count, count, nullptr, 0, bits, 8, scratch.get(), error.get<uint32_t>(), s);
  } else {
    where = sort_pairs_u32(keys, values, tmpKeys.get<uint32_t>(), tmpValues.get<uint32_t>(), count, count, nullptr, 0, bits, 8,
                           scratch.get(), error.get<uint32_t>(), s);
  }
  CGC_CUDA(cudaGetLastError());
  uint32_t err = 0;
  CGC_CUDA(cudaMemcpyAsync(&err, error.get(), 4, cudaMemcpyDeviceToHost, s));
  CGC_CUDA(cudaStreamSynchronize(s));
  if (err != 0u) throw std::runtime_error("a radix sort's look-back gave up waiting");
  if (where == 1) return {tmpKeys.get<K>(), tmpValues.get<uint32_t>()};
  return {keys, values};
}

template <class T> T read_one(const T *device, size_t index, cudaStream_t s) {
  T v;
  CGC_CUDA(cudaMemcpyAsync(&v, device + index, sizeof(T), cudaMemcpyDeviceToHost, s));
  CGC_CUDA(cudaStreamSynchronize(s));
  return v;
}

// The k-means codebook of m points of `dims` values: k centres, Lloyd's
// iterations from k distinct points picked by a fixed hash, then the labels
// of the final centres.
void codebook(const float *x, const float *w, uint32_t m, uint32_t dims, uint32_t k, int iterations, std::vector<float> &centres,
              std::vector<uint32_t> &labels, cudaStream_t s) {
  Dev c((size_t)k * dims * 4), lab((size_t)m * 4), labVal((size_t)m * 4), tk, tv, first((size_t)k * 4), last((size_t)k * 4);
  {
    Dev keys((size_t)m * 4), vals((size_t)m * 4);
    k_seed_keys<<<blocks_for(m), 256, 0, s>>>(m, 12345u, keys.get<uint32_t>(), vals.get<uint32_t>());
    const auto sorted = sort_pairs<uint32_t>(keys.get<uint32_t>(), vals.get<uint32_t>(), tk, tv, m, 32, s);
    k_gather_centres<<<blocks_for((size_t)k * dims), 256, 0, s>>>(k, dims, sorted.second, x, c.get<float>());
    CGC_CUDA(cudaStreamSynchronize(s));
  }
  const auto assign = [&] {
    switch (dims) {
    case 9: k_assign<9><<<blocks_for(m), 256, 0, s>>>(m, k, x, c.get<float>(), lab.get<uint32_t>(), labVal.get<uint32_t>()); break;
    case 24: k_assign<24><<<blocks_for(m), 256, 0, s>>>(m, k, x, c.get<float>(), lab.get<uint32_t>(), labVal.get<uint32_t>()); break;
    default: k_assign<45><<<blocks_for(m), 256, 0, s>>>(m, k, x, c.get<float>(), lab.get<uint32_t>(), labVal.get<uint32_t>()); break;
    }
    CGC_CUDA(cudaGetLastError());
  };
  int labelBits = 1;
  while ((1u << labelBits) < k) ++labelBits;
  for (int it = 0; it < iterations; ++it) {
    assign();
    const auto sorted = sort_pairs<uint32_t>(lab.get<uint32_t>(), labVal.get<uint32_t>(), tk, tv, m, labelBits, s);
    CGC_CUDA(cudaMemsetAsync(first.get(), 0, (size_t)k * 4, s));
    CGC_CUDA(cudaMemsetAsync(last.get(), 0, (size_t)k * 4, s));
    k_runs<<<blocks_for(m), 256, 0, s>>>(m, sorted.first, first.get<uint32_t>(), last.get<uint32_t>());
    k_means<<<blocks_for((size_t)k * dims), 256, 0, s>>>(k, dims, first.get<uint32_t>(), last.get<uint32_t>(), sorted.second, x, w,
                                                        c.get<float>());
    CGC_CUDA(cudaGetLastError());
  }
  assign();
  centres.resize((size_t)k * dims);
  labels.resize(m);
  CGC_CUDA(cudaMemcpyAsync(centres.data(), c.get(), (size_t)k * dims * 4, cudaMemcpyDeviceToHost, s));
  CGC_CUDA(cudaMemcpyAsync(labels.data(), lab.get(), (size_t)m * 4, cudaMemcpyDeviceToHost, s));
  CGC_CUDA(cudaStreamSynchronize(s));
}

template <class T> void put(std::vector<uint8_t> &out, const T &value) {
  const uint8_t *b = reinterpret_cast<const uint8_t *>(&value);
  out.insert(out.end(), b, b + sizeof(T));
}

struct Saved {
  uint64_t bytes = 0;
  uint64_t layerCounts[kLayers] = {0, 0, 0};
};

Saved save(const splat_cloud &cloud, const std::string &path, int preset, bool fast) {
  if (cloud.count < 0 || cloud.sh_degree < 0 || cloud.sh_degree > 3) throw std::invalid_argument("invalid cloud");
  const uint32_t n = (uint32_t)cloud.count, degree = (uint32_t)cloud.sh_degree;
  const uint32_t coeffs = (degree + 1) * (degree + 1), dims = (coeffs - 1) * 3;
  if (n > 0 && (!cloud.positions || !cloud.scales || !cloud.rotations || !cloud.opacities || !cloud.sh))
    throw std::invalid_argument("null cloud array");
  const auto params = layer_params(preset);
  float center[3] = {0.f, 0.f, 0.f}, radius = 1.f;
  LayerHeader headers[kLayers];
  std::vector<std::vector<uint8_t>> columns;
  Saved saved;
  if (n > 0) {
    Stream st;
    const cudaStream_t s = st.s;
    Dev pos((size_t)n * 12), sca((size_t)n * 12), rot((size_t)n * 16), op((size_t)n * 4), sh((size_t)n * coeffs * 12);
    CGC_CUDA(cudaMemcpyAsync(pos.get(), cloud.positions, (size_t)n * 12, cudaMemcpyHostToDevice, s));
    CGC_CUDA(cudaMemcpyAsync(sca.get(), cloud.scales, (size_t)n * 12, cudaMemcpyHostToDevice, s));
    CGC_CUDA(cudaMemcpyAsync(rot.get(), cloud.rotations, (size_t)n * 16, cudaMemcpyHostToDevice, s));
    CGC_CUDA(cudaMemcpyAsync(op.get(), cloud.opacities, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    CGC_CUDA(cudaMemcpyAsync(sh.get(), cloud.sh, (size_t)n * coeffs * 12, cudaMemcpyHostToDevice, s));
    Dev bad(4), axis[3], importance((size_t)n * 4), impKeys((size_t)n * 4), canon((size_t)n * 28), ycocg((size_t)n * 12),
        sig((size_t)n * 4), weight((size_t)n * 4), values((size_t)n * 4), tk, tv;
    for (Dev &a : axis) a.resize((size_t)n * 4);
    Dev axisAll((size_t)n * 12);
    CGC_CUDA(cudaMemsetAsync(bad.get(), 0, 4, s));
    k_splats<<<blocks_for(n), 256, 0, s>>>(n, coeffs, pos.get<float>(), sca.get<float>(), rot.get<float>(), op.get<float>(),
                                           sh.get<float>(), bad.get<uint32_t>(), axisAll.get<uint32_t>(), importance.get<float>(),
                                           impKeys.get<uint32_t>(), canon.get<float>(), ycocg.get<float>(), sig.get<float>(),
                                           weight.get<float>());
    CGC_CUDA(cudaGetLastError());
    if (read_one(bad.get<uint32_t>(), 0, s) != 0u)
      throw std::invalid_argument(path + ": cannot save a cloud with NaN or infinite values");
    // The centre: the median of each coordinate; the radius: the 90th
    // percentile of the distances from it, at least 1e-3.
    for (int a = 0; a < 3; ++a) {
      CGC_CUDA(cudaMemcpyAsync(axis[a].get(), axisAll.get<uint32_t>() + (size_t)a * n, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
      k_iota<<<blocks_for(n), 256, 0, s>>>(n, values.get<uint32_t>());
      const auto sorted = sort_pairs<uint32_t>(axis[a].get<uint32_t>(), values.get<uint32_t>(), tk, tv, n, 32, s);
      center[a] = key_float(read_one(sorted.first, n / 2, s));
    }
    {
      Dev keys((size_t)n * 4);
      k_distance_keys<<<blocks_for(n), 256, 0, s>>>(n, pos.get<float>(), center[0], center[1], center[2], keys.get<uint32_t>(),
                                                    values.get<uint32_t>());
      const auto sorted = sort_pairs<uint32_t>(keys.get<uint32_t>(), values.get<uint32_t>(), tk, tv, n, 32, s);
      radius = std::max(key_float(read_one(sorted.first, std::min<size_t>(n - 1, (size_t)n * 9 / 10), s)), 1e-3f);
    }
    // The layers: importance percentiles, most important first.
    float cuts[kLayers];
    {
      k_iota<<<blocks_for(n), 256, 0, s>>>(n, values.get<uint32_t>());
      const auto sorted = sort_pairs<uint32_t>(impKeys.get<uint32_t>(), values.get<uint32_t>(), tk, tv, n, 32, s);
      for (int l = 0; l < kLayers; ++l)
        cuts[l] = key_float(read_one(sorted.first, (size_t)(params[l].fromPercentile / 100.0 * (double)(n - 1)), s));
    }
    Dev layerKeys((size_t)n * 4), counts(16);
    CGC_CUDA(cudaMemsetAsync(counts.get(), 0, 16, s));
    k_layer_keys<<<blocks_for(n), 256, 0, s>>>(n, importance.get<float>(), cuts[0], cuts[1], layerKeys.get<uint32_t>(),
                                               values.get<uint32_t>(), counts.get<uint32_t>());
    uint32_t layerCount[4];
    CGC_CUDA(cudaMemcpyAsync(layerCount, counts.get(), 16, cudaMemcpyDeviceToHost, s));
    const auto grouped = sort_pairs<uint32_t>(layerKeys.get<uint32_t>(), values.get<uint32_t>(), tk, tv, n, 2, s);
    uint32_t start = 0;
    for (int l = 0; l < kLayers; ++l) {
      const LayerParams &pl = params[l];
      LayerHeader &h = headers[l];
      const uint32_t m = layerCount[l];
      saved.layerCounts[l] = m;
      h.count = m;
      h.posBits = pl.posBits;
      h.rotBits = pl.rotBits;
      h.alphaBits = pl.alphaBits;
      for (int a = 0; a < 3; ++a) h.colorBits[a] = pl.colorBits[a];
      if (m == 0) continue;
      Dev members((size_t)m * 4), warped((size_t)m * 12), extremes(32), colourKeys((size_t)m * 12), colourValues((size_t)m * 12);
      CGC_CUDA(cudaMemcpyAsync(members.get(), grouped.second + start, (size_t)m * 4, cudaMemcpyDeviceToDevice, s));
      start += m;
      const uint32_t init[8] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u, 0u, 0u};
      CGC_CUDA(cudaMemcpyAsync(extremes.get(), init, sizeof(init), cudaMemcpyHostToDevice, s));
      k_layer_prepare<<<blocks_for(m), 256, 0, s>>>(m, members.get<uint32_t>(), pos.get<float>(), sca.get<float>(),
                                                    ycocg.get<float>(), center[0], center[1], center[2], radius,
                                                    warped.get<float>(), extremes.get<uint32_t>(), colourKeys.get<uint32_t>(),
                                                    colourValues.get<uint32_t>());
      uint32_t ex[8];
      CGC_CUDA(cudaMemcpyAsync(ex, extremes.get(), sizeof(ex), cudaMemcpyDeviceToHost, s));
      CGC_CUDA(cudaStreamSynchronize(s));
      float hi[3];
      for (int a = 0; a < 3; ++a) {
        h.posLo[a] = key_float(ex[a]);
        hi[a] = key_float(ex[3 + a]);
      }
      const float extent = std::max({hi[0] - h.posLo[0], hi[1] - h.posLo[1], hi[2] - h.posLo[2]});
      h.posStep = extent > 0.f ? extent / (float)((1u << pl.posBits) - 1) : 1.f;
      const float largest = std::max(kMinLogScale, key_float(ex[6]));
      h.scaleLo = kMinLogScale;
      h.scaleStep = std::max(pl.scaleStep, (largest - kMinLogScale) / 255.f);
      h.gap1Step = pl.gap1Step;
      h.gap2Step = pl.gap2Step;
      // Morton order, ties by index (the members are in index order and the sort is stable).
      Dev codes((size_t)m * 8), order((size_t)m * 4), ck, cv;
      k_morton<<<blocks_for(m), 256, 0, s>>>(m, warped.get<float>(), h.posLo[0], h.posLo[1], h.posLo[2], h.posStep,
                                             codes.get<unsigned long long>(), order.get<uint32_t>());
      const auto morton = sort_pairs<unsigned long long>(codes.get<unsigned long long>(), order.get<uint32_t>(), ck, cv, m,
                                                         (int)pl.posBits * 3, s);
      // The robust colour ranges: skip the most extreme values at each end.
      const size_t skip = m < 64 ? 0 : std::max<size_t>(1, m / 10000);
      for (int a = 0; a < 3; ++a) {
        Dev keys((size_t)m * 4), vals((size_t)m * 4), sk, sv;
        CGC_CUDA(cudaMemcpyAsync(keys.get(), colourKeys.get<uint32_t>() + (size_t)a * m, (size_t)m * 4, cudaMemcpyDeviceToDevice, s));
        CGC_CUDA(cudaMemcpyAsync(vals.get(), colourValues.get<uint32_t>() + (size_t)a * m, (size_t)m * 4, cudaMemcpyDeviceToDevice, s));
        const auto sorted = sort_pairs<uint32_t>(keys.get<uint32_t>(), vals.get<uint32_t>(), sk, sv, m, 32, s);
        const float lo = key_float(read_one(sorted.first, skip, s)), top = key_float(read_one(sorted.first, m - 1 - skip, s));
        h.colorLo[a] = lo;
        h.colorStep[a] = top > lo ? (top - lo) / (float)((1u << pl.colorBits[a]) - 1) : 1.f;
      }
      ColumnArgs ca{};
      ca.planes = (pl.posBits * 3 + 7) / 8;
      ca.rotationTop = (1u << (pl.rotBits - 1)) - 1;
      for (int a = 0; a < 3; ++a) {
        ca.colourTop[a] = (1u << pl.colorBits[a]) - 1;
        ca.colourLo[a] = h.colorLo[a];
        ca.colourStep[a] = h.colorStep[a];
      }
      ca.scaleLo = h.scaleLo;
      ca.scaleStep = h.scaleStep;
      ca.gap1Step = h.gap1Step;
      ca.gap2Step = h.gap2Step;
      ca.levels = (float)(1u << pl.alphaBits);
      const size_t fixedColumns = ca.planes + 10;
      Dev bytes(fixedColumns * m);
      k_columns<<<blocks_for(m), 256, 0, s>>>(m, morton.first, morton.second, members.get<uint32_t>(), canon.get<float>(),
                                              ycocg.get<float>(), sig.get<float>(), ca, bytes.get<uint8_t>());
      CGC_CUDA(cudaGetLastError());
      std::vector<uint8_t> host(fixedColumns * m);
      CGC_CUDA(cudaMemcpyAsync(host.data(), bytes.get(), host.size(), cudaMemcpyDeviceToHost, s));
      CGC_CUDA(cudaStreamSynchronize(s));
      for (size_t c = 0; c < fixedColumns; ++c) columns.emplace_back(host.begin() + c * m, host.begin() + (c + 1) * m);
      if (dims == 0) continue;
      // The higher SH bands: one codebook for the layer, most used entries first.
      Dev x((size_t)m * dims * 4), wts((size_t)m * 4);
      k_sh_points<<<blocks_for(m), 256, 0, s>>>(m, coeffs, morton.second, members.get<uint32_t>(), sh.get<float>(),
                                                weight.get<float>(), x.get<float>(), wts.get<float>());
      size_t wanted = std::min<size_t>({std::max<size_t>({m / pl.splatsPerCode, std::min<size_t>(m / 4, 1024), 1}), m,
                                        kMaxCodebook});
      if (fast) wanted = std::min<size_t>(wanted, 1024);
      std::vector<float> centres;
      std::vector<uint32_t> labels;
      codebook(x.get<float>(), wts.get<float>(), m, dims, (uint32_t)wanted, fast ? 4 : 10, centres, labels, s);
      const size_t book = wanted;
      h.codebookSize = (uint32_t)book;
      h.codebookStep = kCodebookStep;
      std::vector<uint32_t> uses(book, 0u), byUse(book), rank(book);
      for (uint32_t label : labels) ++uses[label];
      std::iota(byUse.begin(), byUse.end(), 0u);
      std::stable_sort(byUse.begin(), byUse.end(), [&](uint32_t a, uint32_t b) { return uses[a] > uses[b]; });
      for (size_t t = 0; t < book; ++t) rank[byUse[t]] = (uint32_t)t;
      std::vector<uint8_t> low(m), high(m), bookLow(book * dims), bookHigh(book * dims);
      for (size_t j = 0; j < m; ++j) {
        low[j] = (uint8_t)rank[labels[j]];
        high[j] = (uint8_t)(rank[labels[j]] >> 8);
      }
      for (size_t a = 0; a < dims; ++a)
        for (size_t t = 0; t < book; ++t) {
          const float v = centres[byUse[t] * dims + a];
          const uint32_t z = zigzag(std::clamp((int)std::round(v / kCodebookStep), -32767, 32767));
          bookLow[a * book + t] = (uint8_t)z;
          bookHigh[a * book + t] = (uint8_t)(z >> 8);
        }
      columns.push_back(std::move(low));
      columns.push_back(std::move(high));
      columns.push_back(std::move(bookLow));
      columns.push_back(std::move(bookHigh));
    }
  } else {
    for (int l = 0; l < kLayers; ++l) {
      headers[l].posBits = params[l].posBits;
      headers[l].rotBits = params[l].rotBits;
      headers[l].alphaBits = params[l].alphaBits;
      for (int a = 0; a < 3; ++a) headers[l].colorBits[a] = params[l].colorBits[a];
    }
  }
  // Each column its own LZMA stream (lc = lp = pb = 0 suits byte columns).
  std::vector<std::vector<uint8_t>> streams(columns.size());
  on_threads(columns.size(), [&](size_t i) { streams[i] = lzma_pack(columns[i].data(), columns[i].size(), fast ? 1 : 6, false, 0, 0, 0); });
  std::vector<uint8_t> file(kMagic, kMagic + 4);
  put(file, kVersion);
  put(file, n);
  put(file, degree);
  put(file, (uint32_t)kLayers);
  for (float v : center) put(file, v);
  put(file, radius);
  for (const LayerHeader &h : headers) put(file, h);
  for (const auto &stream : streams) {
    put(file, (uint32_t)stream.size());
    file.insert(file.end(), stream.begin(), stream.end());
  }
  std::ofstream out(path, std::ios::binary);
  if (!out) throw std::runtime_error("Cannot write '" + path + "'");
  out.write(reinterpret_cast<const char *>(file.data()), (std::streamsize)file.size());
  if (!out) throw std::runtime_error("Failed writing '" + path + "'");
  saved.bytes = file.size();
  return saved;
}

} // namespace cgc
} // namespace sb

namespace {

template <class F> int cgc_guarded(F &&body) {
  try {
    body();
    sb::set_last_error("");
    return SPLAT_OK;
  } catch (const std::invalid_argument &e) {
    sb::set_last_error(e.what());
    return SPLAT_ERR_INVALID;
  } catch (const std::bad_alloc &) {
    sb::set_last_error("out of memory");
    return SPLAT_ERR_DEVICE;
  } catch (const std::exception &e) {
    const std::string what = e.what();
    sb::set_last_error(what.c_str());
    return what.rfind("CUDA: ", 0) == 0 ? SPLAT_ERR_DEVICE : SPLAT_ERR_INVALID;
  }
}

} // namespace

extern "C" int splat_cloud_save_cgc(const char *path, const splat_cloud *cloud, const splat_cgc_options *options,
                                    splat_cgc_stats *stats) {
  return cgc_guarded([&] {
    if (path == nullptr || cloud == nullptr) throw std::invalid_argument("null argument");
    const int preset = options != nullptr ? options->preset : SPLAT_CGC_BALANCED;
    if (preset != SPLAT_CGC_BALANCED && preset != SPLAT_CGC_SMALL) throw std::invalid_argument("unknown CGC preset");
    const sb::cgc::Saved s = sb::cgc::save(*cloud, path, preset, options != nullptr && options->fast != 0);
    if (stats != nullptr) {
      stats->bytes = s.bytes;
      for (int l = 0; l < 3; ++l) stats->layer_counts[l] = s.layerCounts[l];
    }
  });
}

extern "C" int splat_cloud_load_cgc(const char *path, int32_t *count, int32_t *sh_degree, float *positions, float *scales,
                                    float *rotations, float *opacities, float *sh) {
  return cgc_guarded([&] {
    if (path == nullptr || count == nullptr || sh_degree == nullptr) throw std::invalid_argument("null argument");
    const bool headerOnly = !positions && !scales && !rotations && !opacities && !sh;
    if (!headerOnly && (!positions || !scales || !rotations || !opacities || !sh))
      throw std::invalid_argument("either every array or none");
    const sb::cgc::Cloud c = sb::cgc::load(path);
    if (c.count > 0x7FFFFFFFu) throw std::runtime_error(std::string(path) + ": more Gaussians than the cloud's count holds");
    if (!headerOnly) {
      std::memcpy(positions, c.positions.data(), c.positions.size() * 4);
      std::memcpy(scales, c.scales.data(), c.scales.size() * 4);
      std::memcpy(rotations, c.rotations.data(), c.rotations.size() * 4);
      std::memcpy(opacities, c.opacities.data(), c.opacities.size() * 4);
      std::memcpy(sh, c.sh.data(), c.sh.size() * 4);
    }
    *count = (int32_t)c.count;
    *sh_degree = c.degree;
  });
}

extern "C" uint64_t splat_cgc_morton_code(uint32_t x, uint32_t y, uint32_t z) { return sb::cgc::morton(x, y, z); }

extern "C" int splat_cgc_canonicalize_axes(float *log_scales, float *wxyz) {
  return cgc_guarded([&] {
    if (log_scales == nullptr || wxyz == nullptr) throw std::invalid_argument("null argument");
    sb::cgc::canonicalize(log_scales, wxyz);
  });
}

extern "C" int splat_lzma_compress(const uint8_t *data, size_t size, int32_t level, int32_t extreme, int32_t lc, int32_t lp,
                                   int32_t pb, uint8_t *out, size_t capacity, size_t *written) {
  return cgc_guarded([&] {
    if ((data == nullptr && size > 0) || written == nullptr) throw std::invalid_argument("null argument");
    if (lc < 0 || lc > 4 || lp < 0 || lp > 4 || pb < 0 || pb > 4) throw std::invalid_argument("lc, lp and pb must be 0..4");
    const std::vector<uint8_t> packed = sb::cgc::lzma_pack(data, size, level, extreme != 0, lc, lp, pb);
    *written = packed.size();
    if (out != nullptr) std::memcpy(out, packed.data(), std::min(capacity, packed.size()));
  });
}

extern "C" int splat_lzma_decompress(const uint8_t *stream, size_t size, uint8_t *out, size_t expected) {
  return cgc_guarded([&] {
    if (stream == nullptr || (out == nullptr && expected > 0)) throw std::invalid_argument("null argument");
    const std::vector<uint8_t> data = sb::cgc::lzma_unpack(stream, size, expected);
    if (expected > 0) std::memcpy(out, data.data(), expected);
  });
}
