// ORACLE (test infrastructure only; never linked into the product).
//
// The reference's LZMA wrapper interface (src/splat/lzma.hpp: lzma_compress,
// lzma_decompress) implemented over the system's liblzma.so.5, loaded at run
// time: the image has the library but not its headers, so the reference's own
// src/splat/lzma.cpp (which includes <lzma.h>) cannot be compiled here. With
// this file in its place, the reference's CGC writer and reader
// (src/splat/cgc.cpp) compile unmodified into oracle/_ref.
//
// The wrapper's behaviour: an "alone" (.lzma) stream from the preset `level`
// (with the extreme flag when asked) and the given lc, lp, pb; decompression
// fails on a corrupt or truncated stream and on any size other than the one
// expected. Only the first fields of liblzma's option and stream structures
// are touched; their offsets are checked against what lzma_lzma_preset writes
// before any use.
#include "splat/lzma.hpp"

#include <dlfcn.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

namespace splat {

namespace {

// The leading fields of lzma_stream; the rest of liblzma's structure lies in
// the padding, which starts (and, for lzma_end, stays) zero.
struct StreamHead {
  const std::uint8_t *nextIn;
  std::size_t availIn;
  std::uint64_t totalIn;
  std::uint8_t *nextOut;
  std::size_t availOut;
  std::uint64_t totalOut;
};
struct alignas(16) StreamBox {
  StreamHead head;
  unsigned char rest[464];
};
// lzma_options_lzma: dict_size at 0, lc, lp, pb at 20, 24, 28.
struct alignas(16) OptionsBox {
  unsigned char bytes[256];
};

constexpr int kOk = 0, kStreamEnd = 1, kBufError = 10, kFinish = 3;
constexpr std::uint32_t kPresetExtreme = 0x80000000u;

struct Lib {
  unsigned char (*preset)(void *, std::uint32_t) = nullptr;
  int (*aloneEncoder)(void *, const void *) = nullptr;
  int (*aloneDecoder)(void *, std::uint64_t) = nullptr;
  int (*code)(void *, int) = nullptr;
  void (*end)(void *) = nullptr;
};

const Lib &lib() {
  static const Lib l = [] {
    Lib out;
    void *h = dlopen("liblzma.so.5", RTLD_NOW | RTLD_LOCAL);
    if (h == nullptr) throw std::runtime_error("liblzma.so.5 is not available");
    out.preset = reinterpret_cast<unsigned char (*)(void *, std::uint32_t)>(dlsym(h, "lzma_lzma_preset"));
    out.aloneEncoder = reinterpret_cast<int (*)(void *, const void *)>(dlsym(h, "lzma_alone_encoder"));
    out.aloneDecoder = reinterpret_cast<int (*)(void *, std::uint64_t)>(dlsym(h, "lzma_alone_decoder"));
    out.code = reinterpret_cast<int (*)(void *, int)>(dlsym(h, "lzma_code"));
    out.end = reinterpret_cast<void (*)(void *)>(dlsym(h, "lzma_end"));
    if (!out.preset || !out.aloneEncoder || !out.aloneDecoder || !out.code || !out.end)
      throw std::runtime_error("liblzma.so.5 lacks an expected symbol");
    return out;
  }();
  return l;
}

std::uint32_t word_at(const OptionsBox &o, int offset) {
  std::uint32_t v;
  std::memcpy(&v, o.bytes + offset, 4);
  return v;
}

void pump(StreamBox &s, std::span<const std::byte> input, std::vector<std::byte> &out, std::size_t limit) {
  s.head.nextIn = reinterpret_cast<const std::uint8_t *>(input.data());
  s.head.availIn = input.size();
  std::size_t used = 0;
  for (;;) {
    if (s.head.availOut == 0) {
      used = out.size();
      if (used >= limit) throw std::runtime_error("LZMA output is larger than expected");
      out.resize(std::min(limit, std::max<std::size_t>(used * 2, 1 << 16)));
      s.head.nextOut = reinterpret_cast<std::uint8_t *>(out.data()) + used;
      s.head.availOut = out.size() - used;
    }
    const int r = lib().code(&s, kFinish);
    if (r == kStreamEnd) break;
    if (r == kBufError) throw std::runtime_error("LZMA stream ends early");
    if (r != kOk) throw std::runtime_error("LZMA failure " + std::to_string(r));
  }
  out.resize(out.size() - s.head.availOut);
}

} // namespace

std::vector<std::byte> lzma_compress(std::span<const std::byte> data, int level, bool extreme, int lc, int lp, int pb) {
  OptionsBox o{};
  if (lib().preset(&o, static_cast<std::uint32_t>(level) | (extreme ? kPresetExtreme : 0u)) != 0)
    throw std::runtime_error("bad LZMA preset");
  if (word_at(o, 20) != 3u || word_at(o, 24) != 0u || word_at(o, 28) != 2u || word_at(o, 0) == 0u)
    throw std::runtime_error("liblzma's option layout is not the expected one");
  const std::uint32_t l[3] = {static_cast<std::uint32_t>(lc), static_cast<std::uint32_t>(lp), static_cast<std::uint32_t>(pb)};
  std::memcpy(o.bytes + 20, l, sizeof(l));
  StreamBox s{};
  if (lib().aloneEncoder(&s, &o) != kOk) throw std::runtime_error("the LZMA encoder did not start");
  std::vector<std::byte> out;
  try {
    pump(s, data, out, SIZE_MAX);
  } catch (...) {
    lib().end(&s);
    throw;
  }
  lib().end(&s);
  return out;
}

std::vector<std::byte> lzma_decompress(std::span<const std::byte> stream, std::size_t expectedSize) {
  StreamBox s{};
  if (lib().aloneDecoder(&s, UINT64_MAX) != kOk) throw std::runtime_error("the LZMA decoder did not start");
  std::vector<std::byte> out;
  try {
    pump(s, stream, out, expectedSize + 1);
  } catch (...) {
    lib().end(&s);
    throw;
  }
  lib().end(&s);
  if (out.size() != expectedSize) throw std::runtime_error("LZMA data of the wrong size");
  return out;
}

} // namespace splat
