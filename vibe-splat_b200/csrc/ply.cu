// 3DGS .ply files on the host (the reference's load_ply / save_ply,
// src/splat/gaussian_cloud.cpp:236-365): binary little-endian or ASCII in,
// binary little-endian out in the standard layout other splat tools read
// (x y z, three zero normals, f_dc_0..2, f_rest_* channel-major, opacity,
// scale_0..2, rot_0..3, all float). Properties the cloud has no use for are
// skipped; elements after the vertex element are never read. A file whose
// vertex properties are all float is read record by record with no per-value
// type dispatch.
#include <cstdint>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "splat_b200.h"

namespace sb {

void set_last_error(const char *message);

namespace {

enum class Kind { I8, U8, I16, U16, I32, U32, F32, F64 };

bool kind_of(const std::string &name, Kind &kind, size_t &bytes) {
  static const std::unordered_map<std::string, std::pair<Kind, size_t>> kinds = {
      {"char", {Kind::I8, 1}},   {"int8", {Kind::I8, 1}},     {"uchar", {Kind::U8, 1}},   {"uint8", {Kind::U8, 1}},
      {"short", {Kind::I16, 2}}, {"int16", {Kind::I16, 2}},   {"ushort", {Kind::U16, 2}}, {"uint16", {Kind::U16, 2}},
      {"int", {Kind::I32, 4}},   {"int32", {Kind::I32, 4}},   {"uint", {Kind::U32, 4}},   {"uint32", {Kind::U32, 4}},
      {"float", {Kind::F32, 4}}, {"float32", {Kind::F32, 4}}, {"double", {Kind::F64, 8}}, {"float64", {Kind::F64, 8}}};
  const auto it = kinds.find(name);
  if (it == kinds.end()) return false;
  kind = it->second.first;
  bytes = it->second.second;
  return true;
}

template <class T> T little(const unsigned char *p) {
  T v;
  std::memcpy(&v, p, sizeof v); // hosts here are little-endian, as the files
  return v;
}

float value_of(Kind kind, const unsigned char *p) {
  switch (kind) {
  case Kind::I8: return (float)little<int8_t>(p);
  case Kind::U8: return (float)little<uint8_t>(p);
  case Kind::I16: return (float)little<int16_t>(p);
  case Kind::U16: return (float)little<uint16_t>(p);
  case Kind::I32: return (float)little<int32_t>(p);
  case Kind::U32: return (float)little<uint32_t>(p);
  case Kind::F32: return little<float>(p);
  case Kind::F64: return (float)little<double>(p);
  }
  return 0.0f;
}

struct Column {
  std::string name;
  Kind kind;
  size_t offset;
};

struct PlyHeader {
  bool binary = true;
  size_t vertices = 0;
  std::vector<Column> columns;
  size_t recordBytes = 0;
  bool allFloat = true;
};

PlyHeader read_header(std::istream &in, const std::string &path) {
  std::string line;
  if (!std::getline(in, line) || line.compare(0, 3, "ply") != 0) throw std::runtime_error(path + ": not a PLY file");
  PlyHeader h;
  bool vertexOpen = false, haveVertex = false, haveFormat = false;
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::istringstream words(line);
    std::string word;
    words >> word;
    if (word == "end_header") break;
    if (word.empty() || word == "comment" || word == "obj_info") continue;
    if (word == "format") {
      std::string format;
      words >> format;
      if (format == "binary_little_endian") h.binary = true;
      else if (format == "ascii") h.binary = false;
      else throw std::runtime_error(path + ": unsupported PLY format '" + format + "'");
      haveFormat = true;
    } else if (word == "element") {
      std::string name;
      size_t count = 0;
      words >> name >> count;
      if (name == "vertex") {
        if (haveVertex) throw std::runtime_error(path + ": more than one vertex element");
        vertexOpen = haveVertex = true;
        h.vertices = count;
      } else {
        if (!haveVertex && count > 0) throw std::runtime_error(path + ": element '" + name + "' before the vertex element");
        vertexOpen = false;
      }
    } else if (word == "property" && vertexOpen) {
      std::string type, name;
      words >> type;
      if (type == "list") throw std::runtime_error(path + ": list properties on vertices are not supported");
      words >> name;
      Kind kind;
      size_t bytes = 0;
      if (!kind_of(type, kind, bytes)) throw std::runtime_error(path + ": unknown property type '" + type + "'");
      h.columns.push_back({name, kind, h.recordBytes});
      h.recordBytes += bytes;
      h.allFloat = h.allFloat && kind == Kind::F32;
    }
  }
  if (!haveFormat || !haveVertex) throw std::runtime_error(path + ": PLY header has no format or vertex element");
  return h;
}

int degree_of_rest(size_t rest) {
  switch (rest) {
  case 0: return 0;
  case 9: return 1;
  case 24: return 2;
  case 45: return 3;
  default: return -1;
  }
}

// Where each cloud attribute comes from in a vertex record: columns of the
// positions, scales, rotations, opacity, DC and rest (file order).
struct Layout {
  size_t position[3], scale[3], rotation[4], opacity, dc[3];
  std::vector<size_t> rest;
  int degree;
};

Layout layout_of(const PlyHeader &h, const std::string &path) {
  std::unordered_map<std::string, size_t> column;
  for (size_t i = 0; i < h.columns.size(); ++i) column[h.columns[i].name] = i;
  // Every property a splat needs, looked up at once; one message names all
  // the missing ones.
  std::string missing;
  const auto find = [&](const std::string &name) -> size_t {
    const auto it = column.find(name);
    if (it != column.end()) return it->second;
    missing += (missing.empty() ? "" : ", ") + name;
    return 0;
  };
  Layout l;
  size_t rest = 0;
  while (column.count("f_rest_" + std::to_string(rest)) != 0) ++rest;
  l.degree = degree_of_rest(rest);
  static const char *const kAxes[3] = {"x", "y", "z"};
  for (int a = 0; a < 3; ++a) {
    l.position[a] = find(kAxes[a]);
    l.scale[a] = find("scale_" + std::to_string(a));
    l.dc[a] = find("f_dc_" + std::to_string(a));
  }
  for (int a = 0; a < 4; ++a) l.rotation[a] = find("rot_" + std::to_string(a));
  l.opacity = find("opacity");
  if (!missing.empty()) throw std::runtime_error(path + ": not a Gaussian splat file, missing property: " + missing);
  if (l.degree < 0)
    throw std::runtime_error(path + ": " + std::to_string(rest) + " f_rest properties, where a splat file has 0, 9, 24 or 45");
  for (size_t i = 0; i < rest; ++i) l.rest.push_back(column.at("f_rest_" + std::to_string(i)));
  return l;
}

struct Cloud {
  int degree = 0;
  size_t count = 0;
  std::vector<float> positions, scales, rotations, opacities, sh;
};

// One vertex's values (one float per column) into Gaussian v of the cloud; the
// file's f_rest is channel-major: every red coefficient, then green, then blue.
void store_vertex(const Layout &l, const float *values, Cloud &c, size_t v) {
  const size_t coeffs = (size_t)(c.degree + 1) * (c.degree + 1);
  for (int a = 0; a < 3; ++a) {
    c.positions[v * 3 + a] = values[l.position[a]];
    c.scales[v * 3 + a] = values[l.scale[a]];
    c.sh[v * coeffs * 3 + a] = values[l.dc[a]];
  }
  for (int a = 0; a < 4; ++a) c.rotations[v * 4 + a] = values[l.rotation[a]];
  c.opacities[v] = values[l.opacity];
  for (size_t ch = 0; ch < 3 && coeffs > 1; ++ch)
    for (size_t k = 1; k < coeffs; ++k) c.sh[(v * coeffs + k) * 3 + ch] = values[l.rest[ch * (coeffs - 1) + (k - 1)]];
}

Cloud load(const std::string &path, bool headerOnly) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw std::runtime_error("cannot open '" + path + "'");
  const PlyHeader h = read_header(in, path);
  const Layout l = layout_of(h, path);
  Cloud c;
  c.degree = l.degree;
  c.count = h.vertices;
  if (headerOnly) return c;
  const size_t coeffs = (size_t)(c.degree + 1) * (c.degree + 1);
  c.positions.resize(c.count * 3);
  c.scales.resize(c.count * 3);
  c.rotations.resize(c.count * 4);
  c.opacities.resize(c.count);
  c.sh.resize(c.count * coeffs * 3);
  std::vector<float> values(h.columns.size());
  const auto short_file = [&](size_t read) {
    return std::runtime_error(path + ": the file ends after " + std::to_string(read) + " of " + std::to_string(c.count) +
                              " vertices");
  };
  if (h.binary) {
    // Whole vertices in blocks of about 16 MB.
    const size_t perBlock = std::max<size_t>(1, ((size_t)16 << 20) / std::max<size_t>(h.recordBytes, 1));
    std::vector<unsigned char> block(h.recordBytes * std::min(perBlock, std::max<size_t>(c.count, 1)));
    for (size_t first = 0; first < c.count; first += perBlock) {
      const size_t n = std::min(perBlock, c.count - first);
      in.read(reinterpret_cast<char *>(block.data()), (std::streamsize)(n * h.recordBytes));
      const size_t got = (size_t)in.gcount();
      if (got != n * h.recordBytes) throw short_file(first + got / std::max<size_t>(h.recordBytes, 1));
      for (size_t i = 0; i < n; ++i) {
        const unsigned char *record = block.data() + i * h.recordBytes;
        if (h.allFloat) {
          std::memcpy(values.data(), record, h.recordBytes);
        } else {
          for (size_t p = 0; p < h.columns.size(); ++p) values[p] = value_of(h.columns[p].kind, record + h.columns[p].offset);
        }
        store_vertex(l, values.data(), c, first + i);
      }
    }
  } else {
    for (size_t v = 0; v < c.count; ++v) {
      for (size_t p = 0; p < h.columns.size(); ++p) {
        double d = 0.0;
        if (!(in >> d)) throw short_file(v);
        values[p] = (float)d;
      }
      store_vertex(l, values.data(), c, v);
    }
  }
  return c;
}

void save(const splat_cloud &cloud, const std::string &path) {
  if (cloud.count < 0 || cloud.sh_degree < 0 || cloud.sh_degree > 3) throw std::invalid_argument("bad cloud sizes");
  const size_t n = (size_t)cloud.count, coeffs = (size_t)(cloud.sh_degree + 1) * (cloud.sh_degree + 1);
  if (n > 0 && (cloud.positions == nullptr || cloud.scales == nullptr || cloud.rotations == nullptr || cloud.opacities == nullptr ||
                cloud.sh == nullptr))
    throw std::invalid_argument("null cloud array");
  std::ofstream out(path, std::ios::binary);
  if (!out) throw std::runtime_error("cannot write '" + path + "'");
  std::string header = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(n) + "\n";
  for (const char *name : {"x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"})
    header += std::string("property float ") + name + "\n";
  for (size_t i = 0; i < 3 * (coeffs - 1); ++i) header += "property float f_rest_" + std::to_string(i) + "\n";
  for (const char *name : {"opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"})
    header += std::string("property float ") + name + "\n";
  header += "end_header\n";
  out.write(header.data(), (std::streamsize)header.size());
  const size_t perVertex = 9 + 3 * (coeffs - 1) + 8;
  constexpr size_t kChunk = 1 << 14;
  std::vector<float> records(perVertex * kChunk);
  for (size_t first = 0; first < n; first += kChunk) {
    const size_t m = std::min(kChunk, n - first);
    for (size_t i = 0; i < m; ++i) {
      const size_t v = first + i;
      float *r = records.data() + i * perVertex;
      for (int a = 0; a < 3; ++a) *r++ = cloud.positions[v * 3 + a];
      for (int a = 0; a < 3; ++a) *r++ = 0.0f;
      for (int a = 0; a < 3; ++a) *r++ = cloud.sh[v * coeffs * 3 + a];
      for (size_t ch = 0; ch < 3 && coeffs > 1; ++ch)
        for (size_t k = 1; k < coeffs; ++k) *r++ = cloud.sh[(v * coeffs + k) * 3 + ch];
      *r++ = cloud.opacities[v];
      for (int a = 0; a < 3; ++a) *r++ = cloud.scales[v * 3 + a];
      for (int a = 0; a < 4; ++a) *r++ = cloud.rotations[v * 4 + a];
    }
    out.write(reinterpret_cast<const char *>(records.data()), (std::streamsize)(m * perVertex * sizeof(float)));
  }
  if (!out) throw std::runtime_error("failed writing '" + path + "'");
}

} // namespace
} // namespace sb

extern "C" int splat_cloud_load_ply(const char *path, int32_t *count, int32_t *sh_degree, float *positions, float *scales,
                                    float *rotations, float *opacities, float *sh) {
  try {
    if (path == nullptr || count == nullptr || sh_degree == nullptr) throw std::invalid_argument("null argument");
    const bool headerOnly = positions == nullptr && scales == nullptr && rotations == nullptr && opacities == nullptr && sh == nullptr;
    if (!headerOnly && (positions == nullptr || scales == nullptr || rotations == nullptr || opacities == nullptr || sh == nullptr))
      throw std::invalid_argument("either every array or none");
    const sb::Cloud c = sb::load(path, headerOnly);
    if (c.count > 0x7FFFFFFFull) throw std::runtime_error(std::string(path) + ": more Gaussians than the cloud's count holds");
    if (!headerOnly) {
      std::memcpy(positions, c.positions.data(), c.positions.size() * 4);
      std::memcpy(scales, c.scales.data(), c.scales.size() * 4);
      std::memcpy(rotations, c.rotations.data(), c.rotations.size() * 4);
      std::memcpy(opacities, c.opacities.data(), c.opacities.size() * 4);
      std::memcpy(sh, c.sh.data(), c.sh.size() * 4);
    }
    *count = (int32_t)c.count;
    *sh_degree = c.degree;
    sb::set_last_error("");
    return SPLAT_OK;
  } catch (const std::invalid_argument &e) {
    sb::set_last_error(e.what());
    return SPLAT_ERR_INVALID;
  } catch (const std::exception &e) {
    sb::set_last_error(e.what());
    return SPLAT_ERR_INVALID;
  }
}

extern "C" int splat_cloud_save_ply(const char *path, const splat_cloud *cloud) {
  try {
    if (path == nullptr || cloud == nullptr) throw std::invalid_argument("null argument");
    sb::save(*cloud, path);
    sb::set_last_error("");
    return SPLAT_OK;
  } catch (const std::invalid_argument &e) {
    sb::set_last_error(e.what());
    return SPLAT_ERR_INVALID;
  } catch (const std::exception &e) {
    sb::set_last_error(e.what());
    return SPLAT_ERR_INVALID;
  }
}
