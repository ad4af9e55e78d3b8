// A composite transform in ITK's text transform-file form, for the files antsRegistration writes with
// --write-composite-transform 1 (Examples/antsRegistrationTemplateHeader.h:1394-1424) and
// --save-state (:1307-1346) and reads with --restore-state (:293-328).  The reference writes these
// as HDF5 (.h5), which needs a library this build does not have; ITK's text form carries the same
// transforms and is what ITK's transform reader takes for a .txt/.tfm name:
//
//   #Insight Transform File V1.0
//   #Transform 0
//   Transform: CompositeTransform_double_3_3
//   #Transform 1
//   Transform: AffineTransform_double_3_3
//   Parameters: <A row-major, then t>
//   FixedParameters: <center>
//   #Transform 2
//   Transform: DisplacementFieldTransform_float_3_3
//   Parameters: <the field's vectors, voxel by voxel with x fastest, D components each>
//   FixedParameters: <size, origin, spacing, direction row-major>
//
// The first transform of the composite acts last on a point (ITK's composite queue order), as in
// antsApplyTransforms' -t list.  Field values are written in the shortest form that reads back to
// the same float.
#pragma once

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <new>
#include <stdexcept>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "synx.h"

namespace ants_b200 {
namespace composite {

struct Item {
  std::string type;             // e.g. "AffineTransform_double_3_3"
  std::vector<double> params;   // linear transforms
  std::vector<float> field;     // displacement fields (interleaved vectors)
  std::vector<double> fixed;    // fixed parameters
  bool is_field() const { return type.rfind("DisplacementFieldTransform_", 0) == 0; }
};

inline std::string suffix(const char* scalar, int dim) {
  return std::string("_") + scalar + "_" + std::to_string(dim) + "_" + std::to_string(dim);
}

inline Item linear_item(const synx_linear& t, int dim) {
  Item it;
  it.type = "AffineTransform" + suffix("double", dim);
  for (int r = 0; r < dim; ++r)
    for (int c = 0; c < dim; ++c) it.params.push_back(t.matrix[r * 3 + c]);
  for (int r = 0; r < dim; ++r) it.params.push_back(t.translation[r]);
  for (int r = 0; r < dim; ++r) it.fixed.push_back(t.center[r]);
  return it;
}

// A displacement field on grid g (interleaved vectors, D per voxel).
inline Item field_item(const synx_geom& g, const std::vector<float>& v, bool double_type) {
  Item it;
  const int dim = g.dim;
  it.type = "DisplacementFieldTransform" + suffix(double_type ? "double" : "float", dim);
  it.field = v;
  for (int k = 0; k < dim; ++k) it.fixed.push_back((double)g.size[k]);
  for (int k = 0; k < dim; ++k) it.fixed.push_back(g.origin[k]);
  for (int k = 0; k < dim; ++k) it.fixed.push_back(g.spacing[k]);
  for (int r = 0; r < dim; ++r)
    for (int c = 0; c < dim; ++c) it.fixed.push_back(g.direction[r * 3 + c]);
  return it;
}

// A linear entry (any type synx_read_linear_transform reads: affine, translation, identity, the
// rigid and similarity families) in matrix-offset form.
inline synx_linear to_linear(const Item& it, int dim) {
  synx_linear t;
  if (synx_linear_from_parameters(it.type.c_str(), it.params.data(), (int)it.params.size(), it.fixed.data(),
                                  (int)it.fixed.size(), dim, &t) != SYNX_OK)
    throw std::runtime_error(std::string("composite transform: ") + synx_last_error(nullptr));
  return t;
}

inline synx_geom field_geom(const Item& it, int dim) {
  if ((int)it.fixed.size() != dim * (3 + dim)) throw std::runtime_error("composite transform: bad field geometry");
  synx_geom g;
  std::memset(&g, 0, sizeof(g));
  g.dim = dim;
  g.size[0] = g.size[1] = g.size[2] = 1;
  g.spacing[0] = g.spacing[1] = g.spacing[2] = 1.0;
  g.direction[0] = g.direction[4] = g.direction[8] = 1.0;
  for (int k = 0; k < dim; ++k) {
    const double sz = it.fixed[k];
    if (!(sz >= 1.0 && sz <= 1e9 && sz == (double)(int64_t)sz) || !(it.fixed[2 * dim + k] > 0.0))
      throw std::runtime_error("composite transform: field sizes must be positive integers and spacings positive");
    g.size[k] = (int64_t)sz;
    g.origin[k] = it.fixed[dim + k];
    g.spacing[k] = it.fixed[2 * dim + k];
  }
  for (int r = 0; r < dim; ++r)
    for (int c = 0; c < dim; ++c) g.direction[r * 3 + c] = it.fixed[3 * dim + r * dim + c];
  const long long n = g.size[0] * g.size[1] * g.size[2];
  if ((long long)it.field.size() != n * dim)
    throw std::runtime_error("composite transform: field parameters do not match its size");
  return g;
}

inline bool text_name(const std::string& path) {
  auto ends = [&](const char* e) {
    const size_t n = std::strlen(e);
    if (path.size() < n) return false;
    for (size_t i = 0; i < n; ++i)
      if (std::tolower((unsigned char)path[path.size() - n + i]) != e[i]) return false;
    return true;
  };
  return ends(".txt") || ends(".tfm");
}

// " v_i0 v_i0+1 ... v_i1-1" into s (shortest round-trip forms).
template <class V>
inline void format_numbers(const V& v, size_t i0, size_t i1, std::string& s) {
  constexpr size_t kMaxNumber = 32;  // a sign, 17 digits, a point and a 5-character exponent fit
  s.resize((i1 - i0) * (kMaxNumber + 1));
  char* p = &s[0];
  char* const e = p + s.size();
  for (size_t i = i0; i < i1; ++i) {
    *p++ = ' ';
    p = std::to_chars(p, e, v[i]).ptr;
  }
  s.resize((size_t)(p - s.data()));
}

// One "key: v0 v1 ..." line.  A displacement field holds tens of millions of numbers: they are
// formatted in blocks of 4 M, each block split over the host's threads, and written in order, so the
// bytes are those of a sequential pass and the text held at once stays near 150 MB.
template <class V>
inline void write_numbers(std::FILE* f, const char* key, const V& v) {
  std::fputs(key, f);
  const size_t n = v.size();
  constexpr size_t kBlock = size_t(1) << 22, kSerial = size_t(1) << 16;
  const unsigned hw = n < kSerial ? 1u : std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::string> parts(hw);
  for (size_t b0 = 0; b0 < n; b0 += kBlock) {
    const size_t b1 = std::min(n, b0 + kBlock), per = (b1 - b0 + hw - 1) / hw;
    std::vector<char> ok(hw, 1);
    auto part = [&](unsigned t) {
      const size_t i0 = std::min(b1, b0 + t * per), i1 = std::min(b1, i0 + per);
      try {
        format_numbers(v, i0, i1, parts[t]);
      } catch (const std::bad_alloc&) {
        ok[t] = 0;  // thrown below, not across the thread
      }
    };
    std::vector<std::thread> pool;
    unsigned started = 1;
    try {
      for (; started < hw; ++started) pool.emplace_back(part, started);
    } catch (const std::system_error&) {
      // no more threads: the parts not started are formatted here
    }
    part(0);
    for (unsigned t = started; t < hw; ++t) part(t);
    for (std::thread& th : pool) th.join();
    if (std::find(ok.begin(), ok.end(), 0) != ok.end()) throw std::bad_alloc();
    for (const std::string& s : parts) std::fwrite(s.data(), 1, s.size(), f);
  }
  std::fputc('\n', f);
}

inline void write(const std::string& path, int dim, const std::vector<Item>& items) {
  if (!text_name(path))
    throw std::runtime_error("'" + path + "': composite transforms are written in ITK's text form (.txt or .tfm); "
                             "HDF5 (.h5) is not available in this build");
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot write '" + path + "'");
  std::fprintf(f, "#Insight Transform File V1.0\n#Transform 0\nTransform: CompositeTransform%s\n",
               suffix("double", dim).c_str());
  for (size_t k = 0; k < items.size(); ++k) {
    std::fprintf(f, "#Transform %zu\nTransform: %s\n", k + 1, items[k].type.c_str());
    if (items[k].is_field()) write_numbers(f, "Parameters:", items[k].field);
    else write_numbers(f, "Parameters:", items[k].params);
    write_numbers(f, "FixedParameters:", items[k].fixed);
  }
  const bool ok = std::ferror(f) == 0;
  if (std::fclose(f) != 0 || !ok) throw std::runtime_error("error writing '" + path + "'");
}

inline bool blank(char c) { return c == ' ' || c == '\t' || c == '\r'; }

// The numbers of [p, e) appended to v; false at the first text that is not a number.
template <class T>
inline bool parse_span(const char* p, const char* e, std::vector<T>& v) {
  while (true) {
    while (p < e && blank(*p)) ++p;
    if (p >= e) return true;
    T x{};
    auto r = std::from_chars(p, e, x);
    if (r.ec != std::errc()) return false;
    v.push_back(x);
    p = r.ptr;
  }
}

// The numbers of a parameter line from offset `from`.  A long line (a displacement field's) is cut at
// blanks into one span per host thread, the spans parsed at once and joined in order: cutting only at
// blanks keeps every number whole, so the result is that of one pass.
template <class T>
inline std::vector<T> parse_numbers(const std::string& s, size_t from, const std::string& path) {
  const char* const p = s.data() + from;
  const char* const e = s.data() + s.size();
  const size_t len = (size_t)(e - p);
  const unsigned hw =
      len < (size_t(1) << 20) ? 1u : std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<const char*> cut(hw + 1, e);
  cut[0] = p;
  for (unsigned t = 1; t < hw; ++t) {
    const char* c = std::max(cut[t - 1], p + len / hw * t);
    while (c < e && !blank(*c)) ++c;
    cut[t] = c;
  }
  std::vector<std::vector<T>> parts(hw);
  std::vector<char> ok(hw, 0);
  std::vector<char> oom(hw, 0);
  auto part = [&](unsigned t) {
    try {
      ok[t] = parse_span(cut[t], cut[t + 1], parts[t]) ? 1 : 0;
    } catch (const std::bad_alloc&) {
      oom[t] = 1;  // thrown below, not across the thread
    }
  };
  std::vector<std::thread> pool;
  unsigned started = 1;
  try {
    for (; started < hw; ++started) pool.emplace_back(part, started);
  } catch (const std::system_error&) {
    // no more threads: the spans not started are parsed here
  }
  part(0);
  for (unsigned t = started; t < hw; ++t) part(t);
  for (std::thread& th : pool) th.join();
  if (std::find(oom.begin(), oom.end(), 1) != oom.end()) throw std::bad_alloc();
  if (std::find(ok.begin(), ok.end(), 0) != ok.end())
    throw std::runtime_error("'" + path + "': bad number in a parameter line");
  if (hw == 1) return std::move(parts[0]);
  size_t total = 0;
  for (const auto& v : parts) total += v.size();
  std::vector<T> v;
  v.reserve(total);
  for (const auto& q : parts) v.insert(v.end(), q.begin(), q.end());
  return v;
}

// The transforms of a composite file, in its order (the composite's own entry left out).  A file
// holding a single transform reads as a composite of one.
inline std::vector<Item> read(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw std::runtime_error("cannot read '" + path + "'");
  std::vector<Item> items;
  std::string line;
  bool header = false;
  while (std::getline(in, line)) {
    if (line.rfind("#Insight Transform File", 0) == 0) {
      header = true;
      continue;
    }
    if (line.empty() || line[0] == '#') continue;
    const size_t colon = line.find(':');
    if (colon == std::string::npos) throw std::runtime_error("'" + path + "': unexpected line");
    const std::string key = line.substr(0, colon);
    if (key == "Transform") {
      size_t b = colon + 1;
      while (b < line.size() && line[b] == ' ') ++b;
      size_t e = line.size();
      while (e > b && (line[e - 1] == ' ' || line[e - 1] == '\r')) --e;
      const std::string type = line.substr(b, e - b);
      if (type.rfind("CompositeTransform_", 0) == 0) continue;
      items.push_back(Item{type, {}, {}, {}});
    } else if (key == "Parameters" || key == "FixedParameters") {
      if (items.empty()) throw std::runtime_error("'" + path + "': parameters before any transform");
      Item& it = items.back();
      if (key == "FixedParameters") it.fixed = parse_numbers<double>(line, colon + 1, path);
      else if (it.is_field()) it.field = parse_numbers<float>(line, colon + 1, path);
      else it.params = parse_numbers<double>(line, colon + 1, path);
    } else {
      throw std::runtime_error("'" + path + "': unexpected key '" + key + "'");
    }
  }
  if (!header) throw std::runtime_error("'" + path + "' is not an ITK text transform file");
  return items;
}

}  // namespace composite
}  // namespace ants_b200
