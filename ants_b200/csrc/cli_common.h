// Helpers shared by the command-line front ends (antsRegistration and antsApplyTransforms
// subsets): option-value parsing in the reference's name[p0,p1,...] syntax, NIfTI <-> synx_geom
// conversion, and device round trips through the synx C ABI step entry points.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "nifti_io.h"
#include "synx.h"

namespace ants_b200 {
namespace cli {

struct OptionCall {
  std::string name;                 // text before '[' (or the whole value)
  std::vector<std::string> params;  // comma-separated parameters inside [...]
};

// name[p0,p1,...] -> {name, params}; "[a,b]" -> {"", {a, b}}
inline OptionCall parse_call(const std::string& v) {
  OptionCall c;
  const size_t lb = v.find('[');
  if (lb == std::string::npos) {
    c.name = v;
    return c;
  }
  const size_t rb = v.rfind(']');
  if (rb == std::string::npos || rb < lb) throw std::runtime_error("unbalanced brackets in '" + v + "'");
  c.name = v.substr(0, lb);
  std::string inner = v.substr(lb + 1, rb - lb - 1);
  std::stringstream ss(inner);
  std::string item;
  while (std::getline(ss, item, ',')) c.params.push_back(item);
  return c;
}

template <class T>
inline std::vector<T> parse_x_vector(const std::string& s) {
  std::vector<T> out;
  std::stringstream ss(s);
  std::string item;
  while (std::getline(ss, item, 'x')) {
    if (item.empty()) continue;
    std::stringstream is(item);
    T v;
    is >> v;
    if (is.fail()) throw std::runtime_error("cannot parse '" + s + "' as an x-separated vector");
    out.push_back(v);
  }
  return out;
}

inline std::string lower(std::string s) {
  std::transform(s.begin(), s.end(), s.begin(), ::tolower);
  return s;
}

inline synx_geom to_geom(const nifti::Image& im, int dim) {
  synx_geom g;
  std::memset(&g, 0, sizeof(g));
  g.dim = dim;
  for (int k = 0; k < 3; ++k) {
    g.size[k] = k < dim ? im.size[k] : 1;
    g.spacing[k] = k < dim ? im.spacing[k] : 1.0;
    g.origin[k] = k < dim ? im.origin[k] : 0.0;
  }
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      g.direction[r * 3 + c] = (r < dim && c < dim) ? im.direction[r * 3 + c] : (r == c ? 1.0 : 0.0);
  return g;
}

inline nifti::Image field_image(const synx_geom& g, const std::vector<float>& interleaved) {
  nifti::Image im;
  im.dim = g.dim;
  im.components = g.dim;
  for (int k = 0; k < 3; ++k) {
    im.size[k] = g.size[k];
    im.spacing[k] = g.spacing[k];
    im.origin[k] = g.origin[k];
  }
  for (int k = 0; k < 9; ++k) im.direction[k] = g.direction[k];
  const long long N = im.voxels();
  im.data.resize((size_t)N * g.dim);
  for (long long i = 0; i < N; ++i)
    for (int c = 0; c < g.dim; ++c) im.data[(size_t)c * N + i] = interleaved[(size_t)i * g.dim + c];
  return im;
}

#define CLI_CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) throw std::runtime_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// An affine map p -> M p + b (3x3 row-major; a 2-D map keeps the third row and column identity).
struct Map {
  double M[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  double b[3] = {0, 0, 0};
};

inline Map mul(const Map& second, const Map& first) {  // second(first(p))
  Map r;
  for (int i = 0; i < 3; ++i) {
    r.b[i] = second.b[i];
    for (int k = 0; k < 3; ++k) {
      double s = 0.0;
      for (int m = 0; m < 3; ++m) s += second.M[i * 3 + m] * first.M[m * 3 + k];
      r.M[i * 3 + k] = s;
      r.b[i] += second.M[i * 3 + k] * first.b[k];
    }
  }
  return r;
}

inline bool inverse(const Map& a, Map& r) {
  const double* m = a.M;
  const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                     m[2] * (m[3] * m[7] - m[4] * m[6]);
  double scale = 0.0;
  for (int k = 0; k < 9; ++k) scale = std::max(scale, std::fabs(m[k]));
  if (!(std::fabs(det) > 1e-12 * scale * scale * scale)) return false;
  const double id = 1.0 / det;
  r.M[0] = (m[4] * m[8] - m[5] * m[7]) * id;
  r.M[1] = (m[2] * m[7] - m[1] * m[8]) * id;
  r.M[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  r.M[3] = (m[5] * m[6] - m[3] * m[8]) * id;
  r.M[4] = (m[0] * m[8] - m[2] * m[6]) * id;
  r.M[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  r.M[6] = (m[3] * m[7] - m[4] * m[6]) * id;
  r.M[7] = (m[1] * m[6] - m[0] * m[7]) * id;
  r.M[8] = (m[0] * m[4] - m[1] * m[3]) * id;
  for (int i = 0; i < 3; ++i) {
    r.b[i] = 0.0;
    for (int k = 0; k < 3; ++k) r.b[i] -= r.M[i * 3 + k] * a.b[k];
  }
  return true;
}

// T(p) = A (p - c) + t + c, or its inverse.
inline Map map_of(const synx_linear& t, bool invert) {
  Map m;
  for (int k = 0; k < 9; ++k) m.M[k] = t.matrix[k];
  if (t.dim == 2) {
    m.M[2] = m.M[5] = m.M[6] = m.M[7] = 0.0;
    m.M[8] = 1.0;
  }
  for (int i = 0; i < 3; ++i) {
    m.b[i] = i < t.dim ? t.translation[i] + t.center[i] : 0.0;
    for (int k = 0; k < t.dim; ++k) m.b[i] -= m.M[i * 3 + k] * t.center[k];
  }
  if (!invert) return m;
  Map r;
  if (!inverse(m, r)) throw std::runtime_error("a linear transform of the stack has a singular matrix, no inverse");
  return r;
}

// The grid whose voxel i sits at L(p_i), p_i the voxel of g: direction M D, origin M o + b.
inline synx_geom push_forward(const synx_geom& g, const Map& L) {
  synx_geom r = g;
  for (int i = 0; i < 3; ++i) {
    r.origin[i] = L.b[i];
    for (int k = 0; k < 3; ++k) {
      r.origin[i] += L.M[i * 3 + k] * g.origin[k];
      double s = 0.0;
      for (int m = 0; m < 3; ++m) s += L.M[i * 3 + m] * g.direction[m * 3 + k];
      r.direction[i * 3 + k] = s;
    }
  }
  return r;
}

// One linear transform of a .mat/.txt/.tfm file, in application order.
struct LinearItem {
  synx_linear linear;
  Map map;  // the map applied (already inverted for [file,1])
};

// The transforms of a linear transform file in the order they act on a point: the composite the
// file holds applies its last transform first; its inverse ([file,1]) applies the inverse of the
// first one first (itkantsRegistrationHelper.h:1440-1451 expands a composite in that order).
inline std::vector<LinearItem> read_linear_file(const std::string& file, int dim, bool invert) {
  const int n = synx_read_linear_transform(file.c_str(), dim, 0, nullptr);
  if (n < 0) throw std::runtime_error(synx_last_error(nullptr));
  std::vector<LinearItem> items;
  for (int i = 0; i < n; ++i) {
    LinearItem li;
    if (synx_read_linear_transform(file.c_str(), dim, i, &li.linear) < 0)
      throw std::runtime_error(synx_last_error(nullptr));
    li.map = map_of(li.linear, invert);
    items.push_back(li);
  }
  if (!invert) std::reverse(items.begin(), items.end());
  return items;
}

// The AffineTransform form of a map with a chosen center: A = M, t = b - c + M c.
inline synx_linear linear_of(const Map& m, int dim, const double center[3]) {
  synx_linear t;
  std::memset(&t, 0, sizeof(t));
  t.dim = dim;
  t.has_center = 1;
  for (int k = 0; k < 9; ++k) t.matrix[k] = m.M[k];
  for (int i = 0; i < dim; ++i) {
    t.center[i] = center[i];
    t.translation[i] = m.b[i] - center[i];
    for (int k = 0; k < dim; ++k) t.translation[i] += m.M[i * 3 + k] * center[k];
  }
  return t;
}

// out(x) = img(x + u(x)) on grid `grid` (u interleaved on that grid), through synx_warp_image.
inline std::vector<float> warp_on_device(const nifti::Image& img, const synx_geom& gimg, const std::vector<float>& u_inter,
                                  const synx_geom& grid) {
  const long long Ni = img.voxels(), No = grid.size[0] * grid.size[1] * grid.size[2];
  const int D = grid.dim;
  std::vector<float> planes((size_t)No * D);
  for (long long i = 0; i < No; ++i)
    for (int c = 0; c < D; ++c) planes[(size_t)c * No + i] = u_inter[(size_t)i * D + c];
  float *di = nullptr, *du = nullptr, *dout = nullptr;
  CLI_CK(cudaMalloc(&di, 4 * Ni));
  CLI_CK(cudaMalloc(&du, 4 * No * D));
  CLI_CK(cudaMalloc(&dout, 4 * No));
  CLI_CK(cudaMemcpy(di, img.data.data(), 4 * Ni, cudaMemcpyHostToDevice));
  CLI_CK(cudaMemcpy(du, planes.data(), 4 * No * D, cudaMemcpyHostToDevice));
  int rc = synx_warp_image(di, &gimg, du, &grid, dout, nullptr);
  std::vector<float> out((size_t)No);
  if (rc == 0) CLI_CK(cudaMemcpy(out.data(), dout, 4 * No, cudaMemcpyDeviceToHost));
  cudaFree(di);
  cudaFree(du);
  cudaFree(dout);
  if (rc) throw std::runtime_error(std::string("synx_warp_image: ") + synx_last_error(nullptr));
  return out;
}

// u (interleaved, on grid a) resampled onto grid b, through synx_resample_field.
inline std::vector<float> resample_on_device(const std::vector<float>& u_inter, const synx_geom& a, const synx_geom& b) {
  const int D = a.dim;
  const long long Na = a.size[0] * a.size[1] * a.size[2], Nb = b.size[0] * b.size[1] * b.size[2];
  std::vector<float> planes((size_t)Na * D), out_planes((size_t)Nb * D), out((size_t)Nb * D);
  for (long long i = 0; i < Na; ++i)
    for (int c = 0; c < D; ++c) planes[(size_t)c * Na + i] = u_inter[(size_t)i * D + c];
  float *din = nullptr, *dout = nullptr;
  CLI_CK(cudaMalloc(&din, 4 * Na * D));
  CLI_CK(cudaMalloc(&dout, 4 * Nb * D));
  CLI_CK(cudaMemcpy(din, planes.data(), 4 * Na * D, cudaMemcpyHostToDevice));
  int rc = synx_resample_field(din, &a, dout, &b, nullptr);
  if (rc == 0) CLI_CK(cudaMemcpy(out_planes.data(), dout, 4 * Nb * D, cudaMemcpyDeviceToHost));
  cudaFree(din);
  cudaFree(dout);
  if (rc) throw std::runtime_error(std::string("synx_resample_field: ") + synx_last_error(nullptr));
  for (long long i = 0; i < Nb; ++i)
    for (int c = 0; c < D; ++c) out[(size_t)i * D + c] = out_planes[(size_t)c * Nb + i];
  return out;
}

}  // namespace cli
}  // namespace ants_b200
