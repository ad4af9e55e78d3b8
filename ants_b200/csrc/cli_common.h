// Helpers shared by the command-line front ends (antsRegistration and antsApplyTransforms
// subsets): option-value parsing in the reference's name[p0,p1,...] syntax, NIfTI <-> synx_geom
// conversion, and device round trips through the synx C ABI step entry points.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
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
