// Linear transforms of ITK transform files, as antsApplyTransforms reads them in its transform
// stack (Utilities/itkantsReadWriteTransform.h:19-120 hands .mat/.txt files to ITK's transform
// file reader), and their displacement fields on a grid.  Host code only.
//
// File forms:
//  * MATLAB v4 binary (.mat), the form ITK's MATLAB transform IO writes: a sequence of variables,
//    each a 20-byte header of 32-bit integers (type, rows, columns, imaginary flag, name length
//    including its NUL), the name, then rows x columns values.  The type's decimal digits M O P T
//    are: M byte order (0 little, 1 big endian), O storage order (0 by columns, 1 by rows; vnl
//    writes either, a vector reads the same both ways), P element type (0 double, 1 float) and
//    T = 0 (a full numeric matrix).  A variable named after a transform type holds that
//    transform's parameters; the variable "fixed" after it holds its fixed parameters.
//  * Insight text (.txt, or .tfm, the other name ITK's text transform IO takes): "#Insight Transform
//    File V1.0", then per transform a "Transform: <type>"
//    line, a "Parameters:" line and a "FixedParameters:" line (the form
//    Scripts/ANTSAverage3DAffine.sh:94-98 writes).
// Type names are <Base>_<double|float>_<D>_<D>.  Every supported type is reduced to the
// matrix-offset form T(p) = A (p - c) + t + c on physical points, with ITK's parameter layouts:
//   AffineTransform, MatrixOffsetTransformBase  A (row-major, D*D), t (D)      fixed: c
//   TranslationTransform                        t (D)                          A = I, c = 0
//   IdentityTransform                           -                              A = I, t = c = 0
//   Euler2DTransform, Rigid2DTransform          angle, t (2)                   fixed: c
//   Similarity2DTransform                       scale, angle, t (2)            fixed: c
//   Euler3DTransform                            angles x, y, z, t (3)          fixed: c [, ZYX flag]
//       A = Rz Rx Ry, or Rz Ry Rx when the fourth fixed parameter is non-zero
//   VersorRigid3DTransform                      versor x, y, z, t (3)          fixed: c
//   Similarity3DTransform                       versor x, y, z, t (3), scale   fixed: c
// A versor (x, y, z) is the unit quaternion with w = sqrt(1 - x^2 - y^2 - z^2).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/synx.h"
#include "synx_host.h"

namespace {

struct RawTransform {
  std::string type;  // full type name
  std::vector<double> params, fixed;
};

struct ReadError {
  int code;
  std::string msg;
};

[[noreturn]] void fail(int code, const std::string& msg) { throw ReadError{code, msg}; }

std::string lower_ext(const std::string& path) {
  const size_t dot = path.find_last_of('.');
  const size_t slash = path.find_last_of('/');
  if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) return "";
  std::string e = path.substr(dot);
  for (char& ch : e) ch = (char)std::tolower((unsigned char)ch);
  return e;
}

std::vector<char> slurp(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) fail(SYNX_E_ARG, "cannot open transform file '" + path + "'");
  return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

uint32_t bswap32(uint32_t v) {
  return (v >> 24) | ((v >> 8) & 0xff00u) | ((v << 8) & 0xff0000u) | (v << 24);
}

// ---- MATLAB v4 --------------------------------------------------------------------------------
std::vector<RawTransform> parse_mat(const std::vector<char>& buf, const std::string& path) {
  std::vector<RawTransform> out;
  size_t pos = 0;
  while (pos < buf.size()) {
    if (buf.size() - pos < 20) fail(SYNX_E_ARG, "'" + path + "': truncated MATLAB variable header");
    uint32_t h[5];
    std::memcpy(h, buf.data() + pos, 20);
    bool big = false;
    if (h[0] / 1000 != 0 || h[0] > 199) {  // not a little-endian type word: try big endian
      for (uint32_t& v : h) v = bswap32(v);
      big = true;
      if (h[0] / 1000 != 1 || h[0] % 1000 > 199)
        fail(SYNX_E_ARG, "'" + path + "' is not a MATLAB v4 file (type word " + std::to_string(h[0]) + ")");
    }
    const uint32_t type = h[0] % 1000, rows = h[1], cols = h[2], imag = h[3], namelen = h[4];
    const uint32_t prec = (type / 10) % 10, kind = type % 10;
    if (kind != 0 || imag != 0) fail(SYNX_E_ARG, "'" + path + "': only real numeric MATLAB matrices are supported");
    if (prec > 1) fail(SYNX_E_ARG, "'" + path + "': only double or single MATLAB matrices are supported");
    if (namelen < 1 || namelen > 4096) fail(SYNX_E_ARG, "'" + path + "': bad MATLAB variable name length");
    const uint64_t count = (uint64_t)rows * cols;
    if (rows > 1 && cols > 1) fail(SYNX_E_ARG, "'" + path + "': a transform variable must be a vector");
    if (count > (1u << 20)) fail(SYNX_E_ARG, "'" + path + "': MATLAB variable too large");
    const size_t esize = prec == 0 ? 8 : 4;
    pos += 20;
    if (buf.size() - pos < namelen + count * esize) fail(SYNX_E_ARG, "'" + path + "': truncated MATLAB variable");
    std::string name(buf.data() + pos, strnlen(buf.data() + pos, namelen));
    pos += namelen;
    std::vector<double> vals(count);
    for (uint64_t i = 0; i < count; ++i) {
      const char* p = buf.data() + pos + i * esize;
      if (esize == 8) {
        uint64_t u;
        std::memcpy(&u, p, 8);
        if (big) u = ((uint64_t)bswap32((uint32_t)u) << 32) | bswap32((uint32_t)(u >> 32));
        double d;
        std::memcpy(&d, &u, 8);
        vals[i] = d;
      } else {
        uint32_t u;
        std::memcpy(&u, p, 4);
        if (big) u = bswap32(u);
        float f;
        std::memcpy(&f, &u, 4);
        vals[i] = f;
      }
    }
    pos += count * esize;
    if (name == "fixed") {
      if (out.empty()) fail(SYNX_E_ARG, "'" + path + "': fixed parameters before any transform");
      out.back().fixed = vals;
    } else {
      out.push_back(RawTransform{name, vals, {}});
    }
  }
  return out;
}

// ---- Insight text ------------------------------------------------------------------------------
std::vector<double> parse_numbers(const std::string& s, const std::string& path) {
  std::vector<double> v;
  std::istringstream in(s);
  std::string tok;
  while (in >> tok) {
    char* end = nullptr;
    const double d = std::strtod(tok.c_str(), &end);
    if (end == tok.c_str() || *end != '\0') fail(SYNX_E_ARG, "'" + path + "': bad number '" + tok + "'");
    v.push_back(d);
  }
  return v;
}

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

std::vector<RawTransform> parse_txt(const std::vector<char>& buf, const std::string& path) {
  std::vector<RawTransform> out;
  std::istringstream in(std::string(buf.begin(), buf.end()));
  std::string line;
  bool header = false;
  while (std::getline(in, line)) {
    const std::string t = trim(line);
    if (t.empty()) continue;
    if (t[0] == '#') {
      if (t.find("Insight Transform File") != std::string::npos) header = true;
      continue;
    }
    const size_t colon = t.find(':');
    if (colon == std::string::npos) fail(SYNX_E_ARG, "'" + path + "': unexpected line '" + t + "'");
    const std::string key = trim(t.substr(0, colon)), val = trim(t.substr(colon + 1));
    if (key == "Transform") {
      out.push_back(RawTransform{val, {}, {}});
    } else if (key == "Parameters" || key == "FixedParameters") {
      if (out.empty()) fail(SYNX_E_ARG, "'" + path + "': " + key + " before any Transform line");
      (key == "Parameters" ? out.back().params : out.back().fixed) = parse_numbers(val, path);
    } else {
      fail(SYNX_E_ARG, "'" + path + "': unexpected key '" + key + "'");
    }
  }
  if (!header) fail(SYNX_E_ARG, "'" + path + "' is not an Insight transform text file");
  return out;
}

// ---- type names and parameter layouts ------------------------------------------------------
void split_type(const std::string& full, std::string& base, int& d1, int& d2, const std::string& path) {
  // <Base>_<precision>_<D>_<D>
  std::vector<std::string> parts;
  size_t start = 0;
  for (size_t i = 0; i <= full.size(); ++i)
    if (i == full.size() || full[i] == '_') {
      parts.push_back(full.substr(start, i - start));
      start = i + 1;
    }
  if (parts.size() < 4 || (parts[parts.size() - 3] != "double" && parts[parts.size() - 3] != "float"))
    fail(SYNX_E_ARG, "'" + path + "': unrecognised transform type '" + full + "'");
  base.clear();
  for (size_t i = 0; i + 3 < parts.size(); ++i) base += (i ? "_" : "") + parts[i];
  d1 = std::atoi(parts[parts.size() - 2].c_str());
  d2 = std::atoi(parts[parts.size() - 1].c_str());
}

void need(const RawTransform& r, size_t np, const std::string& path) {
  if (r.params.size() != np)
    fail(SYNX_E_ARG, "'" + path + "': " + r.type + " has " + std::to_string(r.params.size()) + " parameters, expected " +
                         std::to_string(np));
}

void set_center(synx_linear& L, const RawTransform& r, int D, const std::string& path) {
  if (r.fixed.empty()) return;
  if ((int)r.fixed.size() < D)
    fail(SYNX_E_ARG, "'" + path + "': " + r.type + " has " + std::to_string(r.fixed.size()) + " fixed parameters");
  for (int k = 0; k < D; ++k) L.center[k] = r.fixed[k];
}

void versor_matrix(double x, double y, double z, double A[9], const std::string& path) {
  const double n2 = x * x + y * y + z * z;
  if (n2 > 1.0 + 1e-9) fail(SYNX_E_ARG, "'" + path + "': versor with norm above 1");
  const double w = std::sqrt(std::max(0.0, 1.0 - n2));
  A[0] = 1 - 2 * (y * y + z * z);
  A[1] = 2 * (x * y - z * w);
  A[2] = 2 * (x * z + y * w);
  A[3] = 2 * (x * y + z * w);
  A[4] = 1 - 2 * (x * x + z * z);
  A[5] = 2 * (y * z - x * w);
  A[6] = 2 * (x * z - y * w);
  A[7] = 2 * (y * z + x * w);
  A[8] = 1 - 2 * (x * x + y * y);
}

void matmul3(const double a[9], const double b[9], double c[9]) {
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) c[r * 3 + k] = a[r * 3] * b[k] + a[r * 3 + 1] * b[3 + k] + a[r * 3 + 2] * b[6 + k];
}

// Returns false for a composite placeholder (skipped); fails for unsupported types.
bool to_linear(const RawTransform& r, int dim, synx_linear& L, const std::string& path) {
  std::string base;
  int d1 = 0, d2 = 0;
  split_type(r.type, base, d1, d2, path);
  if (base == "CompositeTransform") return false;
  if (d1 != dim || d2 != dim)
    fail(SYNX_E_ARG, "'" + path + "': " + r.type + " is not a " + std::to_string(dim) + "-D transform");
  std::memset(&L, 0, sizeof(L));
  L.dim = dim;
  L.matrix[0] = L.matrix[4] = L.matrix[8] = 1.0;
  L.has_center = (base == "TranslationTransform" || base == "IdentityTransform") ? 0 : 1;
  const int D = dim;
  const std::vector<double>& p = r.params;
  if (base == "AffineTransform" || base == "MatrixOffsetTransformBase") {
    need(r, (size_t)(D * D + D), path);
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) L.matrix[i * 3 + j] = p[i * D + j];
    for (int k = 0; k < D; ++k) L.translation[k] = p[D * D + k];
    set_center(L, r, D, path);
  } else if (base == "TranslationTransform") {
    need(r, (size_t)D, path);
    for (int k = 0; k < D; ++k) L.translation[k] = p[k];
  } else if (base == "IdentityTransform") {
    if (!p.empty()) need(r, 0, path);
  } else if (D == 2 && (base == "Euler2DTransform" || base == "Rigid2DTransform" || base == "Similarity2DTransform")) {
    const bool sim = base == "Similarity2DTransform";
    need(r, sim ? 4 : 3, path);
    const double s = sim ? p[0] : 1.0, th = p[sim ? 1 : 0];
    L.matrix[0] = s * std::cos(th);
    L.matrix[1] = -s * std::sin(th);
    L.matrix[3] = s * std::sin(th);
    L.matrix[4] = s * std::cos(th);
    L.translation[0] = p[sim ? 2 : 1];
    L.translation[1] = p[sim ? 3 : 2];
    set_center(L, r, D, path);
  } else if (D == 3 && base == "Euler3DTransform") {
    need(r, 6, path);
    const double cx = std::cos(p[0]), sx = std::sin(p[0]), cy = std::cos(p[1]), sy = std::sin(p[1]),
                 cz = std::cos(p[2]), sz = std::sin(p[2]);
    const double Rx[9] = {1, 0, 0, 0, cx, -sx, 0, sx, cx};
    const double Ry[9] = {cy, 0, sy, 0, 1, 0, -sy, 0, cy};
    const double Rz[9] = {cz, -sz, 0, sz, cz, 0, 0, 0, 1};
    const bool zyx = r.fixed.size() > 3 && r.fixed[3] != 0.0;
    double T[9];
    matmul3(Rz, zyx ? Ry : Rx, T);
    matmul3(T, zyx ? Rx : Ry, L.matrix);
    for (int k = 0; k < 3; ++k) L.translation[k] = p[3 + k];
    set_center(L, r, D, path);
  } else if (D == 3 && (base == "VersorRigid3DTransform" || base == "Similarity3DTransform")) {
    const bool sim = base == "Similarity3DTransform";
    need(r, sim ? 7 : 6, path);
    versor_matrix(p[0], p[1], p[2], L.matrix, path);
    if (sim)
      for (double& a : L.matrix) a *= p[6];
    for (int k = 0; k < 3; ++k) L.translation[k] = p[3 + k];
    set_center(L, r, D, path);
  } else {
    fail(SYNX_E_UNSUPPORTED, "'" + path + "': transform type " + r.type + " is not supported");
  }
  return true;
}

bool invert_matrix(const double A[9], int dim, double Ai[9]) {
  double M[9];
  std::memcpy(M, A, sizeof(M));
  if (dim == 2) {
    M[2] = M[5] = M[6] = M[7] = 0.0;
    M[8] = 1.0;
  }
  const double c00 = M[4] * M[8] - M[5] * M[7], c01 = M[5] * M[6] - M[3] * M[8], c02 = M[3] * M[7] - M[4] * M[6];
  const double det = M[0] * c00 + M[1] * c01 + M[2] * c02;
  double scale = 0.0;
  for (double v : M) scale = std::max(scale, std::fabs(v));
  if (!(std::fabs(det) > 1e-12 * scale * scale * scale)) return false;
  const double id = 1.0 / det;
  Ai[0] = c00 * id;
  Ai[1] = (M[2] * M[7] - M[1] * M[8]) * id;
  Ai[2] = (M[1] * M[5] - M[2] * M[4]) * id;
  Ai[3] = c01 * id;
  Ai[4] = (M[0] * M[8] - M[2] * M[6]) * id;
  Ai[5] = (M[2] * M[3] - M[0] * M[5]) * id;
  Ai[6] = c02 * id;
  Ai[7] = (M[1] * M[6] - M[0] * M[7]) * id;
  Ai[8] = (M[0] * M[4] - M[1] * M[3]) * id;
  return true;
}

}  // namespace

extern "C" {

int synx_read_linear_transform(const char* path, int dim, int index, synx_linear* out) {
  const char* fn = "synx_read_linear_transform: ";
  if (!path) return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "null path");
  if (dim != 2 && dim != 3) return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "dim must be 2 or 3");
  try {
    const std::string p(path);
    const std::string ext = lower_ext(p);
    if (ext != ".mat" && ext != ".txt" && ext != ".tfm")
      fail(SYNX_E_UNSUPPORTED, "'" + p + "': linear transforms are read from .mat, .txt or .tfm files");
    const std::vector<char> buf = slurp(p);
    const std::vector<RawTransform> raw = ext == ".mat" ? parse_mat(buf, p) : parse_txt(buf, p);
    std::vector<synx_linear> lin;
    for (const RawTransform& r : raw) {
      synx_linear L;
      if (to_linear(r, dim, L, p)) lin.push_back(L);
    }
    if (lin.empty()) fail(SYNX_E_ARG, "'" + p + "' holds no transform");
    if (out) {
      if (index < 0 || index >= (int)lin.size())
        fail(SYNX_E_ARG, "'" + p + "': transform index " + std::to_string(index) + " out of range");
      *out = lin[index];
    }
    return (int)lin.size();
  } catch (const ReadError& e) {
    return synx::set_global_error(e.code, fn + e.msg);
  } catch (const std::exception& e) {
    return synx::set_global_error(SYNX_E_ARG, fn + std::string(e.what()));
  }
}

int synx_linear_from_parameters(const char* type, const double* params, int n_params, const double* fixed,
                                int n_fixed, int dim, synx_linear* out) {
  const char* fn = "synx_linear_from_parameters: ";
  if (!type || !out || n_params < 0 || n_fixed < 0 || (n_params > 0 && !params) || (n_fixed > 0 && !fixed))
    return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "null pointer or negative count");
  if (dim != 2 && dim != 3) return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "dim must be 2 or 3");
  try {
    RawTransform r{type, std::vector<double>(params, params + n_params), std::vector<double>(fixed, fixed + n_fixed)};
    synx_linear L;
    if (!to_linear(r, dim, L, r.type)) fail(SYNX_E_ARG, "'" + r.type + "': a composite is not a linear transform");
    *out = L;
    return SYNX_OK;
  } catch (const ReadError& e) {
    return synx::set_global_error(e.code, fn + e.msg);
  } catch (const std::exception& e) {
    return synx::set_global_error(SYNX_E_ARG, fn + std::string(e.what()));
  }
}

int synx_linear_field(const synx_linear* t, int invert, const synx_geom* g, float* field) {
  const char* fn = "synx_linear_field: ";
  if (!t || !g || !field) return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "null argument");
  const int D = g->dim;
  if ((D != 2 && D != 3) || t->dim != D)
    return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "transform and grid dimensions differ");
  if (g->size[0] < 1 || g->size[1] < 1 || g->size[2] < 1 || (D == 2 && g->size[2] != 1))
    return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "bad grid size");
  // T(p) = A (p - c) + t + c, or T^-1(p) = A^-1 (p - t - c) + c: both are M p + b
  double M[9], b[3];
  if (invert) {
    if (!invert_matrix(t->matrix, D, M))
      return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "the matrix is singular, no inverse");
  } else {
    std::memcpy(M, t->matrix, sizeof(M));
  }
  if (D == 2) {
    M[2] = M[5] = M[6] = M[7] = 0.0;
    M[8] = 1.0;
  }
  double q[3];  // the point M is applied to is p - q
  for (int k = 0; k < 3; ++k) q[k] = k < D ? (invert ? t->translation[k] + t->center[k] : t->center[k]) : 0.0;
  for (int r = 0; r < 3; ++r) {
    b[r] = r < D ? (invert ? t->center[r] : t->translation[r] + t->center[r]) : 0.0;
    for (int k = 0; k < 3; ++k) b[r] -= M[r * 3 + k] * q[k];
  }
  // p(i) = origin + Dir diag(spacing) i; u = (M - I) p + b
  double E[9];  // (M - I) Dir diag(spacing)
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) {
      double s = 0.0;
      for (int m = 0; m < 3; ++m) {
        const double mi = M[r * 3 + m] - (r == m ? 1.0 : 0.0);
        const double dir = (m < D && k < D) ? g->direction[m * 3 + k] : (m == k ? 1.0 : 0.0);
        s += mi * dir;
      }
      E[r * 3 + k] = k < D ? s * g->spacing[k] : 0.0;
    }
  double u0[3];
  for (int r = 0; r < 3; ++r) {
    u0[r] = b[r];
    for (int m = 0; m < D; ++m) u0[r] += (M[r * 3 + m] - (r == m ? 1.0 : 0.0)) * g->origin[m];
  }
  // component planes: component r of voxel i at field[r * N + i]
  const int64_t nx = g->size[0], ny = g->size[1], nz = D == 3 ? g->size[2] : 1;
  const size_t N = (size_t)(nx * ny * nz);
  size_t i = 0;
  for (int64_t z = 0; z < nz; ++z)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t x = 0; x < nx; ++x, ++i) {
        const double i0 = (double)x, i1 = (double)y, i2 = (double)z;
        for (int r = 0; r < D; ++r)
          field[(size_t)r * N + i] = (float)(u0[r] + E[r * 3] * i0 + E[r * 3 + 1] * i1 + E[r * 3 + 2] * i2);
      }
  return SYNX_OK;
}

int synx_initial_translation(const float* F, const synx_geom* gf, const float* M, const synx_geom* gm, int feature,
                             synx_linear* out) {
  const char* fn = "synx_initial_translation: ";
  if (!gf || !gm || !out) return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "null argument");
  const int D = gf->dim;
  if ((D != 2 && D != 3) || gm->dim != D)
    return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "the images' dimensions differ or are not 2 or 3");
  if (feature < 0 || feature > 2)
    return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "feature must be 0 (centers), 1 (centers of mass) "
                                                                "or 2 (origins)");
  if (feature == 1 && (!F || !M)) return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "images are needed");
  // physical point of continuous index idx: origin + Dir diag(spacing) idx
  auto point = [D](const synx_geom* g, const double idx[3], double p[3]) {
    for (int r = 0; r < 3; ++r) {
      p[r] = r < D ? g->origin[r] : 0.0;
      if (r < D)
        for (int c = 0; c < D; ++c) p[r] += g->direction[r * 3 + c] * g->spacing[c] * idx[c];
    }
  };
  double cf[3] = {0, 0, 0}, cm[3] = {0, 0, 0};
  for (int k = 0; k < 2; ++k) {
    const synx_geom* g = k ? gm : gf;
    double* c = k ? cm : cf;
    if (feature == 2) {
      for (int r = 0; r < D; ++r) c[r] = g->origin[r];
    } else if (feature == 0) {
      double idx[3] = {0, 0, 0};
      for (int r = 0; r < D; ++r) idx[r] = (double)(g->size[r] - 1) / 2.0;
      point(g, idx, c);
    } else {
      const float* img = k ? M : F;
      const int64_t nx = g->size[0], ny = g->size[1], nz = D == 3 ? g->size[2] : 1;
      double m0 = 0.0, m1[3] = {0, 0, 0};
      size_t i = 0;
      for (int64_t z = 0; z < nz; ++z)
        for (int64_t y = 0; y < ny; ++y)
          for (int64_t x = 0; x < nx; ++x, ++i) {
            const double v = img[i];
            const double idx[3] = {(double)x, (double)y, (double)z};
            double p[3];
            point(g, idx, p);
            m0 += v;
            for (int r = 0; r < D; ++r) m1[r] += v * p[r];
          }
      if (m0 == 0.0)
        return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "the total mass of the " +
                                                      (k ? "moving" : "fixed") + " image is zero");
      for (int r = 0; r < D; ++r) c[r] = m1[r] / m0;
    }
  }
  std::memset(out, 0, sizeof(*out));
  out->dim = D;
  out->has_center = 1;
  out->matrix[0] = out->matrix[4] = out->matrix[8] = 1.0;
  for (int r = 0; r < D; ++r) {
    out->center[r] = cf[r];
    out->translation[r] = cm[r] - cf[r];
  }
  return SYNX_OK;
}

int synx_write_linear_transform(const char* path, const synx_linear* t) {
  const char* fn = "synx_write_linear_transform: ";
  if (!path || !t) return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "null argument");
  const int D = t->dim;
  if (D != 2 && D != 3) return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "dim must be 2 or 3");
  const std::string p(path), ext = lower_ext(p);
  if (ext != ".mat" && ext != ".txt" && ext != ".tfm")
    return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "'" + p + "': write a .mat, .txt or .tfm file");
  std::vector<double> params, fixed;
  for (int i = 0; i < D; ++i)
    for (int j = 0; j < D; ++j) params.push_back(t->matrix[i * 3 + j]);
  for (int k = 0; k < D; ++k) params.push_back(t->translation[k]);
  for (int k = 0; k < D; ++k) fixed.push_back(t->center[k]);
  const std::string type = "AffineTransform_double_" + std::to_string(D) + "_" + std::to_string(D);
  std::ofstream f(p, std::ios::binary);
  if (!f) return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "cannot write '" + p + "'");
  if (ext == ".mat") {
    auto var = [&](const std::string& name, const std::vector<double>& v) {
      // type 0: little-endian IEEE, column-wise, double, full numeric matrix; a column vector
      const int32_t h[5] = {0, (int32_t)v.size(), 1, 0, (int32_t)name.size() + 1};
      char hb[20];
      for (int k = 0; k < 5; ++k) {
        const uint32_t u = (uint32_t)h[k];
        for (int b = 0; b < 4; ++b) hb[k * 4 + b] = (char)((u >> (8 * b)) & 0xff);
      }
      f.write(hb, 20);
      f.write(name.c_str(), (std::streamsize)name.size() + 1);
      for (double d : v) {
        uint64_t u;
        std::memcpy(&u, &d, 8);
        char db[8];
        for (int b = 0; b < 8; ++b) db[b] = (char)((u >> (8 * b)) & 0xff);
        f.write(db, 8);
      }
    };
    var(type, params);
    var("fixed", fixed);
  } else {
    char buf[64];
    auto line = [&](const char* key, const std::vector<double>& v) {
      f << key;
      for (double d : v) {
        std::snprintf(buf, sizeof(buf), " %.17g", d);
        f << buf;
      }
      f << "\n";
    };
    f << "#Insight Transform File V1.0\n#Transform 0\nTransform: " << type << "\n";
    line("Parameters:", params);
    line("FixedParameters:", fixed);
  }
  f.close();
  if (!f) return synx::set_global_error(SYNX_E_ARG, std::string(fn) + "cannot write '" + p + "'");
  return SYNX_OK;
}

}  // extern "C"
