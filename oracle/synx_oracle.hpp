// synx CPU oracle -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement of the arithmetic that antsRegistration's SyN stage with the
// neighbourhood cross-correlation metric runs per iteration (-t SyN[eta,varU,varT]
// -m CC[f,m,1,r]).  It exists to check the CUDA path; the product never links it.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu-baseline leg may load it.
//
// PARITY UNPINNED.  The hot-path arithmetic of the reference lives in ITK (pinned by the
// reference SuperBuild at ITK v6 18d89fd6538769ac83d8e21ba0e10593c6c68751, or v5.4.6
// f7ff6ad56d487d9f52e6ba1dbbd9a816a14b5158), which is not vendored in the reference tree,
// cannot be fetched here and ships no golden vectors for SyN+CC.  Each function below
// restates ITK's published algorithm and cites the in-tree ANTs twin or call site it follows;
// where the in-tree twin and the ITK behaviour differ the comment says which one is used.
// Known-answer tests (analytic fields, independent Bessel evaluation, brute-force CC) pin the
// restatement in tests/test_oracle_*.py.
//
// Layouts: images are x-fastest arrays of n[0]*n[1]*n[2] values (n[2] = 1 in 2-D).  Vector
// fields are component planes ("SoA"): component c of voxel i lives at f[c*N + i].
//
// T is the storage/arithmetic type (float mirrors `antsRegistration --float 1`, double is the
// FP64 oracle).  Window sums of the CC metric, metric means, inverse-residual means and
// intensity statistics accumulate in double in both instantiations.
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace synx_oracle {

inline double omp_seconds() {
#ifdef _OPENMP
  return omp_get_wtime();
#else
  return 0.0;
#endif
}

// ------------------------------------------------------------------------------------------
// Geometry: ITK image information (index -> physical point p = origin + D * diag(sp) * idx).
// ------------------------------------------------------------------------------------------
struct Geom {
  int dim = 3;
  int64_t n[3] = {1, 1, 1};
  double sp[3] = {1, 1, 1};
  double org[3] = {0, 0, 0};
  double dir[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};  // row-major direction cosines
  double i2p[9];  // D * diag(sp)
  double p2i[9];  // inverse of i2p

  int64_t count() const { return n[0] * n[1] * n[2]; }

  void finalize() {
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) i2p[r * 3 + c] = dir[r * 3 + c] * sp[c];
    if (dim == 2) {
      i2p[2] = i2p[5] = i2p[6] = i2p[7] = 0.0;
      i2p[8] = 1.0;
      n[2] = 1;
    }
    const double* a = i2p;
    double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                 a[2] * (a[3] * a[7] - a[4] * a[6]);
    double id = 1.0 / det;
    p2i[0] = (a[4] * a[8] - a[5] * a[7]) * id;
    p2i[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    p2i[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    p2i[3] = (a[5] * a[6] - a[3] * a[8]) * id;
    p2i[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    p2i[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    p2i[6] = (a[3] * a[7] - a[4] * a[6]) * id;
    p2i[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    p2i[8] = (a[0] * a[4] - a[1] * a[3]) * id;
  }
  void index_to_point(const double idx[3], double p[3]) const {
    for (int r = 0; r < 3; ++r)
      p[r] = org[r] + i2p[r * 3 + 0] * idx[0] + i2p[r * 3 + 1] * idx[1] + i2p[r * 3 + 2] * idx[2];
    if (dim == 2) p[2] = 0.0;
  }
  void point_to_cindex(const double p[3], double c[3]) const {
    double d[3] = {p[0] - org[0], p[1] - org[1], dim == 3 ? p[2] - org[2] : 0.0};
    for (int r = 0; r < 3; ++r) c[r] = p2i[r * 3 + 0] * d[0] + p2i[r * 3 + 1] * d[1] + p2i[r * 3 + 2] * d[2];
    if (dim == 2) c[2] = 0.0;
  }
};

// ------------------------------------------------------------------------------------------
// Linear interpolation with ITK's buffer rule.
//
// ITK's ImageFunction::IsInsideBuffer accepts a continuous index c when
// start-0.5 <= c < end+0.5 on every axis; LinearInterpolateImageFunction and
// VectorLinearInterpolateImageFunction then clamp the base index to the buffer and drop the
// upper neighbour beyond the last index, which is clamp-to-edge multilinear interpolation in
// the half-voxel rim.  Points outside the buffer take the caller's default (0 for resampling,
// "no displacement" for composition).  Pattern used in antsRegistration's warps
// (Examples/itkantsRegistrationHelper.hxx:721-763) and in the observer's resampling
// (Examples/antsDisplacementAndVelocityFieldRegistrationCommandIterationUpdate.h:342-381).
// ------------------------------------------------------------------------------------------
inline bool inside_buffer(const Geom& g, const double c[3]) {
  for (int d = 0; d < g.dim; ++d)
    if (!(c[d] >= -0.5 && c[d] < (double)g.n[d] - 0.5)) return false;
  return true;
}

struct LerpCell {
  int64_t i0[3], i1[3];
  double w[3];
};

inline void lerp_cell(const Geom& g, const double c[3], LerpCell& L) {
  for (int d = 0; d < 3; ++d) {
    if (d >= g.dim) {
      L.i0[d] = L.i1[d] = 0;
      L.w[d] = 0.0;
      continue;
    }
    double f = std::floor(c[d]);
    int64_t b = (int64_t)f;
    double w = c[d] - f;
    if (b < 0) {  // rim below index 0: clamp to edge
      b = 0;
      w = 0.0;
    }
    int64_t u = b + 1;
    if (u > g.n[d] - 1) {  // rim above the last index: clamp to edge
      u = g.n[d] - 1;
      w = 0.0;
    }
    L.i0[d] = b;
    L.i1[d] = u;
    L.w[d] = w;
  }
}

template <class T>
inline T lerp_plane(const T* a, const Geom& g, const LerpCell& L) {
  const int64_t nx = g.n[0], nxy = g.n[0] * g.n[1];
  auto at = [&](int64_t x, int64_t y, int64_t z) { return a[z * nxy + y * nx + x]; };
  T wx = (T)L.w[0], wy = (T)L.w[1], wz = (T)L.w[2];
  T v00 = at(L.i0[0], L.i0[1], L.i0[2]), v10 = at(L.i1[0], L.i0[1], L.i0[2]);
  T v01 = at(L.i0[0], L.i1[1], L.i0[2]), v11 = at(L.i1[0], L.i1[1], L.i0[2]);
  T a0 = v00 + (v10 - v00) * wx;
  T a1 = v01 + (v11 - v01) * wx;
  T b0 = a0 + (a1 - a0) * wy;
  if (g.dim == 2) return b0;
  T u00 = at(L.i0[0], L.i0[1], L.i1[2]), u10 = at(L.i1[0], L.i0[1], L.i1[2]);
  T u01 = at(L.i0[0], L.i1[1], L.i1[2]), u11 = at(L.i1[0], L.i1[1], L.i1[2]);
  T c0 = u00 + (u10 - u00) * wx;
  T c1 = u01 + (u11 - u01) * wx;
  T b1 = c0 + (c1 - c0) * wy;
  return b0 + (b1 - b0) * wz;
}

// ------------------------------------------------------------------------------------------
// Discrete Gaussian kernel (ITK GaussianOperator::GenerateCoefficients).
//
// Lindeberg's discrete analogue of the Gaussian: k(n) = e^{-t} I_n(t), t = variance in pixel
// units.  I_0 and I_1 use the polynomial approximations of Abramowitz & Stegun 9.8.1-9.8.4
// (the published approximations ITK evaluates); higher orders use the recurrence
// I_{n}(t) = I_{n-2}(t) - 2 (n-1) I_{n-1}(t) / t.  Coefficients are added until the two-sided
// sum reaches 1 - maxError, or the half-kernel exceeds maxWidth, then normalised to sum 1 and
// mirrored.  Callers: field smoothing (max error 0.001, max width = field size,
// Examples/SmoothDisplacementField.cxx:70-125) and the level pyramid (max error 0.01,
// max width 32, ITK DiscreteGaussianImageFilter defaults).
// ------------------------------------------------------------------------------------------
inline double bessel_i0_as(double y) {
  double ay = std::fabs(y);
  if (ay < 3.75) {
    double t = (y / 3.75) * (y / 3.75);
    return 1.0 + t * (3.5156229 + t * (3.0899424 + t * (1.2067492 + t * (0.2659732 + t * (0.0360768 + t * 0.0045813)))));
  }
  double t = 3.75 / ay;
  return (std::exp(ay) / std::sqrt(ay)) *
         (0.39894228 + t * (0.01328592 + t * (0.00225319 + t * (-0.00157565 + t * (0.00916281 +
          t * (-0.02057706 + t * (0.02635537 + t * (-0.01647633 + t * 0.00392377))))))));
}

inline double bessel_i1_as(double y) {
  double ay = std::fabs(y), ans;
  if (ay < 3.75) {
    double t = (y / 3.75) * (y / 3.75);
    ans = ay * (0.5 + t * (0.87890594 + t * (0.51498869 + t * (0.15084934 + t * (0.02658733 + t * (0.00301532 + t * 0.00032411))))));
  } else {
    double t = 3.75 / ay;
    ans = 0.02282967 + t * (-0.02895312 + t * (0.01787654 - t * 0.00420059));
    ans = 0.39894228 + t * (-0.03988024 + t * (-0.00362018 + t * (0.00163801 + t * (-0.01031555 + t * ans))));
    ans *= std::exp(ay) / std::sqrt(ay);
  }
  return y < 0.0 ? -ans : ans;
}

// Returns the full symmetric kernel (odd length 2R+1), in double.
inline std::vector<double> gaussian_kernel(double variance, double max_error, size_t max_width) {
  std::vector<double> half;
  const double t = variance;
  const double et = std::exp(-t);
  const double cap = 1.0 - max_error;
  double sum = 0.0;
  half.push_back(et * bessel_i0_as(t));
  sum += half[0];
  half.push_back(et * bessel_i1_as(t));
  sum += half[1] * 2.0;
  for (int i = 2; sum < cap; ++i) {
    half.push_back(half[i - 2] - 2.0 * (i - 1) * half[i - 1] / t);
    sum += half[i] * 2.0;
    if (half[i] <= 0.0) break;               // recurrence underflow: stop (ITK warns)
    if (half.size() > max_width) break;      // kernel wider than allowed: truncate (ITK warns)
  }
  for (double& c : half) c /= sum;
  const size_t R = half.size() - 1;
  std::vector<double> k(2 * R + 1);
  for (size_t i = 0; i <= R; ++i) k[R + i] = k[R - i] = half[i];
  return k;
}

// One separable pass along `axis` with zero-flux Neumann (replicate-edge) boundary, the
// default boundary condition of ITK's NeighborhoodOperatorImageFilter family.
template <class Tin, class Tacc, class Tout>
inline void convolve_axis(const Tin* in, Tout* out, const Geom& g, int axis, const std::vector<double>& k) {
  const int64_t nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int64_t stride = axis == 0 ? 1 : (axis == 1 ? nx : nx * ny);
  const int64_t len = g.n[axis];
  const int R = (int)(k.size() / 2);
  std::vector<Tacc> kk(k.size());
  for (size_t i = 0; i < k.size(); ++i) kk[i] = (Tacc)k[i];
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t z = 0; z < nz; ++z)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t x = 0; x < nx; ++x) {
        int64_t base = z * nx * ny + y * nx + x;
        int64_t pos = axis == 0 ? x : (axis == 1 ? y : z);
        int64_t line0 = base - pos * stride;
        Tacc s = 0;
        for (int j = -R; j <= R; ++j) {
          int64_t q = std::min<int64_t>(std::max<int64_t>(pos + j, 0), len - 1);
          s += kk[j + R] * (Tacc)in[line0 + q * stride];
        }
        out[base] = (Tout)s;
      }
}

// Pyramid smoothing of a full-resolution image (ITK DiscreteGaussianImageFilter as configured
// by ImageRegistrationMethodv4 per level: variance sigma^2, max error 0.01, max kernel width 32,
// variance in voxel units for `-s ...vox`, or divided by spacing^2 per axis for `mm`).  The
// filter chains its axis passes from the last axis to the first and carries double between
// passes.  Smoothing sigmas per level: Examples/itkantsRegistrationHelper.hxx:1276-1289,
// :2141-2150.
template <class T>
inline void smooth_image(const T* in, T* out, const Geom& g, double sigma, bool sigma_in_mm) {
  const int64_t N = g.count();
  if (sigma <= 0.0) {
    std::memcpy(out, in, sizeof(T) * N);
    return;
  }
  std::vector<double> a(in, in + N), b(N);
  for (int axis = g.dim - 1; axis >= 0; --axis) {
    double var = sigma * sigma;
    if (sigma_in_mm) var /= g.sp[axis] * g.sp[axis];
    auto k = gaussian_kernel(var, 0.01, 32);
    convolve_axis<double, double, double>(a.data(), b.data(), g, axis, k);
    std::swap(a, b);
  }
  for (int64_t i = 0; i < N; ++i) out[i] = (T)a[i];
}

// ------------------------------------------------------------------------------------------
// Level geometry.  CalculateShrinkFactorsPerDimension: Examples/itkantsRegistrationHelper.hxx
// :593-641.  Shrunk grid: ShrinkImageFilter::GenerateOutputInformation as called through
// GetShrinkImageOutputInformation (hxx:16-39): size = max(1, floor(n/f)), spacing * f,
// origin shifted so that the physical centres of both grids coincide.
// ------------------------------------------------------------------------------------------
inline void shrink_factors_per_dim(int dim, unsigned factor, const double sp[3], unsigned out[3]) {
  double minSp = sp[0];
  int minIdx = 0;
  for (int n = 1; n < dim; ++n)
    if (minSp > sp[n]) { minSp = sp[n]; minIdx = n; }
  for (int n = 0; n < 3; ++n) out[n] = 0;
  out[minIdx] = factor;
  double newSpMin = sp[minIdx] * factor;
  for (int n = 0; n < dim; ++n) {
    if (out[n] != 0) continue;
    double best = std::fabs(sp[n] * factor - newSpMin);
    unsigned bestF = factor;
    for (unsigned f = factor - 1; f > 0; --f) {
      double d = std::fabs(sp[n] * f - newSpMin);
      if (d <= best) { best = d; bestF = f; }
    }
    out[n] = bestF;
  }
  if (dim == 2) out[2] = 1;
}

inline Geom shrink_geom(const Geom& in, const unsigned f[3]) {
  Geom out = in;
  for (int d = 0; d < in.dim; ++d) {
    out.sp[d] = in.sp[d] * (double)f[d];
    int64_t s = (int64_t)std::floor((double)in.n[d] / (double)f[d]);
    out.n[d] = s < 1 ? 1 : s;
  }
  out.finalize();
  double ci[3] = {0, 0, 0}, co[3] = {0, 0, 0};
  for (int d = 0; d < in.dim; ++d) {
    ci[d] = (in.n[d] - 1) / 2.0;
    co[d] = (out.n[d] - 1) / 2.0;
  }
  double pin[3], pout[3];
  in.index_to_point(ci, pin);
  out.index_to_point(co, pout);
  for (int d = 0; d < 3; ++d) out.org[d] = in.org[d] + (pin[d] - pout[d]);
  if (in.dim == 2) out.org[2] = in.org[2];
  out.finalize();
  return out;
}

// ------------------------------------------------------------------------------------------
// Histogram quantile with linear interpolation inside the bin that reaches p, as ITK's
// Histogram::Quantile computes it (ITK 5.4.6, Modules/Numerics/Statistics/include/itkHistogram.hxx;
// the version is pinned in SuperBuild/External_ITKv5.cmake:155).  Equal-width bins: bin b spans
// [lo + b*bw, lo + (b+1)*bw).  Below p = 0.5 the frequencies are accumulated from the first bin
// upward, otherwise from the last bin downward.
// ------------------------------------------------------------------------------------------
inline double histogram_quantile(const std::vector<double>& freq, double lo, double bw, double p) {
  const int nb = (int)freq.size();
  double total = 0.0;
  for (double f : freq) total += f;
  auto bin_min = [&](int b) { return lo + b * bw; };
  auto bin_max = [&](int b) { return lo + (b + 1) * bw; };
  double cum = 0.0, pn = 0.0, pprev = 0.0, fn = 0.0;
  if (p < 0.5) {
    int n = 0;
    do {
      fn = freq[n];
      cum += fn;
      pprev = pn;
      pn = cum / total;
      ++n;
    } while (n < nb && pn < p);
    double prop = fn / total;
    return bin_min(n - 1) + ((p - pprev) / prop) * (bin_max(n - 1) - bin_min(n - 1));
  }
  int n = nb - 1, m = 0;
  pn = 1.0;
  do {
    fn = freq[n];
    cum += fn;
    pprev = pn;
    pn = 1.0 - cum / total;
    --n;
    ++m;
  } while (m < nb && pn > p);
  double prop = fn / total;
  return bin_max(n + 1) - ((pprev - p) / prop) * (bin_max(n + 1) - bin_min(n + 1));
}

// ------------------------------------------------------------------------------------------
// Intensity preprocessing (PreprocessImage, Examples/itkantsRegistrationHelper.hxx:76-136):
// 256-bin histogram with automatic min/max and marginal scale 10 (the upper bound is raised by
// (max-min)/256/10), quantiles -> intensity window -> linear map to [0, 1] with clamping.
// ------------------------------------------------------------------------------------------
template <class T>
inline void preprocess_image(const T* in, T* out, int64_t N, float qlo, float qhi) {
  float mn = (float)in[0], mx = (float)in[0];
  for (int64_t i = 1; i < N; ++i) {
    mn = std::min(mn, (float)in[i]);
    mx = std::max(mx, (float)in[i]);
  }
  const int nb = 256;
  float margin = ((mx - mn) / (float)nb) / 10.0f;
  float hi = mx + margin;
  std::vector<double> freq(nb, 0.0);
  double bw = ((double)hi - (double)mn) / nb;
  for (int64_t i = 0; i < N; ++i) {
    int b = bw > 0 ? (int)(((double)in[i] - (double)mn) / bw) : 0;
    b = std::min(std::max(b, 0), nb - 1);
    freq[b] += 1.0;
  }
  auto quantile = [&](double p) { return histogram_quantile(freq, (double)mn, bw, p); };
  float wlo = (float)quantile(qlo), whi = (float)quantile(qhi);
  double scale = (1.0 - 0.0) / ((double)whi - (double)wlo);
  double shift = 0.0 - (double)wlo * scale;
  for (int64_t i = 0; i < N; ++i) {
    float a = (float)in[i];
    if (a < wlo) out[i] = (T)0;
    else if (a > whi) out[i] = (T)1;
    else out[i] = (T)((double)a * scale + shift);
  }
}

// ------------------------------------------------------------------------------------------
// Warp an image onto a grid through a displacement field defined on that grid:
// out(i) = img(x_i + u(x_i)), linear, 0 outside the image buffer.  This is the resampling
// SyN runs each iteration with DownsampleImagesForMetricDerivatives on
// (Examples/itkantsRegistrationHelper.hxx:2138), mirrored in-tree by the observer
// (Examples/antsDisplacementAndVelocityFieldRegistrationCommandIterationUpdate.h:342-381).
// ------------------------------------------------------------------------------------------
template <class T>
inline void warp_image(const T* img, const Geom& gi, const T* u, const Geom& gv, T* out) {
  const int64_t N = gv.count();
  const int64_t nx = gv.n[0], ny = gv.n[1];
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; ++i) {
    double idx[3] = {(double)(i % nx), (double)((i / nx) % ny), (double)(i / (nx * ny))};
    double p[3];
    gv.index_to_point(idx, p);
    for (int d = 0; d < gv.dim; ++d) p[d] += (double)u[d * N + i];
    double c[3];
    gi.point_to_cindex(p, c);
    if (!inside_buffer(gi, c)) {
      out[i] = (T)0;
      continue;
    }
    LerpCell L;
    lerp_cell(gi, c, L);
    out[i] = lerp_plane(img, gi, L);
  }
}

// Same warp with nearest-neighbour sampling, as antsApplyTransforms -n NearestNeighbor selects it
// (Examples/make_interpolator_snip.tmpl:24-28): ITK's NearestNeighborInterpolateImageFunction
// reads, inside the buffer, the voxel at RoundHalfIntegerUp(c) = floor(c + 0.5) per axis.
template <class T>
inline void warp_image_nearest(const T* img, const Geom& gi, const T* u, const Geom& gv, T* out) {
  const int64_t N = gv.count();
  const int64_t nx = gv.n[0], ny = gv.n[1];
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; ++i) {
    double idx[3] = {(double)(i % nx), (double)((i / nx) % ny), (double)(i / (nx * ny))};
    double p[3];
    gv.index_to_point(idx, p);
    for (int d = 0; d < gv.dim; ++d) p[d] += (double)u[d * N + i];
    double c[3];
    gi.point_to_cindex(p, c);
    if (!inside_buffer(gi, c)) {
      out[i] = (T)0;
      continue;
    }
    int64_t k[3] = {0, 0, 0};
    for (int d = 0; d < gi.dim; ++d) k[d] = std::min<int64_t>(std::max<int64_t>((int64_t)std::floor(c[d] + 0.5), 0), gi.n[d] - 1);
    out[i] = img[(k[2] * gi.n[1] + k[1]) * gi.n[0] + k[0]];
  }
}

// Same warp with the generic label interpolation antsApplyTransforms -n GenericLabel[Linear] selects
// (Examples/make_interpolator_snip.tmpl:112-117): ITK's LabelImageGenericInterpolateImageFunction
// interpolates the indicator image of every label with the linear interpolator and returns the label
// with the largest value, scanning its (sorted) label set and keeping a strictly larger value, so a
// tie goes to the smaller label.  With linear interpolation the value of a label is the sum of the
// weights of the cell corners that carry it; labels absent from the cell have value 0 and never win.
template <class T>
inline void warp_image_label(const T* img, const Geom& gi, const T* u, const Geom& gv, T* out) {
  const int64_t N = gv.count();
  const int64_t nx = gv.n[0], ny = gv.n[1];
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; ++i) {
    double idx[3] = {(double)(i % nx), (double)((i / nx) % ny), (double)(i / (nx * ny))};
    double p[3];
    gv.index_to_point(idx, p);
    for (int d = 0; d < gv.dim; ++d) p[d] += (double)u[d * N + i];
    double c[3];
    gi.point_to_cindex(p, c);
    if (!inside_buffer(gi, c)) {
      out[i] = (T)0;
      continue;
    }
    LerpCell L;
    lerp_cell(gi, c, L);
    double lab[8], acc[8];
    int n = 0;
    const int corners = gi.dim == 3 ? 8 : 4;
    for (int k = 0; k < corners; ++k) {
      const int bx = k & 1, by = (k >> 1) & 1, bz = (k >> 2) & 1;
      const int64_t x = bx ? L.i1[0] : L.i0[0], y = by ? L.i1[1] : L.i0[1], z = bz ? L.i1[2] : L.i0[2];
      const double w = (bx ? L.w[0] : 1.0 - L.w[0]) * (by ? L.w[1] : 1.0 - L.w[1]) *
                       (gi.dim == 3 ? (bz ? L.w[2] : 1.0 - L.w[2]) : 1.0);
      const double v = (double)img[(z * gi.n[1] + y) * gi.n[0] + x];
      int j = 0;
      while (j < n && lab[j] != v) ++j;
      if (j == n) {
        lab[n] = v;
        acc[n] = 0.0;
        ++n;
      }
      acc[j] += w;
    }
    int best = 0;
    for (int j = 1; j < n; ++j)
      if (acc[j] > acc[best] || (acc[j] == acc[best] && lab[j] < lab[best])) best = j;
    out[i] = (T)lab[best];
  }
}

// ------------------------------------------------------------------------------------------
// Neighbourhood cross-correlation value and derivatives.
//
// ITK ANTSNeighborhoodCorrelationImageToImageMetricv4 (configured at
// Examples/itkantsRegistrationHelper.hxx:938-945 and :1154-1156) restated with the in-tree
// twin ImageRegistration/itkCrossCorrelationRegistrationFunction.cxx:
//   * sums over the in-bounds voxels of the (2r+1)^D box, n = their count (:179-306, Qcount);
//   * sFF = SFF - 2 mF SF + n mF^2, sMM likewise, sFM = SFM - mM SF - mF SM + n mM mF with
//     mF = SF/n (:291-296);  F^ = F(x) - mF, M^ = M(x) - mM;
//   * cc = sFM^2 / (sFF sMM) when sFF > eps and sMM > eps, else cc = 1 and no derivative;
//   * the derivative with respect to a displacement of the metric's moving image,
//     2 sFM/(sFF sMM) (F^ - sFM/sMM M^) grad M (twin :443-504, ascent sign of the v4 metric);
//     SyN evaluates it once per half with the roles swapped (fixed-to-middle update uses
//     grad of the warped moving image, moving-to-middle uses grad of the warped fixed image);
//   * value = -mean(cc) over the grid.
// Metric masks (antsRegistration -x [fixedMask,movingMask], Examples/antsRegistration.cxx:471-480,
// set on the metric at Examples/itkantsRegistrationHelper.hxx:1159-1166): SyN resamples each mask
// into the virtual domain through the same half-field as its image, nearest-neighbour with 0
// outside, and a virtual voxel is valid where both warped masks are nonzero.  Invalid voxels add
// nothing to the window sums or to n (the count of valid voxels in the window, ITK's Qcount), and
// an invalid centre has no cc and no derivative; the value is -mean(cc) over the valid centres.
// (ITK's mask handling in SyN and in the metric's scan is restated as recalled: unpinned.)
// grad: ITK CentralDifferenceImageFunction at grid points, i.e. (I(x+h/2) - I(x-h/2)) / h with
// linear interpolation and the buffer rule above: (I[x+1]-I[x-1])/(2h) inside, 0.5(I[1]-I[0])/h
// at index 0 (x-h/2 lies on the buffer rim), 0 at the last index (x+h/2 is outside), then
// rotated by the direction matrix.  Sums accumulate in double.
// ------------------------------------------------------------------------------------------
struct CCResult {
  double value;      // -mean cc
  double sum_cc;
};

template <class T>
inline double grad_axis(const T* I, const Geom& g, int64_t x, int64_t y, int64_t z, int axis) {
  const int64_t nx = g.n[0], nxy = g.n[0] * g.n[1];
  int64_t pos = axis == 0 ? x : (axis == 1 ? y : z);
  int64_t len = g.n[axis];
  int64_t stride = axis == 0 ? 1 : (axis == 1 ? nx : nxy);
  int64_t i = z * nxy + y * nx + x;
  if (len < 2 || pos == len - 1) return 0.0;
  double h = g.sp[axis];
  if (pos == 0) return 0.5 * ((double)I[i + stride] - (double)I[i]) / h;
  return ((double)I[i + stride] - (double)I[i - stride]) / (2.0 * h);
}

template <class T>
inline CCResult cc_metric(const T* F, const T* M, const Geom& g, int r, T* gradF_upd, T* gradM_upd,
                          T* cc_out = nullptr, double eps = 1.1920928955078125e-07,
                          const unsigned char* valid = nullptr) {
  const int64_t nx = g.n[0], ny = g.n[1], nz = g.n[2], N = g.count();
  const int rz = g.dim == 3 ? r : 0;
  // separable running box sums in double: 5 quantities, and with metric masks a sixth, the number
  // of valid voxels in the window (invalid voxels add nothing to any sum)
  const int NQ = valid ? 6 : 5;
  std::vector<double> q[6], t[6];
  for (int k = 0; k < NQ; ++k) {
    q[k].resize(N);
    t[k].resize(N);
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; ++i) {
    const double v = valid ? (valid[i] ? 1.0 : 0.0) : 1.0;
    double f = v != 0.0 ? (double)F[i] : 0.0, m = v != 0.0 ? (double)M[i] : 0.0;
    q[0][i] = f;
    q[1][i] = m;
    q[2][i] = f * f;
    q[3][i] = m * m;
    q[4][i] = f * m;
    if (valid) q[5][i] = v;
  }
  auto box_axis = [&](std::vector<double>* src, std::vector<double>* dst, int axis, int rad) {
    const int64_t stride = axis == 0 ? 1 : (axis == 1 ? nx : nx * ny);
    const int64_t len = g.n[axis];
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t z = 0; z < nz; ++z)
      for (int64_t y = 0; y < ny; ++y)
        for (int64_t x = 0; x < nx; ++x) {
          int64_t pos = axis == 0 ? x : (axis == 1 ? y : z);
          int64_t base = z * nx * ny + y * nx + x;
          int64_t line0 = base - pos * stride;
          int64_t lo = std::max<int64_t>(pos - rad, 0), hi = std::min<int64_t>(pos + rad, len - 1);
          for (int k = 0; k < NQ; ++k) {
            double s = 0.0;
            for (int64_t j = lo; j <= hi; ++j) s += src[k][line0 + j * stride];
            dst[k][base] = s;
          }
        }
  };
  box_axis(q, t, 0, r);
  box_axis(t, q, 1, r);
  if (g.dim == 3) box_axis(q, t, 2, rz);
  std::vector<double>* S = g.dim == 3 ? t : q;
  double sum_cc = 0.0;
  std::vector<double> slice_cc(nz, 0.0);
  std::vector<int64_t> slice_n(nz, 0);
#pragma omp parallel for schedule(static)
  for (int64_t z = 0; z < nz; ++z) {
    double acc = 0.0;
    int64_t cnt = 0;
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t x = 0; x < nx; ++x) {
        int64_t i = z * nx * ny + y * nx + x;
        if (valid && !valid[i]) {  // a masked-out voxel: no value, no update
          if (cc_out) cc_out[i] = (T)0;
          for (int d = 0; d < g.dim; ++d) gradF_upd[d * N + i] = gradM_upd[d * N + i] = (T)0;
          continue;
        }
        ++cnt;
        double cx = (double)(std::min<int64_t>(x + r, nx - 1) - std::max<int64_t>(x - r, 0) + 1);
        double cy = (double)(std::min<int64_t>(y + r, ny - 1) - std::max<int64_t>(y - r, 0) + 1);
        double cz = (double)(std::min<int64_t>(z + rz, nz - 1) - std::max<int64_t>(z - rz, 0) + 1);
        double n = valid ? S[5][i] : cx * cy * cz;
        double sF = S[0][i], sM = S[1][i], sFF2 = S[2][i], sMM2 = S[3][i], sFM2 = S[4][i];
        double mF = sF / n, mM = sM / n;
        double sFF = sFF2 - mF * sF - mF * sF + n * mF * mF;
        double sMM = sMM2 - mM * sM - mM * sM + n * mM * mM;
        double sFM = sFM2 - mM * sF - mF * sM + n * mM * mF;
        double fh = (double)F[i] - mF, mh = (double)M[i] - mM;
        double cc = 1.0;
        double aF = 0.0, aM = 0.0;  // scalar factors multiplying grad M and grad F
        if (sFF > eps && sMM > eps) {
          double sFFsMM = sFF * sMM;
          cc = sFM * sFM / sFFsMM;
          double coef = 2.0 * sFM / sFFsMM;
          aF = coef * (fh - sFM / sMM * mh);
          aM = coef * (mh - sFM / sFF * fh);
        }
        acc += cc;
        if (cc_out) cc_out[i] = (T)cc;
        double gM[3] = {0, 0, 0}, gF[3] = {0, 0, 0};
        for (int a = 0; a < g.dim; ++a) {
          gM[a] = grad_axis(M, g, x, y, z, a);
          gF[a] = grad_axis(F, g, x, y, z, a);
        }
        // index-axis derivatives -> physical (direction matrix)
        for (int d = 0; d < g.dim; ++d) {
          double pm = 0.0, pf = 0.0;
          for (int a = 0; a < g.dim; ++a) {
            pm += g.dir[d * 3 + a] * gM[a];
            pf += g.dir[d * 3 + a] * gF[a];
          }
          gradF_upd[d * N + i] = (T)(aF * pm);
          gradM_upd[d * N + i] = (T)(aM * pf);
        }
      }
    slice_cc[z] = acc;
    slice_n[z] = cnt;
  }
  int64_t n_valid = 0;
  for (int64_t z = 0; z < nz; ++z) {
    sum_cc += slice_cc[z];
    n_valid += slice_n[z];
  }
  return CCResult{n_valid > 0 ? -sum_cc / (double)n_valid : 0.0, sum_cc};
}

// ------------------------------------------------------------------------------------------
// Gaussian smoothing of a displacement field as SyN configures it (ITK
// SyNImageRegistrationMethod::GaussianSmoothDisplacementField; in-tree twin
// Examples/SmoothDisplacementField.cxx:70-125): per axis a GaussianOperator of the given
// variance (voxel units), max error 0.001, max width = field size along that axis, applied
// x, y, z in T with replicate-edge boundary; then boundary voxels are set to zero and, for
// variance < 0.5, the result is blended with the input (w1 = 1 - variance/0.5).
// variance <= 0 returns a copy.
// ------------------------------------------------------------------------------------------
template <class T>
inline void smooth_field(const T* in, T* out, const Geom& g, double variance) {
  const int64_t N = g.count();
  const int D = g.dim;
  std::memcpy(out, in, sizeof(T) * N * D);
  if (variance <= 0.0) return;
  std::vector<T> tmp(N);
  for (int c = 0; c < D; ++c) {
    T* o = out + c * N;
    for (int axis = 0; axis < D; ++axis) {
      auto k = gaussian_kernel(variance, 0.001, (size_t)g.n[axis]);
      convolve_axis<T, T, T>(o, tmp.data(), g, axis, k);
      std::memcpy(o, tmp.data(), sizeof(T) * N);
    }
  }
  T w1 = (T)1;
  if (variance < 0.5) w1 = (T)1 - (T)1 * ((T)variance / (T)0.5);
  T w2 = (T)1 - w1;
  const int64_t nx = g.n[0], ny = g.n[1], nz = g.n[2];
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; ++i) {
    int64_t x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
    bool edge = x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || (D == 3 && (z == 0 || z == nz - 1));
    for (int c = 0; c < D; ++c) {
      if (edge) out[c * N + i] = (T)0;
      else out[c * N + i] = out[c * N + i] * w1 + in[c * N + i] * w2;
    }
  }
}

// max_x || u(x) / spacing ||  (SyN ScaleUpdateField), then u *= eta / max (if max > 0).
template <class T>
inline double scale_update(T* u, const Geom& g, double eta) {
  const int64_t N = g.count();
  double mx = 0.0;
#pragma omp parallel for reduction(max : mx) schedule(static)
  for (int64_t i = 0; i < N; ++i) {
    T s = 0;
    for (int d = 0; d < g.dim; ++d) {
      T v = u[d * N + i] / (T)g.sp[d];
      s += v * v;
    }
    double nrm = (double)std::sqrt(s);
    if (nrm > mx) mx = nrm;
  }
  T scale = (T)eta;
  if (mx > 0.0) scale = (T)(eta / mx);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)g.dim * N; ++i) u[i] *= scale;
  return mx;
}

// ------------------------------------------------------------------------------------------
// Composition out(x) = w(x) + d(x + w(x)) (ITK ComposeDisplacementFieldsImageFilter with
// displacement field d and warping field w; in-tree twins
// Utilities/itkComposeDiffeomorphismsImageFilter.hxx:70-105, used by SyN each iteration and for
// the final fields, Examples/antsDisplacementAndVelocityFieldRegistrationCommandIterationUpdate.h
// :415-432).  d is interpolated linearly; a point outside d's buffer adds no displacement
// (out = w), which is the ITK filter's rule (the legacy in-tree twin leaves 0 there instead).
// ------------------------------------------------------------------------------------------
template <class T>
inline void compose(const T* d, const T* w, const Geom& g, T* out, T d_scale = (T)1) {
  const int64_t N = g.count(), nx = g.n[0], ny = g.n[1];
  const int D = g.dim;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; ++i) {
    double idx[3] = {(double)(i % nx), (double)((i / nx) % ny), (double)(i / (nx * ny))};
    double p[3];
    g.index_to_point(idx, p);
    double wv[3] = {0, 0, 0};
    for (int c = 0; c < D; ++c) {
      wv[c] = (double)w[c * N + i];
      p[c] += wv[c];
    }
    double c3[3];
    g.point_to_cindex(p, c3);
    if (inside_buffer(g, c3)) {
      LerpCell L;
      lerp_cell(g, c3, L);
      for (int c = 0; c < D; ++c) out[c * N + i] = w[c * N + i] + d_scale * lerp_plane(d + c * N, g, L);
    } else {
      for (int c = 0; c < D; ++c) out[c * N + i] = w[c * N + i];
    }
  }
}

// ------------------------------------------------------------------------------------------
// Fixed-point inverse (ITK InvertDisplacementFieldImageFilter as SyN calls it: at most 20
// iterations, mean tolerance 0.001, max tolerance 0.1, warm start from `psi`, boundary voxels
// pinned to zero).  In-tree twin: ImageRegistration/itkANTSImageRegistrationOptimizer.h
// :1845-1988 (residual by composition :1938, negation :1947, epsilon 0.75 then 0.5 :1964-1968,
// step clamp :1970-1978).  Per iteration: E = psi + phi(x + psi) (compose with d = phi,
// w = psi); norm = ||E/spacing||; mean and max over the grid; step = -E clamped to
// eps*max in norm; psi += eps * step.  Loop runs while it < maxIter && max > maxTol &&
// mean > meanTol, the statistics being those of the previous iteration.
// Returns the number of iterations run.
// ------------------------------------------------------------------------------------------
template <class T>
inline int invert_field(const T* phi, T* psi, const Geom& g, int max_iter = 20, double mean_tol = 0.001,
                        double max_tol = 0.1, double* out_mean = nullptr, double* out_max = nullptr) {
  const int64_t N = g.count(), nx = g.n[0], ny = g.n[1], nz = g.n[2];
  const int D = g.dim;
  std::vector<T> E((size_t)N * D);
  std::vector<T> nrm(N);
  double meanE = DBL_MAX, maxE = DBL_MAX;
  int it = 0;
  std::vector<double> slice_sum(nz);
  while (it++ < max_iter && maxE > max_tol && meanE > mean_tol) {
    compose(phi, psi, g, E.data());
    double mx = 0.0;
#pragma omp parallel for reduction(max : mx) schedule(static)
    for (int64_t z = 0; z < nz; ++z) {
      double acc = 0.0;
      for (int64_t j = 0; j < nx * ny; ++j) {
        int64_t i = z * nx * ny + j;
        T s = 0;
        for (int c = 0; c < D; ++c) {
          T v = E[c * N + i] / (T)g.sp[c];
          s += v * v;
        }
        T n = std::sqrt(s);
        nrm[i] = n;
        acc += (double)n;
        if ((double)n > mx) mx = (double)n;
        for (int c = 0; c < D; ++c) E[c * N + i] = -E[c * N + i];
      }
      slice_sum[z] = acc;
    }
    double sum = 0.0;
    for (int64_t z = 0; z < nz; ++z) sum += slice_sum[z];
    meanE = sum / (double)N;
    maxE = mx;
    T eps = it == 1 ? (T)0.75 : (T)0.5;
    T lim = eps * (T)maxE;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
      int64_t x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
      bool edge = x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || (D == 3 && (z == 0 || z == nz - 1));
      T f = (T)1;
      if (nrm[i] > lim) f = lim / nrm[i];
      for (int c = 0; c < D; ++c) {
        T v = psi[c * N + i] + E[c * N + i] * f * eps;
        psi[c * N + i] = edge ? (T)0 : v;
      }
    }
  }
  if (out_mean) *out_mean = meanE;
  if (out_max) *out_max = maxE;
  return it - 1;
}

// ------------------------------------------------------------------------------------------
// Index map between two grids: voxel index i of `src` lands at continuous index
// c = t + B i of `dst`.  Grids of one registration pyramid share the fixed image's direction
// cosines, and then the map is formed in the grids' common frame: B = diag(sp_src / sp_dst)
// with exact zeros off the diagonal, t = D^-1 (org_src - org_dst) / sp_dst.  Formed through
// the physical frame instead, B picks up ~1e-17 off-diagonal terms from the rotation, and a
// shrink by an even factor puts the finer grid's rim voxels exactly on the coarser grid's
// half-voxel buffer bounds (c = -0.5 and c = n - 0.5, the ShrinkImageFilter centring of
// Examples/itkantsRegistrationHelper.hxx:16-39), where that noise decides inside or outside.
// In the common frame those rim points come out exact for power-of-two shrink factors, so the
// buffer rule (inside at -0.5, outside at n - 0.5) is applied to the exact point.  The same
// t and B, evaluated as ((t + B0 x) + B1 y) + B2 z in double, are what the device library's
// level resampling uses.
// ------------------------------------------------------------------------------------------
inline bool same_direction(const Geom& a, const Geom& b) {
  if (a.dim != b.dim) return false;
  for (int r = 0; r < a.dim; ++r)
    for (int c = 0; c < a.dim; ++c)
      if (a.dir[r * 3 + c] != b.dir[r * 3 + c]) return false;
  return true;
}

inline void index_map(const Geom& src, const Geom& dst, double t[3], double B[9]) {
  const double dorg[3] = {src.org[0] - dst.org[0], src.org[1] - dst.org[1],
                          src.dim == 3 ? src.org[2] - dst.org[2] : 0.0};
  if (same_direction(src, dst)) {
    double D[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, Di[9];
    for (int r = 0; r < src.dim; ++r)
      for (int c = 0; c < src.dim; ++c) D[r * 3 + c] = src.dir[r * 3 + c];
    const double* a = D;
    const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                       a[2] * (a[3] * a[7] - a[4] * a[6]);
    const double id = 1.0 / det;
    Di[0] = (a[4] * a[8] - a[5] * a[7]) * id;
    Di[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    Di[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    Di[3] = (a[5] * a[6] - a[3] * a[8]) * id;
    Di[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    Di[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    Di[6] = (a[3] * a[7] - a[4] * a[6]) * id;
    Di[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    Di[8] = (a[0] * a[4] - a[1] * a[3]) * id;
    for (int r = 0; r < 3; ++r) {
      const bool on = r < src.dim;
      for (int c = 0; c < 3; ++c) B[r * 3 + c] = (r == c && on) ? src.sp[r] / dst.sp[r] : 0.0;
      t[r] = on ? (Di[r * 3 + 0] * dorg[0] + Di[r * 3 + 1] * dorg[1] + Di[r * 3 + 2] * dorg[2]) / dst.sp[r] : 0.0;
    }
    return;
  }
  for (int r = 0; r < 3; ++r) {
    double tt = 0.0;
    for (int c = 0; c < 3; ++c) {
      tt += dst.p2i[r * 3 + c] * dorg[c];
      double b = 0.0;
      for (int k = 0; k < 3; ++k) b += dst.p2i[r * 3 + k] * src.i2p[k * 3 + c];
      B[r * 3 + c] = b;
    }
    t[r] = tt;
  }
  if (src.dim == 2) {
    t[2] = 0.0;
    B[2] = B[5] = B[6] = B[7] = B[8] = 0.0;
  }
}

inline void apply_index_map(const double t[3], const double B[9], const double idx[3], double c[3]) {
  for (int r = 0; r < 3; ++r) {
    double v = t[r] + B[r * 3 + 0] * idx[0];
    v = v + B[r * 3 + 1] * idx[1];
    c[r] = v + B[r * 3 + 2] * idx[2];
  }
}

// Resample a vector field onto another grid (DisplacementFieldTransformParametersAdaptor at
// each level, Examples/itkantsRegistrationHelper.hxx:2028-2055): linear, 0 outside.
template <class T>
inline void resample_field(const T* in, const Geom& gi, T* out, const Geom& go) {
  const int64_t No = go.count(), Ni = gi.count(), nx = go.n[0], ny = go.n[1];
  const int D = go.dim;
  double mt[3], mB[9];
  index_map(go, gi, mt, mB);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < No; ++i) {
    double idx[3] = {(double)(i % nx), (double)((i / nx) % ny), (double)(i / (nx * ny))};
    double c[3];
    apply_index_map(mt, mB, idx, c);
    if (D == 2) c[2] = 0.0;
    if (!inside_buffer(gi, c)) {
      for (int k = 0; k < D; ++k) out[k * No + i] = (T)0;
      continue;
    }
    LerpCell L;
    lerp_cell(gi, c, L);
    for (int k = 0; k < D; ++k) out[k * No + i] = lerp_plane(in + k * Ni, gi, L);
  }
}

// ------------------------------------------------------------------------------------------
// Convergence monitor (ITK WindowConvergenceMonitoringFunction as configured at
// Examples/itkantsRegistrationHelper.hxx:2157-2158; defaults 1e-6 / 10 at
// Examples/antsRegistrationTemplateHeader.h:547-548).  The energies of the last `window`
// iterations, each divided by the running sum of |energy| of the level, are fitted with a
// single-span linear B-spline on [0,1] by one level of multilevel B-spline approximation
// (Lee, Wolberg & Shin 1997); the convergence value is minus the fitted slope at the window's
// end.  Fewer than `window` values gives +inf (no stop).
// ------------------------------------------------------------------------------------------
inline double convergence_value(const std::vector<double>& energies, double total_abs, int window) {
  if ((int)energies.size() < window) return DBL_MAX;
  double num0 = 0, den0 = 0, num1 = 0, den1 = 0;
  size_t b = energies.size() - window;
  for (int k = 0; k < window; ++k) {
    double u = (double)k / (double)(window - 1);
    double z = energies[b + k] / total_abs;
    double w0 = 1.0 - u, w1 = u;
    double ws = w0 * w0 + w1 * w1;
    double phi0 = w0 * z / ws, phi1 = w1 * z / ws;
    num0 += w0 * w0 * phi0;
    den0 += w0 * w0;
    num1 += w1 * w1 * phi1;
    den1 += w1 * w1;
  }
  double c0 = den0 > 0 ? num0 / den0 : 0.0, c1 = den1 > 0 ? num1 / den1 : 0.0;
  return -(c1 - c0);
}

// ------------------------------------------------------------------------------------------
// Full SyN stage (ITK SyNImageRegistrationMethod: level loop, per-iteration update of the
// fixed-to-middle and moving-to-middle fields and their inverses; configured at
// Examples/itkantsRegistrationHelper.hxx:1983-2164, final fields composed as in
// Examples/antsDisplacementAndVelocityFieldRegistrationCommandIterationUpdate.h:415-432).
// ------------------------------------------------------------------------------------------
// ------------------------------------------------------------------------------------------
// Histogram matching (--use-histogram-matching 1): PreprocessImage matches the windowed moving
// image to the preprocessed fixed one with ITK's HistogramMatchingImageFilter, 256 histogram
// levels, 12 match points, threshold at the mean intensity
// (Examples/itkantsRegistrationHelper.hxx:111-122, called at :1135-1143).  The filter's algorithm
// (ITK 5.4.6, Modules/Filtering/ImageIntensity/include/itkHistogramMatchingImageFilter.hxx):
//  * per image: min, max and mean (a double sum in voxel order, the mean cast to the pixel type);
//  * per image: a histogram of `levels` equal bins spanning [min, max] of the voxels in
//    [threshold, max], the threshold being the mean (or the min without thresholding);
//  * a table of match points: row 0 the thresholds, rows 1..points the quantiles j/(points+1)
//    of the two histograms, the last row the maxima; the slope between consecutive points,
//    0 where two source points coincide; below the first point the line through
//    (source min, reference min), above the last the one through the maxima;
//  * each source voxel s mapped through that piecewise-linear function, in double, then cast.
// ------------------------------------------------------------------------------------------
struct HistogramMatchTable {
  int points = 0;                      // match points; the table has points + 2 rows
  std::vector<double> src, ref, grad;  // rows of the table; slopes of the points + 1 segments
  double src_min = 0, src_max = 0, ref_min = 0, ref_max = 0, lower_grad = 0, upper_grad = 0;
};

template <class T>
inline void intensity_stats(const T* x, int64_t n, T& mn, T& mx, T& mean) {
  mn = std::numeric_limits<T>::max();
  mx = std::numeric_limits<T>::lowest();
  double sum = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    sum += (double)x[i];
    if (x[i] < mn) mn = x[i];
    if (x[i] > mx) mx = x[i];
  }
  mean = (T)(sum / (double)n);
}

// Frequencies of the voxels in [vlo, vhi], `levels` equal bins over [lo, hi]; the top value
// falls in the last bin.
template <class T>
inline std::vector<double> thresholded_histogram(const T* x, int64_t n, double lo, double hi, double vlo, double vhi,
                                                 int levels) {
  std::vector<double> freq(levels, 0.0);
  const double bw = (hi - lo) / levels;
  for (int64_t i = 0; i < n; ++i) {
    const double v = (double)x[i];
    if (!(v >= vlo && v <= vhi)) continue;
    int b = bw > 0 ? (int)((v - lo) / bw) : 0;
    b = std::min(std::max(b, 0), levels - 1);
    freq[b] += 1.0;
  }
  return freq;
}

template <class T>
inline HistogramMatchTable histogram_match_table(const T* src, int64_t ns, const T* ref, int64_t nr, int levels,
                                                 int points, bool threshold_at_mean) {
  T smin, smax, smean, rmin, rmax, rmean;
  intensity_stats(src, ns, smin, smax, smean);
  intensity_stats(ref, nr, rmin, rmax, rmean);
  const double sthr = threshold_at_mean ? (double)smean : (double)smin;
  const double rthr = threshold_at_mean ? (double)rmean : (double)rmin;
  const auto hs = thresholded_histogram(src, ns, (double)smin, (double)smax, sthr, (double)smax, levels);
  const auto hr = thresholded_histogram(ref, nr, (double)rmin, (double)rmax, rthr, (double)rmax, levels);
  const double bws = ((double)smax - (double)smin) / levels, bwr = ((double)rmax - (double)rmin) / levels;
  HistogramMatchTable t;
  t.points = points;
  t.src.assign(points + 2, 0.0);
  t.ref.assign(points + 2, 0.0);
  t.src[0] = sthr;
  t.ref[0] = rthr;
  t.src[points + 1] = (double)smax;
  t.ref[points + 1] = (double)rmax;
  const double delta = 1.0 / ((double)points + 1.0);
  for (int j = 1; j <= points; ++j) {
    t.src[j] = histogram_quantile(hs, (double)smin, bws, j * delta);
    t.ref[j] = histogram_quantile(hr, (double)rmin, bwr, j * delta);
  }
  t.grad.assign(points + 1, 0.0);
  for (int j = 0; j <= points; ++j) {
    const double den = t.src[j + 1] - t.src[j];
    t.grad[j] = den != 0.0 ? (t.ref[j + 1] - t.ref[j]) / den : 0.0;
  }
  t.src_min = (double)smin;
  t.src_max = (double)smax;
  t.ref_min = (double)rmin;
  t.ref_max = (double)rmax;
  const double dlo = t.src[0] - t.src_min;
  t.lower_grad = dlo != 0.0 ? (t.ref[0] - t.ref_min) / dlo : 0.0;
  const double dhi = t.src[points + 1] - t.src_max;
  t.upper_grad = dhi != 0.0 ? (t.ref[points + 1] - t.ref_max) / dhi : 0.0;
  return t;
}

// The piecewise-linear map of one source value.
inline double histogram_match_value(const HistogramMatchTable& t, double s) {
  int j = 0;
  while (j < t.points + 2 && !(s < t.src[j])) ++j;
  if (j == 0) return t.ref_min + (s - t.src_min) * t.lower_grad;
  if (j == t.points + 2) return t.ref_max + (s - t.src_max) * t.upper_grad;
  return t.ref[j - 1] + (s - t.src[j - 1]) * t.grad[j - 1];
}

template <class T>
inline void histogram_match(const T* src, int64_t ns, const T* ref, int64_t nr, int levels, int points,
                            bool threshold_at_mean, T* out) {
  const HistogramMatchTable t = histogram_match_table(src, ns, ref, nr, levels, points, threshold_at_mean);
  for (int64_t i = 0; i < ns; ++i) out[i] = (T)histogram_match_value(t, (double)src[i]);
}

struct SynParams {
  double eta = 0.1, var_update = 3.0, var_total = 0.0;
  int radius = 4;
  int n_levels = 1;
  unsigned shrink[8] = {1};
  double sigma[8] = {0};
  int iters[8] = {1};
  bool sigma_mm = false;
  double conv_thresh = 1e-6;
  int conv_window = 10;
  bool preprocess = true;
  float q_lo = 0.0f, q_hi = 1.0f;
  bool histogram_match = false;  // the moving image matched to the fixed one after the window
};

struct SynLog {
  std::vector<int> level, iter, inv_iters;
  std::vector<double> metric, conv;
};

template <class T>
struct SynState {
  Geom g;  // current level grid
  std::vector<T> phiF, psiF, phiM, psiM;
  // metric masks on their own grids (nonzero = inside), or null
  const T* maskF = nullptr;
  const T* maskM = nullptr;
  Geom gmF, gmM;
};

// Validity of the virtual voxels under the metric masks: both masks, warped nearest-neighbour
// through the half-fields (fixed mask at x + psiF(x), moving mask at x + psiM(x)), nonzero.
template <class T>
inline void mask_validity(const SynState<T>& S, std::vector<unsigned char>& valid) {
  const Geom& g = S.g;
  const int64_t N = g.count();
  valid.assign(N, 1);
  std::vector<T> w(N);
  if (S.maskF) {
    warp_image_nearest(S.maskF, S.gmF, S.psiF.data(), g, w.data());
    for (int64_t i = 0; i < N; ++i) valid[i] = valid[i] && w[i] != (T)0;
  }
  if (S.maskM) {
    warp_image_nearest(S.maskM, S.gmM, S.psiM.data(), g, w.data());
    for (int64_t i = 0; i < N; ++i) valid[i] = valid[i] && w[i] != (T)0;
  }
}

template <class T>
inline void syn_iteration(const T* Fs, const Geom& gF, const T* Ms, const Geom& gM, const SynParams& P,
                          SynState<T>& S, double* metric, int* inv_iters, std::vector<T>* scratch_cc = nullptr) {
  const Geom& g = S.g;
  const int64_t N = g.count();
  const int D = g.dim;
  std::vector<T> Ft(N), Mt(N), uF((size_t)N * D), uM((size_t)N * D), sF((size_t)N * D), sM((size_t)N * D);
  warp_image(Fs, gF, S.psiF.data(), g, Ft.data());
  warp_image(Ms, gM, S.psiM.data(), g, Mt.data());
  std::vector<unsigned char> valid;
  if (S.maskF || S.maskM) mask_validity(S, valid);
  CCResult r = cc_metric(Ft.data(), Mt.data(), g, P.radius, uF.data(), uM.data(),
                         scratch_cc ? scratch_cc->data() : nullptr, 1.1920928955078125e-07,
                         valid.empty() ? nullptr : valid.data());
  smooth_field(uF.data(), sF.data(), g, P.var_update);
  smooth_field(uM.data(), sM.data(), g, P.var_update);
  scale_update(sF.data(), g, P.eta);
  scale_update(sM.data(), g, P.eta);
  std::vector<T> tF((size_t)N * D), tM((size_t)N * D);
  compose(sF.data(), S.phiF.data(), g, tF.data());
  compose(sM.data(), S.phiM.data(), g, tM.data());
  if (P.var_total > 0.0) {
    std::vector<T> a((size_t)N * D);
    smooth_field(tF.data(), a.data(), g, P.var_total);
    tF.swap(a);
    smooth_field(tM.data(), a.data(), g, P.var_total);
    tM.swap(a);
  }
  int k = 0;
  k += invert_field(tF.data(), S.psiF.data(), g);  // psiF warm-starts from the previous inverse
  S.phiF = tF;
  k += invert_field(S.psiF.data(), S.phiF.data(), g);  // phiF warm-starts from the composed field
  k += invert_field(tM.data(), S.psiM.data(), g);
  S.phiM = tM;
  k += invert_field(S.psiM.data(), S.phiM.data(), g);
  *metric = r.value;  // both halves evaluate the same symmetric value; SyN reports their mean
  if (inv_iters) *inv_iters = k;
}

// A stage run that can be advanced a bounded number of SyN iterations at a time (the CPU
// baseline splits one complete registration over its timed steps).  Level set-up (image
// smoothing, field resampling) happens when the first iteration of a level is due; the final
// composition when the last level ends.  Running it to the end is syn_register.
template <class T>
struct SynRun {
  SynParams P;
  Geom gF, gM;
  std::vector<T> F, M, Fs, Ms;
  SynState<T> S;
  int level = -1;   // current level (-1: none set up yet)
  int k = 0;        // iterations run in the current level
  bool level_done = true;
  bool done = false;
  std::vector<double> energies;
  double total_abs = 0.0;
  std::vector<T> fwd, inv;
  SynLog log;
  std::vector<int64_t> level_voxels;
  std::vector<double> level_seconds;

  std::vector<T> maskF, maskM;
  // Initial half-fields phiF, psiF, phiM, psiM (component planes on grid gI), or none: a SyN stage
  // initialized from a saved registration state (Examples/itkantsRegistrationHelper.hxx:2093-2125
  // sets the restored FixedToMiddle and MovingToMiddle transforms on the SyN method, whose per-level
  // initialization resamples their fields to each level's domain, the first level's included).
  std::vector<T> init[4];
  Geom gI;
  bool have_init = false;

  void set_initial_half_fields(const T* phiF0, const T* psiF0, const T* phiM0, const T* psiM0, const Geom& g) {
    const T* src[4] = {phiF0, psiF0, phiM0, psiM0};
    const size_t n = (size_t)g.count() * g.dim;
    for (int k = 0; k < 4; ++k) init[k].assign(src[k], src[k] + n);
    gI = g;
    have_init = true;
  }

  // Metric masks (nonzero = inside) on their own grids; null for none.  Call before advancing.
  void set_masks(const T* mF, const Geom* gmF, const T* mM, const Geom* gmM) {
    if (mF && gmF) {
      maskF.assign(mF, mF + gmF->count());
      S.maskF = maskF.data();
      S.gmF = *gmF;
    }
    if (mM && gmM) {
      maskM.assign(mM, mM + gmM->count());
      S.maskM = maskM.data();
      S.gmM = *gmM;
    }
  }

  SynRun(const T* F_in, const Geom& gF_, const T* M_in, const Geom& gM_, const SynParams& P_)
      : P(P_), gF(gF_), gM(gM_) {
    const int64_t NF = gF.count(), NM = gM.count();
    F.resize(NF);
    M.resize(NM);
    if (P.preprocess) {
      preprocess_image(F_in, F.data(), NF, P.q_lo, P.q_hi);
      preprocess_image(M_in, M.data(), NM, P.q_lo, P.q_hi);
    } else {
      std::memcpy(F.data(), F_in, sizeof(T) * NF);
      std::memcpy(M.data(), M_in, sizeof(T) * NM);
    }
    if (P.histogram_match) histogram_match(M.data(), NM, F.data(), NF, 256, 12, true, M.data());
    Fs.resize(NF);
    Ms.resize(NM);
    level_voxels.assign(P.n_levels, 0);
    level_seconds.assign(P.n_levels, 0.0);
  }

  void setup_level(int l) {
    unsigned f[3];
    shrink_factors_per_dim(gF.dim, P.shrink[l], gF.sp, f);
    Geom gl = shrink_geom(gF, f);
    const int64_t N = gl.count();
    const int D = gl.dim;
    smooth_image(F.data(), Fs.data(), gF, P.sigma[l], P.sigma_mm);
    smooth_image(M.data(), Ms.data(), gM, P.sigma[l], P.sigma_mm);
    if (l == 0) {
      S.g = gl;
      std::vector<T>* fl[4] = {&S.phiF, &S.psiF, &S.phiM, &S.psiM};
      for (int q = 0; q < 4; ++q) {
        fl[q]->assign((size_t)N * D, (T)0);
        if (have_init) resample_field(init[q].data(), gI, fl[q]->data(), gl);
      }
    } else {
      std::vector<T>* fl[4] = {&S.phiF, &S.psiF, &S.phiM, &S.psiM};
      for (auto* v : fl) {
        std::vector<T> o((size_t)N * D);
        resample_field(v->data(), S.g, o.data(), gl);
        v->swap(o);
      }
      S.g = gl;
    }
    level = l;
    k = 0;
    level_done = false;
    energies.clear();
    total_abs = 0.0;
  }

  void finish() {
    const int64_t N = S.g.count();
    const int D = S.g.dim;
    fwd.assign((size_t)N * D, (T)0);
    inv.assign((size_t)N * D, (T)0);
    compose(S.psiM.data(), S.phiF.data(), S.g, fwd.data());
    compose(S.psiF.data(), S.phiM.data(), S.g, inv.data());
    done = true;
  }

  // Runs up to n SyN iterations (with the level set-ups they need, and the final composition once
  // the last level ends).  Returns the voxel-iterations run.
  int64_t advance(int64_t n) {
    int64_t vi = 0;
    while (!done && n > 0) {
      if (level_done) {
        if (level + 1 >= P.n_levels) {
          finish();
          break;
        }
        setup_level(level + 1);
        if (P.iters[level] <= 0) {
          level_done = true;
          continue;
        }
      }
      double metric = 0.0;
      int ki = 0;
      const double t0 = omp_seconds();
      syn_iteration(Fs.data(), gF, Ms.data(), gM, P, S, &metric, &ki);
      level_seconds[level] += omp_seconds() - t0;
      ++k;
      --n;
      vi += S.g.count();
      level_voxels[level] += S.g.count();
      energies.push_back(metric);
      total_abs += std::fabs(metric);
      const double cv = convergence_value(energies, total_abs, P.conv_window);
      log.level.push_back(level);
      log.iter.push_back(k);
      log.metric.push_back(metric);
      log.conv.push_back(cv);
      log.inv_iters.push_back(ki);
      if (cv < P.conv_thresh || k >= P.iters[level]) level_done = true;
    }
    if (!done && level_done && level + 1 >= P.n_levels) finish();
    return vi;
  }
};

// Initial half-fields of a stage (component planes on grid g), or all null.
template <class T>
struct SynInit {
  const T* f[4] = {nullptr, nullptr, nullptr, nullptr};  // phiF, psiF, phiM, psiM
  Geom g;
};

template <class T>
inline void syn_register(const T* F_in, const Geom& gF, const T* M_in, const Geom& gM, const SynParams& P,
                         std::vector<T>& fwd, std::vector<T>& inv, Geom& gOut, SynLog* log = nullptr,
                         const T* maskF = nullptr, const Geom* gmF = nullptr, const T* maskM = nullptr,
                         const Geom* gmM = nullptr, const SynInit<T>* init = nullptr,
                         std::vector<T>* half_out = nullptr) {
  SynRun<T> R(F_in, gF, M_in, gM, P);
  R.set_masks(maskF, gmF, maskM, gmM);
  if (init && init->f[0]) R.set_initial_half_fields(init->f[0], init->f[1], init->f[2], init->f[3], init->g);
  while (!R.done) R.advance(INT64_MAX);
  fwd.swap(R.fwd);
  inv.swap(R.inv);
  gOut = R.S.g;
  if (log) *log = R.log;
  if (half_out) {  // the final half-fields phiF, psiF, phiM, psiM, one after the other
    half_out->clear();
    for (const std::vector<T>* v : {&R.S.phiF, &R.S.psiF, &R.S.phiM, &R.S.psiM})
      half_out->insert(half_out->end(), v->begin(), v->end());
  }
}

}  // namespace synx_oracle
