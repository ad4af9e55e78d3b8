// Test infrastructure: the C ABI step functions the command lines call (warps, compose, resample),
// routed to the CPU oracle on host memory, so that the command lines' own logic (option parsing,
// transform chains, geometry folding, output files) can be tested without a GPU.  The product's
// step functions are the CUDA kernels in libsynx.so; this file is never linked into it.
#include <string>
#include "synx.h"
#include "synx_host.h"
extern "C" {
void oracle_warp_image_f32(const float*, const synx_geom*, const float*, const synx_geom*, float*);
void oracle_warp_image_nearest_f32(const float*, const synx_geom*, const float*, const synx_geom*, float*);
void oracle_warp_image_label_f32(const float*, const synx_geom*, const float*, const synx_geom*, float*);
void oracle_compose_f32(const float*, const float*, const synx_geom*, float*, double);
void oracle_resample_field_f32(const float*, const synx_geom*, float*, const synx_geom*);
}
static thread_local std::string g_err;
int synx::set_global_error(int code, const std::string& m) { g_err = m; return code; }
extern "C" {
const char* synx_last_error(const synx_ctx*) { return g_err.c_str(); }
int synx_warp_image(const float* img, const synx_geom* gi, const float* u, const synx_geom* gv, float* out, void*) {
  oracle_warp_image_f32(img, gi, u, gv, out); return 0; }
int synx_warp_image_nearest(const float* img, const synx_geom* gi, const float* u, const synx_geom* gv, float* out,
                            void*) {
  oracle_warp_image_nearest_f32(img, gi, u, gv, out); return 0; }
int synx_warp_image_label(const float* img, const synx_geom* gi, const float* u, const synx_geom* gv, float* out,
                          void*) {
  oracle_warp_image_label_f32(img, gi, u, gv, out); return 0; }
int synx_field_affine_update(const float* u, const float* w, const synx_geom* g, const double* M, float* out,
                             void*) {
  const long long N = g->size[0] * g->size[1] * g->size[2];
  const int D = g->dim;
  for (long long i = 0; i < N; ++i) {
    double wv[3] = {0, 0, 0}, uv[3] = {0, 0, 0};
    for (int c = 0; c < D; ++c) { wv[c] = w[c * N + i]; uv[c] = u[c * N + i]; }
    for (int r = 0; r < D; ++r) {
      double s = uv[r];
      for (int k = 0; k < D; ++k) s += M[r * 3 + k] * wv[k];
      out[r * N + i] = (float)s;
    }
  }
  return 0;
}
int synx_compose(const float* d, const float* w, const synx_geom* g, float s, float* out, void*) {
  oracle_compose_f32(d, w, g, out, s); return 0; }
int synx_resample_field(const float* in, const synx_geom* gi, float* out, const synx_geom* go, void*) {
  oracle_resample_field_f32(in, gi, out, go); return 0; }
}
