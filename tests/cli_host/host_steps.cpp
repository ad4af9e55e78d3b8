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
int synx_compose(const float* d, const float* w, const synx_geom* g, float s, float* out, void*) {
  oracle_compose_f32(d, w, g, out, s); return 0; }
int synx_resample_field(const float* in, const synx_geom* gi, float* out, const synx_geom* go, void*) {
  oracle_resample_field_f32(in, gi, out, go); return 0; }
}
