// Test infrastructure: the stage and batch entry points the registration command line and the
// serving loop call, backed by the CPU oracle's whole registration (run when a stage reaches its
// last level), so that their plumbing (initial transforms, output names, written transforms, warped
// images; admission, pooling and request lifecycle) can be tested without a GPU.  The footprint is
// a stand-in that grows with both images.  Never part of the product.
#include <cstring>
#include <string>
#include <vector>
#include "synx.h"
extern "C" int oracle_syn_register_full_f32(const float*, const synx_geom*, const float*, const synx_geom*,
                                            const synx_params*, const float*, const synx_geom*, const float*,
                                            const synx_geom*, const float*, const float*, const float*, const float*,
                                            const synx_geom*, float*, float*, float*, synx_geom*, int32_t*, int32_t*,
                                            double*, double*, int32_t*, int);
extern "C" void oracle_shrink_geom(const synx_geom*, unsigned, synx_geom*);
struct synx_ctx {
  synx_params p;
  std::vector<float> F, M, fwd, inv;
  synx_geom gf, gm, go;
  std::vector<float> mF, mM;  // metric masks (empty: none)
  synx_geom gmF, gmM;
  std::vector<float> init[4];  // initial half-fields, component planes (empty: none)
  synx_geom gI;
  std::vector<float> half;     // final half-fields, component planes one after the other
  std::vector<int32_t> lv, it, ki;
  std::vector<double> me, cv;
  bool done = false;
  int level = 0;  // next level a batch step runs
};
struct synx_batch {
  int device;
};
static int g_created = 0;  // contexts created, so a test can see pooled contexts being reused
extern "C" {
int synx_params_default(synx_params* p, int dim) {
  memset(p, 0, sizeof(*p));
  p->dim = dim; p->n_levels = 1; p->learning_rate = 0.1; p->update_variance = 3.0; p->cc_radius = 4;
  p->iterations[0] = 1; p->shrink_factors[0] = 1; p->convergence_threshold = 1e-6; p->convergence_window = 10;
  p->preprocess = 1; p->winsor_upper = 1.0f; p->inv_max_iter = 20; p->inv_mean_tol = 0.001; p->inv_max_tol = 0.1;
  return 0;
}
int synx_create(const synx_params* p, int, void*, synx_ctx** out) {
  *out = new synx_ctx;
  (*out)->p = *p;
  ++g_created;
  return 0;
}
int host_stage_created() { return g_created; }
int synx_destroy(synx_ctx* c) { delete c; return 0; }
int synx_set_images(synx_ctx* c, const float* F, const synx_geom* gf, const float* M, const synx_geom* gm) {
  c->gf = *gf; c->gm = *gm;
  c->F.assign(F, F + gf->size[0] * gf->size[1] * gf->size[2]);
  c->M.assign(M, M + gm->size[0] * gm->size[1] * gm->size[2]);
  c->done = false;
  c->level = 0;
  return 0;
}
int synx_set_masks(synx_ctx* c, const float* mf, const synx_geom* gmf, const float* mm, const synx_geom* gmm) {
  c->mF.clear();
  c->mM.clear();
  if (mf) { c->gmF = *gmf; c->mF.assign(mf, mf + gmf->size[0] * gmf->size[1] * gmf->size[2]); }
  if (mm) { c->gmM = *gmm; c->mM.assign(mm, mm + gmm->size[0] * gmm->size[1] * gmm->size[2]); }
  return 0;
}
int synx_set_initial_half_fields(synx_ctx* c, const float* a, const float* b, const float* d, const float* e,
                                 const synx_geom* g) {
  for (auto& v : c->init) v.clear();
  if (!a) return 0;
  c->gI = *g;
  const size_t N = g->size[0] * g->size[1] * g->size[2], D = g->dim;
  const float* src[4] = {a, b, d, e};
  for (int k = 0; k < 4; ++k) {
    c->init[k].resize(N * D);
    for (size_t i = 0; i < N; ++i)
      for (size_t q = 0; q < D; ++q) c->init[k][q * N + i] = src[k][i * D + q];
  }
  return 0;
}
int synx_run_level(synx_ctx* c, int level) {
  if (c->done || level != c->p.n_levels - 1) return 0;  // the whole stage runs at the last level
  synx_geom go;
  oracle_shrink_geom(&c->gf, c->p.shrink_factors[c->p.n_levels - 1], &go);
  const size_t N = go.size[0] * go.size[1] * go.size[2], D = c->p.dim;
  std::vector<float> f(N * D), v(N * D);
  const int cap = 100000;
  c->lv.resize(cap); c->it.resize(cap); c->ki.resize(cap); c->me.resize(cap); c->cv.resize(cap);
  const bool ini = !c->init[0].empty();
  c->half.resize(4 * N * D);
  int n = oracle_syn_register_full_f32(c->F.data(), &c->gf, c->M.data(), &c->gm, &c->p,
                                       c->mF.empty() ? nullptr : c->mF.data(), c->mF.empty() ? nullptr : &c->gmF,
                                       c->mM.empty() ? nullptr : c->mM.data(), c->mM.empty() ? nullptr : &c->gmM,
                                       ini ? c->init[0].data() : nullptr, ini ? c->init[1].data() : nullptr,
                                       ini ? c->init[2].data() : nullptr, ini ? c->init[3].data() : nullptr,
                                       ini ? &c->gI : nullptr, f.data(), v.data(), c->half.data(), &c->go,
                                       c->lv.data(), c->it.data(), c->me.data(), c->cv.data(), c->ki.data(), cap);
  for (auto* a : {&c->lv, &c->it, &c->ki}) a->resize(n);
  c->me.resize(n); c->cv.resize(n);
  c->fwd.resize(N * D); c->inv.resize(N * D);
  for (size_t i = 0; i < N; ++i)
    for (size_t k = 0; k < D; ++k) { c->fwd[i * D + k] = f[k * N + i]; c->inv[i * D + k] = v[k * N + i]; }
  c->done = true;
  return 0;
}
int synx_get_output_geom(const synx_ctx* c, synx_geom* g) { *g = c->go; return 0; }
int synx_get_half_fields(synx_ctx* c, float* a, float* b, float* d, float* e) {
  const size_t N = c->go.size[0] * c->go.size[1] * c->go.size[2], D = c->p.dim;
  float* dst[4] = {a, b, d, e};
  for (int k = 0; k < 4; ++k)
    if (dst[k])
      for (size_t i = 0; i < N; ++i)
        for (size_t q = 0; q < D; ++q) dst[k][i * D + q] = c->half[(k * D + q) * N + i];
  return 0;
}
int synx_get_fields(synx_ctx* c, float* fw, float* iv) {
  std::memcpy(fw, c->fwd.data(), 4 * c->fwd.size()); std::memcpy(iv, c->inv.data(), 4 * c->inv.size()); return 0; }
int synx_get_log(synx_ctx* c, int32_t* level, int32_t* iter, double* metric, double* conv, int32_t* inv, int64_t cap, int64_t* count) {
  *count = (int64_t)c->me.size();
  for (int64_t i = 0; i < cap && i < *count; ++i) {
    if (level) level[i] = c->lv[i]; if (iter) iter[i] = c->it[i]; if (metric) metric[i] = c->me[i];
    if (conv) conv[i] = c->cv[i]; if (inv) inv[i] = c->ki[i];
  }
  return 0;
}
}

extern "C" {
int synx_batch_create(int device, synx_batch** out) { *out = new synx_batch{device}; return 0; }
int synx_batch_destroy(synx_batch* b) { delete b; return 0; }
const char* synx_batch_last_error(const synx_batch*) { return ""; }
int synx_batch_step(synx_batch*, synx_ctx* const* cs, int n, void*, int* advanced) {
  int a = 0;
  for (int i = 0; i < n; ++i) {
    synx_ctx* c = cs[i];
    if (c->level >= c->p.n_levels) continue;
    synx_run_level(c, c->level);
    ++c->level;
    ++a;
  }
  if (advanced) *advanced = a;
  return 0;
}
int synx_footprint(const synx_params* p, const synx_geom* gf, const synx_geom* gm, int64_t* bytes) {
  const int64_t nf = gf->size[0] * gf->size[1] * gf->size[2], nm = gm->size[0] * gm->size[1] * gm->size[2];
  *bytes = 4 * (nf + nm) + 40 * nf * p->dim;
  return 0;
}
}
