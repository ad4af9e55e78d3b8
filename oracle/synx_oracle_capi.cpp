// extern "C" wrappers around the CPU oracle (synx_oracle.hpp) for the Python test harness.
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg as the checker; never by the product path.  Parity unpinned (see header).
#include "synx_oracle.hpp"

#include "../include/synx.h"

using namespace synx_oracle;

static Geom to_geom(const synx_geom* s) {
  Geom g;
  g.dim = s->dim;
  for (int d = 0; d < 3; ++d) {
    g.n[d] = s->size[d];
    g.sp[d] = s->spacing[d];
    g.org[d] = s->origin[d];
  }
  for (int k = 0; k < 9; ++k) g.dir[k] = s->direction[k];
  if (g.dim == 2) g.n[2] = 1;
  g.finalize();
  return g;
}

static void from_geom(const Geom& g, synx_geom* s) {
  s->dim = g.dim;
  s->reserved0 = 0;
  for (int d = 0; d < 3; ++d) {
    s->size[d] = g.n[d];
    s->spacing[d] = g.sp[d];
    s->origin[d] = g.org[d];
  }
  for (int k = 0; k < 9; ++k) s->direction[k] = g.dir[k];
}

static SynParams to_params(const synx_params* p) {
  SynParams P;
  P.eta = p->learning_rate;
  P.var_update = p->update_variance;
  P.var_total = p->total_variance;
  P.radius = p->cc_radius;
  P.n_levels = p->n_levels;
  for (int l = 0; l < p->n_levels && l < 8; ++l) {
    P.shrink[l] = (unsigned)p->shrink_factors[l];
    P.sigma[l] = p->smoothing_sigmas[l];
    P.iters[l] = p->iterations[l];
  }
  P.sigma_mm = p->sigmas_in_mm != 0;
  P.conv_thresh = p->convergence_threshold;
  P.conv_window = p->convergence_window;
  P.preprocess = p->preprocess != 0;
  P.q_lo = p->winsor_lower;
  P.q_hi = p->winsor_upper;
  P.histogram_match = p->histogram_match != 0;
  return P;
}

extern "C" {

int oracle_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int oracle_gaussian_kernel(double variance, double max_error, int max_width, double* out, int cap) {
  auto k = gaussian_kernel(variance, max_error, (size_t)max_width);
  for (int i = 0; i < (int)k.size() && i < cap; ++i) out[i] = k[i];
  return (int)k.size();
}

void oracle_shrink_geom(const synx_geom* in, unsigned factor, synx_geom* out) {
  Geom g = to_geom(in);
  unsigned f[3];
  shrink_factors_per_dim(g.dim, factor, g.sp, f);
  from_geom(shrink_geom(g, f), out);
}

#define ORACLE_TYPED(SUF, T)                                                                         \
  void oracle_preprocess_##SUF(const T* in, T* out, int64_t n, float qlo, float qhi) {               \
    preprocess_image(in, out, n, qlo, qhi);                                                          \
  }                                                                                                  \
  void oracle_histogram_match_##SUF(const T* src, int64_t ns, const T* ref, int64_t nr, int levels,    \
                                    int points, int thr_mean, T* out) {                              \
    histogram_match(src, ns, ref, nr, levels, points, thr_mean != 0, out);                           \
  }                                                                                                  \
  /* table rows src[points+2], ref[points+2], slopes grad[points+1]; ends: src min, src max, */       \
  /* ref min, ref max, lower slope, upper slope */                                                   \
  void oracle_histogram_match_table_##SUF(const T* src, int64_t ns, const T* ref, int64_t nr,         \
                                          int levels, int points, int thr_mean, double* tsrc,        \
                                          double* tref, double* grad, double* ends) {                \
    HistogramMatchTable t = histogram_match_table(src, ns, ref, nr, levels, points, thr_mean != 0);   \
    for (int j = 0; j < points + 2; ++j) tsrc[j] = t.src[j], tref[j] = t.ref[j];                     \
    for (int j = 0; j < points + 1; ++j) grad[j] = t.grad[j];                                        \
    const double e[6] = {t.src_min, t.src_max, t.ref_min, t.ref_max, t.lower_grad, t.upper_grad};    \
    for (int k = 0; k < 6; ++k) ends[k] = e[k];                                                      \
  }                                                                                                  \
  void oracle_smooth_image_##SUF(const T* in, T* out, const synx_geom* g, double sigma, int mm) {    \
    smooth_image(in, out, to_geom(g), sigma, mm != 0);                                               \
  }                                                                                                  \
  void oracle_warp_image_##SUF(const T* img, const synx_geom* gi, const T* u, const synx_geom* gv,   \
                               T* out) {                                                             \
    warp_image(img, to_geom(gi), u, to_geom(gv), out);                                               \
  }                                                                                                  \
  void oracle_warp_image_nearest_##SUF(const T* img, const synx_geom* gi, const T* u, const synx_geom* gv,   \
                               T* out) {                                                             \
    warp_image_nearest(img, to_geom(gi), u, to_geom(gv), out);                                               \
  }                                                                                                  \
  void oracle_warp_image_label_##SUF(const T* img, const synx_geom* gi, const T* u, const synx_geom* gv,   \
                               T* out) {                                                             \
    warp_image_label(img, to_geom(gi), u, to_geom(gv), out);                                               \
  }                                                                                                  \
  double oracle_cc_##SUF(const T* F, const T* M, const synx_geom* g, int r, T* gF, T* gM, T* cc) {   \
    return cc_metric(F, M, to_geom(g), r, gF, gM, cc).value;                                         \
  }                                                                                                  \
  /* CC over the valid voxels only (valid: one byte per voxel, nonzero = valid). */                  \
  double oracle_cc_masked_##SUF(const T* F, const T* M, const synx_geom* g, int r,                   \
                                const unsigned char* valid, T* gF, T* gM, T* cc) {                   \
    return cc_metric(F, M, to_geom(g), r, gF, gM, cc, 1.1920928955078125e-07, valid).value;          \
  }                                                                                                  \
  void oracle_smooth_field_##SUF(const T* in, T* out, const synx_geom* g, double var) {              \
    smooth_field(in, out, to_geom(g), var);                                                          \
  }                                                                                                  \
  double oracle_scale_update_##SUF(T* u, const synx_geom* g, double eta) {                           \
    return scale_update(u, to_geom(g), eta);                                                         \
  }                                                                                                  \
  void oracle_compose_##SUF(const T* d, const T* w, const synx_geom* g, T* out, double s) {          \
    compose(d, w, to_geom(g), out, (T)s);                                                            \
  }                                                                                                  \
  int oracle_invert_##SUF(const T* phi, T* psi, const synx_geom* g, int maxit, double mt, double xt, \
                          double* mean, double* mx) {                                                \
    return invert_field(phi, psi, to_geom(g), maxit, mt, xt, mean, mx);                              \
  }                                                                                                  \
  void oracle_resample_field_##SUF(const T* in, const synx_geom* gi, T* out, const synx_geom* go) {  \
    resample_field(in, to_geom(gi), out, to_geom(go));                                               \
  }                                                                                                  \
  /* One SyN iteration on the four half-fields in place (grid g), images already smoothed. */       \
  double oracle_syn_iteration_##SUF(const T* Fs, const synx_geom* gF, const T* Ms, const synx_geom* gM, \
                                    const synx_params* p, const synx_geom* g, T* phiF, T* psiF,      \
                                    T* phiM, T* psiM, int* inv_iters) {                              \
    SynParams P = to_params(p);                                                                      \
    SynState<T> S;                                                                                   \
    S.g = to_geom(g);                                                                                \
    const size_t n = (size_t)S.g.count() * S.g.dim;                                                  \
    S.phiF.assign(phiF, phiF + n);                                                                   \
    S.psiF.assign(psiF, psiF + n);                                                                   \
    S.phiM.assign(phiM, phiM + n);                                                                   \
    S.psiM.assign(psiM, psiM + n);                                                                   \
    double metric = 0.0;                                                                             \
    syn_iteration(Fs, to_geom(gF), Ms, to_geom(gM), P, S, &metric, inv_iters);                       \
    std::copy(S.phiF.begin(), S.phiF.end(), phiF);                                                   \
    std::copy(S.psiF.begin(), S.psiF.end(), psiF);                                                   \
    std::copy(S.phiM.begin(), S.phiM.end(), phiM);                                                   \
    std::copy(S.psiM.begin(), S.psiM.end(), psiM);                                                   \
    return metric;                                                                                   \
  }                                                                                                  \
  /* Full stage.  fwd/inv must hold the last level grid (query it with oracle_shrink_geom);       \
     log arrays hold log_cap records; returns the number of records. */                             \
  int oracle_syn_register_masked_##SUF(const T* F, const synx_geom* gF, const T* M, const synx_geom* gM, \
                                       const synx_params* p, const T* maskF, const synx_geom* gmF,   \
                                       const T* maskM, const synx_geom* gmM, T* fwd, T* inv,         \
                                       synx_geom* gout, int32_t* log_level, int32_t* log_iter,       \
                                       double* log_metric, double* log_conv, int32_t* log_inv,       \
                                       int log_cap);                                                 \
  int oracle_syn_register_full_##SUF(const T* F, const synx_geom* gF, const T* M, const synx_geom* gM, \
                                     const synx_params* p, const T* maskF, const synx_geom* gmF,     \
                                     const T* maskM, const synx_geom* gmM, const T* iphiF,           \
                                     const T* ipsiF, const T* iphiM, const T* ipsiM,                 \
                                     const synx_geom* gI, T* fwd, T* inv, T* half, synx_geom* gout,  \
                                     int32_t* log_level, int32_t* log_iter, double* log_metric,      \
                                     double* log_conv, int32_t* log_inv, int log_cap);               \
  int oracle_syn_register_##SUF(const T* F, const synx_geom* gF, const T* M, const synx_geom* gM,    \
                                const synx_params* p, T* fwd, T* inv, synx_geom* gout,               \
                                int32_t* log_level, int32_t* log_iter, double* log_metric,           \
                                double* log_conv, int32_t* log_inv, int log_cap) {                   \
    return oracle_syn_register_masked_##SUF(F, gF, M, gM, p, nullptr, nullptr, nullptr, nullptr, fwd,   \
                                            inv, gout, log_level, log_iter, log_metric, log_conv,    \
                                            log_inv, log_cap);                                       \
  }                                                                                                  \
  /* The same with metric masks (null for none), each on its own grid. */                           \
  int oracle_syn_register_masked_##SUF(const T* F, const synx_geom* gF, const T* M, const synx_geom* gM, \
                                       const synx_params* p, const T* maskF, const synx_geom* gmF,   \
                                       const T* maskM, const synx_geom* gmM, T* fwd, T* inv,         \
                                       synx_geom* gout, int32_t* log_level, int32_t* log_iter,       \
                                       double* log_metric, double* log_conv, int32_t* log_inv,       \
                                       int log_cap) {                                                \
    return oracle_syn_register_full_##SUF(F, gF, M, gM, p, maskF, gmF, maskM, gmM, nullptr, nullptr, \
                                          nullptr, nullptr, nullptr, fwd, inv, nullptr, gout,        \
                                          log_level, log_iter, log_metric, log_conv, log_inv, log_cap); \
  }                                                                                                  \
  /* The same, also with initial half-fields phiF, psiF, phiM, psiM (component planes on grid gI; \
     null for none) and the final half-fields written one after the other to `half` (4 x D x N of  \
     the last level grid; null: not wanted). */                                                      \
  int oracle_syn_register_full_##SUF(const T* F, const synx_geom* gF, const T* M, const synx_geom* gM, \
                                     const synx_params* p, const T* maskF, const synx_geom* gmF,     \
                                     const T* maskM, const synx_geom* gmM, const T* iphiF,           \
                                     const T* ipsiF, const T* iphiM, const T* ipsiM,                 \
                                     const synx_geom* gI, T* fwd, T* inv, T* half, synx_geom* gout,  \
                                     int32_t* log_level, int32_t* log_iter, double* log_metric,      \
                                     double* log_conv, int32_t* log_inv, int log_cap) {              \
    SynParams P = to_params(p);                                                                      \
    std::vector<T> f, v, hv;                                                                         \
    Geom go;                                                                                         \
    SynLog L;                                                                                        \
    Geom a, b;                                                                                       \
    if (gmF) a = to_geom(gmF);                                                                       \
    if (gmM) b = to_geom(gmM);                                                                       \
    SynInit<T> init;                                                                                 \
    if (iphiF && ipsiF && iphiM && ipsiM && gI) {                                                    \
      init.f[0] = iphiF;                                                                             \
      init.f[1] = ipsiF;                                                                             \
      init.f[2] = iphiM;                                                                             \
      init.f[3] = ipsiM;                                                                             \
      init.g = to_geom(gI);                                                                          \
    }                                                                                                \
    syn_register(F, to_geom(gF), M, to_geom(gM), P, f, v, go, &L, maskF, gmF ? &a : nullptr, maskM,  \
                 gmM ? &b : nullptr, &init, half ? &hv : nullptr);                                   \
    std::copy(f.begin(), f.end(), fwd);                                                              \
    std::copy(v.begin(), v.end(), inv);                                                              \
    if (half) std::copy(hv.begin(), hv.end(), half);                                                 \
    from_geom(go, gout);                                                                             \
    int nrec = (int)L.metric.size();                                                                 \
    for (int i = 0; i < nrec && i < log_cap; ++i) {                                                  \
      if (log_level) log_level[i] = L.level[i];                                                      \
      if (log_iter) log_iter[i] = L.iter[i];                                                         \
      if (log_metric) log_metric[i] = L.metric[i];                                                   \
      if (log_conv) log_conv[i] = L.conv[i];                                                         \
      if (log_inv) log_inv[i] = L.inv_iters[i];                                                      \
    }                                                                                                \
    return nrec;                                                                                     \
  }

ORACLE_TYPED(f32, float)
ORACLE_TYPED(f64, double)

/* A float stage run advanced in bounded pieces (the CPU baseline's timed steps).  advance returns
   the voxel-iterations it ran; the run is done once the final composition has been made. */
void* oracle_run_create_f32(const float* F, const synx_geom* gF, const float* M, const synx_geom* gM,
                            const synx_params* p) {
  return new SynRun<float>(F, to_geom(gF), M, to_geom(gM), to_params(p));
}
int64_t oracle_run_advance_f32(void* h, int64_t n) { return static_cast<SynRun<float>*>(h)->advance(n); }
int oracle_run_done_f32(void* h) { return static_cast<SynRun<float>*>(h)->done ? 1 : 0; }
/* Per level: voxel-iterations run and seconds spent in its iterations; returns the record count. */
int oracle_run_levels_f32(void* h, int64_t* voxel_iters, double* seconds, int32_t* iterations, int cap) {
  auto* R = static_cast<SynRun<float>*>(h);
  const int L = R->P.n_levels;
  for (int l = 0; l < L && l < cap; ++l) {
    voxel_iters[l] = R->level_voxels[l];
    seconds[l] = R->level_seconds[l];
    int n = 0;
    for (int v : R->log.level) n += v == l;
    iterations[l] = n;
  }
  return L;
}
void oracle_run_destroy_f32(void* h) { delete static_cast<SynRun<float>*>(h); }

}  // extern "C"
