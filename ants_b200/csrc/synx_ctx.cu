// synx C ABI: registration context, level loop and step entry points.
//
// One context = one fixed/moving pair on one GPU.  All pair state (images, the pyramid
// level images, the four half-fields and the iteration work buffers) lives in one device
// arena allocated at synx_set_images; a level is enqueued without host synchronisation (the
// convergence test and the fixed-point loop bounds are evaluated on the device), and is
// optionally captured once as a CUDA graph and replayed per iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "../../include/synx.h"
#include "synx_host.h"
#include "synx_nvtx.h"
#include "synx_kernels.cuh"
#include "synx_level.cuh"

using namespace synx;

namespace {

thread_local std::string g_last_error;

// ---- discrete Gaussian kernel --------------------------------------------------------------
// Lindeberg's discrete Gaussian k(n) = e^{-t} I_n(t) with I_0, I_1 from the polynomial
// approximations of Abramowitz & Stegun (9.8.1-9.8.4) and the recurrence
// I_n = I_{n-2} - 2 (n-1) I_{n-1} / t, grown until the two-sided mass reaches 1 - max_error
// or the half-kernel exceeds max_width, then normalised and mirrored (the construction of
// ITK's GaussianOperator that SyN's field smoothing and the level pyramid use).
double as_i0(double y) {
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
double as_i1(double y) {
  double ay = std::fabs(y), r;
  if (ay < 3.75) {
    double t = (y / 3.75) * (y / 3.75);
    r = ay * (0.5 + t * (0.87890594 + t * (0.51498869 + t * (0.15084934 + t * (0.02658733 + t * (0.00301532 + t * 0.00032411))))));
  } else {
    double t = 3.75 / ay;
    r = 0.02282967 + t * (-0.02895312 + t * (0.01787654 - t * 0.00420059));
    r = 0.39894228 + t * (-0.03988024 + t * (-0.00362018 + t * (0.00163801 + t * (-0.01031555 + t * r))));
    r *= std::exp(ay) / std::sqrt(ay);
  }
  return y < 0 ? -r : r;
}
std::vector<double> gauss_kernel(double variance, double max_error, size_t max_width) {
  std::vector<double> h;
  const double et = std::exp(-variance), cap = 1.0 - max_error;
  double sum = 0.0;
  h.push_back(et * as_i0(variance));
  sum += h[0];
  h.push_back(et * as_i1(variance));
  sum += 2.0 * h[1];
  for (int i = 2; sum < cap; ++i) {
    h.push_back(h[i - 2] - 2.0 * (i - 1) * h[i - 1] / variance);
    sum += 2.0 * h[i];
    if (h[i] <= 0.0) break;
    if (h.size() > max_width) break;
  }
  for (double& c : h) c /= sum;
  const size_t R = h.size() - 1;
  std::vector<double> k(2 * R + 1);
  for (size_t i = 0; i <= R; ++i) k[R + i] = k[R - i] = h[i];
  return k;
}

// ---- level geometry (CalculateShrinkFactorsPerDimension + ShrinkImageFilter) ----------------
void shrink_factors(int dim, unsigned factor, const double sp[3], unsigned out[3]) {
  double minSp = sp[0];
  int minIdx = 0;
  for (int n = 1; n < dim; ++n)
    if (minSp > sp[n]) {
      minSp = sp[n];
      minIdx = n;
    }
  out[0] = out[1] = out[2] = 0;
  out[minIdx] = factor;
  const double target = sp[minIdx] * factor;
  for (int n = 0; n < dim; ++n) {
    if (out[n]) continue;
    double best = std::fabs(sp[n] * factor - target);
    unsigned bf = factor;
    for (unsigned f = factor - 1; f > 0; --f) {
      double dd = std::fabs(sp[n] * f - target);
      if (dd <= best) {
        best = dd;
        bf = f;
      }
    }
    out[n] = bf;
  }
  if (dim == 2) out[2] = 1;
}

void geom_to_grid(const synx_geom& g, GridInfo& gi) {
  gi = make_grid(g.dim, g.size, g.spacing, g.origin, g.direction);
}

synx_geom shrink(const synx_geom& in, unsigned factor) {
  unsigned f[3];
  shrink_factors(in.dim, factor, in.spacing, f);
  synx_geom out = in;
  for (int d = 0; d < in.dim; ++d) {
    out.spacing[d] = in.spacing[d] * f[d];
    int64_t s = (int64_t)std::floor((double)in.size[d] / (double)f[d]);
    out.size[d] = s < 1 ? 1 : s;
  }
  if (in.dim == 2) out.size[2] = 1;
  GridInfo gin, gout;
  geom_to_grid(in, gin);
  geom_to_grid(out, gout);
  double ci[3] = {0, 0, 0}, co[3] = {0, 0, 0};
  for (int d = 0; d < in.dim; ++d) {
    ci[d] = (in.size[d] - 1) / 2.0;
    co[d] = (out.size[d] - 1) / 2.0;
  }
  for (int r = 0; r < 3; ++r) {
    double pin = gin.org[r], pout = gout.org[r];
    for (int c = 0; c < 3; ++c) {
      pin += gin.i2p[r * 3 + c] * ci[c];
      pout += gout.i2p[r * 3 + c] * co[c];
    }
    out.origin[r] = in.origin[r] + (pin - pout);
  }
  if (in.dim == 2) out.origin[2] = in.origin[2];
  return out;
}

bool check_geom(const synx_geom* g, int dim) {
  if (!g || g->dim != dim) return false;
  for (int d = 0; d < dim; ++d)
    if (g->size[d] < 1 || !(g->spacing[d] > 0)) return false;
  if (dim == 2 && g->size[2] != 1) return false;
  long long n = (long long)g->size[0] * g->size[1] * g->size[2];
  if (n * 3 >= (1LL << 31)) return false;
  return true;
}

int set_err(synx_ctx* c, int code, const std::string& msg);

struct LevelProf {
  double setup_ms = 0, iterate_ms = 0, inv_ms = 0, cc_ms = 0;
  long long iterations = 0, inv_sub = 0, voxels = 0;
};

}  // namespace

struct synx_ctx {
  synx_params P;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaStream_t aux = nullptr;        // captures the inverse loop bodies of the level graphs
  bool loop_graphs_failed = false;   // the driver refused conditional nodes: graphs use plain launches
  bool pdl_failed = false;           // the driver refused programmatic edges in a captured graph
  std::string err;
  bool images_set = false;
  synx_geom geF{}, geM{};
  GridInfo gF{}, gM{};
  std::vector<synx_geom> lgeom;
  std::vector<GridInfo> lv;
  long long Nmax = 0, NF = 0, NM = 0;
  int D = 3;
  // arena
  char* arena = nullptr;
  size_t arena_bytes = 0;
  float *F0 = nullptr, *M0 = nullptr, *Fs = nullptr, *Ms = nullptr, *tmpI = nullptr;
  float *phiF = nullptr, *psiF = nullptr, *phiM = nullptr, *psiM = nullptr;
  float *Ft = nullptr, *Mt = nullptr;
  float *gFu = nullptr, *gMu = nullptr, *t1F = nullptr, *t1M = nullptr, *t2F = nullptr, *t2M = nullptr;
  double* cc_partials = nullptr;
  int cc_cap = 0;
  double* inv_psum = nullptr;
  float* inv_pmax = nullptr;
  int inv_cap = 0;
  float* coeff_upd = nullptr;   // [3][cap]
  float* coeff_tot = nullptr;   // [3][cap]
  double* coeff_img = nullptr;  // [3][cap]
  int coeff_cap = 0;
  int R_upd[3] = {0, 0, 0}, R_tot[3] = {0, 0, 0};
  IterCtl* ctl = nullptr;
  LogDev logdev{};
  int coop_max = 0;  // largest cooperative grid of the level kernel (0: not queried)
  unsigned* hist = nullptr;  // 256 bins + 2 min/max
  // host mirrors
  std::vector<float> h_coeff_upd, h_coeff_tot;
  std::vector<double> h_coeff_img;
  int cur_level = -1;
  GridInfo cur_grid{};
  std::vector<int32_t> log_level, log_iter, log_inv;
  std::vector<double> log_metric, log_conv;
  // read-back staging of the running level
  IterCtl h_ctl{};
  std::vector<double> h_lm, h_lc;
  std::vector<int> h_li;
  // tile plan per level (stage parameters, then the tuning table, then the cost models)
  LevelPlan plan[SYNX_MAX_LEVELS] = {};
  // metric masks (synx_set_masks): one byte per voxel on their own grids, null for none; the
  // per-iteration validity of the virtual voxels lives in the arena
  unsigned char* maskF = nullptr;
  unsigned char* maskM = nullptr;
  GridInfo gmF{}, gmM{};
  unsigned char* valid = nullptr;
  // initial half-fields phiF, psiF, phiM, psiM (component planes, one after the other, on init_grid),
  // resampled to the first level's grid when it starts, or null: zero fields
  float* init_half = nullptr;
  GridInfo init_grid{};
  int* inv_list[2] = {nullptr, nullptr};  // deferred voxels of the single-pass inverse, per half
  // canonical buffer assignment (level changes swap field and work buffers)
  float* canon[8] = {};
  // graphs: one executable per level, valid while the arena and grids are unchanged
  cudaGraphExec_t gexec_lv[SYNX_MAX_LEVELS] = {};
  long long graph_nodes[SYNX_MAX_LEVELS] = {};
  // profiling
  cudaEvent_t lev_ev[3] = {};
  LevelProf lprof[SYNX_MAX_LEVELS];
  double prof_inv_ms = 0, prof_cc_ms = 0;
  long long prof_inv_launches = 0, prof_inv_vox = 0, prof_cc_launches = 0, prof_cc_vox = 0;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, int>> ev_pairs_inv, ev_pairs_cc;  // indices into ev_pool
  size_t ev_used = 0;
};

namespace {

int set_err(synx_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  g_last_error = msg;
  return code;
}

#define CUDA_TRY(ctx, call)                                                                  \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return set_err(ctx, SYNX_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));  \
  } while (0)

size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

// Device scratch of histogram_match_dev: `levels` bins and the min/max pair, then the per-block sums.
size_t hm_sums_offset(int levels) { return (4 * (size_t)levels + 8 + 15) & ~(size_t)15; }
size_t hm_scratch_bytes(int levels) { return hm_sums_offset(levels) + 8 * (size_t)HM_STATS_BLOCKS; }

void drop_graphs(synx_ctx* c) {
  for (auto& g : c->gexec_lv) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
}

void free_arena(synx_ctx* c) {
  drop_graphs(c);
  if (c->arena) cudaFree(c->arena);
  c->arena = nullptr;
  c->arena_bytes = 0;
}

int build_levels(synx_ctx* c) {
  c->lgeom.clear();
  c->lv.clear();
  c->Nmax = 0;
  for (int l = 0; l < c->P.n_levels; ++l) {
    synx_geom g = shrink(c->geF, (unsigned)c->P.shrink_factors[l]);
    GridInfo gi;
    geom_to_grid(g, gi);
    c->lgeom.push_back(g);
    c->lv.push_back(gi);
    c->Nmax = std::max(c->Nmax, gi.d.N);
  }
  return SYNX_OK;
}

long long level_inv_units(const GridInfo& g);

// Byte offsets of everything a context keeps on the device, for its images and schedule.
struct ArenaPlan {
  size_t F0, M0, Fs, Ms, Tmp, Field[4], Ft, Mt, Work[6], CC, IS, IM, Cu, Ct, Ci, Ctl, Lm, Lc, Li, H, V, IL[2];
  size_t total;
  int ccb, invb, coeff_cap, max_iters;
};

ArenaPlan arena_plan(const synx_ctx* c) {
  ArenaPlan a{};
  const int D = c->D;
  const long long Nmax = c->Nmax, NI = std::max(c->NF, c->NM);
  int ccb = 0, invb = 0;
  for (auto& g : c->lv) {
    ccb = std::max(ccb, cc_blocks_max(g, c->P.cc_radius));  // any chunk count a tile plan picks
    invb = std::max(invb, inv_blocks(g));
  }
  invb = std::max(invb, 2048);
  // level kernel: two slots per tile (its sub-iterations alternate between them)
  for (auto& g : c->lv) invb = (int)std::max<long long>(invb, 2 * level_inv_units(g));
  // step entry points on arbitrary grids reuse nothing from here
  const int coeff_cap = 1024;
  int max_iters = 1;
  for (int l = 0; l < c->P.n_levels; ++l) max_iters = std::max(max_iters, c->P.iterations[l]);
  size_t sz = 0;
  auto add = [&](size_t bytes) {
    size_t o = sz;
    sz += align_up(bytes);
    return o;
  };
  a.F0 = add(4 * c->NF), a.M0 = add(4 * c->NM), a.Fs = add(4 * c->NF), a.Ms = add(4 * c->NM), a.Tmp = add(4 * NI);
  for (int k = 0; k < 4; ++k) a.Field[k] = add(4 * (size_t)D * Nmax);
  a.Ft = add(4 * Nmax), a.Mt = add(4 * Nmax);
  for (int k = 0; k < 6; ++k) a.Work[k] = add(4 * (size_t)D * Nmax);
  // CC partials: the block sums and, with metric masks, the blocks' valid counts after them
  a.CC = add(8 * 2 * (size_t)ccb), a.IS = add(8 * 2 * (size_t)invb), a.IM = add(4 * 2 * (size_t)invb);
  a.Cu = add(4 * 3 * coeff_cap), a.Ct = add(4 * 3 * coeff_cap), a.Ci = add(8 * 3 * coeff_cap);
  a.Ctl = add(sizeof(IterCtl));
  a.Lm = add(8 * (size_t)max_iters), a.Lc = add(8 * (size_t)max_iters), a.Li = add(4 * (size_t)max_iters);
  a.H = add(std::max((size_t)4 * 258, hm_scratch_bytes(256)));
  a.V = add((size_t)Nmax);  // metric-mask validity, one byte per voxel of the largest level
  // the single-pass inverse's deferred-voxel lists, one per half, room for every voxel
  for (int k = 0; k < 2; ++k) a.IL[k] = add(4 * (size_t)Nmax);
  a.total = sz;
  a.ccb = ccb;
  a.invb = invb;
  a.coeff_cap = coeff_cap;
  a.max_iters = max_iters;
  return a;
}

int allocate(synx_ctx* c) {
  const ArenaPlan pl = arena_plan(c);
  const size_t sz = pl.total;
  const int ccb = pl.ccb, invb = pl.invb, coeff_cap = pl.coeff_cap, max_iters = pl.max_iters;
  const size_t oF0 = pl.F0, oM0 = pl.M0, oFs = pl.Fs, oMs = pl.Ms, oTmp = pl.Tmp, oFt = pl.Ft, oMt = pl.Mt;
  const size_t *oField = pl.Field, *oWork = pl.Work;
  const size_t oCC = pl.CC, oIS = pl.IS, oIM = pl.IM, oCu = pl.Cu, oCt = pl.Ct, oCi = pl.Ci, oCtl = pl.Ctl;
  const size_t oLm = pl.Lm, oLc = pl.Lc, oLi = pl.Li, oH = pl.H;
  if (c->arena && c->arena_bytes >= sz) {
    // reuse
  } else {
    free_arena(c);
    cudaError_t e = c->P.test_inject == SYNX_INJECT_ALLOC_FAILURE ? cudaErrorMemoryAllocation
                                                                 : cudaMalloc((void**)&c->arena, sz);
    if (e != cudaSuccess) {
      c->arena = nullptr;
      cudaGetLastError();
      return set_err(c, SYNX_E_NOMEM, std::string("device arena of ") + std::to_string(sz) + " bytes: " +
                                          cudaGetErrorString(e));
    }
    c->arena_bytes = sz;
  }
  char* a = c->arena;
  c->F0 = (float*)(a + oF0);
  c->M0 = (float*)(a + oM0);
  c->Fs = (float*)(a + oFs);
  c->Ms = (float*)(a + oMs);
  c->tmpI = (float*)(a + oTmp);
  c->phiF = (float*)(a + oField[0]);
  c->psiF = (float*)(a + oField[1]);
  c->phiM = (float*)(a + oField[2]);
  c->psiM = (float*)(a + oField[3]);
  c->Ft = (float*)(a + oFt);
  c->Mt = (float*)(a + oMt);
  c->gFu = (float*)(a + oWork[0]);
  c->gMu = (float*)(a + oWork[1]);
  c->t1F = (float*)(a + oWork[2]);
  c->t1M = (float*)(a + oWork[3]);
  c->t2F = (float*)(a + oWork[4]);
  c->t2M = (float*)(a + oWork[5]);
  c->cc_partials = (double*)(a + oCC);
  c->cc_cap = ccb;
  c->inv_psum = (double*)(a + oIS);
  c->inv_pmax = (float*)(a + oIM);
  c->inv_cap = invb;
  c->coeff_upd = (float*)(a + oCu);
  c->coeff_tot = (float*)(a + oCt);
  c->coeff_img = (double*)(a + oCi);
  c->coeff_cap = coeff_cap;
  c->ctl = (IterCtl*)(a + oCtl);
  c->logdev.metric = (double*)(a + oLm);
  c->logdev.conv = (double*)(a + oLc);
  c->logdev.inv_iters = (int*)(a + oLi);
  c->logdev.cap = max_iters;
  c->hist = (unsigned*)(a + oH);
  c->valid = (unsigned char*)(a + pl.V);
  for (int k = 0; k < 2; ++k) c->inv_list[k] = (int*)(a + pl.IL[k]);
  CUDA_TRY(c, cudaMemsetAsync(c->ctl, 0, sizeof(IterCtl), c->stream));
  return SYNX_OK;
}

// Quantile of a histogram with equal bins [lo + b*bw, lo + (b+1)*bw), interpolated inside the bin
// that reaches p: ITK's Histogram::Quantile (ITK 5.4.6, the version SuperBuild/External_ITKv5.cmake:155
// pins), accumulating from the first bin below p = 0.5 and from the last one above.
double hist_quantile(const std::vector<unsigned>& h, double lo, double bw, double p) {
  const int nb = (int)h.size();
  double total = 0.0;
  for (unsigned v : h) total += (double)v;
  auto bmin = [&](int b) { return lo + b * bw; };
  auto bmax = [&](int b) { return lo + (b + 1) * bw; };
  double cum = 0, pn = 0, pprev = 0, fn = 0;
  if (p < 0.5) {
    int k = 0;
    do {
      fn = h[k];
      cum += fn;
      pprev = pn;
      pn = cum / total;
      ++k;
    } while (k < nb && pn < p);
    return bmin(k - 1) + ((p - pprev) / (fn / total)) * (bmax(k - 1) - bmin(k - 1));
  }
  int k = nb - 1, m = 0;
  pn = 1.0;
  do {
    fn = h[k];
    cum += fn;
    pprev = pn;
    pn = 1.0 - cum / total;
    --k;
    ++m;
  } while (m < nb && pn > p);
  return bmax(k + 1) - ((pprev - p) / (fn / total)) * (bmax(k + 1) - bmin(k + 1));
}

struct ImageStats {
  float mn, mx, mean;
};

// Min, max and mean of one image (the mean cast to float, as ITK casts it to the pixel type).  The
// per-block sums come back and are added in block order, so the result does not depend on timing.
int image_stats(synx_ctx* c, const float* x, long long n, void* scratch, int levels, cudaStream_t s, ImageStats& st) {
  unsigned* mm = (unsigned*)scratch + levels;
  double* part = (double*)((char*)scratch + hm_sums_offset(levels));
  unsigned init[2] = {float_to_ordered(FLT_MAX), float_to_ordered(-FLT_MAX)};
  CUDA_TRY(c, cudaMemcpyAsync(mm, init, 8, cudaMemcpyHostToDevice, s));
  launch_stats(x, n, part, HM_STATS_BLOCKS, mm, s);
  unsigned hm[2];
  std::vector<double> hp(HM_STATS_BLOCKS);
  CUDA_TRY(c, cudaMemcpyAsync(hm, mm, 8, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaMemcpyAsync(hp.data(), part, 8 * (size_t)HM_STATS_BLOCKS, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(c, cudaStreamSynchronize(s));
  double sum = 0.0;
  for (double v : hp) sum += v;
  st.mn = ordered_to_float(hm[0]);
  st.mx = ordered_to_float(hm[1]);
  st.mean = (float)(sum / (double)n);
  return SYNX_OK;
}

// Histogram matching of `src` to `ref` (ITK's HistogramMatchingImageFilter; PreprocessImage runs it
// with 256 levels, 12 match points and the threshold at the mean, Examples/itkantsRegistrationHelper.hxx:111-122).
// Statistics and thresholded histograms of both images on the device; the table of match points
// on the host in double (points + 2 rows: the thresholds, the quantiles j/(points+1), the maxima;
// slope 0 between coincident source points; below the first point the line through the minima,
// above the last the one through the maxima); one mapping pass writes `out` (may be `src`).
int histogram_match_dev(synx_ctx* c, const float* src, long long ns, const float* ref, long long nr, int levels,
                        int points, bool thr_mean, float* out, void* scratch, cudaStream_t s) {
  ImageStats a, b;
  int rc = image_stats(c, src, ns, scratch, levels, s, a);
  if (rc) return rc;
  rc = image_stats(c, ref, nr, scratch, levels, s, b);
  if (rc) return rc;
  unsigned* bins = (unsigned*)scratch;
  auto histogram = [&](const float* x, long long n, const ImageStats& st, double thr,
                       std::vector<unsigned>& h) -> int {
    CUDA_TRY(c, cudaMemsetAsync(bins, 0, 4 * (size_t)levels, s));
    launch_histogram_range(x, n, (double)st.mn, (double)st.mx, levels, thr, (double)st.mx, bins, s);
    h.assign(levels, 0u);
    CUDA_TRY(c, cudaMemcpyAsync(h.data(), bins, 4 * (size_t)levels, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(c, cudaStreamSynchronize(s));
    return SYNX_OK;
  };
  const double sthr = thr_mean ? (double)a.mean : (double)a.mn, rthr = thr_mean ? (double)b.mean : (double)b.mn;
  std::vector<unsigned> hs, hr;
  if ((rc = histogram(src, ns, a, sthr, hs))) return rc;
  if ((rc = histogram(ref, nr, b, rthr, hr))) return rc;
  const double bws = ((double)a.mx - (double)a.mn) / levels, bwr = ((double)b.mx - (double)b.mn) / levels;
  HistMatchMap t = {};
  t.points = points;
  t.src[0] = sthr;
  t.ref[0] = rthr;
  t.src[points + 1] = (double)a.mx;
  t.ref[points + 1] = (double)b.mx;
  const double delta = 1.0 / ((double)points + 1.0);
  for (int j = 1; j <= points; ++j) {
    t.src[j] = hist_quantile(hs, (double)a.mn, bws, j * delta);
    t.ref[j] = hist_quantile(hr, (double)b.mn, bwr, j * delta);
  }
  for (int j = 0; j <= points; ++j) {
    const double den = t.src[j + 1] - t.src[j];
    t.grad[j] = den != 0.0 ? (t.ref[j + 1] - t.ref[j]) / den : 0.0;
  }
  t.src_min = (double)a.mn;
  t.src_max = (double)a.mx;
  t.ref_min = (double)b.mn;
  t.ref_max = (double)b.mx;
  const double dlo = t.src[0] - t.src_min, dhi = t.src[points + 1] - t.src_max;
  t.lower_grad = dlo != 0.0 ? (t.ref[0] - t.ref_min) / dlo : 0.0;
  t.upper_grad = dhi != 0.0 ? (t.ref[points + 1] - t.ref_max) / dhi : 0.0;
  launch_histogram_map(src, out, ns, t, s);
  CUDA_TRY(c, cudaGetLastError());
  return SYNX_OK;
}

// Preprocess one image in place on the device: histogram quantiles -> window -> [0, 1].
int preprocess(synx_ctx* c, float* img, long long n) {
  unsigned init[2] = {float_to_ordered(FLT_MAX), float_to_ordered(-FLT_MAX)};
  unsigned* mm = c->hist + 256;
  CUDA_TRY(c, cudaMemcpyAsync(mm, init, 8, cudaMemcpyHostToDevice, c->stream));
  launch_minmax(img, n, mm, c->stream);
  unsigned hm[2];
  CUDA_TRY(c, cudaMemcpyAsync(hm, mm, 8, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  const float mn = ordered_to_float(hm[0]), mx = ordered_to_float(hm[1]);
  const int nb = 256;
  const float margin = ((mx - mn) / (float)nb) / 10.0f;
  const float hi = mx + margin;
  CUDA_TRY(c, cudaMemsetAsync(c->hist, 0, 4 * nb, c->stream));
  launch_histogram(img, n, mn, hi, nb, c->hist, c->stream);
  std::vector<unsigned> hh(nb);
  CUDA_TRY(c, cudaMemcpyAsync(hh.data(), c->hist, 4 * nb, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  const double bw = ((double)hi - (double)mn) / nb;
  auto quantile = [&](double p) { return hist_quantile(hh, (double)mn, bw, p); };
  const float wlo = (float)quantile(c->P.winsor_lower), whi = (float)quantile(c->P.winsor_upper);
  const double scale = 1.0 / ((double)whi - (double)wlo);
  const double shift = -(double)wlo * scale;
  launch_window(img, img, n, wlo, whi, scale, shift, c->stream);
  return SYNX_OK;
}

// Kernels for the current level: pyramid (per image axis) and field smoothing (per field
// axis, width limited by the level size).
int upload_level_kernels(synx_ctx* c, int level) {
  const GridInfo& g = c->lv[level];
  c->h_coeff_upd.assign(3 * c->coeff_cap, 0.0f);
  c->h_coeff_tot.assign(3 * c->coeff_cap, 0.0f);
  for (int a = 0; a < c->D; ++a) {
    const int n = a == 0 ? g.d.nx : (a == 1 ? g.d.ny : g.d.nz);
    auto ku = gauss_kernel(c->P.update_variance, 0.001, (size_t)n);
    auto kt = gauss_kernel(c->P.total_variance, 0.001, (size_t)n);
    if ((int)ku.size() > c->coeff_cap || (int)kt.size() > c->coeff_cap)
      return set_err(c, SYNX_E_UNSUPPORTED, "field smoothing kernel wider than 1024 taps");
    c->R_upd[a] = (int)ku.size() / 2;
    c->R_tot[a] = (int)kt.size() / 2;
    for (size_t j = 0; j < ku.size(); ++j) c->h_coeff_upd[a * c->coeff_cap + j] = (float)ku[j];
    for (size_t j = 0; j < kt.size(); ++j) c->h_coeff_tot[a * c->coeff_cap + j] = (float)kt[j];
  }
  CUDA_TRY(c, cudaMemcpyAsync(c->coeff_upd, c->h_coeff_upd.data(), 4 * 3 * c->coeff_cap, cudaMemcpyHostToDevice,
                              c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->coeff_tot, c->h_coeff_tot.data(), 4 * 3 * c->coeff_cap, cudaMemcpyHostToDevice,
                              c->stream));
  return SYNX_OK;
}

int smooth_images_for_level(synx_ctx* c, int level) {
  const double sigma = c->P.smoothing_sigmas[level];
  struct Img {
    const float* src;
    float* dst;
    const GridInfo* g;
  } imgs[2] = {{c->F0, c->Fs, &c->gF}, {c->M0, c->Ms, &c->gM}};
  for (auto& im : imgs) {
    const GridInfo& g = *im.g;
    if (sigma <= 0.0) {
      CUDA_TRY(c, cudaMemcpyAsync(im.dst, im.src, 4 * g.d.N, cudaMemcpyDeviceToDevice, c->stream));
      continue;
    }
    // per-axis kernels, last axis first (chained as DiscreteGaussianImageFilter does)
    std::vector<double> hk(3 * c->coeff_cap, 0.0);
    int R[3] = {0, 0, 0};
    for (int a = 0; a < c->D; ++a) {
      double var = sigma * sigma;
      if (c->P.sigmas_in_mm) var /= g.sp[a] * g.sp[a];
      auto k = gauss_kernel(var, 0.01, 32);
      R[a] = (int)k.size() / 2;
      for (size_t j = 0; j < k.size(); ++j) hk[a * c->coeff_cap + j] = k[j];
    }
    c->h_coeff_img = hk;
    CUDA_TRY(c, cudaMemcpyAsync(c->coeff_img, c->h_coeff_img.data(), 8 * 3 * c->coeff_cap, cudaMemcpyHostToDevice,
                                c->stream));
    // ping-pong between dst and tmpI so the final pass (axis 0) lands in dst
    const float* src = im.src;
    int passes = c->D;
    for (int p = 0; p < passes; ++p) {
      const int axis = c->D - 1 - p;
      float* out = ((passes - 1 - p) % 2 == 0) ? im.dst : c->tmpI;
      launch_conv_image_axis(src, out, g, axis, c->coeff_img + axis * c->coeff_cap, R[axis], c->stream);
      src = out;
    }
    // no synchronisation: a copy from pageable host memory has taken its data when it returns, and the
    // next image's coefficient upload is ordered after these passes on the stream
  }
  return SYNX_OK;
}

// Smooth both halves: the fused all-axes kernel when its shared-memory tile fits, otherwise
// one pass per axis through `tmp` (in != out; orig is read only at each output voxel).
void smooth_halves(synx_ctx* c, const float* const* in, float* const* out, const float* const* orig,
                   float* const* tmp, const float* coeff_base, const float* host_base, const int R[3], bool epilogue,
                   float w1, float w2, bool maxnorm) {
  const GridInfo& g = c->cur_grid;
  const float* k[3] = {coeff_base, coeff_base + c->coeff_cap, coeff_base + 2 * c->coeff_cap};
  if (smooth3_supported(c->D, R)) {
    const float* kh[3] = {host_base, host_base + c->coeff_cap, host_base + 2 * c->coeff_cap};
    const int rows = c->cur_level >= 0 ? c->plan[c->cur_level].smooth_rows : -1;
    // tile rows > 0: the slab kernel; -1: xy kernel + z kernel; -2 / -3: pipelined xy kernel with
    // 32 / 64-row tiles + z kernel
    const SmoothPlan sp{rows > 0 ? rows : 0, 0, rows == -2 ? 32 : (rows == -3 ? 64 : 0)};
    launch_smooth_field(in, out, orig, tmp, 2, g, kh, R, epilogue, w1, w2, maxnorm, c->ctl, c->stream, &sp);
    return;
  }
  const int D = c->D;
  const float* src[2] = {in[0], in[1]};
  for (int a = 0; a < D; ++a) {
    const bool last = a == D - 1;
    float* const* dst = last ? out : (((D - 1 - a) % 2 == 0) ? out : tmp);
    launch_smooth_field_pass(src, dst, last ? orig : nullptr, 2, g, a, k[a], R[a], last && epilogue, w1, w2,
                             last && maxnorm, c->ctl, c->stream);
    src[0] = dst[0];
    src[1] = dst[1];
  }
}

// One SyN iteration on the current level (all launches asynchronous, stop-aware).
// Enqueues one SyN iteration on c->stream.  loops (only while the stream is being captured into a
// graph): each fixed-point inverse becomes its k = 0 launch followed by a conditional WHILE node
// whose body is one sub-iteration launch plus the loop-control kernel, instead of all
// max_iter + 1 launches of which the converged tail does nothing.
// Scope in which the library's launches use programmatic dependent launch (see launch_k).
struct PdlScope {
  int saved;
  explicit PdlScope(bool on) : saved(t_pdl) {
    t_pdl = on ? 1 : 0;
    t_pdl_skip = 1;  // the first launch follows whatever came before the iteration
  }
  ~PdlScope() {
    t_pdl = saved;
    t_pdl_skip = 0;
  }
};

cudaError_t enqueue_iteration(synx_ctx* c, bool profile, bool loops = false, bool with_pdl = true) {
  const GridInfo& g = c->cur_grid;
  cudaStream_t s = c->stream;
  PdlScope pdl(with_pdl && !profile && !c->pdl_failed && (c->P.flags & SYNX_F_NO_PDL) == 0);
  auto ev = [&](void) -> int {
    if (c->ev_used >= c->ev_pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      c->ev_pool.push_back(e);
    }
    int idx = (int)c->ev_used++;
    cudaEventRecord(c->ev_pool[idx], s);
    return idx;
  };
  // Sweep orders: each kernel walks its grid opposite to the kernel whose output it reads, so it
  // starts on that kernel's last-written tiles while they are in L2 (warp backwards after the
  // inversions' forward walks, CC forwards, xy smoothing backwards, z smoothing forwards, composition
  // backwards, the inversions forwards).  Only the order of the tiles changes, not any result.
  struct SweepReset {
    ~SweepReset() { t_rev = 0; }
  } sweep_reset;
  t_rev = 1;
  launch_warp_pair(c->Fs, c->gF, c->psiF, c->Ms, c->gM, c->psiM, g, c->Ft, c->Mt, c->ctl, s);
  t_rev = 0;
  const bool masked = c->maskF != nullptr || c->maskM != nullptr;
  if (masked) launch_mask_validity(c->maskF, c->gmF, c->psiF, c->maskM, c->gmM, c->psiM, g, c->valid, c->ctl, s);
  int e0 = profile ? ev() : -1;
  launch_cc(c->Ft, c->Mt, g, c->P.cc_radius, c->gFu, c->gMu, c->cc_partials, c->ctl, s, nullptr,
            (c->P.flags & SYNX_F_CC_FP32_SUMS) != 0, c->plan[c->cur_level].cc_chunks, masked ? c->valid : nullptr);
  if (profile) c->ev_pairs_cc.push_back({e0, ev()});
  // update-field smoothing, SyN epilogue (boundary zero, blend) and max ||u/spacing||
  const float* upd[2] = {c->t1F, c->t1M};
  const double var = c->P.update_variance;
  t_rev = 1;  // xy pass backwards, z pass forwards
  {
    const float* in[2] = {c->gFu, c->gMu};
    float* out[2] = {c->t1F, c->t1M};
    float* tmp[2] = {c->t2F, c->t2M};
    if (var > 0.0) {
      const float w1 = var < 0.5 ? (float)(1.0 - var / 0.5) : 1.0f;
      smooth_halves(c, in, out, in, tmp, c->coeff_upd, c->h_coeff_upd.data(), c->R_upd, true, w1, 1.0f - w1, true);
    } else {
      // no smoothing (the kernel is [0 1 0]): a copy plus the max norm, boundary untouched
      launch_smooth_field_pass(in, out, nullptr, 2, g, 0, c->coeff_upd, c->R_upd[0], false, 1.f, 0.f, true, c->ctl,
                               s);
    }
  }
  // scale + compose into the forward half-fields (in place), or into t2 followed by the
  // total-field smoothing back into the half-fields when its variance is positive
  t_rev = 1;  // composition backwards
  if (c->P.total_variance > 0.0) {
    const double vt = c->P.total_variance;
    const float w1 = vt < 0.5 ? (float)(1.0 - vt / 0.5) : 1.0f;
    const float* w[2] = {c->phiF, c->phiM};
    float* t2[2] = {c->t2F, c->t2M};
    launch_compose(upd, w, t2, 2, g, (float)c->P.learning_rate, c->ctl, s);
    const float* in[2] = {c->t2F, c->t2M};
    float* out[2] = {c->phiF, c->phiM};
    float* tmp[2] = {c->gFu, c->gMu};
    t_rev = 0;
    smooth_halves(c, in, out, in, tmp, c->coeff_tot, c->h_coeff_tot.data(), c->R_tot, true, w1, 1.0f - w1, false);
  } else {
    const float* w[2] = {c->phiF, c->phiM};
    float* o[2] = {c->phiF, c->phiM};
    launch_compose(upd, w, o, 2, g, (float)c->P.learning_rate, c->ctl, s);
  }
  t_rev = 0;
  // precision study: half-fields stored in half precision (rounded after every step that writes them)
  const bool fp16 = (c->P.flags & SYNX_F_FIELDS_FP16) != 0;
  auto round_pair = [&](float* a, float* b) {
    float* f[2] = {a, b};
    launch_round_half(f, 2, (long long)c->D * g.d.N, s);
  };
  if (fp16) round_pair(c->phiF, c->phiM);
  // fixed-point inverses: psi <- inv(phi) warm from psi, then phi <- inv(psi) warm from phi
  PartialBufs pb{c->inv_psum, c->inv_pmax, c->inv_cap};
  const int mi = c->P.inv_max_iter;
  int e1 = profile ? ev() : -1;
  // the CC derivative buffers are free until the next iteration: they carry the inverse residual
  float* ecache[2] = {c->gFu, c->gMu};
  // single-pass form (one streaming pass per sub-iteration plus a short pass over the deferred
  // voxels) unless the stage asks for the two-pass form; both give the same bits
  const bool single = (c->P.flags & SYNX_F_INV_TWO_PASS) == 0;
  int* lists[2] = {c->inv_list[0], c->inv_list[1]};
  auto inversion = [&](int phase, const float* const* phi, float* const* psi) -> cudaError_t {
    const double mt = c->P.inv_mean_tol, xt = c->P.inv_max_tol;
    auto sub = [&](int k, cudaStream_t st) {
      if (single) {
        launch_invert_spec(phi, psi, 2, g, k, mi, mt, xt, c->ctl, phase, pb, st, true, ecache, lists);
        launch_invert_fix(phi, psi, 2, g, k, mi, c->ctl, phase, st, true, ecache, lists);
      } else {
        launch_invert_step(phi, psi, 2, g, k, mi, mt, xt, c->ctl, phase, pb, st, true, ecache);
      }
    };
    auto control = [&](cudaGraphConditionalHandle h, bool init, cudaStream_t st) {
      if (single) launch_inv_spec_control(c->ctl, phase, h, mi, init, st);
      else launch_inv_loop_control(c->ctl, phase, h, mi, init, st);
    };
    if (!loops) {
      for (int k = 0; k < (single ? mi : mi + 1); ++k) sub(k, s);
      return cudaSuccess;
    }
    sub(0, s);
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(s, &st, nullptr, &cg, &deps, &nd);
    if (e != cudaSuccess) return e;
    if (st != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureInvalidated;
    cudaGraphConditionalHandle h = 0;
    if ((e = cudaGraphConditionalHandleCreate(&h, cg, 0, 0)) != cudaSuccess) return e;
    control(h, true, s);
    if ((e = cudaStreamGetCaptureInfo(s, &st, nullptr, &cg, &deps, &nd)) != cudaSuccess) return e;
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if ((e = cudaGraphAddNode(&node, cg, deps, nd, &np)) != cudaSuccess) return e;
    if ((e = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
      return e;
    if ((e = cudaStreamBeginCaptureToGraph(c->aux, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return e;
    t_pdl_skip = 1;  // the body's first kernel has no kernel before it
    sub(-1, c->aux);
    control(h, false, c->aux);
    cudaGraph_t body = nullptr;
    e = cudaStreamEndCapture(c->aux, &body);
    t_pdl_skip = 1;  // the next launch on s follows the conditional node
    return e;
  };
  {
    const float* phi[2] = {c->phiF, c->phiM};
    float* psi[2] = {c->psiF, c->psiM};
    const cudaError_t e = inversion(0, phi, psi);
    if (e != cudaSuccess) return e;
  }
  if (fp16) round_pair(c->psiF, c->psiM);
  {
    const float* phi[2] = {c->psiF, c->psiM};
    float* psi[2] = {c->phiF, c->phiM};
    const cudaError_t e = inversion(1, phi, psi);
    if (e != cudaSuccess) return e;
  }
  if (fp16) round_pair(c->phiF, c->phiM);
  if (profile) c->ev_pairs_inv.push_back({e1, ev()});
  launch_converge(c->ctl, c->logdev, c->P.convergence_threshold, c->P.convergence_window, s);
  return cudaSuccess;
}

// The persistent level kernel serves small levels (launch latency dominates there) when the
// stage uses the common options it implements; larger levels, the event-profiled mode and the
// rarer options (total-field smoothing, no update smoothing, wide kernels) take the per-kernel
// path.
// Measured on the 182x218x182 pyramid: 0.1 M voxels 4.2 ms in the level kernel vs ~9 ms as separate
// kernels; 0.9 M voxels 16.0 ms vs 14.3 ms.
constexpr long long kPersistentMaxVoxels = 400000;

// Inversion tiles per half-field of the level kernel on grid g (two residual partial slots each).
long long level_inv_units(const GridInfo& g) {
  const int zb = level_zb(g.d, 2);
  return (long long)((g.d.nx + 31) / 32) * ((g.d.ny + 7) / 8) * ((g.d.nz + zb - 1) / zb);
}

// Whether a level runs in the level kernel (alone or in a batch): the options it implements, and
// a level small enough that launch latency, not bandwidth, dominates the per-kernel path.
// Whether the level kernel implements the stage's options on grid g (whatever its size).
bool persistent_capable(synx_ctx* c, const GridInfo& g, bool profile) {
  if (profile || (c->P.flags & (SYNX_F_NO_PERSISTENT | SYNX_F_CC_FP32_SUMS | SYNX_F_FIELDS_FP16))) return false;
  if (c->maskF || c->maskM) return false;  // metric masks run the per-kernel path
  if (c->P.total_variance > 0.0 || !(c->P.update_variance > 0.0)) return false;
  int rs = 1;
  for (int a = 0; a < c->D; ++a) rs = std::max(rs, c->R_upd[a]);
  if (rs > kLevelMaxSmoothRadius) return false;
  if (c->P.cc_radius < 1 || c->P.cc_radius > 7) return false;
  return 2 * level_inv_units(g) <= c->inv_cap;
}

bool persistent_eligible(synx_ctx* c, const GridInfo& g, bool profile) {
  const long long max_vox = c->P.persistent_max_voxels > 0 ? c->P.persistent_max_voxels : kPersistentMaxVoxels;
  return g.d.N <= max_vox && persistent_capable(c, g, profile);
}

// Radius of the update-field smoothing kernel on a level grid (the widest axis).
int level_smooth_radius(const synx_ctx* c, const GridInfo& g) {
  int rs = 1;
  for (int a = 0; a < c->D; ++a) {
    const int n = a == 0 ? g.d.nx : (a == 1 ? g.d.ny : g.d.nz);
    rs = std::max(rs, (int)gauss_kernel(c->P.update_variance, 0.001, (size_t)n).size() / 2);
  }
  return rs;
}

// The tile plan of a level: the tuning table's entry for its grid (unless the stage opts out),
// overridden by explicit stage parameters; without either, the cost models (xy and z smoothing
// kernels, the CC chunk model, the persistent kernel up to the size threshold).
LevelPlan resolve_plan(synx_ctx* c, int level) {
  const GridInfo& g = c->lv[level];
  LevelPlan p{-1, -1, 0};
  LevelPlan t{};
  if (c->P.tuning == 0 &&
      tuning_lookup(c->D, c->P.cc_radius, level_smooth_radius(c, g), g.d.nx, g.d.ny, g.d.nz, &t))
    p = t;
  if (c->P.smooth_tile_rows != 0) p.smooth_rows = c->P.smooth_tile_rows;
  if ((c->P.flags & SYNX_F_SMOOTH_TWO_PASS) && p.smooth_rows > 0) p.smooth_rows = -1;
  if (c->P.cc_z_chunks > 0) p.cc_chunks = c->P.cc_z_chunks;
  if (c->P.persistent_max_voxels > 0) p.persistent = -1;  // an explicit size threshold decides
  return p;
}

bool use_persistent(synx_ctx* c, int level, const GridInfo& g, bool profile, int* blocks) {
  const int choice = c->plan[level].persistent;
  const bool ok = choice == 1 ? persistent_capable(c, g, profile)
                              : (choice == 0 ? false : persistent_eligible(c, g, profile));
  if (!ok) return false;
  if (c->coop_max <= 0) c->coop_max = level_max_blocks(c->D, c->P.cc_radius, kLevelMaxSmoothRadius, c->device);
  if (c->coop_max <= 0) return false;
  // every co-resident block: the phases are latency-bound at these sizes, so more warps in
  // flight shorten each phase by more than the wider barrier costs (measured at 13k-900k voxels)
  *blocks = c->coop_max;
  if (c->P.persistent_blocks > 0) *blocks = std::min(c->P.persistent_blocks, c->coop_max);
  return *blocks > 0;
}

LevelArgs make_level_args(synx_ctx* c, const GridInfo& g, int iters) {
  LevelArgs A;
  memset(&A, 0, sizeof(A));
  const int D = c->D;
  const int gx = (g.d.nx + 31) / 32, gy = (g.d.ny + 7) / 8;
  const int zw = level_zb(g.d, 1), zc2 = level_zb(g.d, 2);
  A.warp = WarpArgs{c->Fs, c->Ms, c->psiF, c->psiM, c->Ft, c->Mt, c->gF.d, c->gM.d, g.d,
                    make_affine(g, c->gF), make_affine(g, c->gM), zw};
  A.cc = make_cc_params(g, c->P.cc_radius);
  A.cc_gx = gx;
  A.cc_gy = gy;
  A.cc_gz = (g.d.nz + A.cc.ZC - 1) / A.cc.ZC;
  A.gF = c->gFu;
  A.gM = c->gMu;
  const double var = c->P.update_variance;
  const float w1 = var < 0.5 ? (float)(1.0 - var / 0.5) : 1.0f;
  const float* kh[3] = {c->h_coeff_upd.data(), c->h_coeff_upd.data() + c->coeff_cap,
                        c->h_coeff_upd.data() + 2 * c->coeff_cap};
  const float* in[2] = {c->gFu, c->gMu};
  float* t2[2] = {c->t2F, c->t2M};
  float* t1[2] = {c->t1F, c->t1M};
  int RR = 1;
  A.sxy = make_smooth_args(in, D == 3 ? t2 : t1, in, 2, g, kh, c->R_upd, true, w1, 1.0f - w1, true, &RR);
  A.sz = A.sxy;
  A.sz.in = Ptr2c{{c->t2F, c->t2M}};
  A.sz.out = Ptr2{{c->t1F, c->t1M}};
  A.sz.ZC = smooth_z_chunk(g.d, 2, RR, 296);
  A.sz_gz = (g.d.nz + A.sz.ZC - 1) / A.sz.ZC;
  A.r_smooth = RR;
  A.comp.d = Ptr2c{{c->t1F, c->t1M}};
  A.comp.w = Ptr2c{{c->phiF, c->phiM}};
  A.comp.o = Ptr2{{c->phiF, c->phiM}};
  A.comp.g = g.d;
  A.comp.m = make_affine(g, g);
  A.comp.eta = c->P.learning_rate;
  A.comp.zb = zc2;
  const float* phis[2] = {c->phiF, c->phiM};
  float* psis[2] = {c->psiF, c->psiM};
  const float* psic[2] = {c->psiF, c->psiM};
  float* phim[2] = {c->phiF, c->phiM};
  // the CC derivative buffers are free from the composition to the next iteration's CC phase:
  // they carry the inverse residual between sub-iterations
  float* ecache[2] = {c->gFu, c->gMu};
  A.invA = make_inv_args(phis, psis, 2, g, zc2, ecache);
  A.invB = make_inv_args(psic, phim, 2, g, zc2, ecache);
  A.g = g.d;
  A.ctl = c->ctl;
  A.log = c->logdev;
  A.cc_partials = c->cc_partials;
  A.inv_psum = c->inv_psum;
  A.inv_pmax = c->inv_pmax;
  A.pcap = c->inv_cap;
  A.iters = iters;
  A.el_gx = gx;
  A.el_gy = gy;
  A.warp_gz = (g.d.nz + zw - 1) / zw;
  A.comp_gz = (g.d.nz + zc2 - 1) / zc2;
  A.inv_gz = A.comp_gz;
  A.inv_max_iter = c->P.inv_max_iter;
  A.inv_mean_tol = c->P.inv_mean_tol;
  A.inv_max_tol = c->P.inv_max_tol;
  A.conv_threshold = c->P.convergence_threshold;
  A.conv_window = c->P.convergence_window;
  A.diag = affine_diag_host(A.warp.mF) && affine_diag_host(A.warp.mM) && affine_diag_host(A.comp.m);
  // failure-detection test: every barrier waits for one block that was never launched, with a short
  // poll limit, so the first wait runs out, sets the error flag and the kernel ends
  const bool inject = c->P.test_inject == SYNX_INJECT_BARRIER_TIMEOUT;
  A.bar_extra = inject ? 1 : 0;
  A.bar_spins = inject ? (1ll << 14) : (1ll << 24);
  return A;
}

// Level set-up, enqueued on c->stream: pyramid smoothing of both images, resampling (or zeroing)
// of the four half-fields, reset of the control block.
int level_begin(synx_ctx* c, int level) {
  synx::NvtxRange range("synx level setup", level);
  if (!c->images_set) return set_err(c, SYNX_E_STATE, "synx_run_level: images not set");
  if (level != c->cur_level + 1 || level >= c->P.n_levels)
    return set_err(c, SYNX_E_STATE, "synx_run_level: levels must run in order 0.." + std::to_string(c->P.n_levels - 1));
  CUDA_TRY(c, cudaSetDevice(c->device));
  const GridInfo& gl = c->lv[level];
  const int D = c->D;
  CUDA_TRY(c, cudaEventRecord(c->lev_ev[0], c->stream));
  int rc = smooth_images_for_level(c, level);
  if (rc) return rc;
  rc = upload_level_kernels(c, level);
  if (rc) return rc;
  c->plan[level] = resolve_plan(c, level);
  if (level == 0 && c->init_half) {
    const size_t n = (size_t)D * c->init_grid.d.N;
    const float* in[4] = {c->init_half, c->init_half + n, c->init_half + 2 * n, c->init_half + 3 * n};
    float* out[4] = {c->phiF, c->psiF, c->phiM, c->psiM};
    launch_resample_fields(in, c->init_grid, out, gl, 4, c->stream);
    if (c->P.flags & SYNX_F_FIELDS_FP16) launch_round_half(out, 4, (long long)D * gl.d.N, c->stream);
  } else if (level == 0) {
    for (float* f : {c->phiF, c->psiF, c->phiM, c->psiM})
      CUDA_TRY(c, cudaMemsetAsync(f, 0, 4 * (size_t)D * gl.d.N, c->stream));
  } else {
    const float* in[4] = {c->phiF, c->psiF, c->phiM, c->psiM};
    float* out[4] = {c->gFu, c->gMu, c->t1F, c->t1M};
    launch_resample_fields(in, c->cur_grid, out, gl, 4, c->stream);
    std::swap(c->phiF, c->gFu);
    std::swap(c->psiF, c->gMu);
    std::swap(c->phiM, c->t1F);
    std::swap(c->psiM, c->t1M);
    if (c->P.flags & SYNX_F_FIELDS_FP16) {
      float* hf[4] = {c->phiF, c->psiF, c->phiM, c->psiM};
      launch_round_half(hf, 4, (long long)D * gl.d.N, c->stream);
    }
  }
  c->cur_grid = gl;
  c->cur_level = level;
  launch_zero_ctl_level(c->ctl, c->stream);
  CUDA_TRY(c, cudaGetLastError());
  c->ev_used = 0;
  c->ev_pairs_inv.clear();
  c->ev_pairs_cc.clear();
  CUDA_TRY(c, cudaEventRecord(c->lev_ev[1], c->stream));
  return SYNX_OK;
}

// The level's iterations, enqueued on c->stream: the level kernel, graph replay of one iteration,
// or plain launches.
int level_iterate(synx_ctx* c, int level) {
  synx::NvtxRange range("synx level iterate", level);
  const GridInfo& gl = c->lv[level];
  const int D = c->D;
  const int iters = c->P.iterations[level];
  const bool profile = (c->P.flags & SYNX_F_PROFILE_EVENTS) != 0;
  const bool graphs = (c->P.flags & SYNX_F_USE_GRAPHS) != 0 && !profile;
  int coop_blocks = 0;
  const bool persistent = iters > 0 && use_persistent(c, level, gl, profile, &coop_blocks);
  if (persistent) {
    // every iteration of this level in one cooperative launch
    LevelArgs A = make_level_args(c, gl, iters);
    CUDA_TRY(c, launch_level(A, D, c->P.cc_radius, coop_blocks, c->stream));
  } else if (graphs && iters > 0) {
    // one iteration is captured once per level and context (all its launch arguments are fixed
    // for a given level: the buffers are reset to the same assignment by synx_set_images) and
    // replayed `iters` times; the device-side stop flag ends a converged level early
    if (!c->gexec_lv[level]) {
      if (!c->aux && !c->loop_graphs_failed &&
          cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        c->aux = nullptr;
        c->loop_graphs_failed = true;
      }
      // with the inverse loops as conditional nodes first; if the driver refuses them, again
      // with plain launches
      // attempts: conditional loops with programmatic dependent launch, then without PDL (a driver
      // that refuses programmatic edges in captured graphs), then plain launches
      const bool pdl0 = !c->pdl_failed && (c->P.flags & SYNX_F_NO_PDL) == 0;
      const bool loops0 = !c->loop_graphs_failed;
      const std::pair<bool, bool> tries[3] = {{loops0, pdl0}, {loops0, false}, {false, false}};
      for (int tr = 0; tr < 3; ++tr) {
        const bool loops = tries[tr].first, with_pdl = tries[tr].second;
        if (tr > 0 && tries[tr] == tries[tr - 1]) continue;
        const long long before = launch_count();
        CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t eq = enqueue_iteration(c, false, loops, with_pdl);
        cudaGraph_t graph = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(c->stream, &graph);
        c->graph_nodes[level] = launch_count() - before;
        add_launch_count(-c->graph_nodes[level]);  // capture launches nothing
        cudaError_t e = eq != cudaSuccess ? eq : ee;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&c->gexec_lv[level], graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e == cudaSuccess) break;
        c->gexec_lv[level] = nullptr;
        if (loops && c->aux) {
          cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
          if (cudaStreamIsCapturing(c->aux, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone) {
            cudaGraph_t dead = nullptr;
            cudaStreamEndCapture(c->aux, &dead);
            if (dead) cudaGraphDestroy(dead);
          }
        }
        cudaGetLastError();
        if (!loops && !with_pdl) return set_err(c, SYNX_E_CUDA, std::string("level graph: ") + cudaGetErrorString(e));
        if (with_pdl) c->pdl_failed = true;
        else c->loop_graphs_failed = true;
      }
    }
    for (int k = 0; k < iters; ++k) CUDA_TRY(c, cudaGraphLaunch(c->gexec_lv[level], c->stream));
    add_launch_count(c->graph_nodes[level] * (long long)iters);
  } else {
    for (int k = 0; k < iters; ++k) CUDA_TRY(c, enqueue_iteration(c, profile));
  }
  return SYNX_OK;
}

// Enqueue the read-back of the level's control block and log (host staging in the context).
int level_readback(synx_ctx* c, int level) {
  synx::NvtxRange range("synx level readback", level);
  const int iters = c->P.iterations[level];
  CUDA_TRY(c, cudaEventRecord(c->lev_ev[2], c->stream));
  CUDA_TRY(c, cudaGetLastError());
  // collect the level's log
  CUDA_TRY(c, cudaMemcpyAsync(&c->h_ctl, c->ctl, sizeof(IterCtl), cudaMemcpyDeviceToHost, c->stream));
  c->h_lm.assign(std::max(iters, 1), 0.0);
  c->h_lc.assign(std::max(iters, 1), 0.0);
  c->h_li.assign(std::max(iters, 1), 0);
  if (iters > 0) {
    CUDA_TRY(c, cudaMemcpyAsync(c->h_lm.data(), c->logdev.metric, 8 * iters, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(c->h_lc.data(), c->logdev.conv, 8 * iters, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(c->h_li.data(), c->logdev.inv_iters, 4 * iters, cudaMemcpyDeviceToHost, c->stream));
  }
  return SYNX_OK;
}

// After the stream has drained: append the level's log and profile.
int level_finish(synx_ctx* c, int level) {
  const GridInfo& gl = c->lv[level];
  const int iters = c->P.iterations[level];
  const bool profile = (c->P.flags & SYNX_F_PROFILE_EVENTS) != 0;
  const IterCtl& hctl = c->h_ctl;
  const std::vector<double>& lm = c->h_lm;
  const std::vector<double>& lc = c->h_lc;
  const std::vector<int>& li = c->h_li;
  if (hctl.bar_err == 2)
    return set_err(c, SYNX_E_CUDA, "level " + std::to_string(level) +
                                       ": the level kernel was launched with less shared memory than its tiles use");
  if (hctl.bar_err)
    return set_err(c, SYNX_E_CUDA, "level " + std::to_string(level) + ": a grid barrier of the level kernel timed out");
  const int done = std::min(hctl.iter, iters);
  long long sub_iters = 0;
  for (int k = 0; k < done; ++k) {
    c->log_level.push_back(level);
    c->log_iter.push_back(k + 1);
    c->log_metric.push_back(lm[k]);
    c->log_conv.push_back(lc[k]);
    c->log_inv.push_back(li[k]);
    sub_iters += li[k];
  }
  LevelProf& lp = c->lprof[level];
  {
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, c->lev_ev[0], c->lev_ev[1]);
    cudaEventElapsedTime(&b, c->lev_ev[1], c->lev_ev[2]);
    lp.setup_ms += a;
    lp.iterate_ms += b;
    lp.iterations += done;
    lp.inv_sub += sub_iters;
    lp.voxels = gl.d.N;
  }
  if (profile) {
    for (auto& pr : c->ev_pairs_inv) {
      float ms = 0;
      cudaEventElapsedTime(&ms, c->ev_pool[pr.first], c->ev_pool[pr.second]);
      c->prof_inv_ms += ms;
      lp.inv_ms += ms;
    }
    for (auto& pr : c->ev_pairs_cc) {
      float ms = 0;
      cudaEventElapsedTime(&ms, c->ev_pool[pr.first], c->ev_pool[pr.second]);
      c->prof_cc_ms += ms;
      lp.cc_ms += ms;
      c->prof_cc_launches += 1;
      c->prof_cc_vox += gl.d.N;
    }
    // each executed fixed-point iteration is one working launch over one half-field
    c->prof_inv_launches += sub_iters;
    c->prof_inv_vox += sub_iters * gl.d.N;
  }
  return SYNX_OK;
}

int run_level_impl(synx_ctx* c, int level) {
  int rc = level_begin(c, level);
  if (!rc) rc = level_iterate(c, level);
  if (!rc) rc = level_readback(c, level);
  if (rc) return rc;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return level_finish(c, level);
}

bool valid_ctx(const synx_ctx* c) { return c != nullptr; }

// Blocks of a batched level launch for pairs with work w[i]: at least one each, the rest in
// proportion to the work (largest remainders first).  Depends on nothing but w and G.
std::vector<int> split_blocks(const std::vector<double>& w, int G) {
  const int n = (int)w.size();
  std::vector<int> g(n, 1);
  double W = 0.0;
  for (double x : w) W += x;
  int left = G - n;
  if (left <= 0 || W <= 0.0) return g;
  std::vector<std::pair<double, int>> frac;
  int used = 0;
  for (int i = 0; i < n; ++i) {
    const double share = left * (w[i] / W);
    const int whole = (int)share;
    g[i] += whole;
    used += whole;
    frac.push_back({share - whole, i});
  }
  std::sort(frac.begin(), frac.end(), [](const auto& a, const auto& b) {
    return a.first != b.first ? a.first > b.first : a.second < b.second;
  });
  for (int k = 0; k < left - used && k < n; ++k) g[frac[k].second] += 1;
  return g;
}

}  // namespace

struct synx_batch {
  int device = 0;
  std::string err;
  LevelArgs* d_args = nullptr;  // device staging of the per-pair level arguments
  int* d_first = nullptr;
  int cap = 0;
  std::vector<LevelArgs> h_args;
  std::vector<int> h_first;
  cudaEvent_t ev = nullptr;
  // lanes: the levels that run their own kernels (too large for the level kernel) run on these
  // streams concurrently, pair by pair round robin, so one pair's launch gaps and kernel tails
  // overlap another pair's work
  std::vector<cudaStream_t> lanes;
  std::vector<cudaEvent_t> lane_ev;
};

constexpr int kBatchLanes = 4;

namespace {

int batch_err(synx_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  g_last_error = msg;
  return code;
}

int batch_reserve(synx_batch* b, int n) {
  if (n <= b->cap) return SYNX_OK;
  if (b->d_args) cudaFree(b->d_args);
  if (b->d_first) cudaFree(b->d_first);
  b->d_args = nullptr;
  b->d_first = nullptr;
  b->cap = 0;
  const int cap = std::max(n, 64);
  if (cudaMalloc((void**)&b->d_args, sizeof(LevelArgs) * (size_t)cap) != cudaSuccess ||
      cudaMalloc((void**)&b->d_first, sizeof(int) * (size_t)(cap + 1)) != cudaSuccess) {
    cudaGetLastError();
    return batch_err(b, SYNX_E_NOMEM, "synx_batch: staging allocation failed");
  }
  b->cap = cap;
  return SYNX_OK;
}

// Restores each context's own stream when the batch step ends.
struct StreamSwap {
  std::vector<std::pair<synx_ctx*, cudaStream_t>> saved;
  ~StreamSwap() {
    for (auto& p : saved) p.first->stream = p.second;
  }
};

// One batch step: every context with a level left runs its next level.  Levels that the level
// kernel serves share cooperative launches (one per dimension and CC radius); the others run
// their own per-kernel path on the same stream.  One host synchronisation for the whole step.
int batch_step(synx_batch* b, synx_ctx* const* cs, int n, cudaStream_t s, int* advanced) {
  synx::NvtxRange range("synx batch step", n);
  if (advanced) *advanced = 0;
  if (!b || (n > 0 && !cs) || n < 0) return batch_err(b, SYNX_E_ARG, "synx_batch_step: bad arguments");
  std::vector<synx_ctx*> act;
  for (int i = 0; i < n; ++i) {
    synx_ctx* c = cs[i];
    if (!c) return batch_err(b, SYNX_E_ARG, "synx_batch_step: null context");
    if (c->device != b->device) return batch_err(b, SYNX_E_ARG, "synx_batch_step: context on another device");
    if (!c->images_set) return batch_err(b, SYNX_E_STATE, "synx_batch_step: images not set");
    if (std::find(act.begin(), act.end(), c) != act.end())
      return batch_err(b, SYNX_E_ARG, "synx_batch_step: a context appears twice");
    if (c->cur_level + 1 < c->P.n_levels) act.push_back(c);
  }
  if (act.empty()) return SYNX_OK;
  if (cudaSetDevice(b->device) != cudaSuccess) return batch_err(b, SYNX_E_CUDA, "synx_batch_step: cudaSetDevice");
  StreamSwap swap;
  for (synx_ctx* c : act) {
    if (c->stream != s) {
      // work already queued on the context's own stream comes first
      if (cudaEventRecord(b->ev, c->stream) != cudaSuccess || cudaStreamWaitEvent(s, b->ev, 0) != cudaSuccess)
        return batch_err(b, SYNX_E_CUDA, "synx_batch_step: stream ordering failed");
    }
    swap.saved.push_back({c, c->stream});
    c->stream = s;
  }
  auto fail = [&](synx_ctx* c, int rc) { return batch_err(b, rc, c->err); };
  for (synx_ctx* c : act) {
    const int rc = level_begin(c, c->cur_level + 1);
    if (rc) return fail(c, rc);
  }
  // group the levels the level kernel serves by (dimension, CC radius)
  std::vector<synx_ctx*> rest;
  std::vector<std::vector<synx_ctx*>> groups;
  for (synx_ctx* c : act) {
    const int l = c->cur_level;
    const bool profile = (c->P.flags & SYNX_F_PROFILE_EVENTS) != 0;
    if (c->P.iterations[l] > 0 && persistent_eligible(c, c->lv[l], profile)) {
      bool placed = false;
      for (auto& g : groups)
        if (g[0]->D == c->D && g[0]->P.cc_radius == c->P.cc_radius) {
          g.push_back(c);
          placed = true;
          break;
        }
      if (!placed) groups.push_back({c});
    } else {
      rest.push_back(c);
    }
  }
  for (auto& grp : groups) {
    const int D = grp[0]->D, rcc = grp[0]->P.cc_radius;
    const int Gmax = level_batch_max_blocks(D, rcc, b->device);
    if (Gmax <= 0) {
      for (synx_ctx* c : grp) rest.push_back(c);
      continue;
    }
    for (size_t at = 0; at < grp.size(); at += (size_t)Gmax) {
      const int m = (int)std::min(grp.size() - at, (size_t)Gmax);
      int rc = batch_reserve(b, m);
      if (rc) return rc;
      b->h_args.resize(m);
      b->h_first.assign(m + 1, 0);
      std::vector<double> w(m);
      for (int i = 0; i < m; ++i) {
        synx_ctx* c = grp[at + i];
        const int l = c->cur_level;
        b->h_args[i] = make_level_args(c, c->lv[l], c->P.iterations[l]);
        w[i] = (double)c->lv[l].d.N * c->P.iterations[l];
      }
      const std::vector<int> gsz = split_blocks(w, Gmax);
      for (int i = 0; i < m; ++i) b->h_first[i + 1] = b->h_first[i] + gsz[i];
      if (cudaMemcpyAsync(b->d_args, b->h_args.data(), sizeof(LevelArgs) * m, cudaMemcpyHostToDevice, s) !=
              cudaSuccess ||
          cudaMemcpyAsync(b->d_first, b->h_first.data(), sizeof(int) * (m + 1), cudaMemcpyHostToDevice, s) !=
              cudaSuccess)
        return batch_err(b, SYNX_E_CUDA, "synx_batch_step: argument upload failed");
      BatchLevelArgs B{b->d_args, b->d_first, m};
      const cudaError_t e = launch_level_batch(B, D, rcc, b->h_first[m], s);
      if (e != cudaSuccess)
        return batch_err(b, SYNX_E_CUDA, std::string("synx_batch_step: batched level launch: ") + cudaGetErrorString(e));
    }
  }
  if (!rest.empty()) {
    // fork: every lane waits for the set-up enqueued on s, runs its pairs' levels, and s joins
    const int L = (int)std::min(b->lanes.size(), rest.size());
    if (L > 1) {
      if (cudaEventRecord(b->ev, s) != cudaSuccess) return batch_err(b, SYNX_E_CUDA, "synx_batch_step: fork");
      for (int l = 0; l < L; ++l)
        if (cudaStreamWaitEvent(b->lanes[l], b->ev, 0) != cudaSuccess)
          return batch_err(b, SYNX_E_CUDA, "synx_batch_step: fork");
    }
    for (size_t i = 0; i < rest.size(); ++i) {
      synx_ctx* c = rest[i];
      if (L > 1) c->stream = b->lanes[i % L];
      const int rc = level_iterate(c, c->cur_level);
      c->stream = s;
      if (rc) return fail(c, rc);
    }
    if (L > 1)
      for (int l = 0; l < L; ++l)
        if (cudaEventRecord(b->lane_ev[l], b->lanes[l]) != cudaSuccess ||
            cudaStreamWaitEvent(s, b->lane_ev[l], 0) != cudaSuccess)
          return batch_err(b, SYNX_E_CUDA, "synx_batch_step: join");
  }
  for (synx_ctx* c : act) {
    const int rc = level_readback(c, c->cur_level);
    if (rc) return fail(c, rc);
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) {
    const std::string m = cudaGetErrorString(cudaGetLastError());
    return batch_err(b, SYNX_E_CUDA, "synx_batch_step: " + m);
  }
  for (synx_ctx* c : act) {
    const int rc = level_finish(c, c->cur_level);
    if (rc) return fail(c, rc);
  }
  if (advanced) *advanced = (int)act.size();
  return SYNX_OK;
}

}  // namespace

int synx::set_global_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

extern "C" {

int synx_params_default(synx_params* p, int dim) {
  if (!p) return set_err(nullptr, SYNX_E_ARG, "synx_params_default: null");
  if (dim != 2 && dim != 3) return set_err(nullptr, SYNX_E_ARG, "synx_params_default: dim must be 2 or 3");
  memset(p, 0, sizeof(*p));
  p->dim = dim;
  p->n_levels = 1;
  p->learning_rate = 0.1;
  p->update_variance = 3.0;
  p->total_variance = 0.0;
  p->cc_radius = 4;
  p->sigmas_in_mm = 0;
  p->iterations[0] = 1;
  p->shrink_factors[0] = 1;
  p->smoothing_sigmas[0] = 0.0;
  p->convergence_threshold = 1e-6;
  p->convergence_window = 10;
  p->preprocess = 1;
  p->winsor_lower = 0.0f;
  p->winsor_upper = 1.0f;
  p->inv_max_iter = 20;
  p->inv_mean_tol = 0.001;
  p->inv_max_tol = 0.1;
  p->flags = 0;
  return SYNX_OK;
}

const char* synx_last_error(const synx_ctx* ctx) {
  if (ctx) return ctx->err.c_str();
  return g_last_error.c_str();
}

int synx_create(const synx_params* params, int device, void* cuda_stream, synx_ctx** out) {
  if (!params || !out) return set_err(nullptr, SYNX_E_ARG, "synx_create: null argument");
  *out = nullptr;
  const synx_params& p = *params;
  if (p.dim != 2 && p.dim != 3) return set_err(nullptr, SYNX_E_ARG, "synx_create: dim must be 2 or 3");
  if (p.n_levels < 1 || p.n_levels > SYNX_MAX_LEVELS)
    return set_err(nullptr, SYNX_E_ARG, "synx_create: n_levels must be in 1..8");
  for (int l = 0; l < p.n_levels; ++l) {
    if (p.iterations[l] < 0) return set_err(nullptr, SYNX_E_ARG, "synx_create: negative iteration count");
    if (p.shrink_factors[l] < 1) return set_err(nullptr, SYNX_E_ARG, "synx_create: shrink factors must be >= 1");
    if (p.smoothing_sigmas[l] < 0) return set_err(nullptr, SYNX_E_ARG, "synx_create: negative smoothing sigma");
  }
  if (!cc_radius_supported(p.dim, p.cc_radius))
    return set_err(nullptr, SYNX_E_UNSUPPORTED, "synx_create: CC radius must be in 1..7");
  if (!(p.learning_rate > 0)) return set_err(nullptr, SYNX_E_ARG, "synx_create: learning rate must be > 0");
  if (p.convergence_window < 2 || p.convergence_window > kMaxWindow)
    return set_err(nullptr, SYNX_E_ARG, "synx_create: convergence window must be in 2..64");
  if (p.inv_max_iter < 1 || p.inv_max_iter > 1000)
    return set_err(nullptr, SYNX_E_ARG, "synx_create: inverse iteration cap must be in 1..1000");
  if (p.update_variance < 0 || p.total_variance < 0)
    return set_err(nullptr, SYNX_E_ARG, "synx_create: negative smoothing variance");
  if (p.test_inject != 0 && p.test_inject != SYNX_INJECT_BARRIER_TIMEOUT && p.test_inject != SYNX_INJECT_ALLOC_FAILURE)
    return set_err(nullptr, SYNX_E_ARG, "synx_create: unknown test_inject value");
  if (p.histogram_match != 0 && p.histogram_match != 1)
    return set_err(nullptr, SYNX_E_ARG, "synx_create: histogram_match must be 0 or 1");
  if (p.tuning != 0 && p.tuning != 1) return set_err(nullptr, SYNX_E_ARG, "synx_create: tuning must be 0 or 1");
  if (p.smooth_tile_rows != 0 && p.smooth_tile_rows != 8 && p.smooth_tile_rows != 16 &&
      (p.smooth_tile_rows < -3 || p.smooth_tile_rows > -1))
    return set_err(nullptr, SYNX_E_ARG, "synx_create: smooth_tile_rows must be 0, 8, 16, -1, -2 or -3");
  if (p.cc_z_chunks < 0 || p.cc_z_chunks > 4096)
    return set_err(nullptr, SYNX_E_ARG, "synx_create: cc_z_chunks must be in 0..4096");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_err(nullptr, SYNX_E_CUDA, "synx_create: no CUDA device");
  }
  if (device < 0 || device >= ndev) return set_err(nullptr, SYNX_E_ARG, "synx_create: bad device index");
  synx_ctx* c = new synx_ctx();
  c->P = p;
  c->D = p.dim;
  c->device = device;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete c;
    return set_err(nullptr, SYNX_E_CUDA, "synx_create: cudaSetDevice failed");
  }
  if (cuda_stream) {
    c->stream = (cudaStream_t)cuda_stream;
  } else {
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete c;
      return set_err(nullptr, SYNX_E_CUDA, "synx_create: stream creation failed");
    }
    c->own_stream = true;
  }
  if (p.tuning == 0) tuning_ensure_loaded();
  cudaError_t e = cc_prepare(p.dim, p.cc_radius);
  if (e == cudaSuccess) e = smooth3_prepare();
  for (auto& ev : c->lev_ev)
    if (e == cudaSuccess) e = cudaEventCreate(&ev);
  if (e != cudaSuccess) {
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return set_err(nullptr, SYNX_E_CUDA, std::string("synx_create: CC kernel setup: ") + cudaGetErrorString(e));
  }
  *out = c;
  return SYNX_OK;
}

int synx_destroy(synx_ctx* ctx) {
  if (!ctx) return SYNX_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_arena(ctx);
  if (ctx->maskF) cudaFree(ctx->maskF);
  if (ctx->maskM) cudaFree(ctx->maskM);
  if (ctx->init_half) cudaFree(ctx->init_half);
  for (auto e : ctx->ev_pool) cudaEventDestroy(e);
  for (auto e : ctx->lev_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->aux) cudaStreamDestroy(ctx->aux);
  delete ctx;
  return SYNX_OK;
}

static int set_images_common(synx_ctx* c, const float* F, const synx_geom* gf, const float* M, const synx_geom* gm,
                             cudaMemcpyKind kind) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  if (!F || !M) return set_err(c, SYNX_E_ARG, "synx_set_images: null image pointer");
  if (!check_geom(gf, c->D) || !check_geom(gm, c->D))
    return set_err(c, SYNX_E_ARG, "synx_set_images: image geometry does not match the stage dimension or is invalid");
  CUDA_TRY(c, cudaSetDevice(c->device));
  if (memcmp(&c->geF, gf, sizeof(synx_geom)) != 0 || memcmp(&c->geM, gm, sizeof(synx_geom)) != 0) drop_graphs(c);
  c->geF = *gf;
  c->geM = *gm;
  geom_to_grid(c->geF, c->gF);
  geom_to_grid(c->geM, c->gM);
  c->NF = c->gF.d.N;
  c->NM = c->gM.d.N;
  int rc = build_levels(c);
  if (rc) return rc;
  rc = allocate(c);
  if (rc) return rc;
  CUDA_TRY(c, cudaMemcpyAsync(c->F0, F, 4 * c->NF, kind, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->M0, M, 4 * c->NM, kind, c->stream));
  if (c->P.preprocess) {
    rc = preprocess(c, c->F0, c->NF);
    if (rc) return rc;
    rc = preprocess(c, c->M0, c->NM);
    if (rc) return rc;
  }
  if (c->P.histogram_match) {
    rc = histogram_match_dev(c, c->M0, c->NM, c->F0, c->NF, 256, 12, true, c->M0, c->hist, c->stream);
    if (rc) return rc;
  }
  c->images_set = true;
  c->cur_level = -1;
  c->log_level.clear();
  c->log_iter.clear();
  c->log_metric.clear();
  c->log_conv.clear();
  c->log_inv.clear();
  CUDA_TRY(c, cudaGetLastError());
  return SYNX_OK;
}

int synx_set_masks(synx_ctx* c, const float* fixed_mask, const synx_geom* gfm, const float* moving_mask,
                   const synx_geom* gmm) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  if ((fixed_mask && !check_geom(gfm, c->D)) || (moving_mask && !check_geom(gmm, c->D)))
    return set_err(c, SYNX_E_ARG, "synx_set_masks: mask geometry does not match the stage dimension or is invalid");
  CUDA_TRY(c, cudaSetDevice(c->device));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  auto upload = [&](const float* m, const synx_geom* gm, unsigned char** dst, GridInfo* gi) -> int {
    if (*dst) {
      cudaFree(*dst);
      *dst = nullptr;
    }
    if (!m) return SYNX_OK;
    geom_to_grid(*gm, *gi);
    const size_t n = (size_t)gi->d.N;
    std::vector<unsigned char> b(n);
    for (size_t i = 0; i < n; ++i) b[i] = m[i] != 0.0f ? 1 : 0;
    cudaError_t e = cudaMalloc((void**)dst, n);
    if (e != cudaSuccess) {
      *dst = nullptr;
      cudaGetLastError();
      return set_err(c, SYNX_E_NOMEM, std::string("synx_set_masks: ") + cudaGetErrorString(e));
    }
    // on the context's stream, which does not synchronise with the legacy default stream: a plain
    // cudaMemcpy from pageable memory may return before its data reach the device
    CUDA_TRY(c, cudaMemcpyAsync(*dst, b.data(), n, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));  // b is released on return
    return SYNX_OK;
  };
  int rc = upload(fixed_mask, gfm, &c->maskF, &c->gmF);
  if (!rc) rc = upload(moving_mask, gmm, &c->maskM, &c->gmM);
  drop_graphs(c);  // the iteration's launches change with the masks
  return rc;
}

int synx_set_initial_half_fields(synx_ctx* c, const float* phi_f, const float* psi_f, const float* phi_m,
                                 const float* psi_m, const synx_geom* grid) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  const int given = (phi_f != nullptr) + (psi_f != nullptr) + (phi_m != nullptr) + (psi_m != nullptr);
  if (given != 0 && given != 4)
    return set_err(c, SYNX_E_ARG, "synx_set_initial_half_fields: give all four half-fields or none");
  if (given == 4 && !check_geom(grid, c->D))
    return set_err(c, SYNX_E_ARG, "synx_set_initial_half_fields: grid does not match the stage dimension or is invalid");
  if (c->cur_level >= 0 && c->cur_level + 1 < c->P.n_levels)
    return set_err(c, SYNX_E_STATE, "synx_set_initial_half_fields: a run is in progress");
  CUDA_TRY(c, cudaSetDevice(c->device));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (c->init_half) {
    cudaFree(c->init_half);
    c->init_half = nullptr;
  }
  if (given == 0) return SYNX_OK;
  geom_to_grid(*grid, c->init_grid);
  const size_t n = (size_t)c->D * c->init_grid.d.N;
  float* inter = nullptr;
  cudaError_t e = cudaMalloc((void**)&c->init_half, 4 * 4 * n);
  if (e == cudaSuccess) e = cudaMalloc((void**)&inter, 4 * n);
  if (e != cudaSuccess) {
    if (c->init_half) cudaFree(c->init_half);
    c->init_half = nullptr;
    cudaGetLastError();
    return set_err(c, SYNX_E_NOMEM, std::string("synx_set_initial_half_fields: ") + cudaGetErrorString(e));
  }
  const float* src[4] = {phi_f, psi_f, phi_m, psi_m};
  for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
    // the copy on the context's stream, ordered before the kernel that reads it (a plain cudaMemcpy from
    // pageable memory may return before its data reach the device, and this stream does not
    // synchronise with the legacy default stream)
    e = cudaMemcpyAsync(inter, src[k], 4 * n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
      launch_deinterleave(inter, c->init_half + k * n, c->init_grid.d.N, c->D, c->stream);
      e = cudaStreamSynchronize(c->stream);
    }
  }
  cudaFree(inter);
  if (e != cudaSuccess) {
    cudaFree(c->init_half);
    c->init_half = nullptr;
    return set_err(c, SYNX_E_CUDA, std::string("synx_set_initial_half_fields: ") + cudaGetErrorString(e));
  }
  return SYNX_OK;
}

int synx_set_images(synx_ctx* c, const float* F, const synx_geom* gf, const float* M, const synx_geom* gm) {
  return set_images_common(c, F, gf, M, gm, cudaMemcpyHostToDevice);
}
int synx_set_images_device(synx_ctx* c, const float* F, const synx_geom* gf, const float* M, const synx_geom* gm) {
  return set_images_common(c, F, gf, M, gm, cudaMemcpyDeviceToDevice);
}

int synx_run_level(synx_ctx* c, int level) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  return run_level_impl(c, level);
}

int synx_footprint(const synx_params* p, const synx_geom* fixed_geom, const synx_geom* moving_geom, int64_t* bytes) {
  if (!p || !fixed_geom || !moving_geom || !bytes) return set_err(nullptr, SYNX_E_ARG, "synx_footprint: null argument");
  if (p->dim != 2 && p->dim != 3) return set_err(nullptr, SYNX_E_ARG, "synx_footprint: dim must be 2 or 3");
  if (p->n_levels < 1 || p->n_levels > SYNX_MAX_LEVELS)
    return set_err(nullptr, SYNX_E_ARG, "synx_footprint: n_levels must be in 1..8");
  for (int l = 0; l < p->n_levels; ++l)
    if (p->shrink_factors[l] < 1) return set_err(nullptr, SYNX_E_ARG, "synx_footprint: shrink factors must be >= 1");
  if (!check_geom(fixed_geom, p->dim) || !check_geom(moving_geom, p->dim))
    return set_err(nullptr, SYNX_E_ARG, "synx_footprint: invalid geometry");
  synx_ctx c;
  c.P = *p;
  c.D = p->dim;
  c.geF = *fixed_geom;
  c.geM = *moving_geom;
  geom_to_grid(c.geF, c.gF);
  geom_to_grid(c.geM, c.gM);
  c.NF = c.gF.d.N;
  c.NM = c.gM.d.N;
  build_levels(&c);
  *bytes = (int64_t)arena_plan(&c).total;
  return SYNX_OK;
}

int synx_batch_create(int device, synx_batch** out) {
  if (!out) return set_err(nullptr, SYNX_E_ARG, "synx_batch_create: null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_err(nullptr, SYNX_E_CUDA, "synx_batch_create: no CUDA device");
  }
  if (device < 0 || device >= ndev) return set_err(nullptr, SYNX_E_ARG, "synx_batch_create: bad device index");
  if (cudaSetDevice(device) != cudaSuccess) return set_err(nullptr, SYNX_E_CUDA, "synx_batch_create: cudaSetDevice");
  synx_batch* b = new synx_batch();
  b->device = device;
  bool lanes_ok = true;
  for (int l = 0; l < kBatchLanes && lanes_ok; ++l) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    lanes_ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess &&
               cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
    if (st) b->lanes.push_back(st);
    if (ev) b->lane_ev.push_back(ev);
  }
  if (!lanes_ok || cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess) {
    for (auto st : b->lanes) cudaStreamDestroy(st);
    for (auto ev : b->lane_ev) cudaEventDestroy(ev);
    delete b;
    return set_err(nullptr, SYNX_E_CUDA, "synx_batch_create: event creation failed");
  }
  *out = b;
  return SYNX_OK;
}

int synx_batch_destroy(synx_batch* b) {
  if (!b) return SYNX_OK;
  cudaSetDevice(b->device);
  if (b->d_args) cudaFree(b->d_args);
  if (b->d_first) cudaFree(b->d_first);
  if (b->ev) cudaEventDestroy(b->ev);
  for (auto st : b->lanes) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (auto ev : b->lane_ev) cudaEventDestroy(ev);
  delete b;
  return SYNX_OK;
}

const char* synx_batch_last_error(const synx_batch* b) { return b ? b->err.c_str() : g_last_error.c_str(); }

int synx_batch_step(synx_batch* b, synx_ctx* const* ctxs, int n, void* cuda_stream, int* advanced) {
  return batch_step(b, ctxs, n, (cudaStream_t)cuda_stream, advanced);
}

int synx_batch_run(synx_batch* b, synx_ctx* const* ctxs, int n, void* cuda_stream) {
  for (;;) {
    int adv = 0;
    const int rc = batch_step(b, ctxs, n, (cudaStream_t)cuda_stream, &adv);
    if (rc) return rc;
    if (adv == 0) return SYNX_OK;
  }
}

int synx_run(synx_ctx* c) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  if (!c->images_set) return set_err(c, SYNX_E_STATE, "synx_run: images not set");
  for (int l = c->cur_level + 1; l < c->P.n_levels; ++l) {
    int rc = run_level_impl(c, l);
    if (rc) return rc;
  }
  return SYNX_OK;
}

int synx_get_output_geom(const synx_ctx* c, synx_geom* out) {
  if (!valid_ctx(c) || !out) return set_err(nullptr, SYNX_E_ARG, "synx_get_output_geom: null argument");
  if (c->cur_level < 0) return set_err(const_cast<synx_ctx*>(c), SYNX_E_STATE, "no level has run");
  *out = c->lgeom[c->cur_level];
  return SYNX_OK;
}

static int final_fields(synx_ctx* c, float* fwd_planes, float* inv_planes) {
  const GridInfo& g = c->cur_grid;
  {
    const float* d[1] = {c->psiM};
    const float* w[1] = {c->phiF};
    float* o[1] = {fwd_planes};
    launch_compose(d, w, o, 1, g, -1.0f, nullptr, c->stream);
  }
  {
    const float* d[1] = {c->psiF};
    const float* w[1] = {c->phiM};
    float* o[1] = {inv_planes};
    launch_compose(d, w, o, 1, g, -1.0f, nullptr, c->stream);
  }
  return SYNX_OK;
}

static int get_fields_common(synx_ctx* c, float* fwd, float* inv, bool host) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  if (c->cur_level < 0) return set_err(c, SYNX_E_STATE, "synx_get_fields: no level has run");
  CUDA_TRY(c, cudaSetDevice(c->device));
  const GridInfo& g = c->cur_grid;
  const size_t n = (size_t)c->D * g.d.N;
  // final composition into work buffers, then interleave
  final_fields(c, c->t2F, c->t2M);
  launch_interleave(c->t2F, c->gFu, g.d.N, c->D, c->stream);
  launch_interleave(c->t2M, c->gMu, g.d.N, c->D, c->stream);
  const cudaMemcpyKind kind = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  if (fwd) CUDA_TRY(c, cudaMemcpyAsync(fwd, c->gFu, 4 * n, kind, c->stream));
  if (inv) CUDA_TRY(c, cudaMemcpyAsync(inv, c->gMu, 4 * n, kind, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return SYNX_OK;
}

int synx_get_fields(synx_ctx* c, float* fwd, float* inv) { return get_fields_common(c, fwd, inv, true); }
int synx_get_fields_device(synx_ctx* c, float* fwd, float* inv) { return get_fields_common(c, fwd, inv, false); }

int synx_get_half_fields(synx_ctx* c, float* phi_f, float* psi_f, float* phi_m, float* psi_m) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  if (c->cur_level < 0) return set_err(c, SYNX_E_STATE, "synx_get_half_fields: no level has run");
  CUDA_TRY(c, cudaSetDevice(c->device));
  const GridInfo& g = c->cur_grid;
  const size_t n = (size_t)c->D * g.d.N;
  float* outs[4] = {phi_f, psi_f, phi_m, psi_m};
  const float* srcs[4] = {c->phiF, c->psiF, c->phiM, c->psiM};
  for (int k = 0; k < 4; ++k) {
    if (!outs[k]) continue;
    launch_interleave(srcs[k], c->t2F, g.d.N, c->D, c->stream);
    CUDA_TRY(c, cudaMemcpyAsync(outs[k], c->t2F, 4 * n, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  return SYNX_OK;
}

int synx_set_half_fields(synx_ctx* c, const float* phi_f, const float* psi_f, const float* phi_m, const float* psi_m,
                         const synx_geom* grid) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  if (!c->images_set) return set_err(c, SYNX_E_STATE, "synx_set_half_fields: images not set");
  if (!phi_f || !psi_f || !phi_m || !psi_m || !check_geom(grid, c->D))
    return set_err(c, SYNX_E_ARG, "synx_set_half_fields: bad arguments");
  // the grid must be one of the level grids; the next level to run is the one after it
  int lvl = -1;
  for (int l = 0; l < (int)c->lgeom.size(); ++l) {
    const synx_geom& g = c->lgeom[l];
    bool same = true;
    for (int d = 0; d < 3; ++d) same = same && g.size[d] == grid->size[d];
    if (same) {
      lvl = l;
      break;
    }
  }
  if (lvl < 0) return set_err(c, SYNX_E_ARG, "synx_set_half_fields: grid is not a level grid of this stage");
  CUDA_TRY(c, cudaSetDevice(c->device));
  const GridInfo& g = c->lv[lvl];
  const size_t n = (size_t)c->D * g.d.N;
  const float* ins[4] = {phi_f, psi_f, phi_m, psi_m};
  float* dsts[4] = {c->phiF, c->psiF, c->phiM, c->psiM};
  for (int k = 0; k < 4; ++k) {
    CUDA_TRY(c, cudaMemcpyAsync(c->t2F, ins[k], 4 * n, cudaMemcpyHostToDevice, c->stream));
    launch_deinterleave(c->t2F, dsts[k], g.d.N, c->D, c->stream);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  c->cur_grid = g;
  c->cur_level = lvl;
  return SYNX_OK;
}

int synx_get_log(synx_ctx* c, int32_t* level, int32_t* iteration, double* metric, double* convergence,
                 int32_t* inverse_iterations, int64_t capacity, int64_t* count) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  const int64_t n = (int64_t)c->log_metric.size();
  if (count) *count = n;
  for (int64_t i = 0; i < n && i < capacity; ++i) {
    if (level) level[i] = c->log_level[i];
    if (iteration) iteration[i] = c->log_iter[i];
    if (metric) metric[i] = c->log_metric[i];
    if (convergence) convergence[i] = c->log_conv[i];
    if (inverse_iterations) inverse_iterations[i] = c->log_inv[i];
  }
  return SYNX_OK;
}

int synx_get_profile(synx_ctx* c, double* inv_ms, int64_t* inv_launches, int64_t* inv_vox, double* cc_ms,
                     int64_t* cc_launches, int64_t* cc_vox) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  if (inv_ms) *inv_ms = c->prof_inv_ms;
  if (inv_launches) *inv_launches = c->prof_inv_launches;
  if (inv_vox) *inv_vox = c->prof_inv_vox;
  if (cc_ms) *cc_ms = c->prof_cc_ms;
  if (cc_launches) *cc_launches = c->prof_cc_launches;
  if (cc_vox) *cc_vox = c->prof_cc_vox;
  return SYNX_OK;
}

int synx_reset_profile(synx_ctx* c) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  c->prof_inv_ms = c->prof_cc_ms = 0;
  c->prof_inv_launches = c->prof_inv_vox = c->prof_cc_launches = c->prof_cc_vox = 0;
  for (auto& l : c->lprof) l = LevelProf();
  return SYNX_OK;
}

int synx_get_level_profile(synx_ctx* c, int level, double* setup_ms, double* iterate_ms, double* inverse_ms,
                           double* cc_ms, int64_t* iterations, int64_t* inverse_subiterations, int64_t* voxels) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  if (level < 0 || level >= SYNX_MAX_LEVELS) return set_err(c, SYNX_E_ARG, "synx_get_level_profile: bad level");
  const LevelProf& l = c->lprof[level];
  if (setup_ms) *setup_ms = l.setup_ms;
  if (iterate_ms) *iterate_ms = l.iterate_ms;
  if (inverse_ms) *inverse_ms = l.inv_ms;
  if (cc_ms) *cc_ms = l.cc_ms;
  if (iterations) *iterations = l.iterations;
  if (inverse_subiterations) *inverse_subiterations = l.inv_sub;
  if (voxels) *voxels = l.voxels;
  return SYNX_OK;
}

int synx_level_plan(synx_ctx* c, int level, int32_t* persistent, int32_t* smooth_rows, int32_t* cc_z_chunks) {
  if (!valid_ctx(c)) return set_err(nullptr, SYNX_E_ARG, "null context");
  if (!c->images_set) return set_err(c, SYNX_E_STATE, "synx_level_plan: images not set");
  if (level < 0 || level >= c->P.n_levels) return set_err(c, SYNX_E_ARG, "synx_level_plan: bad level");
  CUDA_TRY(c, cudaSetDevice(c->device));
  // the smoothing radii of that level decide eligibility: computed as level_begin would
  const int saved[3] = {c->R_upd[0], c->R_upd[1], c->R_upd[2]};
  const GridInfo& g = c->lv[level];
  for (int a = 0; a < c->D; ++a) {
    const int n = a == 0 ? g.d.nx : (a == 1 ? g.d.ny : g.d.nz);
    c->R_upd[a] = (int)gauss_kernel(c->P.update_variance, 0.001, (size_t)n).size() / 2;
  }
  const LevelPlan p = resolve_plan(c, level);
  const LevelPlan keep = c->plan[level];
  c->plan[level] = p;
  int blocks = 0;
  const bool pers = c->P.iterations[level] > 0 &&
                    use_persistent(c, level, g, (c->P.flags & SYNX_F_PROFILE_EVENTS) != 0, &blocks);
  c->plan[level] = keep;
  for (int a = 0; a < 3; ++a) c->R_upd[a] = saved[a];
  if (persistent) *persistent = pers ? 1 : 0;
  if (smooth_rows) *smooth_rows = p.smooth_rows;
  if (cc_z_chunks) *cc_z_chunks = p.cc_chunks;
  return SYNX_OK;
}

int synx_get_launch_count(int64_t* count) {
  if (!count) return set_err(nullptr, SYNX_E_ARG, "synx_get_launch_count: null");
  *count = (int64_t)launch_count();
  return SYNX_OK;
}

int synx_get_device_bytes(const synx_ctx* c, int64_t* bytes) {
  if (!valid_ctx(c) || !bytes) return set_err(nullptr, SYNX_E_ARG, "null argument");
  *bytes = (int64_t)c->arena_bytes;
  return SYNX_OK;
}

// ------------------------------------------------------------------------------------------
// Step entry points
// ------------------------------------------------------------------------------------------
int synx_gaussian_kernel(double variance, double max_error, int max_width, double* coeffs, int cap, int* len) {
  if (max_width < 1 || !(max_error > 0) || max_error >= 1)
    return set_err(nullptr, SYNX_E_ARG, "synx_gaussian_kernel: bad arguments");
  auto k = gauss_kernel(variance, max_error, (size_t)max_width);
  if (len) *len = (int)k.size();
  for (int i = 0; i < (int)k.size() && i < cap && coeffs; ++i) coeffs[i] = k[i];
  return SYNX_OK;
}

int synx_shrink_geom(const synx_geom* in, int factor, synx_geom* out) {
  if (!in || !out || factor < 1 || (in->dim != 2 && in->dim != 3))
    return set_err(nullptr, SYNX_E_ARG, "synx_shrink_geom: bad arguments");
  *out = shrink(*in, (unsigned)factor);
  return SYNX_OK;
}

namespace {
struct TempCtl {
  IterCtl* ctl = nullptr;
  double* part = nullptr;
  float* pmax = nullptr;
  int cap = 0;
  cudaError_t alloc(int partials) {
    cap = partials;
    cudaError_t e = cudaMalloc((void**)&ctl, sizeof(IterCtl));
    if (e) return e;
    e = cudaMalloc((void**)&part, 8 * 2 * (size_t)std::max(partials, 1));
    if (e) return e;
    e = cudaMalloc((void**)&pmax, 4 * 2 * (size_t)std::max(partials, 1));
    return e;
  }
  ~TempCtl() {
    if (ctl) cudaFree(ctl);
    if (part) cudaFree(part);
    if (pmax) cudaFree(pmax);
  }
};
}  // namespace

#define STEP_TRY(call)                                                                              \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess)                                                                          \
      return set_err(nullptr, SYNX_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

int synx_smooth_image(const float* in, float* out, const synx_geom* gg, double sigma, int mm, void* stream) {
  if (!in || !out || !gg || (gg->dim != 2 && gg->dim != 3) || !check_geom(gg, gg->dim) || sigma < 0)
    return set_err(nullptr, SYNX_E_ARG, "synx_smooth_image: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  GridInfo g;
  geom_to_grid(*gg, g);
  if (sigma == 0.0) {
    STEP_TRY(cudaMemcpyAsync(out, in, 4 * g.d.N, cudaMemcpyDeviceToDevice, s));
    return SYNX_OK;
  }
  double* dk = nullptr;
  float* tmp = nullptr;
  STEP_TRY(cudaMalloc((void**)&dk, 8 * 3 * 64));
  STEP_TRY(cudaMalloc((void**)&tmp, 4 * g.d.N));
  std::vector<double> hk(3 * 64, 0.0);
  int R[3] = {0, 0, 0};
  for (int a = 0; a < gg->dim; ++a) {
    double var = sigma * sigma;
    if (mm) var /= g.sp[a] * g.sp[a];
    auto k = gauss_kernel(var, 0.01, 32);
    R[a] = (int)k.size() / 2;
    for (size_t j = 0; j < k.size(); ++j) hk[a * 64 + j] = k[j];
  }
  STEP_TRY(cudaMemcpyAsync(dk, hk.data(), 8 * 3 * 64, cudaMemcpyHostToDevice, s));
  const float* src = in;
  const int D = gg->dim;
  for (int p = 0; p < D; ++p) {
    const int axis = D - 1 - p;
    float* o = ((D - 1 - p) % 2 == 0) ? out : tmp;
    launch_conv_image_axis(src, o, g, axis, dk + axis * 64, R[axis], s);
    src = o;
  }
  STEP_TRY(cudaStreamSynchronize(s));
  cudaFree(dk);
  cudaFree(tmp);
  STEP_TRY(cudaGetLastError());
  return SYNX_OK;
}

int synx_warp_image(const float* img, const synx_geom* gi, const float* u, const synx_geom* gv, float* out,
                    void* stream) {
  if (!img || !u || !out || !gi || !gv || !check_geom(gi, gi->dim) || !check_geom(gv, gi->dim))
    return set_err(nullptr, SYNX_E_ARG, "synx_warp_image: bad arguments");
  GridInfo a, b;
  geom_to_grid(*gi, a);
  geom_to_grid(*gv, b);
  launch_warp_image(img, a, u, b, out, (cudaStream_t)stream);
  STEP_TRY(cudaGetLastError());
  return SYNX_OK;
}

int synx_warp_image_nearest(const float* img, const synx_geom* gi, const float* u, const synx_geom* gv, float* out,
                            void* stream) {
  if (!img || !u || !out || !gi || !gv || !check_geom(gi, gi->dim) || !check_geom(gv, gi->dim))
    return set_err(nullptr, SYNX_E_ARG, "synx_warp_image_nearest: bad arguments");
  GridInfo a, b;
  geom_to_grid(*gi, a);
  geom_to_grid(*gv, b);
  launch_warp_image_nearest(img, a, u, b, out, (cudaStream_t)stream);
  STEP_TRY(cudaGetLastError());
  return SYNX_OK;
}

int synx_warp_image_label(const float* img, const synx_geom* gi, const float* u, const synx_geom* gv, float* out,
                          void* stream) {
  if (!img || !u || !out || !gi || !gv || !check_geom(gi, gi->dim) || !check_geom(gv, gi->dim))
    return set_err(nullptr, SYNX_E_ARG, "synx_warp_image_label: bad arguments");
  GridInfo a, b;
  geom_to_grid(*gi, a);
  geom_to_grid(*gv, b);
  launch_warp_image_label(img, a, u, b, out, (cudaStream_t)stream);
  STEP_TRY(cudaGetLastError());
  return SYNX_OK;
}

int synx_histogram_match(const float* src, int64_t n_src, const float* ref, int64_t n_ref, int32_t levels,
                         int32_t match_points, int32_t threshold_at_mean, float* out, void* stream) {
  if (!src || !ref || !out || n_src < 1 || n_ref < 1 || levels < 1 || levels > 4096 || match_points < 1 ||
      match_points > HM_MAX_POINTS || (threshold_at_mean != 0 && threshold_at_mean != 1))
    return set_err(nullptr, SYNX_E_ARG, "synx_histogram_match: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  void* scratch = nullptr;
  STEP_TRY(cudaMalloc(&scratch, hm_scratch_bytes(levels)));
  const int rc = histogram_match_dev(nullptr, src, n_src, ref, n_ref, levels, match_points, threshold_at_mean != 0, out,
                                     scratch, s);
  cudaStreamSynchronize(s);
  cudaFree(scratch);
  return rc;
}

int synx_field_affine_update(const float* u, const float* w, const synx_geom* g, const double* matrix, float* out,
                             void* stream) {
  if (!u || !w || !out || !g || !matrix || !check_geom(g, g->dim))
    return set_err(nullptr, SYNX_E_ARG, "synx_field_affine_update: bad arguments");
  launch_field_affine_update(u, w, matrix, g->dim, g->size[0] * g->size[1] * g->size[2], out, (cudaStream_t)stream);
  STEP_TRY(cudaGetLastError());
  return SYNX_OK;
}

int synx_cc_metric(const float* F, const float* M, const synx_geom* gg, int radius, float* gF, float* gM,
                   double* value, void* stream) {
  return synx_cc_metric_ex(F, M, gg, radius, 0, gF, gM, value, stream);
}

int synx_cc_metric_masked(const float* F, const float* M, const uint8_t* valid, const synx_geom* gg, int radius,
                          float* gF, float* gM, double* value, void* stream) {
  if (!F || !M || !valid || !gF || !gM || !gg || !check_geom(gg, gg->dim))
    return set_err(nullptr, SYNX_E_ARG, "synx_cc_metric_masked: bad arguments");
  if (!cc_radius_supported(gg->dim, radius))
    return set_err(nullptr, SYNX_E_UNSUPPORTED, "synx_cc_metric_masked: radius");
  cudaStream_t s = (cudaStream_t)stream;
  GridInfo g;
  geom_to_grid(*gg, g);
  STEP_TRY(cc_prepare(gg->dim, radius));
  TempCtl t;
  STEP_TRY(t.alloc(2 * cc_blocks(g, radius)));  // block sums, then block counts
  STEP_TRY(cudaMemsetAsync(t.ctl, 0, sizeof(IterCtl), s));
  launch_cc(F, M, g, radius, gF, gM, t.part, t.ctl, s, nullptr, false, 0, valid);
  IterCtl h;
  STEP_TRY(cudaMemcpyAsync(&h, t.ctl, sizeof(IterCtl), cudaMemcpyDeviceToHost, s));
  STEP_TRY(cudaStreamSynchronize(s));
  if (value) *value = h.metric;
  STEP_TRY(cudaGetLastError());
  return SYNX_OK;
}

int synx_cc_metric_ex(const float* F, const float* M, const synx_geom* gg, int radius, int flags, float* gF, float* gM,
                      double* value, void* stream) {
  if (!F || !M || !gF || !gM || !gg || !check_geom(gg, gg->dim) || (flags & ~SYNX_F_CC_FP32_SUMS))
    return set_err(nullptr, SYNX_E_ARG, "synx_cc_metric: bad arguments");
  if (!cc_radius_supported(gg->dim, radius)) return set_err(nullptr, SYNX_E_UNSUPPORTED, "synx_cc_metric: radius");
  cudaStream_t s = (cudaStream_t)stream;
  GridInfo g;
  geom_to_grid(*gg, g);
  STEP_TRY(cc_prepare(gg->dim, radius));
  TempCtl t;
  STEP_TRY(t.alloc(cc_blocks(g, radius)));
  STEP_TRY(cudaMemsetAsync(t.ctl, 0, sizeof(IterCtl), s));
  launch_cc(F, M, g, radius, gF, gM, t.part, t.ctl, s, nullptr, (flags & SYNX_F_CC_FP32_SUMS) != 0);
  IterCtl h;
  STEP_TRY(cudaMemcpyAsync(&h, t.ctl, sizeof(IterCtl), cudaMemcpyDeviceToHost, s));
  STEP_TRY(cudaStreamSynchronize(s));
  if (value) *value = h.metric;
  STEP_TRY(cudaGetLastError());
  return SYNX_OK;
}

int synx_smooth_field(const float* in, float* out, const synx_geom* gg, double variance, double* max_norm,
                      void* stream) {
  if (!in || !out || !gg || !check_geom(gg, gg->dim) || variance < 0)
    return set_err(nullptr, SYNX_E_ARG, "synx_smooth_field: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  GridInfo g;
  geom_to_grid(*gg, g);
  const int D = gg->dim;
  const size_t n = (size_t)D * g.d.N;
  TempCtl t;
  STEP_TRY(t.alloc(1));
  STEP_TRY(cudaMemsetAsync(t.ctl, 0, sizeof(IterCtl), s));
  float* coeff = nullptr;
  float *ta = nullptr, *tb = nullptr;
  STEP_TRY(cudaMalloc((void**)&coeff, 4 * 3 * 1024));
  STEP_TRY(cudaMalloc((void**)&ta, 4 * n));
  STEP_TRY(cudaMalloc((void**)&tb, 4 * n));
  std::vector<float> hk(3 * 1024, 0.0f);
  int R[3] = {0, 0, 0};
  for (int a = 0; a < D; ++a) {
    const int len = a == 0 ? g.d.nx : (a == 1 ? g.d.ny : g.d.nz);
    auto k = gauss_kernel(variance, 0.001, (size_t)len);
    if (k.size() > 1024) return set_err(nullptr, SYNX_E_UNSUPPORTED, "synx_smooth_field: kernel too wide");
    R[a] = (int)k.size() / 2;
    for (size_t j = 0; j < k.size(); ++j) hk[a * 1024 + j] = (float)k[j];
  }
  STEP_TRY(cudaMemcpyAsync(coeff, hk.data(), 4 * 3 * 1024, cudaMemcpyHostToDevice, s));
  if (variance <= 0.0) {
    const float* i0[1] = {in};
    float* o0[1] = {out};
    launch_smooth_field_pass(i0, o0, nullptr, 1, g, 0, coeff, R[0], false, 1.f, 0.f, true, t.ctl, s);
  } else if (smooth3_supported(D, R)) {
    const float w1 = variance < 0.5 ? (float)(1.0 - variance / 0.5) : 1.0f, w2 = 1.0f - w1;
    STEP_TRY(smooth3_prepare());
    const float* i0[1] = {in};
    float* o0[1] = {out};
    const float* k[3] = {hk.data(), hk.data() + 1024, hk.data() + 2048};
    float* tt[1] = {ta};
    launch_smooth_field(i0, o0, i0, tt, 1, g, k, R, true, w1, w2, true, t.ctl, s);
  } else {
    const float w1 = variance < 0.5 ? (float)(1.0 - variance / 0.5) : 1.0f, w2 = 1.0f - w1;
    const float* orig[1] = {in};
    const float* src = in;
    for (int a = 0; a < D; ++a) {
      const bool last = a == D - 1;
      float* dst = last ? out : (a % 2 == 0 ? ta : tb);
      const float* i0[1] = {src};
      float* o0[1] = {dst};
      launch_smooth_field_pass(i0, o0, last ? orig : nullptr, 1, g, a, coeff + a * 1024, R[a], last, w1, w2, last,
                               t.ctl, s);
      src = dst;
    }
  }
  IterCtl h;
  STEP_TRY(cudaMemcpyAsync(&h, t.ctl, sizeof(IterCtl), cudaMemcpyDeviceToHost, s));
  STEP_TRY(cudaStreamSynchronize(s));
  if (max_norm) {
    float f;
    memcpy(&f, &h.maxnorm[0], 4);
    *max_norm = f;
  }
  cudaFree(coeff);
  cudaFree(ta);
  cudaFree(tb);
  STEP_TRY(cudaGetLastError());
  return SYNX_OK;
}

int synx_compose(const float* d, const float* w, const synx_geom* gg, float scale, float* out, void* stream) {
  if (!d || !w || !out || !gg || !check_geom(gg, gg->dim))
    return set_err(nullptr, SYNX_E_ARG, "synx_compose: bad arguments");
  GridInfo g;
  geom_to_grid(*gg, g);
  const float* dd[1] = {d};
  const float* ww[1] = {w};
  float* oo[1] = {out};
  if (scale == 1.0f) {
    launch_compose(dd, ww, oo, 1, g, -1.0f, nullptr, (cudaStream_t)stream);
  } else {
    // scale via a constant max-norm: maxnorm = 1 / scale with eta = 1 gives scale
    TempCtl t;
    STEP_TRY(t.alloc(1));
    IterCtl h;
    memset(&h, 0, sizeof(h));
    float inv = 1.0f / scale;
    memcpy(&h.maxnorm[0], &inv, 4);
    STEP_TRY(cudaMemcpyAsync(t.ctl, &h, sizeof(IterCtl), cudaMemcpyHostToDevice, (cudaStream_t)stream));
    launch_compose(dd, ww, oo, 1, g, 1.0f, t.ctl, (cudaStream_t)stream);
    STEP_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  }
  STEP_TRY(cudaGetLastError());
  return SYNX_OK;
}

int synx_invert_field(const float* phi, float* psi, const synx_geom* gg, int max_iter, double mean_tol, double max_tol,
                      int* iterations, void* stream) {
  if (!phi || !psi || !gg || !check_geom(gg, gg->dim) || max_iter < 1)
    return set_err(nullptr, SYNX_E_ARG, "synx_invert_field: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  GridInfo g;
  geom_to_grid(*gg, g);
  TempCtl t;
  const int nb = inv_blocks(g);
  STEP_TRY(t.alloc(nb));
  STEP_TRY(cudaMemsetAsync(t.ctl, 0, sizeof(IterCtl), s));
  PartialBufs pb{t.part, t.pmax, nb};
  const float* pp[1] = {phi};
  float* ps[1] = {psi};
  // the single-pass form: residual cache and deferred-voxel list for the one half
  struct Scratch {
    float* ec = nullptr;
    int* list = nullptr;
    ~Scratch() {
      if (ec) cudaFree(ec);
      if (list) cudaFree(list);
    }
  } sc;
  STEP_TRY(cudaMalloc((void**)&sc.ec, 4 * (size_t)g.d.dim * g.d.N));
  STEP_TRY(cudaMalloc((void**)&sc.list, 4 * (size_t)g.d.N));
  float* ecs[1] = {sc.ec};
  int* lists[1] = {sc.list};
  for (int k = 0; k < max_iter; ++k) {
    launch_invert_spec(pp, ps, 1, g, k, max_iter, mean_tol, max_tol, t.ctl, 0, pb, s, true, ecs, lists);
    launch_invert_fix(pp, ps, 1, g, k, max_iter, t.ctl, 0, s, true, ecs, lists);
  }
  IterCtl h;
  STEP_TRY(cudaMemcpyAsync(&h, t.ctl, sizeof(IterCtl), cudaMemcpyDeviceToHost, s));
  STEP_TRY(cudaStreamSynchronize(s));
  if (iterations) *iterations = h.inv[0][0].iters;
  STEP_TRY(cudaGetLastError());
  return SYNX_OK;
}

int synx_resample_field(const float* in, const synx_geom* gi, float* out, const synx_geom* go, void* stream) {
  if (!in || !out || !gi || !go || !check_geom(gi, gi->dim) || !check_geom(go, gi->dim))
    return set_err(nullptr, SYNX_E_ARG, "synx_resample_field: bad arguments");
  GridInfo a, b;
  geom_to_grid(*gi, a);
  geom_to_grid(*go, b);
  const float* ii[1] = {in};
  float* oo[1] = {out};
  launch_resample_fields(ii, a, oo, b, 1, (cudaStream_t)stream);
  STEP_TRY(cudaGetLastError());
  return SYNX_OK;
}

}  // extern "C"
