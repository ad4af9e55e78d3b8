// Host-side launch interface of the synx kernels (C++ linkage, internal to libsynx).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "synx_device.cuh"

namespace synx {

// Programmatic dependent launch.  The kernels of one SyN iteration are launched with programmatic
// stream serialisation when t_pdl is set (the stage sets it while it enqueues an iteration), so a
// kernel's launch and block scheduling overlap the end of the kernel before it; each such kernel
// waits at its start (griddep_wait, before touching global memory) until its predecessor has
// completed and its writes are visible.  Without the attribute the wait returns at once.
extern thread_local int t_pdl;       // launches from this host thread use the attribute
extern thread_local int t_pdl_skip;  // the next launch does not (it follows a graph node that is not a kernel)
// Sweep order of the launches from this host thread that take one (warp, CC, xy and z smoothing,
// composition): 1 = the grid in reverse (see sweep_block).  The z smoothing pass takes the
// opposite of its xy pass.
extern thread_local int t_rev;
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  const bool pdl = t_pdl && !t_pdl_skip;
  t_pdl_skip = 0;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Fixed-point inverse control block, one per (phase, half).  Slot k%2 holds the decision
// and statistics consumed by launch k; launch k writes slot (k+1)%2.
struct InvCtl {
  int exec[2];
  float maxv[2];
  double mean[2];
  int iters;
  unsigned counter;
  int kdev;  // sub-iteration index for launches that read it from the device (graph loop bodies)
  int pad;
  // single-pass form: a running lower bound of the residual maximum (float bits), the deferred
  // voxels' list length, the arrival counter of the deferred-update pass, and per sub-iteration
  // parity the residual maximum the deferred updates clamp against
  unsigned mrun;
  unsigned lcount;
  unsigned fcount;
  float maxk[2];
  int pad2;
};

constexpr int kMaxWindow = 64;

// Device-resident control block of one registration context.
struct IterCtl {
  int stop;                   // 1 once the level converged: iteration kernels return at once
  int iter;                   // iterations completed in the current level
  unsigned maxnorm[2];        // float bits of max ||u / spacing|| per half (fixed, moving)
  unsigned cc_counter;        // block arrival counter of the CC reduction
  int pad0;
  double cc_sum;              // sum of local cc of the last evaluation
  double metric;              // -mean cc of the last evaluation
  double total_abs;           // running sum of |metric| over the level
  double energies[kMaxWindow];
  InvCtl inv[2][2];           // [phase A (psi), phase B (phi)][half]
  unsigned bar_count;         // grid barrier of the persistent level kernel: arrivals,
  unsigned bar_gen;           // generation,
  int bar_err;                // and 1 if a wait gave up, 2 if the launch's shared memory was too
                              // small (the kernel then returns)
  int pad1;
};

struct LogDev {
  double* metric;
  double* conv;
  int* inv_iters;
  int cap;
};

// Geometry helpers (host).
struct GridInfo {
  Dims d;
  double sp[3], org[3], dir[9], i2p[9], p2i[9];
};

GridInfo make_grid(int dim, const int64_t size[3], const double sp[3], const double org[3], const double dir[9]);
// c = t + B i + A u mapping voxel i of `src` displaced by u into continuous index of `dst`.
Affine make_affine(const GridInfo& src, const GridInfo& dst);
// The index part of that map in double (c = t + B i); exact zeros off the diagonal when both
// grids share their direction cosines.
void index_map(const GridInfo& src, const GridInfo& dst, double t[3], double B[9]);

struct PartialBufs {
  double* sum;       // per-block partial sums
  float* maxv;       // per-block partial max
  int capacity;      // entries per half
};

// ---- launchers (all asynchronous on `s`) -----------------------------------------------
void launch_zero_ctl_level(IterCtl* ctl, cudaStream_t s);

void launch_warp_pair(const float* F, const GridInfo& gF, const float* psiF, const float* M, const GridInfo& gM,
                      const float* psiM, const GridInfo& gv, float* Ft, float* Mt, IterCtl* ctl, cudaStream_t s);
void launch_warp_image(const float* img, const GridInfo& gi, const float* u, const GridInfo& gv, float* out,
                       cudaStream_t s);
void launch_warp_image_nearest(const float* img, const GridInfo& gi, const float* u, const GridInfo& gv, float* out,
                               cudaStream_t s);
void launch_warp_image_label(const float* img, const GridInfo& gi, const float* u, const GridInfo& gv, float* out,
                             cudaStream_t s);
// Metric-mask validity (one byte per voxel of gv): both masks, warped nearest-neighbour through
// their half-fields, nonzero; a null mask is inside everywhere.
void launch_mask_validity(const unsigned char* mF, const GridInfo& gmF, const float* psiF, const unsigned char* mM,
                          const GridInfo& gmM, const float* psiM, const GridInfo& gv, unsigned char* valid,
                          IterCtl* ctl, cudaStream_t s);
void launch_field_affine_update(const float* u, const float* w, const double M[9], int dim, long long N, float* out,
                                cudaStream_t s);

// Returns the number of blocks the CC launch uses (partials needed); chunks > 0 fixes the number
// of z chunks (at most nz / radius), 0 takes the cost model's.
int cc_blocks(const GridInfo& g, int radius, int chunks = 0);
// The most blocks any chunk count can give on g.
int cc_blocks_max(const GridInfo& g, int radius);
size_t cc_smem_bytes(int dim, int radius, bool masked = false);
bool cc_radius_supported(int dim, int radius);
// Raise the dynamic shared-memory limit of the CC kernel (once per device, outside capture).
cudaError_t cc_prepare(int dim, int radius);
// fp32_sums: window sums and variance terms in float (the precision study's variant).
// valid (metric masks): one byte per voxel, nonzero = valid; `partials` then needs twice the blocks.
void launch_cc(const float* Ft, const float* Mt, const GridInfo& g, int radius, float* gF, float* gM, double* partials,
               IterCtl* ctl, cudaStream_t s, float* cc_out = nullptr, bool fp32_sums = false, int chunks = 0,
               const unsigned char* valid = nullptr);
// Round nf fields of n floats each to the nearest half-precision value, in place (the
// precision study's FP16 field storage).
void launch_round_half(float* const* f, int nf, long long n, cudaStream_t s);

// Gaussian smoothing of `halves` fields along every axis: an xy-tile kernel and, in 3-D, a
// z-column kernel (host kernels khost[a] of radius R[a] per axis, passed by value in the
// launch parameters).  `epilogue` applies SyN's boundary zeroing and the blend with `orig`
// (w2 != 0); `maxnorm` reduces max ||u/spacing|| into ctl->maxnorm[h].  Radii up to 12.
bool smooth3_supported(int dim, const int R[3]);
cudaError_t smooth3_prepare();
// How a 3-D field is smoothed: slab_ty > 0 runs the fused slab kernel with 32 x slab_ty column
// tiles (8 or 16) and slab_zc output slices per block (0: chosen by a waves x work model);
// slab_ty = 0 runs an xy kernel and then the z kernel through `tmp`.
struct SmoothPlan {
  int slab_ty;
  int slab_zc;
  int xy_ty;  // two-kernel path: 0 = the xy kernel (one slice per block), 32 / 64 = the pipelined xy
              // kernel (double-buffered tiles over a chunk of slices) with 32 x xy_ty tiles
};
extern SmoothPlan g_smooth_plan;  // the default plan
// In 3-D on the two-kernel path the xy pass writes `tmp` (same shape as `out`), which the z pass
// reads.  plan = null uses g_smooth_plan.
void launch_smooth_field(const float* const* in, float* const* out, const float* const* orig, float* const* tmp,
                         int halves, const GridInfo& g, const float* const khost[3], const int R[3], bool epilogue,
                         float w1, float w2, bool maxnorm, IterCtl* ctl, cudaStream_t s,
                         const SmoothPlan* plan = nullptr);

// Separable smoothing of `halves` fields (each dim components) along one axis.
// `last` applies the SyN epilogue: zero boundary, blend with `orig` (w2 != 0), and the max
// ||u/spacing|| reduction into ctl->maxnorm when `maxnorm` is set.
void launch_smooth_field_pass(const float* const* in, float* const* out, const float* const* orig, int halves,
                              const GridInfo& g, int axis, const float* coeffs, int R, bool last, float w1, float w2,
                              bool maxnorm, IterCtl* ctl, cudaStream_t s);

// out = w + scale * d(x + w); scale = eta / maxnorm[h] when eta > 0, else 1.  In place when
// out == w.
void launch_compose(const float* const* d, const float* const* w, float* const* out, int halves, const GridInfo& g,
                    float eta, IterCtl* ctl, cudaStream_t s);

// One launch of the fused fixed-point inverse (k = 0 .. max_iter) for `halves` pairs.
int inv_blocks(const GridInfo& g);
// ecache: per-half residual buffers (D x N floats each) that carry the residual from a launch's
// statistics pass to the next launch's update; null recomputes it there.  k < 0: the launch is a
// CUDA-graph loop body and reads its sub-iteration index from the control block (kdev).
void launch_invert_step(const float* const* phi, float* const* psi, int halves, const GridInfo& g, int k, int max_iter,
                        double mean_tol, double max_tol, IterCtl* ctl, int phase, PartialBufs pb, cudaStream_t s,
                        bool stop_aware = true, float* const* ecache = nullptr);
// Single-pass fixed-point inverse: sub-iteration k evaluates the residual of the iterate, its
// statistics and the update in one pass over the field (launch_invert_spec), deferring the voxels
// whose clamp factor is not yet known to a short second pass (launch_invert_fix) over a list of
// their indices (`list`: per half, room for every voxel of g).  `ecache` (required) holds the
// deferred voxels' residuals.  k < 0: graph loop body (index from the control block).
void launch_invert_spec(const float* const* phi, float* const* psi, int halves, const GridInfo& g, int k, int max_iter,
                        double mean_tol, double max_tol, IterCtl* ctl, int phase, PartialBufs pb, cudaStream_t s,
                        bool stop_aware, float* const* ecache, int* const* list);
void launch_invert_fix(const float* const* phi, float* const* psi, int halves, const GridInfo& g, int k, int max_iter,
                       IterCtl* ctl, int phase, cudaStream_t s, bool stop_aware, float* const* ecache,
                       int* const* list);
// Loop control of the single-pass form's WHILE node: init (after sub-iteration 0) sets kdev = 1,
// the step form advances kdev; both set the condition to "level running, kdev < max_iter and some
// half continues", so the loop ends within max_iter bodies.
void launch_inv_spec_control(IterCtl* ctl, int phase, cudaGraphConditionalHandle handle, int max_iter, bool init,
                             cudaStream_t s);
// Loop control of a fixed-point inverse captured as a conditional WHILE graph node: init (after
// the k = 0 statistics launch) sets kdev = 1 and the loop condition to "level still running";
// the step form (the loop body's second kernel) advances kdev and sets the condition to "some
// half still iterating and kdev <= max_iter".  It always sets the condition, so the loop ends
// within max_iter bodies.
void launch_inv_loop_control(IterCtl* ctl, int phase, cudaGraphConditionalHandle handle, int max_iter, bool init,
                             cudaStream_t s);

void launch_converge(IterCtl* ctl, LogDev log, double threshold, int window, cudaStream_t s);

void launch_resample_fields(const float* const* in, const GridInfo& gi, float* const* out, const GridInfo& go,
                            int nfields, cudaStream_t s);

// Image pyramid: one axis pass, double accumulation.
void launch_conv_image_axis(const float* in, float* out, const GridInfo& g, int axis, const double* coeffs, int R,
                            cudaStream_t s);

// Intensity statistics / window.
void launch_minmax(const float* x, long long n, unsigned* mm /* [2]: ordered-int min, max */, cudaStream_t s);
void launch_histogram(const float* x, long long n, float lo, float hi, int nbins, unsigned* hist, cudaStream_t s);
// Histogram matching: the table of match points (rows src/ref, points + 2 of them; slopes of
// the points + 1 segments between them; the lines below the first and above the last point).
constexpr int HM_MAX_POINTS = 64;
constexpr int HM_STATS_BLOCKS = 592;  // fixed grid of the statistics pass (4 x 148 SMs)
struct HistMatchMap {
  int points;
  double src[HM_MAX_POINTS + 2], ref[HM_MAX_POINTS + 2], grad[HM_MAX_POINTS + 1];
  double src_min, src_max, ref_min, ref_max, lower_grad, upper_grad;
};
void launch_stats(const float* x, long long n, double* part /* [nblocks] */, int nblocks, unsigned* mm,
                  cudaStream_t s);
void launch_histogram_range(const float* x, long long n, double lo, double hi, int nbins, double vlo, double vhi,
                            unsigned* hist, cudaStream_t s);
void launch_histogram_map(const float* in, float* out, long long n, const HistMatchMap& t, cudaStream_t s);
void launch_window(const float* in, float* out, long long n, float wlo, float whi, double scale, double shift,
                   cudaStream_t s);

// Layout conversion: interleaved (x,y,z per voxel) <-> component planes.
void launch_interleave(const float* planes, float* inter, long long N, int D, cudaStream_t s);
void launch_deinterleave(const float* inter, float* planes, long long N, int D, cudaStream_t s);

// Process-wide kernel launch counter (graph replays are added by the caller).
long long launch_count();
void add_launch_count(long long n);

// Ordered-int encoding of floats for atomic min/max.
unsigned float_to_ordered(float f);
float ordered_to_float(unsigned u);

}  // namespace synx
