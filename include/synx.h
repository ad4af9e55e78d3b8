/*
 * synx.h -- C ABI of the B200 SyN + neighbourhood-CC registration stage.
 *
 * This is the boundary a host binds to: plain C types, opaque handles, int status codes,
 * no exceptions and no C++ or torch types.  It replaces the reference's stage object,
 * itk::SyNImageRegistrationMethod configured with
 * itk::ANTSNeighborhoodCorrelationImageToImageMetricv4, which antsRegistration builds and runs
 * in Examples/itkantsRegistrationHelper.hxx:1983-2220 (construct :2001-2008, configure
 * :2138-2164, run `Update()` :2198, harvest :2207-2218).  The command line front end
 * (Examples/antsRegistration.cxx:554, library entry
 * `int ants::antsRegistration(std::vector<std::string>, std::ostream*)` in
 * Examples/include/antsRegistration.h:7-9) is provided by the C++ host in
 * ants_b200/csrc/ants_registration.cpp on top of these calls.
 *
 * Conventions
 *   - Return value 0 = success, negative = error class (SYNX_E_*); synx_last_error() gives
 *     the message of the last failing call on that context (or the thread's last global
 *     error when ctx is NULL).
 *   - Images are float32, x fastest.  Displacement fields are physical-space vectors (mm).
 *     The stage's field exchange (synx_get_fields, synx_get/set_half_fields) uses ITK's
 *     interleaved in-memory layout (x,y[,z] per voxel, voxel order x fastest); the step entry
 *     points and synx_linear_field use component planes (component c of voxel i at f[c*N+i]),
 *     the order in which a vector NIfTI such as prefix0Warp.nii.gz stores its components.
 *   - "host" pointers are ordinary CPU memory; "dev" pointers are CUDA device memory on the
 *     context's device.  Every call is ordered on the context's CUDA stream.
 *   - A context is used by one host thread at a time; several contexts may run concurrently.
 */
#ifndef SYNX_H
#define SYNX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SYNX_OK 0
#define SYNX_E_ARG -1       /* invalid argument (size, dimension, pointer, option) */
#define SYNX_E_STATE -2     /* call out of order (e.g. run before set_images) */
#define SYNX_E_CUDA -3      /* CUDA runtime error */
#define SYNX_E_NOMEM -4     /* device allocation failed / budget exceeded */
#define SYNX_E_UNSUPPORTED -5

#define SYNX_MAX_LEVELS 8

/* Image grid: ITK image information.  p = origin + direction * diag(spacing) * index. */
typedef struct synx_geom {
  int32_t dim;          /* 2 or 3 */
  int32_t reserved0;
  int64_t size[3];      /* size[2] = 1 for 2-D */
  double spacing[3];
  double origin[3];
  double direction[9];  /* row-major direction cosines */
} synx_geom;

/* Stage parameters, the values antsRegistration parses from
 *   -t SyN[learningRate, updateFieldVariance, totalFieldVariance]
 *      (Examples/antsRegistrationTemplateHeader.h:801-815, defaults 3 and 0)
 *   -m CC[fixed, moving, weight, radius]   (radius default 4, :1013, :1081-1087)
 *   -c [iterations, threshold, window]     (defaults 1e-6 / 10, :545-592)
 *   -f shrink factors, -s sigmas[vox|mm]   (:622-651)
 *   --winsorize-image-intensities [lo,hi]  (:440-458)                                   */
typedef struct synx_params {
  int32_t dim;
  int32_t n_levels;
  double learning_rate;
  double update_variance;
  double total_variance;
  int32_t cc_radius;
  int32_t sigmas_in_mm;
  int32_t iterations[SYNX_MAX_LEVELS];
  int32_t shrink_factors[SYNX_MAX_LEVELS];
  double smoothing_sigmas[SYNX_MAX_LEVELS];
  double convergence_threshold;
  int32_t convergence_window;
  int32_t preprocess;        /* 1: rescale both images to [0,1] as antsRegistration does */
  float winsor_lower;        /* quantiles of the intensity window (0 and 1 by default) */
  float winsor_upper;
  int32_t inv_max_iter;      /* fixed-point inverse: 20 / 0.001 / 0.1 in SyN */
  int32_t flags;             /* SYNX_F_* */
  double inv_mean_tol;
  double inv_max_tol;
  int32_t persistent_blocks;     /* grid of the persistent level kernel; 0: automatic */
  int32_t persistent_max_voxels; /* largest level run by it; 0: automatic (400,000) */
  int32_t test_inject;           /* 0; SYNX_INJECT_* makes a failure happen for tests */
  int32_t histogram_match;       /* 1: match the moving image's histogram to the fixed one's after the
                                    window, or on the images as given when preprocess is 0
                                    (--use-histogram-matching 1; synx_histogram_match) */
  /* Tile plan of the per-kernel path (none of these changes the results beyond rounding order; the
   * smoothing choice not at all).  0 = the tuning table's entry for the level grid (see
   * synx_tuning_load), or the built-in cost models when the table has none. */
  int32_t smooth_tile_rows;      /* 3-D update smoothing: 8 or 16 = fused slab kernel with 32 x rows
                                    column tiles; -1 = xy kernel + z kernel through a temporary;
                                    -2 / -3 = the same with the pipelined xy kernel (double-buffered
                                    32 x 32 / 32 x 64 tiles over chunks of slices) */
  int32_t cc_z_chunks;           /* z chunks of the CC kernel's column walks (>= 1), 0 = table/model */
  int32_t tuning;                /* 0: use the tuning table; 1: built-in cost models only */
  int32_t reserved[1];
} synx_params;

#define SYNX_F_PROFILE_EVENTS 0x1 /* time the dominant kernel class with CUDA events */
#define SYNX_F_USE_GRAPHS 0x2     /* capture each iteration as a CUDA graph and replay it */
#define SYNX_F_NO_PERSISTENT 0x4 /* run small levels as separate kernels too (no persistent level kernel) */
/* Precision-study variants (not antsRegistration behaviour; both run the per-kernel path): */
#define SYNX_F_CC_FP32_SUMS 0x8  /* CC window sums and variance terms in float instead of double */
#define SYNX_F_FIELDS_FP16 0x10  /* half-fields rounded to half precision wherever they are stored */
#define SYNX_F_SMOOTH_TWO_PASS 0x20 /* 3-D field smoothing as an xy kernel and a z kernel through a
                                       temporary even where a tuning table picks the fused slab
                                       kernel (same results) */
#define SYNX_F_INV_TWO_PASS 0x40    /* fixed-point inverse with a statistics pass and an update pass per
                                       sub-iteration instead of the single-pass form (same results) */
#define SYNX_F_NO_PDL 0x80          /* launch an iteration's kernels without programmatic dependent launch
                                       (same results) */

/* Failure injection for tests (host-side; nothing faults): the level kernel's grid barrier waits for
 * one block more than it launched, with a short poll limit, so the wait runs out, the kernel ends
 * and synx_run / synx_run_level return SYNX_E_CUDA with a barrier-timeout message.  The context
 * and the GPU stay usable. */
#define SYNX_INJECT_BARRIER_TIMEOUT 1
/* The context's device arena allocation reports failure without calling the device allocator, so
 * synx_set_images returns SYNX_E_NOMEM as it would when the GPU is out of memory; the context can
 * still be destroyed and other contexts are unaffected. */
#define SYNX_INJECT_ALLOC_FAILURE 2

/* Fill *p with antsRegistration's defaults for a SyN stage of dimension dim
 * (SyN[0.1,3,0], CC radius 4, one level, 1 iteration, shrink 1, sigma 0 vox). */
int synx_params_default(synx_params* p, int dim);

typedef struct synx_ctx synx_ctx;

/* Context lifetime.  stream may be NULL (the context creates its own). */
int synx_create(const synx_params* params, int device, void* cuda_stream, synx_ctx** out);
int synx_destroy(synx_ctx* ctx);
const char* synx_last_error(const synx_ctx* ctx);

/* Inputs from host memory (copied host->device on the context stream). The fixed image grid
 * is the virtual domain of the stage, as in antsRegistration (hxx:1154). */
int synx_set_images(synx_ctx* ctx, const float* fixed_host, const synx_geom* fixed_geom,
                    const float* moving_host, const synx_geom* moving_geom);
/* Same with device-resident inputs (copied device->device into the context arena). */
int synx_set_images_device(synx_ctx* ctx, const float* fixed_dev, const synx_geom* fixed_geom,
                           const float* moving_dev, const synx_geom* moving_geom);

/* Run every level (synx_run) or one level (levels must be run in order 0..L-1). */
int synx_run(synx_ctx* ctx);
int synx_run_level(synx_ctx* ctx, int level);

/* Batched pairs.  No reference counterpart: antsRegistration registers one pair per process
 * (antsRegistration.cxx:554-777); these entry points advance many contexts together.
 * A batch holds only device staging for the launch arguments.  synx_batch_step advances every
 * listed context that has a level left by its next level (synx_run_level semantics per
 * context, same results bit for bit whatever else is in the batch); levels that the persistent
 * level kernel serves share one cooperative launch per (dimension, CC radius); *advanced gets
 * the number of contexts that ran a level.  All work goes on cuda_stream (ordered after work
 * already queued on each context's own stream); the call returns after the step has finished.
 * synx_batch_run repeats steps until every context has run all its levels.  Contexts must be on
 * the batch's device and must not be used elsewhere during the call. */
typedef struct synx_batch synx_batch;
int synx_batch_create(int device, synx_batch** out);
int synx_batch_destroy(synx_batch* batch);
const char* synx_batch_last_error(const synx_batch* batch);
int synx_batch_step(synx_batch* batch, synx_ctx* const* ctxs, int n, void* cuda_stream, int* advanced);
int synx_batch_run(synx_batch* batch, synx_ctx* const* ctxs, int n, void* cuda_stream);

/* Device bytes a context holds for this stage and these image grids (what synx_set_images
 * allocates); no device work. */
int synx_footprint(const synx_params* params, const synx_geom* fixed_geom, const synx_geom* moving_geom,
                   int64_t* bytes);

/* Serving loop.  No reference counterpart (the reference runs one registration per process).
 * A server thread owns one stream and a batch; requests queue on submission and are admitted in
 * arrival order whenever their footprint (synx_footprint) fits the device-memory budget and the
 * active limit (a request that does not fit yet does not block smaller ones behind it).  Every
 * admitted request keeps its images, pyramid and fields resident; each loop step advances every
 * resident request by one level in one synx_batch_step, so requests that arrive while others
 * run join at the next step.  A finished request's context is kept in a pool with its device
 * arena and reused by a later request with the same stage parameters whose footprint it covers
 * (no device allocation on that path); pooled contexts are freed when admission needs the memory.
 * A request's result is bit-identical to running it alone.  The caller's input buffers must
 * stay valid until the request is admitted (status >= 1), output buffers until it is done. */
typedef struct synx_server synx_server;
typedef struct synx_server_config {
  int32_t device;
  int32_t max_active;        /* most resident requests (0: no limit) */
  int64_t hbm_budget_bytes;  /* device bytes resident requests may hold (0: 90% of free memory) */
  int32_t reserved[8];
} synx_server_config;
typedef struct synx_request_info {
  int32_t status;            /* 0 queued, 1 resident, 2 done, negative: SYNX_E_* failure */
  int32_t levels_done;
  int64_t device_bytes;      /* its footprint */
  double t_submit, t_admit, t_done;  /* seconds since the server started (steady clock) */
  char error[256];
} synx_request_info;
typedef struct synx_server_stats {
  int64_t submitted, completed, failed, queued, resident;
  int64_t bytes_resident;    /* arenas of resident requests */
  int64_t bytes_peak;        /* peak of resident + pooled */
  int64_t budget;
  int64_t bytes_pooled;      /* arenas of finished contexts kept for reuse */
  int64_t steps;
  double step_seconds;       /* host time spent inside batch steps */
  double resident_byte_seconds;  /* integral of bytes_resident over time (mean occupancy = / elapsed) */
  double elapsed;
} synx_server_stats;
int synx_server_create(const synx_server_config* cfg, synx_server** out);
/* Stops the loop after the resident requests finish; queued requests fail with SYNX_E_STATE.  No
 * other call on this server (submit, wait, stats) may run concurrently with it or follow it. */
int synx_server_destroy(synx_server* server);
const char* synx_server_last_error(const synx_server* server);
int synx_server_submit(synx_server* server, const synx_params* params, const float* fixed_host,
                       const synx_geom* fixed_geom, const float* moving_host, const synx_geom* moving_geom,
                       float* forward_host, float* inverse_host, int64_t* request_id);
/* Waits up to timeout_s (< 0: no limit) for the request to finish; fills *info (may be NULL).
 * Returns 0 when it is done, SYNX_E_STATE on timeout, or its failure code. */
int synx_server_wait(synx_server* server, int64_t request_id, double timeout_s, synx_request_info* info);
int synx_server_get_stats(synx_server* server, synx_server_stats* stats);

/* Geometry of the grid the output fields live on (the last level run). */
int synx_get_output_geom(const synx_ctx* ctx, synx_geom* out);
/* Final forward (prefix0Warp) and inverse (prefix0InverseWarp) fields, interleaved, host. */
int synx_get_fields(synx_ctx* ctx, float* forward_host, float* inverse_host);
/* Same into device memory. */
int synx_get_fields_device(synx_ctx* ctx, float* forward_dev, float* inverse_dev);
/* The four half-fields (fixed-to-middle, its inverse, moving-to-middle, its inverse) on the
 * current level grid, interleaved, host; any pointer may be NULL. */
int synx_get_half_fields(synx_ctx* ctx, float* phi_f, float* psi_f, float* phi_m, float* psi_m);
/* Replace the four half-fields on the current level grid (resume / test hook). */
int synx_set_half_fields(synx_ctx* ctx, const float* phi_f, const float* psi_f, const float* phi_m,
                         const float* psi_m, const synx_geom* grid);

/* Per-iteration log of everything run so far: level, iteration, metric value, convergence
 * value, fixed-point sub-iterations (sum over the four inversions).  Returns the number of
 * records through *count; arrays may be NULL to query the count. */
int synx_get_log(synx_ctx* ctx, int32_t* level, int32_t* iteration, double* metric, double* convergence,
                 int32_t* inverse_iterations, int64_t capacity, int64_t* count);

/* Device time of the dominant kernel class (fixed-point inverse sub-iterations) recorded
 * with CUDA events when SYNX_F_PROFILE_EVENTS is set: total ms, launches, voxels processed. */
int synx_get_profile(synx_ctx* ctx, double* inverse_ms, int64_t* inverse_launches, int64_t* inverse_voxels,
                     double* cc_ms, int64_t* cc_launches, int64_t* cc_voxels);
int synx_reset_profile(synx_ctx* ctx);
/* Per-level device times (CUDA events on the context stream) accumulated since the last
 * reset: level set-up (pyramid smoothing, field resampling), the iterations, and in
 * SYNX_F_PROFILE_EVENTS mode the inverse and CC shares; iterations run, fixed-point
 * sub-iterations (sum over the four inversions) and grid voxels. */
int synx_get_level_profile(synx_ctx* ctx, int level, double* setup_ms, double* iterate_ms, double* inverse_ms,
                           double* cc_ms, int64_t* iterations, int64_t* inverse_subiterations, int64_t* voxels);

/* Device memory held by the context, bytes. */
int synx_get_device_bytes(const synx_ctx* ctx, int64_t* bytes);

/* Kernel launches issued by this library in this process so far (all contexts; each node
 * of a replayed CUDA graph counts once per replay).  Instrumentation, no reference
 * counterpart. */
int synx_get_launch_count(int64_t* count);

/* ---------------------------------------------------------------------------------------
 * Step entry points (device pointers, component-plane fields: component c of voxel i at
 * f[c*N + i]).  These are the per-step hooks of the stage, used for parity checks; each
 * names the reference behaviour it replaces.  All take a CUDA stream (NULL = default).
 * --------------------------------------------------------------------------------------- */

/* Discrete Gaussian kernel (ITK GaussianOperator: e^-t I_n(t), max error, max width).
 * Writes up to cap coefficients of the full symmetric kernel; returns its length in *len. */
int synx_gaussian_kernel(double variance, double max_error, int max_width, double* coeffs, int cap, int* len);

/* Pyramid smoothing of an image (ITK DiscreteGaussianImageFilter, per level of
 * ImageRegistrationMethodv4; max error 0.01, width 32). */
int synx_smooth_image(const float* in_dev, float* out_dev, const synx_geom* g, double sigma, int sigma_in_mm,
                      void* stream);

/* out(i) = img(x_i + u(x_i)), linear, 0 outside (ResampleImageFilter through a
 * displacement field; itkantsRegistrationHelper.hxx:2138, observer .h:342-381). */
int synx_warp_image(const float* img_dev, const synx_geom* img_geom, const float* u_dev, const synx_geom* grid,
                    float* out_dev, void* stream);
/* Same with nearest-neighbour sampling (antsApplyTransforms -n NearestNeighbor,
 * Examples/make_interpolator_snip.tmpl:24-28): inside the image buffer, the voxel at
 * floor(c + 0.5) per axis of the continuous index c (ITK's NearestNeighborInterpolateImageFunction),
 * 0 outside.  For label images. */
int synx_warp_image_nearest(const float* img_dev, const synx_geom* img_geom, const float* u_dev, const synx_geom* grid,
                            float* out_dev, void* stream);
/* Same with generic label interpolation (antsApplyTransforms -n GenericLabel[Linear],
 * Examples/make_interpolator_snip.tmpl:112-117; ITK's LabelImageGenericInterpolateImageFunction over
 * the linear interpolator): inside the buffer, the label with the largest sum of linear cell-corner
 * weights, a tie going to the smaller label; 0 outside. */
int synx_warp_image_label(const float* img_dev, const synx_geom* img_geom, const float* u_dev, const synx_geom* grid,
                          float* out_dev, void* stream);

/* Histogram matching of `src` to `ref` (device float arrays of n_src and n_ref voxels); `out` may be
 * `src`.  Replaces ITK's HistogramMatchingImageFilter as PreprocessImage runs it for
 * --use-histogram-matching 1 (Examples/itkantsRegistrationHelper.hxx:111-122: levels 256,
 * match_points 12, threshold_at_mean 1).  Each image's histogram holds the voxels in
 * [threshold, max] (threshold: the mean, or the min with threshold_at_mean 0) in `levels` equal
 * bins over [min, max]; the match points are the thresholds, the quantiles j/(match_points+1) and
 * the maxima, and each voxel is mapped through the piecewise-linear function between them.
 * levels in 1..4096, match_points in 1..64 (ImageMath HistogramMatch runs 255 and 64 by default,
 * Examples/ImageMath_Templates.hxx:1758-1789).  Synchronises the stream. */
int synx_histogram_match(const float* src_dev, int64_t n_src, const float* ref_dev, int64_t n_ref, int32_t levels,
                         int32_t match_points, int32_t threshold_at_mean, float* out_dev, void* stream);

/* Metric masks of the stage (antsRegistration -x [fixedMask,movingMask], Examples/antsRegistration.cxx:
 * 471-480, set on the metric at Examples/itkantsRegistrationHelper.hxx:863-890, :1159-1166): host
 * arrays on their own grids, nonzero = inside; NULL for none (both NULL clears them).  Each mask is
 * resampled into the virtual domain through its image's inverse half-field (nearest neighbour, 0
 * outside) every iteration; CC sums, counts, values and updates then cover only the voxels inside
 * both.  Masks stay set across synx_set_images; a masked stage runs the per-kernel path. */
int synx_set_masks(synx_ctx* ctx, const float* fixed_mask, const synx_geom* fixed_mask_geom,
                   const float* moving_mask, const synx_geom* moving_mask_geom);

/* Initial half-fields of the stage: a SyN stage initialized from a saved registration state
 * (antsRegistration --restore-state with --initialize-transforms-per-stage 1; the restored
 * FixedToMiddle and MovingToMiddle transforms are set on the SyN method at
 * Examples/itkantsRegistrationHelper.hxx:2093-2125, and its per-level initialization resamples their
 * fields to each level's domain).  Host arrays, interleaved like synx_get_half_fields' (phiF = fixed
 * to middle, psiF its inverse, phiM = moving to middle, psiM its inverse), on `grid`; all NULL
 * clears them.  The first level resamples them to its grid instead of starting from zero fields.
 * They stay set across runs and synx_set_images; refused while a run is between levels. */
int synx_set_initial_half_fields(synx_ctx* ctx, const float* phi_f, const float* psi_f, const float* phi_m,
                                 const float* psi_m, const synx_geom* grid);

/* Tile plans chosen by the project's autotuner (python -m ants_b200.autotune): a text table of
 * measured winners per level grid, one line per (dim, nx, ny, nz, CC radius, smoothing radius) with
 * the chosen persistent-kernel use, smoothing tile rows and CC z chunks.  Loaded once per process at
 * the first synx_create from $SYNX_TUNING_TABLE or, if unset, tuning_b200.txt beside libsynx.so.
 * synx_tuning_load(path) (re)loads a table explicitly (an unreadable path is SYNX_E_ARG); NULL
 * reloads the default (absent: an empty table); returns the number of entries.  A level grid without an exact entry takes the entry of the
 * nearest size (same dim and radii, voxel count within a factor of 1.5), else the cost models.
 * No counterpart in the reference (ITK has no device tiles). */
int synx_tuning_load(const char* path);
const char* synx_tuning_path(void);
/* The plan level `level` of a context runs with (after synx_set_images): persistent = 1 if the
 * level runs in the persistent level kernel, smoothing tile rows (or -1), CC z chunks. */
int synx_level_plan(synx_ctx* ctx, int level, int32_t* persistent, int32_t* smooth_rows, int32_t* cc_z_chunks);

/* Windowed CC on two images on the same grid: value (-mean cc), the fixed-to-middle update
 * direction (uses grad of `moving`) and the moving-to-middle one (uses grad of `fixed`)
 * (ITK ANTSNeighborhoodCorrelationImageToImageMetricv4; in-tree twin
 * ImageRegistration/itkCrossCorrelationRegistrationFunction.cxx:179-504). */
int synx_cc_metric(const float* fixed_dev, const float* moving_dev, const synx_geom* g, int radius,
                   float* grad_fixed_dev, float* grad_moving_dev, double* value_host, void* stream);
/* CC over the valid voxels only: valid_dev holds one byte per voxel (nonzero = valid, as the
 * metric masks make it); invalid voxels add nothing to the window sums or counts and get no
 * value and zero updates; the value is -mean cc over the valid voxels. */
int synx_cc_metric_masked(const float* fixed_dev, const float* moving_dev, const uint8_t* valid_dev,
                          const synx_geom* g, int radius, float* grad_fixed_dev, float* grad_moving_dev,
                          double* value_host, void* stream);
/* Same with flags: SYNX_F_CC_FP32_SUMS selects float window sums (precision study). */
int synx_cc_metric_ex(const float* fixed_dev, const float* moving_dev, const synx_geom* g, int radius, int flags,
                      float* grad_fixed_dev, float* grad_moving_dev, double* value, void* cuda_stream);

/* Same computation as synx_cc_metric, for callers that must not allocate device memory: a
 * plug-in whose host application (a viewer, a framework with its own caching allocator, a
 * serving process) owns the GPU's memory budget, or a latency-bound loop that cannot afford the
 * device-wide synchronisation of a cudaMalloc/cudaFree pair.  No counterpart in the reference.
 * It calls no cudaMalloc/cudaFree: the kernel's scratch (control block and per-block partial
 * sums, about 260 KB) is a fixed array in device memory that each GPU using the library holds
 * until the process exits.  Limit: grids needing more than 32768 CC blocks (for example more
 * than 8192 x 1024 voxels per slice) are rejected with SYNX_E_ARG.  The first call on a device
 * looks the array's device address up, so make that first call before any stream capture.  All
 * calls on a device share the array and find the previous call's contents in it (the control
 * block is cleared before each launch): calls that overlap on the GPU (other streams, other
 * host threads) race.  value_host may be NULL; otherwise the call waits for its stream to read
 * the value.  While the stream is being captured into a CUDA graph value_host must be NULL (a
 * capture cannot wait for its stream; the call returns SYNX_E_ARG otherwise): the gradients are
 * written on each replay, and the value stays in the shared array until the next call.  Errors are
 * reported by synx_noalloc_last_error(). */
int synx_cc_metric_noalloc(const float* fixed_dev, const float* moving_dev, const synx_geom* g, int radius,
                           float* grad_fixed_dev, float* grad_moving_dev, double* value_host, void* stream);
const char* synx_noalloc_last_error(void);

/* Gaussian smoothing of a displacement field as SyN does it (Examples/SmoothDisplacementField
 * .cxx:70-125 twin).  If max_norm_host is not NULL, also returns max ||u/spacing||. */
int synx_smooth_field(const float* in_dev, float* out_dev, const synx_geom* g, double variance,
                      double* max_norm_host, void* stream);

/* out = w + scale * d(x + w)  (ITK ComposeDisplacementFieldsImageFilter; twin
 * Utilities/itkComposeDiffeomorphismsImageFilter.hxx:70-105). */
int synx_compose(const float* d_dev, const float* w_dev, const synx_geom* g, float scale, float* out_dev,
                 void* stream);
/* out = u + M w at every voxel of `g` (component planes; out may alias u or w; M row-major 3x3, its
 * leading dim x dim block used).  The composition step of a transform stack where compose's
 * interpolation does not apply: a linear transform T(p) = A p + b after w, T(x + w) - x =
 * (T(x) - x) + A w with u = synx_linear_field(T) and M = A; and a field d on another grid,
 * w + d(x + w) with u sampled from d's own grid by synx_warp_image per component and M = I. */
int synx_field_affine_update(const float* u_dev, const float* w_dev, const synx_geom* g, const double* matrix,
                             float* out_dev, void* stream);

/* Fixed-point inverse of phi, warm-started from psi_inout (ITK
 * InvertDisplacementFieldImageFilter; twin itkANTSImageRegistrationOptimizer.h:1845-1988).
 * Returns the number of iterations run in *iterations (may be NULL). */
int synx_invert_field(const float* phi_dev, float* psi_inout_dev, const synx_geom* g, int max_iter,
                      double mean_tol, double max_tol, int* iterations, void* stream);

/* Linear resampling of a field onto another grid, 0 outside (DisplacementFieldTransform
 * ParametersAdaptor, itkantsRegistrationHelper.hxx:2028-2055). */
int synx_resample_field(const float* in_dev, const synx_geom* in_geom, float* out_dev, const synx_geom* out_geom,
                        void* stream);

/* Level grid for a shrink factor (CalculateShrinkFactorsPerDimension hxx:593-641 +
 * ShrinkImageFilter output information hxx:16-39). */
int synx_shrink_geom(const synx_geom* in, int factor, synx_geom* out);

/* ---- Linear transforms (host only, no CUDA call) --------------------------------------------
 * The linear transforms antsRegistration writes next to its warps (prefix0GenericAffine.mat, or
 * Rigid/Similarity/Translation/Affine .mat files without collapsing) and antsApplyTransforms reads
 * in its transform stack: Utilities/itkantsReadWriteTransform.h:19-120 hands .mat/.txt files to
 * ITK's transform file reader.  Every supported type is stored as the matrix-offset form ITK's
 * MatrixOffsetTransformBase applies to physical (LPS) points:  T(p) = A (p - c) + t + c.        */
typedef struct synx_linear {
  int32_t dim;            /* 2 or 3 */
  int32_t has_center;     /* 1 for the matrix-offset family (it has a center), 0 for Translation and
                           * Identity transforms (c = 0); collapsing keeps the first center applied */
  double matrix[9];       /* A, row-major 3x3; a 2-D transform fills the leading 2x2 block */
  double translation[3];  /* t */
  double center[3];       /* c, the transform's fixed parameters */
} synx_linear;

/* Reads linear transform `index` (0-based, file order) of an ITK transform file: the MATLAB v4
 * binary form (.mat; a parameter variable named after the transform type, then "fixed") or the
 * Insight text form (.txt or .tfm: "Transform:", "Parameters:", "FixedParameters:" lines).  Types, double
 * or float, `dim` x `dim`: AffineTransform, MatrixOffsetTransformBase, TranslationTransform,
 * IdentityTransform, Euler2DTransform, Rigid2DTransform, Similarity2DTransform, Euler3DTransform,
 * VersorRigid3DTransform, Similarity3DTransform; a CompositeTransform entry is skipped (its
 * components follow it, in the order a composite adds them).  `out` may be NULL to count.
 * Returns the number of linear transforms in the file (>= 1), or SYNX_E_ARG (missing, malformed
 * or empty file, dimension mismatch, index out of range) / SYNX_E_UNSUPPORTED (another transform
 * type); synx_last_error(NULL) names the reason. */
int synx_read_linear_transform(const char* path, int dim, int index, synx_linear* out);

/* The same conversion for one transform given by its type name ("<Base>_<double|float>_<D>_<D>",
 * a type listed above) and its parameters and fixed parameters as an ITK transform file holds them
 * (the entries of a composite transform read elsewhere, e.g. a saved registration state).  The
 * counterpart of ITK's transform factory for these types.  `params`/`fixed` may be NULL when their
 * count is 0.  SYNX_OK, or SYNX_E_ARG (malformed name, wrong counts, dimension mismatch, a
 * CompositeTransform) / SYNX_E_UNSUPPORTED (another type). */
int synx_linear_from_parameters(const char* type, const double* params, int n_params, const double* fixed,
                                int n_fixed, int dim, synx_linear* out);

/* Displacement field of a linear transform on `grid`, in host memory, as component planes
 * (component c of voxel i at field[c*N + i], the layout of the step entry points, ready to copy
 * to the device for synx_compose / synx_warp_image): u(p) = T(p) - p at every voxel centre p,
 * or T^-1(p) - p with invert = 1 (SYNX_E_ARG when A is singular).  Double arithmetic, float
 * output. */
int synx_linear_field(const synx_linear* transform, int invert, const synx_geom* grid, float* field_host);

/* The translation antsRegistration derives from a pair of images for -r [fixed,moving,feature]
 * (Examples/itkantsRegistrationHelper.h:1297-1360; ITK's CenteredTransformInitializer for 0 and 1):
 * a rigid transform with identity rotation, center c_F and translation c_M - c_F, where c is per
 * image 0: the geometric center (the physical point of continuous index (size-1)/2), 1: the center
 * of intensity mass (sum of value * physical point over sum of value, raw intensities), 2: the
 * origin.  Images are host memory (x fastest) and may be NULL for features 0 and 2.  SYNX_E_ARG for
 * a zero total mass.  Host arithmetic in double. */
int synx_initial_translation(const float* fixed_host, const synx_geom* fixed_geom, const float* moving_host,
                             const synx_geom* moving_geom, int feature, synx_linear* out);

/* Writes `transform` as an ITK AffineTransform_double_<dim>_<dim> file: MATLAB v4 (.mat,
 * little-endian double column vectors "AffineTransform_double_D_D" = A row-major then t, and
 * "fixed" = c), the form antsRegistration writes prefix0GenericAffine.mat in, or Insight text
 * (.txt or .tfm).  SYNX_E_ARG for another extension or a file that cannot be written. */
int synx_write_linear_transform(const char* path, const synx_linear* transform);

#ifdef __cplusplus
}
#endif

#endif /* SYNX_H */
