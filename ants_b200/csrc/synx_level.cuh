// Persistent level kernel interface (see synx_level.cu).
#pragma once

#include "synx_cc_tile.cuh"
#include "synx_phases.cuh"

namespace synx {

struct LevelArgs {
  WarpArgs warp;        // images, inverse half-fields, warped images; warp.zb set for warp_gz
  CCParams cc;          // with cc.ZC of the standalone CC decomposition
  float* gF;            // CC update directions (fixed half, moving half)
  float* gM;
  Smooth3Args sxy;      // xy smoothing: in = {gF, gM}, out = tmp (3-D) or update (2-D)
  Smooth3Args sz;       // z smoothing (3-D): in = tmp, out = update, ZC set
  ComposeArgs comp;     // d = update, w = o = forward half-fields (in place); comp.zb for comp_gz
  InvArgs invA;         // phi = forward half-fields, psi = inverse half-fields
  InvArgs invB;         // phi = inverse half-fields, psi = forward half-fields
  Dims g;
  IterCtl* ctl;
  LogDev log;
  double* cc_partials;
  double* inv_psum;
  float* inv_pmax;
  int pcap;             // partial slots per half (>= 2 x inversion tiles per half)
  int iters;            // iterations of the level
  int r_smooth;         // update-field smoothing radius (1..8)
  int cc_gx, cc_gy, cc_gz;
  int el_gx, el_gy;     // 32 x 8 tiles in x, y
  int warp_gz, comp_gz, inv_gz, sz_gz;
  int inv_max_iter;
  double inv_mean_tol, inv_max_tol;
  double conv_threshold;
  int conv_window;
  int diag;             // index maps without rotation
  int bar_extra;        // blocks a barrier waits for beyond the group (0; 1 in the failure-detection test)
  long long bar_spins;  // polls of a barrier wait before it gives up and sets IterCtl::bar_err
};

// Several pairs in one launch of the level kernel (same dimension and CC radius).
struct BatchLevelArgs {
  const LevelArgs* pairs;  // device array of npairs
  const int* first_block;  // device array of npairs + 1: pair p owns [first_block[p], first_block[p+1])
  int npairs;
};

constexpr int kLevelMaxSmoothRadius = 8;
constexpr int kLevelSmoothTY = 32;  // rows of the xy smoothing tiles in the level kernel

size_t level_smem_bytes(int dim, int cc_radius, int r_smooth);
// Largest cooperative grid for the level kernel on `device` (0 if unsupported).
int level_max_blocks(int dim, int cc_radius, int r_smooth, int device);
cudaError_t launch_level(const LevelArgs& A, int dim, int cc_radius, int blocks, cudaStream_t s);
// Largest cooperative grid of the batched level kernel, and its launch (blocks = first_block[npairs]).
int level_batch_max_blocks(int dim, int cc_radius, int device);
cudaError_t launch_level_batch(const BatchLevelArgs& B, int dim, int cc_radius, int blocks, cudaStream_t s);

// Tile depth (z slices) of the level kernel's per-voxel phases for `halves` field halves; depends
// on the level grid only.
int level_zb(const Dims& d, int halves);

// Helpers shared with the standalone launchers (synx_kernels.cu, synx_cc.cu).
bool affine_diag_host(const Affine& m);
CCParams make_cc_params(const GridInfo& g, int radius, int chunks = 0);
Smooth3Args make_smooth_args(const float* const* in, float* const* out, const float* const* orig, int halves,
                             const GridInfo& g, const float* const khost[3], const int R[3], bool epilogue, float w1,
                             float w2, bool maxnorm, int* radius);
int smooth_z_chunk(const Dims& d, int halves, int RR, int slots);
InvArgs make_inv_args(const float* const* phi, float* const* psi, int halves, const GridInfo& g, int zb,
                      float* const* ecache = nullptr);

}  // namespace synx
