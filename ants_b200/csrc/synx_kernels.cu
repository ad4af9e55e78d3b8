// synx kernels for sm_100a: the per-voxel steps of one SyN + neighbourhood-CC iteration
// (the CC kernel itself is in synx_cc.cu).
//
// Everything here is memory-bound stencil / gather work (no contraction), so the design goals
// are coalesced component-plane access, shared-memory staging of stencil halos, FP64 only
// where the arithmetic needs it (global means), 32-bit index arithmetic with a 3-D launch
// mapping (a block covers 32 x 8 voxels in x, y and a chunk of z slices, so no thread divides
// a linear index), and device-side loop control so that a whole level can be enqueued (or
// graph-replayed) without host round trips.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>

#include <cuda_fp16.h>

#include "synx_level.cuh"
#include "synx_phases.cuh"

namespace synx {

thread_local int t_pdl = 0;
thread_local int t_pdl_skip = 0;
thread_local int t_rev = 0;

// Process-wide count of kernel launches issued by this library (instrumentation).
std::atomic<long long> g_launches{0};
static inline void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(); }
void add_launch_count(long long n) { g_launches.fetch_add(n); }

// ------------------------------------------------------------------------------------------
// Host geometry helpers
// ------------------------------------------------------------------------------------------
static void inv3(const double* a, double* o) {
  double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
               a[2] * (a[3] * a[7] - a[4] * a[6]);
  double id = 1.0 / det;
  o[0] = (a[4] * a[8] - a[5] * a[7]) * id;
  o[1] = (a[2] * a[7] - a[1] * a[8]) * id;
  o[2] = (a[1] * a[5] - a[2] * a[4]) * id;
  o[3] = (a[5] * a[6] - a[3] * a[8]) * id;
  o[4] = (a[0] * a[8] - a[2] * a[6]) * id;
  o[5] = (a[2] * a[3] - a[0] * a[5]) * id;
  o[6] = (a[3] * a[7] - a[4] * a[6]) * id;
  o[7] = (a[1] * a[6] - a[0] * a[7]) * id;
  o[8] = (a[0] * a[4] - a[1] * a[3]) * id;
}

GridInfo make_grid(int dim, const int64_t size[3], const double sp[3], const double org[3], const double dir[9]) {
  GridInfo g;
  g.d.dim = dim;
  g.d.nx = (int)size[0];
  g.d.ny = (int)size[1];
  g.d.nz = dim == 3 ? (int)size[2] : 1;
  g.d.N = (long long)g.d.nx * g.d.ny * g.d.nz;
  for (int k = 0; k < 3; ++k) {
    g.sp[k] = sp[k];
    g.org[k] = org[k];
  }
  for (int k = 0; k < 9; ++k) g.dir[k] = dir[k];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) g.i2p[r * 3 + c] = dir[r * 3 + c] * sp[c];
  if (dim == 2) {
    g.i2p[2] = g.i2p[5] = g.i2p[6] = g.i2p[7] = 0.0;
    g.i2p[8] = 1.0;
    g.org[2] = 0.0;
  }
  inv3(g.i2p, g.p2i);
  return g;
}

// Grids of one pyramid share the fixed image's direction cosines.  Between such grids the
// index map is formed in their common frame, B = diag(sp_src / sp_dst) with exact zeros and
// t = D^-1 (org_src - org_dst) / sp_dst, so that an even shrink factor's half-voxel rim points
// (c = -0.5, c = n - 0.5) come out exact instead of carrying the rotation's rounding noise
// into ITK's inside-buffer test.  Other grid pairs go through the physical frame.
static bool same_direction(const GridInfo& a, const GridInfo& b) {
  const int dim = a.d.dim;
  if (dim != b.d.dim) return false;
  for (int r = 0; r < dim; ++r)
    for (int c = 0; c < dim; ++c)
      if (a.dir[r * 3 + c] != b.dir[r * 3 + c]) return false;
  return true;
}

void index_map(const GridInfo& src, const GridInfo& dst, double t[3], double B[9]) {
  const int dim = src.d.dim;
  const double dorg[3] = {src.org[0] - dst.org[0], src.org[1] - dst.org[1], dim == 3 ? src.org[2] - dst.org[2] : 0.0};
  if (same_direction(src, dst)) {
    double D[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, Di[9];
    for (int r = 0; r < dim; ++r)
      for (int c = 0; c < dim; ++c) D[r * 3 + c] = src.dir[r * 3 + c];
    inv3(D, Di);
    for (int r = 0; r < 3; ++r) {
      const bool on = r < dim;
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
  if (dim == 2) {
    t[2] = 0.0;
    B[2] = B[5] = B[6] = B[7] = B[8] = 0.0;
  }
}

Affine make_affine(const GridInfo& src, const GridInfo& dst) {
  Affine a;
  double t[3], B[9];
  index_map(src, dst, t, B);
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) {
      a.B[r * 3 + c] = (float)B[r * 3 + c];
      a.A[r * 3 + c] = (float)dst.p2i[r * 3 + c];
    }
    a.t[r] = (float)t[r];
  }
  return a;
}

unsigned float_to_ordered(float f) {
  unsigned u;
  memcpy(&u, &f, 4);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
float ordered_to_float(unsigned u) {
  unsigned v = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  float f;
  memcpy(&f, &v, 4);
  return f;
}
__device__ __forceinline__ unsigned d_float_to_ordered(float f) {
  unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

static inline int grid_for(long long n, int threads, int cap = 148 * 16) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

// 3-D launch mapping: 32 x 8 threads per block, each thread walks `zb` consecutive slices.
struct Map3 {
  dim3 grid;
  int zb;
  int nblocks;  // blocks per field (per half)
};
static Map3 map3(const Dims& d, int halves = 1, int target = 148 * 24) {
  Map3 m;
  const int gx = (d.nx + 31) / 32, gy = (d.ny + 7) / 8;
  int per = target / (gx * gy * halves);
  if (per < 1) per = 1;
  int zb = (d.nz + per - 1) / per;
  if (zb < 1) zb = 1;
  const int gz = (d.nz + zb - 1) / zb;
  m.grid = dim3(gx, gy, gz * halves);
  m.zb = zb;
  m.nblocks = gx * gy * gz;
  return m;
}

// Thread coordinates of a 3-D mapped block; h = half selected by blockIdx.z.
struct Coord3 {
  int x, y, z0, z1, h, bid;
  bool ok;
};
__device__ __forceinline__ Coord3 coord3(const Dims& d, int zb, int halves) {
  Coord3 c;
  const int gz = gridDim.z / halves;
  c.h = blockIdx.z / gz;
  const int zc = blockIdx.z - c.h * gz;
  c.x = blockIdx.x * 32 + (threadIdx.x & 31);
  c.y = blockIdx.y * 8 + (threadIdx.x >> 5);
  c.z0 = zc * zb;
  c.z1 = min(c.z0 + zb, d.nz);
  c.ok = c.x < d.nx && c.y < d.ny;
  c.bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * zc);
  return c;
}

static bool affine_diag(const Affine& m) {
  const int off[6] = {1, 2, 3, 5, 6, 7};
  for (int k : off)
    if (m.B[k] != 0.0f || m.A[k] != 0.0f) return false;
  return true;
}
bool affine_diag_host(const Affine& m) { return affine_diag(m); }

// ------------------------------------------------------------------------------------------
// Level control reset
// ------------------------------------------------------------------------------------------
__global__ void k_zero_ctl_level(IterCtl* ctl) {
  ctl->stop = 0;
  ctl->iter = 0;
  ctl->total_abs = 0.0;
  ctl->maxnorm[0] = ctl->maxnorm[1] = 0u;
  ctl->cc_counter = 0u;
  ctl->bar_count = 0u;
  ctl->bar_err = 0;
  for (int p = 0; p < 2; ++p)
    for (int h = 0; h < 2; ++h) {
      ctl->inv[p][h].counter = 0u;
      ctl->inv[p][h].iters = 0;
      ctl->inv[p][h].exec[0] = ctl->inv[p][h].exec[1] = 0;
      ctl->inv[p][h].mrun = 0u;
      ctl->inv[p][h].lcount = 0u;
      ctl->inv[p][h].fcount = 0u;
    }
}
void launch_zero_ctl_level(IterCtl* ctl, cudaStream_t s) {
  count_launch();
  k_zero_ctl_level<<<1, 1, 0, s>>>(ctl);
}


// ------------------------------------------------------------------------------------------
// Warps (one tile per block).
// ------------------------------------------------------------------------------------------
template <int DIM, bool DIAG>
__global__ void __launch_bounds__(256) k_warp_pair(const WarpArgs a, IterCtl* ctl, int rev) {
  griddep_wait();
  if (ctl != nullptr && ctl->stop) return;
  if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && ctl != nullptr) {
    ctl->maxnorm[0] = 0u;  // the update scaling of this iteration starts from zero
    ctl->maxnorm[1] = 0u;
  }
  const uint3 b = sweep_block(rev);
  warp_pair_tile<DIM, DIAG>(a, b.x, b.y, b.z);
}

void launch_warp_pair(const float* F, const GridInfo& gF, const float* psiF, const float* M, const GridInfo& gM,
                      const float* psiM, const GridInfo& gv, float* Ft, float* Mt, IterCtl* ctl, cudaStream_t s) {
  count_launch();
  WarpArgs a{F, M, psiF, psiM, Ft, Mt, gF.d, gM.d, gv.d, make_affine(gv, gF), make_affine(gv, gM), 0};
  const Map3 m = map3(gv.d);
  a.zb = m.zb;
  const bool dg = affine_diag(a.mF) && affine_diag(a.mM);
  if (gv.d.dim == 3) {
    if (dg) launch_k(k_warp_pair<3, true>, m.grid, 256, 0, s, a, ctl, t_rev);
    else launch_k(k_warp_pair<3, false>, m.grid, 256, 0, s, a, ctl, t_rev);
  } else {
    if (dg) launch_k(k_warp_pair<2, true>, m.grid, 256, 0, s, a, ctl, t_rev);
    else launch_k(k_warp_pair<2, false>, m.grid, 256, 0, s, a, ctl, t_rev);
  }
}

template <int DIM>
__global__ void __launch_bounds__(256) k_warp_image(const float* __restrict__ img, Dims di, Affine m,
                                                    const float* __restrict__ u, Dims dv, int zb,
                                                    float* __restrict__ out) {
  const Coord3 c = coord3(dv, zb, 1);
  if (!c.ok) return;
  const int N = (int)dv.N, nxy = dv.nx * dv.ny;
  for (int z = c.z0; z < c.z1; ++z) {
    const int i = z * nxy + c.y * dv.nx + c.x;
    out[i] = sample<DIM, false>(img, di, m, (float)c.x, (float)c.y, (float)z, u[i], u[N + i],
                                DIM == 3 ? u[2 * N + i] : 0.0f);
  }
}

void launch_warp_image(const float* img, const GridInfo& gi, const float* u, const GridInfo& gv, float* out,
                       cudaStream_t s) {
  count_launch();
  Affine a = make_affine(gv, gi);
  const Map3 m = map3(gv.d);
  if (gv.d.dim == 3)
    k_warp_image<3><<<m.grid, 256, 0, s>>>(img, gi.d, a, u, gv.d, m.zb, out);
  else
    k_warp_image<2><<<m.grid, 256, 0, s>>>(img, gi.d, a, u, gv.d, m.zb, out);
}

// Nearest-neighbour variant (antsApplyTransforms -n NearestNeighbor): ITK's
// NearestNeighborInterpolateImageFunction reads, inside the buffer, the voxel at
// RoundHalfIntegerUp(c) = floor(c + 0.5) per axis.  Inside the buffer -0.5 <= c < n - 0.5, so the
// index is in [0, n - 1]; the clamp only absorbs the float rounding of c + 0.5 at the upper rim.
__device__ __forceinline__ int nearest_index(float c, int n) {
  const int i = (int)floorf(c + 0.5f);
  return min(max(i, 0), n - 1);
}

template <int DIM>
__global__ void __launch_bounds__(256) k_warp_image_nearest(const float* __restrict__ img, Dims di, Affine m,
                                                            const float* __restrict__ u, Dims dv, int zb,
                                                            float* __restrict__ out) {
  const Coord3 c = coord3(dv, zb, 1);
  if (!c.ok) return;
  const int N = (int)dv.N, nxy = dv.nx * dv.ny;
  for (int z = c.z0; z < c.z1; ++z) {
    const int i = z * nxy + c.y * dv.nx + c.x;
    float cx, cy, cz;
    map_point<DIM, false>(m, (float)c.x, (float)c.y, (float)z, u[i], u[N + i], DIM == 3 ? u[2 * N + i] : 0.0f, cx, cy,
                          cz);
    float v = 0.0f;
    if (inside_buffer<DIM>(di, cx, cy, cz)) {
      const int x = nearest_index(cx, di.nx), y = nearest_index(cy, di.ny);
      const int zz = DIM == 3 ? nearest_index(cz, di.nz) : 0;
      v = __ldg(img + (zz * di.ny + y) * di.nx + x);
    }
    out[i] = v;
  }
}

// Generic label interpolation (antsApplyTransforms -n GenericLabel[Linear]): ITK's
// LabelImageGenericInterpolateImageFunction returns the label whose indicator image interpolates
// highest; with linear interpolation that is the label with the largest sum of cell-corner weights,
// ties going to the smaller label.  The cell is the linear interpolator's (clamp-to-edge), so every
// corner offset is inside the image; at most 8 distinct labels per cell.
template <int DIM>
__global__ void __launch_bounds__(256) k_warp_image_label(const float* __restrict__ img, Dims di, Affine m,
                                                          const float* __restrict__ u, Dims dv, int zb,
                                                          float* __restrict__ out) {
  const Coord3 c = coord3(dv, zb, 1);
  if (!c.ok) return;
  const int N = (int)dv.N, nxy = dv.nx * dv.ny;
  for (int z = c.z0; z < c.z1; ++z) {
    const int i = z * nxy + c.y * dv.nx + c.x;
    float cx, cy, cz;
    map_point<DIM, false>(m, (float)c.x, (float)c.y, (float)z, u[i], u[N + i], DIM == 3 ? u[2 * N + i] : 0.0f, cx, cy,
                          cz);
    float v = 0.0f;
    if (inside_buffer<DIM>(di, cx, cy, cz)) {
      const Cell cl = make_cell<DIM>(di, cx, cy, cz);
      float lab[8], acc[8];
      int n = 0;
#pragma unroll
      for (int k = 0; k < (DIM == 3 ? 8 : 4); ++k) {
        const int bx = k & 1, by = (k >> 1) & 1, bz = (k >> 2) & 1;
        const int o = cl.o000 + (bx ? cl.dx : 0) + (by ? cl.dy : 0) + (bz ? cl.dz : 0);
        const float w = (bx ? cl.wx : 1.0f - cl.wx) * (by ? cl.wy : 1.0f - cl.wy) *
                        (DIM == 3 ? (bz ? cl.wz : 1.0f - cl.wz) : 1.0f);
        const float l = __ldg(img + o);
        int j = 0;
        while (j < n && lab[j] != l) ++j;
        if (j == n) {
          lab[n] = l;
          acc[n] = 0.0f;
          ++n;
        }
        acc[j] += w;
      }
      int best = 0;
      for (int j = 1; j < n; ++j)
        if (acc[j] > acc[best] || (acc[j] == acc[best] && lab[j] < lab[best])) best = j;
      v = lab[best];
    }
    out[i] = v;
  }
}

// out = u + M w per voxel, fields as component planes (out may alias u or w: each voxel is read
// before it is written, by the same thread).  A transform stack's composition step for a linear
// transform (u = T(x) - x, M = A) or for a field sampled from its own grid (u = d(x + w), M = I).
struct AffineUpdate {
  float M[9];
};

template <int DIM>
__global__ void __launch_bounds__(256) k_field_affine_update(const float* u, const float* w, AffineUpdate a,
                                                             long long N, float* out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    float wv[3] = {w[i], w[N + i], DIM == 3 ? w[2 * N + i] : 0.0f};
    float uv[3] = {u[i], u[N + i], DIM == 3 ? u[2 * N + i] : 0.0f};
#pragma unroll
    for (int r = 0; r < DIM; ++r) {
      float s = uv[r];
#pragma unroll
      for (int k = 0; k < DIM; ++k) s = fmaf(a.M[r * 3 + k], wv[k], s);
      out[r * N + i] = s;
    }
  }
}

void launch_field_affine_update(const float* u, const float* w, const double M[9], int dim, long long N, float* out,
                                cudaStream_t s) {
  count_launch();
  AffineUpdate a;
  for (int k = 0; k < 9; ++k) a.M[k] = (float)M[k];
  const int blocks = grid_for(N, 256);
  if (dim == 3)
    k_field_affine_update<3><<<blocks, 256, 0, s>>>(u, w, a, N, out);
  else
    k_field_affine_update<2><<<blocks, 256, 0, s>>>(u, w, a, N, out);
}

void launch_warp_image_label(const float* img, const GridInfo& gi, const float* u, const GridInfo& gv, float* out,
                             cudaStream_t s) {
  count_launch();
  Affine a = make_affine(gv, gi);
  const Map3 m = map3(gv.d);
  if (gv.d.dim == 3)
    k_warp_image_label<3><<<m.grid, 256, 0, s>>>(img, gi.d, a, u, gv.d, m.zb, out);
  else
    k_warp_image_label<2><<<m.grid, 256, 0, s>>>(img, gi.d, a, u, gv.d, m.zb, out);
}

void launch_warp_image_nearest(const float* img, const GridInfo& gi, const float* u, const GridInfo& gv, float* out,
                               cudaStream_t s) {
  count_launch();
  Affine a = make_affine(gv, gi);
  const Map3 m = map3(gv.d);
  if (gv.d.dim == 3)
    k_warp_image_nearest<3><<<m.grid, 256, 0, s>>>(img, gi.d, a, u, gv.d, m.zb, out);
  else
    k_warp_image_nearest<2><<<m.grid, 256, 0, s>>>(img, gi.d, a, u, gv.d, m.zb, out);
}

// Metric-mask validity of the virtual voxels (antsRegistration -x [fixedMask,movingMask]): SyN
// resamples each mask into the virtual domain through its image's inverse half-field, nearest
// neighbour with 0 outside (ITK's NearestNeighborInterpolateImageFunction: the voxel at
// floor(c + 0.5) inside the buffer), and a voxel is valid where both are nonzero.  A null mask
// counts as inside everywhere.
template <int DIM>
__global__ void __launch_bounds__(256) k_mask_validity(const unsigned char* __restrict__ mF, Dims dF, Affine aF,
                                                       const float* __restrict__ psiF,
                                                       const unsigned char* __restrict__ mM, Dims dM, Affine aM,
                                                       const float* __restrict__ psiM, Dims dv, int zb,
                                                       unsigned char* __restrict__ valid, IterCtl* ctl) {
  griddep_wait();
  if (ctl != nullptr && ctl->stop) return;
  const Coord3 c = coord3(dv, zb, 1);
  if (!c.ok) return;
  const int N = (int)dv.N, nxy = dv.nx * dv.ny;
  auto inside = [&](const unsigned char* m, const Dims& dm, const Affine& a, const float* u, int i, int z) -> bool {
    if (m == nullptr) return true;
    float cx, cy, cz;
    map_point<DIM, false>(a, (float)c.x, (float)c.y, (float)z, u[i], u[N + i], DIM == 3 ? u[2 * N + i] : 0.0f, cx,
                          cy, cz);
    if (!inside_buffer<DIM>(dm, cx, cy, cz)) return false;
    const int x = nearest_index(cx, dm.nx), y = nearest_index(cy, dm.ny);
    const int zz = DIM == 3 ? nearest_index(cz, dm.nz) : 0;
    return __ldg(m + (zz * dm.ny + y) * dm.nx + x) != 0;
  };
  for (int z = c.z0; z < c.z1; ++z) {
    const int i = z * nxy + c.y * dv.nx + c.x;
    valid[i] = (inside(mF, dF, aF, psiF, i, z) && inside(mM, dM, aM, psiM, i, z)) ? 1 : 0;
  }
}

void launch_mask_validity(const unsigned char* mF, const GridInfo& gmF, const float* psiF, const unsigned char* mM,
                          const GridInfo& gmM, const float* psiM, const GridInfo& gv, unsigned char* valid,
                          IterCtl* ctl, cudaStream_t s) {
  count_launch();
  const Affine aF = make_affine(gv, gmF), aM = make_affine(gv, gmM);
  const Map3 m = map3(gv.d);
  if (gv.d.dim == 3)
    launch_k(k_mask_validity<3>, m.grid, 256, 0, s, mF, gmF.d, aF, psiF, mM, gmM.d, aM, psiM, gv.d, m.zb, valid, ctl);
  else
    launch_k(k_mask_validity<2>, m.grid, 256, 0, s, mF, gmF.d, aF, psiF, mM, gmM.d, aM, psiM, gv.d, m.zb, valid, ctl);
}

// ------------------------------------------------------------------------------------------
// Gaussian smoothing of displacement fields: an xy kernel (one block per tile, slice and field)
// and, in 3-D, a z kernel (one thread per column chunk).  The SyN epilogue (boundary zeroing,
// blend for small variances) and the max ||u/h|| reduction run in the last pass.
// ------------------------------------------------------------------------------------------
// rows of the standalone xy smoothing tile: 32 x 64 (2R halo rows per 64 output rows); measured at
// full resolution (R = 6): 231 / 229 / 207 us for 16 / 32 / 64 rows
constexpr int kSmoothTileY = 64;

template <int DIM, int R>
__global__ void __launch_bounds__(256) k_smooth_xy(const Smooth3Args a, Dims d, IterCtl* ctl, int rev) {
  griddep_wait();
  if (ctl != nullptr && ctl->stop) return;
  extern __shared__ __align__(16) float sm3[];
  __shared__ float red[32];
  const uint3 b = sweep_block(rev);
  const int h = b.z / d.nz;
  const int z = b.z - h * d.nz;
  const float mx = smooth_xy_tile<DIM, R, kSmoothTileY, TileLoad::Batched>(a, d, b.x, b.y, z, h, sm3);
  if (DIM == 2 && a.do_max) {
    const float bm = block_max_f(mx, red);
    if (threadIdx.x == 0) atomic_max_nonneg(&ctl->maxnorm[h], bm);
  }
}

// 3-D xy smoothing over a chunk of ZC slices per block, the halo tiles double-buffered: the tile of
// the next slice is copied in with cp.async while the current one is convolved, so the load latency
// overlaps the arithmetic instead of stalling each block between its barriers.  Writes the
// xy-smoothed fields for the z kernel; the arithmetic is k_smooth_xy's (the same bits).
template <int R, int TY>
__global__ void __launch_bounds__(256) k_smooth_xy_pipe(const Smooth3Args a, Dims d, IterCtl* ctl) {
  griddep_wait();
  if (ctl != nullptr && ctl->stop) return;
  constexpr int HX = 32 + 2 * R, HXP = (HX + 3) & ~3, HY = TY + 2 * R, RPT = TY / 8;
  constexpr int TILE = 3 * HY * HXP;
  extern __shared__ __align__(16) float smp[];
  float* xsum = smp + 2 * TILE;
  const int nzc = gridDim.z / a.halves;
  const int h = blockIdx.z / nzc, zc = blockIdx.z - h * nzc;
  const int z0 = zc * a.ZC, z1 = min(z0 + a.ZC, d.nz);
  if (z0 >= z1) return;  // the same for every thread of the block
  const int nx = d.nx, ny = d.ny, nxy = nx * ny, N = (int)d.N;
  float* __restrict__ dst = h ? a.out.p[1] : a.out.p[0];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int ox = blockIdx.x * 32 + tx, oy0 = blockIdx.y * TY + ty * RPT;
  smooth_xy_load_tile<3, R, TY, TileLoad::Async>(a, d, blockIdx.x, blockIdx.y, z0, h, smp);
  cp_async_commit();
  for (int z = z0; z < z1; ++z) {
    const int k = z - z0;
    if (z + 1 < z1) {
      // buffer (k + 1) & 1 was last read by the convolution of slice z - 1, which ended in a barrier
      smooth_xy_load_tile<3, R, TY, TileLoad::Async>(a, d, blockIdx.x, blockIdx.y, z + 1, h, smp + ((k + 1) & 1) * TILE);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    float y[3][RPT];
    smooth_xy_convolve<3, R, TY>(a, smp + (k & 1) * TILE, xsum, y);
    if (ox < nx) {
#pragma unroll
      for (int r = 0; r < RPT; ++r) {
        const int oy = oy0 + r;
        if (oy >= ny) break;
        const int i = z * nxy + oy * nx + ox;
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[c * N + i] = y[c][r];
      }
    }
  }
}

size_t smooth_xy_pipe_smem_bytes(int R, int TY) {
  const int HXP = (32 + 2 * R + 3) & ~3, HY = TY + 2 * R;
  return (size_t)(2 * 3 * HY * HXP + 3 * HY * 32) * sizeof(float);
}

template <int R>
// the ring lives in shared memory ((2R+1) x 3 x 256 floats, smooth_z_smem_bytes), so few registers
// are needed: 5 resident blocks per SM up to R = 6 (40 KB of ring each), 3 up to R = 12
__global__ void __launch_bounds__(kSmoothZThreads, (R <= 6 ? 5 : 3))
    k_smooth_z(const Smooth3Args a, Dims d, IterCtl* ctl, int rev) {
  griddep_wait();
  if (ctl != nullptr && ctl->stop) return;
  extern __shared__ float zring[];
  __shared__ float red[32];
  const uint3 b = sweep_block(rev);
  const int nzc = gridDim.z / a.halves;
  const int h = b.z / nzc;
  const int zc = b.z - h * nzc;
  const float mx = smooth_z_column_smem<R>(a, d, b.x, b.y, zc, h, zring);
  if (a.do_max) {
    const float bm = block_max_f(mx, red);
    if (threadIdx.x == 0) atomic_max_nonneg(&ctl->maxnorm[h], bm);
  }
}

// Fused 3-D smoothing: xy and z in one pass over a slab.  A block owns a 32 x TY tile of columns of
// one half-field and a chunk of ZC output slices.  It convolves slices z0 - R .. z1 - 1 + R in xy
// (the xy kernel's shared-memory halo tile, replicate edges) and keeps the last 2R + 1 xy-smoothed
// slices in a shared-memory ring whose slots are thread-private (each thread's ring entries are its
// own outputs, so the ring needs no barrier); every output slice is then convolved along z from the
// ring, with the SyN epilogue and the max norm.  The xy intermediate never reaches global memory
// (48 B per voxel of traffic less than the two-kernel path), at the price of recomputing the 2R halo
// slices of each chunk.  The arithmetic and its order are those of the two-kernel path: the same bits.
template <int R, int TY>
__global__ void __launch_bounds__(256) k_smooth_slab(const Smooth3Args a, Dims d, IterCtl* ctl) {
  griddep_wait();
  if (ctl != nullptr && ctl->stop) return;
  constexpr int K = 2 * R + 1, RPT = TY / 8;
  extern __shared__ __align__(16) float sms[];
  float* ring = sms + smooth3_smem_floats(3, R, TY);  // [K][3][RPT][256]
  __shared__ float red[32];
  const int nzc = gridDim.z / a.halves;
  const int h = blockIdx.z / nzc;
  const int zc = blockIdx.z - h * nzc;
  const int nx = d.nx, ny = d.ny, nz = d.nz, nxy = nx * ny, N = (int)d.N;
  const int z0 = zc * a.ZC, z1 = min(z0 + a.ZC, nz);
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int ox = blockIdx.x * 32 + tx, oy0 = blockIdx.y * TY + ty * RPT;
  float* __restrict__ dst = h ? a.out.p[1] : a.out.p[0];
  const float* __restrict__ org = h ? a.orig.p[1] : a.orig.p[0];
  const bool xedge = ox == 0 || ox == nx - 1;
  float mx = 0.0f;
  int sq = 0;  // ring slot of slice zs: (zs - z0 + R) mod K
  for (int zs = z0 - R; zs < z1 + R; ++zs) {
    float y[3][RPT];
    smooth_xy_compute<3, R, TY>(a, d, blockIdx.x, blockIdx.y, min(max(zs, 0), nz - 1), h, sms, y);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = 0; r < RPT; ++r) ring[((sq * 3 + c) * RPT + r) * 256 + tid] = y[c][r];
    sq = sq == K - 1 ? 0 : sq + 1;  // now the slot of slice zs + 1, i.e. of slice z - R below
    const int z = zs - R;  // output slice whose window z - R .. z + R is complete
    if (z >= z0 && ox < nx) {
#pragma unroll
      for (int r = 0; r < RPT; ++r) {
        const int oy = oy0 + r;
        if (oy >= ny) break;
        const int i = z * nxy + oy * nx + ox;
        const bool edge = a.epilogue && (xedge || oy == 0 || oy == ny - 1 || z == 0 || z == nz - 1);
        float nrm2 = 0.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float acc = 0.0f;
          int s2 = sq;
#pragma unroll
          for (int j = 0; j < K; ++j) {
            acc = fmaf(a.k[2][j], ring[((s2 * 3 + c) * RPT + r) * 256 + tid], acc);
            s2 = s2 == K - 1 ? 0 : s2 + 1;
          }
          if (a.epilogue) {
            if (edge) acc = 0.0f;
            else if (a.w2 != 0.0f) acc = acc * a.w1 + org[c * N + i] * a.w2;
          }
          const float qv = acc * a.ih[c];
          nrm2 += qv * qv;
          dst[c * N + i] = acc;
        }
        mx = fmaxf(mx, sqrtf(nrm2));
      }
    }
  }
  if (a.do_max) {
    const float bm = block_max_f(mx, red);
    if (threadIdx.x == 0) atomic_max_nonneg(&ctl->maxnorm[h], bm);
  }
}

size_t smooth_slab_smem_bytes(int R, int TY) {
  return (smooth3_smem_floats(3, R, TY) + (size_t)(2 * R + 1) * 3 * (TY / 8) * 256) * sizeof(float);
}

static int smooth3_radius(int dim, const int R[3]) {
  int r = 0;
  for (int a = 0; a < dim; ++a) r = std::max(r, R[a]);
  return std::max(r, 1);
}

bool smooth3_supported(int dim, const int R[3]) { return smooth3_radius(dim, R) <= kSmoothRMax; }

static size_t smooth_z_smem_bytes(int R) { return (size_t)(2 * R + 1) * 3 * kSmoothZThreads * sizeof(float); }

template <int R>
static cudaError_t smooth3_attr_both() {
  cudaError_t e = cudaFuncSetAttribute(k_smooth_xy<3, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(smooth3_smem_floats(3, R, kSmoothTileY) * 4));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_smooth_xy<2, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(smooth3_smem_floats(2, R, kSmoothTileY) * 4));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_smooth_z<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smooth_z_smem_bytes(R));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_smooth_xy_pipe<R, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smooth_xy_pipe_smem_bytes(R, 32));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_smooth_xy_pipe<R, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smooth_xy_pipe_smem_bytes(R, 64));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_smooth_slab<R, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smooth_slab_smem_bytes(R, 8));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_smooth_slab<R, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smooth_slab_smem_bytes(R, 16));
  return e;
}

cudaError_t smooth3_prepare() {
  cudaError_t e = cudaSuccess;
  e = e ? e : smooth3_attr_both<1>();
  e = e ? e : smooth3_attr_both<2>();
  e = e ? e : smooth3_attr_both<3>();
  e = e ? e : smooth3_attr_both<4>();
  e = e ? e : smooth3_attr_both<5>();
  e = e ? e : smooth3_attr_both<6>();
  e = e ? e : smooth3_attr_both<7>();
  e = e ? e : smooth3_attr_both<8>();
  e = e ? e : smooth3_attr_both<9>();
  e = e ? e : smooth3_attr_both<10>();
  e = e ? e : smooth3_attr_both<11>();
  e = e ? e : smooth3_attr_both<12>();
  return e;
}

Smooth3Args make_smooth_args(const float* const* in, float* const* out, const float* const* orig, int halves,
                             const GridInfo& g, const float* const khost[3], const int R[3], bool epilogue, float w1,
                             float w2, bool maxnorm, int* radius) {
  const int dim = g.d.dim;
  const int RR = smooth3_radius(dim, R);
  Smooth3Args a;
  memset(&a, 0, sizeof(a));
  a.in = Ptr2c{{in[0], halves > 1 ? in[1] : in[0]}};
  a.out = Ptr2{{out[0], halves > 1 ? out[1] : out[0]}};
  a.orig = Ptr2c{{orig ? orig[0] : nullptr, orig ? (halves > 1 ? orig[1] : orig[0]) : nullptr}};
  for (int ax = 0; ax < 3; ++ax) {
    a.ih[ax] = (float)(1.0 / g.sp[ax]);
    if (ax < dim) {
      for (int j = 0; j <= 2 * R[ax]; ++j) a.k[ax][RR - R[ax] + j] = khost[ax][j];
    } else {
      a.k[ax][RR] = 1.0f;
    }
  }
  a.halves = halves;
  a.epilogue = epilogue ? 1 : 0;
  a.do_max = maxnorm ? 1 : 0;
  a.w1 = w1;
  a.w2 = w2;
  *radius = RR;
  return a;
}

int smooth_z_chunk(const Dims& d, int halves, int RR, int slots) {
  // z chunk of one column walk of the level kernel's z phase: minimises the waves of walks over
  // `slots` blocks times the work of a walk (its slices plus the ring fill, 2R loads, about R
  // slices)
  const int cols = ((d.nx + 31) / 32) * ((d.ny + 7) / 8) * halves;
  int best_zc = d.nz;
  double best = -1.0;
  for (int zc = 1; zc <= d.nz; ++zc) {
    const long long blocks = (long long)cols * ((d.nz + zc - 1) / zc);
    const double cost = (double)((blocks + slots - 1) / slots) * (zc + RR);
    if (best < 0 || cost < best) {
      best = cost;
      best_zc = zc;
    }
  }
  return best_zc;
}

// Slab plan of the fused 3-D smoothing: tile rows (8 or 16) and output slices per block; 0 = the
// two-kernel path.  The chunk is chosen by waves of resident blocks times the slices a block
// convolves in xy (its chunk plus the 2R halo slices), unless a plan fixes it.
static int slab_chunk(const Dims& d, int halves, int R, int TY) {
  const size_t smem = smooth_slab_smem_bytes(R, TY);
  int per_sm = (int)std::min<size_t>(8, (227 * 1024) / (smem + 1024));
  if (per_sm < 1) per_sm = 1;
  const int slots = 148 * per_sm;
  const int cols = ((d.nx + 31) / 32) * ((d.ny + TY - 1) / TY) * halves;
  int best_zc = d.nz;
  double best = -1.0;
  for (int zc = 1; zc <= d.nz; ++zc) {
    const long long blocks = (long long)cols * ((d.nz + zc - 1) / zc);
    const double cost = (double)((blocks + slots - 1) / slots) * (zc + 2 * R);
    if (best < 0 || cost < best) {
      best = cost;
      best_zc = zc;
    }
  }
  return best_zc;
}

static void launch_smooth_slab(const Smooth3Args& a0, const GridInfo& g, int RR, int TY, int ZC, IterCtl* ctl,
                               cudaStream_t s) {
  Smooth3Args a = a0;
  a.ZC = ZC > 0 ? std::min(ZC, g.d.nz) : slab_chunk(g.d, a.halves, RR, TY);
  const dim3 grid((g.d.nx + 31) / 32, (g.d.ny + TY - 1) / TY, ((g.d.nz + a.ZC - 1) / a.ZC) * a.halves);
  const size_t smem = smooth_slab_smem_bytes(RR, TY);
  count_launch();
#define SYNX_SSLAB(RV)                                                              \
  case RV:                                                                          \
    if (TY == 16)                                                                   \
      launch_k(k_smooth_slab<RV, 16>, grid, 256, smooth_slab_smem_bytes(RV, 16), s, a, g.d, ctl); \
    else                                                                            \
      launch_k(k_smooth_slab<RV, 8>, grid, 256, smooth_slab_smem_bytes(RV, 8), s, a, g.d, ctl);   \
    break;
  (void)smem;
  switch (RR) {
    SYNX_SSLAB(1)
    SYNX_SSLAB(2)
    SYNX_SSLAB(3)
    SYNX_SSLAB(4)
    SYNX_SSLAB(5)
    SYNX_SSLAB(6)
    SYNX_SSLAB(7)
    SYNX_SSLAB(8)
    SYNX_SSLAB(9)
    SYNX_SSLAB(10)
    SYNX_SSLAB(11)
    SYNX_SSLAB(12)
    default:
      break;
  }
#undef SYNX_SSLAB
}

// Default: the xy and z kernels.  The autotuner measured the slab kernel slower at every level of
// the 182x218x182 pyramid (a block's slices are convolved one after another, three barriers each,
// with too few blocks in flight), so it runs only where a tuning table picks it.
SmoothPlan g_smooth_plan{0, 0, 0};

void launch_smooth_field(const float* const* in, float* const* out, const float* const* orig, float* const* tmp,
                         int halves, const GridInfo& g, const float* const khost[3], const int R[3], bool epilogue,
                         float w1, float w2, bool maxnorm, IterCtl* ctl, cudaStream_t s, const SmoothPlan* plan) {
  const int dim = g.d.dim;
  const SmoothPlan P = plan ? *plan : g_smooth_plan;
  if (dim == 3 && P.slab_ty > 0) {
    int RR = 1;
    Smooth3Args a = make_smooth_args(in, out, orig, halves, g, khost, R, epilogue, w1, w2, maxnorm, &RR);
    launch_smooth_slab(a, g, RR, P.slab_ty, P.slab_zc, ctl, s);
    return;
  }
  int RR = 1;
  Smooth3Args a = make_smooth_args(in, dim == 3 ? tmp : out, orig, halves, g, khost, R, epilogue, w1, w2, maxnorm, &RR);
  // xy tiles are 32 x kSmoothTileY; the z pass below keeps 32 x 8 columns
  const int gx = (g.d.nx + 31) / 32, gy = (g.d.ny + 7) / 8;
  if (dim == 3 && (P.xy_ty == 32 || P.xy_ty == 64)) {
    // the pipelined xy kernel: chunks of slices per block by waves of resident blocks times the
    // slices a block walks (plus one for the pipeline's fill)
    const int TY = P.xy_ty;
    const size_t smem = smooth_xy_pipe_smem_bytes(RR, TY);
    const int per_sm = std::max(1, (int)std::min<size_t>(8, (227 * 1024) / (smem + 1024)));
    const int cols = gx * ((g.d.ny + TY - 1) / TY) * halves;
    int best_zc = g.d.nz;
    double best = -1.0;
    for (int zc = 1; zc <= g.d.nz; ++zc) {
      const long long blocks = (long long)cols * ((g.d.nz + zc - 1) / zc);
      const double cost = (double)((blocks + 148 * per_sm - 1) / (148 * per_sm)) * (zc + 1);
      if (best < 0 || cost < best) {
        best = cost;
        best_zc = zc;
      }
    }
    Smooth3Args ap = a;
    ap.ZC = best_zc;
    const dim3 gp(gx, (g.d.ny + TY - 1) / TY, ((g.d.nz + best_zc - 1) / best_zc) * halves);
    count_launch();
#define SYNX_SXYP(RV)                                                                           \
  case RV:                                                                                      \
    if (TY == 64)                                                                               \
      launch_k(k_smooth_xy_pipe<RV, 64>, gp, 256, smooth_xy_pipe_smem_bytes(RV, 64), s, ap, g.d, ctl); \
    else                                                                                        \
      launch_k(k_smooth_xy_pipe<RV, 32>, gp, 256, smooth_xy_pipe_smem_bytes(RV, 32), s, ap, g.d, ctl); \
    break;
    switch (RR) {
      SYNX_SXYP(1)
      SYNX_SXYP(2)
      SYNX_SXYP(3)
      SYNX_SXYP(4)
      SYNX_SXYP(5)
      SYNX_SXYP(6)
      SYNX_SXYP(7)
      SYNX_SXYP(8)
      SYNX_SXYP(9)
      SYNX_SXYP(10)
      SYNX_SXYP(11)
      SYNX_SXYP(12)
      default:
        break;
    }
#undef SYNX_SXYP
  } else {
  const dim3 gxy(gx, (g.d.ny + kSmoothTileY - 1) / kSmoothTileY, g.d.nz * halves);
  const size_t smem = smooth3_smem_floats(dim, RR, kSmoothTileY) * 4;
  count_launch();
#define SYNX_SXY(RV)                                             \
  case RV:                                                       \
    if (dim == 3)                                                \
      launch_k(k_smooth_xy<3, RV>, gxy, 256, smem, s, a, g.d, ctl, t_rev);    \
    else                                                         \
      launch_k(k_smooth_xy<2, RV>, gxy, 256, smem, s, a, g.d, ctl, t_rev);    \
    break;
  switch (RR) {
    SYNX_SXY(1)
    SYNX_SXY(2)
    SYNX_SXY(3)
    SYNX_SXY(4)
    SYNX_SXY(5)
    SYNX_SXY(6)
    SYNX_SXY(7)
    SYNX_SXY(8)
    SYNX_SXY(9)
    SYNX_SXY(10)
    SYNX_SXY(11)
    SYNX_SXY(12)
    default:
      break;
  }
#undef SYNX_SXY
  }
  if (dim != 3) return;
  // z pass: tmp -> out with the epilogue
  a.in = Ptr2c{{tmp[0], halves > 1 ? tmp[1] : tmp[0]}};
  a.out = Ptr2{{out[0], halves > 1 ? out[1] : out[0]}};
  {
    // about 8 column walks per SM of at least 2R + 1 slices (longer walks measured slower here)
    const int cols = gx * gy * halves;
    const int chunks = std::max(1, (148 * 8 + cols - 1) / cols);
    a.ZC = std::min(std::max((g.d.nz + chunks - 1) / chunks, 2 * RR + 1), g.d.nz);
  }
  const dim3 gz(gx, gy, ((g.d.nz + a.ZC - 1) / a.ZC) * halves);
  count_launch();
#define SYNX_SZ(RV)                                    \
  case RV:                                             \
    launch_k(k_smooth_z<RV>, gz, kSmoothZThreads, smooth_z_smem_bytes(RV), s, a, g.d, ctl, t_rev ^ 1); \
    break;
  switch (RR) {
    SYNX_SZ(1)
    SYNX_SZ(2)
    SYNX_SZ(3)
    SYNX_SZ(4)
    SYNX_SZ(5)
    SYNX_SZ(6)
    SYNX_SZ(7)
    SYNX_SZ(8)
    SYNX_SZ(9)
    SYNX_SZ(10)
    SYNX_SZ(11)
    SYNX_SZ(12)
    default:
      break;
  }
#undef SYNX_SZ
}


// Single-axis fallback for kernels too wide for the fused pass.
template <int DIM>
__global__ void __launch_bounds__(256)
    k_smooth_pass(Ptr2c in, Ptr2 out, Ptr2c orig, Dims d, int zb, int axis, const float* __restrict__ coeffs, int R,
                  int last, float w1, float w2, int do_max, float ihx, float ihy, float ihz, IterCtl* ctl) {
  griddep_wait();
  if (ctl != nullptr && ctl->stop) return;
  __shared__ float red[32];
  const Coord3 c3 = coord3(d, zb, gridDim.z / ((d.nz + zb - 1) / zb));
  const int h = c3.h;
  const float* __restrict__ src = (h ? in.p[1] : in.p[0]);
  float* __restrict__ dst = (h ? out.p[1] : out.p[0]);
  const float* __restrict__ org = (h ? orig.p[1] : orig.p[0]);
  const int N = (int)d.N, nxy = d.nx * d.ny;
  const int len = axis == 0 ? d.nx : (axis == 1 ? d.ny : d.nz);
  const int astride = axis == 0 ? 1 : (axis == 1 ? d.nx : nxy);
  const float ih[3] = {ihx, ihy, ihz};
  float mx = 0.0f;
  if (c3.ok) {
    for (int z = c3.z0; z < c3.z1; ++z) {
      const int i = z * nxy + c3.y * d.nx + c3.x;
      const int pos = axis == 0 ? c3.x : (axis == 1 ? c3.y : z);
      const bool edge = last && (c3.x == 0 || c3.x == d.nx - 1 || c3.y == 0 || c3.y == d.ny - 1 ||
                                 (DIM == 3 && (z == 0 || z == d.nz - 1)));
      float nrm2 = 0.0f;
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        const float* line = src + c * N + i - pos * astride;
        float s = 0.0f;
        for (int j = 0; j <= 2 * R; ++j) {
          const int qq = min(max(pos + j - R, 0), len - 1);
          s = fmaf(__ldg(coeffs + j), __ldg(line + qq * astride), s);
        }
        if (last) {
          if (edge) s = 0.0f;
          else if (w2 != 0.0f) s = s * w1 + org[c * N + i] * w2;
        }
        if (do_max) {
          const float v = s * ih[c];
          nrm2 += v * v;
        }
        dst[c * N + i] = s;
      }
      if (do_max) mx = fmaxf(mx, sqrtf(nrm2));
    }
  }
  if (do_max) {
    float bm = block_max_f(mx, red);
    if (threadIdx.x == 0) atomic_max_nonneg(&ctl->maxnorm[h], bm);
  }
}

void launch_smooth_field_pass(const float* const* in, float* const* out, const float* const* orig, int halves,
                              const GridInfo& g, int axis, const float* coeffs, int R, bool last, float w1, float w2,
                              bool maxnorm, IterCtl* ctl, cudaStream_t s) {
  count_launch();
  Ptr2c pi{{in[0], halves > 1 ? in[1] : in[0]}};
  Ptr2 po{{out[0], halves > 1 ? out[1] : out[0]}};
  Ptr2c pg{{orig ? orig[0] : nullptr, orig ? (halves > 1 ? orig[1] : orig[0]) : nullptr}};
  const Map3 m = map3(g.d, halves);
  float ih[3] = {(float)(1.0 / g.sp[0]), (float)(1.0 / g.sp[1]), (float)(1.0 / g.sp[2])};
  if (g.d.dim == 3)
    launch_k(k_smooth_pass<3>, m.grid, 256, 0, s, pi, po, pg, g.d, m.zb, axis, coeffs, R, last ? 1 : 0, w1, w2,
                                            maxnorm ? 1 : 0, ih[0], ih[1], ih[2], ctl);
  else
    launch_k(k_smooth_pass<2>, m.grid, 256, 0, s, pi, po, pg, g.d, m.zb, axis, coeffs, R, last ? 1 : 0, w1, w2,
                                            maxnorm ? 1 : 0, ih[0], ih[1], ih[2], ctl);
}


// ------------------------------------------------------------------------------------------
// Composition (one tile per block, both halves by blockIdx.z).
// ------------------------------------------------------------------------------------------
template <int DIM, bool DIAG>
__global__ void __launch_bounds__(256) k_compose(const ComposeArgs a, int halves, IterCtl* ctl, int rev) {
  griddep_wait();
  if (ctl != nullptr && ctl->stop) return;
  const uint3 b = sweep_block(rev);
  const int gz = gridDim.z / halves;
  const int h = b.z / gz;
  compose_tile<DIM, DIAG>(a, ctl, h, b.x, b.y, b.z - h * gz);
}

void launch_compose(const float* const* d, const float* const* w, float* const* out, int halves, const GridInfo& g,
                    float eta, IterCtl* ctl, cudaStream_t s) {
  count_launch();
  ComposeArgs a;
  a.d = Ptr2c{{d[0], halves > 1 ? d[1] : d[0]}};
  a.w = Ptr2c{{w[0], halves > 1 ? w[1] : w[0]}};
  a.o = Ptr2{{out[0], halves > 1 ? out[1] : out[0]}};
  a.g = g.d;
  a.m = make_affine(g, g);
  a.eta = (double)eta;
  const Map3 m = map3(g.d, halves);
  a.zb = m.zb;
  const bool dg = affine_diag(a.m);
  if (g.d.dim == 3) {
    if (dg) launch_k(k_compose<3, true>, m.grid, 256, 0, s, a, halves, ctl, t_rev);
    else launch_k(k_compose<3, false>, m.grid, 256, 0, s, a, halves, ctl, t_rev);
  } else {
    if (dg) launch_k(k_compose<2, true>, m.grid, 256, 0, s, a, halves, ctl, t_rev);
    else launch_k(k_compose<2, false>, m.grid, 256, 0, s, a, halves, ctl, t_rev);
  }
}

// ------------------------------------------------------------------------------------------
// Fused fixed-point inverse.  Launch k applies iteration k (statistics from launch k-1) and,
// if iteration k+1 is due, computes its residual statistics from the updated iterate, so each
// sub-iteration streams the iterate once.  The loop condition lives on the device
// (InvCtl.exec), so all max_iter+1 launches are enqueued up front and the ones past
// convergence return at once.
// ------------------------------------------------------------------------------------------
struct InvLaunch {
  int k, max_iter, phase, stop_aware, halves;
  int tx, ty, tz;  // 32 x 8 x zb tiles of one half
  double mean_tol, max_tol;
};

template <int DIM, bool DIAG>
__global__ void __launch_bounds__(256, 4) k_invert_step(const InvArgs a, InvLaunch L, IterCtl* ctl,
                                                        double* __restrict__ psum, float* __restrict__ pmax,
                                                        int pcap) {
  griddep_wait();
  if (L.stop_aware && ctl->stop) return;
  __shared__ double redd[32];
  __shared__ float redf[32];
  __shared__ int am_last;
  // gridDim.x / halves blocks per half walk that half's tiles: one wave of blocks, so the
  // launches that find their half converged cost one short launch
  const int nb = gridDim.x / L.halves;
  const int h = blockIdx.x / nb;
  const int bid = blockIdx.x - h * nb;
  InvCtl& C = ctl->inv[L.phase][h];
  const int k = L.k >= 0 ? L.k : *(volatile const int*)&ctl->inv[L.phase][0].kdev;
  bool apply = false, stats = true;
  float eps = 0.0f, lim = 0.0f;
  if (k > 0) {
    const int s = k & 1;
    if (!C.exec[s]) {
      if (bid == 0 && threadIdx.x == 0) C.exec[s ^ 1] = 0;
      return;
    }
    apply = true;
    eps = k == 1 ? 0.75f : 0.5f;
    const float mx = C.maxv[s];
    const double mean = C.mean[s];
    lim = eps * mx;
    stats = (k + 1 <= L.max_iter) && ((double)mx > L.max_tol) && (mean > L.mean_tol);
    if (!stats && bid == 0 && threadIdx.x == 0) {
      C.exec[s ^ 1] = 0;
      C.iters = k;
    }
  }
  double acc = 0.0;
  float mxl = 0.0f;
  const int ntiles = L.tx * L.ty * L.tz;
  for (int t = bid; t < ntiles; t += nb) {
    const int bx = t % L.tx, r = t / L.tx;
    invert_tile<DIM, DIAG>(a, h, bx, r % L.ty, r / L.ty, apply, stats, eps, lim, acc, mxl);
  }
  if (!stats) return;
  const double bs = block_sum_d(acc, redd);
  const float bm = block_max_f(mxl, redf);
  if (threadIdx.x == 0) {
    psum[h * pcap + bid] = bs;
    pmax[h * pcap + bid] = bm;
    __threadfence();
    const unsigned t = atomicAdd(&C.counter, 1u);
    am_last = (t == (unsigned)nb - 1);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    double s = 0.0;
    float m = 0.0f;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      s += __ldcg(psum + h * pcap + b);
      m = fmaxf(m, __ldcg(pmax + h * pcap + b));
    }
    s = block_sum_d(s, redd);
    m = block_max_f(m, redf);
    if (threadIdx.x == 0) {
      const int s1 = (k + 1) & 1;
      C.mean[s1] = s / (double)a.g.N;
      C.maxv[s1] = m;
      C.exec[s1] = 1;
      C.iters = k;
      C.counter = 0u;
    }
  }
}

constexpr int kInvTarget = 148 * 24;    // tiles: short per-thread z walks
constexpr int kInvBlocksPerHalf = 296;  // 148 SMs x 4 resident blocks shared by two halves
int inv_blocks(const GridInfo& g) { return std::max(map3(g.d, 2, kInvTarget).nblocks, kInvBlocksPerHalf); }

InvArgs make_inv_args(const float* const* phi, float* const* psi, int halves, const GridInfo& g, int zb,
                      float* const* ecache) {
  InvArgs a;
  a.phi = Ptr2c{{phi[0], halves > 1 ? phi[1] : phi[0]}};
  a.psi = Ptr2{{psi[0], halves > 1 ? psi[1] : psi[0]}};
  a.ecache = ecache ? Ptr2{{ecache[0], halves > 1 ? ecache[1] : ecache[0]}} : Ptr2{{nullptr, nullptr}};
  a.g = g.d;
  const Affine m = make_affine(g, g);
  for (int j = 0; j < 9; ++j) a.A[j] = m.A[j];
  for (int j = 0; j < 3; ++j) a.ih[j] = (float)(1.0 / g.sp[j]);
  a.zb = zb;
  return a;
}

void launch_invert_step(const float* const* phi, float* const* psi, int halves, const GridInfo& g, int k, int max_iter,
                        double mean_tol, double max_tol, IterCtl* ctl, int phase, PartialBufs pb, cudaStream_t s,
                        bool stop_aware, float* const* ecache) {
  count_launch();
  // tiles of one half (the same decomposition for one or two halves); blocks per half: one
  // wave, at most the partial slots inv_blocks() sized
  const Map3 m2 = map3(g.d, 2, kInvTarget);
  const int tz = (int)m2.grid.z / 2;
  const int ntiles = (int)m2.grid.x * (int)m2.grid.y * tz;
  const int nb = std::max(1, std::min({ntiles, kInvBlocksPerHalf, pb.capacity}));
  const InvArgs a = make_inv_args(phi, psi, halves, g, m2.zb, ecache);
  InvLaunch L{k, max_iter, phase, stop_aware ? 1 : 0, halves, (int)m2.grid.x, (int)m2.grid.y, tz, mean_tol, max_tol};
  Affine am = make_affine(g, g);
  const bool dg = affine_diag(am);
  const dim3 grid((unsigned)(nb * halves));
  if (g.d.dim == 3) {
    if (dg) launch_k(k_invert_step<3, true>, grid, 256, 0, s, a, L, ctl, pb.sum, pb.maxv, pb.capacity);
    else launch_k(k_invert_step<3, false>, grid, 256, 0, s, a, L, ctl, pb.sum, pb.maxv, pb.capacity);
  } else {
    if (dg) launch_k(k_invert_step<2, true>, grid, 256, 0, s, a, L, ctl, pb.sum, pb.maxv, pb.capacity);
    else launch_k(k_invert_step<2, false>, grid, 256, 0, s, a, L, ctl, pb.sum, pb.maxv, pb.capacity);
  }
}

// ------------------------------------------------------------------------------------------
// Single-pass fixed-point inverse.  Sub-iteration k (k_invert_spec) evaluates the residual E_k of
// the iterate psi_k, its statistics, and the update of iteration k in the same pass:
// psi_{k+1} = psi_k + (-E_k f) eps_k with f = lim / ||E_k / h|| where that exceeds lim and 1
// elsewhere, lim = eps_k max ||E_k / h|| (ITK's clamp; eps 0.75 then 0.5; boundary voxels pinned
// to 0).  lim needs the maximum over the whole field, known only when the pass ends, but f = 1
// wherever ||E_k / h|| <= eps_k M for any lower bound M of that maximum.  Every thread keeps such
// a bound (its own running maximum and, through a global atomic maximum read at each tile, what the
// other blocks have seen so far) and updates those voxels at once; the rest keep psi_k, store E_k
// in the residual cache and append their index to a list, and k_invert_fix applies their updates
// with the final lim.  The two passes perform exactly the two-pass form's operations on the same
// values, so the results are bit-identical; the field is streamed once per sub-iteration instead of
// twice.  Control: S(k) runs when k = 0 or S(k-1) found the half not converged (exec[k & 1]); its
// last block decides exec[(k + 1) & 1] from the statistics and k + 1 < max_iter.
// ------------------------------------------------------------------------------------------
struct InvList {
  int* idx[2];
};

template <int DIM, bool DIAG>
__device__ __forceinline__ void invert_spec_tile(const InvArgs& a, int h, int bx, int by, int bz, float eps,
                                                 double& acc, float& mx, unsigned* gbound, int* __restrict__ list,
                                                 unsigned* lcount) {
  const Dims& d = a.g;
  const int x = bx * 32 + (threadIdx.x & 31), y = by * 8 + (threadIdx.x >> 5);
  // every lane of the warp arrives here; the lanes inside the grid walk the same slices below, so
  // they form one active set for the warp-wide list reservation and maximum
  const bool inside = x < d.nx && y < d.ny;
  const unsigned act = __ballot_sync(0xffffffffu, inside);
  if (!inside) return;
  const int lane = threadIdx.x & 31, leader = __ffs(act) - 1;
  const float* __restrict__ phi = h ? a.phi.p[1] : a.phi.p[0];
  float* __restrict__ psi = h ? a.psi.p[1] : a.psi.p[0];
  float* __restrict__ ec = h ? a.ecache.p[1] : a.ecache.p[0];
  const int z0 = bz * a.zb, z1 = min(z0 + a.zb, d.nz);
  const int N = (int)d.N, nxy = d.nx * d.ny;
  const float fx = (float)x, fy = (float)y;
  const bool xyedge = x == 0 || x == d.nx - 1 || y == 0 || y == d.ny - 1;
  const unsigned seen = __ldcg(gbound);
  float bound = fmaxf(mx, __uint_as_float(seen));
  const int i0 = z0 * nxy + y * d.nx + x;
  float pn[3] = {0.0f, 0.0f, 0.0f};
  if (z0 < z1) {
    pn[0] = psi[i0];
    pn[1] = psi[N + i0];
    pn[2] = DIM == 3 ? psi[2 * N + i0] : 0.0f;
  }
  for (int z = z0; z < z1; ++z) {
    const int i = z * nxy + y * d.nx + x;
    float p[3] = {pn[0], pn[1], pn[2]};
    if (z + 1 < z1) {
      pn[0] = psi[i + nxy];
      pn[1] = psi[N + i + nxy];
      pn[2] = DIM == 3 ? psi[2 * N + i + nxy] : 0.0f;
    }
    float e[3];
    inv_residual<DIM, DIAG>(phi, d, a.A, fx, fy, (float)z, p, e);
    float s2 = 0.0f;
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      const float v = e[c] * a.ih[c];
      s2 += v * v;
    }
    const float nrm = sqrtf(s2);
    acc += (double)nrm;
    mx = fmaxf(mx, nrm);
    bound = fmaxf(bound, nrm);
    const bool edge = xyedge || (DIM == 3 && (z == 0 || z == d.nz - 1));
    const bool now = edge || nrm <= eps * bound;  // f = 1 here whatever the final maximum
    if (now) {
      const float f = 1.0f;
#pragma unroll
      for (int c = 0; c < DIM; ++c) p[c] = edge ? 0.0f : p[c] + ((-e[c]) * f) * eps;
      psi[i] = p[0];
      psi[N + i] = p[1];
      if (DIM == 3) psi[2 * N + i] = p[2];
    } else {
      ec[i] = e[0];
      ec[N + i] = e[1];
      if (DIM == 3) ec[2 * N + i] = e[2];
    }
    // deferred voxels: list slots reserved once per warp
    const unsigned def = __ballot_sync(act, !now);
    if (def) {
      unsigned base = 0;
      if (lane == leader) base = atomicAdd(lcount, (unsigned)__popc(def));
      base = __shfl_sync(act, base, leader);
      if (!now) list[base + __popc(def & ((1u << lane) - 1u))] = i;
    }
  }
  // share the warp's maximum with the other blocks (non-negative floats order as their bits)
  const unsigned wmax = __reduce_max_sync(act, __float_as_uint(mx));
  if (lane == leader && wmax > seen) atomicMax(gbound, wmax);
}

// Resident blocks per SM of the single-pass inverse; a launch is one wave of them, shared by the two
// halves.  (3 blocks with up to 80 registers measured the same; staging the corner gathers in shared
// memory with cp.async, two voxels in flight per thread, took 328 instead of 224 us per full-resolution
// launch: more instructions per voxel and no gain in latency hiding.)
constexpr int kInvSpecBlocksPerSM = 4;

template <int DIM, bool DIAG>
__global__ void __launch_bounds__(256, kInvSpecBlocksPerSM) k_invert_spec(const InvArgs a, InvLaunch L, IterCtl* ctl,
                                                        double* __restrict__ psum, float* __restrict__ pmax, int pcap,
                                                        InvList list) {
  griddep_wait();
  if (L.stop_aware && ctl->stop) return;
  __shared__ double redd[32];
  __shared__ float redf[32];
  __shared__ int am_last;
  const int nb = gridDim.x / L.halves;
  const int h = blockIdx.x / nb;
  const int bid = blockIdx.x - h * nb;
  InvCtl& C = ctl->inv[L.phase][h];
  const int k = L.k >= 0 ? L.k : *(volatile const int*)&ctl->inv[L.phase][0].kdev;
  if (k > 0 && !*(volatile const int*)&C.exec[k & 1]) {
    if (bid == 0 && threadIdx.x == 0) C.exec[(k + 1) & 1] = 0;
    return;
  }
  const float eps = k == 0 ? 0.75f : 0.5f;
  // Seed the running bound before the tiles: one lane per warp evaluates the residual norm of the
  // current iterate at one voxel, exactly as the pass computes it, so the maximum of these is a lower
  // bound of the field's maximum.  The voxels lie in this block's own tiles (warp w samples the tile
  // w/8 of the way through the block's walk), which no other block writes and this one has not
  // started, so each sample is the residual of the iterate the pass starts from; a voxel of another
  // block's tile could already hold its update.  The blocks' walks interleave over the whole grid, so
  // the samples (~4700 at full resolution) spread over the field.  Without them the first tiles,
  // before any bound is known, defer most of their voxels; with one sample per thread the scattered
  // gathers cost more DRAM traffic than the deferrals they save.
  {
    float nrm = 0.0f;
    const int ntiles = L.tx * L.ty * L.tz;
    const int nw = blockDim.x >> 5, w = threadIdx.x >> 5;
    const int J = bid < ntiles ? (ntiles - 1 - bid) / nb + 1 : 0;  // tiles of this block's walk
    if ((threadIdx.x & 31) == 0 && J > 0) {
      const Dims& d = a.g;
      const int t = bid + (w * J / nw) * nb;
      const int bx = t % L.tx, r = t / L.tx, by = r % L.ty, bz = r / L.ty;
      const int x = bx * 32 + ((w * 13 + 5) & 31), y = by * 8 + (w & 7);
      const int z = bz * a.zb + (w * 3) % a.zb;
      if (x < d.nx && y < d.ny && z < d.nz) {
        const long long N = d.N;
        const long long j = ((long long)z * d.ny + y) * d.nx + x;
        const float* __restrict__ psi = h ? a.psi.p[1] : a.psi.p[0];
        const float* __restrict__ phi = h ? a.phi.p[1] : a.phi.p[0];
        float p[3] = {psi[j], psi[N + j], DIM == 3 ? psi[2 * N + j] : 0.0f};
        float e[3];
        inv_residual<DIM, DIAG>(phi, d, a.A, (float)x, (float)y, (float)z, p, e);
        float s2 = 0.0f;
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
          const float v = e[c] * a.ih[c];
          s2 += v * v;
        }
        nrm = sqrtf(s2);
      }
    }
    const float bm = block_max_f(nrm, redf);
    if (threadIdx.x == 0) atomicMax(&C.mrun, __float_as_uint(bm));
    __syncthreads();  // redf is reused by the reductions below
  }
  double acc = 0.0;
  float mxl = 0.0f;
  const int ntiles = L.tx * L.ty * L.tz;
  for (int t = bid; t < ntiles; t += nb) {
    const int bx = t % L.tx, r = t / L.tx;
    invert_spec_tile<DIM, DIAG>(a, h, bx, r % L.ty, r / L.ty, eps, acc, mxl, &C.mrun, list.idx[h], &C.lcount);
  }
  const double bs = block_sum_d(acc, redd);
  const float bm = block_max_f(mxl, redf);
  if (threadIdx.x == 0) {
    psum[h * pcap + bid] = bs;
    pmax[h * pcap + bid] = bm;
    __threadfence();
    const unsigned t = atomicAdd(&C.counter, 1u);
    am_last = (t == (unsigned)nb - 1);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    double sm = 0.0;
    float m = 0.0f;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      sm += __ldcg(psum + h * pcap + b);
      m = fmaxf(m, __ldcg(pmax + h * pcap + b));
    }
    sm = block_sum_d(sm, redd);
    m = block_max_f(m, redf);
    if (threadIdx.x == 0) {
      const double mean = sm / (double)a.g.N;
      C.maxk[k & 1] = m;
      C.mean[(k + 1) & 1] = mean;
      C.maxv[(k + 1) & 1] = m;
      C.exec[(k + 1) & 1] = (k + 1 < L.max_iter && (double)m > L.max_tol && mean > L.mean_tol) ? 1 : 0;
      C.iters = k + 1;
      C.counter = 0u;
    }
  }
}

// The deferred updates of sub-iteration k: psi = psi + (-E f) eps with the final clamp.  The last
// block to finish clears the list and the running bound for the next sub-iteration.
template <int DIM>
__global__ void __launch_bounds__(256) k_invert_fix(const InvArgs a, InvLaunch L, IterCtl* ctl, InvList list) {
  griddep_wait();
  if (L.stop_aware && ctl->stop) return;
  __shared__ int am_last;
  const int nb = gridDim.x / L.halves;
  const int h = blockIdx.x / nb;
  const int bid = blockIdx.x - h * nb;
  InvCtl& C = ctl->inv[L.phase][h];
  const int k = L.k >= 0 ? L.k : *(volatile const int*)&ctl->inv[L.phase][0].kdev;
  if (k > 0 && !*(volatile const int*)&C.exec[k & 1]) return;
  const float eps = k == 0 ? 0.75f : 0.5f;
  const float lim = eps * *(volatile const float*)&C.maxk[k & 1];
  const unsigned n = *(volatile const unsigned*)&C.lcount;
  const int N = (int)a.g.N;
  float* __restrict__ psi = h ? a.psi.p[1] : a.psi.p[0];
  const float* __restrict__ ec = h ? a.ecache.p[1] : a.ecache.p[0];
  const int* __restrict__ idx = list.idx[h];
  for (unsigned j = (unsigned)bid * blockDim.x + threadIdx.x; j < n; j += (unsigned)nb * blockDim.x) {
    const int i = idx[j];
    float e[3], p[3];
    e[0] = ec[i];
    e[1] = ec[N + i];
    e[2] = DIM == 3 ? ec[2 * N + i] : 0.0f;
    p[0] = psi[i];
    p[1] = psi[N + i];
    p[2] = DIM == 3 ? psi[2 * N + i] : 0.0f;
    float s2 = 0.0f;
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      const float v = e[c] * a.ih[c];
      s2 += v * v;
    }
    const float nrm = sqrtf(s2);
    const float f = nrm > lim ? lim / nrm : 1.0f;
#pragma unroll
    for (int c = 0; c < DIM; ++c) p[c] = p[c] + ((-e[c]) * f) * eps;
    psi[i] = p[0];
    psi[N + i] = p[1];
    if (DIM == 3) psi[2 * N + i] = p[2];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    am_last = atomicAdd(&C.fcount, 1u) == (unsigned)nb - 1;
  }
  __syncthreads();
  if (am_last && threadIdx.x == 0) {
    C.lcount = 0u;
    C.mrun = 0u;
    C.fcount = 0u;
  }
}

void launch_invert_spec(const float* const* phi, float* const* psi, int halves, const GridInfo& g, int k, int max_iter,
                        double mean_tol, double max_tol, IterCtl* ctl, int phase, PartialBufs pb, cudaStream_t s,
                        bool stop_aware, float* const* ecache, int* const* list) {
  count_launch();
  const Map3 m2 = map3(g.d, 2, kInvTarget);
  const int tz = (int)m2.grid.z / 2;
  const int ntiles = (int)m2.grid.x * (int)m2.grid.y * tz;
  const int nb = std::max(1, std::min({ntiles, 148 * kInvSpecBlocksPerSM / 2, pb.capacity}));
  const InvArgs a = make_inv_args(phi, psi, halves, g, m2.zb, ecache);
  InvLaunch L{k, max_iter, phase, stop_aware ? 1 : 0, halves, (int)m2.grid.x, (int)m2.grid.y, tz, mean_tol, max_tol};
  const InvList il{{list[0], halves > 1 ? list[1] : list[0]}};
  const bool dg = affine_diag(make_affine(g, g));
  const dim3 grid((unsigned)(nb * halves));
  if (g.d.dim == 3) {
    if (dg) launch_k(k_invert_spec<3, true>, grid, 256, 0, s, a, L, ctl, pb.sum, pb.maxv, pb.capacity, il);
    else launch_k(k_invert_spec<3, false>, grid, 256, 0, s, a, L, ctl, pb.sum, pb.maxv, pb.capacity, il);
  } else {
    if (dg) launch_k(k_invert_spec<2, true>, grid, 256, 0, s, a, L, ctl, pb.sum, pb.maxv, pb.capacity, il);
    else launch_k(k_invert_spec<2, false>, grid, 256, 0, s, a, L, ctl, pb.sum, pb.maxv, pb.capacity, il);
  }
}

constexpr int kInvFixBlocksPerHalf = 148;

void launch_invert_fix(const float* const* phi, float* const* psi, int halves, const GridInfo& g, int k, int max_iter,
                       IterCtl* ctl, int phase, cudaStream_t s, bool stop_aware, float* const* ecache,
                       int* const* list) {
  count_launch();
  const InvArgs a = make_inv_args(phi, psi, halves, g, 1, ecache);
  InvLaunch L{k, max_iter, phase, stop_aware ? 1 : 0, halves, 0, 0, 0, 0.0, 0.0};
  const InvList il{{list[0], halves > 1 ? list[1] : list[0]}};
  const dim3 grid((unsigned)(kInvFixBlocksPerHalf * halves));
  if (g.d.dim == 3)
    launch_k(k_invert_fix<3>, grid, 256, 0, s, a, L, ctl, il);
  else
    launch_k(k_invert_fix<2>, grid, 256, 0, s, a, L, ctl, il);
}

__global__ void k_inv_spec_control(IterCtl* ctl, int phase, cudaGraphConditionalHandle handle, int max_iter, int init) {
  griddep_wait();
  InvCtl* C = ctl->inv[phase];
  const int next = init ? 1 : C[0].kdev + 1;
  const int s = next & 1;
  const unsigned go = (!ctl->stop && next < max_iter && (C[0].exec[s] || C[1].exec[s])) ? 1u : 0u;
  C[0].kdev = next;
  cudaGraphSetConditional(handle, go);
}

void launch_inv_spec_control(IterCtl* ctl, int phase, cudaGraphConditionalHandle handle, int max_iter, bool init,
                             cudaStream_t s) {
  count_launch();
  launch_k(k_inv_spec_control, 1, 1, 0, s, ctl, phase, handle, max_iter, init ? 1 : 0);
}

__global__ void k_inv_loop_control(IterCtl* ctl, int phase, cudaGraphConditionalHandle handle, int max_iter,
                                   int init) {
  griddep_wait();
  InvCtl* C = ctl->inv[phase];
  unsigned go = 0;
  if (init) {
    C[0].kdev = 1;
    go = ctl->stop ? 0u : 1u;
  } else {
    const int next = C[0].kdev + 1;
    const int s = next & 1;
    go = (!ctl->stop && next <= max_iter && (C[0].exec[s] || C[1].exec[s])) ? 1u : 0u;
    C[0].kdev = next;
  }
  cudaGraphSetConditional(handle, go);
}

void launch_inv_loop_control(IterCtl* ctl, int phase, cudaGraphConditionalHandle handle, int max_iter, bool init,
                             cudaStream_t s) {
  count_launch();
  launch_k(k_inv_loop_control, 1, 1, 0, s, ctl, phase, handle, max_iter, init ? 1 : 0);
}

// ------------------------------------------------------------------------------------------
// Convergence monitor and per-iteration log (one warp).
// ------------------------------------------------------------------------------------------
__global__ void k_converge(IterCtl* ctl, LogDev log, double threshold, int window) {
  griddep_wait();
  if (ctl->stop) return;
  converge_step(ctl, log, threshold, window);
}

void launch_converge(IterCtl* ctl, LogDev log, double threshold, int window, cudaStream_t s) {
  count_launch();
  launch_k(k_converge, 1, 32, 0, s, ctl, log, threshold, window);
}


// ------------------------------------------------------------------------------------------
// Field resampling between level grids (linear, 0 outside), up to 4 fields per launch.
// ------------------------------------------------------------------------------------------
struct Ptr4c {
  const float* p[4];
};
struct Ptr4 {
  float* p[4];
};

// Index map in double: c = ((t + B0 x) + B1 y) + B2 z, each operation rounded on its own (no
// fused multiply-add), so the inside-buffer decision at a half-voxel rim tie is the one the
// host-side map's exact arithmetic gives.  Once per level and field, so the FP64 cost is nil.
struct MapD {
  double t[3];
  double B[9];
};

__device__ __forceinline__ double map_axis_d(const MapD& m, int r, double x, double y, double z) {
  double v = __dadd_rn(m.t[r], __dmul_rn(m.B[r * 3 + 0], x));
  v = __dadd_rn(v, __dmul_rn(m.B[r * 3 + 1], y));
  return __dadd_rn(v, __dmul_rn(m.B[r * 3 + 2], z));
}

// Clamp-to-edge cell from a double continuous index (weights rounded to float once).
__device__ __forceinline__ void axis_cell_d(double c, int n, int& i0, int& i1, float& w) {
  const double f = floor(c);
  int b = (int)f;
  double wd = c - f;
  if (b < 0) {
    b = 0;
    wd = 0.0;
  }
  int u = b + 1;
  if (u > n - 1) {
    u = n - 1;
    wd = 0.0;
  }
  i0 = b;
  i1 = u;
  w = (float)wd;
}

template <int DIM>
__global__ void __launch_bounds__(256) k_resample(Ptr4c in, Dims di, Ptr4 out, Dims dout, int zb, MapD m, int nf) {
  const Coord3 c3 = coord3(dout, zb, 1);
  if (!c3.ok) return;
  const int No = (int)dout.N, Ni = (int)di.N, nxy = dout.nx * dout.ny;
  for (int z = c3.z0; z < c3.z1; ++z) {
    const int i = z * nxy + c3.y * dout.nx + c3.x;
    const double fx = (double)c3.x, fy = (double)c3.y, fz = (double)z;
    const double cx = map_axis_d(m, 0, fx, fy, fz), cy = map_axis_d(m, 1, fx, fy, fz);
    const double cz = DIM == 3 ? map_axis_d(m, 2, fx, fy, fz) : 0.0;
    bool ok = (cx >= -0.5) && (cx < (double)di.nx - 0.5) && (cy >= -0.5) && (cy < (double)di.ny - 0.5);
    if (DIM == 3) ok = ok && (cz >= -0.5) && (cz < (double)di.nz - 0.5);
    Cell c{};
    if (ok) {
      int x0, x1, y0, y1, z0 = 0, z1 = 0;
      axis_cell_d(cx, di.nx, x0, x1, c.wx);
      axis_cell_d(cy, di.ny, y0, y1, c.wy);
      if (DIM == 3) axis_cell_d(cz, di.nz, z0, z1, c.wz);
      const int sy = di.nx, sz = di.nx * di.ny;
      c.o000 = z0 * sz + y0 * sy + x0;
      c.dx = x1 - x0;
      c.dy = (y1 - y0) * sy;
      c.dz = (z1 - z0) * sz;
    }
    for (int f = 0; f < nf; ++f)
#pragma unroll
      for (int k = 0; k < DIM; ++k) out.p[f][k * No + i] = ok ? lerp_at<DIM>(in.p[f] + k * Ni, c) : 0.0f;
  }
}

__global__ void __launch_bounds__(256) k_round_half(Ptr4 f, int nf, long long n) {
  griddep_wait();
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    for (int k = 0; k < nf; ++k) f.p[k][i] = __half2float(__float2half_rn(f.p[k][i]));
}

void launch_round_half(float* const* f, int nf, long long n, cudaStream_t s) {
  count_launch();
  Ptr4 p{};
  for (int k = 0; k < nf && k < 4; ++k) p.p[k] = f[k];
  const long long blocks = std::min<long long>((n + 255) / 256, 148 * 16);
  launch_k(k_round_half, (unsigned)std::max<long long>(blocks, 1), 256, 0, s, p, std::min(nf, 4), n);
}

void launch_resample_fields(const float* const* in, const GridInfo& gi, float* const* out, const GridInfo& go,
                            int nfields, cudaStream_t s) {
  count_launch();
  Ptr4c pi{};
  Ptr4 po{};
  for (int f = 0; f < nfields && f < 4; ++f) {
    pi.p[f] = in[f];
    po.p[f] = out[f];
  }
  MapD a;
  index_map(go, gi, a.t, a.B);
  const Map3 m = map3(go.d);
  if (go.d.dim == 3)
    k_resample<3><<<m.grid, 256, 0, s>>>(pi, gi.d, po, go.d, m.zb, a, nfields);
  else
    k_resample<2><<<m.grid, 256, 0, s>>>(pi, gi.d, po, go.d, m.zb, a, nfields);
}

// ------------------------------------------------------------------------------------------
// Image pyramid: one separable pass, replicate-edge boundary, FP64 accumulation.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_conv_image_axis(const float* __restrict__ in, float* __restrict__ out, Dims d,
                                                         int zb, int axis, const double* __restrict__ coeffs, int R) {
  const Coord3 c3 = coord3(d, zb, 1);
  if (!c3.ok) return;
  const int nxy = d.nx * d.ny;
  const int len = axis == 0 ? d.nx : (axis == 1 ? d.ny : d.nz);
  const int astride = axis == 0 ? 1 : (axis == 1 ? d.nx : nxy);
  for (int z = c3.z0; z < c3.z1; ++z) {
    const int i = z * nxy + c3.y * d.nx + c3.x;
    const int pos = axis == 0 ? c3.x : (axis == 1 ? c3.y : z);
    const float* line = in + i - pos * astride;
    double s = 0.0;
    // unrolled so that the taps' loads are issued ahead of the accumulation chain (the order of the
    // additions, j ascending, is unchanged)
#pragma unroll 8
    for (int j = 0; j <= 2 * R; ++j) {
      const int q = min(max(pos + j - R, 0), len - 1);
      s += __ldg(coeffs + j) * (double)__ldg(line + q * astride);
    }
    out[i] = (float)s;
  }
}

// The same pass with the radius a compile-time constant, in two forms whose sums are the generic
// kernel's (coefficient j times the replicate-edge sample pos - R + j, j ascending, in FP64 FMAs):
//  * along x, each warp converts its row segment and halo to double once into shared memory and sums
//    from there (the taps are immediate offsets);
//  * along y or z, each thread walks a chunk of its line with the last 2R+1 samples in registers
//    (unrolled by 2R+1 so every ring index is a compile-time constant): one load and one conversion
//    per output instead of 2R+1.
constexpr int kConvImageMaxR = 16;

constexpr int kConvImageXSlices = 8;  // rows of consecutive slices per warp of the x pass

template <int R>
__global__ void __launch_bounds__(256) k_conv_image_x(const float* __restrict__ in, float* __restrict__ out, Dims d,
                                                      const double* __restrict__ coeffs) {
  constexpr int K = 2 * R + 1, W = 32 + 2 * R;
  __shared__ double buf[8][W];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int x0 = blockIdx.x * 32, y = blockIdx.y * 8 + w;
  if (y >= d.ny) return;  // the whole warp; no block-wide barrier below
  double c[K];
#pragma unroll
  for (int j = 0; j < K; ++j) c[j] = __ldg(coeffs + j);
  const int x = x0 + lane;
  const int z0 = blockIdx.z * kConvImageXSlices, z1 = min(z0 + kConvImageXSlices, d.nz);
  for (int z = z0; z < z1; ++z) {
    const long long row = ((long long)z * d.ny + y) * d.nx;
    const float* line = in + row;
    __syncwarp();  // the previous row's reads of buf are done
    for (int k = lane; k < W; k += 32) buf[w][k] = (double)__ldg(line + min(max(x0 - R + k, 0), d.nx - 1));
    __syncwarp();
    if (x < d.nx) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < K; ++j) acc = fma(c[j], buf[w][lane + j], acc);
      out[row + x] = (float)acc;
    }
  }
}

template <int R, int AXIS>
__global__ void __launch_bounds__(256) k_conv_image_walk(const float* __restrict__ in, float* __restrict__ out, Dims d,
                                                         const double* __restrict__ coeffs, int chunk) {
  constexpr int K = 2 * R + 1;
  const int x = blockIdx.x * 32 + (threadIdx.x & 31);
  const int o = blockIdx.y * 8 + (threadIdx.x >> 5);  // z for a y walk, y for a z walk
  const int len = AXIS == 1 ? d.ny : d.nz;
  if (x >= d.nx || o >= (AXIS == 1 ? d.nz : d.ny)) return;
  const long long stride = AXIS == 1 ? (long long)d.nx : (long long)d.nx * d.ny;
  const long long base = AXIS == 1 ? (long long)o * d.nx * d.ny + x : (long long)o * d.nx + x;
  const int p0 = blockIdx.z * chunk, p1 = min(p0 + chunk, len);
  double c[K];
#pragma unroll
  for (int j = 0; j < K; ++j) c[j] = __ldg(coeffs + j);
  double ring[K];
#pragma unroll
  for (int u = 0; u < 2 * R; ++u) ring[u] = (double)__ldg(in + base + min(max(p0 - R + u, 0), len - 1) * stride);
  for (int pb = p0; pb < p1; pb += K) {
#pragma unroll
    for (int u = 0; u < K; ++u) {
      const int p = pb + u;
      if (p < p1) {
        ring[(u + 2 * R) % K] = (double)__ldg(in + base + min(p + R, len - 1) * stride);
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < K; ++j) acc = fma(c[j], ring[(u + j) % K], acc);
        out[base + p * stride] = (float)acc;
      }
    }
  }
}

template <int R>
static void conv_image_axis_t(const float* in, float* out, const GridInfo& g, int axis, const double* coeffs,
                              cudaStream_t s) {
  const Dims& d = g.d;
  const int gx = (d.nx + 31) / 32;
  if (axis == 0) {
    k_conv_image_x<R><<<dim3(gx, (d.ny + 7) / 8, (d.nz + kConvImageXSlices - 1) / kConvImageXSlices), 256, 0, s>>>(
        in, out, d, coeffs);
    return;
  }
  const int other = axis == 1 ? d.nz : d.ny, len = axis == 1 ? d.ny : d.nz;
  const int cols = gx * ((other + 7) / 8);
  // about 8 walking warps per SM; a chunk is at least 2R + 1 long, its warm-up being 2R loads
  const int chunks = std::max(1, std::min(len, (148 * 8 + cols - 1) / cols));
  const int chunk = std::min(len, std::max((len + chunks - 1) / chunks, 2 * R + 1));
  const dim3 grid(gx, (other + 7) / 8, (len + chunk - 1) / chunk);
  if (axis == 1) k_conv_image_walk<R, 1><<<grid, 256, 0, s>>>(in, out, d, coeffs, chunk);
  else k_conv_image_walk<R, 2><<<grid, 256, 0, s>>>(in, out, d, coeffs, chunk);
}

void launch_conv_image_axis(const float* in, float* out, const GridInfo& g, int axis, const double* coeffs, int R,
                            cudaStream_t s) {
  count_launch();
  switch (R) {
#define SYNX_CONV_IMG(RV)                                   \
  case RV:                                                  \
    conv_image_axis_t<RV>(in, out, g, axis, coeffs, s);     \
    return;
    SYNX_CONV_IMG(1)
    SYNX_CONV_IMG(2)
    SYNX_CONV_IMG(3)
    SYNX_CONV_IMG(4)
    SYNX_CONV_IMG(5)
    SYNX_CONV_IMG(6)
    SYNX_CONV_IMG(7)
    SYNX_CONV_IMG(8)
    SYNX_CONV_IMG(9)
    SYNX_CONV_IMG(10)
    SYNX_CONV_IMG(11)
    SYNX_CONV_IMG(12)
    SYNX_CONV_IMG(13)
    SYNX_CONV_IMG(14)
    SYNX_CONV_IMG(15)
    SYNX_CONV_IMG(16)
#undef SYNX_CONV_IMG
    default:
      break;
  }
  static_assert(kConvImageMaxR == 16, "the switch covers 1..kConvImageMaxR");
  const Map3 m = map3(g.d);
  k_conv_image_axis<<<m.grid, 256, 0, s>>>(in, out, g.d, m.zb, axis, coeffs, R);
}

// ------------------------------------------------------------------------------------------
// Intensity statistics and window (antsRegistration's preprocessing).
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_minmax(const float* __restrict__ x, long long n, unsigned* mm) {
  float lo = FLT_MAX, hi = -FLT_MAX;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float v = x[i];
    lo = fminf(lo, v);
    hi = fmaxf(hi, v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_down_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_down_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&mm[0], d_float_to_ordered(lo));
    atomicMax(&mm[1], d_float_to_ordered(hi));
  }
}
void launch_minmax(const float* x, long long n, unsigned* mm, cudaStream_t s) {
  count_launch();
  k_minmax<<<grid_for(n, 256), 256, 0, s>>>(x, n, mm);
}

__global__ void __launch_bounds__(256) k_hist(const float* __restrict__ x, long long n, double lo, double bw, int nb,
                                              unsigned* hist) {
  extern __shared__ unsigned sh[];
  for (int b = threadIdx.x; b < nb; b += blockDim.x) sh[b] = 0u;
  __syncthreads();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int b = bw > 0.0 ? (int)(((double)x[i] - lo) / bw) : 0;
    b = min(max(b, 0), nb - 1);
    atomicAdd(&sh[b], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
    if (sh[b]) atomicAdd(&hist[b], sh[b]);
}
void launch_histogram(const float* x, long long n, float lo, float hi, int nbins, unsigned* hist, cudaStream_t s) {
  count_launch();
  const double bw = ((double)hi - (double)lo) / nbins;
  k_hist<<<grid_for(n, 256), 256, nbins * sizeof(unsigned), s>>>(x, n, (double)lo, bw, nbins, hist);
}

__global__ void __launch_bounds__(256) k_window(const float* __restrict__ in, float* __restrict__ out, long long n,
                                                float wlo, float whi, double scale, double shift) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float a = in[i];
    out[i] = a < wlo ? 0.0f : (a > whi ? 1.0f : (float)((double)a * scale + shift));
  }
}
void launch_window(const float* in, float* out, long long n, float wlo, float whi, double scale, double shift,
                   cudaStream_t s) {
  count_launch();
  k_window<<<grid_for(n, 256), 256, 0, s>>>(in, out, n, wlo, whi, scale, shift);
}

// ------------------------------------------------------------------------------------------
// Histogram matching (ITK's HistogramMatchingImageFilter): an image's min, max and per-block
// double sums (a fixed grid, so the mean's summation order is the same on every run), the
// histogram of the voxels inside [vlo, vhi], and the piecewise-linear map through the table of
// match points.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_stats(const float* __restrict__ x, long long n, double* part, unsigned* mm) {
  __shared__ double ws[8];
  double sum = 0.0;
  float lo = FLT_MAX, hi = -FLT_MAX;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float v = x[i];
    sum += (double)v;
    lo = fminf(lo, v);
    hi = fmaxf(hi, v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_down_sync(0xffffffffu, sum, o);
    lo = fminf(lo, __shfl_down_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_down_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    ws[threadIdx.x >> 5] = sum;
    atomicMin(&mm[0], d_float_to_ordered(lo));
    atomicMax(&mm[1], d_float_to_ordered(hi));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
    part[blockIdx.x] = t;
  }
}
void launch_stats(const float* x, long long n, double* part, int nblocks, unsigned* mm, cudaStream_t s) {
  count_launch();
  k_stats<<<nblocks, 256, 0, s>>>(x, n, part, mm);
}

__global__ void __launch_bounds__(256) k_hist_range(const float* __restrict__ x, long long n, double lo, double bw,
                                                    int nb, double vlo, double vhi, unsigned* hist) {
  extern __shared__ unsigned sh[];
  for (int b = threadIdx.x; b < nb; b += blockDim.x) sh[b] = 0u;
  __syncthreads();
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = (double)x[i];
    if (!(v >= vlo && v <= vhi)) continue;  // also drops NaN
    int b = bw > 0.0 ? (int)((v - lo) / bw) : 0;
    b = min(max(b, 0), nb - 1);
    atomicAdd(&sh[b], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
    if (sh[b]) atomicAdd(&hist[b], sh[b]);
}
void launch_histogram_range(const float* x, long long n, double lo, double hi, int nbins, double vlo, double vhi,
                            unsigned* hist, cudaStream_t s) {
  count_launch();
  const double bw = (hi - lo) / nbins;
  k_hist_range<<<grid_for(n, 256), 256, nbins * sizeof(unsigned), s>>>(x, n, lo, bw, nbins, vlo, vhi, hist);
}

// Unfused double arithmetic (no FMA contraction), as the host computes the same map.
__global__ void __launch_bounds__(256) k_hist_map(const float* in, float* out, long long n,
                                                  HistMatchMap t) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = (double)in[i];
    int j = 0;
    while (j < t.points + 2 && !(v < t.src[j])) ++j;
    double r;
    if (j == 0)
      r = __dadd_rn(t.ref_min, __dmul_rn(__dsub_rn(v, t.src_min), t.lower_grad));
    else if (j == t.points + 2)
      r = __dadd_rn(t.ref_max, __dmul_rn(__dsub_rn(v, t.src_max), t.upper_grad));
    else
      r = __dadd_rn(t.ref[j - 1], __dmul_rn(__dsub_rn(v, t.src[j - 1]), t.grad[j - 1]));
    out[i] = (float)r;
  }
}
void launch_histogram_map(const float* in, float* out, long long n, const HistMatchMap& t, cudaStream_t s) {
  count_launch();
  k_hist_map<<<grid_for(n, 256), 256, 0, s>>>(in, out, n, t);
}

// ------------------------------------------------------------------------------------------
// Layout conversion.
// ------------------------------------------------------------------------------------------
__global__ void k_interleave(const float* __restrict__ planes, float* __restrict__ inter, long long N, int D) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    for (int c = 0; c < D; ++c) inter[i * D + c] = planes[c * N + i];
}
__global__ void k_deinterleave(const float* __restrict__ inter, float* __restrict__ planes, long long N, int D) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
    for (int c = 0; c < D; ++c) planes[c * N + i] = inter[i * D + c];
}
void launch_interleave(const float* planes, float* inter, long long N, int D, cudaStream_t s) {
  count_launch();
  k_interleave<<<grid_for(N, 256), 256, 0, s>>>(planes, inter, N, D);
}
void launch_deinterleave(const float* inter, float* planes, long long N, int D, cudaStream_t s) {
  count_launch();
  k_deinterleave<<<grid_for(N, 256), 256, 0, s>>>(inter, planes, N, D);
}

}  // namespace synx
