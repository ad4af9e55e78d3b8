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

#include "synx_kernels.cuh"

namespace synx {

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

Affine make_affine(const GridInfo& src, const GridInfo& dst) {
  Affine a;
  double dorg[3] = {src.org[0] - dst.org[0], src.org[1] - dst.org[1], src.org[2] - dst.org[2]};
  for (int r = 0; r < 3; ++r) {
    double t = 0.0;
    for (int c = 0; c < 3; ++c) {
      t += dst.p2i[r * 3 + c] * dorg[c];
      double b = 0.0;
      for (int k = 0; k < 3; ++k) b += dst.p2i[r * 3 + k] * src.i2p[k * 3 + c];
      a.B[r * 3 + c] = (float)b;
      a.A[r * 3 + c] = (float)dst.p2i[r * 3 + c];
    }
    a.t[r] = (float)t;
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

// DIAG: the grids share axis directions (no rotation between them), the common case; the
// map is then one FMA pair per axis.
template <int DIM, bool DIAG = false>
__device__ __forceinline__ void map_point(const Affine& m, float fx, float fy, float fz, float ux, float uy, float uz,
                                          float& cx, float& cy, float& cz) {
  if (DIAG) {
    cx = fmaf(m.A[0], ux, fmaf(m.B[0], fx, m.t[0]));
    cy = fmaf(m.A[4], uy, fmaf(m.B[4], fy, m.t[1]));
    cz = DIM == 3 ? fmaf(m.A[8], uz, fmaf(m.B[8], fz, m.t[2])) : 0.0f;
    return;
  }
  cx = m.t[0] + m.B[0] * fx + m.B[1] * fy + m.A[0] * ux + m.A[1] * uy;
  cy = m.t[1] + m.B[3] * fx + m.B[4] * fy + m.A[3] * ux + m.A[4] * uy;
  cz = 0.0f;
  if (DIM == 3) {
    cx += m.B[2] * fz + m.A[2] * uz;
    cy += m.B[5] * fz + m.A[5] * uz;
    cz = m.t[2] + m.B[6] * fx + m.B[7] * fy + m.B[8] * fz + m.A[6] * ux + m.A[7] * uy + m.A[8] * uz;
  }
}

// ------------------------------------------------------------------------------------------
// Level control reset
// ------------------------------------------------------------------------------------------
__global__ void k_zero_ctl_level(IterCtl* ctl) {
  ctl->stop = 0;
  ctl->iter = 0;
  ctl->total_abs = 0.0;
  ctl->maxnorm[0] = ctl->maxnorm[1] = 0u;
  ctl->cc_counter = 0u;
  for (int p = 0; p < 2; ++p)
    for (int h = 0; h < 2; ++h) {
      ctl->inv[p][h].counter = 0u;
      ctl->inv[p][h].iters = 0;
      ctl->inv[p][h].exec[0] = ctl->inv[p][h].exec[1] = 0;
    }
}
void launch_zero_ctl_level(IterCtl* ctl, cudaStream_t s) {
  count_launch();
  k_zero_ctl_level<<<1, 1, 0, s>>>(ctl);
}

// ------------------------------------------------------------------------------------------
// Warp of both images through their inverse half-fields onto the level grid.
// ------------------------------------------------------------------------------------------
template <int DIM, bool DIAG>
__device__ __forceinline__ float sample(const float* __restrict__ img, const Dims& di, const Affine& m, float fx,
                                        float fy, float fz, float ux, float uy, float uz) {
  float cx, cy, cz;
  map_point<DIM, DIAG>(m, fx, fy, fz, ux, uy, uz, cx, cy, cz);
  if (!inside_buffer<DIM>(di, cx, cy, cz)) return 0.0f;
  return lerp_at<DIM>(img, make_cell<DIM>(di, cx, cy, cz));
}

template <int DIM, bool DIAG>
__global__ void __launch_bounds__(256)
    k_warp_pair(const float* __restrict__ F, Dims dF, Affine mF, const float* __restrict__ psiF,
                const float* __restrict__ M, Dims dM, Affine mM, const float* __restrict__ psiM, Dims dv, int zb,
                float* __restrict__ Ft, float* __restrict__ Mt, IterCtl* ctl) {
  if (ctl != nullptr && ctl->stop) return;
  if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && ctl != nullptr) {
    ctl->maxnorm[0] = 0u;
    ctl->maxnorm[1] = 0u;
  }
  const Coord3 c = coord3(dv, zb, 1);
  if (!c.ok) return;
  const int N = (int)dv.N, nxy = dv.nx * dv.ny;
  const float fx = (float)c.x, fy = (float)c.y;
  const int i0 = c.z0 * nxy + c.y * dv.nx + c.x;
  float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, b0 = 0.0f, b1 = 0.0f, b2 = 0.0f;
  if (c.z0 < c.z1) {
    a0 = psiF[i0];
    a1 = psiF[N + i0];
    a2 = DIM == 3 ? psiF[2 * N + i0] : 0.0f;
    b0 = psiM[i0];
    b1 = psiM[N + i0];
    b2 = DIM == 3 ? psiM[2 * N + i0] : 0.0f;
  }
  for (int z = c.z0; z < c.z1; ++z) {
    const int i = z * nxy + c.y * dv.nx + c.x;
    const float fz = (float)z;
    const float u0 = a0, u1 = a1, u2 = a2, v0 = b0, v1 = b1, v2 = b2;
    if (z + 1 < c.z1) {  // next slice's displacements, loaded ahead of this slice's gathers
      const int j = i + nxy;
      a0 = psiF[j];
      a1 = psiF[N + j];
      a2 = DIM == 3 ? psiF[2 * N + j] : 0.0f;
      b0 = psiM[j];
      b1 = psiM[N + j];
      b2 = DIM == 3 ? psiM[2 * N + j] : 0.0f;
    }
    Ft[i] = sample<DIM, DIAG>(F, dF, mF, fx, fy, fz, u0, u1, u2);
    Mt[i] = sample<DIM, DIAG>(M, dM, mM, fx, fy, fz, v0, v1, v2);
  }
}

void launch_warp_pair(const float* F, const GridInfo& gF, const float* psiF, const float* M, const GridInfo& gM,
                      const float* psiM, const GridInfo& gv, float* Ft, float* Mt, IterCtl* ctl, cudaStream_t s) {
  count_launch();
  Affine mF = make_affine(gv, gF), mM = make_affine(gv, gM);
  const Map3 m = map3(gv.d);
  const bool dg = affine_diag(mF) && affine_diag(mM);
  if (gv.d.dim == 3) {
    if (dg)
      k_warp_pair<3, true><<<m.grid, 256, 0, s>>>(F, gF.d, mF, psiF, M, gM.d, mM, psiM, gv.d, m.zb, Ft, Mt, ctl);
    else
      k_warp_pair<3, false><<<m.grid, 256, 0, s>>>(F, gF.d, mF, psiF, M, gM.d, mM, psiM, gv.d, m.zb, Ft, Mt, ctl);
  } else {
    if (dg)
      k_warp_pair<2, true><<<m.grid, 256, 0, s>>>(F, gF.d, mF, psiF, M, gM.d, mM, psiM, gv.d, m.zb, Ft, Mt, ctl);
    else
      k_warp_pair<2, false><<<m.grid, 256, 0, s>>>(F, gF.d, mF, psiF, M, gM.d, mM, psiM, gv.d, m.zb, Ft, Mt, ctl);
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
    out[i] = sample<DIM, false>(img, di, m, (float)c.x, (float)c.y, (float)z, u[i], u[N + i], DIM == 3 ? u[2 * N + i] : 0.0f);
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

// ------------------------------------------------------------------------------------------
// Gaussian smoothing of displacement fields, all axes in one pass.
//
// A block owns a 32 x 8 tile of output columns of one field and marches along z.  For each
// input slice it stages the (32+2Rx) x (8+2Ry) halo tile of every component in shared
// memory (replicate-edge indices), convolves along x, then y (each thread its own column),
// and keeps the xy-smoothed slices of the last 2Rz+1 z positions in a per-thread shared
// ring; the z convolution of that ring gives the output.  The pass order (x, y, z) and the
// float rounding after each axis follow the separable filter.  The epilogue applies SyN's
// boundary zeroing and blend, and reduces max ||u / spacing|| for the update scaling.
// ------------------------------------------------------------------------------------------
struct Ptr2c {
  const float* p[2];
};
struct Ptr2 {
  float* p[2];
};

constexpr int kSmoothRMax = 12;

struct Smooth3Args {
  Ptr2c in, orig;
  Ptr2 out;
  float k[3][2 * kSmoothRMax + 1];  // per-axis kernels, zero-padded and centred to radius R
  int ZC, halves, epilogue, do_max;
  float w1, w2;
  float ih[3];
};

__host__ __device__ inline size_t smooth3_smem_floats(int dim, int R) {
  const int HXP = (32 + 2 * R + 3) & ~3, HY = 8 + 2 * R;
  return (size_t)dim * HY * HXP + (size_t)dim * HY * 32;
}

// xy part: one block per (32 x 8 tile, slice, field).  The halo tile of every component is
// staged in shared memory with replicate-edge indices, convolved along x (each work item makes
// four consecutive outputs from float4 loads) and then along y.  In 2-D this is the whole
// filter and the SyN epilogue runs here; in 3-D the xy-smoothed slice goes to `out` for the z
// kernel.
template <int DIM, int R>
__global__ void __launch_bounds__(256) k_smooth_xy(const Smooth3Args a, Dims d, IterCtl* ctl) {
  if (ctl != nullptr && ctl->stop) return;
  constexpr int K = 2 * R + 1;
  constexpr int HX = 32 + 2 * R, HXP = (HX + 3) & ~3, HY = 8 + 2 * R;
  constexpr int NQ = (2 * R + 3) / 4 + 1;  // float4 loads covering 4 + 2R taps
  extern __shared__ __align__(16) float sm3[];
  __shared__ float red[32];
  float* tile = sm3;                    // [DIM][HY][HXP]
  float* xsum = tile + DIM * HY * HXP;  // [DIM][HY][32]
  const int nx = d.nx, ny = d.ny, nz = d.nz, nxy = nx * ny, N = (int)d.N;
  const int h = blockIdx.z / nz;
  const int z = blockIdx.z - h * nz;
  const float* __restrict__ src = h ? a.in.p[1] : a.in.p[0];
  float* __restrict__ dst = h ? a.out.p[1] : a.out.p[0];
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 8;
  const float* plane = src + z * nxy;
  for (int row = ty; row < DIM * HY; row += 8) {
    const int c = row / HY, hy = row - c * HY;
    const int gy = min(max(y0 - R + hy, 0), ny - 1);
    const float* line = plane + c * N + gy * nx;
    float* trow = tile + row * HXP;
#pragma unroll
    for (int hx = tx; hx < HX; hx += 32) trow[hx] = __ldg(line + min(max(x0 - R + hx, 0), nx - 1));
  }
  __syncthreads();
  for (int it = tid; it < DIM * HY * 8; it += 256) {
    const int row = it >> 3, q = it & 7;
    const float4* t4 = reinterpret_cast<const float4*>(tile + row * HXP) + q;
    float w[4 * NQ];
#pragma unroll
    for (int m = 0; m < NQ; ++m) {
      const float4 v = t4[m];
      w[4 * m] = v.x;
      w[4 * m + 1] = v.y;
      w[4 * m + 2] = v.z;
      w[4 * m + 3] = v.w;
    }
    float o[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      float acc = 0.0f;
#pragma unroll
      for (int j = 0; j < K; ++j) acc = fmaf(a.k[0][j], w[i + j], acc);
      o[i] = acc;
    }
    reinterpret_cast<float4*>(xsum + row * 32)[q] = make_float4(o[0], o[1], o[2], o[3]);
  }
  __syncthreads();
  const int ox = x0 + tx, oy = y0 + ty;
  const bool ok = ox < nx && oy < ny;
  float y[DIM];
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    const float* col = xsum + (c * HY + ty) * 32 + tx;
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < K; ++j) acc = fmaf(a.k[1][j], col[j * 32], acc);
    y[c] = acc;
  }
  if (DIM == 3) {
    if (ok) {
      const int i = z * nxy + oy * nx + ox;
#pragma unroll
      for (int c = 0; c < DIM; ++c) dst[c * N + i] = y[c];
    }
    return;
  }
  // 2-D: SyN epilogue and max norm
  float mx = 0.0f;
  if (ok) {
    const int i = oy * nx + ox;
    const float* __restrict__ org = h ? a.orig.p[1] : a.orig.p[0];
    const bool edge = a.epilogue && (ox == 0 || ox == nx - 1 || oy == 0 || oy == ny - 1);
    float nrm2 = 0.0f;
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      float r = y[c];
      if (a.epilogue) {
        if (edge) r = 0.0f;
        else if (a.w2 != 0.0f) r = r * a.w1 + org[c * N + i] * a.w2;
      }
      const float q = r * a.ih[c];
      nrm2 += q * q;
      dst[c * N + i] = r;
    }
    mx = sqrtf(nrm2);
  }
  if (a.do_max) {
    const float bm = block_max_f(mx, red);
    if (tid == 0) atomic_max_nonneg(&ctl->maxnorm[h], bm);
  }
}

// z part (3-D): each thread owns one (x, y) column of one field over a chunk of slices and
// keeps the last 2R+1 xy-smoothed values per component in registers; the z loop is unrolled
// by 2R+1 so every ring index is a compile-time constant.  No shared memory, no barriers in
// the loop.  Applies the SyN epilogue and reduces the max norm.
template <int R>
__global__ void __launch_bounds__(256) k_smooth_z(const Smooth3Args a, Dims d, IterCtl* ctl) {
  if (ctl != nullptr && ctl->stop) return;
  constexpr int K = 2 * R + 1, RD = K;
  __shared__ float red[32];
  const int nx = d.nx, ny = d.ny, nz = d.nz, nxy = nx * ny, N = (int)d.N;
  const int nzc = gridDim.z / a.halves;
  const int h = blockIdx.z / nzc;
  const int zc = blockIdx.z - h * nzc;
  const float* __restrict__ src = h ? a.in.p[1] : a.in.p[0];
  float* __restrict__ dst = h ? a.out.p[1] : a.out.p[0];
  const float* __restrict__ org = h ? a.orig.p[1] : a.orig.p[0];
  const int ox = blockIdx.x * 32 + (threadIdx.x & 31), oy = blockIdx.y * 8 + (threadIdx.x >> 5);
  const int z0 = zc * a.ZC, z1 = min(z0 + a.ZC, nz);
  float mx = 0.0f;
  if (ox < nx && oy < ny) {
    const float* col = src + oy * nx + ox;
    float ring[3][RD];
#pragma unroll
    for (int u = 0; u < 2 * R; ++u) {
      const int zs = min(max(z0 - R + u, 0), nz - 1);
#pragma unroll
      for (int c = 0; c < 3; ++c) ring[c][u] = __ldg(col + c * N + zs * nxy);
    }
    const bool xyedge = ox == 0 || ox == nx - 1 || oy == 0 || oy == ny - 1;
    for (int zb = z0; zb < z1; zb += RD) {
#pragma unroll
      for (int u = 0; u < RD; ++u) {
        const int z = zb + u;
        if (z < z1) {
          const int zs = min(z + R, nz - 1);
#pragma unroll
          for (int c = 0; c < 3; ++c) ring[c][(u + 2 * R) % RD] = __ldg(col + c * N + zs * nxy);
          const int i = z * nxy + oy * nx + ox;
          const bool edge = a.epilogue && (xyedge || z == 0 || z == nz - 1);
          float nrm2 = 0.0f;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            float acc = 0.0f;
#pragma unroll
            for (int j = 0; j < K; ++j) acc = fmaf(a.k[2][j], ring[c][(u + j) % RD], acc);
            if (a.epilogue) {
              if (edge) acc = 0.0f;
              else if (a.w2 != 0.0f) acc = acc * a.w1 + org[c * N + i] * a.w2;
            }
            const float q = acc * a.ih[c];
            nrm2 += q * q;
            dst[c * N + i] = acc;
          }
          mx = fmaxf(mx, sqrtf(nrm2));
        }
      }
    }
  }
  if (a.do_max) {
    const float bm = block_max_f(mx, red);
    if (threadIdx.x == 0) atomic_max_nonneg(&ctl->maxnorm[h], bm);
  }
}

static int smooth3_radius(int dim, const int R[3]) {
  int r = 0;
  for (int a = 0; a < dim; ++a) r = std::max(r, R[a]);
  return std::max(r, 1);
}

bool smooth3_supported(int dim, const int R[3]) { return smooth3_radius(dim, R) <= kSmoothRMax; }

template <int R>
static cudaError_t smooth3_attr_both() {
  cudaError_t e = cudaFuncSetAttribute(k_smooth_xy<3, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(smooth3_smem_floats(3, R) * 4));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_smooth_xy<2, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(smooth3_smem_floats(2, R) * 4));
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

void launch_smooth_field(const float* const* in, float* const* out, const float* const* orig, float* const* tmp,
                         int halves, const GridInfo& g, const float* const khost[3], const int R[3], bool epilogue,
                         float w1, float w2, bool maxnorm, IterCtl* ctl, cudaStream_t s) {
  const int dim = g.d.dim;
  const int RR = smooth3_radius(dim, R);
  Smooth3Args a;
  memset(&a, 0, sizeof(a));
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
  const int gx = (g.d.nx + 31) / 32, gy = (g.d.ny + 7) / 8;
  // xy pass: in -> (3-D: tmp, 2-D: out)
  a.in = Ptr2c{{in[0], halves > 1 ? in[1] : in[0]}};
  float* const* xyout = dim == 3 ? tmp : out;
  a.out = Ptr2{{xyout[0], halves > 1 ? xyout[1] : xyout[0]}};
  const dim3 gxy(gx, gy, g.d.nz * halves);
  const size_t smem = smooth3_smem_floats(dim, RR) * 4;
  count_launch();
#define SYNX_SXY(RV)                                             \
  case RV:                                                       \
    if (dim == 3)                                                \
      k_smooth_xy<3, RV><<<gxy, 256, smem, s>>>(a, g.d, ctl);    \
    else                                                         \
      k_smooth_xy<2, RV><<<gxy, 256, smem, s>>>(a, g.d, ctl);    \
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
  if (dim != 3) return;
  // z pass: tmp -> out with the epilogue
  a.in = Ptr2c{{tmp[0], halves > 1 ? tmp[1] : tmp[0]}};
  a.out = Ptr2{{out[0], halves > 1 ? out[1] : out[0]}};
  const int target = 148 * 8;
  const int chunks = std::max(1, (target + gx * gy * halves - 1) / (gx * gy * halves));
  int zc = (g.d.nz + chunks - 1) / chunks;
  zc = std::min(std::max(zc, 2 * RR + 1), g.d.nz);
  a.ZC = zc;
  const dim3 gz(gx, gy, ((g.d.nz + zc - 1) / zc) * halves);
  count_launch();
#define SYNX_SZ(RV)                                    \
  case RV:                                             \
    k_smooth_z<RV><<<gz, 256, 0, s>>>(a, g.d, ctl);    \
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
    k_smooth_pass<3><<<m.grid, 256, 0, s>>>(pi, po, pg, g.d, m.zb, axis, coeffs, R, last ? 1 : 0, w1, w2,
                                            maxnorm ? 1 : 0, ih[0], ih[1], ih[2], ctl);
  else
    k_smooth_pass<2><<<m.grid, 256, 0, s>>>(pi, po, pg, g.d, m.zb, axis, coeffs, R, last ? 1 : 0, w1, w2,
                                            maxnorm ? 1 : 0, ih[0], ih[1], ih[2], ctl);
}

// ------------------------------------------------------------------------------------------
// Composition out = w + s * d(x + w), s = eta / max||d/spacing|| (SyN's update scaling fused).
// Reads w only at its own voxel, so it runs in place (out == w).
// ------------------------------------------------------------------------------------------
template <int DIM, bool DIAG>
__global__ void __launch_bounds__(256) k_compose(Ptr2c dd, Ptr2c ww, Ptr2 oo, Dims d, int zb, int halves, Affine m,
                                                 double eta, IterCtl* ctl) {
  if (ctl != nullptr && ctl->stop) return;
  const Coord3 c3 = coord3(d, zb, halves);
  if (!c3.ok) return;
  const int h = c3.h;
  const float* __restrict__ D = (h ? dd.p[1] : dd.p[0]);
  const float* W = (h ? ww.p[1] : ww.p[0]);
  float* O = (h ? oo.p[1] : oo.p[0]);
  float scale = 1.0f;
  if (eta > 0.0) {
    const float mx = __uint_as_float(ctl->maxnorm[h]);
    scale = mx > 0.0f ? (float)(eta / (double)mx) : (float)eta;
  }
  const int N = (int)d.N, nxy = d.nx * d.ny;
  const float fx = (float)c3.x, fy = (float)c3.y;
  const int i0 = c3.z0 * nxy + c3.y * d.nx + c3.x;
  float n0 = 0.0f, n1 = 0.0f, n2 = 0.0f;
  if (c3.z0 < c3.z1) {
    n0 = W[i0];
    n1 = W[N + i0];
    n2 = DIM == 3 ? W[2 * N + i0] : 0.0f;
  }
  for (int z = c3.z0; z < c3.z1; ++z) {
    const int i = z * nxy + c3.y * d.nx + c3.x;
    const float w0 = n0, w1 = n1, w2 = n2;
    if (z + 1 < c3.z1) {  // next slice's warp vector, loaded ahead of this slice's gathers
      n0 = W[i + nxy];
      n1 = W[N + i + nxy];
      n2 = DIM == 3 ? W[2 * N + i + nxy] : 0.0f;
    }
    float cx, cy, cz;
    map_point<DIM, DIAG>(m, fx, fy, (float)z, w0, w1, w2, cx, cy, cz);
    if (inside_buffer<DIM>(d, cx, cy, cz)) {
      const Cell c = make_cell<DIM>(d, cx, cy, cz);
      O[i] = fmaf(scale, lerp_at<DIM>(D, c), w0);
      O[N + i] = fmaf(scale, lerp_at<DIM>(D + N, c), w1);
      if (DIM == 3) O[2 * N + i] = fmaf(scale, lerp_at<DIM>(D + 2 * N, c), w2);
    } else {
      O[i] = w0;
      O[N + i] = w1;
      if (DIM == 3) O[2 * N + i] = w2;
    }
  }
}

void launch_compose(const float* const* d, const float* const* w, float* const* out, int halves, const GridInfo& g,
                    float eta, IterCtl* ctl, cudaStream_t s) {
  count_launch();
  Ptr2c pd{{d[0], halves > 1 ? d[1] : d[0]}};
  Ptr2c pw{{w[0], halves > 1 ? w[1] : w[0]}};
  Ptr2 po{{out[0], halves > 1 ? out[1] : out[0]}};
  Affine a = make_affine(g, g);
  const Map3 m = map3(g.d, halves);
  const bool dg = affine_diag(a);
  if (g.d.dim == 3) {
    if (dg)
      k_compose<3, true><<<m.grid, 256, 0, s>>>(pd, pw, po, g.d, m.zb, halves, a, (double)eta, ctl);
    else
      k_compose<3, false><<<m.grid, 256, 0, s>>>(pd, pw, po, g.d, m.zb, halves, a, (double)eta, ctl);
  } else {
    if (dg)
      k_compose<2, true><<<m.grid, 256, 0, s>>>(pd, pw, po, g.d, m.zb, halves, a, (double)eta, ctl);
    else
      k_compose<2, false><<<m.grid, 256, 0, s>>>(pd, pw, po, g.d, m.zb, halves, a, (double)eta, ctl);
  }
}

// ------------------------------------------------------------------------------------------
// Fused fixed-point inverse.  Launch k applies iteration k (statistics from launch k-1) and,
// if iteration k+1 is due, computes its residual statistics from the updated iterate, so each
// sub-iteration streams the iterate once.  The loop condition lives on the device
// (InvCtl.exec), so all max_iter+1 launches are enqueued up front and the ones past
// convergence return at once.
// ------------------------------------------------------------------------------------------
struct InvParams {
  float A[9];
  float ih[3];
  int k, max_iter, phase, stop_aware, zb, halves;
  double mean_tol, max_tol;
};

template <int DIM, bool DIAG>
__device__ __forceinline__ void residual(const float* __restrict__ phi, const Dims& d, const float* A, float fx,
                                         float fy, float fz, const float p[3], float e[3]) {
  float cx, cy, cz;
  if (DIAG) {
    cx = fmaf(A[0], p[0], fx);
    cy = fmaf(A[4], p[1], fy);
    cz = DIM == 3 ? fmaf(A[8], p[2], fz) : 0.0f;
  } else {
  cx = fx + A[0] * p[0] + A[1] * p[1];
  cy = fy + A[3] * p[0] + A[4] * p[1];
  cz = 0.0f;
  if (DIM == 3) {
    cx += A[2] * p[2];
    cy += A[5] * p[2];
    cz = fz + A[6] * p[0] + A[7] * p[1] + A[8] * p[2];
  }
  }
  e[0] = p[0];
  e[1] = p[1];
  e[2] = DIM == 3 ? p[2] : 0.0f;
  if (inside_buffer<DIM>(d, cx, cy, cz)) {
    const Cell c = make_cell<DIM>(d, cx, cy, cz);
    const int N = (int)d.N;
    e[0] += lerp_at<DIM>(phi, c);
    e[1] += lerp_at<DIM>(phi + N, c);
    if (DIM == 3) e[2] += lerp_at<DIM>(phi + 2 * N, c);
  }
}

template <int DIM, bool DIAG>
__global__ void __launch_bounds__(256, 4) k_invert_step(Ptr2c phis, Ptr2 psis, Dims d, InvParams P, IterCtl* ctl,
                                                     double* __restrict__ psum, float* __restrict__ pmax, int pcap) {
  if (P.stop_aware && ctl->stop) return;
  __shared__ double redd[32];
  __shared__ float redf[32];
  __shared__ int am_last;
  const Coord3 c3 = coord3(d, P.zb, P.halves);
  const int h = c3.h;
  InvCtl& C = ctl->inv[P.phase][h];
  const float* __restrict__ phi = (h ? phis.p[1] : phis.p[0]);
  float* __restrict__ psi = (h ? psis.p[1] : psis.p[0]);
  const int k = P.k;
  bool apply = false, stats = true;
  float eps = 0.0f, lim = 0.0f;
  if (k > 0) {
    const int s = k & 1;
    if (!C.exec[s]) {
      if (c3.bid == 0 && threadIdx.x == 0) C.exec[s ^ 1] = 0;
      return;
    }
    apply = true;
    eps = k == 1 ? 0.75f : 0.5f;
    const float mx = C.maxv[s];
    const double mean = C.mean[s];
    lim = eps * mx;
    stats = (k + 1 <= P.max_iter) && ((double)mx > P.max_tol) && (mean > P.mean_tol);
    if (!stats && c3.bid == 0 && threadIdx.x == 0) {
      C.exec[s ^ 1] = 0;
      C.iters = k;
    }
  }
  if (!stats && !c3.ok) return;
  const int N = (int)d.N, nxy = d.nx * d.ny;
  double acc = 0.0;
  float mxl = 0.0f;
  if (c3.ok) {
    const float fx = (float)c3.x, fy = (float)c3.y;
    const bool xyedge = c3.x == 0 || c3.x == d.nx - 1 || c3.y == 0 || c3.y == d.ny - 1;
    // the iterate of the next slice is loaded before this slice's gathers (one dependent
    // memory round trip per slice instead of two)
    const int i0 = c3.z0 * nxy + c3.y * d.nx + c3.x;
    float pn[3] = {0.0f, 0.0f, 0.0f};
    if (c3.z0 < c3.z1) {
      pn[0] = psi[i0];
      pn[1] = psi[N + i0];
      pn[2] = DIM == 3 ? psi[2 * N + i0] : 0.0f;
    }
    for (int z = c3.z0; z < c3.z1; ++z) {
      const int i = z * nxy + c3.y * d.nx + c3.x;
      const float fz = (float)z;
      float p[3] = {pn[0], pn[1], pn[2]};
      if (z + 1 < c3.z1) {
        pn[0] = psi[i + nxy];
        pn[1] = psi[N + i + nxy];
        pn[2] = DIM == 3 ? psi[2 * N + i + nxy] : 0.0f;
      }
      float e[3];
      if (apply) {
        residual<DIM, DIAG>(phi, d, P.A, fx, fy, fz, p, e);
        float s2 = 0.0f;
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
          const float v = e[c] * P.ih[c];
          s2 += v * v;
        }
        const float nrm = sqrtf(s2);
        const float f = nrm > lim ? lim / nrm : 1.0f;
        const bool edge = xyedge || (DIM == 3 && (z == 0 || z == d.nz - 1));
#pragma unroll
        for (int c = 0; c < DIM; ++c) p[c] = edge ? 0.0f : p[c] + ((-e[c]) * f) * eps;
        psi[i] = p[0];
        psi[N + i] = p[1];
        if (DIM == 3) psi[2 * N + i] = p[2];
      }
      if (stats) {
        residual<DIM, DIAG>(phi, d, P.A, fx, fy, fz, p, e);
        float s2 = 0.0f;
#pragma unroll
        for (int c = 0; c < DIM; ++c) {
          const float v = e[c] * P.ih[c];
          s2 += v * v;
        }
        const float nrm = sqrtf(s2);
        acc += (double)nrm;
        mxl = fmaxf(mxl, nrm);
      }
    }
  }
  if (!stats) return;
  const double bs = block_sum_d(acc, redd);
  const float bm = block_max_f(mxl, redf);
  const int nb = gridDim.x * gridDim.y * (gridDim.z / P.halves);
  if (threadIdx.x == 0) {
    psum[h * pcap + c3.bid] = bs;
    pmax[h * pcap + c3.bid] = bm;
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
      C.mean[s1] = s / (double)N;
      C.maxv[s1] = m;
      C.exec[s1] = 1;
      C.iters = k;
      C.counter = 0u;
    }
  }
}

constexpr int kInvTarget = 148 * 24;  // blocks: short per-thread z walks, small last-wave tail
int inv_blocks(const GridInfo& g) { return map3(g.d, 2, kInvTarget).nblocks; }

void launch_invert_step(const float* const* phi, float* const* psi, int halves, const GridInfo& g, int k, int max_iter,
                        double mean_tol, double max_tol, IterCtl* ctl, int phase, PartialBufs pb, cudaStream_t s,
                        bool stop_aware) {
  count_launch();
  Ptr2c pp{{phi[0], halves > 1 ? phi[1] : phi[0]}};
  Ptr2 ps{{psi[0], halves > 1 ? psi[1] : psi[0]}};
  InvParams P;
  Affine a = make_affine(g, g);
  for (int j = 0; j < 9; ++j) P.A[j] = a.A[j];
  for (int j = 0; j < 3; ++j) P.ih[j] = (float)(1.0 / g.sp[j]);
  // the block decomposition is the same for one or two halves, so the partial buffers sized
  // by inv_blocks() fit either
  const Map3 m2 = map3(g.d, 2, kInvTarget);
  Map3 m = m2;
  m.grid.z = (m2.grid.z / 2) * halves;
  P.k = k;
  P.max_iter = max_iter;
  P.phase = phase;
  P.stop_aware = stop_aware ? 1 : 0;
  P.zb = m.zb;
  P.halves = halves;
  P.mean_tol = mean_tol;
  P.max_tol = max_tol;
  const bool dg = affine_diag(a);
  if (g.d.dim == 3) {
    if (dg)
      k_invert_step<3, true><<<m.grid, 256, 0, s>>>(pp, ps, g.d, P, ctl, pb.sum, pb.maxv, pb.capacity);
    else
      k_invert_step<3, false><<<m.grid, 256, 0, s>>>(pp, ps, g.d, P, ctl, pb.sum, pb.maxv, pb.capacity);
  } else {
    if (dg)
      k_invert_step<2, true><<<m.grid, 256, 0, s>>>(pp, ps, g.d, P, ctl, pb.sum, pb.maxv, pb.capacity);
    else
      k_invert_step<2, false><<<m.grid, 256, 0, s>>>(pp, ps, g.d, P, ctl, pb.sum, pb.maxv, pb.capacity);
  }
}

// ------------------------------------------------------------------------------------------
// Convergence monitor and per-iteration log (one thread).
// ------------------------------------------------------------------------------------------
__global__ void k_converge(IterCtl* ctl, LogDev log, double threshold, int window) {
  if (ctl->stop) return;
  const int k = ctl->iter;
  const double v = ctl->metric;
  ctl->total_abs += fabs(v);
  const int W = window < 2 ? 2 : (window > kMaxWindow ? kMaxWindow : window);
  ctl->energies[k % W] = v;
  const int k1 = k + 1;
  double conv = DBL_MAX;
  if (k1 >= W) {
    double num0 = 0, den0 = 0, num1 = 0, den1 = 0;
    for (int j = 0; j < W; ++j) {
      const double u = (double)j / (double)(W - 1);
      const double z = ctl->energies[(k1 - W + j) % W] / ctl->total_abs;
      const double w0 = 1.0 - u, w1 = u, ws = w0 * w0 + w1 * w1;
      num0 += w0 * w0 * (w0 * z / ws);
      den0 += w0 * w0;
      num1 += w1 * w1 * (w1 * z / ws);
      den1 += w1 * w1;
    }
    const double c0 = den0 > 0 ? num0 / den0 : 0.0, c1 = den1 > 0 ? num1 / den1 : 0.0;
    conv = -(c1 - c0);
  }
  if (k < log.cap) {
    log.metric[k] = v;
    log.conv[k] = conv;
    log.inv_iters[k] = ctl->inv[0][0].iters + ctl->inv[0][1].iters + ctl->inv[1][0].iters + ctl->inv[1][1].iters;
  }
  ctl->iter = k1;
  if (conv < threshold) ctl->stop = 1;
}

void launch_converge(IterCtl* ctl, LogDev log, double threshold, int window, cudaStream_t s) {
  count_launch();
  k_converge<<<1, 1, 0, s>>>(ctl, log, threshold, window);
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

template <int DIM>
__global__ void __launch_bounds__(256) k_resample(Ptr4c in, Dims di, Ptr4 out, Dims dout, int zb, Affine m, int nf) {
  const Coord3 c3 = coord3(dout, zb, 1);
  if (!c3.ok) return;
  const int No = (int)dout.N, Ni = (int)di.N, nxy = dout.nx * dout.ny;
  for (int z = c3.z0; z < c3.z1; ++z) {
    const int i = z * nxy + c3.y * dout.nx + c3.x;
    float cx, cy, cz;
    map_point<DIM>(m, (float)c3.x, (float)c3.y, (float)z, 0.0f, 0.0f, 0.0f, cx, cy, cz);
    const bool ok = inside_buffer<DIM>(di, cx, cy, cz);
    Cell c{};
    if (ok) c = make_cell<DIM>(di, cx, cy, cz);
    for (int f = 0; f < nf; ++f)
#pragma unroll
      for (int k = 0; k < DIM; ++k) out.p[f][k * No + i] = ok ? lerp_at<DIM>(in.p[f] + k * Ni, c) : 0.0f;
  }
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
  Affine a = make_affine(go, gi);
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
    for (int j = 0; j <= 2 * R; ++j) {
      const int q = min(max(pos + j - R, 0), len - 1);
      s += __ldg(coeffs + j) * (double)__ldg(line + q * astride);
    }
    out[i] = (float)s;
  }
}

void launch_conv_image_axis(const float* in, float* out, const GridInfo& g, int axis, const double* coeffs, int R,
                            cudaStream_t s) {
  count_launch();
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
