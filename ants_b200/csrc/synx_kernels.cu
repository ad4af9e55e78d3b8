// synx kernels for sm_100a: the per-voxel steps of one SyN + neighbourhood-CC iteration.
//
// Everything here is memory-bound stencil / gather work (no contraction), so the design goals
// are coalesced component-plane access, shared-memory staging of stencil halos, FP64 only
// where the arithmetic needs it (CC window sums, global means), and device-side loop control
// so that a whole level can be enqueued (or graph-replayed) without host round trips.
#include <cfloat>
#include <cmath>
#include <atomic>
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

__device__ __forceinline__ void voxel_xyz(long long i, const Dims& d, int& x, int& y, int& z) {
  x = (int)(i % d.nx);
  long long r = i / d.nx;
  y = (int)(r % d.ny);
  z = (int)(r / d.ny);
}

template <int DIM>
__device__ __forceinline__ void map_point(const Affine& m, float fx, float fy, float fz, float ux, float uy, float uz,
                                          float& cx, float& cy, float& cz) {
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
template <int DIM>
__global__ void __launch_bounds__(256)
    k_warp_pair(const float* __restrict__ F, Dims dF, Affine mF, const float* __restrict__ psiF,
                const float* __restrict__ M, Dims dM, Affine mM, const float* __restrict__ psiM, Dims dv,
                float* __restrict__ Ft, float* __restrict__ Mt, IterCtl* ctl) {
  if (ctl != nullptr && ctl->stop) return;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && ctl != nullptr) {
    ctl->maxnorm[0] = 0u;
    ctl->maxnorm[1] = 0u;
  }
  const long long N = dv.N, stride = (long long)gridDim.x * blockDim.x;
  for (; i < N; i += stride) {
    int x, y, z;
    voxel_xyz(i, dv, x, y, z);
    const float fx = (float)x, fy = (float)y, fz = (float)z;
    float cx, cy, cz;
    {
      float ux = psiF[i], uy = psiF[N + i], uz = DIM == 3 ? psiF[2 * N + i] : 0.0f;
      map_point<DIM>(mF, fx, fy, fz, ux, uy, uz, cx, cy, cz);
      float v = 0.0f;
      if (inside_buffer<DIM>(dF, cx, cy, cz)) v = lerp_at<DIM>(F, make_cell<DIM>(dF, cx, cy, cz));
      Ft[i] = v;
    }
    {
      float ux = psiM[i], uy = psiM[N + i], uz = DIM == 3 ? psiM[2 * N + i] : 0.0f;
      map_point<DIM>(mM, fx, fy, fz, ux, uy, uz, cx, cy, cz);
      float v = 0.0f;
      if (inside_buffer<DIM>(dM, cx, cy, cz)) v = lerp_at<DIM>(M, make_cell<DIM>(dM, cx, cy, cz));
      Mt[i] = v;
    }
  }
}

void launch_warp_pair(const float* F, const GridInfo& gF, const float* psiF, const float* M, const GridInfo& gM,
                      const float* psiM, const GridInfo& gv, float* Ft, float* Mt, IterCtl* ctl, cudaStream_t s) {
  count_launch();
  Affine mF = make_affine(gv, gF), mM = make_affine(gv, gM);
  int blocks = grid_for(gv.d.N, 256);
  if (gv.d.dim == 3)
    k_warp_pair<3><<<blocks, 256, 0, s>>>(F, gF.d, mF, psiF, M, gM.d, mM, psiM, gv.d, Ft, Mt, ctl);
  else
    k_warp_pair<2><<<blocks, 256, 0, s>>>(F, gF.d, mF, psiF, M, gM.d, mM, psiM, gv.d, Ft, Mt, ctl);
}

template <int DIM>
__global__ void __launch_bounds__(256) k_warp_image(const float* __restrict__ img, Dims di, Affine m,
                                                    const float* __restrict__ u, Dims dv, float* __restrict__ out) {
  const long long N = dv.N, stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    int x, y, z;
    voxel_xyz(i, dv, x, y, z);
    float ux = u[i], uy = u[N + i], uz = DIM == 3 ? u[2 * N + i] : 0.0f;
    float cx, cy, cz;
    map_point<DIM>(m, (float)x, (float)y, (float)z, ux, uy, uz, cx, cy, cz);
    float v = 0.0f;
    if (inside_buffer<DIM>(di, cx, cy, cz)) v = lerp_at<DIM>(img, make_cell<DIM>(di, cx, cy, cz));
    out[i] = v;
  }
}

void launch_warp_image(const float* img, const GridInfo& gi, const float* u, const GridInfo& gv, float* out,
                       cudaStream_t s) {
  count_launch();
  Affine m = make_affine(gv, gi);
  int blocks = grid_for(gv.d.N, 256);
  if (gv.d.dim == 3)
    k_warp_image<3><<<blocks, 256, 0, s>>>(img, gi.d, m, u, gv.d, out);
  else
    k_warp_image<2><<<blocks, 256, 0, s>>>(img, gi.d, m, u, gv.d, out);
}

// ------------------------------------------------------------------------------------------
// Neighbourhood cross-correlation: value and both update directions.
//
// A block owns a 32 x 8 tile of output columns and marches along z over a chunk of ZC
// slices.  Each thread keeps FP64 running z-window sums of F, M, F^2, M^2, FM for up to CPT
// halo columns; the raw (F, M) values of the last 2R+1 slices sit in a shared-memory ring so
// the leaving slice is subtracted without a second global read.  Per slice the column sums
// are box-summed along x and then y in shared memory (FP64), giving the five window sums of
// each output voxel, from which the CC terms and derivatives follow.  The in-bounds count is
// separable (cx*cy*cz) and computed analytically.
// ------------------------------------------------------------------------------------------
struct CCParams {
  float h[3];      // spacing
  float dir[9];    // direction cosines
  int identity_dir;
  double eps;
  int ZC;          // z-chunk per block
};

__device__ __forceinline__ int pmod(int a, int m) {
  int r = a % m;
  return r < 0 ? r + m : r;
}

__device__ __forceinline__ float grad1(float vm, float v0, float vp, int pos, int n, float h) {
  if (n < 2 || pos == n - 1) return 0.0f;
  if (pos == 0) return 0.5f * (vp - v0) / h;
  return (vp - vm) / (2.0f * h);
}

template <int R, int DIM>
struct CCShape {
  static constexpr int TX = 32, TY = 8;
  static constexpr int HX = TX + 2 * R, HY = TY + 2 * R, HC = HX * HY;
  static constexpr int RZ = DIM == 3 ? R : 0;
  static constexpr int RD = 2 * RZ + 1;
  static constexpr int CPT = (HC + 255) / 256;
  static constexpr size_t smem = (size_t)RD * HC * sizeof(float2) + (size_t)5 * HC * sizeof(double) +
                                 (size_t)5 * HY * TX * sizeof(double);
};

template <int R, int DIM>
__global__ void __launch_bounds__(256)
    k_cc(const float* __restrict__ Ft, const float* __restrict__ Mt, Dims d, CCParams P, float* __restrict__ gF,
         float* __restrict__ gM, double* __restrict__ partials, IterCtl* ctl, float* __restrict__ cc_out) {
  using S = CCShape<R, DIM>;
  constexpr int TX = S::TX, HX = S::HX, HY = S::HY, HC = S::HC, RZ = S::RZ, RD = S::RD, CPT = S::CPT;
  if (ctl != nullptr && ctl->stop) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* ring = reinterpret_cast<float2*>(smem_raw);
  double* cs = reinterpret_cast<double*>(ring + RD * HC);
  double* xs = cs + 5 * HC;
  __shared__ double red[32];
  __shared__ int am_last;

  const int tid = threadIdx.x;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const long long nxy = (long long)nx * ny, N = d.N;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * S::TY;
  const int z0 = blockIdx.z * P.ZC;
  const int z1 = min(z0 + P.ZC, nz);

  // owned halo columns
  int gofs[CPT];
  bool gval[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    int col = tid + c * 256;
    int hx = col % HX, hy = col / HX;
    int gx = x0 - R + hx, gy = y0 - R + hy;
    gval[c] = col < HC && gx >= 0 && gx < nx && gy >= 0 && gy < ny;
    gofs[c] = gval[c] ? gy * nx + gx : 0;
  }
  double acc[CPT][5];
#pragma unroll
  for (int c = 0; c < CPT; ++c)
#pragma unroll
    for (int q = 0; q < 5; ++q) acc[c][q] = 0.0;

  // warm-up: slices z0-RZ .. z0+RZ-1
  for (int zs = z0 - RZ; zs < z0 + RZ; ++zs) {
    const bool zin = zs >= 0 && zs < nz;
    const int slot = pmod(zs, RD);
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      int col = tid + c * 256;
      if (col < HC) {
        float2 v = make_float2(0.0f, 0.0f);
        if (zin && gval[c]) {
          long long o = (long long)zs * nxy + gofs[c];
          v.x = __ldg(Ft + o);
          v.y = __ldg(Mt + o);
          double f = v.x, m = v.y;
          acc[c][0] += f;
          acc[c][1] += m;
          acc[c][2] += f * f;
          acc[c][3] += m * m;
          acc[c][4] += f * m;
        }
        ring[slot * HC + col] = v;
      }
    }
  }

  double cc_acc = 0.0;
  const int tx = tid & 31, ty = tid >> 5;
  const int ox = x0 + tx, oy = y0 + ty;
  const bool out_ok = ox < nx && oy < ny;
  const double cxn = (double)(min(ox + R, nx - 1) - max(ox - R, 0) + 1);
  const double cyn = (double)(min(oy + R, ny - 1) - max(oy - R, 0) + 1);

  for (int zc = z0; zc < z1; ++zc) {
    // slide the z window: subtract slice zc-RZ-1 (if it was added), add slice zc+RZ
    const int ze = zc + RZ, zl = zc - RZ - 1;
    const int slot = pmod(ze, RD);
    const bool sub = zc > z0 && zl >= 0;
    const bool zin = ze < nz;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      int col = tid + c * 256;
      if (col < HC) {
        if (sub && gval[c]) {
          float2 o = ring[slot * HC + col];
          double f = o.x, m = o.y;
          acc[c][0] -= f;
          acc[c][1] -= m;
          acc[c][2] -= f * f;
          acc[c][3] -= m * m;
          acc[c][4] -= f * m;
        }
        float2 v = make_float2(0.0f, 0.0f);
        if (zin && gval[c]) {
          long long o = (long long)ze * nxy + gofs[c];
          v.x = __ldg(Ft + o);
          v.y = __ldg(Mt + o);
          double f = v.x, m = v.y;
          acc[c][0] += f;
          acc[c][1] += m;
          acc[c][2] += f * f;
          acc[c][3] += m * m;
          acc[c][4] += f * m;
        }
        ring[slot * HC + col] = v;
#pragma unroll
        for (int q = 0; q < 5; ++q) cs[q * HC + col] = acc[c][q];
      }
    }
    __syncthreads();
    // x box sums: HY rows x TX outputs
    for (int p = tid; p < HY * TX; p += 256) {
      const int hy = p / TX, px = p % TX;
      const double* src = cs + hy * HX + px;
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j <= 2 * R; ++j) s += src[q * HC + j];
        xs[q * HY * TX + p] = s;
      }
    }
    __syncthreads();
    if (out_ok) {
      double Sq[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j <= 2 * R; ++j) s += xs[q * HY * TX + (ty + j) * TX + tx];
        Sq[q] = s;
      }
      const double czn = (double)(min(zc + RZ, nz - 1) - max(zc - RZ, 0) + 1);
      const double n = cxn * cyn * czn;
      const double inv_n = __drcp_rn(n);
      const double mF = Sq[0] * inv_n, mM = Sq[1] * inv_n;
      const double sFF = Sq[2] - mF * Sq[0] - mF * Sq[0] + n * mF * mF;
      const double sMM = Sq[3] - mM * Sq[1] - mM * Sq[1] + n * mM * mM;
      const double sFM = Sq[4] - mM * Sq[0] - mF * Sq[1] + n * mM * mF;
      const int cidx = (ty + R) * HX + (tx + R);
      const float2* rc = ring + pmod(zc, RD) * HC;
      const float2 v0 = rc[cidx];
      const double fh = (double)v0.x - mF, mh = (double)v0.y - mM;
      double cc = 1.0, aF = 0.0, aM = 0.0;
      if (sFF > P.eps && sMM > P.eps) {
        const double prod = sFF * sMM;
        const double ip = __drcp_rn(prod);
        cc = sFM * sFM * ip;
        const double coef = 2.0 * sFM * ip;
        aF = coef * (fh - sFM * sFF * ip * mh);
        aM = coef * (mh - sFM * sMM * ip * fh);
      }
      cc_acc += cc;
      // central differences of both warped images (index axes)
      float gMi[3], gFi[3];
      {
        const float2 xm = rc[cidx - 1], xp = rc[cidx + 1];
        gMi[0] = grad1(xm.y, v0.y, xp.y, ox, nx, P.h[0]);
        gFi[0] = grad1(xm.x, v0.x, xp.x, ox, nx, P.h[0]);
        const float2 ym = rc[cidx - HX], yp = rc[cidx + HX];
        gMi[1] = grad1(ym.y, v0.y, yp.y, oy, ny, P.h[1]);
        gFi[1] = grad1(ym.x, v0.x, yp.x, oy, ny, P.h[1]);
        gMi[2] = gFi[2] = 0.0f;
        if (DIM == 3) {
          const float2 zm = ring[pmod(zc - 1, RD) * HC + cidx], zp = ring[pmod(zc + 1, RD) * HC + cidx];
          gMi[2] = grad1(zm.y, v0.y, zp.y, zc, nz, P.h[2]);
          gFi[2] = grad1(zm.x, v0.x, zp.x, zc, nz, P.h[2]);
        }
      }
      const long long oi = (long long)zc * nxy + (long long)oy * nx + ox;
#pragma unroll
      for (int dd = 0; dd < DIM; ++dd) {
        float pm, pf;
        if (P.identity_dir) {
          pm = gMi[dd];
          pf = gFi[dd];
        } else {
          pm = 0.0f;
          pf = 0.0f;
#pragma unroll
          for (int a = 0; a < DIM; ++a) {
            pm += P.dir[dd * 3 + a] * gMi[a];
            pf += P.dir[dd * 3 + a] * gFi[a];
          }
        }
        gF[dd * N + oi] = (float)(aF * (double)pm);
        gM[dd * N + oi] = (float)(aM * (double)pf);
      }
      if (cc_out != nullptr) cc_out[oi] = (float)cc;
    }
    __syncthreads();
  }

  // deterministic reduction of sum(cc): block partials, the last block sums them in order
  const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
  const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  double bs = block_sum_d(cc_acc, red);
  if (tid == 0) {
    partials[bid] = bs;
    __threadfence();
    unsigned t = atomicAdd(&ctl->cc_counter, 1u);
    am_last = (t == nblocks - 1);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    double s = 0.0;
    for (unsigned b = tid; b < nblocks; b += 256) s += __ldcg(partials + b);
    s = block_sum_d(s, red);
    if (tid == 0) {
      ctl->cc_sum = s;
      ctl->metric = -s / (double)N;
      ctl->cc_counter = 0u;
    }
  }
}

template <int R, int DIM>
static void cc_launch_t(const float* Ft, const float* Mt, const GridInfo& g, float* gF, float* gM, double* partials,
                        IterCtl* ctl, cudaStream_t s, float* cc_out, dim3 grid, const CCParams& P) {
  using S = CCShape<R, DIM>;
  k_cc<R, DIM><<<grid, 256, S::smem, s>>>(Ft, Mt, g.d, P, gF, gM, partials, ctl, cc_out);
}

static int cc_zchunk(const GridInfo& g, int radius) {
  if (g.d.dim == 2) return 1;
  const int bx = (g.d.nx + 31) / 32, by = (g.d.ny + 7) / 8;
  const int target = 148 * 6;
  int chunks = (target + bx * by - 1) / (bx * by);
  int zc = (g.d.nz + chunks - 1) / chunks;
  zc = zc < 4 * radius ? 4 * radius : zc;
  if (zc > g.d.nz) zc = g.d.nz;
  if (zc < 1) zc = 1;
  return zc;
}

int cc_blocks(const GridInfo& g, int radius) {
  const int bx = (g.d.nx + 31) / 32, by = (g.d.ny + 7) / 8;
  const int zc = cc_zchunk(g, radius);
  return bx * by * ((g.d.nz + zc - 1) / zc);
}

size_t cc_smem_bytes(int dim, int radius) {
  const size_t TX = 32, TY = 8, HX = TX + 2 * radius, HY = TY + 2 * radius, HC = HX * HY;
  const size_t RD = dim == 3 ? 2 * radius + 1 : 1;
  return RD * HC * 8 + 5 * HC * 8 + 5 * HY * TX * 8;
}

template <int R, int DIM>
static cudaError_t cc_prepare_t() {
  return cudaFuncSetAttribute(k_cc<R, DIM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CCShape<R, DIM>::smem);
}

cudaError_t cc_prepare(int dim, int radius) {
#define SYNX_CC_PREP(RR) \
  case RR:               \
    return dim == 3 ? cc_prepare_t<RR, 3>() : cc_prepare_t<RR, 2>();
  switch (radius) {
    SYNX_CC_PREP(1)
    SYNX_CC_PREP(2)
    SYNX_CC_PREP(3)
    SYNX_CC_PREP(4)
    SYNX_CC_PREP(5)
    SYNX_CC_PREP(6)
    SYNX_CC_PREP(7)
    default:
      return cudaErrorInvalidValue;
  }
#undef SYNX_CC_PREP
}

bool cc_radius_supported(int dim, int radius) {
  return radius >= 1 && radius <= 7 && cc_smem_bytes(dim, radius) <= 227 * 1024;
}

void launch_cc(const float* Ft, const float* Mt, const GridInfo& g, int radius, float* gF, float* gM, double* partials,
               IterCtl* ctl, cudaStream_t s, float* cc_out) {
  count_launch();
  CCParams P;
  for (int k = 0; k < 3; ++k) P.h[k] = (float)g.sp[k];
  bool ident = true;
  for (int k = 0; k < 9; ++k) {
    P.dir[k] = (float)g.dir[k];
    if (g.dir[k] != ((k % 4) == 0 ? 1.0 : 0.0)) ident = false;
  }
  P.identity_dir = ident ? 1 : 0;
  P.eps = 1.1920928955078125e-07;  // FLT_EPSILON: the reference metric's float guard
  P.ZC = cc_zchunk(g, radius);
  dim3 grid((g.d.nx + 31) / 32, (g.d.ny + 7) / 8, (g.d.nz + P.ZC - 1) / P.ZC);
#define SYNX_CC_CASE(RR)                                                                         \
  case RR:                                                                                       \
    if (g.d.dim == 3)                                                                            \
      cc_launch_t<RR, 3>(Ft, Mt, g, gF, gM, partials, ctl, s, cc_out, grid, P);                  \
    else                                                                                         \
      cc_launch_t<RR, 2>(Ft, Mt, g, gF, gM, partials, ctl, s, cc_out, grid, P);                  \
    break;
  switch (radius) {
    SYNX_CC_CASE(1)
    SYNX_CC_CASE(2)
    SYNX_CC_CASE(3)
    SYNX_CC_CASE(4)
    SYNX_CC_CASE(5)
    SYNX_CC_CASE(6)
    SYNX_CC_CASE(7)
    default:
      break;
  }
#undef SYNX_CC_CASE
}

// ------------------------------------------------------------------------------------------
// Separable Gaussian smoothing of displacement fields (both halves per launch, blockIdx.y).
// ------------------------------------------------------------------------------------------
struct Ptr2c {
  const float* p[2];
};
struct Ptr2 {
  float* p[2];
};

template <int DIM>
__global__ void __launch_bounds__(256)
    k_smooth_pass(Ptr2c in, Ptr2 out, Ptr2c orig, Dims d, int axis, const float* __restrict__ coeffs, int R, int last,
                  float w1, float w2, int do_max, float ihx, float ihy, float ihz, IterCtl* ctl) {
  if (ctl != nullptr && ctl->stop) return;
  __shared__ float red[32];
  const int h = blockIdx.y;
  const float* __restrict__ src = in.p[h];
  float* __restrict__ dst = out.p[h];
  const float* __restrict__ org = orig.p[h];
  const long long N = d.N, stride = (long long)gridDim.x * blockDim.x;
  const int len = axis == 0 ? d.nx : (axis == 1 ? d.ny : d.nz);
  const long long astride = axis == 0 ? 1 : (axis == 1 ? d.nx : (long long)d.nx * d.ny);
  const float ih[3] = {ihx, ihy, ihz};
  float mx = 0.0f;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    int x, y, z;
    voxel_xyz(i, d, x, y, z);
    const int pos = axis == 0 ? x : (axis == 1 ? y : z);
    const bool edge = last && (x == 0 || x == d.nx - 1 || y == 0 || y == d.ny - 1 ||
                               (DIM == 3 && (z == 0 || z == d.nz - 1)));
    float nrm2 = 0.0f;
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      const float* line = src + c * N + i - pos * astride;
      float s = 0.0f;
      if (pos >= R && pos + R < len) {
        const float* q = line + (long long)(pos - R) * astride;
        for (int j = 0; j <= 2 * R; ++j) s = fmaf(__ldg(coeffs + j), __ldg(q + j * astride), s);
      } else {
        for (int j = 0; j <= 2 * R; ++j) {
          int qq = min(max(pos + j - R, 0), len - 1);
          s = fmaf(__ldg(coeffs + j), __ldg(line + (long long)qq * astride), s);
        }
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
  dim3 grid(grid_for(g.d.N, 256), halves);
  float ih[3] = {(float)(1.0 / g.sp[0]), (float)(1.0 / g.sp[1]), (float)(1.0 / g.sp[2])};
  if (g.d.dim == 3)
    k_smooth_pass<3><<<grid, 256, 0, s>>>(pi, po, pg, g.d, axis, coeffs, R, last ? 1 : 0, w1, w2, maxnorm ? 1 : 0,
                                          ih[0], ih[1], ih[2], ctl);
  else
    k_smooth_pass<2><<<grid, 256, 0, s>>>(pi, po, pg, g.d, axis, coeffs, R, last ? 1 : 0, w1, w2, maxnorm ? 1 : 0,
                                          ih[0], ih[1], ih[2], ctl);
}

// ------------------------------------------------------------------------------------------
// Composition out = w + s * d(x + w), s = eta / max||d/spacing|| (SyN's update scaling fused).
// Reads w only at its own voxel, so it runs in place (out == w).
// ------------------------------------------------------------------------------------------
template <int DIM>
__global__ void __launch_bounds__(256) k_compose(Ptr2c dd, Ptr2c ww, Ptr2 oo, Dims d, Affine m, double eta,
                                                 IterCtl* ctl) {
  if (ctl != nullptr && ctl->stop) return;
  const int h = blockIdx.y;
  const float* __restrict__ D = dd.p[h];
  const float* W = ww.p[h];
  float* O = oo.p[h];
  float scale = 1.0f;
  if (eta > 0.0) {
    const float mx = __uint_as_float(ctl->maxnorm[h]);
    scale = mx > 0.0f ? (float)(eta / (double)mx) : (float)eta;
  }
  const long long N = d.N, stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    int x, y, z;
    voxel_xyz(i, d, x, y, z);
    const float w0 = W[i], w1 = W[N + i], w2 = DIM == 3 ? W[2 * N + i] : 0.0f;
    float cx, cy, cz;
    map_point<DIM>(m, (float)x, (float)y, (float)z, w0, w1, w2, cx, cy, cz);
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
  Affine m = make_affine(g, g);
  dim3 grid(grid_for(g.d.N, 256), halves);
  if (g.d.dim == 3)
    k_compose<3><<<grid, 256, 0, s>>>(pd, pw, po, g.d, m, (double)eta, ctl);
  else
    k_compose<2><<<grid, 256, 0, s>>>(pd, pw, po, g.d, m, (double)eta, ctl);
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
  int k, max_iter, phase, stop_aware;
  double mean_tol, max_tol;
};

template <int DIM>
__device__ __forceinline__ void residual(const float* __restrict__ phi, const Dims& d, const float* A, int x, int y,
                                         int z, long long i, const float p[3], float e[3]) {
  float cx, cy, cz;
  cx = (float)x + A[0] * p[0] + A[1] * p[1];
  cy = (float)y + A[3] * p[0] + A[4] * p[1];
  cz = 0.0f;
  if (DIM == 3) {
    cx += A[2] * p[2];
    cy += A[5] * p[2];
    cz = (float)z + A[6] * p[0] + A[7] * p[1] + A[8] * p[2];
  }
  e[0] = p[0];
  e[1] = p[1];
  e[2] = DIM == 3 ? p[2] : 0.0f;
  if (inside_buffer<DIM>(d, cx, cy, cz)) {
    const Cell c = make_cell<DIM>(d, cx, cy, cz);
    const long long N = d.N;
    e[0] += lerp_at<DIM>(phi, c);
    e[1] += lerp_at<DIM>(phi + N, c);
    if (DIM == 3) e[2] += lerp_at<DIM>(phi + 2 * N, c);
  }
  (void)i;
}

template <int DIM>
__global__ void __launch_bounds__(256) k_invert_step(Ptr2c phis, Ptr2 psis, Dims d, InvParams P, IterCtl* ctl,
                                                     double* __restrict__ psum, float* __restrict__ pmax, int pcap) {
  if (P.stop_aware && ctl->stop) return;
  __shared__ double redd[32];
  __shared__ float redf[32];
  __shared__ int am_last;
  const int h = blockIdx.y;
  InvCtl& C = ctl->inv[P.phase][h];
  const float* __restrict__ phi = phis.p[h];
  float* __restrict__ psi = psis.p[h];
  const int k = P.k;
  bool apply = false, stats = true;
  float eps = 0.0f, lim = 0.0f;
  if (k > 0) {
    const int s = k & 1;
    if (!C.exec[s]) {
      if (blockIdx.x == 0 && threadIdx.x == 0) C.exec[s ^ 1] = 0;
      return;
    }
    apply = true;
    eps = k == 1 ? 0.75f : 0.5f;
    const float mx = C.maxv[s];
    const double mean = C.mean[s];
    lim = eps * mx;
    stats = (k + 1 <= P.max_iter) && ((double)mx > P.max_tol) && (mean > P.mean_tol);
    if (!stats) {
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        C.exec[s ^ 1] = 0;
        C.iters = k;
      }
    }
  }
  const long long N = d.N, stride = (long long)gridDim.x * blockDim.x;
  double acc = 0.0;
  float mxl = 0.0f;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    int x, y, z;
    voxel_xyz(i, d, x, y, z);
    float p[3];
    p[0] = psi[i];
    p[1] = psi[N + i];
    p[2] = DIM == 3 ? psi[2 * N + i] : 0.0f;
    float e[3];
    if (apply) {
      residual<DIM>(phi, d, P.A, x, y, z, i, p, e);
      float s2 = 0.0f;
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        const float v = e[c] * P.ih[c];
        s2 += v * v;
      }
      const float nrm = sqrtf(s2);
      const float f = nrm > lim ? lim / nrm : 1.0f;
      const bool edge = x == 0 || x == d.nx - 1 || y == 0 || y == d.ny - 1 || (DIM == 3 && (z == 0 || z == d.nz - 1));
#pragma unroll
      for (int c = 0; c < DIM; ++c) p[c] = edge ? 0.0f : p[c] + ((-e[c]) * f) * eps;
      psi[i] = p[0];
      psi[N + i] = p[1];
      if (DIM == 3) psi[2 * N + i] = p[2];
    }
    if (stats) {
      residual<DIM>(phi, d, P.A, x, y, z, i, p, e);
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
  if (!stats) return;
  const double bs = block_sum_d(acc, redd);
  const float bm = block_max_f(mxl, redf);
  if (threadIdx.x == 0) {
    psum[h * pcap + blockIdx.x] = bs;
    pmax[h * pcap + blockIdx.x] = bm;
    __threadfence();
    const unsigned t = atomicAdd(&C.counter, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    double s = 0.0;
    float m = 0.0f;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
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

int inv_blocks(const GridInfo& g) { return grid_for(g.d.N, 256, 148 * 8); }

void launch_invert_step(const float* const* phi, float* const* psi, int halves, const GridInfo& g, int k, int max_iter,
                        double mean_tol, double max_tol, IterCtl* ctl, int phase, PartialBufs pb, cudaStream_t s,
                        bool stop_aware) {
  count_launch();
  Ptr2c pp{{phi[0], halves > 1 ? phi[1] : phi[0]}};
  Ptr2 ps{{psi[0], halves > 1 ? psi[1] : psi[0]}};
  InvParams P;
  Affine m = make_affine(g, g);
  for (int j = 0; j < 9; ++j) P.A[j] = m.A[j];
  for (int j = 0; j < 3; ++j) P.ih[j] = (float)(1.0 / g.sp[j]);
  P.k = k;
  P.max_iter = max_iter;
  P.phase = phase;
  P.stop_aware = stop_aware ? 1 : 0;
  P.mean_tol = mean_tol;
  P.max_tol = max_tol;
  dim3 grid(inv_blocks(g), halves);
  if (g.d.dim == 3)
    k_invert_step<3><<<grid, 256, 0, s>>>(pp, ps, g.d, P, ctl, pb.sum, pb.maxv, pb.capacity);
  else
    k_invert_step<2><<<grid, 256, 0, s>>>(pp, ps, g.d, P, ctl, pb.sum, pb.maxv, pb.capacity);
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
__global__ void __launch_bounds__(256) k_resample(Ptr4c in, Dims di, Ptr4 out, Dims dout, Affine m, int nf) {
  const long long No = dout.N, Ni = di.N, stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < No; i += stride) {
    int x, y, z;
    voxel_xyz(i, dout, x, y, z);
    float cx, cy, cz;
    map_point<DIM>(m, (float)x, (float)y, (float)z, 0.0f, 0.0f, 0.0f, cx, cy, cz);
    const bool ok = inside_buffer<DIM>(di, cx, cy, cz);
    Cell c;
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
  Affine m = make_affine(go, gi);
  int blocks = grid_for(go.d.N, 256);
  if (go.d.dim == 3)
    k_resample<3><<<blocks, 256, 0, s>>>(pi, gi.d, po, go.d, m, nfields);
  else
    k_resample<2><<<blocks, 256, 0, s>>>(pi, gi.d, po, go.d, m, nfields);
}

// ------------------------------------------------------------------------------------------
// Image pyramid: one separable pass, replicate-edge boundary, FP64 accumulation.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_conv_image_axis(const float* __restrict__ in, float* __restrict__ out, Dims d,
                                                         int axis, const double* __restrict__ coeffs, int R) {
  const long long N = d.N, stride = (long long)gridDim.x * blockDim.x;
  const int len = axis == 0 ? d.nx : (axis == 1 ? d.ny : d.nz);
  const long long astride = axis == 0 ? 1 : (axis == 1 ? d.nx : (long long)d.nx * d.ny);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    int x, y, z;
    voxel_xyz(i, d, x, y, z);
    const int pos = axis == 0 ? x : (axis == 1 ? y : z);
    const float* line = in + i - pos * astride;
    double s = 0.0;
    for (int j = 0; j <= 2 * R; ++j) {
      const int q = min(max(pos + j - R, 0), len - 1);
      s += __ldg(coeffs + j) * (double)__ldg(line + (long long)q * astride);
    }
    out[i] = (float)s;
  }
}

void launch_conv_image_axis(const float* in, float* out, const GridInfo& g, int axis, const double* coeffs, int R,
                            cudaStream_t s) {
  count_launch();
  k_conv_image_axis<<<grid_for(g.d.N, 256), 256, 0, s>>>(in, out, g.d, axis, coeffs, R);
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
