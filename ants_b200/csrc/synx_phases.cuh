// Per-voxel phases of one SyN iteration as device functions over explicit tiles, shared by the
// standalone kernels (one tile per block) and the persistent level kernel (tiles in a block-
// stride loop).  Tiles are 32 x 8 voxels in x, y; `zb` consecutive slices per thread.
#pragma once

#include <cfloat>

#include "synx_kernels.cuh"

namespace synx {

struct Ptr2c {
  const float* p[2];
};
struct Ptr2 {
  float* p[2];
};

// ---- index maps --------------------------------------------------------------------------------
// DIAG: the grids share axis directions (no rotation between them), the common case; the map is
// then one FMA pair per axis.
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

template <int DIM, bool DIAG>
__device__ __forceinline__ float sample(const float* SYNX_RESTRICT img, const Dims& di, const Affine& m, float fx,
                                        float fy, float fz, float ux, float uy, float uz) {
  float cx, cy, cz;
  map_point<DIM, DIAG>(m, fx, fy, fz, ux, uy, uz, cx, cy, cz);
  if (!inside_buffer<DIM>(di, cx, cy, cz)) return 0.0f;
  float v;
  lerp_planes<DIM, 1>(img, 0, di, cx, cy, cz, &v);
  return v;
}

// ---- warp of both images through their inverse half-fields -----------------------------------
struct WarpArgs {
  const float* F;
  const float* M;
  const float* psiF;
  const float* psiM;
  float* Ft;
  float* Mt;
  Dims dF, dM, dv;
  Affine mF, mM;
  int zb;
};

template <int DIM, bool DIAG>
__device__ __forceinline__ void warp_pair_tile(const WarpArgs& a, int bx, int by, int bz) {
  const int x = bx * 32 + (threadIdx.x & 31), y = by * 8 + (threadIdx.x >> 5);
  const Dims& dv = a.dv;
  if (x >= dv.nx || y >= dv.ny) return;
  const int z0 = bz * a.zb, z1 = min(z0 + a.zb, dv.nz);
  const int N = (int)dv.N, nxy = dv.nx * dv.ny;
  const float* SYNX_RESTRICT psiF = a.psiF;
  const float* SYNX_RESTRICT psiM = a.psiM;
  const float fx = (float)x, fy = (float)y;
  const int i0 = z0 * nxy + y * dv.nx + x;
  float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, b0 = 0.0f, b1 = 0.0f, b2 = 0.0f;
  if (z0 < z1) {
    a0 = psiF[i0];
    a1 = psiF[N + i0];
    a2 = DIM == 3 ? psiF[2 * N + i0] : 0.0f;
    b0 = psiM[i0];
    b1 = psiM[N + i0];
    b2 = DIM == 3 ? psiM[2 * N + i0] : 0.0f;
  }
  for (int z = z0; z < z1; ++z) {
    const int i = z * nxy + y * dv.nx + x;
    const float fz = (float)z;
    const float u0 = a0, u1 = a1, u2 = a2, v0 = b0, v1 = b1, v2 = b2;
    if (z + 1 < z1) {  // next slice's displacements, loaded ahead of this slice's gathers
      const int j = i + nxy;
      a0 = psiF[j];
      a1 = psiF[N + j];
      a2 = DIM == 3 ? psiF[2 * N + j] : 0.0f;
      b0 = psiM[j];
      b1 = psiM[N + j];
      b2 = DIM == 3 ? psiM[2 * N + j] : 0.0f;
    }
    a.Ft[i] = sample<DIM, DIAG>(a.F, a.dF, a.mF, fx, fy, fz, u0, u1, u2);
    a.Mt[i] = sample<DIM, DIAG>(a.M, a.dM, a.mM, fx, fy, fz, v0, v1, v2);
  }
}

// ---- composition out = w + s * d(x + w), s = eta / max||d/h|| (in place when out == w) --------
struct ComposeArgs {
  Ptr2c d, w;
  Ptr2 o;
  Dims g;
  Affine m;
  double eta;
  int zb;
};

template <int DIM, bool DIAG>
__device__ __forceinline__ void compose_tile(const ComposeArgs& a, const IterCtl* ctl, int h, int bx, int by,
                                             int bz) {
  const Dims& d = a.g;
  const int x = bx * 32 + (threadIdx.x & 31), y = by * 8 + (threadIdx.x >> 5);
  if (x >= d.nx || y >= d.ny) return;
  const float* SYNX_RESTRICT D = h ? a.d.p[1] : a.d.p[0];
  const float* W = h ? a.w.p[1] : a.w.p[0];
  float* O = h ? a.o.p[1] : a.o.p[0];
  float scale = 1.0f;
  if (a.eta > 0.0) {
    const float mx = __uint_as_float(ctl->maxnorm[h]);
    scale = mx > 0.0f ? (float)(a.eta / (double)mx) : (float)a.eta;
  }
  const int z0 = bz * a.zb, z1 = min(z0 + a.zb, d.nz);
  const int N = (int)d.N, nxy = d.nx * d.ny;
  const float fx = (float)x, fy = (float)y;
  const int i0 = z0 * nxy + y * d.nx + x;
  float n0 = 0.0f, n1 = 0.0f, n2 = 0.0f;
  if (z0 < z1) {
    n0 = W[i0];
    n1 = W[N + i0];
    n2 = DIM == 3 ? W[2 * N + i0] : 0.0f;
  }
  for (int z = z0; z < z1; ++z) {
    const int i = z * nxy + y * d.nx + x;
    const float w0 = n0, w1 = n1, w2 = n2;
    if (z + 1 < z1) {  // next slice's warp vector, loaded ahead of this slice's gathers
      n0 = W[i + nxy];
      n1 = W[N + i + nxy];
      n2 = DIM == 3 ? W[2 * N + i + nxy] : 0.0f;
    }
    float cx, cy, cz;
    map_point<DIM, DIAG>(a.m, fx, fy, (float)z, w0, w1, w2, cx, cy, cz);
    if (inside_buffer<DIM>(d, cx, cy, cz)) {
      float v[DIM];
      lerp_planes<DIM, DIM>(D, N, d, cx, cy, cz, v);
      O[i] = fmaf(scale, v[0], w0);
      O[N + i] = fmaf(scale, v[1], w1);
      if (DIM == 3) O[2 * N + i] = fmaf(scale, v[DIM - 1], w2);
    } else {
      O[i] = w0;
      O[N + i] = w1;
      if (DIM == 3) O[2 * N + i] = w2;
    }
  }
}

// ---- fixed-point inverse: one sub-iteration on one tile ----------------------------------------
struct InvArgs {
  Ptr2c phi;   // field being inverted (read-only, gathered)
  Ptr2 psi;    // iterate (updated in place at its own voxels)
  Ptr2 ecache; // residual of the current iterate per voxel (written by the statistics pass, read by
               // the next update), or null: the update then recomputes it
  Dims g;
  float A[9];
  float ih[3];
  int zb;
};

// Continuous index of voxel (fx, fy, fz) displaced by p (physical): (fx, fy, fz) + A p.
template <int DIM, bool DIAG>
__device__ __forceinline__ void inv_map(const float* A, float fx, float fy, float fz, const float p[3], float& cx,
                                        float& cy, float& cz) {
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
}

template <int DIM, bool DIAG>
__device__ __forceinline__ void inv_residual(const float* SYNX_RESTRICT phi, const Dims& d, const float* A, float fx,
                                             float fy, float fz, const float p[3], float e[3]) {
  float cx, cy, cz;
  inv_map<DIM, DIAG>(A, fx, fy, fz, p, cx, cy, cz);
  e[0] = p[0];
  e[1] = p[1];
  e[2] = DIM == 3 ? p[2] : 0.0f;
  if (inside_buffer<DIM>(d, cx, cy, cz)) {
    float v[DIM];
    lerp_planes<DIM, DIM>(phi, (int)d.N, d, cx, cy, cz, v);
    e[0] += v[0];
    e[1] += v[1];
    if (DIM == 3) e[2] += v[DIM - 1];
  }
}

// apply: psi += eps * clamp(-E, lim) (boundary voxels pinned to 0); stats: accumulate ||E/h|| of
// the (updated) iterate into acc (sum) and mx (max).  With a residual cache, the statistics pass
// stores E and the next update reads it back instead of gathering phi again: the same values,
// since E depends only on the iterate and phi, which have not changed in between.
template <int DIM, bool DIAG>
__device__ __forceinline__ void invert_tile(const InvArgs& a, int h, int bx, int by, int bz, bool apply, bool stats,
                                            float eps, float lim, double& acc, float& mx) {
  const Dims& d = a.g;
  const int x = bx * 32 + (threadIdx.x & 31), y = by * 8 + (threadIdx.x >> 5);
  if (x >= d.nx || y >= d.ny) return;
  const float* SYNX_RESTRICT phi = h ? a.phi.p[1] : a.phi.p[0];
  float* SYNX_RESTRICT psi = h ? a.psi.p[1] : a.psi.p[0];
  float* SYNX_RESTRICT ec = h ? a.ecache.p[1] : a.ecache.p[0];
  const int z0 = bz * a.zb, z1 = min(z0 + a.zb, d.nz);
  const int N = (int)d.N, nxy = d.nx * d.ny;
  const float fx = (float)x, fy = (float)y;
  const bool xyedge = x == 0 || x == d.nx - 1 || y == 0 || y == d.ny - 1;
  // the iterate of the next slice is loaded before this slice's gathers (one dependent memory
  // round trip per slice instead of two)
  const int i0 = z0 * nxy + y * d.nx + x;
  float pn[3] = {0.0f, 0.0f, 0.0f};
  if (z0 < z1) {
    pn[0] = psi[i0];
    pn[1] = psi[N + i0];
    pn[2] = DIM == 3 ? psi[2 * N + i0] : 0.0f;
  }
  for (int z = z0; z < z1; ++z) {
    const int i = z * nxy + y * d.nx + x;
    const float fz = (float)z;
    float p[3] = {pn[0], pn[1], pn[2]};
    if (z + 1 < z1) {
      pn[0] = psi[i + nxy];
      pn[1] = psi[N + i + nxy];
      pn[2] = DIM == 3 ? psi[2 * N + i + nxy] : 0.0f;
    }
    float e[3];
    if (apply) {
      if (ec != nullptr) {
        e[0] = ec[i];
        e[1] = ec[N + i];
        e[2] = DIM == 3 ? ec[2 * N + i] : 0.0f;
      } else {
        inv_residual<DIM, DIAG>(phi, d, a.A, fx, fy, fz, p, e);
      }
      float s2 = 0.0f;
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        const float v = e[c] * a.ih[c];
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
      inv_residual<DIM, DIAG>(phi, d, a.A, fx, fy, fz, p, e);
      if (ec != nullptr) {
        ec[i] = e[0];
        ec[N + i] = e[1];
        if (DIM == 3) ec[2 * N + i] = e[2];
      }
      float s2 = 0.0f;
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        const float v = e[c] * a.ih[c];
        s2 += v * v;
      }
      const float nrm = sqrtf(s2);
      acc += (double)nrm;
      mx = fmaxf(mx, nrm);
    }
  }
}

// ---- Gaussian smoothing of displacement fields ---------------------------------------------------
constexpr int kSmoothRMax = 12;

struct Smooth3Args {
  Ptr2c in, orig;
  Ptr2 out;
  float k[3][2 * kSmoothRMax + 1];  // per-axis kernels, zero-padded and centred to radius R
  int ZC, halves, epilogue, do_max;
  float w1, w2;
  float ih[3];
};

__host__ __device__ inline size_t smooth3_smem_floats(int dim, int R, int TY = 8) {
  const int HXP = (32 + 2 * R + 3) & ~3, HY = TY + 2 * R;
  return (size_t)dim * HY * HXP + (size_t)dim * HY * 32;
}

// xy smoothing of one (32 x TY tile, slice z, field h): halo tile of every component staged in
// shared memory with replicate-edge indices, convolved along x (each work item makes four
// consecutive outputs from float4 loads) and then along y (each thread makes TY/8 consecutive rows
// of one column from registers).  Taller tiles convolve fewer halo rows along x per output (TY + 2R
// rows for TY outputs).
__device__ __forceinline__ void cp_async4(float* smem, const float* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int NPENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(NPENDING) : "memory");
}

// How a halo tile reaches shared memory: a loop of plain loads and stores (few registers: the
// persistent level kernel), all of a warp's rows of a component loaded into registers before they
// are stored (the loads in flight together: the standalone xy kernel), or cp.async copies that the
// caller commits and waits for.
enum class TileLoad { Loop, Batched, Async };

// Halo tile of one (32 x TY tile, slice z, field h) into shared memory (replicate-edge indices).
template <int DIM, int R, int TY, TileLoad LOAD>
__device__ __forceinline__ void smooth_xy_load_tile(const Smooth3Args& a, const Dims& d, int bx, int by, int z, int h,
                                                    float* tile) {
  constexpr int HX = 32 + 2 * R, HXP = (HX + 3) & ~3, HY = TY + 2 * R;
  static_assert(HX <= 64, "two columns per lane cover a halo row");
  const int nx = d.nx, ny = d.ny, nxy = nx * ny, N = (int)d.N;
  const float* SYNX_RESTRICT src = h ? a.in.p[1] : a.in.p[0];
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int x0 = bx * 32, y0 = by * TY;
  // the halo columns this lane copies (replicate-edge indices) are the same in every row
  const int gx0 = min(max(x0 - R + tx, 0), nx - 1);
  const int gx1 = min(max(x0 - R + 32 + tx, 0), nx - 1);
  const bool second = tx < HX - 32;
  constexpr int RPW = (HY + 7) / 8;  // halo rows per warp and component
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    const float* cplane = src + c * N + z * nxy;
    float* ctile = tile + c * HY * HXP;
    if (LOAD != TileLoad::Batched) {
      for (int hy = ty; hy < HY; hy += 8) {
        const float* line = cplane + min(max(y0 - R + hy, 0), ny - 1) * nx;
        float* trow = ctile + hy * HXP;
        if (LOAD == TileLoad::Async) {
          cp_async4(trow + tx, line + gx0);
          if (second) cp_async4(trow + 32 + tx, line + gx1);
        } else {
          trow[tx] = SYNX_LDG(line + gx0);
          if (second) trow[32 + tx] = SYNX_LDG(line + gx1);
        }
      }
    } else {
      float v0[RPW], v1[RPW];
#pragma unroll
      for (int k = 0; k < RPW; ++k) {
        const int hy = ty + 8 * k;
        if (hy < HY) {
          const float* line = cplane + min(max(y0 - R + hy, 0), ny - 1) * nx;
          v0[k] = SYNX_LDG(line + gx0);
          v1[k] = second ? SYNX_LDG(line + gx1) : 0.0f;
        }
      }
#pragma unroll
      for (int k = 0; k < RPW; ++k) {
        const int hy = ty + 8 * k;
        if (hy < HY) {
          float* trow = ctile + hy * HXP;
          trow[tx] = v0[k];
          if (second) trow[32 + tx] = v1[k];
        }
      }
    }
  }
}

// x and y convolution of a loaded halo tile: thread (tx, ty) gets the outputs at x = bx*32 + tx,
// y = by*TY + ty*(TY/8) + r in y[c][r].  All threads of the block call it; it ends with the
// tile read and xsum free again.
template <int DIM, int R, int TY>
__device__ __forceinline__ void smooth_xy_convolve(const Smooth3Args& a, const float* tile, float* xsum,
                                                   float (&y)[DIM][TY / 8]) {
  static_assert(TY % 8 == 0, "8 warps share the tile rows");
  constexpr int K = 2 * R + 1, RPT = TY / 8;
  constexpr int HX = 32 + 2 * R, HXP = (HX + 3) & ~3, HY = TY + 2 * R;
  constexpr int NQ = (2 * R + 3) / 4 + 1;  // float4 loads covering 4 + 2R taps
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
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
  const int ty0 = ty * RPT;
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    const float* col = xsum + (c * HY + ty0) * 32 + tx;
    float w[RPT + 2 * R];
#pragma unroll
    for (int j = 0; j < RPT + 2 * R; ++j) w[j] = col[j * 32];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      float acc = 0.0f;
#pragma unroll
      for (int j = 0; j < K; ++j) acc = fmaf(a.k[1][j], w[r + j], acc);
      y[c][r] = acc;
    }
  }
  __syncthreads();  // the tile and xsum may be reused by the caller's next tile
}

template <int DIM, int R, int TY, TileLoad LOAD = TileLoad::Loop>
__device__ __forceinline__ void smooth_xy_compute(const Smooth3Args& a, const Dims& d, int bx, int by, int z, int h,
                                                  float* sm, float (&y)[DIM][TY / 8]) {
  static_assert(LOAD != TileLoad::Async, "the caller waits for cp.async copies");
  constexpr int HX = 32 + 2 * R, HXP = (HX + 3) & ~3, HY = TY + 2 * R;
  float* tile = sm;                     // [DIM][HY][HXP]
  float* xsum = tile + DIM * HY * HXP;  // [DIM][HY][32]
  smooth_xy_load_tile<DIM, R, TY, LOAD>(a, d, bx, by, z, h, tile);
  __syncthreads();
  smooth_xy_convolve<DIM, R, TY>(a, tile, xsum, y);
}

// xy part for one (32 x TY tile, slice z, field h), written out: in 3-D the xy-smoothed values go
// to `out` for the z part; in 2-D this is the whole filter and the SyN epilogue runs here (max norm
// returned).  All threads of the block must call it; `sm` holds smooth3_smem_floats(DIM, R, TY)
// floats.
template <int DIM, int R, int TY = 8, TileLoad LOAD = TileLoad::Loop>
__device__ __forceinline__ float smooth_xy_tile(const Smooth3Args& a, const Dims& d, int bx, int by, int z, int h,
                                                float* sm) {
  constexpr int RPT = TY / 8;
  float y[DIM][RPT];
  smooth_xy_compute<DIM, R, TY, LOAD>(a, d, bx, by, z, h, sm, y);
  const int nx = d.nx, ny = d.ny, nxy = nx * ny, N = (int)d.N;
  float* SYNX_RESTRICT dst = h ? a.out.p[1] : a.out.p[0];
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const int x0 = bx * 32, y0 = by * TY;
  const int ox = x0 + tx, ty0 = ty * RPT;
  float mx = 0.0f;
  if (ox >= nx) return mx;
  const float* SYNX_RESTRICT org = h ? a.orig.p[1] : a.orig.p[0];
#pragma unroll
  for (int r = 0; r < RPT; ++r) {
    const int oy = y0 + ty0 + r;
    if (oy >= ny) break;
    const int i = z * nxy + oy * nx + ox;
    if (DIM == 3) {
#pragma unroll
      for (int c = 0; c < DIM; ++c) dst[c * N + i] = y[c][r];
      continue;
    }
    const bool edge = a.epilogue && (ox == 0 || ox == nx - 1 || oy == 0 || oy == ny - 1);
    float nrm2 = 0.0f;
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      float v = y[c][r];
      if (a.epilogue) {
        if (edge) v = 0.0f;
        else if (a.w2 != 0.0f) v = v * a.w1 + org[c * N + i] * a.w2;
      }
      const float q = v * a.ih[c];
      nrm2 += q * q;
      dst[c * N + i] = v;
    }
    mx = fmaxf(mx, sqrtf(nrm2));
  }
  return mx;
}

// z part (3-D) for one (x, y) column of field h over slices [zc*ZC, zc*ZC + ZC): the last 2R+1
// xy-smoothed values per component sit in registers, the z loop is unrolled by 2R+1 so every
// ring index is a compile-time constant; applies the SyN epilogue; returns the max norm.
template <int R>
__device__ __forceinline__ float smooth_z_column(const Smooth3Args& a, const Dims& d, int bx, int by, int zc, int h) {
  constexpr int K = 2 * R + 1, RD = K;
  const int nx = d.nx, ny = d.ny, nz = d.nz, nxy = nx * ny, N = (int)d.N;
  const float* SYNX_RESTRICT src = h ? a.in.p[1] : a.in.p[0];
  float* SYNX_RESTRICT dst = h ? a.out.p[1] : a.out.p[0];
  const float* SYNX_RESTRICT org = h ? a.orig.p[1] : a.orig.p[0];
  const int ox = bx * 32 + (threadIdx.x & 31), oy = by * 8 + (threadIdx.x >> 5);
  const int z0 = zc * a.ZC, z1 = min(z0 + a.ZC, nz);
  float mx = 0.0f;
  if (ox >= nx || oy >= ny) return mx;
  const float* col = src + oy * nx + ox;
  float ring[3][RD];
#pragma unroll
  for (int u = 0; u < 2 * R; ++u) {
    const int zs = min(max(z0 - R + u, 0), nz - 1);
#pragma unroll
    for (int c = 0; c < 3; ++c) ring[c][u] = SYNX_LDG(col + c * N + zs * nxy);
  }
  const bool xyedge = ox == 0 || ox == nx - 1 || oy == 0 || oy == ny - 1;
  for (int zb = z0; zb < z1; zb += RD) {
#pragma unroll
    for (int u = 0; u < RD; ++u) {
      const int z = zb + u;
      if (z < z1) {
        const int zs = min(z + R, nz - 1);
#pragma unroll
        for (int c = 0; c < 3; ++c) ring[c][(u + 2 * R) % RD] = SYNX_LDG(col + c * N + zs * nxy);
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
  return mx;
}

// Threads of a block of the standalone z smoothing kernel.
constexpr int kSmoothZThreads = 256;

// The same z part with the ring in shared memory (`ring` holds (2R+1) x 3 x kSmoothZThreads floats,
// slot-major, thread-minor: each thread touches only its own column, so no barrier is needed and the
// accesses are conflict-free).  Far fewer registers than the register ring, so more blocks fit on
// an SM; the arithmetic and its order are the same, so the results have the same bits.
template <int R>
__device__ __forceinline__ float smooth_z_column_smem(const Smooth3Args& a, const Dims& d, int bx, int by, int zc,
                                                      int h, float* ring) {
  constexpr int K = 2 * R + 1, RD = K;
  const int nx = d.nx, ny = d.ny, nz = d.nz, nxy = nx * ny, N = (int)d.N;
  const float* SYNX_RESTRICT src = h ? a.in.p[1] : a.in.p[0];
  float* SYNX_RESTRICT dst = h ? a.out.p[1] : a.out.p[0];
  const float* SYNX_RESTRICT org = h ? a.orig.p[1] : a.orig.p[0];
  const int ox = bx * 32 + (threadIdx.x & 31), oy = by * 8 + (threadIdx.x >> 5);
  const int z0 = zc * a.ZC, z1 = min(z0 + a.ZC, nz);
  float mx = 0.0f;
  if (ox >= nx || oy >= ny) return mx;
  // a compile-time row length (the kernel's block), so every slot's offset is an immediate
  constexpr int T = kSmoothZThreads;
  float* rt = ring + threadIdx.x;
  auto slot = [&](int s, int c) -> float& { return rt[(s * 3 + c) * T]; };
  const float* col = src + oy * nx + ox;
#pragma unroll
  for (int u = 0; u < 2 * R; ++u) {
    const int zs = min(max(z0 - R + u, 0), nz - 1);
#pragma unroll
    for (int c = 0; c < 3; ++c) slot(u, c) = SYNX_LDG(col + c * N + zs * nxy);
  }
  const bool xyedge = ox == 0 || ox == nx - 1 || oy == 0 || oy == ny - 1;
  // the slices entering the window are loaded two outputs ahead (q0: slice z + R, q1: z + R + 1),
  // so each load's latency overlaps two outputs' convolutions
  float q0[3], q1[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    q0[c] = z0 < z1 ? SYNX_LDG(col + c * N + min(z0 + R, nz - 1) * nxy) : 0.0f;
    q1[c] = z0 + 1 < z1 ? SYNX_LDG(col + c * N + min(z0 + 1 + R, nz - 1) * nxy) : 0.0f;
  }
  for (int zb = z0; zb < z1; zb += RD) {
#pragma unroll
    for (int u = 0; u < RD; ++u) {
      const int z = zb + u;
      if (z < z1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          slot((u + 2 * R) % RD, c) = q0[c];
          q0[c] = q1[c];
          if (z + 2 < z1) q1[c] = SYNX_LDG(col + c * N + min(z + 2 + R, nz - 1) * nxy);
        }
        const int i = z * nxy + oy * nx + ox;
        const bool edge = a.epilogue && (xyedge || z == 0 || z == nz - 1);
        float nrm2 = 0.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float acc = 0.0f;
#pragma unroll
          for (int j = 0; j < K; ++j) acc = fmaf(a.k[2][j], slot((u + j) % RD, c), acc);
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
  return mx;
}

// ---- convergence monitor and per-iteration log (one warp) ------------------------------------------
// The last `window` energies, each divided by the running sum of |energy| of the level, are
// fitted with a single-span linear B-spline on [0,1] by one level of multilevel B-spline
// approximation; the convergence value is minus the fitted slope.
// Called by all 32 lanes of one warp: lane j takes window entries j, j + 32, ... (the newest value
// comes from ctl->metric, the older ones from the ring), the four sums are reduced across the
// warp in a fixed order, and lane 0 updates the ring, the log and the stop flag.
__device__ __forceinline__ void converge_step(IterCtl* ctl, const LogDev& log, double threshold, int window) {
  const int lane = threadIdx.x & 31;
  const int k = ctl->iter;
  const double v = ctl->metric;
  const double tabs = ctl->total_abs + fabs(v);
  const int W = window < 2 ? 2 : (window > kMaxWindow ? kMaxWindow : window);
  const int k1 = k + 1;
  const bool full = k1 >= W;
  double num0 = 0, den0 = 0, num1 = 0, den1 = 0;
  if (full) {
    for (int j = lane; j < W; j += 32) {
      const int slot = (k1 - W + j) % W;
      const double e = slot == k % W ? v : ctl->energies[slot];
      const double u = (double)j / (double)(W - 1);
      const double z = e / tabs;
      const double w0 = 1.0 - u, w1 = u, ws = w0 * w0 + w1 * w1;
      num0 += w0 * w0 * (w0 * z / ws);
      den0 += w0 * w0;
      num1 += w1 * w1 * (w1 * z / ws);
      den1 += w1 * w1;
    }
    num0 = warp_sum_d(num0);
    den0 = warp_sum_d(den0);
    num1 = warp_sum_d(num1);
    den1 = warp_sum_d(den1);
  }
  __syncwarp();
  if (lane != 0) return;
  ctl->total_abs = tabs;
  ctl->energies[k % W] = v;
  double conv = DBL_MAX;
  if (full) {
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

}  // namespace synx
