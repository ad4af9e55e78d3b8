// Device-side building blocks shared by the synx kernels: grid descriptors, ITK's linear
// interpolation buffer rule, deterministic block reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// Loads in the device functions that the per-kernel launches and the persistent level kernel share.
// A per-kernel launch only reads data that earlier launches wrote, so the read-only (non-coherent)
// path and restrict-qualified pointers apply.  The level kernel reads, after a grid barrier, data that
// other blocks wrote earlier in the same launch, which the read-only path may serve stale: its
// translation unit defines SYNX_COHERENT_LOADS, so these are plain (coherent) global loads there and
// no pointer is restrict-qualified (which would let the compiler choose the read-only path itself).
#ifdef SYNX_COHERENT_LOADS
#define SYNX_LDG(p) (*(p))
#define SYNX_RESTRICT
#else
#define SYNX_LDG(p) __ldg(p)
#define SYNX_RESTRICT __restrict__
#endif

namespace synx {

// Voxel counts of one grid.  nz = 1 for 2-D.
struct Dims {
  int nx, ny, nz;
  int dim;
  long long N;
};

// Continuous index into a target grid of a source-grid voxel i displaced by u (physical):
// c = t + B * i + A * u.  For a single grid (composition, inversion) t = 0, B = I and
// A = inverse(direction * diag(spacing)).
struct Affine {
  float t[3];
  float B[9];
  float A[9];
};

// ITK ImageFunction::IsInsideBuffer: start-0.5 <= c < end+0.5 per axis (NaN is outside).
template <int DIM>
__device__ __forceinline__ bool inside_buffer(const Dims& d, float cx, float cy, float cz) {
  bool ok = (cx >= -0.5f) && (cx < (float)d.nx - 0.5f) && (cy >= -0.5f) && (cy < (float)d.ny - 0.5f);
  if (DIM == 3) ok = ok && (cz >= -0.5f) && (cz < (float)d.nz - 0.5f);
  return ok;
}

// Clamp-to-edge cell of ITK's (Vector)LinearInterpolateImageFunction for c inside the buffer.
__device__ __forceinline__ void axis_cell(float c, int n, int& i0, int& i1, float& w) {
  float f = floorf(c);
  int b = (int)f;
  w = c - f;
  if (b < 0) {
    b = 0;
    w = 0.0f;
  }
  int u = b + 1;
  if (u > n - 1) {
    u = n - 1;
    w = 0.0f;
  }
  i0 = b;
  i1 = u;
}

// Grids hold fewer than 2^31 values per component plane (checked on the host), so cell
// offsets are 32-bit.
struct Cell {
  int o000, dx, dy, dz;  // base offset and the per-axis offset to the upper neighbour
  float wx, wy, wz;
};

template <int DIM>
__device__ __forceinline__ Cell make_cell(const Dims& d, float cx, float cy, float cz) {
  Cell c;
  int x0, x1, y0, y1, z0 = 0, z1 = 0;
  axis_cell(cx, d.nx, x0, x1, c.wx);
  axis_cell(cy, d.ny, y0, y1, c.wy);
  c.wz = 0.0f;
  if (DIM == 3) axis_cell(cz, d.nz, z0, z1, c.wz);
  const int sy = d.nx, sz = d.nx * d.ny;
  c.o000 = z0 * sz + y0 * sy + x0;
  c.dx = x1 - x0;
  c.dy = (y1 - y0) * sy;
  c.dz = (z1 - z0) * sz;
  return c;
}

// Multilinear interpolation in the lerp form a + (b - a) w, x then y then z.
template <int DIM>
__device__ __forceinline__ float lerp_at(const float* SYNX_RESTRICT a, const Cell& c) {
  const float* p = a + c.o000;
  float v00 = SYNX_LDG(p), v10 = SYNX_LDG(p + c.dx);
  float v01 = SYNX_LDG(p + c.dy), v11 = SYNX_LDG(p + c.dy + c.dx);
  float a0 = fmaf(v10 - v00, c.wx, v00);
  float a1 = fmaf(v11 - v01, c.wx, v01);
  float b0 = fmaf(a1 - a0, c.wy, a0);
  if (DIM == 2) return b0;
  const float* q = p + c.dz;
  float u00 = SYNX_LDG(q), u10 = SYNX_LDG(q + c.dx);
  float u01 = SYNX_LDG(q + c.dy), u11 = SYNX_LDG(q + c.dy + c.dx);
  float c0 = fmaf(u10 - u00, c.wx, u00);
  float c1 = fmaf(u11 - u01, c.wx, u01);
  float b1 = fmaf(c1 - c0, c.wy, c0);
  return fmaf(b1 - b0, c.wz, b0);
}

// Cell of a point whose every axis has both neighbours inside the grid (0 <= floor(c) < n - 1), so
// that no clamp applies: the upper neighbours sit at +1, +nx and +nx*ny, the weights are c - floor(c).
// Returns false for a point that needs the clamp-to-edge cell (make_cell); the offset and weights it
// computes are then not meant to be used.  Where it returns true, the corners and weights are exactly
// make_cell's, so lerp_interior gives lerp_at's value bit for bit.
template <int DIM>
__device__ __forceinline__ bool interior_cell(const Dims& d, float cx, float cy, float cz, int& o, float& wx,
                                              float& wy, float& wz) {
  const float fx = floorf(cx), fy = floorf(cy), fz = DIM == 3 ? floorf(cz) : 0.0f;
  const int bx = (int)fx, by = (int)fy, bz = (int)fz;
  wx = cx - fx;
  wy = cy - fy;
  wz = DIM == 3 ? cz - fz : 0.0f;
  o = (bz * d.ny + by) * d.nx + bx;
  bool in = (unsigned)bx < (unsigned)(d.nx - 1) && (unsigned)by < (unsigned)(d.ny - 1);
  if (DIM == 3) in = in && (unsigned)bz < (unsigned)(d.nz - 1);
  return in;
}

// lerp_at for an interior cell: p = plane + offset of the lower corner; sy = nx, sz = nx * ny.
template <int DIM>
__device__ __forceinline__ float lerp_interior(const float* SYNX_RESTRICT p, int sy, int sz, float wx, float wy,
                                               float wz) {
  const float* py = p + sy;
  float v00 = SYNX_LDG(p), v10 = SYNX_LDG(p + 1);
  float v01 = SYNX_LDG(py), v11 = SYNX_LDG(py + 1);
  float a0 = fmaf(v10 - v00, wx, v00);
  float a1 = fmaf(v11 - v01, wx, v01);
  float b0 = fmaf(a1 - a0, wy, a0);
  if (DIM == 2) return b0;
  const float* q = p + sz;
  const float* qy = q + sy;
  float u00 = SYNX_LDG(q), u10 = SYNX_LDG(q + 1);
  float u01 = SYNX_LDG(qy), u11 = SYNX_LDG(qy + 1);
  float c0 = fmaf(u10 - u00, wx, u00);
  float c1 = fmaf(u11 - u01, wx, u01);
  float b1 = fmaf(c1 - c0, wy, c0);
  return fmaf(b1 - b0, wz, b0);
}

// Multilinear interpolation of NC planes (plane c at a + c * N) at one point inside the buffer.  A
// warp whose active lanes all have interior cells takes the interior cell's short form; otherwise
// every lane takes the clamp-to-edge cell, so lanes near the edges do not split the warp into both
// forms (on small grids most warps have such a lane).  Either form gives the same value.
template <int DIM, int NC>
__device__ __forceinline__ void lerp_planes(const float* SYNX_RESTRICT a, int N, const Dims& d, float cx, float cy,
                                            float cz, float out[NC]) {
  int o;
  float wx, wy, wz;
  const bool in = interior_cell<DIM>(d, cx, cy, cz, o, wx, wy, wz);
  if (__all_sync(__activemask(), in)) {
    const int sy = d.nx, sz = d.nx * d.ny;
#pragma unroll
    for (int c = 0; c < NC; ++c) out[c] = lerp_interior<DIM>(a + c * N + o, sy, sz, wx, wy, wz);
  } else {
    const Cell cl = make_cell<DIM>(d, cx, cy, cz);
#pragma unroll
    for (int c = 0; c < NC; ++c) out[c] = lerp_at<DIM>(a + c * N, cl);
  }
}

// This block's tile coordinates, in reverse order of the grid when `rev` (block 0 takes the last
// tile).  Blocks start roughly in index order, so a kernel walking the grid backwards begins on the
// tiles that the kernel before it (walking forwards) wrote last, while they are still in L2.
__device__ __forceinline__ uint3 sweep_block(int rev) {
  uint3 b = blockIdx;
  if (rev) {
    b.x = gridDim.x - 1 - b.x;
    b.y = gridDim.y - 1 - b.y;
    b.z = gridDim.z - 1 - b.z;
  }
  return b;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Fixed-order block sum (valid in thread 0).  blockDim.x must be a multiple of 32, <= 1024.
__device__ __forceinline__ double block_sum_d(double v, double* sh /* >= 32 */) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum_d(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = lane < nw ? sh[lane] : 0.0;
    r = warp_sum_d(r);
  }
  return r;
}
__device__ __forceinline__ float block_max_f(float v, float* sh /* >= 32 */) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_max_f(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  float r = 0.0f;
  if (w == 0) {
    r = lane < nw ? sh[lane] : 0.0f;
    r = warp_max_f(r);
  }
  return r;
}

// Sum of a double and max of a float over the block in one pass; the results are valid in
// thread 0 (warp 0).
__device__ __forceinline__ void block_sum_max(double& s, float& m, double* shd, float* shf) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  s = warp_sum_d(s);
  m = warp_max_f(m);
  __syncthreads();
  if (lane == 0) {
    shd[w] = s;
    shf[w] = m;
  }
  __syncthreads();
  if (w == 0) {
    s = lane < nw ? shd[lane] : 0.0;
    m = lane < nw ? shf[lane] : 0.0f;
    s = warp_sum_d(s);
    m = warp_max_f(m);
  }
}

// Non-negative floats order like their bit patterns: atomicMax on the bits is a float max.
__device__ __forceinline__ void atomic_max_nonneg(unsigned int* addr, float v) {
  atomicMax(addr, __float_as_uint(fmaxf(v, 0.0f)));
}

}  // namespace synx
