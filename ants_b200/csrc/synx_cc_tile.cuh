// Neighbourhood cross-correlation tile (value and both SyN update directions), shared by the
// CC kernel and the persistent level kernel.
#include <cfloat>
#include <cmath>

#pragma once

#include "synx_kernels.cuh"

namespace synx {

// ------------------------------------------------------------------------------------------
// Neighbourhood cross-correlation: value and both update directions.
//
// A block owns a 32 x 8 tile of output columns and marches along z over a chunk of ZC
// slices.  Each thread keeps FP64 running z-window sums of F, M, F^2, M^2, FM for up to CPT
// halo columns; the raw (F, M) values of the last 2R+1 slices sit in a shared-memory ring so
// the leaving slice is subtracted without a second global read.  Per slice the column sums
// are box-summed along y and then x in shared memory (FP64) with sliding windows: along y one
// thread per (quantity, halo column) walking down the 8 output rows, along x one thread per
// (quantity, output row, 8-output segment); the x pass reads and writes rows of an odd pitch,
// so the threads of a half-warp, which differ in row, hit distinct banks.  (y first: the x pass
// then runs over the 8 output rows only, not the 8 + 2R halo rows.  Each task's first window is
// summed pairwise and each slide adds the difference of the entering and leaving values, so a
// task's chain of dependent additions is ceil(log2(2R+1)) + 7 long.)  This gives the five
// window sums of each output voxel, from which the CC terms and derivatives follow.  The
// in-bounds count is separable (cx*cy*cz) and computed analytically.
//
// T is the type of the window sums and of the variance terms formed from them: double (the
// default; the sums of F^2 and M^2 cancel badly in float when the window is nearly flat) or
// float (the precision study's variant).  The tile's sum of cc is accumulated in double either
// way.
// ------------------------------------------------------------------------------------------
struct CCParams {
  float h[3];      // spacing
  float dir[9];    // direction cosines
  int identity_dir;
  double eps;
  int ZC;          // z-chunk per block
  const unsigned char* valid;  // metric masks: nonzero = valid voxel (MASKED tiles only)
  // 1/n for n = 0..kCCRcpMax, each the correctly rounded double (the window's voxel count n is an
  // integer, so a table lookup replaces the reciprocal sequence; entry 0 is unused)
  const double* rcp;
};

constexpr int kCCRcpMax = 15 * 15 * 15;  // the largest window, radius 7 in 3-D

__device__ __forceinline__ int pmod(int a, int m) {
  int r = a % m;
  return r < 0 ? r + m : r;
}

__device__ __forceinline__ float grad1(float vm, float v0, float vp, int pos, int n, float h) {
  if (n < 2 || pos == n - 1) return 0.0f;
  if (pos == 0) return 0.5f * (vp - v0) / h;
  return (vp - vm) / (2.0f * h);
}

// With metric masks (MASKED) a sixth quantity, the count of valid voxels, is box-summed beside the
// five sums, and a byte ring holds the validity of the ring's slices.
template <int R, int DIM, typename T = double, bool MASKED = false, int NT = 256>
struct CCShape {
  static constexpr int TX = 32, TY = 8;
  static constexpr int HX = TX + 2 * R, HY = TY + 2 * R, HC = HX * HY;
  static constexpr int RZ = DIM == 3 ? R : 0;
  static constexpr int RD = 2 * RZ + 1;
  static constexpr int CPT = (HC + NT - 1) / NT;  // halo columns per thread
  static_assert(NT % 32 == 0 && NT >= TX * TY, "a thread per output voxel");
  static constexpr int NQ = MASKED ? 6 : 5;
  static constexpr int CSP = HX | 1;   // row pitch of the column sums and of the y box sums (odd)
  static constexpr int XSP = TX + 1;   // row pitch of the window sums (odd)
  static constexpr int XSEG = 8;       // outputs per x-pass task
  static_assert(TX % XSEG == 0, "x segments tile the output row");
  static constexpr bool EXACT = CPT * NT == HC;  // every thread owns exactly CPT halo columns
  static constexpr size_t smem = (size_t)RD * HC * sizeof(float2) + (size_t)NQ * HY * CSP * sizeof(T) +
                                 (size_t)NQ * TY * CSP * sizeof(T) + (size_t)NQ * TY * XSP * sizeof(T) +
                                 (MASKED ? (size_t)RD * HC : 0);
  // The next slice's column update writes the column sums and ring slot (z + 1 + R) mod (2R + 1)
  // while slower warps may still be in this slice's epilogue, which reads the window sums (their
  // own array) and ring slots z - 1, z, z + 1.  Those slots differ from the written one unless
  // R = 1, so only then does a slice end with a barrier.
  static constexpr bool END_BARRIER = DIM == 3 && R < 2;
};

template <typename T>
__device__ __forceinline__ T rcp_rn(T x);
template <>
__device__ __forceinline__ double rcp_rn<double>(double x) {
  return __drcp_rn(x);
}
template <>
__device__ __forceinline__ float rcp_rn<float>(float x) {
  return __frcp_rn(x);
}

// One sliding pass of a task: dst[y * dstride] = sum of src[(y + j) * stride], j = 0..2R, for
// y = 0..NOUT-1.  The first window is summed pairwise (a tree of depth ceil(log2(2R+1)), not a
// chain of 2R+1 dependent additions) and each slide adds (entering - leaving), one dependent
// addition per output.  The 2R + NOUT inputs are loaded once into registers (the slides reuse the
// window's values instead of reloading them past the stores).
template <int R, int NOUT, typename T>
__device__ __forceinline__ void slide_sums(const T* src, int stride, T* dst, int dstride) {
  constexpr int K = 2 * R + 1, L = K + NOUT - 1;
  T v[L];
#pragma unroll
  for (int j = 0; j < L; ++j) v[j] = src[j * stride];
  T w[K];
#pragma unroll
  for (int j = 0; j < K; ++j) w[j] = v[j];
#pragma unroll
  for (int m = 1; m < K; m *= 2)
#pragma unroll
    for (int j = 0; j + m < K; j += 2 * m) w[j] += w[j + m];
  T s = w[0];
  dst[0] = s;
#pragma unroll
  for (int y = 1; y < NOUT; ++y) {
    s += v[y + 2 * R] - v[y - 1];
    dst[y * dstride] = s;
  }
}

// One CC tile: output columns x in [32 bx, 32 bx + 32), y in [8 by, 8 by + 8), z chunk bz.
// Returns the tile's sum of local cc (valid in thread 0).  All NT threads of the block must call
// it; `smem_raw` holds CCShape<R, DIM, T, MASKED>::smem bytes and `red` 32 doubles.
template <int R, int DIM, typename T = double, bool MASKED = false, int NT = 256>
__device__ __forceinline__ double cc_tile(const float* SYNX_RESTRICT Ft, const float* SYNX_RESTRICT Mt, const Dims& d,
                                          const CCParams& P, float* SYNX_RESTRICT gF, float* SYNX_RESTRICT gM,
                                          float* SYNX_RESTRICT cc_out, int bx, int by, int bz,
                                          unsigned char* smem_raw, double* red, double* valid_count = nullptr) {
  using S = CCShape<R, DIM, T, MASKED, NT>;
  constexpr int TX = S::TX, HX = S::HX, HY = S::HY, HC = S::HC, RZ = S::RZ, RD = S::RD, CPT = S::CPT;
  constexpr int CSP = S::CSP, XSP = S::XSP, TY = S::TY, NQ = S::NQ;
  float2* ring = reinterpret_cast<float2*>(smem_raw);
  T* cs = reinterpret_cast<T*>(ring + RD * HC);  // [NQ][HY][CSP] column sums
  T* ys = cs + NQ * HY * CSP;                     // [NQ][TY][CSP] y box sums of the halo columns
  T* ws = ys + NQ * TY * CSP;                     // [NQ][TY][XSP] window sums of the output voxels
  unsigned char* vring = reinterpret_cast<unsigned char*>(ws + NQ * TY * XSP);  // [RD][HC] (MASKED)
  const unsigned char* SYNX_RESTRICT valid = P.valid;

  const int tid = threadIdx.x;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const int nxy = nx * ny, N = (int)d.N;  // 32-bit offsets: the host keeps 3 N below 2^31
  const int x0 = bx * TX, y0 = by * S::TY;
  const int z0 = bz * P.ZC;
  const int z1 = min(z0 + P.ZC, nz);

  // owned halo columns
  int gofs[CPT], sofs[CPT];
  bool gval[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    int col = tid + c * NT;
    int hx = col % HX, hy = col / HX;
    int gx = x0 - R + hx, gy = y0 - R + hy;
    gval[c] = (S::EXACT || col < HC) && gx >= 0 && gx < nx && gy >= 0 && gy < ny;
    gofs[c] = gval[c] ? gy * nx + gx : 0;
    sofs[c] = hy * CSP + hx;
  }
  // sliding-window tasks: x pass (quantity, half, halo row), y pass (quantity, output column)
  T acc[CPT][NQ];
#pragma unroll
  for (int c = 0; c < CPT; ++c)
#pragma unroll
    for (int q = 0; q < NQ; ++q) acc[c][q] = T(0);

  // warm-up: slices z0-RZ .. z0+RZ-1
  for (int zs = z0 - RZ; zs < z0 + RZ; ++zs) {
    const bool zin = zs >= 0 && zs < nz;
    const int slot = pmod(zs, RD);
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      int col = tid + c * NT;
      if (S::EXACT || col < HC) {
        float2 v = make_float2(0.0f, 0.0f);
        unsigned char vb = 0;
        if (zin && gval[c]) {
          const int o = zs * nxy + gofs[c];
          v.x = SYNX_LDG(Ft + o);
          v.y = SYNX_LDG(Mt + o);
          vb = MASKED ? SYNX_LDG(valid + o) : 1;
          if (vb) {
            const T f = v.x, m = v.y;
            acc[c][0] += f;
            acc[c][1] += m;
            acc[c][2] += f * f;
            acc[c][3] += m * m;
            acc[c][4] += f * m;
            if (MASKED) acc[c][NQ - 1] += T(1);
          }
        }
        ring[slot * HC + col] = v;
        if (MASKED) vring[slot * HC + col] = vb;
      }
    }
  }

  double cc_acc = 0.0, n_valid = 0.0;
  const int tx = tid & 31, ty = tid >> 5;
  const int ox = x0 + tx, oy = y0 + ty;
  const bool out_ok = ty < TY && ox < nx && oy < ny;  // threads past the 32 x 8 outputs only sum
  const T cxn = (T)(min(ox + R, nx - 1) - max(ox - R, 0) + 1);
  const T cyn = (T)(min(oy + R, ny - 1) - max(oy - R, 0) + 1);

  // the (F, M) values of the slice entering the z window are loaded one slice ahead, so the
  // loads overlap the previous slice's box sums and CC terms
  float2 nv[CPT];
  unsigned char nvb[CPT];
#pragma unroll
  for (int c = 0; c < CPT; ++c) {
    nv[c] = make_float2(0.0f, 0.0f);
    nvb[c] = 0;
    if (z0 < z1 && z0 + RZ < nz && gval[c]) {
      const int o = (z0 + RZ) * nxy + gofs[c];
      nv[c] = make_float2(SYNX_LDG(Ft + o), SYNX_LDG(Mt + o));
      if (MASKED) nvb[c] = SYNX_LDG(valid + o);
    }
  }
  // ring slots of slices zc (sc), zc - 1 (sm), zc + 1 (sp) and zc + RZ (slot), advanced per slice
  int sc = pmod(z0, RD);
  const int pofs = oy * nx + ox;
  for (int zc = z0; zc < z1; ++zc) {
    const int sp = sc + 1 == RD ? 0 : sc + 1, sm = sc == 0 ? RD - 1 : sc - 1;
    const int slot = sc + RZ >= RD ? sc + RZ - RD : sc + RZ;
    // slide the z window: subtract slice zc-RZ-1 (if it was added), add slice zc+RZ
    const int ze = zc + RZ, zl = zc - RZ - 1;
    const bool sub = zc > z0 && zl >= 0;
    const bool zin = ze < nz;
    const bool znext = zc + 1 < z1 && ze + 1 < nz;
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      int col = tid + c * NT;
      if (S::EXACT || col < HC) {
        if (sub && gval[c] && (!MASKED || vring[slot * HC + col])) {
          float2 o = ring[slot * HC + col];
          const T f = o.x, m = o.y;
          acc[c][0] -= f;
          acc[c][1] -= m;
          acc[c][2] -= f * f;
          acc[c][3] -= m * m;
          acc[c][4] -= f * m;
          if (MASKED) acc[c][NQ - 1] -= T(1);
        }
        const float2 v = nv[c];  // zero outside the volume
        const unsigned char vb = MASKED ? nvb[c] : 1;
        if (zin && gval[c] && vb) {
          const T f = v.x, m = v.y;
          acc[c][0] += f;
          acc[c][1] += m;
          acc[c][2] += f * f;
          acc[c][3] += m * m;
          acc[c][4] += f * m;
          if (MASKED) acc[c][NQ - 1] += T(1);
        }
        ring[slot * HC + col] = v;
        if (MASKED) vring[slot * HC + col] = (zin && gval[c]) ? vb : 0;
#pragma unroll
        for (int q = 0; q < NQ; ++q) cs[q * HY * CSP + sofs[c]] = acc[c][q];
        nv[c] = make_float2(0.0f, 0.0f);
        if (MASKED) nvb[c] = 0;
        if (znext && gval[c]) {
          const int o = (ze + 1) * nxy + gofs[c];
          nv[c] = make_float2(SYNX_LDG(Ft + o), SYNX_LDG(Mt + o));
          if (MASKED) nvb[c] = SYNX_LDG(valid + o);
        }
      }
    }
    __syncthreads();
    // y box sums, sliding down one halo column over the TY output rows (one task per quantity and
    // halo column)
    for (int task = tid; task < NQ * HX; task += NT) {  // one pass when the tasks fit the block
      const int yq = task / HX, ycol = task - yq * HX;
      slide_sums<R, TY>(cs + yq * HY * CSP + ycol, CSP, ys + yq * TY * CSP + ycol, CSP);
      if (NQ * HX <= NT) break;
    }
    __syncthreads();
    // x box sums, sliding along an output row: outputs XSEG k .. XSEG k + XSEG-1 (one task per
    // quantity, output row and segment; consecutive threads take consecutive rows)
    for (int task = tid; task < NQ * TY * (TX / S::XSEG); task += NT) {
      const int row = task % (NQ * TY), seg = task / (NQ * TY);
      slide_sums<R, S::XSEG>(ys + row * CSP + S::XSEG * seg, 1, ws + row * XSP + S::XSEG * seg, 1);
      if (NQ * TY * (TX / S::XSEG) <= NT) break;
    }
    __syncthreads();
    const int cidx = (ty + R) * HX + (tx + R);
    const bool center_ok = out_ok && (!MASKED || vring[sc * HC + cidx]);
    if (MASKED && out_ok && !center_ok) {  // a masked-out voxel: no value, no update
      const int oi = zc * nxy + pofs;
#pragma unroll
      for (int dd = 0; dd < DIM; ++dd) gF[dd * N + oi] = gM[dd * N + oi] = 0.0f;
      if (cc_out != nullptr) cc_out[oi] = 0.0f;
    }
    if (center_ok) {
      T Sq[NQ];
#pragma unroll
      for (int q = 0; q < NQ; ++q) Sq[q] = ws[(q * TY + ty) * XSP + tx];
      const T czn = (T)(min(zc + RZ, nz - 1) - max(zc - RZ, 0) + 1);
      const T n = MASKED ? Sq[NQ - 1] : cxn * cyn * czn;
      if (MASKED) n_valid += 1.0;
      // the same bits either way; the table saves the reciprocal sequence
      const T inv_n = (sizeof(T) == 8 && P.rcp != nullptr) ? (T)SYNX_LDG(P.rcp + (int)n) : rcp_rn(n);
      const T mF = Sq[0] * inv_n, mM = Sq[1] * inv_n;
      const T sFF = Sq[2] - mF * Sq[0] - mF * Sq[0] + n * mF * mF;
      const T sMM = Sq[3] - mM * Sq[1] - mM * Sq[1] + n * mM * mM;
      const T sFM = Sq[4] - mM * Sq[0] - mF * Sq[1] + n * mM * mF;
      const float2* rc = ring + sc * HC;
      const float2 v0 = rc[cidx];
      const T fh = (T)v0.x - mF, mh = (T)v0.y - mM;
      T cc = T(1), aF = T(0), aM = T(0);
      if (sFF > (T)P.eps && sMM > (T)P.eps) {
        const T prod = sFF * sMM;
        const T ip = rcp_rn(prod);
        cc = sFM * sFM * ip;
        const T coef = T(2) * sFM * ip;
        aF = coef * (fh - sFM * sFF * ip * mh);
        aM = coef * (mh - sFM * sMM * ip * fh);
      }
      cc_acc += (double)cc;
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
          const float2 zm = ring[sm * HC + cidx], zp = ring[sp * HC + cidx];
          gMi[2] = grad1(zm.y, v0.y, zp.y, zc, nz, P.h[2]);
          gFi[2] = grad1(zm.x, v0.x, zp.x, zc, nz, P.h[2]);
        }
      }
      const int oi = zc * nxy + pofs;
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
        gF[dd * N + oi] = (float)(aF * (T)pm);
        gM[dd * N + oi] = (float)(aM * (T)pf);
      }
      if (cc_out != nullptr) cc_out[oi] = (float)cc;
    }
    if (S::END_BARRIER) __syncthreads();
    sc = sp;
  }
  if (MASKED) {
    const double nv = block_sum_d(n_valid, red);
    if (tid == 0 && valid_count) *valid_count = nv;
    __syncthreads();  // red is reused below
  }
  return block_sum_d(cc_acc, red);
}

}  // namespace synx
