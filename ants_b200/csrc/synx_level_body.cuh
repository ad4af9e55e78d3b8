// Persistent level kernel: every iteration of one level in a single cooperative launch.
//
// Coarse levels are small (13 k - 900 k voxels for the 182x218x182 pyramid), so one iteration's
// ~47 separate launches cost more in launch latency and grid fill than in work.  This kernel keeps
// one block per resident slot on every SM and walks the phases of an iteration (warps, CC,
// smoothing, composition, both fixed-point inverses, the convergence monitor) with a grid-wide
// barrier between phases; the tiles of each phase are spread over the blocks in a block-stride
// loop using the same device functions as the standalone kernels.  Reductions are
// deterministic: block partials in fixed slots, reduced in a fixed order by every block that
// needs the result.  The grid barrier spins on a generation counter with an iteration limit;
// if a wait gives up, the kernel records the error (IterCtl::bar_err) and every block returns.
//
// The batched form (k_level_batch) runs several pairs in one launch: each pair owns a contiguous
// group of blocks, its own control block and barrier, and advances through its own level
// independently of the others.  Every tile decomposition and every reduction order depends on
// the pair's level grid only, never on how many blocks its group has, so a pair gives the same
// bits alone and in any batch.
#pragma once

#include <cooperative_groups.h>

#include <algorithm>
#include <cstring>

#include "synx_cc_tile.cuh"
#include "synx_level.cuh"
#include "synx_phases.cuh"

namespace synx {

namespace {

// The barrier's spin limit comes from LevelArgs::bar_spins (about 2^24 polls, a second or more,
// unless a failure-detection test shortens it).

__device__ __forceinline__ unsigned ld_volatile_u(const unsigned* p) { return *(volatile const unsigned*)p; }
__device__ __forceinline__ int ld_volatile_i(const int* p) { return *(volatile const int*)p; }

// The blocks that work on one pair: block b of G (a whole cooperative grid, or one pair's group
// in the batched kernel).
struct Grp {
  int b, G;
};

// Barrier over the G blocks of a group (all co-resident: cooperative launch).  Returns false
// once any block's wait has timed out.
__device__ bool grid_barrier(IterCtl* ctl, int G, long long spin_limit) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned gen = ld_volatile_u(&ctl->bar_gen);
    __threadfence();
    const unsigned arrived = atomicAdd(&ctl->bar_count, 1u) + 1u;
    if (arrived == (unsigned)G) {
      ctl->bar_count = 0u;
      __threadfence();
      atomicAdd(&ctl->bar_gen, 1u);
    } else {
      long long spins = 0;
      while (ld_volatile_u(&ctl->bar_gen) == gen) {
        if (ld_volatile_i(&ctl->bar_err) || ++spins > spin_limit) {
          atomicExch(&ctl->bar_err, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = ld_volatile_i(&ctl->bar_err) == 0;
  }
  __syncthreads();
  return s_ok != 0;
}

struct Units {
  int gx, gy, gz, halves;
  __device__ int count() const { return gx * gy * gz * halves; }
  __device__ void at(int u, int& bx, int& by, int& bz, int& h) const {
    bx = u % gx;
    int r = u / gx;
    by = r % gy;
    r /= gy;
    bz = r % gz;
    h = r / gz;
  }
};

template <int DIM, int R>
__device__ __forceinline__ float smooth_xy_r(const LevelArgs& A, int bx, int by, int z, int h, float* sm) {
  return smooth_xy_tile<DIM, R, kLevelSmoothTY>(A.sxy, A.g, bx, by, z, h, sm);
}

template <int DIM>
__device__ float smooth_xy_dispatch(const LevelArgs& A, int bx, int by, int z, int h, float* sm) {
  switch (A.r_smooth) {
    case 1: return smooth_xy_r<DIM, 1>(A, bx, by, z, h, sm);
    case 2: return smooth_xy_r<DIM, 2>(A, bx, by, z, h, sm);
    case 3: return smooth_xy_r<DIM, 3>(A, bx, by, z, h, sm);
    case 4: return smooth_xy_r<DIM, 4>(A, bx, by, z, h, sm);
    case 5: return smooth_xy_r<DIM, 5>(A, bx, by, z, h, sm);
    case 6: return smooth_xy_r<DIM, 6>(A, bx, by, z, h, sm);
    case 7: return smooth_xy_r<DIM, 7>(A, bx, by, z, h, sm);
    default: return smooth_xy_r<DIM, 8>(A, bx, by, z, h, sm);
  }
}

__device__ float smooth_z_dispatch(const LevelArgs& A, int bx, int by, int zc, int h) {
  switch (A.r_smooth) {
    case 1: return smooth_z_column<1>(A.sz, A.g, bx, by, zc, h);
    case 2: return smooth_z_column<2>(A.sz, A.g, bx, by, zc, h);
    case 3: return smooth_z_column<3>(A.sz, A.g, bx, by, zc, h);
    case 4: return smooth_z_column<4>(A.sz, A.g, bx, by, zc, h);
    case 5: return smooth_z_column<5>(A.sz, A.g, bx, by, zc, h);
    case 6: return smooth_z_column<6>(A.sz, A.g, bx, by, zc, h);
    case 7: return smooth_z_column<7>(A.sz, A.g, bx, by, zc, h);
    default: return smooth_z_column<8>(A.sz, A.g, bx, by, zc, h);
  }
}

// Deterministic reduction of the per-tile partials (n per half, starting at slot `off` of each
// half; sum and max per half): every block that runs it gets bit-identical results.
__device__ void reduce_partials(const LevelArgs& A, int n, int off, double out_sum[2], float out_max[2], double* redd,
                                float* redf) {
  __shared__ double s_sum[2];
  __shared__ float s_max[2];
  for (int h = 0; h < 2; ++h) {
    double s = 0.0;
    float m = 0.0f;
    for (int b = threadIdx.x; b < n; b += blockDim.x) {
      s += __ldcg(A.inv_psum + h * A.pcap + off + b);
      m = fmaxf(m, __ldcg(A.inv_pmax + h * A.pcap + off + b));
    }
    block_sum_max(s, m, redd, redf);
    if (threadIdx.x == 0) {
      s_sum[h] = s;
      s_max[h] = m;
    }
  }
  __syncthreads();
  out_sum[0] = s_sum[0];
  out_sum[1] = s_sum[1];
  out_max[0] = s_max[0];
  out_max[1] = s_max[1];
}

// One fixed-point inversion of both halves (psi <- inv(phi), warm-started from psi).  Each tile
// writes its own residual partials, so the statistics do not depend on the group size.  After the
// barrier that ends a sub-iteration every block reads all of that sub-iteration's partials, while
// faster blocks may already write the next one's: consecutive sub-iterations use the two halves of
// each half-field's slots in turn (nh slots each), and two sub-iterations apart a barrier lies between
// the last read and the next write.
template <int DIM, bool DIAG>
__device__ bool inverse_phase(const LevelArgs& A, const InvArgs& I, int phase, const Grp& gp, double* redd,
                              float* redf) {
  IterCtl* ctl = A.ctl;
  const Units U{A.el_gx, A.el_gy, A.inv_gz, 2};
  const int nu = U.count(), nh = nu / 2;
  const double N = (double)A.g.N;
  // statistics of the starting iterate
  for (int u = gp.b; u < nu; u += gp.G) {
    int bx, by, bz, h;
    U.at(u, bx, by, bz, h);
    double acc = 0.0;
    float mx = 0.0f;
    invert_tile<DIM, DIAG>(I, h, bx, by, bz, false, true, 0.0f, 0.0f, acc, mx);
    block_sum_max(acc, mx, redd, redf);
    if (threadIdx.x == 0) {
      A.inv_psum[h * A.pcap + (u - h * nh)] = acc;  // sub-iteration 0: first slot set
      A.inv_pmax[h * A.pcap + (u - h * nh)] = mx;
    }
  }
  if (!grid_barrier(ctl, gp.G + A.bar_extra, A.bar_spins)) return false;
  double sum[2];
  float mxv[2];
  reduce_partials(A, nh, 0, sum, mxv, redd, redf);
  bool exec[2] = {true, true};
  int iters[2] = {0, 0};
  for (int k = 1; k <= A.inv_max_iter; ++k) {
    if (!exec[0] && !exec[1]) break;
    const float eps = k == 1 ? 0.75f : 0.5f;
    bool st[2];
    float lim[2];
    for (int h = 0; h < 2; ++h) {
      st[h] = exec[h] && (k + 1 <= A.inv_max_iter) && ((double)mxv[h] > A.inv_max_tol) &&
              (sum[h] / N > A.inv_mean_tol);
      lim[h] = eps * mxv[h];
      if (exec[h]) iters[h] = k;
    }
    for (int u = gp.b; u < nu; u += gp.G) {
      int bx, by, bz, h;
      U.at(u, bx, by, bz, h);
      if (!exec[h]) continue;  // uniform over the block
      double acc = 0.0;
      float mx = 0.0f;
      invert_tile<DIM, DIAG>(I, h, bx, by, bz, true, st[h], eps, lim[h], acc, mx);
      if (st[h]) {
        block_sum_max(acc, mx, redd, redf);
        if (threadIdx.x == 0) {
          A.inv_psum[h * A.pcap + (k & 1) * nh + (u - h * nh)] = acc;
          A.inv_pmax[h * A.pcap + (k & 1) * nh + (u - h * nh)] = mx;
        }
      }
    }
    if (!grid_barrier(ctl, gp.G + A.bar_extra, A.bar_spins)) return false;
    if (st[0] || st[1]) reduce_partials(A, nh, (k & 1) * nh, sum, mxv, redd, redf);
    exec[0] = st[0];
    exec[1] = st[1];
  }
  if (gp.b == 0 && threadIdx.x == 0) {
    ctl->inv[phase][0].iters = iters[0];
    ctl->inv[phase][1].iters = iters[1];
  }
  return true;
}

template <int DIM, int RCC, bool DIAG>
__device__ void level_body(const LevelArgs& A, const Grp& gp, unsigned char* smem, double* redd, float* redf) {
  IterCtl* ctl = A.ctl;
  const int G = gp.G, b = gp.b, tid = threadIdx.x;
  const Units UW{A.el_gx, A.el_gy, A.warp_gz, 1};
  const Units UC{A.el_gx, A.el_gy, A.comp_gz, 2};
  const Units UXY{A.el_gx, (A.g.ny + kLevelSmoothTY - 1) / kLevelSmoothTY, A.g.nz, 2};
  const Units UZ{A.el_gx, A.el_gy, A.sz_gz, 2};
  const int ncc = A.cc_gx * A.cc_gy * A.cc_gz;
  for (int it = 0; it < A.iters; ++it) {
    if (ld_volatile_i(&ctl->stop)) break;  // set by block 0 before the last barrier
    // 1. warps
    for (int u = b; u < UW.count(); u += G) {
      int bx, by, bz, h;
      UW.at(u, bx, by, bz, h);
      warp_pair_tile<DIM, DIAG>(A.warp, bx, by, bz);
    }
    if (!grid_barrier(ctl, G + A.bar_extra, A.bar_spins)) return;
    // 2. CC tiles (same tiles and partial slots as the standalone kernel)
    for (int t = b; t < ncc; t += G) {
      const int bx = t % A.cc_gx, by = (t / A.cc_gx) % A.cc_gy, bz = t / (A.cc_gx * A.cc_gy);
      const double s = cc_tile<RCC, DIM>(A.warp.Ft, A.warp.Mt, A.g, A.cc, A.gF, A.gM, nullptr, bx, by, bz, smem, redd);
      if (tid == 0) A.cc_partials[t] = s;
    }
    if (!grid_barrier(ctl, G + A.bar_extra, A.bar_spins)) return;
    // 3. update smoothing (xy, then z in 3-D) with the max ||u/h|| per half
    float mxs[2] = {0.0f, 0.0f};
    for (int u = b; u < UXY.count(); u += G) {
      int bx, by, z, h;
      UXY.at(u, bx, by, z, h);
      const float m = smooth_xy_dispatch<DIM>(A, bx, by, z, h, reinterpret_cast<float*>(smem));
      if (DIM == 2) mxs[h] = fmaxf(mxs[h], m);
    }
    if (DIM == 3) {
      if (!grid_barrier(ctl, G + A.bar_extra, A.bar_spins)) return;
      for (int u = b; u < UZ.count(); u += G) {
        int bx, by, zc, h;
        UZ.at(u, bx, by, zc, h);
        mxs[h] = fmaxf(mxs[h], smooth_z_dispatch(A, bx, by, zc, h));
      }
    }
    for (int h = 0; h < 2; ++h) {
      const float bm = block_max_f(mxs[h], redf);
      if (tid == 0) atomic_max_nonneg(&ctl->maxnorm[h], bm);
    }
    if (!grid_barrier(ctl, G + A.bar_extra, A.bar_spins)) return;
    // 4. scale + compose into the forward half-fields, in place
    for (int u = b; u < UC.count(); u += G) {
      int bx, by, bz, h;
      UC.at(u, bx, by, bz, h);
      compose_tile<DIM, DIAG>(A.comp, ctl, h, bx, by, bz);
    }
    if (!grid_barrier(ctl, G + A.bar_extra, A.bar_spins)) return;
    // 5, 6. psi <- inv(phi) warm from psi, then phi <- inv(psi) warm from phi
    if (!inverse_phase<DIM, DIAG>(A, A.invA, 0, gp, redd, redf)) return;
    if (!inverse_phase<DIM, DIAG>(A, A.invB, 1, gp, redd, redf)) return;
    // 7. metric (reduced like the standalone CC kernel) and the convergence monitor
    if (b == 0) {
      double s = 0.0;
      for (int t = tid; t < ncc; t += blockDim.x) s += __ldcg(A.cc_partials + t);
      s = block_sum_d(s, redd);
      if (tid == 0) {
        ctl->cc_sum = s;
        ctl->metric = -s / (double)A.g.N;
        ctl->maxnorm[0] = ctl->maxnorm[1] = 0u;
      }
      if (tid < 32) {
        __syncwarp();
        converge_step(ctl, A.log, A.conv_threshold, A.conv_window);
      }
    }
    if (!grid_barrier(ctl, G + A.bar_extra, A.bar_spins)) return;
  }
}

// The level's phases carve the dynamic shared memory as the CC tile and the xy smoothing tile lay
// it out; a launch that provides less records IterCtl::bar_err = 2 and every block returns, so a
// host-side sizing mistake is reported by the run instead of reaching outside the allocation.
template <int DIM, int RCC>
__device__ __forceinline__ bool level_smem_ok(const LevelArgs& A) {
  unsigned have;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(have));
  const size_t need_cc = CCShape<RCC, DIM>::smem;
  const size_t need_xy = smooth3_smem_floats(DIM, A.r_smooth, kLevelSmoothTY) * sizeof(float);
  if (have >= need_cc && have >= need_xy) return true;
  if (threadIdx.x == 0) atomicExch(&A.ctl->bar_err, 2);
  return false;
}

template <int DIM, int RCC>
__global__ void __launch_bounds__(256, 2) k_level(const __grid_constant__ LevelArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double redd[32];
  __shared__ float redf[32];
  if (!level_smem_ok<DIM, RCC>(A)) return;
  const Grp gp{(int)blockIdx.x, (int)gridDim.x};
  if (A.diag) level_body<DIM, RCC, true>(A, gp, smem, redd, redf);
  else level_body<DIM, RCC, false>(A, gp, smem, redd, redf);
}

// Several pairs in one cooperative launch: pair p owns blocks [first_block[p], first_block[p+1]).
template <int DIM, int RCC>
__global__ void __launch_bounds__(256, 2) k_level_batch(const __grid_constant__ BatchLevelArgs B) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double redd[32];
  __shared__ float redf[32];
  __shared__ __align__(16) unsigned long long a_raw[sizeof(LevelArgs) / 8];
  __shared__ int s_pair;
  if (threadIdx.x == 0) {
    int lo = 0, hi = B.npairs - 1;  // the last pair whose first block is <= blockIdx.x
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (B.first_block[mid] <= (int)blockIdx.x) lo = mid;
      else hi = mid - 1;
    }
    s_pair = lo;
  }
  __syncthreads();
  const int p = s_pair;
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(B.pairs + p);
  for (int i = threadIdx.x; i < (int)(sizeof(LevelArgs) / 8); i += blockDim.x) a_raw[i] = src[i];
  __syncthreads();
  const LevelArgs& A = *reinterpret_cast<const LevelArgs*>(a_raw);
  if (!level_smem_ok<DIM, RCC>(A)) return;
  const Grp gp{(int)blockIdx.x - B.first_block[p], B.first_block[p + 1] - B.first_block[p]};
  if (A.diag) level_body<DIM, RCC, true>(A, gp, smem, redd, redf);
  else level_body<DIM, RCC, false>(A, gp, smem, redd, redf);
}

}  // namespace

}  // namespace synx
