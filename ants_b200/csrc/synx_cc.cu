// Neighbourhood cross-correlation kernel (value and both SyN update directions), sm_100a.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <map>
#include <mutex>
#include <vector>

#include "synx_cc_tile.cuh"
#include "synx_level.cuh"

namespace synx {

// The window counts' reciprocals (CCParams::rcp), one table per device in a file-scope device array
// (no allocation): filled from the host's IEEE divisions, which round correctly like the device's
// reciprocal, by cc_prepare before any launch that reads it; its address is cached per device.
__device__ double g_cc_rcp[kCCRcpMax + 1];

static const double* cc_rcp_table(bool fill) {
  static std::mutex mu;
  static std::map<int, const double*> addr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  auto it = addr.find(dev);
  if (it != addr.end()) return it->second;
  if (!fill) return nullptr;
  std::vector<double> h(kCCRcpMax + 1, 0.0);
  for (int n = 1; n <= kCCRcpMax; ++n) h[n] = 1.0 / (double)n;
  void* p = nullptr;
  if (cudaMemcpyToSymbol(g_cc_rcp, h.data(), sizeof(double) * h.size()) != cudaSuccess ||
      cudaGetSymbolAddress(&p, g_cc_rcp) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  addr[dev] = static_cast<const double*>(p);
  return addr[dev];
}

// Standalone CC kernel: one tile per block, deterministic metric reduction (block partials,
// the last block sums them in order).
// With metric masks (MASKED) the partials hold each block's cc sum and, after them, its count of
// valid voxels; the value is -sum / count.
// Threads per standalone CC block: 320 = 10 warps own the 640 halo columns of a radius-4 tile two
// each (256 threads would leave a third column to half of the warps), and the register cap keeps two
// blocks per SM.
constexpr int CC_THREADS = 320;

template <int R, int DIM, typename T, bool MASKED = false>
__global__ void __launch_bounds__(CC_THREADS, 2)
    k_cc(const float* __restrict__ Ft, const float* __restrict__ Mt, Dims d, CCParams P, float* __restrict__ gF,
         float* __restrict__ gM, double* __restrict__ partials, IterCtl* ctl, float* __restrict__ cc_out, int rev) {
  griddep_wait();
  if (ctl != nullptr && ctl->stop) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  __shared__ double vcount;
  __shared__ int am_last;
  const int tid = threadIdx.x;
  const uint3 b = sweep_block(rev);
  const double bs = cc_tile<R, DIM, T, MASKED, CC_THREADS>(Ft, Mt, d, P, gF, gM, cc_out, b.x, b.y, b.z, smem_raw, red,
                                                           &vcount);
  const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
  const unsigned bid = b.x + gridDim.x * (b.y + gridDim.y * b.z);  // the tile's partial slot
  if (tid == 0) {
    partials[bid] = bs;
    if (MASKED) partials[nblocks + bid] = vcount;
    __threadfence();
    unsigned t = atomicAdd(&ctl->cc_counter, 1u);
    am_last = (t == nblocks - 1);
  }
  __syncthreads();
  if (am_last) {
    __threadfence();
    double s = 0.0, n = 0.0;
    for (unsigned b = tid; b < nblocks; b += CC_THREADS) {
      s += __ldcg(partials + b);
      if (MASKED) n += __ldcg(partials + nblocks + b);
    }
    s = block_sum_d(s, red);
    if (MASKED) {
      __syncthreads();
      n = block_sum_d(n, red);
    }
    if (tid == 0) {
      const double cnt = MASKED ? n : (double)d.N;
      ctl->cc_sum = s;
      ctl->metric = cnt > 0.0 ? -s / cnt : 0.0;
      ctl->cc_counter = 0u;
    }
  }
}

template <int R, int DIM>
static void cc_launch_t(const float* Ft, const float* Mt, const GridInfo& g, float* gF, float* gM, double* partials,
                        IterCtl* ctl, cudaStream_t s, float* cc_out, dim3 grid, const CCParams& P, bool fp32) {
  if (P.valid != nullptr)
    launch_k(k_cc<R, DIM, double, true>, grid, CC_THREADS, CCShape<R, DIM, double, true>::smem, s, Ft, Mt, g.d, P, gF, gM, partials,
                                                                                     ctl, cc_out, t_rev);
  else if (fp32)
    launch_k(k_cc<R, DIM, float>, grid, CC_THREADS, CCShape<R, DIM, float>::smem, s, Ft, Mt, g.d, P, gF, gM, partials,
             ctl, cc_out, t_rev);
  else
    launch_k(k_cc<R, DIM, double>, grid, CC_THREADS, CCShape<R, DIM, double>::smem, s, Ft, Mt, g.d, P, gF, gM, partials, ctl,
                                                                          cc_out, t_rev);
}

// z-chunk of one CC block.  Each block first fills its z window (2R slices, column updates only,
// about a third of a full slice's work each), then marches its chunk; 2 blocks are resident per
// SM.  The chunk count minimises waves x (chunk + warm-up cost), so the last wave is not mostly
// empty (e.g. 182 slices over 6 x 28 tiles: 7 chunks, 1176 blocks = 3.97 waves of 296).  A tile
// plan may fix the number of chunks instead (at most nz / R, chunks of at least R slices).
static int cc_max_chunks(const GridInfo& g, int radius) {
  return g.d.dim == 2 ? 1 : std::max(1, g.d.nz / std::max(radius, 1));
}

static int cc_zchunk(const GridInfo& g, int radius, int chunks = 0) {
  if (g.d.dim == 2) return 1;
  const int nz = g.d.nz;
  const int max_chunks = cc_max_chunks(g, radius);
  if (chunks > 0) {
    chunks = std::min(chunks, max_chunks);
    return (nz + chunks - 1) / chunks;
  }
  const int bxy = ((g.d.nx + 31) / 32) * ((g.d.ny + 7) / 8);
  const int slots = 2 * 148;
  int best_zc = nz;
  double best = 1e30;
  for (int c = 1; c <= max_chunks; ++c) {
    const int zc = (nz + c - 1) / c;
    const int blocks = bxy * ((nz + zc - 1) / zc);
    const double waves = (double)((blocks + slots - 1) / slots);
    const double cost = waves * (zc + 0.35 * 2 * radius);
    if (cost < best - 1e-9) {
      best = cost;
      best_zc = zc;
    }
  }
  return best_zc;
}

int cc_blocks(const GridInfo& g, int radius, int chunks) {
  const int bx = (g.d.nx + 31) / 32, by = (g.d.ny + 7) / 8;
  const int zc = cc_zchunk(g, radius, chunks);
  return bx * by * ((g.d.nz + zc - 1) / zc);
}

int cc_blocks_max(const GridInfo& g, int radius) {
  return cc_blocks(g, radius, cc_max_chunks(g, radius));
}

template <int R, int DIM>
static size_t cc_smem_t(bool masked) {
  return masked ? CCShape<R, DIM, double, true>::smem : CCShape<R, DIM, double>::smem;
}

size_t cc_smem_bytes(int dim, int radius, bool masked) {
  // CCShape<R, DIM, double, masked>::smem for a run-time radius (the tile's own layout, so the
  // persistent level kernel's allocation cannot fall behind it); radii without a kernel: SIZE_MAX
#define SYNX_CC_SMEM(RR) \
  case RR:               \
    return dim == 3 ? cc_smem_t<RR, 3>(masked) : cc_smem_t<RR, 2>(masked);
  switch (radius) {
    SYNX_CC_SMEM(1)
    SYNX_CC_SMEM(2)
    SYNX_CC_SMEM(3)
    SYNX_CC_SMEM(4)
    SYNX_CC_SMEM(5)
    SYNX_CC_SMEM(6)
    SYNX_CC_SMEM(7)
    default:
      return SIZE_MAX;
  }
#undef SYNX_CC_SMEM
}

template <int R, int DIM>
static cudaError_t cc_prepare_t() {
  cudaError_t e = cudaFuncSetAttribute(k_cc<R, DIM, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)CCShape<R, DIM, double>::smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_cc<R, DIM, double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)CCShape<R, DIM, double, true>::smem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_cc<R, DIM, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)CCShape<R, DIM, float>::smem);
}

cudaError_t cc_prepare(int dim, int radius) {
  if (cc_rcp_table(true) == nullptr) return cudaErrorInitializationError;
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
  return radius >= 1 && radius <= 7 && cc_smem_bytes(dim, radius, true) <= 227 * 1024;
}

CCParams make_cc_params(const GridInfo& g, int radius, int chunks) {
  CCParams P;
  for (int k = 0; k < 3; ++k) P.h[k] = (float)g.sp[k];
  bool ident = true;
  for (int k = 0; k < 9; ++k) {
    P.dir[k] = (float)g.dir[k];
    if (g.dir[k] != ((k % 4) == 0 ? 1.0 : 0.0)) ident = false;
  }
  P.identity_dir = ident ? 1 : 0;
  P.eps = 1.1920928955078125e-07;  // FLT_EPSILON: the reference metric's float guard
  P.valid = nullptr;
  P.rcp = cc_rcp_table(false);  // set up by cc_prepare, which every entry point calls first (else null:
                                // the tile computes the reciprocals)
  P.ZC = cc_zchunk(g, radius, chunks);
  return P;
}

void launch_cc(const float* Ft, const float* Mt, const GridInfo& g, int radius, float* gF, float* gM, double* partials,
               IterCtl* ctl, cudaStream_t s, float* cc_out, bool fp32_sums, int chunks, const unsigned char* valid) {
  add_launch_count(1);
  CCParams P = make_cc_params(g, radius, chunks);
  P.valid = valid;
  dim3 grid((g.d.nx + 31) / 32, (g.d.ny + 7) / 8, (g.d.nz + P.ZC - 1) / P.ZC);
#define SYNX_CC_CASE(RR)                                                                         \
  case RR:                                                                                       \
    if (g.d.dim == 3)                                                                            \
      cc_launch_t<RR, 3>(Ft, Mt, g, gF, gM, partials, ctl, s, cc_out, grid, P, fp32_sums);       \
    else                                                                                         \
      cc_launch_t<RR, 2>(Ft, Mt, g, gF, gM, partials, ctl, s, cc_out, grid, P, fp32_sums);       \
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


}  // namespace synx
