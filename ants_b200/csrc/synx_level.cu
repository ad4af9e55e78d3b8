// Persistent level kernel: host side (kernel selection, occupancy, cooperative launch).  The
// kernel itself is in synx_level_body.cuh, instantiated per CC radius by synx_level_inst.cu.
#include <algorithm>

#include "synx_level.cuh"

namespace synx {

void* level_kernel_r1(int dim, bool batch);
void* level_kernel_r2(int dim, bool batch);
void* level_kernel_r3(int dim, bool batch);
void* level_kernel_r4(int dim, bool batch);
void* level_kernel_r5(int dim, bool batch);
void* level_kernel_r6(int dim, bool batch);
void* level_kernel_r7(int dim, bool batch);

namespace {

void* pick_kernel(int dim, int rcc, bool batch) {
  switch (rcc) {
    case 1: return level_kernel_r1(dim, batch);
    case 2: return level_kernel_r2(dim, batch);
    case 3: return level_kernel_r3(dim, batch);
    case 4: return level_kernel_r4(dim, batch);
    case 5: return level_kernel_r5(dim, batch);
    case 6: return level_kernel_r6(dim, batch);
    case 7: return level_kernel_r7(dim, batch);
    default: return nullptr;
  }
}

}  // namespace

size_t level_smem_bytes(int dim, int cc_radius, int r_smooth) {
  const size_t a = cc_smem_bytes(dim, cc_radius);
  const size_t b = smooth3_smem_floats(dim, std::max(r_smooth, kLevelMaxSmoothRadius), kLevelSmoothTY) * 4;
  return std::max(a, b);
}

static int max_blocks_of(void* k, size_t smem, int device) {
  if (!k) return 0;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int per_sm = 0, sms = 0, coop = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 256, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
  if (!coop) return 0;
  return per_sm * sms;
}

int level_max_blocks(int dim, int cc_radius, int r_smooth, int device) {
  return max_blocks_of(pick_kernel(dim, cc_radius, false), level_smem_bytes(dim, cc_radius, r_smooth), device);
}

cudaError_t launch_level(const LevelArgs& A, int dim, int cc_radius, int blocks, cudaStream_t s) {
  void* k = pick_kernel(dim, cc_radius, false);
  if (!k) return cudaErrorInvalidValue;
  add_launch_count(1);
  const size_t smem = level_smem_bytes(dim, cc_radius, A.r_smooth);
  void* args[] = {(void*)&A};
  return cudaLaunchCooperativeKernel(k, dim3(blocks), dim3(256), args, smem, s);
}

int level_batch_max_blocks(int dim, int cc_radius, int device) {
  return max_blocks_of(pick_kernel(dim, cc_radius, true), level_smem_bytes(dim, cc_radius, kLevelMaxSmoothRadius),
                       device);
}

cudaError_t launch_level_batch(const BatchLevelArgs& B, int dim, int cc_radius, int blocks, cudaStream_t s) {
  void* k = pick_kernel(dim, cc_radius, true);
  if (!k || B.npairs < 1 || blocks < B.npairs) return cudaErrorInvalidValue;
  add_launch_count(1);
  const size_t smem = level_smem_bytes(dim, cc_radius, kLevelMaxSmoothRadius);
  void* args[] = {(void*)&B};
  return cudaLaunchCooperativeKernel(k, dim3(blocks), dim3(256), args, smem, s);
}

int level_zb(const Dims& d, int halves) {
  // z depth of the 32 x 8 tiles of a per-voxel phase: minimises the rounds of tiles over a full
  // cooperative grid (296 blocks on 148 SMs) times the work of one tile (its slices plus about
  // half a slice of set-up).  A constant grid size, so the decomposition is the same whatever grid
  // or group runs the level.
  const int G = 296;
  const int gxy = ((d.nx + 31) / 32) * ((d.ny + 7) / 8) * halves;
  int best_zb = d.nz;
  double best = -1.0;
  for (int zb = 1; zb <= d.nz; ++zb) {
    const long long units = (long long)gxy * ((d.nz + zb - 1) / zb);
    const double cost = (double)((units + G - 1) / G) * (zb + 0.5);
    if (best < 0 || cost < best) {
      best = cost;
      best_zb = zb;
    }
  }
  return best_zb;
}

}  // namespace synx
