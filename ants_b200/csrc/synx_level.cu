// Persistent level kernel: host side (kernel selection, occupancy, cooperative launch).  The
// kernel itself is in synx_level_body.cuh, instantiated per CC radius by synx_level_inst.cu.
#include <algorithm>

#include "synx_level.cuh"

namespace synx {

void* level_kernel_r1(int dim);
void* level_kernel_r2(int dim);
void* level_kernel_r3(int dim);
void* level_kernel_r4(int dim);
void* level_kernel_r5(int dim);
void* level_kernel_r6(int dim);
void* level_kernel_r7(int dim);

namespace {

void* pick_kernel(int dim, int rcc) {
  switch (rcc) {
    case 1: return level_kernel_r1(dim);
    case 2: return level_kernel_r2(dim);
    case 3: return level_kernel_r3(dim);
    case 4: return level_kernel_r4(dim);
    case 5: return level_kernel_r5(dim);
    case 6: return level_kernel_r6(dim);
    case 7: return level_kernel_r7(dim);
    default: return nullptr;
  }
}

}  // namespace

size_t level_smem_bytes(int dim, int cc_radius, int r_smooth) {
  const size_t a = cc_smem_bytes(dim, cc_radius);
  const size_t b = smooth3_smem_floats(dim, std::max(r_smooth, kLevelMaxSmoothRadius)) * 4;
  return std::max(a, b);
}

int level_max_blocks(int dim, int cc_radius, int r_smooth, int device) {
  void* k = pick_kernel(dim, cc_radius);
  if (!k) return 0;
  const size_t smem = level_smem_bytes(dim, cc_radius, r_smooth);
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

cudaError_t launch_level(const LevelArgs& A, int dim, int cc_radius, int blocks, cudaStream_t s) {
  void* k = pick_kernel(dim, cc_radius);
  if (!k) return cudaErrorInvalidValue;
  add_launch_count(1);
  const size_t smem = level_smem_bytes(dim, cc_radius, A.r_smooth);
  void* args[] = {(void*)&A};
  return cudaLaunchCooperativeKernel(k, dim3(blocks), dim3(256), args, smem, s);
}

}  // namespace synx
