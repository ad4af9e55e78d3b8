// Allocation-free entry point for the neighbourhood-CC step.
//
// Some callers of this library cannot call cudaMalloc: a plug-in whose host application (a
// viewer, a deep-learning framework with its own caching allocator, a serving process) owns the
// GPU's memory and its budget, or a latency-bound loop that cannot afford the device-wide
// synchronisation a cudaMalloc/cudaFree pair can cause.  synx_cc_metric() allocates a small
// control block and the per-block partial sums of the metric on every call;
// synx_cc_metric_noalloc() runs the same kernel with that scratch taken from a fixed array in
// device memory instead.
//
// The array below is part of the library image: every GPU on which the library is used keeps
// it (about 260 KB) until the process exits.  All calls on a device share it and find the last
// call's contents there; the control block is cleared on the stream before every launch.  The
// first call on a device looks up the array's device address (cudaGetSymbolAddress), so that
// first call should come before any stream capture.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/synx.h"
#include "synx_kernels.cuh"

namespace {

constexpr int kMaxCCBlocks = 32768;  // partial sums of the CC metric (one per block)
constexpr size_t kCtlBytes = (sizeof(synx::IterCtl) + 255) & ~(size_t)255;
constexpr size_t kScratchBytes = kCtlBytes + sizeof(double) * kMaxCCBlocks;
constexpr int kMaxDevices = 64;

// The scratch: a control block (block-arrival counter, metric) followed by the partial sums.
static __device__ __align__(256) unsigned char g_cc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};  // device address of g_cc_scratch, per device

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

// Device address of the scratch array on the current device.  The symbol's host-side name is a
// stand-in, not a device address, so it is looked up once per device with that device current.
int scratch_on_current_device(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(SYNX_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(SYNX_E_UNSUPPORTED, "device index beyond 63");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_cc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fail(SYNX_E_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return SYNX_OK;
}

}  // namespace

extern "C" {

const char* synx_noalloc_last_error(void) { return g_err.c_str(); }

int synx_cc_metric_noalloc(const float* fixed_dev, const float* moving_dev, const synx_geom* g, int radius,
                           float* grad_fixed_dev, float* grad_moving_dev, double* value_host, void* stream) {
  if (!fixed_dev || !moving_dev || !grad_fixed_dev || !grad_moving_dev || !g || (g->dim != 2 && g->dim != 3))
    return fail(SYNX_E_ARG, "synx_cc_metric_noalloc: null pointer or dimension not 2/3");
  for (int d = 0; d < g->dim; ++d)
    if (g->size[d] < 1 || !(g->spacing[d] > 0))
      return fail(SYNX_E_ARG, "synx_cc_metric_noalloc: sizes must be >= 1 and spacings > 0");
  if (g->dim == 2 && g->size[2] != 1) return fail(SYNX_E_ARG, "synx_cc_metric_noalloc: 2-D grid with size[2] != 1");
  const long long n = (long long)g->size[0] * g->size[1] * g->size[2];
  if (n * 3 >= (1LL << 31)) return fail(SYNX_E_ARG, "synx_cc_metric_noalloc: grid too large");
  if (!synx::cc_radius_supported(g->dim, radius))
    return fail(SYNX_E_UNSUPPORTED, "synx_cc_metric_noalloc: radius must be in 1..7");
  synx::GridInfo gi = synx::make_grid(g->dim, g->size, g->spacing, g->origin, g->direction);
  const int blocks = synx::cc_blocks(gi, radius);
  if (blocks > kMaxCCBlocks)
    return fail(SYNX_E_ARG, "synx_cc_metric_noalloc: this grid needs " + std::to_string(blocks) +
                                " CC blocks; the fixed scratch holds at most " + std::to_string(kMaxCCBlocks) +
                                " (for example 8192 x 1024 voxels per slice); use synx_cc_metric");
  cudaStream_t s = (cudaStream_t)stream;
  if (value_host) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t ce = cudaStreamIsCapturing(s, &cap);
    if (ce != cudaSuccess) return fail(SYNX_E_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(ce));
    if (cap != cudaStreamCaptureStatusNone)
      return fail(SYNX_E_ARG, "synx_cc_metric_noalloc: value_host must be NULL while the stream is being captured");
  }
  void* base = nullptr;
  int rc = scratch_on_current_device(&base);
  if (rc) return rc;
  cudaError_t e = synx::cc_prepare(g->dim, radius);
  if (e != cudaSuccess) return fail(SYNX_E_CUDA, std::string("CC kernel setup: ") + cudaGetErrorString(e));
  synx::IterCtl* ctl = reinterpret_cast<synx::IterCtl*>(base);
  double* partials = reinterpret_cast<double*>(static_cast<unsigned char*>(base) + kCtlBytes);
  // the previous call's control block is still there: the arrival counter must start at zero
  e = cudaMemsetAsync(ctl, 0, sizeof(synx::IterCtl), s);
  if (e != cudaSuccess) return fail(SYNX_E_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  synx::launch_cc(fixed_dev, moving_dev, gi, radius, grad_fixed_dev, grad_moving_dev, partials, ctl, s);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SYNX_E_CUDA, std::string("CC launch: ") + cudaGetErrorString(e));
  if (value_host) {
    e = cudaMemcpyAsync(value_host, &ctl->metric, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(SYNX_E_CUDA, std::string("reading the metric: ") + cudaGetErrorString(e));
  }
  return SYNX_OK;
}

}  // extern "C"
