// Host-side declarations shared by the library's translation units (no CUDA types).
#pragma once

#include <string>

namespace synx {

// Records `msg` as the calling thread's last global error, the text synx_last_error(NULL)
// returns, and passes `code` through.
int set_global_error(int code, const std::string& msg);

// Tile plan of one level on the per-kernel path (or whether it runs in the persistent level
// kernel instead), as the autotuner's table records it.
struct LevelPlan {
  int persistent;   // 1: persistent level kernel (when eligible), 0: per-kernel path, -1: size threshold
  int smooth_rows;  // 3-D update smoothing: 8 / 16 slab tile rows, -1: xy + z kernels, -2 / -3: pipelined
                    // xy kernel (32 / 64-row tiles) + z kernel
  int cc_chunks;    // z chunks of the CC kernel, 0: its cost model
};

// Loads the default tuning table once per process.
void tuning_ensure_loaded();
// The table's plan for a level grid (exact dims, else the nearest size within a factor of 1.5).
bool tuning_lookup(int dim, int r_cc, int r_smooth, int nx, int ny, int nz, LevelPlan* out);

}  // namespace synx
