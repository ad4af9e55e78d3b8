// Tuning table: the tile plans the project's autotuner measured fastest per level grid.
//
// The autotuner (ants_b200/autotune.py) registers representative image pairs once per candidate
// plan, reads each level's iteration time from the level profile, and writes the winner of every
// level grid here as one text line:
//
//   dim nx ny nz r_cc r_smooth  persistent smooth_rows cc_z_chunks  ms_best ms_default
//
// persistent: 1 = the persistent level kernel, 0 = the per-kernel path; smooth_rows: 8 or 16 (the
// fused slab smoothing kernel's tile rows), -1 (xy and z kernels) or -2 / -3 (the pipelined xy kernel
// with 32- / 64-row tiles, and the z kernel); cc_z_chunks: z chunks of the
// CC kernel (0 = its cost model).  The two times are informational.  The table is read once per
// process (first synx_create) from $SYNX_TUNING_TABLE or tuning_b200.txt beside libsynx.so.
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/synx.h"
#include "synx_host.h"

namespace synx {

namespace {

struct TuneEntry {
  int dim, nx, ny, nz, r_cc, r_smooth;
  LevelPlan plan;
};

std::mutex g_tune_mu;
std::vector<TuneEntry> g_table;
std::string g_table_path;
bool g_loaded = false;

std::string default_table_path() {
  const char* env = std::getenv("SYNX_TUNING_TABLE");
  if (env && *env) return env;
  Dl_info info;
  if (dladdr(reinterpret_cast<void*>(&default_table_path), &info) && info.dli_fname) {
    std::string p = info.dli_fname;
    const size_t slash = p.rfind('/');
    return (slash == std::string::npos ? std::string(".") : p.substr(0, slash)) + "/tuning_b200.txt";
  }
  return "tuning_b200.txt";
}

// Parses a table; malformed lines are skipped.  Returns the entries read, or -1 if unreadable.
int load_locked(const std::string& path) {
  g_table.clear();
  g_table_path = path;
  g_loaded = true;
  FILE* f = std::fopen(path.c_str(), "r");
  if (!f) return -1;
  char line[512];
  while (std::fgets(line, sizeof line, f)) {
    if (line[0] == '#' || line[0] == '\n') continue;
    TuneEntry e{};
    double a = 0, b = 0;
    const int n = std::sscanf(line, "%d %d %d %d %d %d %d %d %d %lf %lf", &e.dim, &e.nx, &e.ny, &e.nz, &e.r_cc,
                              &e.r_smooth, &e.plan.persistent, &e.plan.smooth_rows, &e.plan.cc_chunks, &a, &b);
    if (n < 9 || (e.dim != 2 && e.dim != 3) || e.nx < 1 || e.ny < 1 || e.nz < 1) continue;
    if (e.plan.persistent != 0 && e.plan.persistent != 1) continue;
    if (e.plan.smooth_rows != 8 && e.plan.smooth_rows != 16 && (e.plan.smooth_rows < -3 || e.plan.smooth_rows > -1))
      continue;
    if (e.plan.cc_chunks < 0 || e.plan.cc_chunks > 4096) continue;
    g_table.push_back(e);
  }
  std::fclose(f);
  return (int)g_table.size();
}

}  // namespace

void tuning_ensure_loaded() {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  if (!g_loaded) load_locked(default_table_path());
}

bool tuning_lookup(int dim, int r_cc, int r_smooth, int nx, int ny, int nz, LevelPlan* out) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  const TuneEntry* best = nullptr;
  double best_cost = 0.0;
  const double N = (double)nx * ny * nz;
  for (const TuneEntry& e : g_table) {
    if (e.dim != dim || e.r_cc != r_cc || e.r_smooth != r_smooth) continue;
    if (e.nx == nx && e.ny == ny && e.nz == nz) {
      *out = e.plan;
      return true;
    }
    const double Ne = (double)e.nx * e.ny * e.nz;
    const double cost = std::fabs(std::log(N / Ne)) + 0.25 * std::fabs(std::log((double)nz / e.nz));
    if (std::fabs(std::log(N / Ne)) <= std::log(1.5) && (!best || cost < best_cost)) {
      best = &e;
      best_cost = cost;
    }
  }
  if (!best) return false;
  *out = best->plan;
  // a chunk count tuned for another depth is rescaled to this one
  if (out->cc_chunks > 0 && best->nz != nz)
    out->cc_chunks = std::max(1, (int)std::lround((double)out->cc_chunks * nz / best->nz));
  return true;
}

}  // namespace synx

extern "C" {

int synx_tuning_load(const char* path) {
  std::lock_guard<std::mutex> lock(synx::g_tune_mu);
  const int n = synx::load_locked(path ? std::string(path) : synx::default_table_path());
  if (n < 0 && path) return synx::set_global_error(SYNX_E_ARG, "synx_tuning_load: cannot read " + std::string(path));
  return n < 0 ? 0 : n;  // no default table: the cost models plan every level
}

const char* synx_tuning_path(void) {
  synx::tuning_ensure_loaded();
  std::lock_guard<std::mutex> lock(synx::g_tune_mu);
  return synx::g_table_path.c_str();
}

}  // extern "C"
