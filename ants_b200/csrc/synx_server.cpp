// Serving loop: continuous batching of SyN registration requests on one GPU.
//
// One server thread owns a CUDA stream and a batch (synx_batch_*).  Submitted requests wait in
// a queue; at every loop step the thread admits, in arrival order, each queued request whose
// device footprint fits the remaining budget (and the resident limit), creates its context and
// uploads its images, then advances every resident request by one pyramid level in a single
// synx_batch_step.  Requests finish at different steps; a finished request's fields are copied
// to the caller's buffers and its context goes to a pool: a later request with the same stage
// parameters whose footprint fits the pooled arena reuses it (synx_set_images keeps an arena
// that is large enough), so steady serving allocates no device memory.  Pooled contexts are
// freed, largest first, when admission needs their memory.  Built on the public C ABI only.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/synx.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  synx_params params{};
  const float* fixed = nullptr;
  const float* moving = nullptr;
  synx_geom fg{}, mg{};
  float* fwd = nullptr;
  float* inv = nullptr;
  int64_t bytes = 0;     // footprint of a new context for this request
  int64_t held = 0;      // device bytes its context holds (a reused arena may be larger)
  synx_ctx* ctx = nullptr;
  bool reused = false;
  synx_request_info info{};
};

struct Pooled {
  synx_params params;
  synx_ctx* ctx;
  int64_t bytes;
};

bool same_params(const synx_params& a, const synx_params& b) { return std::memcmp(&a, &b, sizeof(a)) == 0; }

thread_local std::string t_err;

}  // namespace

struct synx_server {
  int device = 0;
  int max_active = 0;
  int64_t budget = 0;
  cudaStream_t stream = nullptr;
  synx_batch* batch = nullptr;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  int64_t next_id = 1;
  std::deque<Request*> queue;
  std::vector<Request*> resident;           // owned by the loop thread between steps
  std::map<int64_t, Request*> all;          // every request not yet collected by wait()
  std::vector<Pooled> pool;                 // finished contexts kept with their arenas
  synx_server_stats st{};
  double last_t = 0.0;                      // for the occupancy integral
  std::thread loop;
  std::string err;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  // under mu
  void account(double t) {
    st.resident_byte_seconds += (double)st.bytes_resident * (t - last_t);
    last_t = t;
  }
};

namespace {

// Completes a request.  A healthy context goes to the pool, a failed one is destroyed.
void finish(synx_server* s, Request* r, int status, const std::string& msg) {
  synx_ctx* drop = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    const double t = s->now();
    s->account(t);
    if (r->info.status >= 1) s->st.bytes_resident -= r->held;
    if (r->ctx) {
      if (status >= 0 && r->held > 0) {
        s->pool.push_back({r->params, r->ctx, r->held});
        s->st.bytes_pooled += r->held;
      } else {
        drop = r->ctx;
      }
      r->ctx = nullptr;
    }
    r->info.status = status;
    r->info.t_done = t;
    if (status < 0) {
      std::strncpy(r->info.error, msg.c_str(), sizeof(r->info.error) - 1);
      s->st.failed += 1;
    } else {
      s->st.completed += 1;
    }
    s->cv_done.notify_all();
  }
  if (drop) synx_destroy(drop);
}

void run_loop(synx_server* s) {
  cudaSetDevice(s->device);
  for (;;) {
    std::vector<Request*> admit;
    std::vector<synx_ctx*> evict;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty() || !s->resident.empty(); });
      if (s->stop && s->resident.empty()) {
        for (Request* r : s->queue) {
          r->info.status = SYNX_E_STATE;
          std::strncpy(r->info.error, "server stopped before the request was admitted", sizeof(r->info.error) - 1);
          r->info.t_done = s->now();
          s->st.failed += 1;
        }
        s->queue.clear();
        s->cv_done.notify_all();
        return;
      }
      // admission: arrival order, every request that fits (no head-of-line blocking); a pooled
      // context with the same parameters and a large enough arena is reused, otherwise pooled
      // contexts are evicted (largest first) until a new arena fits
      if (!s->stop) {
        const double t = s->now();
        for (auto it = s->queue.begin(); it != s->queue.end();) {
          Request* r = *it;
          const bool slot = s->max_active <= 0 || (int)(s->resident.size() + admit.size()) < s->max_active;
          int best = -1;
          for (int i = 0; i < (int)s->pool.size(); ++i)
            if (same_params(s->pool[i].params, r->params) && s->pool[i].bytes >= r->bytes &&
                (best < 0 || s->pool[i].bytes < s->pool[best].bytes))
              best = i;
          bool ok = false;
          if (slot && best >= 0) {
            r->ctx = s->pool[best].ctx;
            r->held = s->pool[best].bytes;
            r->reused = true;
            s->st.bytes_pooled -= r->held;
            s->pool.erase(s->pool.begin() + best);
            ok = true;
          } else if (slot && s->st.bytes_resident + r->bytes <= s->budget) {
            while (s->st.bytes_resident + s->st.bytes_pooled + r->bytes > s->budget && !s->pool.empty()) {
              auto big = std::max_element(s->pool.begin(), s->pool.end(),
                                          [](const Pooled& a, const Pooled& b) { return a.bytes < b.bytes; });
              evict.push_back(big->ctx);
              s->st.bytes_pooled -= big->bytes;
              s->pool.erase(big);
            }
            r->held = r->bytes;
            ok = true;
          }
          if (ok) {
            s->account(t);
            s->st.bytes_resident += r->held;
            s->st.bytes_peak = std::max(s->st.bytes_peak, s->st.bytes_resident + s->st.bytes_pooled);
            r->info.status = 1;
            r->info.t_admit = t;
            admit.push_back(r);
            it = s->queue.erase(it);
          } else {
            ++it;
          }
        }
      }
    }
    for (synx_ctx* c : evict) synx_destroy(c);
    for (Request* r : admit) {
      int rc = SYNX_OK;
      if (!r->ctx) {
        rc = synx_create(&r->params, s->device, (void*)s->stream, &r->ctx);
        if (rc) {
          finish(s, r, rc, synx_last_error(nullptr));
          continue;
        }
      }
      rc = synx_set_images(r->ctx, r->fixed, &r->fg, r->moving, &r->mg);
      if (rc) {
        finish(s, r, rc, synx_last_error(r->ctx));
        continue;
      }
      s->resident.push_back(r);
    }
    if (s->resident.empty()) continue;
    // one step: every resident request runs its next level
    std::vector<synx_ctx*> cs;
    for (Request* r : s->resident) cs.push_back(r->ctx);
    const auto a = Clock::now();
    int adv = 0;
    const int rc = synx_batch_step(s->batch, cs.data(), (int)cs.size(), (void*)s->stream, &adv);
    const double dt = std::chrono::duration<double>(Clock::now() - a).count();
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->st.steps += 1;
      s->st.step_seconds += dt;
    }
    std::vector<Request*> keep;
    if (rc) {
      const std::string msg = synx_batch_last_error(s->batch);
      for (Request* r : s->resident) finish(s, r, rc, msg);
      s->resident.clear();
      continue;
    }
    for (Request* r : s->resident) {
      int done_levels;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        done_levels = ++r->info.levels_done;
      }
      if (done_levels < r->params.n_levels) {
        keep.push_back(r);
        continue;
      }
      const int g = synx_get_fields(r->ctx, r->fwd, r->inv);
      finish(s, r, g ? g : 2, g ? synx_last_error(r->ctx) : "");
    }
    s->resident.swap(keep);
  }
}

}  // namespace

extern "C" {

int synx_server_create(const synx_server_config* cfg, synx_server** out) {
  if (!cfg || !out) {
    t_err = "synx_server_create: null argument";
    return SYNX_E_ARG;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    t_err = "synx_server_create: no CUDA device";
    return SYNX_E_CUDA;
  }
  if (cfg->device < 0 || cfg->device >= ndev || cfg->hbm_budget_bytes < 0 || cfg->max_active < 0) {
    t_err = "synx_server_create: bad device, budget or resident limit";
    return SYNX_E_ARG;
  }
  cudaSetDevice(cfg->device);
  synx_server* s = new synx_server();
  s->device = cfg->device;
  s->max_active = cfg->max_active;
  s->budget = cfg->hbm_budget_bytes;
  if (s->budget == 0) {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    s->budget = (int64_t)(0.9 * (double)fr);
  }
  s->st.budget = s->budget;
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
      synx_batch_create(s->device, &s->batch) != SYNX_OK) {
    t_err = "synx_server_create: stream or batch creation failed";
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return SYNX_E_CUDA;
  }
  s->t0 = Clock::now();
  s->loop = std::thread(run_loop, s);
  *out = s;
  return SYNX_OK;
}

int synx_server_destroy(synx_server* s) {
  if (!s) return SYNX_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->loop.joinable()) s->loop.join();
  cudaSetDevice(s->device);
  for (auto& p : s->pool) synx_destroy(p.ctx);
  s->pool.clear();
  synx_batch_destroy(s->batch);
  cudaStreamDestroy(s->stream);
  for (auto& kv : s->all) delete kv.second;
  delete s;
  return SYNX_OK;
}

const char* synx_server_last_error(const synx_server* s) {
  (void)s;
  return t_err.c_str();
}

int synx_server_submit(synx_server* s, const synx_params* p, const float* fixed, const synx_geom* fg,
                       const float* moving, const synx_geom* mg, float* fwd, float* inv, int64_t* id) {
  if (!s || !p || !fixed || !fg || !moving || !mg || !fwd || !inv || !id) {
    t_err = "synx_server_submit: null argument";
    return SYNX_E_ARG;
  }
  int64_t bytes = 0;
  int rc = synx_footprint(p, fg, mg, &bytes);
  if (rc) {
    t_err = std::string("synx_server_submit: ") + synx_last_error(nullptr);
    return rc;
  }
  if (bytes > s->budget) {
    t_err = "synx_server_submit: the request needs " + std::to_string(bytes) + " device bytes, above the budget of " +
            std::to_string(s->budget);
    return SYNX_E_NOMEM;
  }
  Request* r = new Request();
  r->params = *p;
  r->fixed = fixed;
  r->moving = moving;
  r->fg = *fg;
  r->mg = *mg;
  r->fwd = fwd;
  r->inv = inv;
  r->bytes = bytes;
  r->info.device_bytes = bytes;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      delete r;
      t_err = "synx_server_submit: server is stopping";
      return SYNX_E_STATE;
    }
    r->id = s->next_id++;
    r->info.t_submit = s->now();
    s->all[r->id] = r;
    s->queue.push_back(r);
    s->st.submitted += 1;
    *id = r->id;
  }
  s->cv_work.notify_all();
  return SYNX_OK;
}

int synx_server_wait(synx_server* s, int64_t id, double timeout_s, synx_request_info* info) {
  if (!s) {
    t_err = "synx_server_wait: null server";
    return SYNX_E_ARG;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) {
    t_err = "synx_server_wait: unknown request id";
    return SYNX_E_ARG;
  }
  Request* r = it->second;
  auto done = [&] { return r->info.status == 2 || r->info.status < 0; };
  if (timeout_s < 0) {
    s->cv_done.wait(lk, done);
  } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) {
    if (info) *info = r->info;
    t_err = "synx_server_wait: timed out";
    return SYNX_E_STATE;
  }
  if (info) *info = r->info;
  const int status = r->info.status;
  if (status < 0) t_err = r->info.error;
  s->all.erase(it);
  delete r;
  return status < 0 ? status : SYNX_OK;
}

int synx_server_get_stats(synx_server* s, synx_server_stats* out) {
  if (!s || !out) {
    t_err = "synx_server_get_stats: null argument";
    return SYNX_E_ARG;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  const double t = s->now();
  s->account(t);
  s->st.queued = (int64_t)s->queue.size();
  s->st.resident = 0;
  for (auto& kv : s->all)
    if (kv.second->info.status == 1) s->st.resident += 1;
  s->st.elapsed = t;
  *out = s->st;
  return SYNX_OK;
}

}  // extern "C"
