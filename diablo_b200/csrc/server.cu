// Continuous-batching ensemble server: independent channel solves of
// different sizes and physics run concurrently on one GPU.
//
// A request carries a dg_params, the GY grid, a compact spectral initial
// state and a step count.  A scheduler thread admits queued requests while a
// slot is free and the device bytes of the active cases plus the newcomer
// (dg_state_bytes) fit the HBM budget; an admitted case gets its own handle
// and stream, its state is uploaded, and, on request, APPLY_BC_VEL,
// REM_DIV_CHAN, APPLY_BC_VEL prepare it as CREATE_FLOW_CHAN does.  An
// admission thread does this set-up (and the first two steps, which capture
// the case's step graph) so that a stepping thread never waits on it; the
// stepping thread keeps up to two RK3 steps of every active case in flight:
// each step is one replay of the case's captured graph (diablo_step) on the
// case's stream, so steps of different cases overlap on the device.  Launch
// shapes are tuned once per grid shape (dg_autotune on the first case of a
// shape, reused for later ones).  A finished case's state is copied back to
// host memory, its device memory is freed, and the slot goes to the next
// request: requests that arrive while others run are admitted as soon as a
// slot and memory free up.  Step latency is the device time between events
// recorded around each step on the case's stream.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "dg_internal.cuh"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
  int64_t id = 0;
  dg_params p{};
  std::vector<double> gy;
  std::vector<std::vector<double>> init;  // compact spectral fields, interleaved re/im
  std::vector<std::vector<double>> out;
  int nsteps = 0;
  int prepare = 0;
  int status = 1;  // 1 queued, 2 running, 0 done, <0 error (negated DG code)
  std::string err;
  double t_submit = 0, t_admit = 0, t_done = 0;
};

struct InFlight {
  cudaEvent_t e0, e1;
};

struct Active {
  std::shared_ptr<Request> r;
  dg_handle *h = nullptr;
  cudaStream_t st = nullptr;
  int launched = 0, completed = 0;
  std::deque<InFlight> inflight;
  std::vector<InFlight> pool;
  int64_t bytes = 0;
};

using ShapeKey = std::tuple<int, int, int, int, int>;

// field ids of the state a request carries: CU1..3, CP, CTH(n)
std::vector<int> state_ids(const dg_params &p) {
  std::vector<int> ids = {DG_CU1, DG_CU2, DG_CU3, DG_CP};
  for (int n = 0; n < p.n_th; n++) ids.push_back(DG_CTH + n);
  return ids;
}

size_t compact_len(const dg_params &p) {
  const size_t nkxp = p.nx / 3 + 1, nkzt = 2 * (p.nz / 3) + 1;
  return 2 * nkxp * nkzt * (size_t)(p.ny + 2);
}

}  // namespace

struct dg_server {
  int max_active = 8;
  int64_t budget = 0;
  int autotune = 1;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_step;
  std::deque<std::shared_ptr<Request>> queue;
  std::map<int64_t, std::shared_ptr<Request>> all;
  std::vector<Active> active;     // stepping thread only
  std::deque<Active> ready;       // prepared, handed to the stepping thread
  int preparing = 0;
  std::map<ShapeKey, std::vector<int>> tuned;
  std::vector<float> step_ms;
  int64_t next_id = 1;
  int64_t bytes_active = 0, bytes_peak = 0;
  int64_t cases_done = 0, steps_done = 0;
  double point_steps = 0;
  double t_first_submit = -1, t_last_done = 0;
  bool stop = false;
  std::thread worker, admitter;
  int device = 0;
  int n_active = 0;               // active.size(), readable under mu

  void fail(Active &a, int code, const char *msg) {
    a.r->status = -code;
    a.r->err = msg ? msg : "";
  }

  // set up one request (on failure its status carries the error code)
  bool try_admit(std::shared_ptr<Request> r, int64_t est) {
    Active a;
    a.r = r;
    a.bytes = est;
    if (cudaStreamCreateWithFlags(&a.st, cudaStreamNonBlocking) != cudaSuccess) {
      std::lock_guard<std::mutex> lk(mu);
      r->status = -DG_ERR_CUDA;
      r->err = "stream creation failed";
      r->t_done = now_s();
      cv_done.notify_all();
      return true;
    }
    int code = diablo_gpu_init(&r->p, r->gy.empty() ? nullptr : r->gy.data(), a.st, &a.h);
    if (code != DG_OK) {
      cudaStreamDestroy(a.st);
      std::lock_guard<std::mutex> lk(mu);
      r->status = -code;
      r->err = dg_last_error();
      r->t_done = now_s();
      cv_done.notify_all();
      return true;  // consumed (failed)
    }
    const std::vector<int> ids = state_ids(r->p);
    for (size_t i = 0; i < ids.size() && code == DG_OK; i++)
      code = diablo_set_field(a.h, ids[i], r->init[i].data(), DG_LAYOUT_COMPACT, DG_HOST);
    if (code == DG_OK) code = diablo_set_time(a.h, 0.0, r->p.delta_t);
    if (code == DG_OK && r->prepare) {
      code = diablo_apply_bc_vel(a.h);
      if (code == DG_OK) code = diablo_rem_div_chan(a.h);
      if (code == DG_OK) code = diablo_apply_bc_vel(a.h);
    }
    if (code == DG_OK && autotune) {
      const ShapeKey key{r->p.nx, r->p.ny, r->p.nz, r->p.n_th, r->p.precision};
      auto it = tuned.find(key);
      if (it == tuned.end()) {
        code = dg_autotune(a.h, 2);
        if (code == DG_OK) {
          std::vector<int> v(4);
          for (int k = 0; k < 4; k++) dg_tune_get(a.h, k, &v[k]);
          tuned[key] = v;
        }
      } else {
        for (int k = 0; k < 4; k++) dg_tune_set(a.h, k, it->second[k]);
      }
    }
    if (code != DG_OK) {
      const std::string msg = dg_last_error();
      diablo_gpu_finalize(a.h);
      cudaStreamDestroy(a.st);
      std::lock_guard<std::mutex> lk(mu);
      r->status = -code;
      r->err = msg;
      r->t_done = now_s();
      cv_done.notify_all();
      return true;
    }
    for (int k = 0; k < 2; k++) {
      InFlight f;
      cudaEventCreate(&f.e0);
      cudaEventCreate(&f.e1);
      a.pool.push_back(f);
    }
    // the first steps run here: the first is eager, the second captures the
    // case's step graph
    const int warm = r->nsteps < 2 ? r->nsteps : 2;
    code = diablo_step(a.h, 1, warm);
    if (code == DG_OK && cudaStreamSynchronize(a.st) != cudaSuccess) code = DG_ERR_CUDA;
    if (code != DG_OK) {
      const std::string msg = dg_last_error();
      for (InFlight &f : a.pool) {
        cudaEventDestroy(f.e0);
        cudaEventDestroy(f.e1);
      }
      diablo_gpu_finalize(a.h);
      cudaStreamDestroy(a.st);
      std::lock_guard<std::mutex> lk(mu);
      r->status = -code;
      r->err = msg;
      r->t_done = now_s();
      cv_done.notify_all();
      return true;
    }
    a.launched = a.completed = warm;
    std::lock_guard<std::mutex> lk(mu);
    r->status = 2;
    r->t_admit = now_s();
    steps_done += warm;
    point_steps += (double)warm * r->p.nx * r->p.ny * r->p.nz;
    ready.push_back(std::move(a));
    return true;
  }

  void retire(size_t idx) {
    Active &a = active[idx];
    std::shared_ptr<Request> r = a.r;
    if (r->status == 2) {
      const std::vector<int> ids = state_ids(r->p);
      r->out.assign(ids.size(), std::vector<double>(compact_len(r->p)));
      int code = DG_OK;
      for (size_t i = 0; i < ids.size() && code == DG_OK; i++)
        code = diablo_get_field(a.h, ids[i], r->out[i].data(), DG_LAYOUT_COMPACT, DG_HOST);
      if (code == DG_OK) {
        double t = 0, dt = 0;
        diablo_get_time(a.h, &t, &dt);
        r->status = 0;
        cases_done++;
      } else {
        r->status = -code;
        r->err = dg_last_error();
      }
    }
    for (InFlight &f : a.pool) {
      cudaEventDestroy(f.e0);
      cudaEventDestroy(f.e1);
    }
    diablo_gpu_finalize(a.h);
    cudaStreamDestroy(a.st);
    bytes_active -= a.bytes;
    r->t_done = now_s();
    t_last_done = r->t_done;
    active.erase(active.begin() + idx);
    cv_done.notify_all();
  }

  // admission thread: set-up of queued requests in arrival order while a
  // slot is free and the budget allows
  void admit_loop() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      cv_work.wait(lk, [&] {
        return stop || (!queue.empty() &&
                        n_active + (int)ready.size() + preparing < max_active);
      });
      if (stop) return;
      std::shared_ptr<Request> r = queue.front();
      const int64_t est = dg_state_bytes(&r->p);
      if (est < 0 || (budget > 0 && est > budget)) {
        queue.pop_front();
        r->status = -DG_ERR_OOM;
        r->err = "case exceeds the HBM budget";
        r->t_done = now_s();
        cv_done.notify_all();
        continue;
      }
      if (budget > 0 && bytes_active + est > budget) {
        // wait for a retirement to free memory
        cv_work.wait(lk, [&] { return stop || bytes_active + est <= budget; });
        continue;
      }
      queue.pop_front();
      preparing++;
      bytes_active += est;
      bytes_peak = std::max(bytes_peak, bytes_active);
      lk.unlock();
      const bool ok = try_admit(r, est);
      lk.lock();
      preparing--;
      if (!ok || r->status < 0) bytes_active -= est;  // failed set-up frees its share
      cv_step.notify_one();
    }
  }

  // stepping thread: collects finished steps and keeps two steps of every
  // active case in flight
  void loop() {
    cudaSetDevice(device);
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu);
        if (active.empty() && ready.empty()) {
          cv_step.wait(lk, [&] {
            return !ready.empty() || (stop && queue.empty() && preparing == 0);
          });
          if (ready.empty() && stop && queue.empty() && preparing == 0) return;
        }
        while (!ready.empty()) {
          active.push_back(std::move(ready.front()));
          ready.pop_front();
        }
        n_active = (int)active.size();
      }
      bool progressed = false;
      for (size_t i = 0; i < active.size();) {
        Active &a = active[i];
        while (!a.inflight.empty() && cudaEventQuery(a.inflight.front().e1) == cudaSuccess) {
          InFlight f = a.inflight.front();
          a.inflight.pop_front();
          float ms = 0.f;
          cudaEventElapsedTime(&ms, f.e0, f.e1);
          {
            std::lock_guard<std::mutex> lk(mu);
            step_ms.push_back(ms);
            steps_done++;
            point_steps += (double)a.r->p.nx * a.r->p.ny * a.r->p.nz;
          }
          a.pool.push_back(f);
          a.completed++;
          progressed = true;
        }
        if (a.r->status != 2 || a.completed >= a.r->nsteps) {
          if (a.inflight.empty()) {
            std::lock_guard<std::mutex> lk(mu);
            retire(i);
            n_active = (int)active.size();
            cv_work.notify_all();
            progressed = true;
            continue;
          }
        } else {
          while (a.launched < a.r->nsteps && !a.pool.empty()) {
            InFlight f = a.pool.back();
            a.pool.pop_back();
            cudaEventRecord(f.e0, a.st);
            const int code = diablo_step(a.h, a.launched + 1, 1);
            cudaEventRecord(f.e1, a.st);
            a.inflight.push_back(f);
            a.launched++;
            progressed = true;
            if (code != DG_OK) {
              std::lock_guard<std::mutex> lk(mu);
              fail(a, code, dg_last_error());
              break;
            }
          }
        }
        i++;
      }
      if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
  }
};

extern "C" int dg_server_create(int max_active, double hbm_budget_gb, int autotune,
                                dg_server **out) {
  if (!out || max_active < 1) return DG_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    dg_set_error("no CUDA device");
    return DG_ERR_NODEV;
  }
  dg_server *s = new dg_server();
  s->max_active = max_active;
  s->budget = (int64_t)(hbm_budget_gb * 1e9);
  s->autotune = autotune;
  cudaGetDevice(&s->device);
  s->worker = std::thread([s] { s->loop(); });
  s->admitter = std::thread([s] { s->admit_loop(); });
  *out = s;
  return DG_OK;
}

extern "C" int dg_server_submit(dg_server *s, const dg_params *p, const double *gy,
                                const double *const *state, int nsteps, int prepare, int64_t *id) {
  if (!s || !p || !state || nsteps < 0 || !id) return DG_ERR_ARG;
  if (p->num_per_dir != 2 || !gy) {
    dg_set_error("the server runs channel cases (num_per_dir = 2, with a GY grid)");
    return DG_ERR_ARG;
  }
  auto r = std::make_shared<Request>();
  r->p = *p;
  r->gy.assign(gy, gy + p->ny + 1);
  const size_t n = compact_len(*p);
  const std::vector<int> ids = state_ids(*p);
  for (size_t i = 0; i < ids.size(); i++) r->init.emplace_back(state[i], state[i] + n);
  r->nsteps = nsteps;
  r->prepare = prepare;
  r->t_submit = now_s();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    if (s->t_first_submit < 0) s->t_first_submit = r->t_submit;
    s->all[r->id] = r;
    s->queue.push_back(r);
  }
  s->cv_work.notify_one();
  *id = r->id;
  return DG_OK;
}

extern "C" int dg_server_wait(dg_server *s, int64_t id, double *const *state, double *times) {
  if (!s) return DG_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return DG_ERR_ARG;
  std::shared_ptr<Request> r = it->second;
  s->cv_done.wait(lk, [&] { return r->status <= 0; });
  if (r->status < 0) {
    dg_set_error(r->err.c_str());
    return -r->status;
  }
  if (state)
    for (size_t i = 0; i < r->out.size(); i++)
      if (state[i]) memcpy(state[i], r->out[i].data(), sizeof(double) * r->out[i].size());
  if (times) {
    times[0] = r->t_admit - r->t_submit;  // queueing
    times[1] = r->t_done - r->t_admit;    // on the device
  }
  r->out.clear();
  r->init.clear();
  return DG_OK;
}

extern "C" int dg_server_query(dg_server *s, dg_server_stats *st) {
  if (!s || !st) return DG_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  memset(st, 0, sizeof(*st));
  st->cases_done = s->cases_done;
  st->steps_done = s->steps_done;
  st->active = s->n_active;
  st->queued = (int)s->queue.size();
  st->bytes_active = s->bytes_active;
  st->bytes_peak = s->bytes_peak;
  if (!s->step_ms.empty()) {
    std::vector<float> v = s->step_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) { return (double)v[(size_t)std::min<double>(v.size() - 1, floor(q * (v.size() - 1) + 0.5))]; };
    st->step_ms_p50 = pct(0.50);
    st->step_ms_p99 = pct(0.99);
  }
  const double span = s->t_last_done - s->t_first_submit;
  if (span > 0 && s->cases_done > 0) {
    st->cases_per_s = s->cases_done / span;
    st->mpoint_steps_per_s = s->point_steps / span / 1e6;
    st->wall_s = span;
  }
  return DG_OK;
}

extern "C" int dg_server_destroy(dg_server *s) {
  if (!s) return DG_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  s->cv_step.notify_all();
  if (s->admitter.joinable()) s->admitter.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    // requests never admitted end with an error
    for (auto &r : s->queue) {
      r->status = -DG_ERR_ARG;
      r->err = "server destroyed before admission";
    }
    s->queue.clear();
  }
  s->cv_step.notify_all();
  if (s->worker.joinable()) s->worker.join();
  s->cv_done.notify_all();
  delete s;
  return DG_OK;
}
