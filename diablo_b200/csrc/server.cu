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
// shape; later cases of the shape take the tuning cache's entry).  A finished case's state is copied back to
// host memory, its device memory is freed, and the slot goes to the next
// request: requests that arrive while others run are admitted as soon as a
// slot and memory free up.  Step latency is the device time between events
// recorded around each step on the case's stream.
//
// Grouped stepping (dg_server_config DG_SERVER_GROUP_CASES = G > 0): active
// cases of similar size advance together in groups of up to G.  One RK3
// step of a group is one CUDA graph: per substep, every member's transform
// stage (z inverse, x-row products, z forward) runs on the member's own
// stream, the members join, and ONE ragged column launch (k_col_cn) does
// the right-hand sides and CN solves of every member's modes -- a (case,
// mode tile, field) work list over all members -- before the members'
// streams fork again for their REM_DIV (and COURANT) kernels.  Groups run
// concurrently on their own streams.  A
// group is re-captured when a member joins or leaves (at step boundaries,
// after the group's steps in flight have finished).  Results are the same
// as per-case stepping: every mode's arithmetic is the single-case kernels'.
// Cases that change their launch sequence from step to step (LES, COURANT
// at an UPDATE_DT cadence other than every step) step alone as above.
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

// a case can join a group: its step's launch sequence is the same every step
bool groupable(const dg_params &p) {
  return !p.les && (!p.variable_dt || p.update_dt == 1);
}

struct Group {
  std::vector<Active *> m;         // members (owned by the server's case list)
  cudaStream_t gs = nullptr;       // the group's stream: graph launches, column launches
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_m;   // one per member: joins into gs
  cudaEvent_t ev_col = nullptr;    // column launch done: members fork from it
  int cmt = 0;                     // the members' modes per column CTA (all the same)
  void *d_cases = nullptr;         // the column kernel's case table
  int4 *d_work = nullptr;          // and its work list
  dg_col_launch cl = {};           // the column launch's sizes
  cudaGraphExec_t exec = nullptr;
  long long gkernels = 0;
  std::deque<InFlight> inflight;
  std::vector<InFlight> pool;
  // cases placed in the group while its steps were in flight: they join the
  // members (and the graph) at the next rebuild, so completions of steps
  // launched before they joined are not counted for them
  std::vector<Active *> joining;
  bool dirty = true;               // membership changed: rebuild before the next step
  double points = 0;               // mean points per member (grouping by size)
};

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

struct dg_server;
void dg_server_run_grouped(dg_server *s);

struct dg_server {
  int max_active = 8;
  int group_cases = 0;            // > 0: grouped stepping with up to this many cases per group
  bool submitted = false;
  int64_t budget = 0;
  int autotune = 1;
  std::mutex mu;
  std::condition_variable cv_work, cv_done, cv_step;
  std::deque<std::shared_ptr<Request>> queue;
  std::map<int64_t, std::shared_ptr<Request>> all;
  std::vector<Active> active;     // stepping thread only
  std::deque<Active> ready;       // prepared, handed to the stepping thread
  int preparing = 0;
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
      // the process-wide tuning cache holds one entry per grid shape: the
      // first case of a shape is tuned, later ones (and later runs that
      // loaded the cache file) reuse it
      int hit = 0;
      code = dg_tune_lookup(a.h, &hit);
      if (code == DG_OK && !hit) code = dg_autotune(a.h, 2);
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
    // case's step graph (a case that will step in a group runs one eager step)
    const bool grouped = group_cases > 0 && groupable(r->p);
    const int warm = r->nsteps < (grouped ? 1 : 2) ? r->nsteps : (grouped ? 1 : 2);
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
    {
      // the mode is fixed by the first submit (dg_server_config comes before it)
      std::unique_lock<std::mutex> lk(mu);
      cv_step.wait(lk, [&] { return submitted || stop; });
    }
    if (group_cases > 0) {
      dg_server_run_grouped(this);
      return;
    }
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

// ------------------------------------------------------ grouped stepping
struct GroupedLoop {
  dg_server *s;
  std::vector<std::unique_ptr<Active>> cases;  // every active case
  std::vector<std::unique_ptr<Group>> groups;
  std::vector<Active *> solo;                   // cases that step alone

  explicit GroupedLoop(dg_server *sv) : s(sv) {}

  static double pts(const Active *a) { return (double)a->r->p.nx * a->r->p.ny * a->r->p.nz; }

  void free_graph(Group &g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    if (g.d_cases) cudaFree(g.d_cases);
    g.d_cases = nullptr;
    if (g.d_work) cudaFree(g.d_work);
    g.d_work = nullptr;
  }

  Group *new_group() {
    auto g = std::make_unique<Group>();
    cudaStreamCreateWithFlags(&g->gs, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&g->ev_col, cudaEventDisableTiming);
    for (int k = 0; k < 2; k++) {
      InFlight f;
      cudaEventCreate(&f.e0);
      cudaEventCreate(&f.e1);
      g->pool.push_back(f);
    }
    groups.push_back(std::move(g));
    return groups.back().get();
  }

  void destroy_group(size_t gi) {
    Group &g = *groups[gi];
    cudaStreamSynchronize(g.gs);
    free_graph(g);
    for (cudaEvent_t e : g.ev_m) cudaEventDestroy(e);
    for (InFlight &f : g.pool) {
      cudaEventDestroy(f.e0);
      cudaEventDestroy(f.e1);
    }
    cudaEventDestroy(g.ev_fork);
    cudaEventDestroy(g.ev_col);
    cudaStreamDestroy(g.gs);
    groups.erase(groups.begin() + gi);
  }

  // join a group of similar size with room, else open one
  void place(Active *a) {
    if (!groupable(a->r->p)) {
      solo.push_back(a);
      return;
    }
    // a group's members share one column launch, so they share its modes per
    // CTA: the width each one runs alone (same kernel instance, same results)
    const int cmt = dg_col_mt_eff(a->h);
    Group *best = nullptr;
    double bd = 1e30;
    for (auto &g : groups) {
      if ((int)(g->m.size() + g->joining.size()) >= s->group_cases || g->cmt != cmt) continue;
      const double d = fabs(log(pts(a) / g->points));
      if (d < log(4.0) && d < bd) {
        bd = d;
        best = g.get();
      }
    }
    if (!best) {
      best = new_group();
      best->cmt = cmt;
    }
    best->joining.push_back(a);
    double sum = 0;
    for (Active *x : best->m) sum += pts(x);
    for (Active *x : best->joining) sum += pts(x);
    best->points = sum / (best->m.size() + best->joining.size());
    best->dirty = true;
  }

  // one RK3 step of every member (captured into the group's graph)
  int step_body(Group &g) {
    const int n = (int)g.m.size();
    DG_CUDA(cudaEventRecord(g.ev_fork, g.gs));
    for (Active *a : g.m) DG_CUDA(cudaStreamWaitEvent(a->st, g.ev_fork, 0));
    for (Active *a : g.m) {
      dg_handle *h = a->h;
      h->defer_tables = true;
      if (h->p.variable_dt) {
        // the CN tables of the DELTA_T the previous step committed
        DG_CUDA(cudaEventRecord(h->ev_fork, h->st));
        DG_CUDA(cudaStreamWaitEvent(h->st2, h->ev_fork, 0));
        cudaStream_t keep = h->st;
        h->st = h->st2;
        const int st = dg_cn_tables(h);
        h->st = keep;
        DG_TRY(st);
        DG_CUDA(cudaEventRecord(h->ev_join, h->st2));
        h->tables_pending = true;
      }
    }
    for (int rk = 1; rk <= 3; rk++) {
      for (int c = 0; c < n; c++) {
        dg_handle *h = g.m[c]->h;
        bool col = false;
        DG_TRY(dg_chan_nonlinear(h, 2, rk, &col));
        if (h->tables_pending) {
          DG_CUDA(cudaStreamWaitEvent(h->st, h->ev_join, 0));
          h->tables_pending = false;
        }
        DG_CUDA(cudaEventRecord(g.ev_m[c], h->st));
        DG_CUDA(cudaStreamWaitEvent(g.gs, g.ev_m[c], 0));
      }
      DG_TRY(dg_col_batch_launch(g.gs, g.cl, g.d_cases, g.d_work, rk));
      DG_CUDA(cudaEventRecord(g.ev_col, g.gs));
      for (Active *a : g.m) {
        dg_handle *h = a->h;
        DG_CUDA(cudaStreamWaitEvent(h->st, g.ev_col, 0));
        if (dg_chan_cfl(h, 2, rk)) DG_TRY(dg_chan_cfl_tail(h, rk));
        else DG_TRY(dg_rem_div_dev(h, 1, rk, true));
      }
    }
    for (int c = 0; c < n; c++) {
      dg_handle *h = g.m[c]->h;
      h->defer_tables = false;
      DG_TRY(diablo_advance_time(h));
      DG_CUDA(cudaEventRecord(g.ev_m[c], h->st));
      DG_CUDA(cudaStreamWaitEvent(g.gs, g.ev_m[c], 0));
    }
    return DG_OK;
  }

  // tables, work list and graph for the current members (group idle)
  int rebuild(Group &g) {
    free_graph(g);
    for (cudaEvent_t e : g.ev_m) cudaEventDestroy(e);
    g.ev_m.assign(g.m.size(), nullptr);
    for (cudaEvent_t &e : g.ev_m) DG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    std::vector<dg_handle *> hs;
    for (Active *a : g.m) {
      hs.push_back(a->h);
      if (a->h->tables_pending) {
        DG_CUDA(cudaStreamWaitEvent(a->h->st, a->h->ev_join, 0));
        a->h->tables_pending = false;
      }
      DG_CUDA(cudaStreamSynchronize(a->h->st));
    }
    const int want = g.cmt;  // every member's own width (place() groups by it)
    {
      std::vector<unsigned char> tab;
      std::vector<int4> work;
      DG_TRY(dg_col_batch_build(hs.data(), (int)hs.size(), want, tab, work, &g.cl));
      DG_CUDA(cudaMalloc(&g.d_cases, tab.size()));
      // on the group's stream (non-blocking: a legacy-stream copy would not be
      // ordered before the graph launches), finished before tab goes away
      DG_CUDA(cudaMemcpyAsync(g.d_cases, tab.data(), tab.size(), cudaMemcpyHostToDevice, g.gs));
      DG_CUDA(cudaMalloc((void **)&g.d_work, sizeof(int4) * work.size()));
      DG_CUDA(cudaMemcpyAsync(g.d_work, work.data(), sizeof(int4) * work.size(),
                              cudaMemcpyHostToDevice, g.gs));
      DG_CUDA(cudaStreamSynchronize(g.gs));
    }
    DG_CUDA(cudaStreamBeginCapture(g.gs, cudaStreamCaptureModeThreadLocal));
    for (dg_handle *h : hs) h->capturing = true;
    const long long k0 = dg_kernel_launches();
    const int st = step_body(g);
    g.gkernels = dg_kernel_launches() - k0;
    for (dg_handle *h : hs) h->capturing = false;
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(g.gs, &graph);
    if (st != DG_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    if (e != cudaSuccess) {
      dg_set_error((std::string("group graph capture: ") + cudaGetErrorString(e)).c_str());
      return DG_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
      g.exec = nullptr;
      dg_set_error((std::string("group graph instantiate: ") + cudaGetErrorString(ei)).c_str());
      return DG_ERR_CUDA;
    }
    g.dirty = false;
    return DG_OK;
  }

  void retire_case(Active *a) {
    // the server's retire() works on its `active` vector: hand it over
    s->active.push_back(std::move(*a));
    std::lock_guard<std::mutex> lk(s->mu);
    s->retire(s->active.size() - 1);
    for (size_t i = 0; i < cases.size(); i++)
      if (cases[i].get() == a) {
        cases.erase(cases.begin() + i);
        break;
      }
    s->n_active = (int)cases.size();
    s->cv_work.notify_all();
  }

  void fail_group(Group &g, int code) {
    const std::string msg = dg_last_error();
    std::lock_guard<std::mutex> lk(s->mu);
    for (Active *a : g.m) s->fail(*a, code, msg.c_str());
  }

  void run() {
    for (;;) {
      bool progressed = false;
      {
        std::unique_lock<std::mutex> lk(s->mu);
        if (cases.empty() && s->ready.empty()) {
          s->cv_step.wait(lk, [&] {
            return !s->ready.empty() || (s->stop && s->queue.empty() && s->preparing == 0);
          });
          if (s->ready.empty() && s->stop && s->queue.empty() && s->preparing == 0) return;
        }
        while (!s->ready.empty()) {
          cases.push_back(std::make_unique<Active>(std::move(s->ready.front())));
          s->ready.pop_front();
          place(cases.back().get());
          progressed = true;
        }
        s->n_active = (int)cases.size();
      }
      // groups: collect finished steps, retire members that are done,
      // rebuild changed groups once idle, keep two steps in flight
      for (size_t gi = 0; gi < groups.size();) {
        Group &g = *groups[gi];
        while (!g.inflight.empty() && cudaEventQuery(g.inflight.front().e1) == cudaSuccess) {
          InFlight f = g.inflight.front();
          g.inflight.pop_front();
          float ms = 0.f;
          cudaEventElapsedTime(&ms, f.e0, f.e1);
          {
            std::lock_guard<std::mutex> lk(s->mu);
            for (Active *a : g.m) {
              s->step_ms.push_back(ms);
              s->steps_done++;
              s->point_steps += pts(a);
            }
          }
          for (Active *a : g.m) a->completed++;
          g.pool.push_back(f);
          progressed = true;
        }
        if (g.inflight.empty()) {
          // members that are done (or failed) leave the group
          for (size_t k = 0; k < g.m.size();) {
            Active *a = g.m[k];
            if (a->r->status != 2 || a->completed >= a->r->nsteps) {
              g.m.erase(g.m.begin() + k);
              g.dirty = true;
              retire_case(a);
              progressed = true;
            } else {
              k++;
            }
          }
          // cases placed meanwhile join now, before the rebuild
          for (Active *a : g.joining) g.m.push_back(a);
          g.joining.clear();
          if (g.m.empty()) {
            destroy_group(gi);
            continue;
          }
          if (g.dirty) {
            const int code = rebuild(g);
            if (code != DG_OK) {
              fail_group(g, code);  // its members leave at the next pass
              gi++;
              continue;
            }
            progressed = true;
          }
        }
        if (!g.dirty) {
          int left = 1 << 30;
          for (Active *a : g.m) left = std::min(left, a->r->nsteps - a->launched);
          while (left > 0 && !g.pool.empty()) {
            InFlight f = g.pool.back();
            g.pool.pop_back();
            cudaEventRecord(f.e0, g.gs);
            const cudaError_t e = cudaGraphLaunch(g.exec, g.gs);
            cudaEventRecord(f.e1, g.gs);
            g.inflight.push_back(f);
            dg_count_launch((int)g.gkernels);
            for (Active *a : g.m) a->launched++;
            left--;
            progressed = true;
            if (e != cudaSuccess) {
              dg_set_error((std::string("group graph launch: ") + cudaGetErrorString(e)).c_str());
              fail_group(g, DG_ERR_CUDA);
              break;
            }
          }
        }
        gi++;
      }
      // cases that step alone: as in dg_server::loop
      for (size_t i = 0; i < solo.size();) {
        Active &a = *solo[i];
        while (!a.inflight.empty() && cudaEventQuery(a.inflight.front().e1) == cudaSuccess) {
          InFlight f = a.inflight.front();
          a.inflight.pop_front();
          float ms = 0.f;
          cudaEventElapsedTime(&ms, f.e0, f.e1);
          {
            std::lock_guard<std::mutex> lk(s->mu);
            s->step_ms.push_back(ms);
            s->steps_done++;
            s->point_steps += pts(&a);
          }
          a.pool.push_back(f);
          a.completed++;
          progressed = true;
        }
        if (a.r->status != 2 || a.completed >= a.r->nsteps) {
          if (a.inflight.empty()) {
            solo.erase(solo.begin() + i);
            retire_case(&a);
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
              std::lock_guard<std::mutex> lk(s->mu);
              s->fail(a, code, dg_last_error());
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

void dg_server_run_grouped(dg_server *s) {
  cudaSetDevice(s->device);
  GroupedLoop gl(s);
  gl.run();
}

extern "C" int dg_server_config(dg_server *s, int key, int value) {
  if (!s) return DG_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->submitted) {
    dg_set_error("dg_server_config must come before the first submit");
    return DG_ERR_ARG;
  }
  if (key == DG_SERVER_GROUP_CASES) {
    if (value < 0 || value > 64) return DG_ERR_ARG;
    s->group_cases = value;
    return DG_OK;
  }
  return DG_ERR_ARG;
}

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
    s->submitted = true;
    if (s->t_first_submit < 0) s->t_first_submit = r->t_submit;
    s->all[r->id] = r;
    s->queue.push_back(r);
  }
  s->cv_work.notify_one();
  s->cv_step.notify_all();
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
