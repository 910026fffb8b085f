// Per-handle kernel timing with CUDA events.
//
// When enabled, each instrumented launch is bracketed by an event pair
// recorded on the launch's stream: dg_kt_begin() records the start event just
// before the launch, and the launch accounting that follows every launch
// (dg_count_launch) records the end event.  Pairs live in a ring; a slot is
// read back (its end event synchronised) only when the ring wraps onto it or
// when the totals are read, so timing adds no host-device synchronisation in
// the common case.
#include <string.h>

#include <string>
#include <vector>

#include "dg_internal.cuh"

struct dg_ktimer {
  bool on = false;
  static constexpr int cap = 2048;
  cudaEvent_t ev0[cap], ev1[cap];
  int slot_kernel[cap];
  long next = 0;
  std::vector<std::string> names;
  std::vector<long long> count;
  std::vector<double> ms;
};

namespace {
thread_local dg_ktimer *t_pending = nullptr;
thread_local int t_slot = -1;
thread_local cudaStream_t t_stream = nullptr;

void settle(dg_ktimer *t, int s) {
  if (t->slot_kernel[s] < 0) return;
  float v = 0.f;
  if (cudaEventSynchronize(t->ev1[s]) == cudaSuccess &&
      cudaEventElapsedTime(&v, t->ev0[s], t->ev1[s]) == cudaSuccess) {
    t->ms[t->slot_kernel[s]] += v;
    t->count[t->slot_kernel[s]] += 1;
  }
  t->slot_kernel[s] = -1;
}
}  // namespace

void dg_kt_begin(dg_handle *h, const char *name, cudaStream_t st) {
  dg_ktimer *t = h ? h->kt : nullptr;
  if (!t || !t->on || h->capturing) return;
  int k = -1;
  for (size_t i = 0; i < t->names.size(); i++)
    if (t->names[i] == name) {
      k = (int)i;
      break;
    }
  if (k < 0) {
    t->names.push_back(name);
    t->count.push_back(0);
    t->ms.push_back(0.0);
    k = (int)t->names.size() - 1;
  }
  const int s = (int)(t->next % dg_ktimer::cap);
  settle(t, s);
  if (cudaEventRecord(t->ev0[s], st) != cudaSuccess) return;
  t->slot_kernel[s] = k;
  t->next++;
  t_pending = t;
  t_slot = s;
  t_stream = st;
}

void dg_kt_end() {
  if (!t_pending) return;
  if (cudaEventRecord(t_pending->ev1[t_slot], t_stream) != cudaSuccess)
    t_pending->slot_kernel[t_slot] = -1;
  t_pending = nullptr;
}

void dg_kt_free(dg_handle *h) {
  if (!h || !h->kt) return;
  dg_ktimer *t = h->kt;
  for (int s = 0; s < dg_ktimer::cap; s++) {
    cudaEventDestroy(t->ev0[s]);
    cudaEventDestroy(t->ev1[s]);
  }
  delete t;
  h->kt = nullptr;
}

extern "C" int dg_timing_enable(dg_handle *h, int on) {
  if (!h) return DG_ERR_ARG;
  if (on && !h->kt) {
    dg_ktimer *t = new dg_ktimer();
    for (int s = 0; s < dg_ktimer::cap; s++) {
      t->slot_kernel[s] = -1;
      if (cudaEventCreate(&t->ev0[s]) != cudaSuccess || cudaEventCreate(&t->ev1[s]) != cudaSuccess) {
        dg_set_error("cudaEventCreate failed (kernel timing)");
        for (int r = 0; r <= s; r++) {
          cudaEventDestroy(t->ev0[r]);
          cudaEventDestroy(t->ev1[r]);
        }
        delete t;
        return DG_ERR_CUDA;
      }
    }
    h->kt = t;
  }
  if (!h->kt) return DG_OK;
  dg_ktimer *t = h->kt;
  if (on) {
    for (int s = 0; s < dg_ktimer::cap; s++) t->slot_kernel[s] = -1;
    t->names.clear();
    t->count.clear();
    t->ms.clear();
    t->next = 0;
  }
  t->on = on != 0;
  return DG_OK;
}

extern "C" int dg_timing_read(dg_handle *h, int i, char *name, int name_len, int64_t *launches,
                              double *total_ms) {
  if (!h || !h->kt || i < 0) return DG_ERR_ARG;
  dg_ktimer *t = h->kt;
  for (int s = 0; s < dg_ktimer::cap; s++) settle(t, s);
  if (i >= (int)t->names.size()) return DG_ERR_ARG;
  if (name && name_len > 0) {
    strncpy(name, t->names[i].c_str(), name_len - 1);
    name[name_len - 1] = 0;
  }
  if (launches) *launches = t->count[i];
  if (total_ms) *total_ms = t->ms[i];
  return DG_OK;
}
