// Tunable launch shapes of the channel substep and the autotuner that picks
// them by timing.
//
//   DG_TUNE_COL_MT      modes per CTA of the REM_DIV column kernel (k_rd_col:
//                       REM_DIV_CHAN, and the substep that runs COURANT): 4, 8
//                       or 16.
//   DG_TUNE_CN_MT       modes per CTA of the substep's column kernel
//                       (k_col_cn: right-hand side and CN solve of one field):
//                       2, 4, 8 or 16.  Fewer modes per CTA means more CTAs
//                       and smaller tiles to stage; more means more sweep
//                       lanes per CTA.
//   DG_TUNE_XROW_CHUNK  y-planes one CTA of the x-row product kernel marches
//                       through (0 = automatic).  Longer marches re-read fewer
//                       halo planes; shorter ones give more CTAs.
//   DG_TUNE_YCHUNK      planes per y-chunk of a substep (0 = all): smaller
//                       chunks keep the intermediate planes in L2.
//   DG_TUNE_PDL         1 (default): the substep kernels are launched with
//                       programmatic dependent launch; 0: plain launches.
//   DG_TUNE_FFT_PLAN    radix order of the x and z transform plans: 0 the
//                       largest radix first (128 = 16 x 8), 1 the reverse
//                       (128 = 8 x 16).  Same transform, different shared-
//                       memory strides, twiddle reuse and registers; lengths
//                       whose factors are all equal have one plan.
//   DG_TUNE_PLANE_XZ    1 (default): the LES model's transforms between
//                       spectral planes and physical rows run as one kernel
//                       per direction where the grid allows (x and z lengths
//                       16, 32, 48, 64, 96 or 128); 0: two launches each,
//                       staged through a half-physical array.  Same passes,
//                       same results.
//   DG_TUNE_WAIT_TEST   test only, not a launch shape: value > 0 makes the
//                       next column-kernel launch poll its bulk-copy barrier at
//                       most `value` times and expect 16 bytes more than its
//                       copies bring, so every copy lands but the wait runs
//                       out; the kernel then flags the failure and skips its
//                       work.  It exercises the bounded-wait error path
//                       without a fault; the setting clears after that launch.
//
// dg_autotune times candidate values one tunable at a time (coordinate
// descent) on the handle's own state with CUDA events over a few eager
// steps, keeps the fastest, and restores the state, TIME and DELTA_T it found.
// The choice depends only on the grid and field count, so a caller that
// serves many cases can tune once per shape and copy the values across with
// dg_tune_set.
#include <stdio.h>
#include <string.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "dg_internal.cuh"

// ------------------------------------------------------------ tuning cache
// The autotuner's choices per grid shape, process-wide: key
// "NXxNYxNZ_thN_fp64|mixed", value the launch-shape tunables.  dg_autotune
// stores its result here; dg_tune_lookup applies a stored one;
// dg_tune_cache_save / _load keep the table in a JSON file between runs:
//   {"128x129x128_th0_fp64": {"col_mt": 8, "xrow_chunk": 0, "ychunk": 0,
//    "cn_mt": 4, "pdl": 1, "fft_plan": 0}, ...}
namespace {

constexpr int kTuneKeys[] = {DG_TUNE_COL_MT, DG_TUNE_XROW_CHUNK, DG_TUNE_YCHUNK, DG_TUNE_CN_MT,
                             DG_TUNE_PDL, DG_TUNE_FFT_PLAN};
constexpr const char *kTuneNames[] = {"col_mt", "xrow_chunk", "ychunk", "cn_mt", "pdl",
                                      "fft_plan"};
constexpr int kNTune = 6;

struct TuneRec {
  int v[kNTune];
};

std::mutex g_tmu;
std::map<std::string, TuneRec> g_tcache;

std::string shape_key(const dg_params &p) {
  char b[96];
  snprintf(b, sizeof(b), "%dx%dx%d_th%d_%s", p.nx, p.ny, p.nz, p.n_th,
           p.precision ? "mixed" : "fp64");
  return b;
}

}  // namespace

int dg_default_col_mt(const dg_handle *h) {
  // enough CTAs for about three per SM
  for (int mt : {16, 8})
    if ((h->ss + mt - 1) / mt >= 3 * 148) return mt;
  return 4;
}

static void invalidate_graphs(dg_handle *h) {
  dg_graphs_free(h);
  h->gwarm[0] = h->gwarm[1] = false;
}

extern "C" int dg_tune_set(dg_handle *h, int key, int value) {
  if (!h) return DG_ERR_ARG;
  switch (key) {
    case DG_TUNE_COL_MT:
      if (value != 4 && value != 8 && value != 16) return DG_ERR_ARG;
      h->col_mt = value;
      break;
    case DG_TUNE_CN_MT:
      if (value != 2 && value != 4 && value != 8 && value != 16) return DG_ERR_ARG;
      h->cn_mt = value;
      break;
    case DG_TUNE_XROW_CHUNK:
      if (value < 0 || value > 1024) return DG_ERR_ARG;
      h->xrow_chunk = value;
      break;
    case DG_TUNE_YCHUNK:
      if (value < 0 || value > 1 << 20) return DG_ERR_ARG;
      h->ychunk = value;
      break;
    case DG_TUNE_PDL:
      if (value != 0 && value != 1) return DG_ERR_ARG;
      h->pdl = value;
      break;
    case DG_TUNE_WAIT_TEST:
      if (value < 0 || value > (1 << 20)) return DG_ERR_ARG;
      h->wait_test = value;
      break;
    case DG_TUNE_FFT_PLAN:
      if (value != 0 && value != 1) return DG_ERR_ARG;
      h->fft_plan = value;
      break;
    case DG_TUNE_PLANE_XZ:
      if (value != 0 && value != 1) return DG_ERR_ARG;
      h->plane_xz = value;
      break;
    default:
      return DG_ERR_ARG;
  }
  invalidate_graphs(h);
  return DG_OK;
}

extern "C" int dg_tune_get(dg_handle *h, int key, int *value) {
  if (!h || !value) return DG_ERR_ARG;
  switch (key) {
    case DG_TUNE_COL_MT: *value = h->col_mt; return DG_OK;
    case DG_TUNE_CN_MT: *value = h->cn_mt; return DG_OK;
    case DG_TUNE_XROW_CHUNK: *value = h->xrow_chunk; return DG_OK;
    case DG_TUNE_YCHUNK: *value = h->ychunk; return DG_OK;
    case DG_TUNE_PDL: *value = h->pdl; return DG_OK;
    case DG_TUNE_WAIT_TEST: *value = h->wait_test; return DG_OK;
    case DG_TUNE_FFT_PLAN: *value = h->fft_plan; return DG_OK;
    case DG_TUNE_PLANE_XZ: *value = h->plane_xz; return DG_OK;
    default: return DG_ERR_ARG;
  }
}

namespace {

struct Saved {
  std::vector<double2 *> bufs;
  double scal[16];
};

int save_state(dg_handle *h, Saved *sv) {
  const size_t bytes = sizeof(double2) * h->nspec;
  auto keep = [&](const double2 *src) -> int {
    double2 *d = nullptr;
    DG_CUDA(dg_malloc(h, (void **)&d, bytes));
    sv->bufs.push_back(d);
    DG_CUDA(cudaMemcpyAsync(d, src, bytes, cudaMemcpyDeviceToDevice, h->st));
    return DG_OK;
  };
  for (int f = 0; f < h->nf; f++) {
    DG_TRY(keep(h->cu[f]));
    DG_TRY(keep(h->cf[f]));
  }
  DG_TRY(keep(h->cp));
  DG_CUDA(cudaMemcpyAsync(sv->scal, h->dscal, sizeof(sv->scal), cudaMemcpyDeviceToHost, h->st));
  DG_CUDA(cudaStreamSynchronize(h->st));
  return DG_OK;
}

int restore_state(dg_handle *h, Saved *sv) {
  const size_t bytes = sizeof(double2) * h->nspec;
  size_t k = 0;
  for (int f = 0; f < h->nf; f++) {
    DG_CUDA(cudaMemcpyAsync(h->cu[f], sv->bufs[k++], bytes, cudaMemcpyDeviceToDevice, h->st));
    DG_CUDA(cudaMemcpyAsync(h->cf[f], sv->bufs[k++], bytes, cudaMemcpyDeviceToDevice, h->st));
  }
  DG_CUDA(cudaMemcpyAsync(h->cp, sv->bufs[k++], bytes, cudaMemcpyDeviceToDevice, h->st));
  DG_CUDA(cudaMemcpyAsync(h->dscal, sv->scal, sizeof(sv->scal), cudaMemcpyHostToDevice, h->st));
  DG_CUDA(cudaStreamSynchronize(h->st));
  return DG_OK;
}

void free_saved(dg_handle *h, Saved *sv) {
  for (double2 *p : sv->bufs) dg_free(h, p);
  sv->bufs.clear();
}

// device time of `steps` eager RK3 steps, in ms
int time_steps(dg_handle *h, int steps, float *ms) {
  cudaEvent_t e0, e1;
  DG_CUDA(cudaEventCreate(&e0));
  DG_CUDA(cudaEventCreate(&e1));
  int s = DG_OK;
  // one untimed step with the new shape (first launches, table joins)
  for (int rk = 1; rk <= 3 && s == DG_OK; rk++) s = diablo_rk_chan_1(h, 1, rk);
  if (s == DG_OK) cudaEventRecord(e0, h->st);
  for (int i = 0; i < steps && s == DG_OK; i++)
    for (int rk = 1; rk <= 3 && s == DG_OK; rk++) s = diablo_rk_chan_1(h, 2 + i, rk);
  if (s == DG_OK) {
    cudaEventRecord(e1, h->st);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(ms, e0, e1) != cudaSuccess)
      s = DG_ERR_CUDA;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return s;
}

}  // namespace

extern "C" int dg_autotune(dg_handle *h, int steps_per_trial) {
  if (!h || steps_per_trial < 1) return DG_ERR_ARG;
  if (h->periodic) return DG_OK;  // the periodic path has no tunable shapes
  Saved sv;
  int s = save_state(h, &sv);
  if (s != DG_OK) {
    free_saved(h, &sv);
    return s;
  }
  struct Knob {
    int key;
    std::vector<int> vals;
  };
  std::vector<Knob> knobs = {
      {DG_TUNE_CN_MT, {2, 4, 8, 16}},
      {DG_TUNE_COL_MT, {4, 8, 16}},
      {DG_TUNE_XROW_CHUNK, {0, 2, 4, 8, 16}},
      {DG_TUNE_YCHUNK, {0, 16, 32, 64}},
      {DG_TUNE_FFT_PLAN, {0, 1}},
  };
  for (const Knob &k : knobs) {
    int best = 0;
    dg_tune_get(h, k.key, &best);
    float best_ms = 1e30f;
    for (int v : k.vals) {
      if (k.key == DG_TUNE_YCHUNK && v != 0 && v >= h->NY) continue;
      if ((s = dg_tune_set(h, k.key, v)) != DG_OK) break;
      float ms = 0.f;
      if ((s = time_steps(h, steps_per_trial, &ms)) != DG_OK) break;
      if ((s = restore_state(h, &sv)) != DG_OK) break;
      if (ms < best_ms) {
        best_ms = ms;
        best = v;
      }
    }
    if (s != DG_OK) break;
    dg_tune_set(h, k.key, best);
  }
  const int r = restore_state(h, &sv);
  free_saved(h, &sv);
  DG_TRY(s);
  DG_TRY(r);
  {
    TuneRec rec;
    for (int k = 0; k < kNTune; k++) dg_tune_get(h, kTuneKeys[k], &rec.v[k]);
    std::lock_guard<std::mutex> lk(g_tmu);
    g_tcache[shape_key(h->p)] = rec;
  }
  // the tables of the restored DELTA_T
  if (h->tables_pending) {
    DG_CUDA(cudaStreamWaitEvent(h->st, h->ev_join, 0));
    h->tables_pending = false;
  }
  DG_TRY(dg_cn_tables(h));
  DG_CUDA(cudaStreamSynchronize(h->st));
  return DG_OK;
}

extern "C" int dg_tune_lookup(dg_handle *h, int *hit) {
  if (!h || !hit) return DG_ERR_ARG;
  *hit = 0;
  TuneRec rec;
  {
    std::lock_guard<std::mutex> lk(g_tmu);
    auto it = g_tcache.find(shape_key(h->p));
    if (it == g_tcache.end()) return DG_OK;
    rec = it->second;
  }
  for (int k = 0; k < kNTune; k++) DG_TRY(dg_tune_set(h, kTuneKeys[k], rec.v[k]));
  *hit = 1;
  return DG_OK;
}

extern "C" int dg_tune_cache_get(const dg_params *p, int key, int *value) {
  if (!p || !value) return DG_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_tmu);
  auto it = g_tcache.find(shape_key(*p));
  if (it == g_tcache.end()) return DG_ERR_ARG;
  for (int k = 0; k < kNTune; k++)
    if (kTuneKeys[k] == key) {
      *value = it->second.v[k];
      return DG_OK;
    }
  return DG_ERR_ARG;
}

extern "C" int dg_tune_cache_save(const char *path) {
  if (!path) return DG_ERR_ARG;
  std::string out = "{";
  {
    std::lock_guard<std::mutex> lk(g_tmu);
    bool first = true;
    for (const auto &kv : g_tcache) {
      out += first ? "\n" : ",\n";
      first = false;
      out += " \"" + kv.first + "\": {";
      for (int k = 0; k < kNTune; k++) {
        char b[48];
        snprintf(b, sizeof(b), "%s\"%s\": %d", k ? ", " : "", kTuneNames[k], kv.second.v[k]);
        out += b;
      }
      out += "}";
    }
  }
  out += "\n}\n";
  FILE *f = fopen(path, "w");
  if (!f) {
    dg_set_error((std::string("cannot write the tuning cache ") + path).c_str());
    return DG_ERR_ARG;
  }
  const bool ok = fwrite(out.data(), 1, out.size(), f) == out.size();
  if (fclose(f) != 0 || !ok) {
    dg_set_error((std::string("writing the tuning cache ") + path + " failed").c_str());
    return DG_ERR_ARG;
  }
  return DG_OK;
}

// Reads the file dg_tune_cache_save writes (a JSON object of objects whose
// values are integers) and merges its entries into the table.  Unknown
// tunable names are ignored; an entry lacking one keeps that tunable's
// default; anything that is not this shape of JSON is an error and leaves
// the table as it was.
extern "C" int dg_tune_cache_load(const char *path) {
  if (!path) return DG_ERR_ARG;
  FILE *f = fopen(path, "r");
  if (!f) {
    dg_set_error((std::string("cannot read the tuning cache ") + path).c_str());
    return DG_ERR_ARG;
  }
  std::string t;
  char buf[4096];
  size_t n;
  while ((n = fread(buf, 1, sizeof(buf), f)) > 0) t.append(buf, n);
  fclose(f);
  size_t i = 0;
  auto ws = [&] {
    while (i < t.size() && (t[i] == ' ' || t[i] == '\n' || t[i] == '\r' || t[i] == '\t')) i++;
  };
  auto str = [&](std::string &o) -> bool {
    ws();
    if (i >= t.size() || t[i] != '"') return false;
    size_t j = t.find('"', i + 1);
    if (j == std::string::npos) return false;
    o = t.substr(i + 1, j - i - 1);
    i = j + 1;
    return true;
  };
  auto ch = [&](char c) -> bool {
    ws();
    if (i < t.size() && t[i] == c) {
      i++;
      return true;
    }
    return false;
  };
  auto bad = [&]() {
    dg_set_error((std::string("the tuning cache ") + path + " is not in the expected format").c_str());
    return DG_ERR_ARG;
  };
  std::map<std::string, TuneRec> got;
  if (!ch('{')) return bad();
  if (!ch('}')) {
    do {
      std::string key;
      if (!str(key) || !ch(':') || !ch('{')) return bad();
      TuneRec rec = {{8, 0, 0, 4, 1, 0}};
      if (!ch('}')) {
        do {
          std::string name;
          if (!str(name) || !ch(':')) return bad();
          ws();
          char *end = nullptr;
          const long v = strtol(t.c_str() + i, &end, 10);
          if (end == t.c_str() + i) return bad();
          i = end - t.c_str();
          for (int k = 0; k < kNTune; k++)
            if (name == kTuneNames[k]) rec.v[k] = (int)v;
        } while (ch(','));
        if (!ch('}')) return bad();
      }
      got[key] = rec;
    } while (ch(','));
    if (!ch('}')) return bad();
  }
  std::lock_guard<std::mutex> lk(g_tmu);
  for (const auto &kv : got) g_tcache[kv.first] = kv.second;
  return DG_OK;
}
