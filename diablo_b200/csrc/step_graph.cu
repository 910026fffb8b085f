// Full RK3 time steps as CUDA graphs.
//
// diablo_step runs what the reference's driver loop does per step
// (for/diablo.f:70-109): RK_CHAN_1 (or RK_PER_1) for RK_STEP = 1, 2, 3 and
// then TIME = TIME + DELTA_T.  The first step of each variant runs eagerly;
// later steps replay a graph captured from the same launch sequence, so the
// host issues one launch per step instead of ~20.  Two variants exist for
// the channel: with and without COURANT (variable DELTA_T at the UPDATE_DT
// cadence).
//
// With variable DELTA_T the CN tables depend on the DELTA_T committed by the
// previous step's COURANT.  Inside a step they are rebuilt on the side stream
// at the start of the step (overlapping substep 1's transforms) and joined
// before substep 1's CN solve; the commit at the end of substep 3 does not
// rebuild them.  The tables are the same ones the per-substep entry point
// builds, so results are identical.
#include "dg_internal.cuh"

namespace {

int step_body(dg_handle *h, int time_step) {
  if (h->periodic) {
    for (int rk = 1; rk <= 3; rk++) DG_TRY(diablo_rk_per_1(h, rk));
    return diablo_advance_time(h);
  }
  if (h->p.variable_dt && !(h->p.les && h->les_nut)) {
    DG_CUDA(cudaEventRecord(h->ev_fork, h->st));
    DG_CUDA(cudaStreamWaitEvent(h->st2, h->ev_fork, 0));
    cudaStream_t keep = h->st;
    h->st = h->st2;
    const int s = dg_cn_tables(h);
    h->st = keep;
    DG_TRY(s);
    DG_CUDA(cudaEventRecord(h->ev_join, h->st2));
    h->tables_pending = true;
  }
  h->defer_tables = true;
  int s = DG_OK;
  for (int rk = 1; rk <= 3 && s == DG_OK; rk++) s = diablo_rk_chan_1(h, time_step, rk);
  h->defer_tables = false;
  DG_TRY(s);
  if (h->tables_pending) {  // not consumed (no CN solve ran): join anyway
    DG_CUDA(cudaStreamWaitEvent(h->st, h->ev_join, 0));
    h->tables_pending = false;
  }
  return diablo_advance_time(h);
}

bool graph_ok(const dg_handle *h) {
  // the periodic forcing reads its coefficient back to the host every substep;
  // an LES that waits for step 100 of a new flow changes its launch sequence
  return !(h->periodic && h->p.epsilon_target != 0.0) && !(h->p.les && h->p.create_new_flow);
}

int capture(dg_handle *h, int time_step, int v) {
  if (h->tables_pending) {
    DG_CUDA(cudaStreamWaitEvent(h->st, h->ev_join, 0));
    h->tables_pending = false;
  }
  DG_CUDA(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
  h->capturing = true;
  const long long k0 = dg_kernel_launches();
  const int s = step_body(h, time_step);
  h->gkernels[v] = dg_kernel_launches() - k0;
  h->capturing = false;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(h->st, &g);
  if (s != DG_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  if (e != cudaSuccess) {
    dg_set_error((std::string("graph capture of the RK3 step: ") + cudaGetErrorString(e)).c_str());
    return DG_ERR_CUDA;
  }
  e = cudaGraphInstantiate(&h->gexec[v], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    h->gexec[v] = nullptr;
    dg_set_error((std::string("graph instantiate: ") + cudaGetErrorString(e)).c_str());
    return DG_ERR_CUDA;
  }
  return DG_OK;
}

}  // namespace

void dg_graphs_free(dg_handle *h) {
  for (int v = 0; v < 2; v++)
    if (h->gexec[v]) {
      cudaGraphExecDestroy(h->gexec[v]);
      h->gexec[v] = nullptr;
    }
}

extern "C" int diablo_step(dg_handle *h, int time_step, int nsteps) {
  if (!h || nsteps < 0) return DG_ERR_ARG;
  for (int i = 0; i < nsteps; i++) {
    const int ts = time_step + i;
    const int v = (!h->periodic && h->p.variable_dt && h->p.update_dt > 0 &&
                   ts % h->p.update_dt == 0) ? 1 : 0;
    if (!graph_ok(h) || !h->gwarm[v]) {
      DG_TRY(step_body(h, ts));
      h->gwarm[v] = true;
      continue;
    }
    if (!h->gexec[v]) DG_TRY(capture(h, ts, v));
    if (h->tables_pending) {
      DG_CUDA(cudaStreamWaitEvent(h->st, h->ev_join, 0));
      h->tables_pending = false;
    }
    DG_CUDA(cudaGraphLaunch(h->gexec[v], h->st));
    dg_count_launch((int)h->gkernels[v]);
  }
  return DG_OK;
}
