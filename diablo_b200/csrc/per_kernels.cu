// Triply periodic substep (RK_PER_1, for/periodic.f:23-285).
#include "dg_internal.cuh"

int dg_per_init(dg_handle *h) {
  (void)h;
  dg_set_error("periodic path not built yet");
  return DG_ERR_ARG;
}

extern "C" int diablo_rk_per_1(dg_handle *h, int) { return h ? DG_ERR_ARG : DG_ERR_ARG; }
extern "C" int diablo_rem_div_per(dg_handle *h) { return h ? DG_ERR_ARG : DG_ERR_ARG; }
extern "C" int diablo_poisson_p_per(dg_handle *h) { return h ? DG_ERR_ARG : DG_ERR_ARG; }
extern "C" int diablo_poisson_p_chan(dg_handle *h) { return h ? DG_ERR_ARG : DG_ERR_ARG; }
