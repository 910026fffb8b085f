// Internal declarations shared by the diablo_b200 CUDA sources.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/diablo_b200.h"

#define DG_MAX_PASSES 12

// ------------------------------------------------------------ error plumbing
void dg_set_error(const char *msg);
void dg_count_launch(int n = 1);

#define DG_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess) {                                                       \
      dg_set_error((std::string(#call) + ": " + cudaGetErrorString(_e)).c_str());  \
      return (_e == cudaErrorMemoryAllocation) ? DG_ERR_OOM : DG_ERR_CUDA;         \
    }                                                                              \
  } while (0)

#define DG_LAUNCHED()                                                              \
  do {                                                                             \
    dg_count_launch();                                                             \
    cudaError_t _e = cudaGetLastError();                                           \
    if (_e != cudaSuccess) {                                                       \
      dg_set_error((std::string("kernel launch: ") + cudaGetErrorString(_e)).c_str()); \
      return DG_ERR_CUDA;                                                          \
    }                                                                              \
  } while (0)

#define DG_TRY(call)                  \
  do {                                \
    int _s = (call);                  \
    if (_s != DG_OK) return _s;       \
  } while (0)

// ------------------------------------------------------------------- FFT plan
struct FftPlan {
  int n;                       // transform length
  int np;                      // number of Stockham passes
  int r[DG_MAX_PASSES];        // radix of each pass (2, 3, 4, 8)
};

bool dg_make_plan(int n, FftPlan *pl);

// up to 3 + DG_MAX_TH field pointers passed by value to kernels.  Device code
// reads them through operator(), an unrolled select: indexing the parameter
// array with a run-time index would make the compiler copy it to local memory.
template <typename T>
struct PtrArray {
  T *p[3 + DG_MAX_TH + 1];
  __device__ __forceinline__ T *operator()(int i) const {
    T *r = p[0];
#pragma unroll
    for (int k = 1; k < 3 + DG_MAX_TH + 1; k++) r = (i == k) ? p[k] : r;
    return r;
  }
};
struct FieldPtrs : PtrArray<double2> {};
struct CFieldPtrs : PtrArray<const double2> {};

// ---------------------------------------------------------- CN system tables
// Per field type, the mode-independent tridiagonal system of one RK substep
// after elimination (rows 0..NY+1): multiplier a'(j), reciprocal pivot 1/b'(j),
// upper diagonal c(j), and what feeds row j's right-hand side.
enum { ROW_ZERO = 0, ROW_RHS = 1, ROW_BC = 2 };

// field slots in the solver (velocity then scalars)
enum { F_U1 = 0, F_U2 = 1, F_U3 = 2, F_TH0 = 3 };

struct dg_ktimer;

struct dg_handle {
  dg_params p;
  int NX, NY, NZ, NTH, NKX, NKZ, TNKZ, NKY, TNKY;
  int nkxp, nkzt, nkyt;
  int nplanes;                  // NY+2 (channel) or TNKY+1 (periodic)
  long ss;                      // retained modes per plane
  long nspec;                   // complex values per spectral field
  int periodic;
  int nf;                       // 3 + N_TH prognostic fields
  int jstart, jend, jstart_th[DG_MAX_TH], jend_th[DG_MAX_TH];
  double pi, eps;

  cudaStream_t st;
  bool own_stream;
  cudaStream_t st2;             // side stream for work off the critical path
  cudaEvent_t ev_fork, ev_join;
  cudaEvent_t ev_cfl0, ev_cfl1;  // COURANT's reduction on the side stream
  bool tables_pending;          // CN tables being rebuilt on st2

  // host copies of the tables
  double *h_gy, *h_gyf, *h_dy, *h_dyf, *h_kx, *h_kz, *h_ky;

  // device tables
  double *gyf, *dy, *dyf, *kx, *kz, *ky, *kx2, *kz2, *ky2;
  double2 *twx, *twz, *twy;     // exp(-2 pi i m / N) for the x, z, y lengths
  float2 *twx_f, *twz_f, *twy_f;  // the same in FP32 (mixed path)
  int mixed;                    // dg_params.precision == 1
  FftPlan plx, plz, ply;

  // device scalars: [0]=time [1]=delta_t [2..4]=h_bar(1..3) [5]=cfl min
  double *dscal;

  // spectral state (compact layout), double2 = (re, im)
  double2 *cu[3 + DG_MAX_TH];   // CU1, CU2, CU3, CTH(n)
  double2 *cf[3 + DG_MAX_TH];   // CF1..3, CFTH(n)
  double2 *cp;
  double2 *cr1;                 // phi from REM_DIV
  double2 *rhs[3 + DG_MAX_TH];  // CN right-hand sides
  double2 *gphi;                // REM_DIV forward-sweep scratch
  double *rem_a, *rem_rb;       // REM_DIV multipliers and reciprocal pivots [NY+2][ss]
  double *cn_tab;               // CN tables [rk][field][5][LP] (LP: NY+2 rounded up to even)
  double *cn_rows;              // CN row templates [field][8][NY+2]

  // work arrays
  double2 *H;                   // half-physical [nf][planes][NZ][nkxp]
  double2 *G;                   // product half-spectra [2nf][planes][NZ][nkxp]
  double2 *work;                // general scratch
  size_t work_bytes;
  unsigned long long *dmin_bits;// CFL min as ordered bits
  int *dflag;                   // non-finite flag

  // periodic extras
  double2 *Hy;                  // y-inverse output [nf][NY][nkzt][nkxp]
  double2 *P;                   // products [9][NY][NZ][nkxp] then [9][NY][nkzt][nkxp]
  double2 *Q;                   // z-forward products [9][NY][nkzt][nkxp]

  dg_ktimer *kt;                // per-kernel event timing (null unless enabled)

  // SAVE_STATS_CHAN running means (host, allocated on first use)
  int nsamples;
  double *h_ubar;               // [3 + N_TH][NY+2]: UBAR, VBAR, WBAR, THBAR(n)

  // full-step CUDA graphs (variant 0: no COURANT, 1: with COURANT)
  cudaGraphExec_t gexec[2];
  bool gwarm[2];
  long long gkernels[2];        // kernels per replay of each variant
  bool capturing;
  bool defer_tables;            // dt commit leaves the CN tables to the next step

  // tunables (dg_tune_set / dg_autotune)
  int pdl;                      // substep kernels use programmatic dependent launch
  int pdl_zinv;                 // the next z inverse follows a kernel of the substep path
  int col_mt;                   // modes per CTA of the REM_DIV column kernel (4, 8, 16)
  int cn_mt;                    // modes per CTA of the column (CN) kernel (2, 4, 8, 16)
  int xrow_chunk;               // planes per CTA of the x-row product kernel (0 = auto)
  int ychunk;                   // planes per y-chunk of a substep (0 = all)
  double *rowc;                 // per-row grid factors of the column kernel [8][LP]
  void *col_dcase;              // device case table of the column kernel (one case)
  int4 *col_dwork;              // and its work list
  int col_dmt, col_dnwork;      // the modes per item they were built for; items
  int fft_plan;                 // radix-order variant of the x and z transform plans (0, 1)
  int zf_nlo;                   // the z forward writes only the nonlinear terms (the
                                // column kernel assembles the right-hand sides)
  int wait_test;                // test only: poll limit of the next column-kernel launch,
                                // whose barrier then expects 16 bytes more than it receives
  int plane_xz;                 // LES transforms: one kernel per direction and plane where
                                // the grid allows (1), or staged through les_H (0)

  // LES (dg_params.les): physical slots [nslots][NY+2][NZ][NX], spectral slots
  // [nslots][NY+2][ss], filter-width factors [2][NY+2] (DYF, DY), mean U1/U3
  double *les_phys;
  double2 *les_spec;
  double *les_dfac;
  double *les_ubar;
  double2 *les_H;               // half-physical staging for LES_HF fields
  double *les_means;            // [2][NY+2]: NU_T_MEAN, EPS_SGS1_MEAN of a requested substep
  double *les_rowtab;           // [6][NY+2] reciprocal grid factors of the LES CN rows
  bool les_stats_req, les_stats_valid;
  bool les_nut;                 // NU_T has been computed (it stays in use from then on)
};

int dg_default_col_mt(const dg_handle *h);
bool dg_mixed_ok(int nx, int nz, int n_th);
bool dg_per_mixed_ok(int nx, int n_th);

void dg_graphs_free(dg_handle *h);

// stream-ordered device allocation of a handle's arrays (on h->st)
cudaError_t dg_malloc(dg_handle *h, void **p, size_t bytes);
void dg_free(dg_handle *h, void *p);

// kernel timing: begin before a launch on stream st; the launch accounting
// after the launch ends it
void dg_kt_begin(dg_handle *h, const char *name, cudaStream_t st);
void dg_kt_end();
void dg_kt_free(dg_handle *h);

// common kernel-launch helpers (defined in fft_kernels.cu)
int dg_cinv_g(dg_handle *h, const double2 *const *fields, int nf, int jmin, int jmax,
              long in_plane, int rowlen, int N, int NK, const FftPlan &pl, const double2 *tw,
              double2 *H, long out_field);
// FP32 working precision (mixed path): FP64 spectral input, FP32 output
int dg_cinv_gf(dg_handle *h, const double2 *const *fields, int nf, int jmin, int jmax,
               long in_plane, int rowlen, int N, int NK, const FftPlan &pl, const float2 *tw,
               float2 *H, long out_field);
int dg_cinv_ff(dg_handle *h, const float2 *const *fields, int nf, int jmin, int jmax,
               long in_plane, int rowlen, int N, int NK, const FftPlan &pl, const float2 *tw,
               float2 *H, long out_field);
int dg_cfwd_ff(dg_handle *h, const float2 *H, long in_field, int nf, int jmin, int jmax,
               int rowlen, int nkt, int N, int NK, const FftPlan &pl, const float2 *tw,
               float2 *const *fields, long out_plane);
int dg_cfwd_g(dg_handle *h, const double2 *H, long in_field, int nf, int jmin, int jmax,
              int rowlen, int nkt, int N, int NK, const FftPlan &pl, const double2 *tw,
              double2 *const *fields, long out_plane);
int dg_zinv(dg_handle *h, const double2 *const *fields, int nf, int jmin, int jmax,
            double2 *H, int field_stride_planes);
int dg_xc2r_planes(dg_handle *h, const double2 *H, int nf, int jmin, int jmax, double *phys,
                   long phys_plane_stride, long phys_row_stride, long field_stride);
int dg_xc2r_cfl(dg_handle *h, const double2 *H, int jmin, int jmax, unsigned long long *out);
int dg_xr2c_planes(dg_handle *h, const double *phys, int nf, int jmin, int jmax,
                   long phys_plane_stride, long phys_row_stride, long field_stride, double2 *H);
int dg_zfwd_planes(dg_handle *h, const double2 *H, int nf, int jmin, int jmax,
                   double2 *const *fields, double2 *raw_ref, long raw_ld);
// whole-plane transforms (spectral planes <-> physical rows, one kernel per
// direction, no staging array): DG_OK once launched, 1 when the grid does not
// allow them (the caller then stages through a half-physical array)
bool dg_plane_ok(const dg_handle *h);
int dg_plane_c2r(dg_handle *h, const double2 *const *in, int nf, int jmin, int jmax, double *phys,
                 long phys_plane_stride, long phys_row_stride, long field_stride);
int dg_plane_r2c(dg_handle *h, const double *phys, int nf, int jmin, int jmax,
                 long phys_plane_stride, long phys_row_stride, long field_stride,
                 double2 *const *out);

// channel / periodic internals
int dg_chan_init(dg_handle *h);
int dg_per_init(dg_handle *h);
int dg_apply_bc_vel_dev(dg_handle *h);
int dg_rem_div_dev(dg_handle *h, int update_cp, int rk_step, bool from_rhs);
int dg_courant_dev(dg_handle *h, const double2 *const *u, bool side = false);
int dg_stats_dev(dg_handle *h, dg_stats *s);
int dg_per_stats(dg_handle *h, dg_stats *s);
int dg_cn_tables(dg_handle *h);
int dg_dt_commit(dg_handle *h);
int dg_courant_phys(dg_handle *h, const double *u_plane1, long pfield);
int dg_les_init(dg_handle *h);
bool dg_les_active(const dg_handle *h, int time_step);
int dg_les_pre(dg_handle *h, int rk_step);
int dg_les_post(dg_handle *h, int time_step, int rk_step, bool sgs);
int dg_chan_nonlinear(dg_handle *h, int time_step, int rk_step, bool *column_next);
bool dg_chan_cfl(const dg_handle *h, int time_step, int rk_step);
int dg_chan_cfl_tail(dg_handle *h, int rk_step);
int dg_col_init(dg_handle *h);
int dg_col_step_dev(dg_handle *h, int rk_step, bool rd);
size_t dg_col_smem(const dg_handle *h, int mt);
bool dg_col_th_to_rhs(const dg_handle *h, int n);
int dg_col_mt_eff(const dg_handle *h);  // modes per CTA the column kernel runs h with
// launch sizes of a column-kernel launch (one case or a server group)
struct dg_col_launch {
  int mt, thr, grid;      // modes per item, threads per CTA, CTAs (one per item)
  int tile, lp, nseg;     // shared-memory layout: the largest case's
  int nwork;              // work items
  size_t smem;
};
int dg_col_batch_build(dg_handle *const *hs, int n, int want_mt, std::vector<unsigned char> &cases,
                       std::vector<int4> &work, dg_col_launch *cl);
int dg_col_batch_launch(cudaStream_t st, const dg_col_launch &cl, const void *dev_cases,
                        const int4 *dev_work, int rk_step);

#define DG_CASE_N(N) \
  case N:            \
    KERNEL_BODY(N);  \
    break;

void dg_big_smem(const void *kern);

static inline int dg_cdiv(long a, long b) { return (int)((a + b - 1) / b); }

// Programmatic dependent launch.  A kernel launched with dg_launch(pdl = 1)
// right after another kernel in the same stream may be scheduled as that
// kernel's CTAs exit, before its completion is flushed: it must call
// dg_pdl_wait() before it reads anything the predecessor writes (or writes
// anything the predecessor reads); only constant tables may be touched
// before.  The predecessors trigger implicitly as their CTAs exit (an explicit
// trigger at kernel entry measured slower: the waiting CTAs held SM slots).
// dg_pdl_wait() is a no-op for a plain launch.
__device__ __forceinline__ void dg_pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// ------------------------------------------------------------------- TMA
// Bulk tensor copies (cp.async.bulk.tensor, no multicast) into shared memory,
// completed on an mbarrier.  Waits are bounded: a copy that does not land
// within the kernel's poll limit (DG_ASYNC_SPIN unless the handle's wait test
// lowers it for one launch) sets dg_handle::dflag[1] (reported by the next
// diablo_stats / diablo_synchronize) and the kernel skips its work.
#define DG_ASYNC_SPIN (1L << 24)

__device__ __forceinline__ unsigned dg_smem_addr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void dg_mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(dg_smem_addr(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void dg_mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(dg_smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
// 2-D tiled load of box (x, y) of the tensor map into shared memory at dst
__device__ __forceinline__ void dg_tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                               unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dg_smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(dg_smem_addr(bar))
      : "memory");
}
// 1-D bulk copy (no multicast) of `bytes` from global to shared memory:
// both addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void dg_bulk_load(void *dst, const void *src, unsigned bytes,
                                             unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dg_smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(src)), "r"(bytes), "r"(dg_smem_addr(bar))
      : "memory");
}
// orders this thread's generic-proxy shared-memory accesses before later
// bulk copies (async proxy) into the same shared memory
__device__ __forceinline__ void dg_fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Folds v >= 0 (or +inf) into the running minimum at *out (the IEEE bit
// patterns of non-negative doubles order like unsigned integers).  The atomic
// runs only when v could lower the stored value: a reduction whose CTAs all
// fold into one address would otherwise serialise on it.
__device__ __forceinline__ void dg_fold_min(unsigned long long *out, double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  if (b < *reinterpret_cast<volatile unsigned long long *>(out)) atomicMin(out, b);
}
// true once phase `parity` of the barrier completed; false after `spin` polls
__device__ __forceinline__ bool dg_mbar_wait(unsigned long long *bar, unsigned parity,
                                             long spin = DG_ASYNC_SPIN) {
  const unsigned a = dg_smem_addr(bar);
  for (long it = 0; it < spin; it++) {
    unsigned done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// host: a 2-D FP64 tensor map over planes of complex modes -- x = 2*ss
// doubles of a plane (row stride ss complex), y = rows planes; box 2*mt x by
int dg_tmap_planes(const void *base, long ss, int rows, int mt, int by, CUtensorMap *out);

template <typename... KArgs, typename... Args>
static inline cudaError_t dg_launch(int pdl, void (*kern)(KArgs...), dim3 grid, dim3 block,
                                    size_t smem, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}
