/*
 * diablo_b200 -- C-ABI of the B200 (sm_100a) replacement for DIABLO's
 * RK3 / Crank-Nicolson hot path.
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (DG_OK = 0) and never aborts the caller.  A Fortran host binds them with
 * ISO_C_BINDING interfaces; the Python mirror in
 * diablo_b200/_lib.py binds them with ctypes.
 *
 * Ownership: the caller's arrays (the reference's COMMON blocks) stay the
 * owner of record on the host; the library keeps device-resident mirrors
 * across substeps and copies only in diablo_set_field / diablo_get_field
 * and in the FFT_XZ / Thomas entry points called on host arrays.
 *
 * Array layouts accepted (DG_LAYOUT_*):
 *   REFERENCE : the reference's own arrays, first index fastest:
 *               spectral  COMPLEX*16 CU(0:NX/2, 0:NZ+1, 0:NY+1)
 *               physical  REAL*8     U (0:NX+1, 0:NZ+1, 0:NY+1)
 *               (for/header:214-245 with NPROCY = NPROCZ = 1)
 *   COMPACT   : retained modes only, [NY+2][TNKZ+1][NKX+1] complex (channel)
 *               or [TNKY+1][TNKZ+1][NKX+1] (periodic); physical [NY+2][NZ][NX]
 *               or [NY][NZ][NX].
 *   REFERENCE_RETAINED : the reference's spectral array, of which only the
 *               retained block (kx 0..NKX, kz slots 0..TNKZ, every plane) is
 *               read or written; diablo_get_field leaves the other entries of
 *               the caller's array as they were.  This is the part the
 *               reference's host consumers read (SAVE_FLOW writes
 *               CU(0:NKX,0:TNKZ,*), for/diablo_io.f:367-391; the statistics
 *               read retained modes), and only it crosses the bus.
 * Complex values are interleaved (re, im) doubles.
 */
#ifndef DIABLO_B200_H
#define DIABLO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DG_MAX_TH 4

enum dg_status {
  DG_OK = 0,
  DG_ERR_ARG = 1,      /* bad argument / unsupported option */
  DG_ERR_DIMS = 2,     /* grid sizes not supported (the reference STOPs) */
  DG_ERR_OOM = 3,      /* device allocation failed */
  DG_ERR_CUDA = 4,     /* CUDA runtime error (message via dg_last_error) */
  DG_ERR_NAN = 5,      /* non-finite value detected in the state */
  DG_ERR_TIMEOUT = 6,  /* a bounded device wait gave up */
  DG_ERR_NODEV = 7     /* no usable sm_100 device */
};

enum { DG_HOST = 0, DG_DEVICE = 1 };
enum { DG_LAYOUT_COMPACT = 0, DG_LAYOUT_REFERENCE = 1, DG_LAYOUT_REFERENCE_RETAINED = 2 };

/* field ids for diablo_set_field / diablo_get_field */
enum {
  DG_CU1 = 0, DG_CU2 = 1, DG_CU3 = 2, DG_CP = 3,
  DG_CF1 = 4, DG_CF2 = 5, DG_CF3 = 6,
  DG_CR1 = 7,               /* phi left by REM_DIV_CHAN (for/channel.f:1189) */
  DG_CTH = 16,              /* + scalar index n (0-based) */
  DG_CFTH = 32              /* + scalar index n */
};

/* What the reference holds in COMMON /INPUT/ and friends (for/header:83-302)
 * plus grid_def's NX, NY, NZ, N_TH.  Field order is ABI. */
typedef struct dg_params {
  int32_t nx, ny, nz, n_th;
  int32_t num_per_dir;        /* 2 = channel (RK_CHAN_1), 3 = periodic (RK_PER_1) */
  int32_t precision;          /* 0 = FP64 throughout, 1 = mixed (FP32 FFT/products) */
  double nu, beta, lx, ly, lz, nu_v_scale;
  double delta_t, cfl;
  int32_t variable_dt, update_dt;
  double i_ro, grav_x, grav_y, grav_z;
  int32_t f_type, pad0;
  double ubulk0, px0, omega0, amp_omega0;
  int32_t u_bc_ymin, v_bc_ymin, w_bc_ymin, u_bc_ymax, v_bc_ymax, w_bc_ymax;
  double u_bc_ymin_c1, v_bc_ymin_c1, w_bc_ymin_c1;
  double u_bc_ymax_c1, v_bc_ymax_c1, w_bc_ymax_c1;
  int32_t th_bc_ymin[DG_MAX_TH], th_bc_ymax[DG_MAX_TH];
  double th_bc_ymin_c1[DG_MAX_TH], th_bc_ymax_c1[DG_MAX_TH];
  double ri[DG_MAX_TH], pr[DG_MAX_TH], drhodx[DG_MAX_TH], drhodz[DG_MAX_TH];
  int32_t background_grad[DG_MAX_TH];
  double epsilon_target;
  int32_t les;                /* USE_LES (input.dat, for/diablo_io.f:25) */
  int32_t les_model_type;     /* for/channel.f:1477; the MPI build runs only 1 */
  int32_t create_new_flow;    /* for/diablo_io.f:31: the model waits 100 steps */
  int32_t pad1;
} dg_params;

/* Parity statistics (SAVE_STATS_CHAN, for/save_stats.f:112-203,470-489). */
typedef struct dg_stats {
  double ubulk, urms_b, vrms_b, wrms_b, ke, div_max;
  double thrms_b[DG_MAX_TH], th_var[DG_MAX_TH];
} dg_stats;

typedef struct dg_handle dg_handle;

/* ---------------------------------------------------------------- misc */
int dg_version(void);
const char *dg_last_error(void);
/* Kernels launched by this library since load (for launch accounting). */
int64_t dg_kernel_launches(void);
/* The ABI structs as compiled: sizeof(dg_params), sizeof(dg_stats), then the
 * offsets of dg_params' nx, nu, f_type, ubulk0, th_bc_ymin, epsilon_target,
 * les, les_model_type, create_new_flow (for binding checks).  Returns the
 * count written; with out = NULL, the count available. */
int dg_abi_layout(int64_t *out, int n);

/* -------------------------------------------------------------- lifecycle
 * Replaces the device-side parts of INITIALIZE: INIT_FFT (for/fft.f:55-147),
 * CREATE_GRID_CHAN's metrics (for/channel.f:1645-1652 via
 * for/hdf5.f:676-703), INIT_CHAN_MPI's JSTART/JEND (for/mpi.f:1067-1135) and
 * the RK3 coefficients (for/diablo_io.f:116-124).
 * gy: GY(1..NY+1) (NY+1 doubles) for the channel, NULL for periodic.
 * stream: a cudaStream_t to run on, or NULL for a library-owned stream. */
int diablo_gpu_init(const dg_params *p, const double *gy, void *stream, dg_handle **out);
int diablo_gpu_finalize(dg_handle *h);
int diablo_synchronize(dg_handle *h);

/* COMMON /RUNTIME_VARS/ TIME and DELTA_T (device-resident; COURANT updates
 * DELTA_T on the device). */
int diablo_set_time(dg_handle *h, double time, double delta_t);
int diablo_get_time(dg_handle *h, double *time, double *delta_t);
/* TIME = TIME + DELTA_T on the device (for/diablo.f:109). */
int diablo_advance_time(dg_handle *h);

/* Host <-> device copies of one spectral field (ids above). */
int diablo_set_field(dg_handle *h, int field, const double *src, int layout, int where);
int diablo_get_field(dg_handle *h, int field, double *dst, int layout, int where);
/* The same for n fields at once (fields[i] <-> arrays[i]); the copies run on
 * two streams and the call synchronises once.  Layouts COMPACT and
 * REFERENCE_RETAINED (and REFERENCE for set, which reads only the retained
 * block anyway). */
int diablo_set_fields(dg_handle *h, int n, const int *fields, const double *const *src,
                      int layout, int where);
int diablo_get_fields(dg_handle *h, int n, const int *fields, double *const *dst, int layout,
                      int where);

/* ------------------------------------------------------- channel hot path */
/* SUBROUTINE RK_CHAN_1 (for/channel.f:62-1073): one RK3 substep on the
 * device-resident state.  time_step/rk_step are COMMON /RUNTIME_VARS/. */
int diablo_rk_chan_1(dg_handle *h, int time_step, int rk_step);
/* LES (dg_params.les = 1, LES_MODEL_TYPE 1): RK_CHAN_1 then also runs
 * les_chan (for/les.f:1-275) and the eddy-viscosity Crank-Nicolson solves on
 * physical columns (for/channel.f:299-372,631-659,748-1029).  NU_T at GY
 * points (COMMON NU_T, for/header:166), physical layout [NY+2][NZ][NX]. */
int diablo_les_nu_t(dg_handle *h, double *dst, int where);
/* les_chan's mean_les output (for/les.f:336-510): after a request, the next
 * LES substep (the reference: MOD(TIME_STEP,SAVE_STATS_INT) = 0, RK_STEP = 1)
 * records the plane means NU_T_MEAN and EPS_SGS1_MEAN, rows 0..NY+1 (host
 * arrays of NY+2). */
int diablo_les_stats_request(dg_handle *h);
int diablo_les_stats(dg_handle *h, double *nu_t_mean, double *eps_sgs1_mean);
/* tkebudget_chan_les (for/save_stats.f:887-964), which SAVE_STATS_CHAN calls
 * with LES: applies APPLY_BC_VEL to the state, then epsilon_sgs rows 1..NY
 * (host array of NY+2; sums over each plane, as the reference's). */
int diablo_les_tke(dg_handle *h, double *epsilon_sgs);
/* SUBROUTINE REM_DIV_CHAN (for/channel.f:1103-1214): projects CU1..3, leaves
 * phi in CR1. */
int diablo_rem_div_chan(dg_handle *h);
/* SUBROUTINE POISSON_P_CHAN (for/channel.f:1217-1453): CP from CU1..3, CTH. */
int diablo_poisson_p_chan(dg_handle *h);
/* APPLY_BC_VEL_MPI = APPLY_BC_VEL_LOWER + _UPPER (for/channel.f:2285-2492). */
int diablo_apply_bc_vel(dg_handle *h);
/* SUBROUTINE COURANT (for/courant.f:1-65) evaluated on the physical velocity
 * of the current spectral state; updates DELTA_T and H_BAR on the device. */
int diablo_courant(dg_handle *h);

/* FFT_XZ_TO_FOURIER(V,VV,JMIN,JMAX) (for/mpi.f:1530-1611) and
 * FFT_XZ_TO_PHYSICAL(VV,V,JMIN,JMAX) (for/mpi.f:1613-1674), REFERENCE layout.
 * V and VV may alias (the reference passes EQUIVALENCEd arrays).
 * where = DG_HOST or DG_DEVICE for both pointers. */
int diablo_fft_xz_to_fourier(dg_handle *h, const double *V, double *VV, int jmin, int jmax,
                             int where);
int diablo_fft_xz_to_physical(dg_handle *h, const double *VV, double *V, int jmin, int jmax,
                              int where);

/* THOMAS_REAL(A,B,C,G,NY,NX) (for/channel.f:2653-2684) and
 * THOMAS_COMPLEX(A,B,C,G,NY,NX) (for/channel.f:2687-2720): NX+1 independent
 * systems of NY+1 rows, arrays (0:NX,0:NY) first index fastest; A and B are
 * destroyed, the solution is returned in G (complex interleaved for
 * THOMAS_COMPLEX).  where = DG_HOST or DG_DEVICE. */
int diablo_thomas_real(double *A, double *B, double *C, double *G, int ny, int nx, int where);
int diablo_thomas_complex(double *A, double *B, double *C, double *G, int ny, int nx,
                          int where);

/* The driver's time-step loop body (for/diablo.f:70-109) for nsteps steps
 * starting at time_step: RK_CHAN_1 / RK_PER_1 for RK_STEP = 1..3, then
 * TIME = TIME + DELTA_T.  After the first step of a kind, steps replay a
 * captured CUDA graph (one host launch per step); results are identical to
 * calling the substep entry points. */
int diablo_step(dg_handle *h, int time_step, int nsteps);

/* ------------------------------------------------------ periodic hot path */
/* SUBROUTINE RK_PER_1 (for/periodic.f:23-285). */
int diablo_rk_per_1(dg_handle *h, int rk_step);
/* SUBROUTINE REM_DIV_PER (for/periodic.f:299-326). */
int diablo_rem_div_per(dg_handle *h);
/* SUBROUTINE POISSON_P_PER (for/periodic.f:329-393). */
int diablo_poisson_p_per(dg_handle *h);
/* FFT_XZY_TO_FOURIER(U,CU) (for/fft.f:223-258) and FFT_XZY_TO_PHYSICAL(CU,U)
 * (for/fft.f:261-299) on REFERENCE-layout arrays U(0:NX+1,0:NZ+1,0:NY+1) and
 * CU(0:NX/2,0:NZ+1,0:NY+1); retained modes at CU(0:NKX,0:TNKZ,0:TNKY), every
 * other slot of the output zeroed.  U and CU may alias.  where = DG_HOST or
 * DG_DEVICE for both pointers. */
int diablo_fft_xzy_to_fourier(dg_handle *h, const double *U, double *CU, int where);
int diablo_fft_xzy_to_physical(dg_handle *h, const double *CU, double *U, int where);

/* ------------------------------------------------------ kernel timing */
/* No counterpart in the reference (measurement and tuning).  on = 1 clears
 * the totals and brackets every later launch of this handle's kernels with a
 * CUDA event pair on the launch's stream; on = 0 stops recording.
 * dg_timing_read waits for the recorded pairs and returns, for the i-th
 * kernel name seen (0-based), its launch count and total device time. */
int dg_timing_enable(dg_handle *h, int on);
int dg_timing_read(dg_handle *h, int i, char *name, int name_len, int64_t *launches,
                   double *total_ms);

/* -------------------------------------------------------------- tuning */
/* No counterpart in the reference.  Launch shapes of the channel substep:
 * modes per CTA of the REM_DIV y-column kernel (4, 8, 16) and of the substep's
 * column kernel (one field's right-hand side and CN solve; 2, 4, 8, 16),
 * y-planes per CTA of the x-row product kernel (0 = automatic), planes per
 * y-chunk of a substep (0 = all).  Results do not depend on them
 * (DG_TUNE_FFT_PLAN below: at round-off level only).  dg_autotune times
 * candidates on the handle's own state (steps_per_trial eager RK3 steps each), keeps the
 * fastest and restores the state, TIME and DELTA_T; it allocates temporary
 * device copies of the state while it runs. */
enum { DG_TUNE_COL_MT = 0, DG_TUNE_XROW_CHUNK = 1, DG_TUNE_YCHUNK = 2, DG_TUNE_CN_MT = 3,
       DG_TUNE_PDL = 4, DG_TUNE_WAIT_TEST = 5, DG_TUNE_FFT_PLAN = 6, DG_TUNE_PLANE_XZ = 7 };
/* DG_TUNE_PLANE_XZ: 1 (default) moves the LES model's fields between
 * spectral planes and physical rows with one kernel per direction and plane
 * where the x and z lengths allow (16, 32, 48, 64, 96 or 128); 0 stages them
 * through a half-physical array in two launches.  Same transforms, same
 * results; the setting is not tuned. */
/* DG_TUNE_FFT_PLAN: radix order of the x and z transform plans of the
 * substep (0: largest radix first, 128 = 16 x 8; 1: the reverse, 8 x 16).
 * The same transform either way; the autotuner times both per grid shape.
 * Unlike the other tunables it changes the order of the transforms'
 * arithmetic, so results differ between the two at round-off level (both
 * are held to the same parity tolerance). */
/* DG_TUNE_WAIT_TEST (test only): value > 0 makes the next Crank-Nicolson
 * column-kernel launch give up on its bulk-copy barrier after `value` polls, with
 * the barrier expecting 16 bytes more than its copies bring (every copy
 * lands; nothing faults).  The kernel skips its work and the next
 * diablo_synchronize / diablo_stats returns DG_ERR_TIMEOUT once.  The
 * setting clears after that one launch. */
int dg_tune_set(dg_handle *h, int key, int value);
int dg_tune_get(dg_handle *h, int key, int *value);
int dg_autotune(dg_handle *h, int steps_per_trial);
/* The autotuner's choices per grid shape (NX, NY, NZ, N_TH, precision) in a
 * process-wide table (no counterpart in the reference; FFTW_MEASURE planning,
 * for/fft.f:77-94, is the reference's own per-size tuning).  dg_autotune
 * stores its result in it; dg_tune_lookup applies the stored values for h's
 * shape (*hit = 1) or leaves h as it is (*hit = 0); dg_tune_cache_get reads
 * one stored value for a shape (DG_ERR_ARG when absent).  The table persists
 * in a JSON file, {"NXxNYxNZ_thN_fp64|mixed": {"col_mt": .., "xrow_chunk": ..,
 * "ychunk": .., "cn_mt": .., "pdl": .., "fft_plan": ..},
 * ...}: _save writes the whole table, _load merges a file's entries into it. */
int dg_tune_lookup(dg_handle *h, int *hit);
int dg_tune_cache_get(const dg_params *p, int key, int *value);
int dg_tune_cache_save(const char *path);
int dg_tune_cache_load(const char *path);

/* ------------------------------------------- allocation-free transform */
/* No counterpart in the reference.  FFT_XZ_TO_FOURIER(V,VV,JMIN,JMAX) on
 * DEVICE arrays in the reference layout (as diablo_fft_xz_to_fourier with
 * DG_DEVICE), for callers that cannot have device memory allocated for
 * them: it needs no dg_handle and allocates no device memory.  Its only
 * scratch is a fixed DG_NOALLOC_SCRATCH_BYTES array in the library's device
 * image, held by every GPU that loads the library until exit; one NX x NZ
 * plane must fit in it (about 1.75 MB at 512 x 384), otherwise DG_ERR_DIMS.
 * The first call in a CUDA context (per device: its primary context, or
 * another context the caller made current) looks up the array's address
 * (cudaGetSymbolAddress) and keeps it for that context; make that first call
 * before any stream capture.  V and VV must be device or managed memory of
 * the current device (checked with cudaPointerGetAttributes; otherwise
 * DG_ERR_ARG before anything is queued).
 * Work is queued on `stream` (NULL: the default stream) and the call
 * returns without waiting.  All calls share the scratch: calls that overlap
 * on the GPU race.  V and VV may alias. */
#define DG_NOALLOC_SCRATCH_BYTES (16 * 1024 * 1024)
int diablo_fft_xz_to_fourier_noalloc(const double *V, double *VV, int nx, int nz, int ny,
                                     int jmin, int jmax, void *stream);

/* ------------------------------------------------------- ensemble server */
/* No counterpart in the reference (it runs one case per job).  Continuous
 * batching of independent channel solves on one GPU: requests are admitted
 * while fewer than max_active cases run and their device bytes
 * (dg_state_bytes) fit hbm_budget_gb (0 = no budget); each active case has
 * its own handle and stream and advances by replayed step graphs, so steps
 * of different cases overlap on the device; launch shapes are autotuned once
 * per grid shape when autotune != 0.  A request's state is the compact
 * spectral CU1, CU2, CU3, CP, CTH(0..N_TH-1), each
 * [NY+2][TNKZ+1][NKX+1] complex; prepare != 0 applies APPLY_BC_VEL,
 * REM_DIV_CHAN, APPLY_BC_VEL on admission (the tail of CREATE_FLOW_CHAN).
 * dg_server_wait blocks until the request is done, copies its final state
 * into `state` (same layout) and, if times != NULL, stores the seconds spent
 * queued and on the device. */
typedef struct dg_server dg_server;
typedef struct dg_server_stats {
  int64_t cases_done, steps_done;
  int32_t active, queued;
  int64_t bytes_active, bytes_peak;
  double step_ms_p50, step_ms_p99;   /* device time of one RK3 step of a case */
  double cases_per_s, mpoint_steps_per_s, wall_s;  /* first submit .. last completion */
} dg_server_stats;
int64_t dg_state_bytes(const dg_params *p);
int dg_server_create(int max_active, double hbm_budget_gb, int autotune, dg_server **out);
int dg_server_submit(dg_server *s, const dg_params *p, const double *gy,
                     const double *const *state, int nsteps, int prepare, int64_t *id);
int dg_server_wait(dg_server *s, int64_t id, double *const *state, double *times);
int dg_server_query(dg_server *s, dg_server_stats *st);
/* Server options, set before the first dg_server_submit.
 * DG_SERVER_GROUP_CASES = G > 0: cases of similar size step together in
 * groups of up to G, one CUDA graph per group step, with one ragged column
 * launch per substep covering every member's (case, mode tile) work list;
 * 0 (default): every case steps on its own.  Results are the same either
 * way.  LES cases and cases with COURANT at an UPDATE_DT other than 1 always
 * step on their own. */
enum { DG_SERVER_GROUP_CASES = 0 };
int dg_server_config(dg_server *s, int key, int value);
int dg_server_destroy(dg_server *s);

/* ------------------------------------------------------------ flow files */
/* SAVE_FLOW / READ_FLOW without HDF5 (for/diablo_io.f:201-404): Fortran
 * unformatted sequential files (4-byte record markers, little-endian), a
 * header record NX, NY, NZ, NUM_PER_DIR, TIME, TIME_STEP and one record of
 * retained modes.  Channel: CU1 J=1..NY, CU2 J=2..NY, CU3 J=1..NY; each
 * scalar in its own file (fname_th[n], NULL to skip), written J=0..NY and
 * read J=1..NY as the reference does (a file written by SAVE_FLOW comes
 * back one plane lower).  Periodic: all ky planes.  Write uses the handle's
 * TIME; read checks NX, NY, NZ and NUM_PER_DIR (DG_ERR_DIMS with the
 * reference's message), sets TIME, returns TIME_STEP and, for the channel,
 * runs APPLY_BC_VEL.  Records above 2 GiB return DG_ERR_DIMS. */
int diablo_save_flow(dg_handle *h, int time_step, const char *fname, const char *const *fname_th);
int diablo_read_flow(dg_handle *h, const char *fname, const char *const *fname_th,
                     int *time_step);
/* The datasets of the HDF5 flow files (WriteHDF5 / ReadHDF5,
 * for/hdf5.f:5-544), channel only, for a host that writes the file with its
 * own HDF5 library: physical U, V, W, TH(n) and P on planes 1..NY as
 * C arrays [NZ][NY][NX] (Fortran tmp(NX,NY,NZ)), V moved onto GYF by G2GF.
 * Any output may be NULL; TH is [N_TH][NZ][NY][NX].  The reverse (ReadHDF5)
 * applies GF2G to V (walls set for zero mass flux), transforms, sets TIME,
 * runs COURANT when VARIABLE_DT and POISSON_P_CHAN when P is NULL. */
int diablo_flow_fields_physical(dg_handle *h, double *U, double *V, double *W, double *TH,
                                double *P);
int diablo_flow_fields_from_physical(dg_handle *h, const double *U, const double *V,
                                     const double *W, const double *TH, const double *P,
                                     double time);

/* ------------------------------------------------------------ statistics */
/* Parity statistics of the current state (channel or periodic); also checks
 * the state for non-finite values (returns DG_ERR_NAN if any). */
int diablo_stats(dg_handle *h, dg_stats *s);

/* SAVE_STATS_CHAN(FINAL=.FALSE.) (for/save_stats.f:4-31,85-690) with
 * tkebudget_chan (for/save_stats.f:963-1173), channel only.  Runs
 * APPLY_BC_VEL on the state (for/save_stats.f:24-36), then fills, for rows
 * j = 0..NY+1,
 *   prof    [DG_PR_COUNT][NY+2]          the columns of mean.txt and tke.txt
 *   prof_th [N_TH][DG_PRT_COUNT][NY+2]   the columns of mean_th.txt (may be
 *                                        NULL when N_TH = 0)
 *   bulk    [5] = UBULK, centreline U1, <urms>, <vrms>, <wrms>
 * Rows 1..NY carry what the reference writes; EPSILON rows 2..NY-1
 * (tke.txt); the means (UME, VME, WME, CP, THME) also rows 0 and NY+1.
 * VME is on GY (mean.txt prints 0.5 (VME(j) + VME(j+1))).  Also advances
 * NSAMPLES and the running means UBAR, VBAR, WBAR, THBAR
 * (for/save_stats.f:99-114).  Replaces the reference's transforms with the
 * discrete Parseval identity on the retained modes; the spectral state is
 * left as it was (the reference's physical round trip changes it only by
 * round-off). */
enum {
  DG_PR_UME = 0, DG_PR_VME, DG_PR_WME, DG_PR_URMS, DG_PR_VRMS, DG_PR_WRMS, DG_PR_UV, DG_PR_UW,
  DG_PR_WV, DG_PR_DUDY, DG_PR_DWDY, DG_PR_CP, DG_PR_SHEAR, DG_PR_OMEGA_X, DG_PR_OMEGA_Y,
  DG_PR_OMEGA_Z, DG_PR_EPSILON, DG_PR_COUNT
};
enum { DG_PRT_THME = 0, DG_PRT_DTHDY, DG_PRT_THRMS, DG_PRT_THV, DG_PRT_PE_DISS, DG_PRT_COUNT };
int diablo_save_stats_chan(dg_handle *h, double *prof, double *prof_th, double *bulk);
/* SAVE_STATS_CHAN's running means, rows 0..NY+1 (rows 1..NY updated):
 * ubar, vbar, wbar [NY+2], thbar [N_TH][NY+2] (may be NULL); *nsamples =
 * NSAMPLES.  What SAVE_STATS_CHAN(FINAL=.TRUE.) writes to stats.txt. */
int diablo_stats_means(dg_handle *h, double *ubar, double *vbar, double *wbar, double *thbar,
                       int *nsamples);

#ifdef __cplusplus
}
#endif
#endif
