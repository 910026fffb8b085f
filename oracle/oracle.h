/*
 * CPU oracle for the DIABLO channel / triply periodic RK3 substeps.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C FP64 restatement of the
 * reference Fortran (johnryantaylor/DIABLO, diablo_2.0/for, Fortran sources) used by the
 * parity tests, by __graft_entry__.smoke() as the checker and by bench.py's
 * CPU-baseline leg.  No product code path may call it.
 *
 * Parity status: the reference ships no tests, golden vectors or runnable
 * build (no Fortran compiler, MPI, FFTW 2.1.5 or HDF5 here), so this oracle
 * is "parity unpinned" against the reference binary.  It is pinned instead
 * against numpy.fft (FFT conventions), dense linear solves (Thomas), exact
 * analytic solutions (Fourier-mode decay, laminar channel steady states)
 * and the divergence-free constraint; see tests/test_oracle.py.
 *
 * Layouts (all row-major, last index fastest):
 *   spectral field  : complex  [NY+2][TNKZ+1][NKX+1]     (retained modes only)
 *   physical field  : double   [NY+2][NZ][NX]
 * Retained modes follow the reference packing (for/fft.f:8-50,
 * for/mpi.f:1530-1611): kx = 0..NKX, kz = 0..NKZ then -NKZ..-1 stored at
 * NKZ+1..TNKZ.  The reference also stores kx = NKX+1..NX/2-1 but keeps them
 * identically zero on the channel path, so they are omitted here.
 */
#ifndef DIABLO_ORACLE_H
#define DIABLO_ORACLE_H

#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_TH 4

typedef struct orc_params {
  int nx, ny, nz, n_th;
  int num_per_dir;            /* 2 = channel, 3 = triply periodic */
  double nu, beta, lx, ly, lz, nu_v_scale;
  double delta_t, cfl;
  int variable_dt, update_dt;
  double i_ro, grav_x, grav_y, grav_z;
  int f_type;
  double ubulk0, px0, omega0, amp_omega0;
  int u_bc_ymin, v_bc_ymin, w_bc_ymin, u_bc_ymax, v_bc_ymax, w_bc_ymax;
  double u_bc_ymin_c1, v_bc_ymin_c1, w_bc_ymin_c1;
  double u_bc_ymax_c1, v_bc_ymax_c1, w_bc_ymax_c1;
  int th_bc_ymin[ORC_MAX_TH], th_bc_ymax[ORC_MAX_TH];
  double th_bc_ymin_c1[ORC_MAX_TH], th_bc_ymax_c1[ORC_MAX_TH];
  double ri[ORC_MAX_TH], pr[ORC_MAX_TH];
  double drhodx[ORC_MAX_TH], drhodz[ORC_MAX_TH];
  int background_grad[ORC_MAX_TH];
  double epsilon_target;      /* periodic linear forcing (user_rhs.f:124) */
  int les;                    /* USE_LES (input.dat, for/diablo_io.f:25) */
  int les_model_type;         /* input_chan.dat (for/channel.f:1477); only 1 runs */
  int create_new_flow;        /* input.dat (for/diablo_io.f:31): LES waits 100 steps */
} orc_params;

typedef struct orc orc;

typedef enum {
  ORC_CU1 = 0, ORC_CU2, ORC_CU3, ORC_CP, ORC_CF1, ORC_CF2, ORC_CF3, ORC_CR1,
  ORC_CTH = 16, ORC_CFTH = 32
} orc_field;

/* lifecycle; gy = GY(1..NY+1) (channel) or NULL (periodic) */
orc *orc_create(const orc_params *p, const double *gy);
void orc_destroy(orc *o);
void orc_set_threads(int n);

/* dims */
int orc_nkx(const orc *o);
int orc_tnkz(const orc *o);
int orc_tnky(const orc *o);
long orc_spec_size(const orc *o);   /* complex elements per spectral field */
long orc_phys_size(const orc *o);   /* doubles per physical field */

/* grid tables (NY+2 doubles each) */
void orc_get_grid(const orc *o, double *gy, double *gyf, double *dy, double *dyf);

/* field access (compact layouts above); field ids orc_field, +n for scalar n */
int orc_get_field(const orc *o, int id, double complex *out);
int orc_set_field(orc *o, int id, const double complex *in);

/* scalars */
void orc_set_time(orc *o, double time, double delta_t);
void orc_get_time(const orc *o, double *time, double *delta_t);

/* ---- transforms (for/mpi.f:1530-1674, for/fft.f:223-299) ---- */
void orc_fft_xz_to_fourier(const orc *o, const double *phys, double complex *spec,
                           int jmin, int jmax);
void orc_fft_xz_to_physical(const orc *o, const double complex *spec, double *phys,
                            int jmin, int jmax);
void orc_fft_xzy_to_fourier(const orc *o, const double *phys, double complex *spec);
void orc_fft_xzy_to_physical(const orc *o, const double complex *spec, double *phys);

/* generic 1-D complex FFT, unnormalised, sign -1 forward / +1 inverse */
void orc_fft1d(int n, double complex *data, int sign);

/* ---- tridiagonal solvers (for/channel.f:2653-2720) ---- */
void orc_thomas_real(double *a, double *b, double *c, double *g, int ny, int nx);
void orc_thomas_complex(double *a, double *b, double *c, double complex *g, int ny, int nx);

/* ---- channel (for/channel.f) ---- */
void orc_rk_chan_1(orc *o, int time_step, int rk_step);
void orc_rem_div_chan(orc *o);
void orc_poisson_p_chan(orc *o);
void orc_apply_bc_vel(orc *o);
void orc_create_flow_chan(orc *o, const double *u1, const double *u2, const double *u3,
                          const double *th);
void orc_courant(orc *o);             /* on the physical U1..U3 currently held */

/* ---- periodic (for/periodic.f) ---- */
void orc_rk_per_1(orc *o, int rk_step);
void orc_rem_div_per(orc *o);
void orc_poisson_p_per(orc *o);
void orc_create_flow_per(orc *o, const double *u1, const double *u2, const double *u3);

/* ---- diagnostics ---- */
typedef struct orc_stats {
  double ubulk, urms_b, vrms_b, wrms_b, ke, div_max;
  double thrms_b[ORC_MAX_TH], th_var[ORC_MAX_TH];
} orc_stats;
void orc_stats_chan(const orc *o, orc_stats *s);
void orc_stats_per(const orc *o, orc_stats *s);
double orc_div_max_chan(const orc *o);

/* SAVE_STATS_CHAN (for/save_stats.f:4-690) and tkebudget_chan
 * (for/save_stats.f:963-1173) profiles, rows j = 0..NY+1 of each:
 * prof [ORC_PR_COUNT][NY+2], prof_th [N_TH][ORC_PRT_COUNT][NY+2],
 * bulk = {UBULK, centreline U, <urms>, <vrms>, <wrms>}.  Rows 1..NY hold
 * the values the reference writes (mean.txt, mean_th.txt); EPSILON rows
 * 2..NY-1 (tke.txt); the means also rows 0 and NY+1. */
enum {
  ORC_PR_UME, ORC_PR_VME, ORC_PR_WME, ORC_PR_URMS, ORC_PR_VRMS, ORC_PR_WRMS, ORC_PR_UV,
  ORC_PR_UW, ORC_PR_WV, ORC_PR_DUDY, ORC_PR_DWDY, ORC_PR_CP, ORC_PR_SHEAR, ORC_PR_OMEGA_X,
  ORC_PR_OMEGA_Y, ORC_PR_OMEGA_Z, ORC_PR_EPSILON, ORC_PR_COUNT
};
enum { ORC_PRT_THME, ORC_PRT_DTHDY, ORC_PRT_THRMS, ORC_PRT_THV, ORC_PRT_PE_DISS, ORC_PRT_COUNT };
void orc_save_stats_chan(orc *o, double *prof, double *prof_th, double *bulk);
void orc_stats_means_update(const orc *o, int nsamples, double *ubar, double *vbar,
                            double *wbar, double *thbar);
double orc_div_max_per(const orc *o);
/* NU_T of the last LES substep, physical layout; -1 without LES */
int orc_get_nu_t(const orc *o, double *out);
/* les_chan's plane means (for/les.f:336-459): the next LES substep records
 * NU_T_MEAN and EPS_SGS1_MEAN (rows 0..NY+1) as it does when
 * MOD(TIME_STEP, SAVE_STATS_INT) = 0 and RK_STEP = 1. */
void orc_les_stats_request(orc *o);
int orc_les_stats(const orc *o, double *nu_t_mean, double *eps_sgs1_mean);
/* tkebudget_chan_les: epsilon_sgs rows 1..NY (sums over the plane); applies
 * APPLY_BC_VEL to the state as SAVE_STATS_CHAN does first. */
void orc_tkebudget_chan_les(orc *o, double *epsilon_sgs);

#ifdef __cplusplus
}
#endif
#endif
