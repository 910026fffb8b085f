/*
 * Oracle restatement of the channel-flow RK3/Crank-Nicolson substep and its
 * helpers.  TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Follows the NPROCS = 1 MPI build of the reference (USE_MPI = .TRUE.,
 * NPROCY = NPROCZ = 1): that is the configuration `mpirun -np 1` runs; the
 * serial stub library cannot link (for/dummy_code/mpi_serial.f lacks
 * FFT_XZ_*).  Consequences restated here:
 *   - JSTART = 2 and JEND = NY whatever the BC (for/mpi.f:1080-1100, the
 *     RANKY = 0 branch wins because RANKY = 0 = NPROCY-1);
 *   - JSTART_TH = 2 (Dirichlet) or 1 (Neumann), JEND_TH = NY;
 *   - both lower and upper BCs are applied (for/mpi.f:1137-1299);
 *   - Thomas solves use the MPI sweeps (for/mpi.f:630-866), including the
 *     zero-pivot guards of the complex and backward-real variants;
 *   - the pressure-Poisson BCs are APPLY_BC_REM_DIV_MPI / APPLY_BC_POISSON_MPI
 *     (for/mpi.f:1293-1369).
 * Spectral loops of the reference run over I = 0..NXP-1; modes NKX < I < NXP
 * are identically zero on this path and are not stored.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle_int.h"

#ifdef _OPENMP
#include <omp.h>
#endif

#define SIDX(o, j, k, i) ((long)(j) * (o)->ss + (long)(k) * (o)->nkxp + (i))
#define PIDX(o, j, k, i) ((long)(j) * (o)->NZ * (o)->NX + (long)(k) * (o)->NX + (i))

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

static void *zalloc(long n, long sz) { return calloc((size_t)(n > 0 ? n : 1), (size_t)sz); }

/* ------------------------------------------------------------------ setup */
orc *orc_create(const orc_params *p, const double *gy) {
  /* LES_MODEL_TYPE 2 and 3 stop the MPI build (for/les.f:269-272) */
  if (p->les && p->num_per_dir == 2 && p->les_model_type != 1) return NULL;
  orc *o = (orc *)calloc(1, sizeof(orc));
  o->p = *p;
  o->NX = p->nx;
  o->NY = p->ny;
  o->NZ = p->nz;
  o->NTH = p->n_th;
  o->NXP = p->nx / 2;
  o->NKX = p->nx / 3;
  o->NKZ = p->nz / 3;
  o->TNKZ = 2 * o->NKZ;
  o->NKY = p->ny / 3;
  o->TNKY = 2 * o->NKY;
  o->nkxp = o->NKX + 1;
  o->nkzt = o->TNKZ + 1;
  o->nkyt = o->TNKY + 1;
  o->ss = (long)o->nkxp * o->nkzt;
  o->pi = 4.0 * atan(1.0);
  const double pi = o->pi;
  const int per = (p->num_per_dir == 3);
  o->nspec = per ? o->ss * o->nkyt : o->ss * (o->NY + 2);
  o->nphys = per ? (long)o->NY * o->NZ * o->NX : (long)(o->NY + 2) * o->NZ * o->NX;
  /* EPS = 0.000000001 is a default-real literal (for/fft.f:74) */
  o->eps = (double)(float)0.000000001;

  /* wavenumbers (for/fft.f:82-129) */
  o->KX = zalloc(o->nkxp, sizeof(double));
  o->KX2 = zalloc(o->nkxp, sizeof(double));
  o->CIKX = zalloc(o->nkxp, sizeof(cplx));
  for (int i = 0; i <= o->NKX; i++) {
    o->KX[i] = (double)i * (2.0 * pi) / p->lx;
    o->KX2[i] = o->KX[i] * o->KX[i];
    o->CIKX[i] = I * o->KX[i];
  }
  o->KZ = zalloc(o->nkzt, sizeof(double));
  o->KZ2 = zalloc(o->nkzt, sizeof(double));
  o->CIKZ = zalloc(o->nkzt, sizeof(cplx));
  for (int k = 0; k <= o->NKZ; k++) o->KZ[k] = (double)k * (2.0 * pi) / p->lz;
  for (int k = 1; k <= o->NKZ; k++) o->KZ[o->TNKZ + 1 - k] = -((double)k * (2.0 * pi) / p->lz);
  for (int k = 0; k <= o->TNKZ; k++) {
    o->KZ2[k] = o->KZ[k] * o->KZ[k];
    o->CIKZ[k] = I * o->KZ[k];
  }
  o->KY = zalloc(o->nkyt, sizeof(double));
  o->KY2 = zalloc(o->nkyt, sizeof(double));
  o->CIKY = zalloc(o->nkyt, sizeof(cplx));
  if (per) {
    for (int j = 1; j <= o->NKY; j++) o->KY[j] = (double)j * (2.0 * pi) / p->ly;
    for (int j = 1; j <= o->NKY; j++) o->KY[o->TNKY + 1 - j] = -((double)j * (2.0 * pi) / p->ly);
    for (int j = 0; j <= o->TNKY; j++) {
      o->KY2[j] = o->KY[j] * o->KY[j];
      o->CIKY[j] = I * o->KY[j];
    }
  }

  /* grid */
  o->GY = zalloc(o->NY + 2, sizeof(double));
  o->GYF = zalloc(o->NY + 2, sizeof(double));
  o->DY = zalloc(o->NY + 2, sizeof(double));
  o->DYF = zalloc(o->NY + 2, sizeof(double));
  o->DX = p->lx / o->NX;
  o->DZ = p->lz / o->NZ;
  const int NY = o->NY;
  if (!per && gy) {
    /* ReadGridHDF5 (for/hdf5.f:676-703) + metrics (for/channel.f:1646-1652) */
    for (int j = 1; j <= NY + 1; j++) o->GY[j] = gy[j - 1];
    for (int j = 1; j <= NY; j++) o->GYF[j] = 0.5 * (o->GY[j] + o->GY[j + 1]);
    o->GYF[0] = 2.0 * o->GYF[1] - o->GYF[2];
    o->GYF[NY + 1] = 2.0 * o->GYF[NY] - o->GYF[NY - 1];
    for (int j = 1; j <= NY + 1; j++) o->DY[j] = o->GYF[j] - o->GYF[j - 1];
    for (int j = 1; j <= NY; j++) o->DYF[j] = o->GY[j + 1] - o->GY[j];
    o->DYF[NY + 1] = o->DYF[NY];
  } else if (per) {
    /* CREATE_GRID_PER (for/periodic.f:415-419) */
    for (int j = 0; j <= NY; j++) {
      o->GY[j] = (j * p->ly) / NY;
      o->DY[j] = p->ly / NY;
    }
  }

  /* RK3 coefficients (for/diablo_io.f:116-124) */
  orc_set_time(o, 0.0, p->delta_t);
  o->beta_bar[0] = 1.0;
  o->beta_bar[1] = 25.0 / 8.0;
  o->beta_bar[2] = 9.0 / 4.0;
  o->zeta_bar[0] = 0.0;
  o->zeta_bar[1] = -17.0 / 8.0;
  o->zeta_bar[2] = -5.0 / 4.0;

  /* INIT_CHAN_MPI with NPROCY = 1 (for/mpi.f:1080-1100) */
  o->jstart = 2;
  o->jend = NY;
  for (int n = 0; n < o->NTH; n++) {
    o->jend_th[n] = NY;
    o->jstart_th[n] = (p->th_bc_ymin[n] == 1) ? 1 : 2;
  }

  const long ns = o->nspec, np = o->nphys;
  cplx **cf[] = {&o->CU1, &o->CU2, &o->CU3, &o->CP, &o->CF1, &o->CF2, &o->CF3,
                 &o->CR1, &o->CR2, &o->CR3, &o->CS1};
  for (unsigned i = 0; i < sizeof(cf) / sizeof(cf[0]); i++) *cf[i] = zalloc(ns, sizeof(cplx));
  double **pf[] = {&o->U1, &o->U2, &o->U3, &o->R1, &o->R2, &o->R3, &o->S1, &o->F1, &o->F2, &o->F3};
  for (unsigned i = 0; i < sizeof(pf) / sizeof(pf[0]); i++) *pf[i] = zalloc(np, sizeof(double));
  for (int n = 0; n < o->NTH; n++) {
    o->CTH[n] = zalloc(ns, sizeof(cplx));
    o->CFTH[n] = zalloc(ns, sizeof(cplx));
    o->CRTH[n] = zalloc(ns, sizeof(cplx));
    o->TH[n] = zalloc(np, sizeof(double));
    o->RTH[n] = zalloc(np, sizeof(double));
  }
  if (p->les && !per) {
    o->NU_T = zalloc(np, sizeof(double));
    o->TEMP = zalloc(np, sizeof(double));
    o->CTEMP = zalloc(ns, sizeof(cplx));
    o->nu_t_mean = zalloc(o->NY + 2, sizeof(double));
    o->eps_sgs1_mean = zalloc(o->NY + 2, sizeof(double));
    for (int c = 0; c < 6; c++) {
      o->Sij[c] = zalloc(np, sizeof(double));
      o->CSij[c] = zalloc(ns, sizeof(cplx));
    }
  }
  return o;
}

void orc_destroy(orc *o) {
  if (!o) return;
  void *ptrs[] = {o->KX, o->KX2, o->CIKX, o->KZ, o->KZ2, o->CIKZ, o->KY, o->KY2, o->CIKY,
                  o->GY, o->GYF, o->DY, o->DYF, o->CU1, o->CU2, o->CU3, o->CP, o->CF1,
                  o->CF2, o->CF3, o->CR1, o->CR2, o->CR3, o->CS1, o->U1, o->U2, o->U3,
                  o->R1, o->R2, o->R3, o->S1, o->F1, o->F2, o->F3};
  for (unsigned i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
  for (int n = 0; n < o->NTH; n++) {
    free(o->CTH[n]);
    free(o->CFTH[n]);
    free(o->CRTH[n]);
    free(o->TH[n]);
    free(o->RTH[n]);
  }
  free(o->NU_T);
  free(o->TEMP);
  free(o->CTEMP);
  free(o->nu_t_mean);
  free(o->eps_sgs1_mean);
  for (int c = 0; c < 6; c++) {
    free(o->Sij[c]);
    free(o->CSij[c]);
  }
  free(o);
}

int orc_nkx(const orc *o) { return o->NKX; }
int orc_tnkz(const orc *o) { return o->TNKZ; }
int orc_tnky(const orc *o) { return o->TNKY; }
long orc_spec_size(const orc *o) { return o->nspec; }
long orc_phys_size(const orc *o) { return o->nphys; }

void orc_get_grid(const orc *o, double *gy, double *gyf, double *dy, double *dyf) {
  size_t n = sizeof(double) * (o->NY + 2);
  if (gy) memcpy(gy, o->GY, n);
  if (gyf) memcpy(gyf, o->GYF, n);
  if (dy) memcpy(dy, o->DY, n);
  if (dyf) memcpy(dyf, o->DYF, n);
}

static cplx *field_ptr(const orc *o, int id) {
  if (id >= ORC_CFTH && id < ORC_CFTH + o->NTH) return o->CFTH[id - ORC_CFTH];
  if (id >= ORC_CTH && id < ORC_CTH + o->NTH) return o->CTH[id - ORC_CTH];
  switch (id) {
    case ORC_CU1: return o->CU1;
    case ORC_CU2: return o->CU2;
    case ORC_CU3: return o->CU3;
    case ORC_CP: return o->CP;
    case ORC_CF1: return o->CF1;
    case ORC_CF2: return o->CF2;
    case ORC_CF3: return o->CF3;
    case ORC_CR1: return o->CR1;
    default: return NULL;
  }
}

int orc_get_field(const orc *o, int id, cplx *out) {
  cplx *f = field_ptr(o, id);
  if (!f) return -1;
  memcpy(out, f, sizeof(cplx) * o->nspec);
  return 0;
}

int orc_set_field(orc *o, int id, const cplx *in) {
  cplx *f = field_ptr(o, id);
  if (!f) return -1;
  memcpy(f, in, sizeof(cplx) * o->nspec);
  return 0;
}

void orc_set_time(orc *o, double time, double delta_t) {
  o->time = time;
  o->delta_t = delta_t;
  o->h_bar[0] = delta_t * (8.0 / 15.0);
  o->h_bar[1] = delta_t * (2.0 / 15.0);
  o->h_bar[2] = delta_t * (5.0 / 15.0);
}

void orc_get_time(const orc *o, double *time, double *delta_t) {
  if (time) *time = o->time;
  if (delta_t) *delta_t = o->delta_t;
}

/* ------------------------------------------------------------ Thomas */
/* THOMAS_REAL(A,B,C,G,NY,NX), for/channel.f:2653-2684: A..G(0:NX,0:NY),
 * first index fastest. */
void orc_thomas_real(double *A, double *B, double *C, double *G, int ny, int nx) {
  const int ld = nx + 1;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i <= nx; i++) {
      long c = (long)(j + 1) * ld + i, p = (long)j * ld + i;
      A[c] = -A[c] / B[p];
      B[c] = B[c] + A[c] * C[p];
      G[c] = G[c] + A[c] * G[p];
    }
  for (int i = 0; i <= nx; i++) G[(long)ny * ld + i] = G[(long)ny * ld + i] / B[(long)ny * ld + i];
  for (int j = ny - 1; j >= 0; j--)
    for (int i = 0; i <= nx; i++) {
      long c = (long)j * ld + i;
      G[c] = (G[c] - C[c] * G[c + ld]) / B[c];
    }
}

/* THOMAS_COMPLEX(A,B,C,G,NY,NX), for/channel.f:2687-2720 */
void orc_thomas_complex(double *A, double *B, double *C, cplx *G, int ny, int nx) {
  const int ld = nx + 1;
  for (int j = 0; j < ny; j++)
    for (int i = 0; i <= nx; i++) {
      long c = (long)(j + 1) * ld + i, p = (long)j * ld + i;
      A[c] = -A[c] / B[p];
      B[c] = B[c] + A[c] * C[p];
      G[c] = G[c] + A[c] * G[p];
    }
  for (int i = 0; i <= nx; i++) G[(long)ny * ld + i] = G[(long)ny * ld + i] / B[(long)ny * ld + i];
  for (int i = 0; i <= nx; i++)
    for (int j = ny - 1; j >= 0; j--) {
      long c = (long)j * ld + i;
      G[c] = (G[c] - C[c] * G[c + ld]) / B[c];
    }
}

/* THOMAS_FORWARD_REAL_MPI + THOMAS_BACKWARD_REAL_MPI for the only rank
 * (RANKY = 0 = NPROCY-1), for/mpi.f:630-703,767-809.  Arrays (0:INX-1,0:INY+1). */
static void thomas_real_mpi(double *A, double *B, double *C, double *G, int iny, int inx) {
  for (int j = 1; j <= iny + 1; j++)
    for (int i = 0; i < inx; i++) {
      long c = (long)j * inx + i, p = c - inx;
      A[c] = -A[c] / B[p];
      B[c] = B[c] + A[c] * C[p];
      G[c] = G[c] + A[c] * G[p];
    }
  for (int i = 0; i < inx; i++) {
    long t = (long)(iny + 1) * inx + i;
    G[t] = G[t] / B[t];
    for (int j = iny; j >= 0; j--) {
      long c = (long)j * inx + i;
      if (B[c] != 0.0)
        G[c] = (G[c] - C[c] * G[c + inx]) / B[c];
      else
        G[c] = 0.0;
    }
  }
}

/* THOMAS_FORWARD_COMPLEX_MPI + THOMAS_BACKWARD_COMPLEX_MPI for the only
 * rank, for/mpi.f:708-764,812-865.  Columns i = 0..ncol-1, rows 1..iny. */
static void thomas_complex_mpi(double *A, double *B, double *C, cplx *G, int iny, int ld,
                               int ncol) {
  for (int i = 0; i < ncol; i++) {
    for (int j = 2; j <= iny; j++) {
      long c = (long)j * ld + i, p = c - ld;
      if (B[p] != 0.0)
        A[c] = -A[c] / B[p];
      else
        A[c] = 0.0;
      B[c] = B[c] + A[c] * C[p];
      G[c] = G[c] + A[c] * G[p];
    }
    long t = (long)iny * ld + i;
    if (B[t] != 0.0)
      G[t] = G[t] / B[t];
    else
      G[t] = 0.0;
    for (int j = iny - 1; j >= 1; j--) {
      long c = (long)j * ld + i;
      if (B[c] != 0.0)
        G[c] = (G[c] - C[c] * G[c + ld]) / B[c];
      else
        G[c] = 0.0;
    }
  }
}

/* --------------------------------------------------- BC rows (physical) */
typedef struct {
  double *L, *D, *U, *V;
  int nx;
} rowset;

static void set_row(rowset *m, int j, double l, double d, double u, double v) {
  for (int i = 0; i < m->nx; i++) {
    long c = (long)j * m->nx + i;
    m->L[c] = l;
    m->D[c] = d;
    m->U[c] = u;
    m->V[c] = v;
  }
}

/* APPLY_BC_1/3/TH_LOWER/UPPER share one form (for/channel.f:1660-1697,
 * 1741-1778, 1967-2004, 2047-2084, 2128-2163, 2205-2241). */
static void bc_gyf_lower(rowset *m, int type, double c1, const orc *o) {
  if (type == 0) {
    set_row(m, 0, 0.0, 1.0, 0.0, 0.0);
    set_row(m, 1, 0.0, 1.0, 0.0, c1);
  } else {
    set_row(m, 0, 0.0, 1.0, 0.0, 0.0);
    set_row(m, 1, 0.0, -1.0, 1.0, o->DY[2] * c1);
  }
}

static void bc_gyf_upper(rowset *m, int type, double c1, const orc *o) {
  const int NY = o->NY;
  if (type == 0) {
    set_row(m, NY + 1, 0.0, 1.0, 0.0, 0.0);
    set_row(m, NY, 0.0, 1.0, 0.0, c1);
  } else {
    set_row(m, NY, -1.0, 1.0, 0.0, o->DY[NY] * c1);
    set_row(m, NY + 1, 0.0, 1.0, 0.0, 0.0);
  }
}

/* APPLY_BC_2_LOWER/UPPER (for/channel.f:1822-1860, 1905-1933) */
static void bc_gy_lower(rowset *m, int type, double c1, const orc *o) {
  if (type == 0) {
    set_row(m, 1, 0.0, 1.0, 0.0, c1);
    set_row(m, 2, 0.0, 1.0, 0.0, c1);
  } else if (type == 1) {
    set_row(m, 1, 0.0, -1.0, 1.0, o->DYF[1] * c1);
  }
  set_row(m, 0, 0.0, 1.0, 0.0, 0.0);
}

static void bc_gy_upper(rowset *m, int type, double c1, const orc *o) {
  const int NY = o->NY;
  if (type == 0) {
    set_row(m, NY + 1, 0.0, 1.0, 0.0, c1);
    set_row(m, NY, 0.0, 1.0, 0.0, c1);
  } else if (type == 1) {
    set_row(m, NY + 1, -1.0, 1.0, 0.0, o->DYF[NY] * c1);
  }
}

/* ------------------------------------------- APPLY_BC_VEL_LOWER/UPPER */
/* for/channel.f:2285-2492, Fourier space, (0,0) mode = index 0 */
void orc_apply_bc_vel(orc *o) {
  const orc_params *p = &o->p;
  const int NY = o->NY;
  const long ss = o->ss;
  cplx *U1 = o->CU1, *U2 = o->CU2, *U3 = o->CU3;
  /* lower */
  if (p->u_bc_ymin == 0) {
    for (long m = 0; m < ss; m++) U1[m] = U1[ss + m] = 0.0;
    U1[ss] = p->u_bc_ymin_c1;
    U1[0] = p->u_bc_ymin_c1;
  } else {
    for (long m = 0; m < ss; m++) {
      U1[ss + m] = U1[2 * ss + m];
      U1[m] = U1[ss + m];
    }
    U1[ss] = U1[2 * ss] - o->DY[2] * p->u_bc_ymin_c1;
    U1[0] = U1[ss] - o->DY[1] * p->u_bc_ymin_c1;
  }
  if (p->w_bc_ymin == 0) {
    for (long m = 0; m < ss; m++) U3[m] = U3[ss + m] = 0.0;
    U3[ss] = p->w_bc_ymin_c1;
    U3[0] = p->w_bc_ymin_c1;
  } else {
    for (long m = 0; m < ss; m++) {
      U3[ss + m] = U3[2 * ss + m];
      U3[m] = U3[ss + m];
    }
    U3[ss] = U3[2 * ss] - o->DY[2] * p->w_bc_ymin_c1;
    U3[0] = U3[ss] - o->DY[1] * p->w_bc_ymin_c1;
  }
  if (p->v_bc_ymin == 0) {
    for (long m = 0; m < ss; m++) {
      U2[ss + m] = 2.0 * p->v_bc_ymin_c1 - U2[2 * ss + m];
      U2[m] = U2[ss + m];
    }
  } else if (p->v_bc_ymin == 1) {
    for (long m = 0; m < ss; m++) {
      U2[ss + m] = U2[2 * ss + m];
      U2[m] = U2[ss + m];
    }
    U2[ss] = U2[2 * ss] - o->DYF[1] * p->v_bc_ymin_c1;
    U2[0] = U2[ss] - o->DYF[1] * p->v_bc_ymin_c1;
  } else if (p->v_bc_ymin == 2) {
    U2[ss] = -U2[2 * ss];
  }
  /* upper */
  const long jn = (long)NY * ss, jn1 = (long)(NY + 1) * ss, jm = (long)(NY - 1) * ss;
  if (p->u_bc_ymax == 0) {
    for (long m = 0; m < ss; m++) U1[jn + m] = U1[jn1 + m] = 0.0;
    U1[jn] = p->u_bc_ymax_c1;
    U1[jn1] = p->u_bc_ymax_c1;
  } else {
    for (long m = 0; m < ss; m++) {
      U1[jn + m] = U1[jm + m];
      U1[jn1 + m] = U1[jn + m];
    }
    U1[jn] = U1[jm] + o->DY[NY] * p->u_bc_ymax_c1;
    U1[jn1] = U1[jn] + o->DY[NY] * p->u_bc_ymax_c1;
  }
  if (p->w_bc_ymax == 0) {
    for (long m = 0; m < ss; m++) U3[jn + m] = U3[jn1 + m] = 0.0;
    U3[jn] = p->w_bc_ymax_c1;
    U3[jn1] = p->w_bc_ymax_c1;
    U3[jn1] = 0.0; /* "Ghost cell not used", for/channel.f:2445 */
  } else {
    for (long m = 0; m < ss; m++) {
      U3[jn + m] = U3[jm + m];
      U3[jn1 + m] = U3[jn + m];
    }
    U3[jn] = U3[jm] + o->DY[NY] * p->w_bc_ymax_c1;
    U3[jn1] = U3[jn] + o->DY[NY] * p->w_bc_ymax_c1;
  }
  if (p->v_bc_ymax == 0) {
    /* only the (0,0) mode is written (for/channel.f:2466-2470) */
    U2[jn1] = 2.0 * p->v_bc_ymax_c1 - U2[jn];
  } else if (p->v_bc_ymax == 1) {
    for (long m = 0; m < ss; m++) {
      U2[jn + m] = U2[jm + m];
      U2[jn1 + m] = U2[jn + m];
    }
    U2[jn1] = U2[jn] + o->DY[NY] * p->v_bc_ymax_c1;
  } else if (p->v_bc_ymax == 2) {
    U2[jn1] = -U2[jn];
  }
}

/* ---------------------------------------------------------- REM_DIV_CHAN */
/* for/channel.f:1103-1214 with APPLY_BC_REM_DIV_MPI (for/mpi.f:1293-1332) and
 * the MPI complex Thomas sweeps.  phi is left in CR1 (rows 1..NY). */
void orc_rem_div_chan(orc *o) {
  const int NY = o->NY, nkxp = o->nkxp;
  const double *DY = o->DY, *DYF = o->DYF;
#pragma omp parallel
  {
    const long n = (long)nkxp * (NY + 2);
    double *L = malloc(sizeof(double) * n), *D = malloc(sizeof(double) * n),
           *U = malloc(sizeof(double) * n);
    cplx *V = malloc(sizeof(cplx) * n);
#pragma omp for schedule(static)
    for (int k = 0; k <= o->TNKZ; k++) {
      for (long c = 0; c < n; c++) {
        L[c] = 0.0;
        D[c] = 1.0;
        U[c] = 0.0;
        V[c] = 0.0;
      }
      for (int j = 1; j <= NY; j++)
        for (int i = 0; i < nkxp; i++) {
          long c = (long)j * nkxp + i;
          L[c] = 1. / (DY[j] * DYF[j]);
          D[c] = -o->KX2[i] - o->KZ2[k] - 1. / (DY[j + 1] * DYF[j]) - 1. / (DY[j] * DYF[j]);
          U[c] = 1. / (DY[j + 1] * DYF[j]);
        }
      for (int j = 1; j <= NY; j++)
        for (int i = 0; i < nkxp; i++)
          V[(long)j * nkxp + i] =
              (o->CIKX[i] * o->CU1[SIDX(o, j, k, i)] +
               (o->CU2[SIDX(o, j + 1, k, i)] - o->CU2[SIDX(o, j, k, i)]) / DYF[j] +
               o->CIKZ[k] * o->CU3[SIDX(o, j, k, i)]);
      for (int i = 0; i < nkxp; i++) {
        long c = nkxp + i;
        if (k == 0 && i == 0) {
          L[c] = 0.;
          D[c] = 1.;
          U[c] = 0.;
          V[c] = 0.;
        } else {
          L[c] = 0.;
          D[c] = 1.;
          U[c] = -1.;
          V[c] = 0.;
        }
        c = (long)NY * nkxp + i;
        L[c] = 1.;
        D[c] = -1.;
        U[c] = 0.;
        V[c] = 0.;
      }
      thomas_complex_mpi(L, D, U, V, NY, nkxp, nkxp);
      for (int j = 1; j <= NY; j++)
        for (int i = 0; i < nkxp; i++) o->CR1[SIDX(o, j, k, i)] = V[(long)j * nkxp + i];
    }
    free(L);
    free(D);
    free(U);
    free(V);
  }
#pragma omp parallel for schedule(static)
  for (int j = 1; j <= NY; j++)
    for (int k = 0; k <= o->TNKZ; k++)
      for (int i = 0; i < nkxp; i++) {
        long c = SIDX(o, j, k, i);
        o->CU1[c] = o->CU1[c] - o->CIKX[i] * o->CR1[c];
        o->CU3[c] = o->CU3[c] - o->CIKZ[k] * o->CR1[c];
      }
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= NY; j++)
    for (int k = 0; k <= o->TNKZ; k++)
      for (int i = 0; i < nkxp; i++) {
        long c = SIDX(o, j, k, i);
        o->CU2[c] = o->CU2[c] - (o->CR1[c] - o->CR1[c - o->ss]) / DY[j];
      }
}

/* ---------------------------------------------------------- helpers */
static void spec_to_phys(orc *o, const cplx *s, double *p, int jmin, int jmax) {
  orc_fft_xz_to_physical(o, s, p, jmin, jmax);
}
static void phys_to_spec(orc *o, const double *p, cplx *s, int jmin, int jmax) {
  orc_fft_xz_to_fourier(o, p, s, jmin, jmax);
}

/* -------------------------------------------------------- POISSON_P_CHAN */
/* for/channel.f:1217-1453 with APPLY_BC_POISSON_MPI (for/mpi.f:1334-1369) */
void orc_poisson_p_chan(orc *o) {
  const int NY = o->NY, nkxp = o->nkxp, nkzt = o->nkzt, NX = o->NX, NZ = o->NZ;
  const double *DY = o->DY, *DYF = o->DYF, *GYF = o->GYF;
  cplx *CF1 = o->CF1, *CF2 = o->CF2, *CF3 = o->CF3, *CS1 = o->CS1;
  const long np = (long)NZ * NX;
#define LOOPJ2 for (int j = 2; j <= NY; j++) for (int k = 0; k < nkzt; k++) for (int i = 0; i < nkxp; i++)
  LOOPJ2 {
    long c = SIDX(o, j, k, i);
    CF1[c] = o->CIKX[i] * o->CU1[c];
    CF2[c] = (o->CU2[c + o->ss] - o->CU2[c]) / DYF[j];
    CF3[c] = o->CIKZ[k] * o->CU3[c];
  }
  spec_to_phys(o, CF1, o->F1, 0, NY + 1);
  spec_to_phys(o, CF2, o->F2, 0, NY + 1);
  spec_to_phys(o, CF3, o->F3, 0, NY + 1);
  for (long c = 2 * np; c < (NY + 1) * np; c++) {
    o->F1[c] = o->F1[c] * o->F1[c];
    o->F2[c] = o->F2[c] * o->F2[c];
    o->F3[c] = o->F3[c] * o->F3[c];
  }
  phys_to_spec(o, o->F1, CF1, 0, NY + 1);
  phys_to_spec(o, o->F2, CF2, 0, NY + 1);
  phys_to_spec(o, o->F3, CF3, 0, NY + 1);
  LOOPJ2 {
    long c = SIDX(o, j, k, i);
    CS1[c] = CF1[c] + CF2[c] + CF3[c];
  }
  for (int pass = 0; pass < 3; pass++) {
    LOOPJ2 {
      long c = SIDX(o, j, k, i);
      if (pass == 0) {
        CF1[c] = (o->CU1[c + o->ss] - o->CU1[c - o->ss]) / (2. * DYF[j]);
        CF2[c] = o->CIKX[i] * 0.5 * (o->CU2[c] + o->CU2[c + o->ss]);
      } else if (pass == 1) {
        CF1[c] = (o->CU3[c + o->ss] - o->CU3[c - o->ss]) / (2. * DYF[j]);
        CF2[c] = o->CIKZ[k] * 0.5 * (o->CU2[c] + o->CU2[c + o->ss]);
      } else {
        CF1[c] = o->CIKZ[k] * o->CU1[c];
        CF2[c] = o->CIKX[i] * o->CU3[c];
      }
    }
    spec_to_phys(o, CF1, o->F1, 0, NY + 1);
    spec_to_phys(o, CF2, o->F2, 0, NY + 1);
    for (long c = 2 * np; c < (NY + 1) * np; c++) o->F1[c] = 2. * o->F1[c] * o->F2[c];
    phys_to_spec(o, o->F1, CF1, 0, NY + 1);
    LOOPJ2 {
      long c = SIDX(o, j, k, i);
      CS1[c] = CS1[c] + CF1[c];
    }
  }
  for (int n = 0; n < o->NTH; n++) {
    LOOPJ2 {
      long c = SIDX(o, j, k, i);
      if (i != 0 || k != 0)
        CS1[c] = CS1[c] + o->p.ri[n] * (o->CTH[n][c + o->ss] - o->CTH[n][c - o->ss]) /
                              (GYF[j + 1] - GYF[j - 1]);
    }
  }
#undef LOOPJ2
  const long n = (long)nkxp * (NY + 2);
  double *L = malloc(sizeof(double) * n), *D = malloc(sizeof(double) * n),
         *U = malloc(sizeof(double) * n);
  cplx *V = malloc(sizeof(cplx) * n);
  for (int k = 0; k < nkzt; k++) {
    for (long c = 0; c < n; c++) {
      L[c] = 0.0;
      D[c] = 1.0;
      U[c] = 0.0;
      V[c] = 0.0;
    }
    for (int j = 2; j <= NY; j++)
      for (int i = 0; i < nkxp; i++) {
        long c = (long)j * nkxp + i;
        L[c] = 1. / (DY[j] * DYF[j]);
        D[c] = -o->KX2[i] - o->KZ2[k] - 1. / (DY[j + 1] * DYF[j]) - 1. / (DY[j] * DYF[j]);
        U[c] = 1. / (DY[j + 1] * DYF[j]);
        V[c] = -1. * CS1[SIDX(o, j, k, i)];
      }
    for (int i = 0; i < nkxp; i++) {
      long c = nkxp + i;
      if (i == 0 && k == 0) {
        D[c] = 1.;
        U[c] = 0.;
        V[c] = 0.;
      } else {
        D[c] = 1.;
        U[c] = -1.;
        V[c] = 0.;
      }
      c = (long)NY * nkxp + i;
      D[c] = -1.;
      L[c] = 1.;
      V[c] = 0.;
    }
    thomas_complex_mpi(L, D, U, V, NY, nkxp, nkxp);
    for (int j = 1; j <= NY; j++)
      for (int i = 0; i < nkxp; i++) o->CP[SIDX(o, j, k, i)] = V[(long)j * nkxp + i];
  }
  free(L);
  free(D);
  free(U);
  free(V);
}

/* --------------------------------------------------------------- COURANT */
/* for/courant.f:1-65, on the physical U1..U3 held in o->U1..U3 */
void orc_courant(orc *o) {
  const orc_params *p = &o->p;
  double dt = 999.0;
  double dmin = o->DX < o->DY[1] ? o->DX : o->DY[1];
  double t = 0.5 * (dmin * dmin) / p->nu;
  dt = dt < t ? dt : t;
  for (int n = 0; n < o->NTH; n++) {
    t = dt * p->nu / (p->nu / p->pr[n]);
    dt = dt < t ? dt : t;
  }
  if (p->i_ro != 0.0) {
    t = 2.0 * o->pi / fabs(p->i_ro) / 20.0;
    dt = dt < t ? dt : t;
  }
  for (int n = 0; n < o->NTH; n++)
    if (p->ri[n] != 0.0) {
      double nmax = sqrt(fabs(p->ri[n] * p->th_bc_ymin_c1[n]));
      t = (double)0.1f * 2.0 * o->pi / nmax; /* 0.1 is a default-real literal */
      dt = dt < t ? dt : t;
    }
  const int NY = o->NY;
  const long np = (long)o->NZ * o->NX;
#pragma omp parallel for reduction(min : dt) schedule(static)
  for (int j = 1; j <= NY; j++) {
    for (long c = 0; c < np; c++) {
      long q = (long)j * np + c;
      double dx = p->cfl * o->DX / fabs(o->U1[q]);
      double dy = p->cfl * o->DY[j] / fabs(o->U2[q]);
      double dz = p->cfl * o->DZ / fabs(o->U3[q]);
      double m = dt;
      if (dx < m) m = dx;
      if (dy < m) m = dy;
      if (dz < m) m = dz;
      dt = m;
    }
  }
  double new_dt;
  if (dt <= 0)
    new_dt = 0.0001;
  else if (dt >= 999.)
    new_dt = 999.0;
  else
    new_dt = dt;
  orc_set_time(o, o->time, new_dt);
}

/* ------------------------------------------------------------ RK_CHAN_1 */
/* for/channel.f:62-1073 (USER_RHS_CHAN_* are empty); the LES parts are in
 * les.c and in the eddy-viscosity terms of the implicit solves below. */
void orc_rk_chan_1(orc *o, int time_step, int rk_step) {
  const orc_params *p = &o->p;
  const int NY = o->NY, NX = o->NX, NZ = o->NZ, nkxp = o->nkxp, nkzt = o->nkzt;
  const long ss = o->ss, np = (long)NZ * NX;
  const double *DY = o->DY, *DYF = o->DYF;
  const int r = rk_step - 1;
  const double NU = p->nu, NUV = p->nu_v_scale;
  const double TEMP1 = NU * o->h_bar[r] / 2.0;
  const double TEMP2 = o->h_bar[r] / 2.0;
  const double *NUT = o->NU_T;
  const double TEMP3 = o->zeta_bar[r] * o->h_bar[r];
  const double TEMP4 = o->h_bar[r];
  const double TEMP5 = o->beta_bar[r] * o->h_bar[r];
  const int JS = o->jstart, JE = o->jend;
  cplx *CU1 = o->CU1, *CU2 = o->CU2, *CU3 = o->CU3, *CP = o->CP;
  cplx *CR1 = o->CR1, *CR2 = o->CR2, *CR3 = o->CR3, *CF1 = o->CF1, *CF2 = o->CF2, *CF3 = o->CF3;
  cplx *CS1 = o->CS1;
  double *U1 = o->U1, *U2 = o->U2, *U3 = o->U3, *S1 = o->S1;
#define LOOPS(J0, J1) \
  _Pragma("omp parallel for schedule(static)") for (int j = (J0); j <= (J1); j++) for (int k = 0; k < nkzt; k++) for (int i = 0; i < nkxp; i++)
#define LOOPP(J0, J1) \
  _Pragma("omp parallel for schedule(static)") for (int j = (J0); j <= (J1); j++) for (int k = 0; k < NZ; k++) for (int i = 0; i < NX; i++)
#define S(j, k, i) SIDX(o, j, k, i)
#define P(j, k, i) PIDX(o, j, k, i)

  LOOPS(JS, JE) {
    CR1[S(j, k, i)] = CU1[S(j, k, i)];
    CR3[S(j, k, i)] = CU3[S(j, k, i)];
  }
  LOOPS(2, NY) { CR2[S(j, k, i)] = CU2[S(j, k, i)]; }
  if (rk_step > 1) {
    LOOPS(JS, JE) {
      CR1[S(j, k, i)] = CR1[S(j, k, i)] + TEMP3 * CF1[S(j, k, i)];
      CR3[S(j, k, i)] = CR3[S(j, k, i)] + TEMP3 * CF3[S(j, k, i)];
    }
    LOOPS(2, NY) { CR2[S(j, k, i)] = CR2[S(j, k, i)] + TEMP3 * CF2[S(j, k, i)]; }
  }
  LOOPS(2, NY) { CS1[S(j, k, i)] = (CP[S(j, k, i)] - CP[S(j - 1, k, i)]) / DY[j]; }
  LOOPS(JS, JE) {
    CR1[S(j, k, i)] = CR1[S(j, k, i)] - TEMP4 * (o->CIKX[i] * CP[S(j, k, i)]);
    CR3[S(j, k, i)] = CR3[S(j, k, i)] - TEMP4 * (o->CIKZ[k] * CP[S(j, k, i)]);
  }
  LOOPS(2, NY) { CR2[S(j, k, i)] = CR2[S(j, k, i)] - TEMP4 * CS1[S(j, k, i)]; }
  if (p->f_type == 1) {
    for (int j = JS; j <= JE; j++) CR1[S(j, 0, 0)] = CR1[S(j, 0, 0)] - TEMP4 * p->px0;
  } else if (p->f_type == 2) {
    for (int j = JS; j <= JE; j++)
      CR1[S(j, 0, 0)] =
          CR1[S(j, 0, 0)] - TEMP4 * (p->px0 + p->amp_omega0 * cos(p->omega0 * o->time));
  }
  /* explicit horizontal viscous terms; BETA is the Laplacian order */
  LOOPS(JS, JE) {
    double kk = pow(o->KX2[i] + o->KZ2[k], p->beta);
    CF1[S(j, k, i)] = -NU * kk * CU1[S(j, k, i)];
    CF3[S(j, k, i)] = -NU * kk * CU3[S(j, k, i)];
  }
  LOOPS(2, NY) {
    double kk = pow(o->KX2[i] + o->KZ2[k], p->beta);
    CF2[S(j, k, i)] = -NU * kk * CU2[S(j, k, i)];
  }
  LOOPS(JS, JE) {
    CF1[S(j, k, i)] = CF1[S(j, k, i)] + p->i_ro * CU3[S(j, k, i)];
    CF3[S(j, k, i)] = CF3[S(j, k, i)] - p->i_ro * CU1[S(j, k, i)];
  }
  for (int n = 0; n < o->NTH; n++) {
    cplx *CTH = o->CTH[n], *CFTH = o->CFTH[n], *CRTH = o->CRTH[n];
    const double RI = p->ri[n], PR = p->pr[n];
    LOOPS(2, NY) {
      if (k == 0 && i == 0) continue;
      CF2[S(j, k, i)] = CF2[S(j, k, i)] + RI * p->grav_y *
                                              (CTH[S(j, k, i)] * DYF[j - 1] +
                                               CTH[S(j - 1, k, i)] * DYF[j]) /
                                              (2.0 * DY[j]);
    }
    LOOPS(JS, JE) { CF1[S(j, k, i)] = CF1[S(j, k, i)] + RI * p->grav_x * CTH[S(j, k, i)]; }
    LOOPS(JS, JE) { CF3[S(j, k, i)] = CF3[S(j, k, i)] + RI * p->grav_z * CTH[S(j, k, i)]; }
    const int JSt = o->jstart_th[n], JEt = o->jend_th[n];
    LOOPS(JSt, JEt) { CRTH[S(j, k, i)] = CTH[S(j, k, i)]; }
    if (rk_step > 1) {
      LOOPS(JSt, JEt) { CRTH[S(j, k, i)] = CRTH[S(j, k, i)] + TEMP3 * CFTH[S(j, k, i)]; }
    }
    LOOPS(JSt, JEt) {
      CFTH[S(j, k, i)] = -(NU / PR) * pow(o->KX2[i] + o->KZ2[k], p->beta) * CTH[S(j, k, i)];
    }
    LOOPS(JSt, JEt) {
      CFTH[S(j, k, i)] =
          CFTH[S(j, k, i)] - CU1[S(j, k, i)] * p->drhodx[n] - CU3[S(j, k, i)] * p->drhodz[n];
    }
  }

  /* the subgrid model waits 100 steps after a new flow (for/channel.f:303) */
  if (p->les && (!p->create_new_flow || time_step > 100)) {
    orc_les_chan(o);
    orc_apply_bc_vel_phys(o);
    for (int n = 0; n < o->NTH; n++) orc_les_scalar_terms(o, n);
    for (int n = 0; n < o->NTH; n++) spec_to_phys(o, o->CTH[n], o->TH[n], 0, NY + 1);
  } else {
    /* to physical space */
    spec_to_phys(o, CU1, U1, 0, NY + 1);
    spec_to_phys(o, CU2, U2, 0, NY + 1);
    spec_to_phys(o, CU3, U3, 0, NY + 1);
    for (int n = 0; n < o->NTH; n++) spec_to_phys(o, o->CTH[n], o->TH[n], 0, NY + 1);
  }

  /* nonlinear terms (for/channel.f:409-571) */
  LOOPP(JS, JE) { S1[P(j, k, i)] = U3[P(j, k, i)] * U1[P(j, k, i)]; }
  phys_to_spec(o, S1, CS1, 0, NY + 1);
  LOOPS(JS, JE) {
    CF1[S(j, k, i)] = CF1[S(j, k, i)] - o->CIKZ[k] * CS1[S(j, k, i)];
    CF3[S(j, k, i)] = CF3[S(j, k, i)] - o->CIKX[i] * CS1[S(j, k, i)];
  }
  LOOPP(JS, JE) { S1[P(j, k, i)] = U1[P(j, k, i)] * U1[P(j, k, i)]; }
  phys_to_spec(o, S1, CS1, 0, NY + 1);
  LOOPS(JS, JE) { CF1[S(j, k, i)] = CF1[S(j, k, i)] - o->CIKX[i] * CS1[S(j, k, i)]; }
  LOOPP(JS, JE) { S1[P(j, k, i)] = U3[P(j, k, i)] * U3[P(j, k, i)]; }
  phys_to_spec(o, S1, CS1, 0, NY + 1);
  LOOPS(JS, JE) { CF3[S(j, k, i)] = CF3[S(j, k, i)] - o->CIKZ[k] * CS1[S(j, k, i)]; }
  LOOPP(2, NY) {
    S1[P(j, k, i)] =
        ((DYF[j] * U1[P(j, k, i)] + DYF[j - 1] * U1[P(j - 1, k, i)]) / (2. * DY[j])) *
        U2[P(j, k, i)];
  }
  phys_to_spec(o, S1, CS1, 0, NY + 1);
  LOOPS(2, NY) { CF2[S(j, k, i)] = CF2[S(j, k, i)] - o->CIKX[i] * CS1[S(j, k, i)]; }
  LOOPP(2, NY) {
    S1[P(j, k, i)] =
        ((DYF[j] * U3[P(j, k, i)] + DYF[j - 1] * U3[P(j - 1, k, i)]) / (2. * DY[j])) *
        U2[P(j, k, i)];
  }
  phys_to_spec(o, S1, CS1, 0, NY + 1);
  LOOPS(2, NY) { CF2[S(j, k, i)] = CF2[S(j, k, i)] - o->CIKZ[k] * CS1[S(j, k, i)]; }
  LOOPP(JS, JE) {
    S1[P(j, k, i)] = (U1[P(j + 1, k, i)] * U2[P(j + 1, k, i)] + U1[P(j, k, i)] * U2[P(j + 1, k, i)] -
                      U1[P(j, k, i)] * U2[P(j, k, i)] - U1[P(j - 1, k, i)] * U2[P(j, k, i)]) /
                     (2.0 * DYF[j]);
  }
  phys_to_spec(o, S1, CS1, 0, NY + 1);
  LOOPS(JS, JE) { CF1[S(j, k, i)] = CF1[S(j, k, i)] - CS1[S(j, k, i)]; }
  LOOPP(JS, JE) {
    S1[P(j, k, i)] = (U3[P(j + 1, k, i)] * U2[P(j + 1, k, i)] + U3[P(j, k, i)] * U2[P(j + 1, k, i)] -
                      U3[P(j, k, i)] * U2[P(j, k, i)] - U3[P(j - 1, k, i)] * U2[P(j, k, i)]) /
                     (2.0 * DYF[j]);
  }
  phys_to_spec(o, S1, CS1, 0, NY + 1);
  LOOPS(JS, JE) { CF3[S(j, k, i)] = CF3[S(j, k, i)] - CS1[S(j, k, i)]; }
  LOOPP(2, NY) {
    double a = U2[P(j, k, i)] + U2[P(j + 1, k, i)], b = U2[P(j, k, i)] + U2[P(j - 1, k, i)];
    S1[P(j, k, i)] = (0.25 * (a * a) - 0.25 * (b * b)) / DY[j];
  }
  phys_to_spec(o, S1, CS1, 0, NY + 1);
  LOOPS(2, NY) { CF2[S(j, k, i)] = CF2[S(j, k, i)] - CS1[S(j, k, i)]; }

  /* CR += beta*h*CF and transform */
  LOOPS(JS, JE) {
    CR1[S(j, k, i)] = CR1[S(j, k, i)] + TEMP5 * CF1[S(j, k, i)];
    CR3[S(j, k, i)] = CR3[S(j, k, i)] + TEMP5 * CF3[S(j, k, i)];
  }
  LOOPS(2, NY) { CR2[S(j, k, i)] = CR2[S(j, k, i)] + TEMP5 * CF2[S(j, k, i)]; }
  spec_to_phys(o, CR1, o->R1, 0, NY + 1);
  spec_to_phys(o, CR2, o->R2, 2, NY);
  spec_to_phys(o, CR3, o->R3, 0, NY + 1);
  double *R1 = o->R1, *R2 = o->R2, *R3 = o->R3;
  /* explicit half of the Crank-Nicolson vertical viscous term */
  LOOPP(JS, JE) {
    R1[P(j, k, i)] = R1[P(j, k, i)] +
                     TEMP1 * NUV *
                         (((U1[P(j + 1, k, i)] - U1[P(j, k, i)]) / DY[j + 1] -
                           (U1[P(j, k, i)] - U1[P(j - 1, k, i)]) / DY[j]) /
                          DYF[j]);
    R3[P(j, k, i)] = R3[P(j, k, i)] +
                     TEMP1 * NUV *
                         (((U3[P(j + 1, k, i)] - U3[P(j, k, i)]) / DY[j + 1] -
                           (U3[P(j, k, i)] - U3[P(j - 1, k, i)]) / DY[j]) /
                          DYF[j]);
  }
  LOOPP(2, NY) {
    R2[P(j, k, i)] = R2[P(j, k, i)] +
                     TEMP1 * NUV *
                         (((U2[P(j + 1, k, i)] - U2[P(j, k, i)]) / DYF[j] -
                           (U2[P(j, k, i)] - U2[P(j - 1, k, i)]) / DYF[j - 1]) /
                          DY[j]);
  }
  /* eddy viscosity, Crank-Nicolson like the molecular term (NU_T on GY
   * points; interpolated to GYF for U2), for/channel.f:631-659 */
  if (p->les) {
    LOOPP(JS, JE) {
      const long q = P(j, k, i), qp = P(j + 1, k, i), qm = P(j - 1, k, i);
      R1[q] = R1[q] + TEMP2 * ((NUT[qp] * (U1[qp] - U1[q]) / DY[j + 1] -
                                NUT[q] * (U1[q] - U1[qm]) / DY[j]) / DYF[j]);
      R3[q] = R3[q] + TEMP2 * ((NUT[qp] * (U3[qp] - U3[q]) / DY[j + 1] -
                                NUT[q] * (U3[q] - U3[qm]) / DY[j]) / DYF[j]);
    }
    LOOPP(2, NY) {
      const long q = P(j, k, i), qp = P(j + 1, k, i), qm = P(j - 1, k, i);
      R2[q] = R2[q] + TEMP2 * ((0.5 * (NUT[q] + NUT[qp]) * (U2[qp] - U2[q]) / DYF[j] -
                                0.5 * (NUT[q] + NUT[qm]) * (U2[q] - U2[qm]) / DYF[j - 1]) /
                               DY[j]);
    }
  }

  /* scalars: nonlinear terms, RHS, implicit solve (for/channel.f:665-836) */
  for (int n = 0; n < o->NTH; n++) {
    cplx *CFTH = o->CFTH[n], *CRTH = o->CRTH[n];
    double *TH = o->TH[n], *RTH = o->RTH[n];
    const int JSt = o->jstart_th[n], JEt = o->jend_th[n];
    const double PR = p->pr[n];
    LOOPP(JSt, JEt) { S1[P(j, k, i)] = TH[P(j, k, i)] * U1[P(j, k, i)]; }
    phys_to_spec(o, S1, CS1, 0, NY + 1);
    LOOPS(JSt, JEt) { CFTH[S(j, k, i)] = CFTH[S(j, k, i)] - o->CIKX[i] * CS1[S(j, k, i)]; }
    LOOPP(JSt, JEt) { S1[P(j, k, i)] = TH[P(j, k, i)] * U3[P(j, k, i)]; }
    phys_to_spec(o, S1, CS1, 0, NY + 1);
    LOOPS(JSt, JEt) { CFTH[S(j, k, i)] = CFTH[S(j, k, i)] - o->CIKZ[k] * CS1[S(j, k, i)]; }
    LOOPP(JSt, JEt) {
      S1[P(j, k, i)] = (TH[P(j + 1, k, i)] * U2[P(j + 1, k, i)] + TH[P(j, k, i)] * U2[P(j + 1, k, i)] -
                        TH[P(j, k, i)] * U2[P(j, k, i)] - TH[P(j - 1, k, i)] * U2[P(j, k, i)]) /
                       (2.0 * DYF[j]);
    }
    phys_to_spec(o, S1, CS1, 0, NY + 1);
    LOOPS(JSt, JEt) { CFTH[S(j, k, i)] = CFTH[S(j, k, i)] - CS1[S(j, k, i)]; }
    LOOPS(JSt, JEt) { CRTH[S(j, k, i)] = CRTH[S(j, k, i)] + TEMP5 * CFTH[S(j, k, i)]; }
    spec_to_phys(o, CRTH, RTH, 0, NY + 1);
    LOOPP(JSt, JEt) {
      RTH[P(j, k, i)] = RTH[P(j, k, i)] +
                        (TEMP1 / PR) * NUV *
                            (((TH[P(j + 1, k, i)] - TH[P(j, k, i)]) / DY[j + 1] -
                              (TH[P(j, k, i)] - TH[P(j - 1, k, i)]) / DY[j]) /
                             DYF[j]);
    }
    if (p->les) {
      /* KAPPA_T = NU_T (for/channel.f:314-322, 748-760) */
      LOOPP(JSt, JEt) {
        const long q = P(j, k, i), qp = P(j + 1, k, i), qm = P(j - 1, k, i);
        RTH[q] = RTH[q] + TEMP2 * ((NUT[qp] * (TH[qp] - TH[q]) / DY[j + 1] -
                                    NUT[q] * (TH[q] - TH[qm]) / DY[j]) / DYF[j]);
      }
    }
#pragma omp parallel
    {
      const long nm = (long)NX * (NY + 2);
      rowset m = {malloc(sizeof(double) * nm), malloc(sizeof(double) * nm),
                  malloc(sizeof(double) * nm), malloc(sizeof(double) * nm), NX};
      const double a = TEMP1 / PR * NUV;
#pragma omp for schedule(static)
      for (int k = 0; k < NZ; k++) {
        for (int j = 0; j <= NY + 1; j++) set_row(&m, j, 0., 1., 0., 0.);
        for (int j = JSt; j <= JEt; j++)
          for (int i = 0; i < NX; i++) {
            long c = (long)j * NX + i;
            m.L[c] = -(a) / (DY[j] * DYF[j]);
            m.D[c] = 1. + (a) / (DY[j + 1] * DYF[j]) + (a) / (DY[j] * DYF[j]);
            m.U[c] = -(a) / (DY[j + 1] * DYF[j]);
            m.V[c] = RTH[P(j, k, i)];
            if (p->les) {
              const double kj = NUT[P(j, k, i)], kp = NUT[P(j + 1, k, i)];
              m.L[c] = m.L[c] - TEMP2 * kj / (DY[j] * DYF[j]);
              m.D[c] = m.D[c] + TEMP2 * kp / (DY[j + 1] * DYF[j]) + TEMP2 * kj / (DY[j] * DYF[j]);
              m.U[c] = m.U[c] - TEMP2 * kp / (DY[j + 1] * DYF[j]);
            }
          }
        bc_gyf_lower(&m, p->th_bc_ymin[n], p->th_bc_ymin_c1[n], o);
        bc_gyf_upper(&m, p->th_bc_ymax[n], p->th_bc_ymax_c1[n], o);
        thomas_real_mpi(m.L, m.D, m.U, m.V, NY, NX);
        for (int j = JSt - 1; j <= JEt + 1; j++)
          for (int i = 0; i < NX; i++) TH[P(j, k, i)] = m.V[(long)j * NX + i];
      }
      free(m.L);
      free(m.D);
      free(m.U);
      free(m.V);
    }
  }

  /* velocity implicit solves: U2, U1, U3 (for/channel.f:838-1029) */
  for (int comp = 0; comp < 3; comp++) {
#pragma omp parallel
    {
      const long nm = (long)NX * (NY + 2);
      rowset m = {malloc(sizeof(double) * nm), malloc(sizeof(double) * nm),
                  malloc(sizeof(double) * nm), malloc(sizeof(double) * nm), NX};
#pragma omp for schedule(static)
      for (int k = 0; k < NZ; k++) {
        for (int j = 0; j <= NY + 1; j++) set_row(&m, j, 0., 1., 0., 0.);
        if (comp == 0) {
          for (int j = 2; j <= NY; j++)
            for (int i = 0; i < NX; i++) {
              long c = (long)j * NX + i;
              m.L[c] = -TEMP1 * NUV / (DYF[j - 1] * DY[j]);
              m.D[c] = 1. + TEMP1 * NUV / (DYF[j] * DY[j]) + TEMP1 * NUV / (DYF[j - 1] * DY[j]);
              m.U[c] = -TEMP1 * NUV / (DYF[j] * DY[j]);
              m.V[c] = R2[P(j, k, i)];
              if (p->les) {
                const double nm = 0.5 * (NUT[P(j, k, i)] + NUT[P(j - 1, k, i)]);
                const double npl = 0.5 * (NUT[P(j, k, i)] + NUT[P(j + 1, k, i)]);
                m.L[c] = m.L[c] - TEMP2 * nm / (DYF[j - 1] * DY[j]);
                m.D[c] = m.D[c] + TEMP2 * npl / (DYF[j] * DY[j]) + TEMP2 * nm / (DYF[j - 1] * DY[j]);
                m.U[c] = m.U[c] - TEMP2 * npl / (DYF[j] * DY[j]);
              }
            }
          bc_gy_lower(&m, p->v_bc_ymin, p->v_bc_ymin_c1, o);
          bc_gy_upper(&m, p->v_bc_ymax, p->v_bc_ymax_c1, o);
          thomas_real_mpi(m.L, m.D, m.U, m.V, NY, NX);
          for (int j = 1; j <= NY + 1; j++)
            for (int i = 0; i < NX; i++) U2[P(j, k, i)] = m.V[(long)j * NX + i];
        } else {
          const double *R = comp == 1 ? R1 : R3;
          double *U = comp == 1 ? U1 : U3;
          for (int j = JS; j <= JE; j++)
            for (int i = 0; i < NX; i++) {
              long c = (long)j * NX + i;
              m.L[c] = -TEMP1 * NUV / (DY[j] * DYF[j]);
              m.D[c] = 1. - TEMP1 * NUV * (-1. / (DY[j + 1] * DYF[j]) - 1. / (DY[j] * DYF[j]));
              m.U[c] = -TEMP1 * NUV / (DY[j + 1] * DYF[j]);
              m.V[c] = R[P(j, k, i)];
              if (p->les) {
                const double nj = NUT[P(j, k, i)], np1 = NUT[P(j + 1, k, i)];
                m.L[c] = m.L[c] - TEMP2 * nj / (DY[j] * DYF[j]);
                m.D[c] = m.D[c] + TEMP2 * np1 / (DY[j + 1] * DYF[j]) + TEMP2 * nj / (DY[j] * DYF[j]);
                m.U[c] = m.U[c] - TEMP2 * np1 / (DY[j + 1] * DYF[j]);
              }
            }
          if (comp == 1) {
            bc_gyf_lower(&m, p->u_bc_ymin, p->u_bc_ymin_c1, o);
            bc_gyf_upper(&m, p->u_bc_ymax, p->u_bc_ymax_c1, o);
          } else {
            bc_gyf_lower(&m, p->w_bc_ymin, p->w_bc_ymin_c1, o);
            bc_gyf_upper(&m, p->w_bc_ymax, p->w_bc_ymax_c1, o);
          }
          thomas_real_mpi(m.L, m.D, m.U, m.V, NY, NX);
          for (int j = JS - 1; j <= JE + 1; j++)
            for (int i = 0; i < NX; i++) U[P(j, k, i)] = m.V[(long)j * NX + i];
        }
      }
      free(m.L);
      free(m.D);
      free(m.U);
      free(m.V);
    }
  }

  if (p->variable_dt && rk_step == 3 && (time_step % p->update_dt) == 0) orc_courant(o);

  phys_to_spec(o, U1, CU1, 0, NY + 1);
  phys_to_spec(o, U2, CU2, 0, NY + 1);
  phys_to_spec(o, U3, CU3, 0, NY + 1);
  for (int n = 0; n < o->NTH; n++) phys_to_spec(o, o->TH[n], o->CTH[n], 0, NY + 1);

  orc_rem_div_chan(o);

  LOOPS(JS, JE) { CP[S(j, k, i)] = CP[S(j, k, i)] + CR1[S(j, k, i)] / TEMP4; }
  (void)ss;
  (void)np;
#undef LOOPS
#undef LOOPP
#undef S
#undef P
}

/* ------------------------------------------------------- initial flow */
/* CREATE_FLOW_CHAN tail (for/set_ics.f:109-182) and CREATE_TH_CHAN's
 * transform (for/set_ics.f:251-253): the caller supplies the physical fields
 * (profile + seeded noise); then FFT, APPLY_BC_VEL, REM_DIV_CHAN and the
 * APPLY_BC_VEL done by SAVE_STATS_CHAN (for/save_stats.f:30-36). */
void orc_create_flow_chan(orc *o, const double *u1, const double *u2, const double *u3,
                          const double *th) {
  const int NY = o->NY;
  phys_to_spec(o, u1, o->CU1, 0, NY + 1);
  phys_to_spec(o, u2, o->CU2, 0, NY + 1);
  phys_to_spec(o, u3, o->CU3, 0, NY + 1);
  memset(o->CP, 0, sizeof(cplx) * o->nspec);
  for (int n = 0; n < o->NTH; n++) {
    if (th) phys_to_spec(o, th + (long)n * o->nphys, o->CTH[n], 0, NY + 1);
    memset(o->CFTH[n], 0, sizeof(cplx) * o->nspec);
  }
  memset(o->CF1, 0, sizeof(cplx) * o->nspec);
  memset(o->CF2, 0, sizeof(cplx) * o->nspec);
  memset(o->CF3, 0, sizeof(cplx) * o->nspec);
  orc_apply_bc_vel(o);
  orc_rem_div_chan(o);
  orc_apply_bc_vel(o);
}

/* ------------------------------------------------------------ statistics */
/* INTEGRATE_Y_VAR (for/mpi.f:1676-1698) */
static double integrate_y(const orc *o, const double *v) {
  double res = 0.;
  for (int j = 2; j <= o->NY; j++) res = res + 0.5 * (v[j] + v[j - 1]) * o->DY[j];
  return res / o->p.ly;
}

/* Parity series from SAVE_STATS_CHAN (for/save_stats.f:112-203,470-489),
 * evaluated on the current spectral state without modifying it. */
void orc_stats_chan(const orc *o, orc_stats *s) {
  const int NY = o->NY, NX = o->NX, NZ = o->NZ;
  const long np = (long)NX * NZ;
  double *ume = calloc(NY + 2, sizeof(double)), *vme = calloc(NY + 2, sizeof(double)),
         *wme = calloc(NY + 2, sizeof(double));
  double *urms = calloc(NY + 2, sizeof(double)), *vrms = calloc(NY + 2, sizeof(double)),
         *wrms = calloc(NY + 2, sizeof(double)), *ke = calloc(NY + 2, sizeof(double));
  for (int j = 0; j <= NY + 1; j++) {
    ume[j] = creal(o->CU1[SIDX(o, j, 0, 0)]);
    vme[j] = creal(o->CU2[SIDX(o, j, 0, 0)]);
    wme[j] = creal(o->CU3[SIDX(o, j, 0, 0)]);
  }
  s->ubulk = integrate_y(o, ume);
  double *u1 = malloc(sizeof(double) * o->nphys), *u2 = malloc(sizeof(double) * o->nphys),
         *u3 = malloc(sizeof(double) * o->nphys);
  orc_fft_xz_to_physical(o, o->CU1, u1, 0, NY + 1);
  orc_fft_xz_to_physical(o, o->CU2, u2, 0, NY + 1);
  orc_fft_xz_to_physical(o, o->CU3, u3, 0, NY + 1);
  for (int j = 1; j <= NY; j++) {
    double a = 0, b = 0, c = 0, e = 0;
    for (long q = 0; q < np; q++) {
      double du = u1[j * np + q] - ume[j], dw = u3[j * np + q] - wme[j];
      double dv0 = u2[j * np + q] - vme[j], dv1 = u2[(j + 1) * np + q] - vme[j + 1];
      a += du * du;
      b += 0.5 * (dv0 * dv0 + dv1 * dv1);
      c += dw * dw;
      double v0 = u2[j * np + q], v1 = u2[(j + 1) * np + q];
      e += u1[j * np + q] * u1[j * np + q] + 0.5 * (v0 * v0 + v1 * v1) +
           u3[j * np + q] * u3[j * np + q];
    }
    urms[j] = sqrt(a / ((double)NZ * NX));
    vrms[j] = sqrt(b / ((double)NZ * NX));
    wrms[j] = sqrt(c / ((double)NZ * NX));
    ke[j] = 0.5 * e / ((double)NZ * NX);
  }
  s->urms_b = integrate_y(o, urms);
  s->vrms_b = integrate_y(o, vrms);
  s->wrms_b = integrate_y(o, wrms);
  s->ke = integrate_y(o, ke);
  for (int n = 0; n < o->NTH && n < ORC_MAX_TH; n++) {
    double *th = u1;
    orc_fft_xz_to_physical(o, o->CTH[n], th, 0, NY + 1);
    double *thrms = urms, *thv = vrms;
    for (int j = 1; j <= NY; j++) {
      double m = creal(o->CTH[n][SIDX(o, j, 0, 0)]), a = 0;
      for (long q = 0; q < np; q++) {
        double d = th[j * np + q] - m;
        a += d * d;
      }
      thrms[j] = sqrt(a / ((double)NZ * NX));
      thv[j] = a / ((double)NZ * NX);
    }
    s->thrms_b[n] = integrate_y(o, thrms);
    s->th_var[n] = integrate_y(o, thv);
  }
  s->div_max = orc_div_max_chan(o);
  free(u1);
  free(u2);
  free(u3);
  free(ume);
  free(vme);
  free(wme);
  free(urms);
  free(vrms);
  free(wrms);
  free(ke);
}

/* max over physical points of |div u| on the rows REM_DIV_CHAN constrains
 * (j = 2..NY-1): ikx U1 + (U2(j+1)-U2(j))/DYF(j) + ikz U3 */
double orc_div_max_chan(const orc *o) {
  const int NY = o->NY;
  cplx *d = calloc(o->nspec, sizeof(cplx));
  double *ph = calloc(o->nphys, sizeof(double));
  for (int j = 2; j <= NY - 1; j++)
    for (int k = 0; k < o->nkzt; k++)
      for (int i = 0; i < o->nkxp; i++) {
        long c = SIDX(o, j, k, i);
        d[c] = o->CIKX[i] * o->CU1[c] + (o->CU2[c + o->ss] - o->CU2[c]) / o->DYF[j] +
               o->CIKZ[k] * o->CU3[c];
      }
  orc_fft_xz_to_physical(o, d, ph, 2, NY - 1);
  double mx = 0;
  const long np = (long)o->NX * o->NZ;
  for (long q = 2 * np; q < (long)NY * np; q++)
    if (fabs(ph[q]) > mx) mx = fabs(ph[q]);
  free(d);
  free(ph);
  return mx;
}
