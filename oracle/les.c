/*
 * Oracle restatement of the channel LES (constant Smagorinsky, the only
 * model the MPI build runs).  TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Follows for/les.f:1-275 (les_chan, LES_MODEL_TYPE = 1) with its plane
 * means for mean_les (for/les.f:336-459), for/les.f:526-569 (compute_strain_chan),
 * for/les.f:805-865 (APPLY_BC_LES), for/mpi.f:352-515 (GHOST_LES_MPI with
 * NPROCY = 1: NU_T = 0 on planes 1, 2, NY, NY+1), for/channel.f:2495-2652
 * (APPLY_BC_VEL_PHYS_LOWER/UPPER) and the scalar eddy-diffusivity block of
 * RK_CHAN_1 (for/channel.f:312-372).  The implicit eddy-viscosity terms of
 * the Crank-Nicolson solves live in channel.c beside the molecular ones.
 *
 * The reference keeps S_ij and CS_ij in EQUIVALENCEd storage; planes that
 * compute_strain_chan does not write (0 and NY+1 of CS_1,2,3,5, plane 0 of
 * CS_4,6) start at zero and stay zero through every call, so they are zero
 * here by construction.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle_int.h"

#define SIDX(o, j, k, i) ((long)(j) * (o)->ss + (long)(k) * (o)->nkxp + (i))
#define PIDX(o, j, k, i) ((long)(j) * (o)->NZ * (o)->NX + (long)(k) * (o)->NX + (i))

/* for/les.f:805-865: with Neumann velocity BCs the ghost planes copy the
 * first interior plane so the model sees no spurious wall gradient. */
static void apply_bc_les(orc *o) {
  const orc_params *p = &o->p;
  const int NY = o->NY;
  const long ss = o->ss;
  cplx *U1 = o->CU1, *U3 = o->CU3;
  for (long m = 0; m < ss; m++) {
    if (p->u_bc_ymax == 1) {
      U1[NY * ss + m] = U1[(NY - 1) * ss + m];
      U1[(NY + 1) * ss + m] = U1[NY * ss + m];
    }
    if (p->w_bc_ymax == 1) {
      U3[NY * ss + m] = U3[(NY - 1) * ss + m];
      U3[(NY + 1) * ss + m] = U3[NY * ss + m];
    }
    if (p->u_bc_ymin == 1) {
      U1[1 * ss + m] = U1[2 * ss + m];
      U1[m] = U1[1 * ss + m];
    }
    if (p->w_bc_ymin == 1) {
      U3[1 * ss + m] = U3[2 * ss + m];
      U3[m] = U3[1 * ss + m];
    }
  }
}

/* APPLY_BC_VEL_PHYS_LOWER / _UPPER (for/channel.f:2495-2652) on U1..U3. */
void orc_apply_bc_vel_phys(orc *o) {
  const orc_params *p = &o->p;
  const int NY = o->NY;
  const long np = (long)o->NZ * o->NX;
  const double *DY = o->DY, *DYF = o->DYF;
  double *U1 = o->U1, *U2 = o->U2, *U3 = o->U3;
  for (long q = 0; q < np; q++) {
    const long j0 = q, j1 = np + q, j2 = 2 * np + q;
    const long jm = (NY - 1) * np + q, jn = NY * np + q, jn1 = (NY + 1) * np + q;
    if (p->u_bc_ymin == 0) {
      U1[j0] = p->u_bc_ymin_c1;
      U1[j1] = p->u_bc_ymin_c1;
    } else {
      U1[j1] = U1[j2] - DY[2] * p->u_bc_ymin_c1;
      U1[j0] = U1[j1] - DY[1] * p->u_bc_ymin_c1;
    }
    if (p->w_bc_ymin == 0) {
      U3[j0] = p->w_bc_ymin_c1;
      U3[j1] = p->w_bc_ymin_c1;
    } else {
      U3[j1] = U3[j2] - DY[2] * p->w_bc_ymin_c1;
      U3[j0] = U3[j1] - DY[1] * p->w_bc_ymin_c1;
    }
    if (p->v_bc_ymin == 0) {
      U2[j1] = 2.0 * p->v_bc_ymin_c1 - U2[j2];
      U2[j0] = U2[j1];
    } else {
      U2[j1] = U2[j2] - DYF[1] * p->v_bc_ymin_c1;
      U2[j0] = U2[j1] - DYF[1] * p->v_bc_ymin_c1;
    }
    if (p->u_bc_ymax == 0) {
      U1[jn] = p->u_bc_ymax_c1;
      U1[jn1] = p->u_bc_ymax_c1;
    } else {
      U1[jn] = U1[jm] + DY[NY] * p->u_bc_ymax_c1;
      U1[jn1] = U1[jn] + DY[NY] * p->u_bc_ymax_c1;
    }
    if (p->w_bc_ymax == 0) {
      U3[jn] = p->w_bc_ymax_c1;
      U3[jn1] = p->w_bc_ymax_c1;
    } else {
      U3[jn] = U3[jm] + DY[NY] * p->w_bc_ymax_c1;
      U3[jn1] = U3[jn] + DY[NY] * p->w_bc_ymax_c1;
    }
    if (p->v_bc_ymax == 0)
      U2[jn1] = 2.0 * p->v_bc_ymax_c1 - U2[jn];
    else
      U2[jn1] = U2[jn] + DY[NY] * p->v_bc_ymax_c1;
  }
}

/* Filter width factor -2 C_S^2 (DX BETA DY 2 DZ BETA)^(2/3) with C_S = 0.13
 * and BETA = 1 (for/les.f:194-217), for a y spacing d. */
static double delta_factor(const orc *o, double d) {
  const double cs = 0.13, beta_sgs = 1.0;
  return -2.0 * cs * cs * pow(o->DX * beta_sgs * d * 2.0 * o->DZ * beta_sgs, 2.0 / 3.0);
}

/* The plane means les_chan writes to mean_les (for/les.f:336-459): NU_T and
 * EPS_SGS1 = <F1 U1 + F3 U3 + F2 U2>, F the SGS stress divergence in physical
 * space (the cross terms of F2 transformed separately, as the reference
 * does), with the velocity as les_chan holds it (before APPLY_BC_VEL_PHYS).
 * CTEMP planes the loops do not write are zero in the reference. */
static void les_means(orc *o, int J1, int J2) {
  const int NY = o->NY, NX = o->NX, NZ = o->NZ, nkxp = o->nkxp, nkzt = o->nkzt;
  const long np = (long)NX * NZ;
  const double *DY = o->DY, *DYF = o->DYF;
  cplx **CS = o->CSij, *CT = o->CTEMP;
  double *T = o->TEMP, *NUT = o->NU_T;
  const double *U[3] = {o->U1, o->U2, o->U3};
  double *eps = o->eps_sgs1_mean, *num = o->nu_t_mean;
  for (int j = 0; j <= NY + 1; j++) {
    double a = 0.0, b = 0.0;
    for (long q = 0; q < np; q++) b += NUT[j * np + q];
    num[j] = b / (double)(NX * NZ);
    eps[j] = a;
  }
  for (int part = 0; part < 5; part++) {
    memset(CT, 0, sizeof(cplx) * o->nspec);
    const double *Uf = part == 0 ? U[0] : part == 1 ? U[2] : U[1];
    if (part < 3) {
      const int j0 = part < 2 ? J1 : 2, j1 = part < 2 ? J2 : NY;
      for (int j = j0; j <= j1; j++)
        for (int k = 0; k < nkzt; k++)
          for (int i = 0; i < nkxp; i++) {
            const long s = SIDX(o, j, k, i), sp = s + o->ss;
            if (part == 0)
              CT[s] = -o->CIKX[i] * CS[0][s] - (CS[3][sp] - CS[3][s]) / DYF[j] - o->CIKZ[k] * CS[4][s];
            else if (part == 1)
              CT[s] = -o->CIKX[i] * CS[4][s] - (CS[5][sp] - CS[5][s]) / DYF[j] - o->CIKZ[k] * CS[2][s];
            else
              CT[s] = -o->CIKX[i] * CS[3][s] - o->CIKZ[k] * CS[5][s];
          }
    } else {
      const double *Ud = part == 3 ? U[0] : U[2];
      for (int j = 2; j <= NY; j++)
        for (long q = 0; q < np; q++)
          T[j * np + q] = NUT[j * np + q] * (Ud[j * np + q] - Ud[(j - 1) * np + q]) / DY[j];
      orc_fft_xz_to_fourier(o, T, CT, 2, NY);
      for (int j = 2; j <= NY; j++)
        for (int k = 0; k < nkzt; k++)
          for (int i = 0; i < nkxp; i++) {
            const long s = SIDX(o, j, k, i);
            CT[s] = (part == 3 ? o->CIKX[i] : o->CIKZ[k]) * CT[s];
          }
    }
    orc_fft_xz_to_physical(o, CT, T, 0, NY + 1);
    for (int j = 0; j <= NY + 1; j++) {
      double a = 0.0;
      for (long q = 0; q < np; q++) a += T[j * np + q] * Uf[j * np + q];
      eps[j] += a;
    }
  }
  for (int j = 0; j <= NY + 1; j++) eps[j] = eps[j] / (double)(NX * NZ);
  o->les_stats_req = 0;
  o->les_stats_valid = 1;
}

/* les_chan for LES_MODEL_TYPE = 1: the velocity is spectral on entry and
 * physical (U1..U3, boundary planes as les_chan leaves them) on exit; NU_T is
 * set and the SGS stress divergence is added to CF1..CF3. */
void orc_les_chan(orc *o) {
  const int NY = o->NY, NX = o->NX, NZ = o->NZ, nkxp = o->nkxp, nkzt = o->nkzt;
  const double *DY = o->DY, *DYF = o->DYF;
  const int JS = o->jstart, JE = o->jend;
  /* J1/J2 of les_chan: the RANKY = NPROCY-1 branch (for/les.f:44-56) */
  const int J1 = JS, J2 = NY - 1;
  cplx *CU1 = o->CU1, *CU2 = o->CU2, *CU3 = o->CU3;
  double *U1 = o->U1, *U2 = o->U2, *U3 = o->U3;
  double **S = o->Sij;
  cplx **CS = o->CSij;
  double *NUT = o->NU_T, *T = o->TEMP;
  const long ns = o->nspec;
#define S_(j, k, i) SIDX(o, j, k, i)
#define P_(j, k, i) PIDX(o, j, k, i)
#define LOOPS(J0, J1_) \
  _Pragma("omp parallel for schedule(static)") for (int j = (J0); j <= (J1_); j++) for (int k = 0; k < nkzt; k++) for (int i = 0; i < nkxp; i++)
#define LOOPP(J0, J1_) \
  _Pragma("omp parallel for schedule(static)") for (int j = (J0); j <= (J1_); j++) for (int k = 0; k < NZ; k++) for (int i = 0; i < NX; i++)

  orc_apply_bc_vel(o);  /* APPLY_BC_VEL_MPI; GHOST_CHAN_MPI is a no-op for one rank */
  apply_bc_les(o);

  /* compute_strain_chan (for/les.f:526-569) */
  for (int c = 0; c < 6; c++) memset(CS[c], 0, sizeof(cplx) * ns);
  LOOPS(1, NY) {
    const long s = S_(j, k, i);
    CS[0][s] = o->CIKX[i] * CU1[s];
    CS[1][s] = (CU2[s + o->ss] - CU2[s]) / DYF[j];
    CS[2][s] = o->CIKZ[k] * CU3[s];
    CS[4][s] = 0.5 * (o->CIKZ[k] * CU1[s] + o->CIKX[i] * CU3[s]);
  }
  LOOPS(1, NY + 1) {
    const long s = S_(j, k, i);
    CS[3][s] = 0.5 * ((CU1[s] - CU1[s - o->ss]) / DY[j] + o->CIKX[i] * CU2[s]);
    CS[5][s] = 0.5 * (o->CIKZ[k] * CU2[s] + (CU3[s] - CU3[s - o->ss]) / DY[j]);
  }
  for (int c = 0; c < 6; c++) orc_fft_xz_to_physical(o, CS[c], S[c], 0, NY + 1);

  double *u1b = calloc(NY + 2, sizeof(double)), *u3b = calloc(NY + 2, sizeof(double));
  for (int j = 0; j <= NY + 1; j++) {
    u1b[j] = creal(CU1[S_(j, 0, 0)]);
    u3b[j] = creal(CU3[S_(j, 0, 0)]);
  }
  orc_fft_xz_to_physical(o, CU1, U1, 0, NY + 1);
  orc_fft_xz_to_physical(o, CU2, U2, 0, NY + 1);
  orc_fft_xz_to_physical(o, CU3, U3, 0, NY + 1);

  /* |S| at GYF points (kept in S1) and at GY points (TEMP) */
  double *S1 = o->S1;
  LOOPP(JS, JE) {
    const long q = P_(j, k, i), qp = P_(j + 1, k, i);
    const double a4 = 0.5 * (S[3][qp] + S[3][q] - 0.5 * (u1b[j] - u1b[j - 1]) / DY[j] -
                             0.5 * (u1b[j + 1] - u1b[j]) / DY[j + 1]);
    const double a6 = 0.5 * (S[5][qp] + S[5][q] - 0.5 * (u3b[j] - u3b[j - 1]) / DY[j] -
                             0.5 * (u3b[j + 1] - u3b[j]) / DY[j + 1]);
    S1[q] = sqrt(2.0 * (S[0][q] * S[0][q]) + 4.0 * (a4 * a4) + 4.0 * (S[4][q] * S[4][q]) +
                 2.0 * (S[1][q] * S[1][q]) + 4.0 * (a6 * a6) + 2.0 * (S[2][q] * S[2][q]));
  }
  LOOPP(2, NY + 1) {
    const long q = P_(j, k, i), qm = P_(j - 1, k, i);
    const double w = 2.0 * DY[j];
    const double b1 = (S[0][q] * DYF[j - 1] + S[0][qm] * DYF[j]) / w;
    const double b4 = S[3][q] - 0.5 * (u1b[j] - u1b[j - 1]) / DY[j];
    const double b5 = (S[4][q] * DYF[j - 1] + S[4][qm] * DYF[j]) / w;
    const double b2 = (S[1][q] * DYF[j - 1] + S[1][qm] * DYF[j]) / w;
    const double b6 = S[5][q] - 0.5 * (u3b[j] - u3b[j - 1]) / DY[j];
    const double b3 = (S[2][q] * DYF[j - 1] + S[2][qm] * DYF[j]) / w;
    T[q] = sqrt(2.0 * (b1 * b1) + 4.0 * (b4 * b4) + 4.0 * (b5 * b5) + 2.0 * (b2 * b2) +
                4.0 * (b6 * b6) + 2.0 * (b3 * b3));
  }
  free(u1b);
  free(u3b);
  /* |S| S_ij at GYF points; S_22 goes through the implicit eddy viscosity */
  LOOPP(JS, JE) {
    const long q = P_(j, k, i);
    S[0][q] = S1[q] * S[0][q];
    S[4][q] = S1[q] * S[4][q];
    S[1][q] = 0.0;
    S[2][q] = S1[q] * S[2][q];
  }
  /* |S| S_ij at GY points, without the dU1/dy, dU3/dy parts (implicit) */
  LOOPP(2, NY + 1) {
    const long q = P_(j, k, i), qm = P_(j - 1, k, i);
    S[3][q] = T[q] * (S[3][q] - 0.5 * (U1[q] - U1[qm]) / DY[j]);
    S[5][q] = T[q] * (S[5][q] - 0.5 * (U3[q] - U3[qm]) / DY[j]);
  }
  double *dyf_f = calloc(NY + 2, sizeof(double)), *dy_f = calloc(NY + 2, sizeof(double));
  for (int j = 1; j <= NY + 1; j++) {
    dyf_f[j] = delta_factor(o, DYF[j]);
    dy_f[j] = delta_factor(o, DY[j]);
  }
  /* NU_T = C_S^2 DELTA^2 |S| at GY points, then GHOST_LES_MPI (one rank) */
  LOOPP(2, NY) {
    const long q = P_(j, k, i);
    NUT[q] = -0.5 * dy_f[j] * T[q];
  }
  const long np = (long)NZ * NX;
  for (long q = 0; q < np; q++) {
    NUT[1 * np + q] = 0.0;
    NUT[2 * np + q] = 0.0;
    NUT[(long)NY * np + q] = 0.0;
    NUT[(long)(NY + 1) * np + q] = 0.0;
  }
  const int fwd[5] = {0, 2, 3, 4, 5};
  for (int c = 0; c < 5; c++) orc_fft_xz_to_fourier(o, S[fwd[c]], CS[fwd[c]], 0, NY + 1);
  LOOPS(1, NY + 1) {
    const long s = S_(j, k, i);
    CS[0][s] = dyf_f[j] * CS[0][s];
    CS[4][s] = dyf_f[j] * CS[4][s];
    CS[2][s] = dyf_f[j] * CS[2][s];
  }
  LOOPS(2, NY + 1) {
    const long s = S_(j, k, i);
    CS[3][s] = dy_f[j] * CS[3][s];
    CS[5][s] = dy_f[j] * CS[5][s];
  }
  free(dyf_f);
  free(dy_f);
  /* SGS stress divergence into CF1..CF3 (for/les.f:279-304) */
  LOOPS(J1, J2) {
    const long s = S_(j, k, i), sp = s + o->ss;
    o->CF1[s] = o->CF1[s] - o->CIKX[i] * CS[0][s] - (CS[3][sp] - CS[3][s]) / DYF[j] -
                o->CIKZ[k] * CS[4][s];
    o->CF3[s] = o->CF3[s] - o->CIKX[i] * CS[4][s] - (CS[5][sp] - CS[5][s]) / DYF[j] -
                o->CIKZ[k] * CS[2][s];
  }
  LOOPS(2, NY) {
    const long s = S_(j, k, i);
    o->CF2[s] = o->CF2[s] - o->CIKX[i] * CS[3][s] - o->CIKZ[k] * CS[5][s];
  }
  /* cross terms NU_T dU1/dy, NU_T dU3/dy at GY, explicit (for/les.f:306-333) */
  for (int c = 0; c < 2; c++) {
    const double *U = c == 0 ? U1 : U3;
    LOOPP(2, NY) {
      const long q = P_(j, k, i), qm = P_(j - 1, k, i);
      T[q] = NUT[q] * (U[q] - U[qm]) / DY[j];
    }
    orc_fft_xz_to_fourier(o, T, o->CTEMP, 2, NY);
    LOOPS(2, NY) {
      const long s = S_(j, k, i);
      o->CF2[s] = o->CF2[s] + (c == 0 ? o->CIKX[i] : o->CIKZ[k]) * o->CTEMP[s];
    }
  }
  if (o->les_stats_req) les_means(o, J1, J2);
#undef LOOPS
#undef LOOPP
#undef S_
#undef P_
}

/* Horizontal eddy diffusion of scalar n with KAPPA_T = NU_T, explicit
 * (for/channel.f:312-372): CFTH += ikx F(K_T F^-1(ikx CTH)) + ikz F(K_T F^-1(ikz CTH)). */
void orc_les_scalar_terms(orc *o, int n) {
  const int NY = o->NY, NX = o->NX, NZ = o->NZ, nkxp = o->nkxp, nkzt = o->nkzt;
  cplx *CTH = o->CTH[n], *CFTH = o->CFTH[n], *CS1 = o->CS1;
  double *S1 = o->S1, *NUT = o->NU_T;
  const int JSt = o->jstart_th[n], JEt = o->jend_th[n];
  for (int c = 0; c < 2; c++) {
    memset(CS1, 0, sizeof(cplx) * o->nspec);
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= NY + 1; j++)
      for (int k = 0; k < nkzt; k++)
        for (int i = 0; i < nkxp; i++) {
          const long s = SIDX(o, j, k, i);
          CS1[s] = (c == 0 ? o->CIKX[i] : o->CIKZ[k]) * CTH[s];
        }
    orc_fft_xz_to_physical(o, CS1, S1, 0, NY + 1);
#pragma omp parallel for schedule(static)
    for (int j = 1; j <= NY + 1; j++)
      for (int k = 0; k < NZ; k++)
        for (int i = 0; i < NX; i++) {
          const long q = PIDX(o, j, k, i);
          S1[q] = NUT[q] * S1[q];
        }
    orc_fft_xz_to_fourier(o, S1, CS1, 0, NY + 1);
#pragma omp parallel for schedule(static)
    for (int j = JSt; j <= JEt; j++)
      for (int k = 0; k < nkzt; k++)
        for (int i = 0; i < nkxp; i++) {
          const long s = SIDX(o, j, k, i);
          CFTH[s] = CFTH[s] + (c == 0 ? o->CIKX[i] : o->CIKZ[k]) * CS1[s];
        }
  }
}

int orc_get_nu_t(const orc *o, double *out) {
  if (!o->NU_T) return -1;
  memcpy(out, o->NU_T, sizeof(double) * o->nphys);
  return 0;
}

void orc_les_stats_request(orc *o) { o->les_stats_req = 1; }

int orc_les_stats(const orc *o, double *nu_t_mean, double *eps_sgs1_mean) {
  if (!o->les_stats_valid) return -1;
  memcpy(nu_t_mean, o->nu_t_mean, sizeof(double) * (o->NY + 2));
  memcpy(eps_sgs1_mean, o->eps_sgs1_mean, sizeof(double) * (o->NY + 2));
  return 0;
}

/* tkebudget_chan_les (for/save_stats.f:887-964), called by SAVE_STATS_CHAN
 * after its APPLY_BC_VEL and the transform of CU1..CU3: per plane J = 1..NY
 * the SUM (not the mean) over the points of U1 d(NU_T dU1/dy)/dy + U3 ... +
 * U2 d(NU_T dU2/dy)/dy with NU_T from the last LES substep.  DYF(0) is never
 * set in the reference (it stays 0), so the U2 term of J = 1 is 0/0. */
void orc_tkebudget_chan_les(orc *o, double *eps) {
  const int NY = o->NY;
  const long np = (long)o->NZ * o->NX;
  const double *DY = o->DY, *DYF = o->DYF, *NUT = o->NU_T;
  orc_apply_bc_vel(o);
  orc_fft_xz_to_physical(o, o->CU1, o->U1, 0, NY + 1);
  orc_fft_xz_to_physical(o, o->CU2, o->U2, 0, NY + 1);
  orc_fft_xz_to_physical(o, o->CU3, o->U3, 0, NY + 1);
  const double *U1 = o->U1, *U2 = o->U2, *U3 = o->U3;
  for (int j = 0; j <= NY + 1; j++) eps[j] = 0.0;
  for (int j = 1; j <= NY; j++) {
    double a = 0.0;
    for (long q = 0; q < np; q++) {
      const long c = j * np + q, p = c + np, m = c - np;
      const double t =
          U1[c] * ((NUT[p] * (U1[p] - U1[c]) / DY[j + 1] - NUT[c] * (U1[c] - U1[m]) / DY[j]) /
                   DYF[j]) +
          U3[c] * ((NUT[p] * (U3[p] - U3[c]) / DY[j + 1] - NUT[c] * (U3[c] - U3[m]) / DY[j]) /
                   DYF[j]) +
          U2[c] * ((0.5 * (NUT[c] + NUT[p]) * (U2[p] - U2[c]) / DYF[j] -
                    0.5 * (NUT[c] + NUT[m]) * (U2[c] - U2[m]) / DYF[j - 1]) /
                   DY[j]);
      a = a + t;
    }
    eps[j] = a;
  }
}
