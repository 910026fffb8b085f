/*
 * Oracle restatement of the triply periodic RK3 substep (for/periodic.f).
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Spectral layout [TNKY+1][TNKZ+1][NKX+1]; physical [NY][NZ][NX].
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle_int.h"

#define SIDX(o, j, k, i) ((long)(j) * (o)->ss + (long)(k) * (o)->nkxp + (i))
#define LOOPK                                                   \
  _Pragma("omp parallel for schedule(static)") for (int j = 0; j < o->nkyt; j++) \
    for (int k = 0; k < o->nkzt; k++) for (int i = 0; i < o->nkxp; i++)

static double ksq(const orc *o, int j, int k, int i) {
  return o->KX2[i] + o->KY2[j] + o->KZ2[k];
}

/* REM_DIV_PER, for/periodic.f:299-326 (phi left in CR1) */
void orc_rem_div_per(orc *o) {
  LOOPK {
    long c = SIDX(o, j, k, i);
    double t5 = -(o->KX2[i] + o->KY2[j] + o->KZ2[k] + o->eps);
    o->CR1[c] = (o->CIKX[i] * o->CU1[c] + o->CIKY[j] * o->CU2[c] + o->CIKZ[k] * o->CU3[c]) / t5;
    o->CU1[c] = o->CU1[c] - o->CIKX[i] * o->CR1[c];
    o->CU2[c] = o->CU2[c] - o->CIKY[j] * o->CR1[c];
    o->CU3[c] = o->CU3[c] - o->CIKZ[k] * o->CR1[c];
  }
}

/* POISSON_P_PER, for/periodic.f:329-393 */
void orc_poisson_p_per(orc *o) {
  const long np = o->nphys;
  LOOPK {
    long c = SIDX(o, j, k, i);
    o->CR1[c] = o->CIKX[i] * o->CU1[c];
    o->CR2[c] = o->CIKZ[k] * o->CU3[c];
  }
  orc_fft_xzy_to_physical(o, o->CR1, o->R1);
  orc_fft_xzy_to_physical(o, o->CR2, o->R2);
  double *P = o->S1;
  for (long q = 0; q < np; q++)
    P[q] = o->R1[q] * o->R1[q] + o->R1[q] * o->R2[q] + o->R2[q] * o->R2[q];
  LOOPK {
    long c = SIDX(o, j, k, i);
    o->CF1[c] = o->CIKY[j] * o->CU1[c];
    o->CF2[c] = o->CIKX[i] * o->CU2[c];
    o->CF3[c] = o->CIKZ[k] * o->CU1[c];
    o->CR1[c] = o->CIKX[i] * o->CU3[c];
    o->CR2[c] = o->CIKZ[k] * o->CU2[c];
    o->CR3[c] = o->CIKY[j] * o->CU3[c];
  }
  orc_fft_xzy_to_physical(o, o->CF1, o->F1);
  orc_fft_xzy_to_physical(o, o->CF2, o->F2);
  orc_fft_xzy_to_physical(o, o->CF3, o->F3);
  orc_fft_xzy_to_physical(o, o->CR1, o->R1);
  orc_fft_xzy_to_physical(o, o->CR2, o->R2);
  orc_fft_xzy_to_physical(o, o->CR3, o->R3);
  for (long q = 0; q < np; q++)
    P[q] = 2 * (P[q] + o->F1[q] * o->F2[q] + o->F3[q] * o->R1[q] + o->R2[q] * o->R3[q]);
  orc_fft_xzy_to_fourier(o, P, o->CP);
  LOOPK {
    long c = SIDX(o, j, k, i);
    o->CP[c] = o->CP[c] / (o->KX2[i] + o->KY2[j] + o->KZ2[k] + o->eps);
  }
  o->CP[0] = 0.0;
}

/* RK_PER_1, for/periodic.f:23-285 */
void orc_rk_per_1(orc *o, int rk_step) {
  const orc_params *p = &o->p;
  const int r = rk_step - 1;
  const double TEMP1 = p->nu * o->h_bar[r] / 2.0;
  const double TEMP2 = o->beta_bar[r] * o->h_bar[r];
  const double TEMP3 = o->zeta_bar[r] * o->h_bar[r];
  const double TEMP4 = o->h_bar[r];
  const long np = o->nphys;
  cplx *CU1 = o->CU1, *CU2 = o->CU2, *CU3 = o->CU3, *CP = o->CP;
  cplx *CR1 = o->CR1, *CR2 = o->CR2, *CR3 = o->CR3, *CF1 = o->CF1, *CF2 = o->CF2, *CF3 = o->CF3;
  cplx *CS1 = o->CS1;
  LOOPK {
    long c = SIDX(o, j, k, i);
    double t5 = 1 - TEMP1 * ksq(o, j, k, i);
    CR1[c] = t5 * CU1[c] - TEMP4 * (o->CIKX[i] * CP[c]);
    CR2[c] = t5 * CU2[c] - TEMP4 * (o->CIKY[j] * CP[c]);
    CR3[c] = t5 * CU3[c] - TEMP4 * (o->CIKZ[k] * CP[c]);
    for (int n = 0; n < o->NTH; n++) {
      double t6 = 1 - (TEMP1 / p->pr[n]) * ksq(o, j, k, i);
      o->CRTH[n][c] = t6 * o->CTH[n][c];
    }
    if (rk_step > 1) {
      CR1[c] = CR1[c] + TEMP3 * CF1[c];
      CR2[c] = CR2[c] + TEMP3 * CF2[c];
      CR3[c] = CR3[c] + TEMP3 * CF3[c];
      for (int n = 0; n < o->NTH; n++) o->CRTH[n][c] = o->CRTH[n][c] + TEMP3 * o->CFTH[n][c];
    }
  }
  for (int n = 0; n < o->NTH; n++) {
    if (p->background_grad[n]) {
      LOOPK { o->CFTH[n][SIDX(o, j, k, i)] = -CU2[SIDX(o, j, k, i)]; }
    } else {
      LOOPK { o->CFTH[n][SIDX(o, j, k, i)] = 0.0; }
    }
  }
  double *U1 = o->U1, *U2 = o->U2, *U3 = o->U3, *F1 = o->F1, *F2 = o->F2, *F3 = o->F3, *S1 = o->S1;
  orc_fft_xzy_to_physical(o, CU1, U1);
  orc_fft_xzy_to_physical(o, CU2, U2);
  orc_fft_xzy_to_physical(o, CU3, U3);
  for (int n = 0; n < o->NTH; n++) orc_fft_xzy_to_physical(o, o->CTH[n], o->TH[n]);
  for (int n = 0; n < o->NTH; n++) {
    const double *TH = o->TH[n];
    for (long q = 0; q < np; q++) {
      F1[q] = U1[q] * TH[q];
      F2[q] = U2[q] * TH[q];
      F3[q] = U3[q] * TH[q];
    }
    orc_fft_xzy_to_fourier(o, F1, CF1);
    orc_fft_xzy_to_fourier(o, F2, CF2);
    orc_fft_xzy_to_fourier(o, F3, CF3);
    LOOPK {
      long c = SIDX(o, j, k, i);
      o->CFTH[n][c] = o->CFTH[n][c] - o->CIKX[i] * CF1[c] - o->CIKY[j] * CF2[c] - o->CIKZ[k] * CF3[c];
    }
  }
  for (long q = 0; q < np; q++) {
    F1[q] = U1[q] * U1[q];
    F2[q] = U1[q] * U2[q];
    F3[q] = U1[q] * U3[q];
    S1[q] = U2[q] * U2[q];
  }
  orc_fft_xzy_to_fourier(o, F1, CF1);
  orc_fft_xzy_to_fourier(o, F2, CF2);
  orc_fft_xzy_to_fourier(o, F3, CF3);
  orc_fft_xzy_to_fourier(o, S1, CS1);
  LOOPK {
    long c = SIDX(o, j, k, i);
    cplx f1 = CF1[c], f2 = CF2[c], f3 = CF3[c], s1 = CS1[c];
    CF1[c] = -o->CIKX[i] * f1 - o->CIKY[j] * f2 - o->CIKZ[k] * f3;
    CF2[c] = -o->CIKX[i] * f2 - o->CIKY[j] * s1;
    CF3[c] = -o->CIKX[i] * f3;
  }
  for (long q = 0; q < np; q++) S1[q] = U2[q] * U3[q];
  orc_fft_xzy_to_fourier(o, S1, CS1);
  LOOPK {
    long c = SIDX(o, j, k, i);
    CF2[c] = CF2[c] - o->CIKZ[k] * CS1[c];
    CF3[c] = CF3[c] - o->CIKY[j] * CS1[c];
  }
  for (long q = 0; q < np; q++) S1[q] = U3[q] * U3[q];
  orc_fft_xzy_to_fourier(o, S1, CS1);
  LOOPK {
    long c = SIDX(o, j, k, i);
    CF3[c] = CF3[c] - o->CIKZ[k] * CS1[c];
  }
  /* USER_RHS_PER_PHYSICAL (for/user_rhs.f:124-194); it adds exactly zero when
   * EPSILON_TARGET = 0, which is the decaying case */
  if (p->epsilon_target != 0.0) {
    double ek = 0.0;
    for (long q = 0; q < np; q++) ek = ek + U1[q] * U1[q] + U2[q] * U2[q] + U3[q] * U3[q];
    ek = ek / (double)((long)o->NX * o->NY * o->NZ);
    ek = 0.8 * ek;
    const double *Us[3] = {U1, U2, U3};
    cplx *CFs[3] = {CF1, CF2, CF3};
    for (int d = 0; d < 3; d++) {
      for (long q = 0; q < np; q++) S1[q] = (p->epsilon_target / ek) * Us[d][q];
      orc_fft_xzy_to_fourier(o, S1, CS1);
      cplx *CF = CFs[d];
      LOOPK {
        long c = SIDX(o, j, k, i);
        CF[c] = CF[c] + CS1[c];
      }
    }
  }
  for (int n = 0; n < o->NTH; n++) {
    orc_fft_xzy_to_fourier(o, o->TH[n], o->CTH[n]);
    LOOPK {
      long c = SIDX(o, j, k, i);
      CF2[c] = CF2[c] + p->ri[n] * o->CTH[n][c];
    }
  }
  LOOPK {
    long c = SIDX(o, j, k, i);
    CR1[c] = CR1[c] + TEMP2 * CF1[c];
    CR2[c] = CR2[c] + TEMP2 * CF2[c];
    CR3[c] = CR3[c] + TEMP2 * CF3[c];
    for (int n = 0; n < o->NTH; n++) o->CRTH[n][c] = o->CRTH[n][c] + TEMP2 * o->CFTH[n][c];
  }
  LOOPK {
    long c = SIDX(o, j, k, i);
    double t5 = 1 + TEMP1 * ksq(o, j, k, i);
    CU1[c] = CR1[c] / t5;
    CU2[c] = CR2[c] / t5;
    CU3[c] = CR3[c] / t5;
    for (int n = 0; n < o->NTH; n++) {
      double t6 = 1 + (TEMP1 / p->pr[n]) * ksq(o, j, k, i);
      o->CTH[n][c] = o->CRTH[n][c] / t6;
    }
  }
  orc_rem_div_per(o);
  LOOPK {
    long c = SIDX(o, j, k, i);
    CP[c] = CP[c] + CR1[c] / TEMP4;
  }
}

void orc_create_flow_per(orc *o, const double *u1, const double *u2, const double *u3) {
  orc_fft_xzy_to_fourier(o, u1, o->CU1);
  orc_fft_xzy_to_fourier(o, u2, o->CU2);
  orc_fft_xzy_to_fourier(o, u3, o->CU3);
  memset(o->CF1, 0, sizeof(cplx) * o->nspec);
  memset(o->CF2, 0, sizeof(cplx) * o->nspec);
  memset(o->CF3, 0, sizeof(cplx) * o->nspec);
  orc_rem_div_per(o);
  orc_poisson_p_per(o);
}

double orc_div_max_per(const orc *o) {
  cplx *d = calloc(o->nspec, sizeof(cplx));
  double *ph = calloc(o->nphys, sizeof(double));
  for (int j = 0; j < o->nkyt; j++)
    for (int k = 0; k < o->nkzt; k++)
      for (int i = 0; i < o->nkxp; i++) {
        long c = SIDX(o, j, k, i);
        d[c] = o->CIKX[i] * o->CU1[c] + o->CIKY[j] * o->CU2[c] + o->CIKZ[k] * o->CU3[c];
      }
  orc_fft_xzy_to_physical(o, d, ph);
  double mx = 0;
  for (long q = 0; q < o->nphys; q++)
    if (fabs(ph[q]) > mx) mx = fabs(ph[q]);
  free(d);
  free(ph);
  return mx;
}

void orc_stats_per(const orc *o, orc_stats *s) {
  memset(s, 0, sizeof(*s));
  const long np = o->nphys;
  double *u = malloc(sizeof(double) * np);
  const cplx *f[3] = {o->CU1, o->CU2, o->CU3};
  double rms[3], e = 0;
  for (int d = 0; d < 3; d++) {
    orc_fft_xzy_to_physical(o, f[d], u);
    double a = 0;
    for (long q = 0; q < np; q++) a += u[q] * u[q];
    rms[d] = sqrt(a / (double)np);
    e += a;
  }
  s->urms_b = rms[0];
  s->vrms_b = rms[1];
  s->wrms_b = rms[2];
  s->ke = 0.5 * e / (double)np;
  for (int n = 0; n < o->NTH && n < ORC_MAX_TH; n++) {
    orc_fft_xzy_to_physical(o, o->CTH[n], u);
    double a = 0, m = creal(o->CTH[n][0]);
    for (long q = 0; q < np; q++) a += (u[q] - m) * (u[q] - m);
    s->th_var[n] = a / (double)np;
    s->thrms_b[n] = sqrt(s->th_var[n]);
  }
  s->div_max = orc_div_max_per(o);
  free(u);
}
