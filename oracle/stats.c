/* Channel flow statistics: SAVE_STATS_CHAN and tkebudget_chan.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * A literal physical-space restatement: the velocity, scalar and derivative
 * fields are taken to physical space with FFT_XZ_TO_PHYSICAL and the plane
 * sums run over the NX x NZ points, in the reference's order.  The state is
 * changed only by the APPLY_BC_VEL the reference runs first; the reference's
 * closing physical -> Fourier round trip of CU and CTH (a round-off-level
 * change) is not repeated. */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_int.h"

#define SIDX(o, j, k, i) ((long)(j) * (o)->ss + (long)(k) * (o)->nkxp + (i))

/* INTEGRATE_Y_VAR (for/mpi.f:1676-1698) */
static double integ_y(const orc *o, const double *v) {
  double res = 0.;
  for (int j = 2; j <= o->NY; j++) res = res + 0.5 * (v[j] + v[j - 1]) * o->DY[j];
  return res / o->p.ly;
}

/* derived spectral field on planes 1..NY (0 and NY+1 zero), to physical */
typedef cplx (*mode_fn)(const orc *o, int j, int k, int i, const void *arg);

static void derived_phys(const orc *o, mode_fn fn, const void *arg, cplx *cs, double *ph) {
  const int NY = o->NY;
  memset(cs, 0, sizeof(cplx) * o->nspec);
  for (int j = 1; j <= NY; j++)
    for (int k = 0; k <= o->TNKZ; k++)
      for (int i = 0; i < o->nkxp; i++) cs[SIDX(o, j, k, i)] = fn(o, j, k, i, arg);
  orc_fft_xz_to_physical(o, cs, ph, 0, NY + 1);
}

static cplx f_ikx(const orc *o, int j, int k, int i, const void *a) {
  return o->CIKX[i] * ((const cplx *)a)[SIDX(o, j, k, i)];
}
static cplx f_ikz(const orc *o, int j, int k, int i, const void *a) {
  return o->CIKZ[k] * ((const cplx *)a)[SIDX(o, j, k, i)];
}
/* omega_x (for/save_stats.f:268-272) */
static cplx f_omx(const orc *o, int j, int k, int i, const void *a) {
  const long c = SIDX(o, j, k, i), s = o->ss;
  return (o->CU3[c + s] - o->CU3[c - s]) / (2.0 * o->DYF[j]) -
         o->CIKZ[k] * 0.5 * (o->CU2[c + s] + o->CU2[c]);
  (void)a;
}
/* omega_y (for/save_stats.f:296-300) */
static cplx f_omy(const orc *o, int j, int k, int i, const void *a) {
  const long c = SIDX(o, j, k, i);
  (void)a;
  return o->CIKZ[k] * o->CU1[c] - o->CIKX[i] * o->CU3[c];
}
/* omega_z (for/save_stats.f:324-329) */
static cplx f_omz(const orc *o, int j, int k, int i, const void *a) {
  const long c = SIDX(o, j, k, i), s = o->ss;
  (void)a;
  return o->CIKX[i] * 0.5 * (o->CU2[c + s] + o->CU2[c]) -
         (o->CU1[c + s] - o->CU1[c - s]) / (2.0 * o->DYF[j]);
}
/* scalar y-gradient (for/save_stats.f:470) */
static cplx f_thy(const orc *o, int j, int k, int i, const void *a) {
  const cplx *t = (const cplx *)a;
  const long c = SIDX(o, j, k, i), s = o->ss;
  return (t[c + s] - t[c - s]) / (o->GYF[j + 1] - o->GYF[j - 1]);
}

void orc_save_stats_chan(orc *o, double *prof, double *prof_th, double *bulk) {
  const int NY = o->NY, NX = o->NX, NZ = o->NZ, NTH = o->NTH;
  const long L = NY + 2, np = (long)NX * NZ;
  const double nxz = (double)NZ * (double)NX;
  const double *DY = o->DY, *DYF = o->DYF, *GYF = o->GYF, *GY = o->GY;
#define PR(q, j) prof[(long)(q) * L + (j)]
  memset(prof, 0, sizeof(double) * ORC_PR_COUNT * L);
  if (prof_th) memset(prof_th, 0, sizeof(double) * ORC_PRT_COUNT * L * NTH);

  /* for/save_stats.f:24-36 */
  orc_apply_bc_vel(o);

  /* centerline velocity (:88-96) and the bulk velocity (:117-124) */
  const int jh = NY / 2;
  bulk[1] = (NY % 2 == 0) ? creal(o->CU1[SIDX(o, jh, 0, 0)])
                          : 0.5 * (creal(o->CU1[SIDX(o, jh - 1, 0, 0)]) +
                                   creal(o->CU1[SIDX(o, jh, 0, 0)]));
  double *ume = calloc(L, sizeof(double)), *vme = calloc(L, sizeof(double)),
         *wme = calloc(L, sizeof(double)), *tmp = calloc(L, sizeof(double));
  for (int j = 0; j < L; j++) {
    ume[j] = creal(o->CU1[SIDX(o, j, 0, 0)]);
    vme[j] = creal(o->CU2[SIDX(o, j, 0, 0)]);
    wme[j] = creal(o->CU3[SIDX(o, j, 0, 0)]);
    PR(ORC_PR_UME, j) = ume[j];
    PR(ORC_PR_VME, j) = vme[j];
    PR(ORC_PR_WME, j) = wme[j];
    PR(ORC_PR_CP, j) = creal(o->CP[SIDX(o, j, 0, 0)]);
  }
  bulk[0] = integ_y(o, ume);

  /* physical velocity (:163-165) */
  double *U1 = malloc(sizeof(double) * o->nphys), *U2 = malloc(sizeof(double) * o->nphys),
         *U3 = malloc(sizeof(double) * o->nphys), *S1 = malloc(sizeof(double) * o->nphys);
  cplx *CS = malloc(sizeof(cplx) * o->nspec);
  orc_fft_xz_to_physical(o, o->CU1, U1, 0, NY + 1);
  orc_fft_xz_to_physical(o, o->CU2, U2, 0, NY + 1);
  orc_fft_xz_to_physical(o, o->CU3, U3, 0, NY + 1);
#define AT(a, j, q) (a)[(long)(j) * np + (q)]

  /* tkebudget_chan (:963-1173): the pseudo-dissipation on GY points */
  double *eps = calloc(L, sizeof(double));
  /* du/dx, interpolated */
  derived_phys(o, f_ikx, o->CU1, CS, S1);
  for (int j = 1; j <= NY; j++)
    for (long q = 0; q < np; q++)
      eps[j] = eps[j] + (DYF[j - 1] * AT(S1, j, q) * AT(S1, j, q) +
                         DYF[j] * AT(S1, j - 1, q) * AT(S1, j - 1, q)) / (2.0 * DY[j]);
  /* dv/dx */
  derived_phys(o, f_ikx, o->CU2, CS, S1);
  for (int j = 1; j <= NY; j++)
    for (long q = 0; q < np; q++) eps[j] = eps[j] + AT(S1, j, q) * AT(S1, j, q);
  /* du/dy at GY, mean removed */
  for (int j = 1; j <= NY; j++)
    for (long q = 0; q < np; q++)
      AT(S1, j, q) = ((AT(U1, j, q) - ume[j]) - (AT(U1, j - 1, q) - ume[j - 1])) / DY[j];
  for (int j = 1; j <= NY; j++)
    for (long q = 0; q < np; q++) eps[j] = eps[j] + AT(S1, j, q) * AT(S1, j, q);
  /* dw/dx, interpolated */
  derived_phys(o, f_ikx, o->CU3, CS, S1);
  for (int j = 1; j <= NY; j++)
    for (long q = 0; q < np; q++)
      eps[j] = eps[j] + (DYF[j - 1] * AT(S1, j, q) * AT(S1, j, q) +
                         DYF[j] * AT(S1, j - 1, q) * AT(S1, j - 1, q)) / (2.0 * DY[j]);
  /* du/dz, interpolated */
  derived_phys(o, f_ikz, o->CU1, CS, S1);
  for (int j = 1; j <= NY; j++)
    for (long q = 0; q < np; q++)
      eps[j] = eps[j] + (DYF[j - 1] * AT(S1, j, q) * AT(S1, j, q) +
                         DYF[j] * AT(S1, j - 1, q) * AT(S1, j - 1, q)) / (2.0 * DY[j]);
  /* dv/dy on j = 2..NY-1 (rows 1 and NY keep the previous S1: du/dz) */
  for (int j = 2; j <= NY - 1; j++)
    for (long q = 0; q < np; q++)
      AT(S1, j, q) = ((AT(U2, j + 1, q) - vme[j]) - (AT(U2, j - 1, q) - vme[j - 1])) /
                     (GY[j + 1] - GY[j - 1]);
  for (int j = 1; j <= NY; j++)
    for (long q = 0; q < np; q++) eps[j] = eps[j] + AT(S1, j, q) * AT(S1, j, q);
  /* dw/dy at GY, mean removed */
  for (int j = 1; j <= NY; j++)
    for (long q = 0; q < np; q++)
      AT(S1, j, q) = ((AT(U3, j, q) - wme[j]) - (AT(U3, j - 1, q) - wme[j - 1])) / DY[j];
  for (int j = 1; j <= NY; j++)
    for (long q = 0; q < np; q++) eps[j] = eps[j] + AT(S1, j, q) * AT(S1, j, q);
  /* dv/dz */
  derived_phys(o, f_ikz, o->CU2, CS, S1);
  for (int j = 1; j <= NY; j++)
    for (long q = 0; q < np; q++) eps[j] = eps[j] + AT(S1, j, q) * AT(S1, j, q);
  /* dw/dz, interpolated */
  derived_phys(o, f_ikz, o->CU3, CS, S1);
  for (int j = 1; j <= NY; j++)
    for (long q = 0; q < np; q++)
      eps[j] = eps[j] + (DYF[j - 1] * AT(S1, j, q) * AT(S1, j, q) +
                         DYF[j] * AT(S1, j - 1, q) * AT(S1, j - 1, q)) / (2.0 * DY[j]);
  /* the reference writes rows 2..NY-1 (tke.txt); rows 1 and NY read
   * scratch planes the reference leaves unset */
  for (int j = 2; j <= NY - 1; j++) PR(ORC_PR_EPSILON, j) = o->p.nu * eps[j] / (double)(NX * NZ);

  /* rms velocities (:168-197) */
  for (int j = 1; j <= NY; j++) {
    double a = 0., b = 0., c = 0.;
    for (long q = 0; q < np; q++) {
      a = a + pow(AT(U1, j, q) - ume[j], 2.);
      b = b + 0.5 * (pow(AT(U2, j, q) - vme[j], 2.) + pow(AT(U2, j + 1, q) - vme[j + 1], 2.));
      c = c + pow(AT(U3, j, q) - wme[j], 2.);
    }
    PR(ORC_PR_URMS, j) = sqrt(a / nxz);
    PR(ORC_PR_VRMS, j) = sqrt(b / nxz);
    PR(ORC_PR_WRMS, j) = sqrt(c / nxz);
  }
  for (int j = 0; j < L; j++) tmp[j] = PR(ORC_PR_URMS, j);
  bulk[2] = integ_y(o, tmp);
  for (int j = 0; j < L; j++) tmp[j] = PR(ORC_PR_VRMS, j);
  bulk[3] = integ_y(o, tmp);
  for (int j = 0; j < L; j++) tmp[j] = PR(ORC_PR_WRMS, j);
  bulk[4] = integ_y(o, tmp);

  /* Reynolds stresses (:205-235): uv and wv on GY, uw on GYF */
  for (int j = 1; j <= NY; j++) {
    double uv = 0., wv = 0., uw = 0.;
    for (long q = 0; q < np; q++) {
      uv = uv + (DYF[j - 1] * (AT(U1, j, q) - ume[j]) + DYF[j] * (AT(U1, j - 1, q) - ume[j - 1])) /
                    (2.0 * DY[j]) * (AT(U2, j, q) - vme[j]);
      wv = wv + (DYF[j - 1] * (AT(U3, j, q) - wme[j]) + DYF[j] * (AT(U3, j - 1, q) - wme[j - 1])) /
                    (2.0 * DY[j]) * (AT(U2, j, q) - vme[j]);
      uw = uw + (AT(U1, j, q) - ume[j]) * (AT(U3, j, q) - wme[j]);
    }
    PR(ORC_PR_UV, j) = uv / nxz;
    PR(ORC_PR_WV, j) = wv / nxz;
    PR(ORC_PR_UW, j) = uw / nxz;
  }
  /* mean gradients on GY (:238-241) */
  for (int j = 1; j <= NY; j++) {
    PR(ORC_PR_DUDY, j) = (ume[j] - ume[j - 1]) / (GYF[j] - GYF[j - 1]);
    PR(ORC_PR_DWDY, j) = (wme[j] - wme[j - 1]) / (GYF[j] - GYF[j - 1]);
  }
  /* mean square shear (:244-258) */
  for (int j = 1; j <= NY; j++) {
    double s = 0.;
    for (long q = 0; q < np; q++)
      s = s + pow((AT(U1, j + 1, q) - AT(U1, j - 1, q)) / (2.0 * DYF[j]), 2.) +
          pow((AT(U3, j + 1, q) - AT(U3, j - 1, q)) / (2.0 * DYF[j]), 2.);
    PR(ORC_PR_SHEAR, j) = s / (double)(NX * NZ);
  }
  /* rms vorticity (:266-348) */
  mode_fn om[3] = {f_omx, f_omy, f_omz};
  for (int c = 0; c < 3; c++) {
    derived_phys(o, om[c], NULL, CS, S1);
    for (int j = 1; j <= NY; j++) {
      double s = 0.;
      for (long q = 0; q < np; q++) s = s + pow(AT(S1, j, q), 2.);
      PR(ORC_PR_OMEGA_X + c, j) = sqrt(s / ((double)NX * (double)NZ));
    }
  }

  /* scalars (:452-560) */
  double *R1 = malloc(sizeof(double) * o->nphys), *R2 = malloc(sizeof(double) * o->nphys),
         *R3 = malloc(sizeof(double) * o->nphys), *TH = malloc(sizeof(double) * o->nphys);
  for (int n = 0; n < NTH && prof_th; n++) {
    double *T = prof_th + (long)n * ORC_PRT_COUNT * L;
    const cplx *ct = o->CTH[n];
    double *thme = tmp;
    for (int j = 0; j < L; j++) thme[j] = creal(ct[SIDX(o, j, 0, 0)]);
    derived_phys(o, f_ikx, ct, CS, R1);
    derived_phys(o, f_thy, ct, CS, R2);
    derived_phys(o, f_ikz, ct, CS, R3);
    orc_fft_xz_to_physical(o, ct, TH, 0, NY + 1);
    for (int j = 1; j <= NY; j++) {
      double a = 0., v = 0., pe = 0.;
      for (long q = 0; q < np; q++) {
        a = a + pow(fabs(AT(TH, j, q) - thme[j]), 2.);
        v = v + (AT(TH, j, q) - thme[j]) * (0.5 * (AT(U2, j, q) + AT(U2, j + 1, q)) -
                                            0.5 * (vme[j] + vme[j + 1]));
        pe = pe + pow(AT(R1, j, q), 2.) + pow(AT(R2, j, q), 2.) + pow(AT(R3, j, q), 2.);
      }
      T[ORC_PRT_THME * L + j] = thme[j];
      T[ORC_PRT_THRMS * L + j] = sqrt(a / nxz);
      T[ORC_PRT_THV * L + j] = v / nxz;
      T[ORC_PRT_DTHDY * L + j] = (thme[j] - thme[j - 1]) / (GYF[j] - GYF[j - 1]);
      T[ORC_PRT_PE_DISS * L + j] = pe / (double)(NX * NZ);
    }
    T[ORC_PRT_THME * L + 0] = thme[0];
    T[ORC_PRT_THME * L + NY + 1] = thme[NY + 1];
  }
#undef AT
#undef PR
  free(R1);
  free(R2);
  free(R3);
  free(TH);
  free(U1);
  free(U2);
  free(U3);
  free(S1);
  free(CS);
  free(eps);
  free(ume);
  free(vme);
  free(wme);
  free(tmp);
}

/* running means of SAVE_STATS_CHAN (:99-114): the weights are REAL*4
 * expressions, 1./FLOAT(NSAMPLES) and (FLOAT(NSAMPLES)-1.)/FLOAT(NSAMPLES) */
void orc_stats_means_update(const orc *o, int nsamples, double *ubar, double *vbar,
                            double *wbar, double *thbar) {
  const float fn = (float)nsamples;
  const double w1 = (double)(1.0f / fn), w2 = (double)((fn - 1.0f) / fn);
  const long L = o->NY + 2;
  for (int j = 1; j <= o->NY; j++) {
    ubar[j] = w1 * creal(o->CU1[SIDX(o, j, 0, 0)]) + w2 * ubar[j];
    vbar[j] = w1 * creal(o->CU2[SIDX(o, j, 0, 0)]) + w2 * vbar[j];
    wbar[j] = w1 * creal(o->CU3[SIDX(o, j, 0, 0)]) + w2 * wbar[j];
    for (int n = 0; n < o->NTH; n++)
      thbar[n * L + j] = w1 * creal(o->CTH[n][SIDX(o, j, 0, 0)]) + w2 * thbar[n * L + j];
  }
}
