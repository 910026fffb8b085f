/* Internal state of the CPU oracle.  TEST INFRASTRUCTURE ONLY (see oracle.h). */
#ifndef DIABLO_ORACLE_INT_H
#define DIABLO_ORACLE_INT_H

#include <complex.h>
#include "oracle.h"

typedef double complex cplx;

struct orc {
  orc_params p;
  int NX, NY, NZ, NTH, NXP, NKX, NKZ, TNKZ, NKY, TNKY;
  int nkxp, nkzt, nkyt;      /* NKX+1, TNKZ+1, TNKY+1 */
  long ss;                   /* spectral plane size nkxp*nkzt */
  long nspec;                /* complex elements per spectral field */
  long nphys;                /* doubles per physical field */
  double pi;
  /* grid (NY+2 each; channel) */
  double *GY, *GYF, *DY, *DYF;
  double DX, DZ;
  /* wavenumbers */
  double *KX, *KZ, *KY, *KX2, *KZ2, *KY2;
  cplx *CIKX, *CIKZ, *CIKY;
  double eps;
  /* RK3 */
  double h_bar[3], beta_bar[3], zeta_bar[3];
  double time, delta_t;
  int jstart, jend, jstart_th[ORC_MAX_TH], jend_th[ORC_MAX_TH];
  /* spectral fields */
  cplx *CU1, *CU2, *CU3, *CP, *CF1, *CF2, *CF3, *CR1, *CR2, *CR3, *CS1;
  cplx *CTH[ORC_MAX_TH], *CFTH[ORC_MAX_TH], *CRTH[ORC_MAX_TH];
  /* physical fields */
  double *U1, *U2, *U3, *R1, *R2, *R3, *S1, *F1, *F2, *F3;
  double *TH[ORC_MAX_TH], *RTH[ORC_MAX_TH];
  /* LES (allocated when p.les): NU_T at GY points, S_ij / CS_ij, TEMP / CTEMP */
  double *NU_T, *Sij[6], *TEMP;
  cplx *CSij[6], *CTEMP;
  int les_stats_req, les_stats_valid;
  double *nu_t_mean, *eps_sgs1_mean;   /* [NY+2] each */
};

void orc_r2c_pair(int n, const double *a, const double *b, cplx *A, cplx *B, cplx *work);
void orc_c2r_pair(int n, const cplx *A, const cplx *B, double *a, double *b, cplx *work);
void orc_plane_to_fourier(const orc *o, const double *phys, cplx *spec, cplx *wk);
void orc_plane_to_physical(const orc *o, const cplx *spec, double *phys, cplx *wk);
long orc_plane_work_size(const orc *o);
void orc_les_chan(orc *o);
void orc_les_scalar_terms(orc *o, int n);
void orc_apply_bc_vel_phys(orc *o);

#endif
