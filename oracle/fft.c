/*
 * Oracle FFTs.  TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The reference delegates its transforms to FFTW 2.1.5 (not vendored; pinned
 * by docs/UsersGuideDiablo.pdf p.1 "tested using FFTW version 2.1.5"; call
 * sites for/fft.f:77-94,112-115,167,199,245,288 and for/mpi.f:1548,1585,1639,
 * 1670).  Published FFTW conventions restated here:
 *   - FFTW_FORWARD = -1 (for/fft.f:64): X[k] = sum_n x[n] exp(-2 pi i n k / N)
 *   - FFTW_BACKWARD = +1, unnormalised; DIABLO divides by NX, NZ (and NY)
 *     itself (for/mpi.f:1552,1589,1604; for/fft.f:249,252).
 *   - real-to-complex keeps bins 0..N/2; complex-to-real reads bins 0..N/2
 *     and ignores the imaginary parts of bins 0 and N/2 (FFTW's halfcomplex
 *     storage has no slot for them).
 * The algorithm is a textbook recursive mixed-radix decimation-in-time
 * Cooley-Tukey transform with an exact twiddle table; real transforms use
 * the "two real rows in one complex transform" identity.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle_int.h"

#define MAX_PLANS 16

typedef struct {
  int n;
  int nfac;
  int fac[64];            /* pairs (p, m) per recursion level */
  cplx *tw_fwd;           /* exp(-2 pi i k / n) */
  cplx *tw_inv;           /* exp(+2 pi i k / n) */
} plan_t;

static plan_t plans[MAX_PLANS];
static int nplans = 0;

static const plan_t *get_plan(int n) {
  for (int i = 0; i < nplans; i++)
    if (plans[i].n == n) return &plans[i];
  plan_t *pl;
#pragma omp critical(orc_fft_plan)
  {
    pl = NULL;
    for (int i = 0; i < nplans; i++)
      if (plans[i].n == n) pl = &plans[i];
    if (!pl) {
      pl = &plans[nplans];
      pl->n = n;
      pl->tw_fwd = (cplx *)malloc(sizeof(cplx) * n);
      pl->tw_inv = (cplx *)malloc(sizeof(cplx) * n);
      for (int k = 0; k < n; k++) {
        long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)k /
                        (long double)n;
        double c = (double)cosl(a), s = (double)sinl(a);
        pl->tw_fwd[k] = c - I * s;
        pl->tw_inv[k] = c + I * s;
      }
      /* factorise: prefer 4, then 2, 3, 5, then any prime */
      int m = n, nf = 0;
      while (m > 1) {
        int p;
        if (m % 4 == 0) p = 4;
        else if (m % 2 == 0) p = 2;
        else if (m % 3 == 0) p = 3;
        else if (m % 5 == 0) p = 5;
        else {
          p = 7;
          while (m % p) p += 2;
        }
        m /= p;
        pl->fac[2 * nf] = p;
        pl->fac[2 * nf + 1] = m;
        nf++;
      }
      pl->nfac = nf;
      __sync_synchronize();
      nplans++;
    }
  }
  return pl;
}

/* Butterfly of radix p on the m interleaved sub-transforms held in out. */
static void bfly(cplx *out, int f, const cplx *tw, int ntop, int m, int p, int sign) {
  if (p == 2) {
    for (int u = 0; u < m; u++) {
      cplx a = out[u];
      cplx b = out[u + m] * tw[(u * f) % ntop];
      out[u] = a + b;
      out[u + m] = a - b;
    }
  } else if (p == 4) {
    for (int u = 0; u < m; u++) {
      cplx y0 = out[u];
      cplx y1 = out[u + m] * tw[((long)u * f) % ntop];
      cplx y2 = out[u + 2 * m] * tw[((long)2 * u * f) % ntop];
      cplx y3 = out[u + 3 * m] * tw[((long)3 * u * f) % ntop];
      cplx s02 = y0 + y2, d02 = y0 - y2, s13 = y1 + y3, d13 = y1 - y3;
      /* multiply d13 by sign*i: forward uses exp(-i pi/2) = -i */
      cplx rd13 = (sign < 0) ? (cimag(d13) - I * creal(d13)) : (-cimag(d13) + I * creal(d13));
      out[u] = s02 + s13;
      out[u + m] = d02 + rd13;
      out[u + 2 * m] = s02 - s13;
      out[u + 3 * m] = d02 - rd13;
    }
  } else {
    cplx scratch[64];
    for (int u = 0; u < m; u++) {
      for (int q = 0; q < p; q++) scratch[q] = out[u + q * m];
      for (int t = 0; t < p; t++) {
        long k = u + (long)t * m;
        cplx acc = scratch[0];
        for (int q = 1; q < p; q++) acc += scratch[q] * tw[(q * k * f) % ntop];
        out[k] = acc;
      }
    }
  }
}

static void work(cplx *out, const cplx *in, int f, int istride, const int *fac, const cplx *tw,
                 int ntop, int sign) {
  const int p = fac[0], m = fac[1];
  if (m == 1) {
    for (int q = 0; q < p; q++) out[q] = in[(long)q * f * istride];
  } else {
    for (int q = 0; q < p; q++)
      work(out + (long)q * m, in + (long)q * f * istride, f * p, istride, fac + 2, tw, ntop, sign);
  }
  bfly(out, f, tw, ntop, m, p, sign);
}

/* out-of-place strided transform helper */
static void fft_oop(int n, const cplx *in, int istride, cplx *out, int sign) {
  const plan_t *pl = get_plan(n);
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  work(out, in, 1, istride, pl->fac, sign < 0 ? pl->tw_fwd : pl->tw_inv, n, sign);
}

void orc_fft1d(int n, cplx *data, int sign) {
  cplx *tmp = (cplx *)malloc(sizeof(cplx) * n);
  fft_oop(n, data, 1, tmp, sign);
  memcpy(data, tmp, sizeof(cplx) * n);
  free(tmp);
}

/* ------------------------------------------------------------------------
 * Real transforms of two rows at once.
 * r2c: z = a + i b, Z = DFT(z); A_k = (Z_k + conj Z_{N-k})/2,
 *      B_k = (Z_k - conj Z_{N-k})/(2i), k = 0..N/2.
 * c2r: Z_k = A_k + i B_k with the Hermitian extension of each; imaginary
 *      parts of bins 0 and N/2 ignored; a = Re IDFT(Z), b = Im IDFT(Z).
 * ---------------------------------------------------------------------- */
void orc_r2c_pair(int n, const double *a, const double *b, cplx *A, cplx *B, cplx *work_) {
  cplx *z = work_, *Z = work_ + n;
  for (int i = 0; i < n; i++) z[i] = a[i] + I * (b ? b[i] : 0.0);
  fft_oop(n, z, 1, Z, -1);
  for (int k = 0; k <= n / 2; k++) {
    cplx zk = Z[k], zm = conj(Z[(n - k) % n]);
    A[k] = 0.5 * (zk + zm);
    if (B) B[k] = -0.5 * I * (zk - zm);
  }
}

void orc_c2r_pair(int n, const cplx *A, const cplx *B, double *a, double *b, cplx *work_) {
  cplx *Z = work_, *z = work_ + n;
  for (int k = 0; k <= n / 2; k++) {
    cplx ak = A[k], bk = B ? B[k] : 0.0;
    if (k == 0 || 2 * k == n) {
      ak = creal(ak);
      bk = creal(bk);
    }
    Z[k] = ak + I * bk;
    if (k > 0 && 2 * k < n) Z[n - k] = conj(ak) + I * conj(bk);
  }
  fft_oop(n, Z, 1, z, +1);
  for (int i = 0; i < n; i++) {
    a[i] = creal(z[i]);
    if (b) b[i] = cimag(z[i]);
  }
}

/* ------------------------------------------------------------------------
 * FFT_XZ_TO_FOURIER for one plane (for/mpi.f:1530-1611 with NPROCZ = 1):
 *   r2c along x, divide bins 0..NKX by NX, drop NKX+1..NX/2;
 *   c2c along z (sign -1) per retained kx; divide by NZ; pack kz = 0..NKZ
 *   then -NKZ..-1 into NKZ+1..TNKZ.
 * ---------------------------------------------------------------------- */
void orc_plane_to_fourier(const orc *o, const double *phys, cplx *spec, cplx *wk) {
  const int NX = o->NX, NZ = o->NZ, NKX = o->NKX, NKZ = o->NKZ, nkxp = o->nkxp;
  cplx *T = wk;                            /* [NZ][nkxp] */
  cplx *A = T + (long)NZ * nkxp;           /* NX/2+1 */
  cplx *B = A + NX / 2 + 1;
  cplx *w = B + NX / 2 + 1;                /* 2*max(NX,NZ) */
  for (int z = 0; z < NZ; z += 2) {
    orc_r2c_pair(NX, phys + (long)z * NX, phys + (long)(z + 1) * NX, A, B, w);
    for (int i = 0; i <= NKX; i++) {
      T[(long)z * nkxp + i] = A[i] / (double)NX;
      T[(long)(z + 1) * nkxp + i] = B[i] / (double)NX;
    }
  }
  cplx *col = w + 2 * (NX > NZ ? NX : NZ);
  for (int i = 0; i <= NKX; i++) {
    fft_oop(NZ, T + i, nkxp, col, -1);
    for (int k = 0; k <= NKZ; k++) spec[(long)k * nkxp + i] = col[k] / (double)NZ;
    for (int k = 1; k <= NKZ; k++)
      spec[(long)(NKZ + k) * nkxp + i] = col[NZ - 1 + k - NKZ] / (double)NZ;
  }
}

/* FFT_XZ_TO_PHYSICAL for one plane (for/mpi.f:1613-1674):
 *   unpack kz, zero |kz| > NKZ, c2c along z (sign +1), zero kx > NKX and the
 *   x-Nyquist bin, c2r along x.  Unnormalised. */
void orc_plane_to_physical(const orc *o, const cplx *spec, double *phys, cplx *wk) {
  const int NX = o->NX, NZ = o->NZ, NKX = o->NKX, NKZ = o->NKZ, nkxp = o->nkxp;
  cplx *T = wk;                            /* [NZ][nkxp] */
  cplx *A = T + (long)NZ * nkxp;
  cplx *B = A + NX / 2 + 1;
  cplx *w = B + NX / 2 + 1;
  cplx *col = w + 2 * (NX > NZ ? NX : NZ);
  cplx *colo = col + NZ;
  for (int i = 0; i <= NKX; i++) {
    for (int k = 0; k < NZ; k++) col[k] = 0.0;
    for (int k = 0; k <= NKZ; k++) col[k] = spec[(long)k * nkxp + i];
    for (int k = 1; k <= NKZ; k++) col[NZ - 1 + k - NKZ] = spec[(long)(NKZ + k) * nkxp + i];
    fft_oop(NZ, col, 1, colo, +1);
    for (int k = 0; k < NZ; k++) T[(long)k * nkxp + i] = colo[k];
  }
  for (int z = 0; z < NZ; z += 2) {
    for (int i = 0; i <= NX / 2; i++) {
      A[i] = (i <= NKX) ? T[(long)z * nkxp + i] : 0.0;
      B[i] = (i <= NKX) ? T[(long)(z + 1) * nkxp + i] : 0.0;
    }
    A[NX / 2] = 0.0;
    B[NX / 2] = 0.0;
    orc_c2r_pair(NX, A, B, phys + (long)z * NX, phys + (long)(z + 1) * NX, w);
  }
}

long orc_plane_work_size(const orc *o) {
  int mx = o->NX > o->NZ ? o->NX : o->NZ;
  if (o->NY > mx) mx = o->NY;
  return (long)o->NZ * o->nkxp + 2 * (o->NX / 2 + 1) + 4 * mx + 2 * o->NZ + 16;
}

void orc_fft_xz_to_fourier(const orc *o, const double *phys, cplx *spec, int jmin, int jmax) {
  const long ps = (long)o->NZ * o->NX, ss = (long)o->nkzt * o->nkxp;
  const long wsz = orc_plane_work_size(o);
#pragma omp parallel
  {
    cplx *wk = (cplx *)malloc(sizeof(cplx) * wsz);
#pragma omp for schedule(static)
    for (int j = jmin; j <= jmax; j++) orc_plane_to_fourier(o, phys + j * ps, spec + j * ss, wk);
    free(wk);
  }
}

void orc_fft_xz_to_physical(const orc *o, const cplx *spec, double *phys, int jmin, int jmax) {
  const long ps = (long)o->NZ * o->NX, ss = (long)o->nkzt * o->nkxp;
  const long wsz = orc_plane_work_size(o);
#pragma omp parallel
  {
    cplx *wk = (cplx *)malloc(sizeof(cplx) * wsz);
#pragma omp for schedule(static)
    for (int j = jmin; j <= jmax; j++) orc_plane_to_physical(o, spec + j * ss, phys + j * ps, wk);
    free(wk);
  }
}

/* ------------------------------------------------------------------------
 * Triply periodic transforms (for/fft.f:223-299).  Spectral layout
 * [TNKY+1][TNKZ+1][NKX+1]; physical [NY][NZ][NX].
 *   to Fourier : FFT_XZ of planes 0..NY-1, then per (kx, kz) a c2c along y
 *                (sign -1), divide by NY, pack ky like kz.
 *   to physical: unpack ky (zero |ky| > NKY), c2c along y (sign +1), then
 *                FFT_XZ_TO_PHYSICAL of planes 0..NY-1.
 * The reference leaves stale values in kx > NKX between substeps on this
 * path (its FFT_XZ_TO_PHYSICAL does not zero them, for/mpi.f:1652-1655);
 * the documented packing contract (for/fft.f:48-50, "higher wavenumbers are
 * SET TO ZERO before the inverse transform") is followed here instead.
 * ---------------------------------------------------------------------- */
void orc_fft_xzy_to_fourier(const orc *o, const double *phys, cplx *spec) {
  const int NY = o->NY, NKY = o->NKY, nkxp = o->nkxp, nkzt = o->nkzt;
  const long ss = (long)nkzt * nkxp;
  cplx *tmp = (cplx *)malloc(sizeof(cplx) * ss * NY);
  orc_fft_xz_to_fourier(o, phys, tmp, 0, NY - 1);
#pragma omp parallel
  {
    cplx *col = (cplx *)malloc(sizeof(cplx) * 2 * NY);
#pragma omp for schedule(static)
    for (long m = 0; m < ss; m++) {
      fft_oop(NY, tmp + m, (int)ss, col, -1);
      for (int j = 0; j <= NKY; j++) spec[j * ss + m] = col[j] / (double)NY;
      for (int j = 1; j <= NKY; j++) spec[(NKY + j) * ss + m] = col[NY - 1 - NKY + j] / (double)NY;
    }
    free(col);
  }
  free(tmp);
}

void orc_fft_xzy_to_physical(const orc *o, const cplx *spec, double *phys) {
  const int NY = o->NY, NKY = o->NKY, nkxp = o->nkxp, nkzt = o->nkzt;
  const long ss = (long)nkzt * nkxp;
  cplx *tmp = (cplx *)malloc(sizeof(cplx) * ss * NY);
#pragma omp parallel
  {
    cplx *col = (cplx *)malloc(sizeof(cplx) * 2 * NY);
#pragma omp for schedule(static)
    for (long m = 0; m < ss; m++) {
      cplx *ci = col, *co = col + NY;
      for (int j = 0; j < NY; j++) ci[j] = 0.0;
      for (int j = 0; j <= NKY; j++) ci[j] = spec[j * ss + m];
      for (int j = 1; j <= NKY; j++) ci[NY - 1 - NKY + j] = spec[(NKY + j) * ss + m];
      fft_oop(NY, ci, 1, co, +1);
      for (int j = 0; j < NY; j++) tmp[j * ss + m] = co[j];
    }
    free(col);
  }
  orc_fft_xz_to_physical(o, tmp, phys, 0, NY - 1);
  free(tmp);
}
