// The per-mode column stage of RK_CHAN_1: explicit terms and the
// Crank-Nicolson right-hand side, the CN solves, and REM_DIV_CHAN with the
// pressure update, for a tile of MT retained (kx, kz) modes and their whole
// y-columns.
//
// Reference steps it replaces, per mode instead of per physical column (the
// operators are linear and the same for every column, so they commute with
// the x-z transform):
//   RHS assembly     for/channel.f:88-167   CR = CU + zeta h CF - h grad P
//   explicit terms   for/channel.f:175-290  CF = -nu k^2 CU + Coriolis,
//                                           buoyancy, GRAV, DRHODX/Z + NL
//   CN explicit half for/channel.f:580-626  R += beta h CF + (nu h/2) d2/dy2 CU
//   CN solves        for/channel.f:771-1029 (THOMAS_*_MPI, for/mpi.f:630-866)
//   REM_DIV_CHAN     for/channel.f:1103-1214, CP += phi / h :1059-1065
//
// Two forms (DG_TUNE_COL_FUSED):
//   split (0): one CTA per (mode tile, field) forms that field's right-hand
//              sides and solves its CN systems, writing the post-CN field;
//              REM_DIV follows as its own launch (k_rd_col).  Every field's
//              sweep runs in its own CTA, so the y-recurrences of a substep
//              spread over three times as many CTAs.
//   fused (1): one CTA per mode tile does every field and then REM_DIV: no
//              round trip of the post-CN velocity, but each CTA runs the CN
//              and the REM_DIV recurrences one after the other.
// The autotuner picks per grid shape.  Both do the same arithmetic per mode
// except for the REM_DIV divergence, which each compiles on its own (results
// agree to round-off).  The split form writes each field as soon as its CTA
// has solved it, so it is used only when no field's right-hand side reads
// another field (no rotation, no buoyancy or GRAV terms, no DRHODX/Z);
// otherwise the fused form runs, which stages every field before it writes
// any.
//
// Layout: every field is [NY+2][ss] complex, modes kx fastest; a CTA owns
// modes m0 .. m0+MT-1.  The CU tiles (all planes x MT modes) arrive by bulk
// tensor copies (TMA, no multicast) on one mbarrier with a bounded wait; the
// nonlinear terms NL (written by the z-forward kernel into the rhs arrays),
// CF and CP are read with plain coalesced loads while the right-hand sides
// are formed.  The right-hand sides, then the CN solutions, live in a second
// set of shared tiles; the CN and REM_DIV row tables are staged in shared
// memory so the sequential sweeps touch nothing else.  Every phase loops
// field by field, so the field's constants and pointers are uniform across
// the CTA.
#include <string.h>

#include <algorithm>
#include <vector>

#include "dg_internal.cuh"

namespace {

constexpr int CS_THR = 128;

struct ColConst {
  int NY, nf, nth, nkxp, JS, JE;
  int JSt[DG_MAX_TH], JEt[DG_MAX_TH];
  long ss;
  double nu, beta, nuv, i_ro, grav_x, grav_y, grav_z, px0, omega0, amp_omega0;
  int f_type;
  double ri[DG_MAX_TH], pr[DG_MAX_TH], drhodx[DG_MAX_TH], drhodz[DG_MAX_TH];
};

// Everything the column stage of one case needs.  The single-case launch
// passes it as a __grid_constant__ parameter; the ragged launch reads it from
// a device array (tensor maps first: 64-byte aligned in either place).
struct ColCase {
  CUtensorMap maps[3 + DG_MAX_TH];  // CU of every field, [plane][2 ss doubles]
  ColConst C;
  const double *dscal, *tab, *kxv, *kzv, *rowc, *ra, *rrb;
  double2 *cu[3 + DG_MAX_TH], *cf[3 + DG_MAX_TH];
  const double2 *nl[3 + DG_MAX_TH];
  double2 *cp, *phi;
  int *err;
  int by, nbox;
  int rd;  // fused form: 1 REM_DIV in the kernel; 0 stop after the CN solves
};

// per-CTA header in shared memory: the case's field pointers, read once
struct Hdr {
  double2 *cu[3 + DG_MAX_TH], *cf[3 + DG_MAX_TH];
  const double2 *nl[3 + DG_MAX_TH];
};

template <typename T>
__device__ __forceinline__ T pick(const T (&a)[DG_MAX_TH], int i) {
  T r = a[0];
#pragma unroll
  for (int k = 1; k < DG_MAX_TH; k++) r = (i == k) ? a[k] : r;
  return r;
}

// rowc: per-row grid factors [8][NY+2]
//   0 1/(DY(j+1) DYF(j))  1 1/(DY(j) DYF(j))       (GYF rows: U1, U3, TH)
//   2 1/(DYF(j) DY(j))    3 1/(DYF(j-1) DY(j))     (GY rows: U2)
//   4 1/DY(j)             5 1/DYF(j)               6 REM_DIV upper diagonal
//   7 DYF(j)
//
// The column stage of modes m0 .. m0+MT-1 of one case: fields f0 .. f0+F-1
// (F = nf in the fused form, 1 in the split form), then, fused and rd,
// REM_DIV.  sbase: the CTA's 128-byte aligned dynamic shared memory.
template <int MT>
__device__ __forceinline__ void col_body(const ColCase &cc, int rk_step, long m0, int f0, int F,
                                         bool fused, long spin, unsigned extra_tx,
                                         unsigned char *sbase) {
  const ColConst &C = cc.C;
  const int NY = C.NY, L = NY + 2, nf = C.nf, nth = C.nth;
  const int by = cc.by, nbox = cc.nbox;
  const long ss = C.ss;
  const int mt = (int)((ss - m0) < MT ? (ss - m0) : MT);
  const bool rd = fused && cc.rd;
  const int tile = nbox * by * MT;                                  // double2 per CU tile
  double2 *CUt = reinterpret_cast<double2 *>(sbase);                // [F][nbox*by][MT]
  double2 *R = CUt + (long)F * tile;                                // [F][L][MT]
  double *TB = reinterpret_cast<double *>(R + (long)F * L * MT);    // [F][5][L] CN tables
  double *RT = TB + (long)F * 5 * L;                                // [3][L] UU, IDY, IDYF
  double *KXS = RT + 3 * L, *KZS = KXS + MT, *KKS = KZS + MT;       // [MT]
  Hdr *hd = reinterpret_cast<Hdr *>(KKS + MT);
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(hd + 1);
  const int tid = threadIdx.x;

  // constant tables first: they do not depend on the preceding kernel
  if (tid == 0) dg_mbar_init(bar, 1);
  if (tid < MT) {
    const long mg = (m0 + tid < ss) ? m0 + tid : 0;
    const double KX = cc.kxv[mg % C.nkxp], KZ = cc.kzv[mg / C.nkxp];
    const double k2 = KX * KX + KZ * KZ;
    KXS[tid] = KX;
    KZS[tid] = KZ;
    KKS[tid] = (C.beta == 1.0) ? k2 : pow(k2, C.beta);
  }
  if (tid < nf) {
    hd->cu[tid] = cc.cu[tid];
    hd->cf[tid] = cc.cf[tid];
    hd->nl[tid] = cc.nl[tid];
  }
  const double *tab_rk = cc.tab + (long)(rk_step - 1) * (3 + DG_MAX_TH) * 5 * L;
  for (int i = tid; i < F * 5 * L; i += CS_THR) TB[i] = tab_rk[(long)f0 * 5 * L + i];
  if (rd) {
    for (int j = tid; j < L; j += CS_THR) {
      RT[j] = cc.rowc[6 * L + j];          // UU
      RT[L + j] = cc.rowc[4 * L + j];      // 1/DY
      RT[2 * L + j] = cc.rowc[5 * L + j];  // 1/DYF
    }
  }
  __syncthreads();
  dg_pdl_wait();  // NL comes from the z-forward kernel
  if (tid == 0) {
    // columns beyond ss and planes beyond L arrive as zeros (extra_tx is 0
    // except in the wait test, where the barrier can then never complete)
    dg_mbar_expect_tx(bar, (unsigned)(sizeof(double2) * F * tile) + extra_tx);
    for (int f = 0; f < F; f++)
      for (int q = 0; q < nbox; q++)
        dg_tma_load_2d(CUt + (long)f * tile + (long)q * by * MT, &cc.maps[f0 + f], (int)(2 * m0),
                       q * by, bar);
  }
  const bool landed = dg_mbar_wait(bar, 0, spin);
  __syncthreads();
  if (!landed) {
    if (tid == 0) atomicExch(cc.err + 1, 1);
    dg_mbar_wait(bar, 0, spin);  // give the copies in flight one more bounded wait
    return;
  }

  // ---- 1. explicit terms, CF and the CN right-hand side, field by field
  const double h = cc.dscal[1 + rk_step];
  const double time = cc.dscal[0];
  const double zeta = (rk_step == 2) ? -17.0 / 8.0 : (rk_step == 3) ? -5.0 / 4.0 : 0.0;
  const double bbar = (rk_step == 2) ? 25.0 / 8.0 : (rk_step == 3) ? 9.0 / 4.0 : 1.0;
  const double T1 = C.nu * h / 2.0, T3 = zeta * h, T4 = h, T5 = bbar * h;
  const double aaU = T1 * C.nuv;
  const double NU = C.nu;
  const double *__restrict__ rowc = cc.rowc;
  double2 *__restrict__ cp = cc.cp;
  // a value of field g at (j, m): from the staged tiles when the CTA holds
  // g, from global memory otherwise (the split form's cross-field terms)
  auto fieldv = [&](int g, int j, int m, long o) -> double2 {
    if (g >= f0 && g < f0 + F) return CUt[(long)(g - f0) * tile + j * MT + m];
    return hd->cu[g][o];
  };
  for (int fl = 0; fl < F; fl++) {
    const int f = f0 + fl;
    int lo, hi;
    if (f == 0 || f == 2) { lo = C.JS; hi = C.JE; }
    else if (f == 1) { lo = 2; hi = NY; }
    else { lo = pick(C.JSt, f - 3); hi = pick(C.JEt, f - 3); }
    const double2 *__restrict__ T = CUt + (long)fl * tile;
    double2 *__restrict__ Rf = R + (long)fl * L * MT;
    const double2 *__restrict__ nlf = hd->nl[f];
    double2 *__restrict__ cff = hd->cf[f];
    // the field's uniform coefficients
    const double sgn = (f == 0) ? 1.0 : -1.0;
    const double gr = (f == 0) ? C.grav_x : C.grav_z;
    const int n = f - 3;
    const double nup = (f >= 3) ? NU / pick(C.pr, n) : NU;
    const double ipr = (f >= 3) ? 1.0 / pick(C.pr, n) : 1.0;
    const double ddx = (f >= 3) ? pick(C.drhodx, n) : 0.0;
    const double ddz = (f >= 3) ? pick(C.drhodz, n) : 0.0;
    for (int i = lo * MT + tid; i < (hi + 1) * MT; i += CS_THR) {
      const int j = i / MT, m = i - j * MT;
      if (m >= mt) continue;
      const long o = (long)j * ss + m0 + m;
      const double2 u = T[i], um = T[i - MT], up = T[i + MT];
      const double2 nlv = nlf[o];
      const double2 old = (rk_step > 1) ? cff[o] : make_double2(0.0, 0.0);
      const double kk = KKS[m];
      double2 fv, r;
      if (f == 0 || f == 2) {
        fv = make_double2(-NU * kk * u.x, -NU * kk * u.y);
        if (C.i_ro != 0.0) {
          const double2 uo = fieldv(2 - f, j, m, o);
          fv.x += sgn * C.i_ro * uo.x;
          fv.y += sgn * C.i_ro * uo.y;
        }
        for (int q = 0; q < nth; q++) {
          const double w = C.ri[q] * gr;
          if (w == 0.0) continue;
          const double2 t = fieldv(3 + q, j, m, o);
          fv.x += w * t.x;
          fv.y += w * t.y;
        }
        fv.x += nlv.x;
        fv.y += nlv.y;
        r = u;
        r.x += T3 * old.x;
        r.y += T3 * old.y;
        const double2 p0 = cp[o];
        const double K = (f == 0) ? KXS[m] : KZS[m];
        r.x -= T4 * (-K * p0.y);
        r.y -= T4 * (K * p0.x);
        if (f == 0 && m0 + m == 0) {
          if (C.f_type == 1) r.x -= T4 * C.px0;
          else if (C.f_type == 2) r.x -= T4 * (C.px0 + C.amp_omega0 * cos(C.omega0 * time));
        }
        r.x += T5 * fv.x;
        r.y += T5 * fv.y;
        const double cup = aaU * rowc[0 * L + j], cdn = aaU * rowc[1 * L + j];
        r.x += cup * (up.x - u.x) - cdn * (u.x - um.x);
        r.y += cup * (up.y - u.y) - cdn * (u.y - um.y);
      } else if (f == 1) {
        fv = make_double2(-NU * kk * u.x, -NU * kk * u.y);
        if (m0 + m != 0) {
          const double dyfj = rowc[7 * L + j], dyfm = rowc[7 * L + j - 1];
          const double bw2 = 0.5 * rowc[4 * L + j];
          for (int q = 0; q < nth; q++) {
            if (C.ri[q] * C.grav_y == 0.0) continue;
            const double w = C.ri[q] * C.grav_y * bw2;
            const double2 t = fieldv(3 + q, j, m, o);
            const double2 tm = fieldv(3 + q, j - 1, m, o - ss);
            fv.x += w * (t.x * dyfm + tm.x * dyfj);
            fv.y += w * (t.y * dyfm + tm.y * dyfj);
          }
        }
        fv.x += nlv.x;
        fv.y += nlv.y;
        r = u;
        r.x += T3 * old.x;
        r.y += T3 * old.y;
        const double2 p0 = cp[o], pm = cp[o - ss];
        const double idy = rowc[4 * L + j];
        r.x -= T4 * ((p0.x - pm.x) * idy);
        r.y -= T4 * ((p0.y - pm.y) * idy);
        r.x += T5 * fv.x;
        r.y += T5 * fv.y;
        const double cup2 = aaU * rowc[2 * L + j], cdn2 = aaU * rowc[3 * L + j];
        r.x += cup2 * (up.x - u.x) - cdn2 * (u.x - um.x);
        r.y += cup2 * (up.y - u.y) - cdn2 * (u.y - um.y);
      } else {
        fv = make_double2(-nup * kk * u.x, -nup * kk * u.y);
        if (ddx != 0.0 || ddz != 0.0) {
          const double2 u1 = fieldv(0, j, m, o), u3 = fieldv(2, j, m, o);
          fv.x = fv.x - u1.x * ddx - u3.x * ddz;
          fv.y = fv.y - u1.y * ddx - u3.y * ddz;
        }
        fv.x += nlv.x;
        fv.y += nlv.y;
        r = u;
        r.x += T3 * old.x;
        r.y += T3 * old.y;
        r.x += T5 * fv.x;
        r.y += T5 * fv.y;
        const double cup = aaU * rowc[0 * L + j], cdn = aaU * rowc[1 * L + j];
        r.x += ipr * (cup * (up.x - u.x) - cdn * (u.x - um.x));
        r.y += ipr * (cup * (up.y - u.y) - cdn * (u.y - um.y));
      }
      cff[o] = fv;
      Rf[i] = r;
    }
  }
  __syncthreads();

  // ---- 2. CN solves, one lane per (field, mode), rows 0..NY+1.  The operator
  // is real, so the real and imaginary parts are two independent recurrences;
  // one lane runs both, interleaved, which hides half of each one's latency.
  for (int t = tid; t < MT * F; t += CS_THR) {
    const int fl = t / MT;
    const int f = f0 + fl;
    const int m = t - fl * MT;
    const double *T = TB + (long)fl * 5 * L;
    const double *Aa = T, *Rb = T + L, *Cc = T + 2 * L, *K = T + 3 * L, *V = T + 4 * L;
    double2 *x = R + (long)fl * L * MT + m;
    constexpr int B = 8;  // rows per register block: loads first, then the recurrences
    const bool mean = (m0 + m == 0);
    const int wlo = (f >= 3) ? pick(C.JSt, f - 3) - 1 : 1;
    double2 g = make_double2(0.0, 0.0);
    for (int j0 = 0; j0 < L; j0 += B) {
      double2 r[B];
      double a[B];
#pragma unroll
      for (int q = 0; q < B; q++) {
        const int j = j0 + q < L ? j0 + q : L - 1;
        const double kind = K[j];
        const double2 xr = x[j * MT];
        // a BC row's value goes to the real part of the (0,0) mode only
        r[q] = (kind == (double)ROW_RHS)
                   ? xr
                   : make_double2((kind == (double)ROW_BC && mean) ? V[j] : 0.0, 0.0);
        a[q] = Aa[j];
      }
#pragma unroll
      for (int q = 0; q < B; q++) {
        if (j0 + q < L) {
          g.x = r[q].x + a[q] * g.x;
          g.y = r[q].y + a[q] * g.y;
          r[q] = g;
        }
      }
#pragma unroll
      for (int q = 0; q < B; q++)
        if (j0 + q < L) x[(j0 + q) * MT] = r[q];
    }
    const double rbl = Rb[L - 1];
    double2 xv = make_double2(g.x * rbl, g.y * rbl);
    x[(L - 1) * MT] = xv;
    for (int j1 = L - 2; j1 >= wlo; j1 -= B) {
      double2 gq[B];
      double cq[B], rq[B];
#pragma unroll
      for (int q = 0; q < B; q++) {
        const int j = j1 - q >= wlo ? j1 - q : wlo;
        gq[q] = x[j * MT];
        cq[q] = Cc[j];
        rq[q] = Rb[j];
      }
#pragma unroll
      for (int q = 0; q < B; q++) {
        if (j1 - q >= wlo) {
          xv.x = (gq[q].x - cq[q] * xv.x) * rq[q];
          xv.y = (gq[q].y - cq[q] * xv.y) * rq[q];
          gq[q] = xv;
        }
      }
#pragma unroll
      for (int q = 0; q < B; q++)
        if (j1 - q >= wlo) x[(j1 - q) * MT] = gq[q];
    }
  }
  __syncthreads();

  if (!rd) {
    // the post-CN fields go out; REM_DIV runs as its own launch
    for (int fl = 0; fl < F; fl++) {
      const int f = f0 + fl;
      const int wlo = (f >= 3) ? pick(C.JSt, f - 3) - 1 : 1;
      double2 *__restrict__ U = hd->cu[f];
      const double2 *__restrict__ Rf = R + (long)fl * L * MT;
      for (int i = wlo * MT + tid; i < L * MT; i += CS_THR) {
        const int j = i / MT, m = i - j * MT;
        if (m < mt) U[(long)j * ss + m0 + m] = Rf[i];
      }
    }
    return;
  }

  // ---- 3. REM_DIV_CHAN (fused form): divergence of the CN velocity, factors, sweeps
  const double2 *U1 = R, *U2 = R + (long)L * MT, *U3 = R + 2L * L * MT;
  double2 *GX = CUt;          // [L][MT]: rhs -> g -> phi
  double2 *RAB = CUt + tile;  // [L][MT]: (multiplier, reciprocal pivot)
  const double *UU = RT, *IDY = RT + L, *IDYF = RT + 2 * L;
  for (int i = tid; i < L * MT; i += CS_THR) {
    const int j = i / MT, m = i - j * MT;
    const bool ok = m < mt && j >= 1 && j <= NY;
    double2 r = make_double2(0.0, 0.0);
    if (ok && j >= 2 && j < NY) {
      const double KX = KXS[m], KZ = KZS[m], id = IDYF[j];
      const double2 a1 = U1[i], a3 = U3[i], b2 = U2[i], b2p = U2[i + MT];
      r.x = (-KX * a1.y) + (b2p.x - b2.x) * id + (-KZ * a3.y);
      r.y = (KX * a1.x) + (b2p.y - b2.y) * id + (KZ * a3.x);
    }
    GX[i] = r;
    const long o = (long)j * ss + m0 + m;
    RAB[i] = ok ? make_double2(cc.ra[o], cc.rrb[o]) : make_double2(0.0, 0.0);
  }
  __syncthreads();
  if (tid < MT) {
    // one lane per mode: the real and imaginary recurrences interleaved
    const int m = tid;
    const bool mean = (m0 + m == 0);
    double2 *x = GX + m;
    const double2 *AB = RAB + m;  // (multiplier, reciprocal pivot) of [j][m]
    constexpr int B = 8;
    double2 g = make_double2(0.0, 0.0);  // row 1 has a zero right-hand side
    x[1 * MT] = g;
    for (int j0 = 2; j0 <= NY; j0 += B) {
      double2 r[B];
      double a[B];
#pragma unroll
      for (int q = 0; q < B; q++) {
        const int j = j0 + q <= NY ? j0 + q : NY;
        r[q] = x[j * MT];
        a[q] = AB[j * MT].x;
      }
#pragma unroll
      for (int q = 0; q < B; q++) {
        if (j0 + q <= NY) {
          g.x = r[q].x + a[q] * g.x;
          g.y = r[q].y + a[q] * g.y;
          r[q] = g;
        }
      }
#pragma unroll
      for (int q = 0; q < B; q++)
        if (j0 + q <= NY) x[(j0 + q) * MT] = r[q];
    }
    const double rbn = AB[NY * MT].y;
    double2 ph = make_double2(g.x * rbn, g.y * rbn);
    x[NY * MT] = ph;
    for (int j1 = NY - 1; j1 >= 2; j1 -= B) {
      double2 gq[B];
      double uq[B], bq[B];
#pragma unroll
      for (int q = 0; q < B; q++) {
        const int j = j1 - q >= 2 ? j1 - q : 2;
        gq[q] = x[j * MT];
        uq[q] = UU[j];
        bq[q] = AB[j * MT].y;
      }
#pragma unroll
      for (int q = 0; q < B; q++) {
        if (j1 - q >= 2) {
          ph.x = (gq[q].x - uq[q] * ph.x) * bq[q];
          ph.y = (gq[q].y - uq[q] * ph.y) * bq[q];
          gq[q] = ph;
        }
      }
#pragma unroll
      for (int q = 0; q < B; q++)
        if (j1 - q >= 2) x[(j1 - q) * MT] = gq[q];
    }
    const double u1r = mean ? 0.0 : -1.0;
    const double2 x1 = x[1 * MT];
    const double rb1 = AB[1 * MT].y;
    ph = make_double2((x1.x - u1r * ph.x) * rb1, (x1.y - u1r * ph.y) * rb1);
    x[1 * MT] = ph;
  }
  __syncthreads();

  // ---- 4. projection, phi, CP += phi / h; every field's rows go out
  const double ihh = 1.0 / h;
  for (int f = 0; f < nf; f++) {
    const int wlo = (f >= 3) ? pick(C.JSt, f - 3) - 1 : 1;
    double2 *__restrict__ U = hd->cu[f];
    const double2 *__restrict__ Rf = R + (long)f * L * MT;
    for (int i = wlo * MT + tid; i < L * MT; i += CS_THR) {
      const int j = i / MT, m = i - j * MT;
      if (m >= mt) continue;
      const long o = (long)j * ss + m0 + m;
      double2 v = Rf[i];
      if (f < 3 && j >= 1 && j <= NY) {
        const double2 ph = GX[i];
        if (f == 0 || f == 2) {
          // U1 -= i kx phi, U3 -= i kz phi
          const double K = (f == 0) ? KXS[m] : KZS[m];
          v.x -= -K * ph.y;
          v.y -= K * ph.x;
        } else if (j >= 2) {
          // U2(j) -= (phi(j) - phi(j-1)) / DY(j)
          const double2 pm = GX[i - MT];
          v.x -= (ph.x - pm.x) * IDY[j];
          v.y -= (ph.y - pm.y) * IDY[j];
        }
        if (f == 0) {
          cc.phi[o] = ph;
          if (j >= C.JS && j <= C.JE) {
            double2 pc = cp[o];
            pc.x = pc.x + ph.x * ihh;
            pc.y = pc.y + ph.y * ihh;
            cp[o] = pc;
          }
        }
      }
      U[o] = v;
    }
  }
}

// dynamic shared memory of one CTA holding F fields' tiles
size_t col_smem_f(int L, int F, int mt, int by, int nbox) {
  return sizeof(double2) * (size_t)F * ((size_t)nbox * by * mt + (size_t)L * mt) +
         sizeof(double) * ((size_t)F * 5 * L + 3 * L + 3 * mt) + sizeof(Hdr) + 8 + 128;
}

// The column kernel: CTA b takes work[b] = (case, mode tile, first field,
// fields) from the case table (fields = the case's nf in the fused form, 1
// in the split form; every case at substep rk_step with MT modes per CTA).
// A single case runs it with a one-case table, so a case computes with the
// same machine code alone and in an ensemble group (whose launch covers
// every member's tiles), and its results are bit-identical either way.
template <int MT>
__global__ void __launch_bounds__(CS_THR) k_col_step(const ColCase *__restrict__ cases,
                                                    const int4 *__restrict__ work, int rk_step,
                                                    int fused, long spin, unsigned extra_tx) {
  extern __shared__ __align__(128) unsigned char cs_raw[];
  unsigned char *sbase = cs_raw + ((128u - (dg_smem_addr(cs_raw) & 127u)) & 127u);
  const int4 w = work[blockIdx.x];
  col_body<MT>(cases[w.x], rk_step, (long)w.y * MT, w.z, w.w, fused != 0, spin, extra_tx,
               sbase);
}

ColConst make_col_const(const dg_handle *h) {
  ColConst c;
  c.NY = h->NY; c.nf = h->nf; c.nth = h->NTH; c.nkxp = h->nkxp; c.ss = h->ss;
  c.JS = h->jstart; c.JE = h->jend;
  for (int n = 0; n < DG_MAX_TH; n++) {
    c.JSt[n] = h->jstart_th[n]; c.JEt[n] = h->jend_th[n];
    c.ri[n] = h->p.ri[n]; c.pr[n] = h->p.pr[n];
    c.drhodx[n] = h->p.drhodx[n]; c.drhodz[n] = h->p.drhodz[n];
  }
  c.nu = h->p.nu; c.beta = h->p.beta; c.nuv = h->p.nu_v_scale; c.i_ro = h->p.i_ro;
  c.grav_x = h->p.grav_x; c.grav_y = h->p.grav_y; c.grav_z = h->p.grav_z;
  c.px0 = h->p.px0; c.omega0 = h->p.omega0; c.amp_omega0 = h->p.amp_omega0;
  c.f_type = h->p.f_type;
  return c;
}

}  // namespace

// Per-row grid factors of the column kernel (once per handle, host side).
int dg_col_init(dg_handle *h) {
  const int L = h->NY + 2;
  double *t = (double *)calloc((size_t)8 * L, sizeof(double));
  if (!t) return DG_ERR_OOM;
  const double *dy = h->h_dy, *dyf = h->h_dyf;
  for (int j = 1; j <= h->NY; j++) {
    t[0 * L + j] = 1.0 / (dy[j + 1] * dyf[j]);
    t[1 * L + j] = 1.0 / (dy[j] * dyf[j]);
    t[2 * L + j] = 1.0 / (dyf[j] * dy[j]);
    t[3 * L + j] = 1.0 / (dyf[j - 1] * dy[j]);
    t[5 * L + j] = 1.0 / dyf[j];
    t[6 * L + j] = (j >= 2 && j < h->NY) ? 1.0 / (dy[j + 1] * dyf[j]) : 0.0;
  }
  for (int j = 1; j < L; j++) t[4 * L + j] = 1.0 / dy[j];
  for (int j = 0; j < L; j++) t[7 * L + j] = dyf[j];
  cudaError_t e = dg_malloc(h, (void **)&h->rowc, sizeof(double) * 8 * L);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h->rowc, t, sizeof(double) * 8 * L, cudaMemcpyHostToDevice, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  free(t);
  DG_CUDA(e);
  return DG_OK;
}

static void col_geometry(const dg_handle *h, int *by, int *nbox) {
  const int L = h->NY + 2;
  // boxes of at most 256 planes; a multiple of 8 planes keeps every box's
  // shared-memory destination 128-byte aligned for any modes per CTA
  *nbox = dg_cdiv(L, 256);
  *by = (dg_cdiv(L, *nbox) + 7) / 8 * 8;
}

// shared memory of one CTA of handle h's column kernel (fused: every field)
size_t dg_col_smem(const dg_handle *h, int mt, bool fused) {
  int by, nbox;
  col_geometry(h, &by, &nbox);
  return col_smem_f(h->NY + 2, fused ? h->nf : 1, mt, by, nbox);
}

// The column-kernel description of handle h for `mt` modes per CTA (builds
// the tensor maps of CU for that tile width).
static int fill_case(dg_handle *h, int mt, bool rd, ColCase *cc) {
  const int L = h->NY + 2;
  int by = 0, nbox = 0;
  col_geometry(h, &by, &nbox);
  if (h->cs_maps_mt != mt) {
    for (int f = 0; f < h->nf; f++)
      DG_TRY(dg_tmap_planes(h->cu[f], h->ss, L, mt, by, &h->cs_maps->m[f]));
    h->cs_maps_mt = mt;
  }
  memset(cc, 0, sizeof(*cc));
  for (int f = 0; f < h->nf; f++) cc->maps[f] = h->cs_maps->m[f];
  cc->C = make_col_const(h);
  cc->dscal = h->dscal;
  cc->tab = h->cn_tab;
  cc->kxv = h->kx;
  cc->kzv = h->kz;
  cc->rowc = h->rowc;
  cc->ra = h->rem_a;
  cc->rrb = h->rem_rb;
  for (int f = 0; f < h->nf; f++) {
    cc->cu[f] = h->cu[f];
    cc->cf[f] = h->cf[f];
    cc->nl[f] = h->rhs[f];
  }
  cc->cp = h->cp;
  cc->phi = h->cr1;
  cc->err = h->dflag;
  cc->by = by;
  cc->nbox = nbox;
  cc->rd = rd ? 1 : 0;
  return DG_OK;
}

// The column form that runs for h: the split form only when no field's
// right-hand side reads another field (see above).
bool dg_col_fused(const dg_handle *h) {
  if (h->col_fused) return true;
  if (h->p.i_ro != 0.0) return true;
  for (int n = 0; n < h->NTH; n++) {
    const double ri = h->p.ri[n];
    if (ri * h->p.grav_x != 0.0 || ri * h->p.grav_y != 0.0 || ri * h->p.grav_z != 0.0 ||
        h->p.drhodx[n] != 0.0 || h->p.drhodz[n] != 0.0)
      return true;
  }
  return false;
}

// modes per CTA for handle h: the tuned value, halved until the tiles fit
static int col_mt(const dg_handle *h, int want, bool fused) {
  int mt = want;
  while (mt > 2 && dg_col_smem(h, mt, fused) > 220 * 1024) mt /= 2;
  return mt;
}

// the work list of one case: (case 0, tile, first field, fields) per CTA
static void case_work(const dg_handle *h, int c, int mt, bool fused, std::vector<int4> &work) {
  const int tiles = dg_cdiv(h->ss, mt);
  if (fused) {
    for (int t = 0; t < tiles; t++) work.push_back(make_int4(c, t, 0, h->nf));
  } else {
    for (int f = 0; f < h->nf; f++)
      for (int t = 0; t < tiles; t++) work.push_back(make_int4(c, t, f, 1));
  }
}

// The handle's device copies of its case table (rd = 0 and 1) and work list
// for (mt, fused), rebuilt when either changes.  The copies are synchronous,
// so they cannot run inside a stream capture: diablo_step's first step of a
// kind, which runs eagerly, builds them before any capture.
static int col_tables(dg_handle *h, int mt, bool fused) {
  if (h->col_dcase && h->col_dmt == mt && h->col_dfused == (int)fused) return DG_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(h->st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
    dg_set_error("the column kernel's case table must be built before a stream capture "
                 "(run one substep eagerly after changing the tuning)");
    return DG_ERR_ARG;
  }
  ColCase cc[2];
  DG_TRY(fill_case(h, mt, false, &cc[0]));
  DG_TRY(fill_case(h, mt, true, &cc[1]));
  std::vector<int4> work;
  case_work(h, 0, mt, fused, work);
  DG_CUDA(cudaStreamSynchronize(h->st));
  if (h->col_dcase) dg_free(h, h->col_dcase);
  if (h->col_dwork) dg_free(h, h->col_dwork);
  h->col_dcase = nullptr;
  h->col_dwork = nullptr;
  DG_CUDA(dg_malloc(h, &h->col_dcase, sizeof(cc)));
  DG_CUDA(dg_malloc(h, (void **)&h->col_dwork, sizeof(int4) * work.size()));
  DG_CUDA(cudaMemcpyAsync(h->col_dcase, cc, sizeof(cc), cudaMemcpyHostToDevice, h->st));
  DG_CUDA(cudaMemcpyAsync(h->col_dwork, work.data(), sizeof(int4) * work.size(),
                          cudaMemcpyHostToDevice, h->st));
  DG_CUDA(cudaStreamSynchronize(h->st));
  h->col_dmt = mt;
  h->col_dfused = fused ? 1 : 0;
  h->col_dnwork = (int)work.size();
  return DG_OK;
}

// The column stage of substep rk_step.  rd = false: stop after the CN
// solves (the velocity goes out unprojected; COURANT and REM_DIV follow).
// The split form always stops there, and REM_DIV runs here after it when rd.
int dg_col_step_dev(dg_handle *h, int rk_step, bool rd) {
  if (h->tables_pending) {
    DG_CUDA(cudaStreamWaitEvent(h->st, h->ev_join, 0));
    h->tables_pending = false;
  }
  const bool fused = dg_col_fused(h);
  const int mt = col_mt(h, h->cn_mt, fused);
  const size_t sm = dg_col_smem(h, mt, fused);
  if (sm > 220 * 1024) {
    dg_set_error("column kernel: the y-columns of two modes do not fit in shared memory");
    return DG_ERR_DIMS;
  }
  DG_TRY(col_tables(h, mt, fused));
  const ColCase *dcase = reinterpret_cast<const ColCase *>(h->col_dcase) + ((fused && rd) ? 1 : 0);
  // the wait test (DG_TUNE_WAIT_TEST) applies to this one launch
  const long spin = h->wait_test > 0 ? (long)h->wait_test : DG_ASYNC_SPIN;
  const unsigned extra_tx = h->wait_test > 0 ? 16u : 0u;
  h->wait_test = 0;
  const char *name = fused ? (rd ? "k_col_step" : "k_col_step_cn") : "k_col_cn";
#define CS_CASE(MTV)                                                                           \
  if (mt == MTV) {                                                                             \
    dg_big_smem((const void *)k_col_step<MTV>);                                                \
    dg_kt_begin(h, name, h->st);                                                               \
    DG_CUDA(dg_launch(h->pdl, k_col_step<MTV>, dim3(h->col_dnwork), dim3(CS_THR), sm, h->st,   \
                      dcase, (const int4 *)h->col_dwork, rk_step, fused ? 1 : 0, spin,         \
                      extra_tx));                                                              \
  }
  CS_CASE(2) CS_CASE(4) CS_CASE(8) CS_CASE(16)
#undef CS_CASE
  DG_LAUNCHED();
  if (!fused && rd) DG_TRY(dg_rem_div_dev(h, 1, rk_step));
  return DG_OK;
}

// ---------------------------------------------------------- ragged launch
// The column stage of several cases at the same substep in one launch (the
// ensemble server's groups).  dg_col_batch_build fills, for the handles, the
// host images of the case table and the work list (one (case, tile, first
// field, fields) entry per CTA) with one MT for all, and returns the launch's
// shared memory; the caller copies them to device memory it owns and
// launches with dg_col_batch_launch.  In the split form (fused = 0) the
// launch stops after the CN solves and each case's REM_DIV follows on its
// own stream.  Results do not depend on the batch: each mode's arithmetic is
// the single-case kernel's.
size_t dg_col_case_bytes() { return sizeof(ColCase); }

int dg_col_batch_build(dg_handle *const *hs, const int *rd, int n, int want_mt, int fused,
                       std::vector<unsigned char> &cases, std::vector<int4> &work, int *mt_out,
                       size_t *smem_out) {
  int mt = want_mt;
  for (int c = 0; c < n; c++) mt = std::min(mt, col_mt(hs[c], want_mt, fused != 0));
  size_t sm = 0;
  for (int c = 0; c < n; c++) sm = std::max(sm, dg_col_smem(hs[c], mt, fused != 0));
  if (sm > 220 * 1024) {
    dg_set_error("column kernel: the y-columns of two modes do not fit in shared memory");
    return DG_ERR_DIMS;
  }
  cases.assign(sizeof(ColCase) * n, 0);
  work.clear();
  for (int c = 0; c < n; c++) {
    ColCase cc;
    DG_TRY(fill_case(hs[c], mt, fused && rd[c] != 0, &cc));
    memcpy(cases.data() + sizeof(ColCase) * c, &cc, sizeof(ColCase));
    case_work(hs[c], c, mt, fused != 0, work);
  }
  *mt_out = mt;
  *smem_out = sm;
  return DG_OK;
}

int dg_col_batch_launch(cudaStream_t st, int mt, size_t smem, const void *dev_cases,
                        const int4 *dev_work, int nwork, int rk_step, int fused) {
#define CR_CASE(MTV)                                                                              \
  if (mt == MTV) {                                                                                \
    dg_big_smem((const void *)k_col_step<MTV>);                                                   \
    k_col_step<MTV><<<nwork, CS_THR, smem, st>>>((const ColCase *)dev_cases, dev_work, rk_step,   \
                                                fused, (long)DG_ASYNC_SPIN, 0u);                  \
  }
  CR_CASE(2) CR_CASE(4) CR_CASE(8) CR_CASE(16)
#undef CR_CASE
  DG_LAUNCHED();
  return DG_OK;
}
