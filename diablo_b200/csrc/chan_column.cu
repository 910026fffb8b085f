// The per-mode column stage of RK_CHAN_1 in one kernel: explicit terms and
// the Crank-Nicolson right-hand side, the CN solves of every field, and
// REM_DIV_CHAN with the pressure update, for a tile of MT retained (kx, kz)
// modes and their whole y-columns.
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
// Layout: every field is [NY+2][ss] complex, modes kx fastest; a CTA owns
// modes m0 .. m0+MT-1.  The CU tiles of every field (all planes x MT modes)
// arrive by bulk tensor copies (TMA, no multicast) on one mbarrier with a
// bounded wait; the nonlinear terms NL (written by the z-forward kernel into
// the rhs arrays), CF and CP are read with plain coalesced loads while the
// right-hand sides are formed.  The right-hand sides, then the CN solutions,
// live in a second set of shared tiles; the CU tiles, no longer needed, hold
// the REM_DIV factors and phi.  Only the three velocity solutions meet in
// REM_DIV, so every field's sweep runs in its own lanes at the same time.
//
// Global traffic per substep (FP64 complex fields of the retained modes):
// read CU, NL, CF (substeps 2, 3), CP, the REM_DIV factors; write CF, CU, CP,
// phi -- each once.
#include <string.h>

#include <algorithm>
#include <vector>

#include "dg_internal.cuh"

namespace {

constexpr int CS_THR = 128;

struct ColConst {
  int NY, nf, nth, nkxp, JS, JE;
  int JSt[DG_MAX_TH], JEt[DG_MAX_TH];
  int wlo[3 + DG_MAX_TH];  // lowest row each field's CN solution writes
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
  int rd;  // 1: REM_DIV in the kernel; 0: stop after the CN solves
};

template <typename T>
__device__ __forceinline__ T pick(const T (&a)[DG_MAX_TH], int i) {
  T r = a[0];
#pragma unroll
  for (int k = 1; k < DG_MAX_TH; k++) r = (i == k) ? a[k] : r;
  return r;
}

__device__ __forceinline__ int pick_w(const int (&a)[3 + DG_MAX_TH], int i) {
  int r = a[0];
#pragma unroll
  for (int k = 1; k < 3 + DG_MAX_TH; k++) r = (i == k) ? a[k] : r;
  return r;
}

// rows of field f's right-hand side (JSTART..JEND, 2..NY for U2)
__device__ __forceinline__ void rhs_rows(const ColConst &C, int f, int &lo, int &hi) {
  if (f == 0 || f == 2) { lo = C.JS; hi = C.JE; }
  else if (f == 1) { lo = 2; hi = C.NY; }
  else { lo = pick(C.JSt, f - 3); hi = pick(C.JEt, f - 3); }
}

// rowc: per-row grid factors [8][NY+2]
//   0 1/(DY(j+1) DYF(j))  1 1/(DY(j) DYF(j))       (GYF rows: U1, U3, TH)
//   2 1/(DYF(j) DY(j))    3 1/(DYF(j-1) DY(j))     (GY rows: U2)
//   4 1/DY(j)             5 1/DYF(j)               6 REM_DIV upper diagonal
//   7 DYF(j)
// The column stage of modes m0 .. m0+MT-1 of one case (all threads of the
// CTA; sbase: the CTA's 128-byte aligned dynamic shared memory).
template <int MT>
__device__ __forceinline__ void col_body(const ColCase &cc, int rk_step, long m0, long spin,
                                         unsigned extra_tx, unsigned char *sbase) {
  const ColConst &C = cc.C;
  const int by = cc.by, nbox = cc.nbox;
  const double *__restrict__ dscal = cc.dscal;
  const double *__restrict__ kxv = cc.kxv;
  const double *__restrict__ kzv = cc.kzv;
  const double *__restrict__ rowc = cc.rowc;
  double2 *__restrict__ cp = cc.cp;
  const int L = C.NY + 2, nf = C.nf;
  const double *__restrict__ tab_rk = cc.tab + (long)(rk_step - 1) * (3 + DG_MAX_TH) * 5 * L;
  const long ss = C.ss;
  const int mt = (int)((ss - m0) < MT ? (ss - m0) : MT);
  const int tile = nbox * by * MT;                                   // double2 per CU tile
  double2 *CUt = reinterpret_cast<double2 *>(sbase);                 // [nf][nbox*by][MT]
  double2 *R = CUt + (long)nf * tile;                                // [nf][L][MT]
  double *KXS = reinterpret_cast<double *>(R + (long)nf * L * MT);   // [MT]
  double *KZS = KXS + MT, *KKS = KZS + MT;                           // [MT]
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(KKS + MT);
  const int tid = threadIdx.x;

  if (tid == 0) dg_mbar_init(bar, 1);
  if (tid < MT) {
    const long mg = (m0 + tid < ss) ? m0 + tid : 0;
    const double KX = kxv[mg % C.nkxp], KZ = kzv[mg / C.nkxp];
    const double k2 = KX * KX + KZ * KZ;
    KXS[tid] = KX;
    KZS[tid] = KZ;
    KKS[tid] = (C.beta == 1.0) ? k2 : pow(k2, C.beta);
  }
  __syncthreads();
  dg_pdl_wait();  // NL comes from the z-forward kernel
  if (tid == 0) {
    // columns beyond ss and planes beyond L arrive as zeros (extra_tx is 0
    // except in the wait test, where the barrier can then never complete)
    dg_mbar_expect_tx(bar, (unsigned)(sizeof(double2) * nf * tile) + extra_tx);
    for (int f = 0; f < nf; f++)
      for (int q = 0; q < nbox; q++)
        dg_tma_load_2d(CUt + (long)f * tile + (long)q * by * MT, &cc.maps[f], (int)(2 * m0), q * by,
                       bar);
  }
  const bool landed = dg_mbar_wait(bar, 0, spin);
  __syncthreads();
  if (!landed) {
    if (tid == 0) atomicExch(cc.err + 1, 1);
    dg_mbar_wait(bar, 0, spin);  // give the copies in flight one more bounded wait
    return;
  }

  // ---- 1. explicit terms, CF and the CN right-hand side, every (field, row, mode)
  const double h = dscal[1 + rk_step];
  const double time = dscal[0];
  const double zeta = (rk_step == 2) ? -17.0 / 8.0 : (rk_step == 3) ? -5.0 / 4.0 : 0.0;
  const double bbar = (rk_step == 2) ? 25.0 / 8.0 : (rk_step == 3) ? 9.0 / 4.0 : 1.0;
  const double T1 = C.nu * h / 2.0, T3 = zeta * h, T4 = h, T5 = bbar * h;
  const double aaU = T1 * C.nuv;
  const double NU = C.nu;
  const int nitems = nf * L * MT;
  for (int i = tid; i < nitems; i += CS_THR) {
    const int f = i / (L * MT);
    const int rem = i - f * L * MT;
    const int j = rem / MT, m = rem - j * MT;
    int lo, hi;
    rhs_rows(C, f, lo, hi);
    if (m >= mt || j < lo || j > hi) continue;
    const long o = (long)j * ss + m0 + m;
    const double2 *T = CUt + (long)f * tile;
    const double2 u = T[j * MT + m], um = T[(j - 1) * MT + m], up = T[(j + 1) * MT + m];
    const double2 nlv = cc.nl[f][o];
    const double2 old = (rk_step > 1) ? cc.cf[f][o] : make_double2(0.0, 0.0);
    const double kk = KKS[m];
    double2 fv, r;
    if (f == 0 || f == 2) {
      const double2 uo = CUt[(long)(2 - f) * tile + j * MT + m];
      const double sgn = (f == 0) ? 1.0 : -1.0;
      const double gr = (f == 0) ? C.grav_x : C.grav_z;
      fv = make_double2(-NU * kk * u.x, -NU * kk * u.y);
      if (C.i_ro != 0.0) {
        fv.x += sgn * C.i_ro * uo.x;
        fv.y += sgn * C.i_ro * uo.y;
      }
#pragma unroll
      for (int n = 0; n < DG_MAX_TH; n++) {
        if (n >= C.nth) break;
        const double2 t = CUt[(long)(3 + n) * tile + j * MT + m];
        fv.x += C.ri[n] * gr * t.x;
        fv.y += C.ri[n] * gr * t.y;
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
#pragma unroll
        for (int n = 0; n < DG_MAX_TH; n++) {
          if (n >= C.nth) break;
          const double2 t = CUt[(long)(3 + n) * tile + j * MT + m];
          const double2 tm = CUt[(long)(3 + n) * tile + (j - 1) * MT + m];
          const double w = C.ri[n] * C.grav_y * bw2;
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
      const int n = f - 3;
      const double nup = NU / pick(C.pr, n);
      fv = make_double2(-nup * kk * u.x, -nup * kk * u.y);
      const double dx = pick(C.drhodx, n), dz = pick(C.drhodz, n);
      if (dx != 0.0 || dz != 0.0) {
        const double2 u1 = CUt[j * MT + m], u3 = CUt[2L * tile + j * MT + m];
        fv.x = fv.x - u1.x * dx - u3.x * dz;
        fv.y = fv.y - u1.y * dx - u3.y * dz;
      }
      fv.x += nlv.x;
      fv.y += nlv.y;
      r = u;
      r.x += T3 * old.x;
      r.y += T3 * old.y;
      r.x += T5 * fv.x;
      r.y += T5 * fv.y;
      const double ipr = 1.0 / pick(C.pr, n);
      const double cup = aaU * rowc[0 * L + j], cdn = aaU * rowc[1 * L + j];
      r.x += ipr * (cup * (up.x - u.x) - cdn * (u.x - um.x));
      r.y += ipr * (cup * (up.y - u.y) - cdn * (u.y - um.y));
    }
    cc.cf[f][o] = fv;
    R[(long)f * L * MT + j * MT + m] = r;
  }
  __syncthreads();

  // ---- 2. CN solves, one lane per (field, mode, re/im part), rows 0..NY+1
  for (int t = tid; t < 2 * MT * nf; t += CS_THR) {
    const int f = t / (2 * MT);
    const int m = (t >> 1) % MT, part = t & 1;
    const double *T = tab_rk + (long)f * 5 * L;
    const double *Aa = T, *Rb = T + L, *Cc = T + 2 * L, *K = T + 3 * L, *V = T + 4 * L;
    double *x = reinterpret_cast<double *>(R + (long)f * L * MT) + 2 * m + part;
    constexpr int st = 2 * MT;
    constexpr int B = 8;  // rows per register block: loads first, then the recurrence
    const bool mean_re = (m0 + m == 0) && part == 0;
    const int wlo = pick_w(C.wlo, f);
    double g = 0.0;
    for (int j0 = 0; j0 < L; j0 += B) {
      double r[B], a[B];
#pragma unroll
      for (int q = 0; q < B; q++) {
        const int j = j0 + q < L ? j0 + q : L - 1;
        const double kind = __ldg(K + j);
        const double xr = x[j * st];
        r[q] = (kind == (double)ROW_RHS) ? xr
                                         : ((kind == (double)ROW_BC && mean_re) ? __ldg(V + j) : 0.0);
        a[q] = __ldg(Aa + j);
      }
#pragma unroll
      for (int q = 0; q < B; q++) {
        if (j0 + q < L) {
          g = r[q] + a[q] * g;
          r[q] = g;
        }
      }
#pragma unroll
      for (int q = 0; q < B; q++)
        if (j0 + q < L) x[(j0 + q) * st] = r[q];
    }
    double xv = g * __ldg(Rb + L - 1);
    x[(L - 1) * st] = xv;
    for (int j1 = L - 2; j1 >= wlo; j1 -= B) {
      double gq[B], cq[B], rq[B];
#pragma unroll
      for (int q = 0; q < B; q++) {
        const int j = j1 - q >= wlo ? j1 - q : wlo;
        gq[q] = x[j * st];
        cq[q] = __ldg(Cc + j);
        rq[q] = __ldg(Rb + j);
      }
#pragma unroll
      for (int q = 0; q < B; q++) {
        if (j1 - q >= wlo) {
          xv = (gq[q] - cq[q] * xv) * rq[q];
          gq[q] = xv;
        }
      }
#pragma unroll
      for (int q = 0; q < B; q++)
        if (j1 - q >= wlo) x[(j1 - q) * st] = gq[q];
    }
  }
  __syncthreads();

  if (!cc.rd) {
    // the post-CN velocity and scalars go out; REM_DIV runs after COURANT
    for (int i = tid; i < nitems; i += CS_THR) {
      const int f = i / (L * MT);
      const int rem = i - f * L * MT;
      const int j = rem / MT, m = rem - j * MT;
      if (m < mt && j >= pick_w(C.wlo, f)) cc.cu[f][(long)j * ss + m0 + m] = R[i];
    }
    return;
  }

  // ---- 3. REM_DIV_CHAN: divergence of the CN velocity, factors, sweeps
  const int NY = C.NY;
  const double2 *U1 = R, *U2 = R + (long)L * MT, *U3 = R + 2L * L * MT;
  double2 *GX = CUt;          // [L][MT]: rhs -> g -> phi
  double2 *RAB = CUt + tile;  // [L][MT]: (multiplier, reciprocal pivot)
  for (int i = tid; i < L * MT; i += CS_THR) {
    const int j = i / MT, m = i - j * MT;
    const bool ok = m < mt && j >= 1 && j <= NY;
    double2 r = make_double2(0.0, 0.0);
    if (ok && j >= 2 && j < NY) {
      const double KX = KXS[m], KZ = KZS[m], id = rowc[5 * L + j];
      const double2 a1 = U1[i], a3 = U3[i], b2 = U2[i], b2p = U2[i + MT];
      r.x = (-KX * a1.y) + (b2p.x - b2.x) * id + (-KZ * a3.y);
      r.y = (KX * a1.x) + (b2p.y - b2.y) * id + (KZ * a3.x);
    }
    GX[i] = r;
    const long o = (long)j * ss + m0 + m;
    RAB[i] = ok ? make_double2(cc.ra[o], cc.rrb[o]) : make_double2(0.0, 0.0);
  }
  __syncthreads();
  if (tid < 2 * MT) {
    const int m = tid >> 1;
    const bool mean = (m0 + m == 0);
    double *x = reinterpret_cast<double *>(GX) + tid;
    const double *RAd = reinterpret_cast<const double *>(RAB) + 2 * m;  // .x of [j][m]
    constexpr int st = 2 * MT;
    constexpr int B = 8;
    double g = 0.0;  // row 1 has a zero right-hand side
    x[1 * st] = 0.0;
    for (int j0 = 2; j0 <= NY; j0 += B) {
      double r[B], a[B];
#pragma unroll
      for (int q = 0; q < B; q++) {
        const int j = j0 + q <= NY ? j0 + q : NY;
        r[q] = x[j * st];
        a[q] = RAd[j * st];
      }
#pragma unroll
      for (int q = 0; q < B; q++) {
        if (j0 + q <= NY) {
          g = r[q] + a[q] * g;
          r[q] = g;
        }
      }
#pragma unroll
      for (int q = 0; q < B; q++)
        if (j0 + q <= NY) x[(j0 + q) * st] = r[q];
    }
    double ph = g * RAd[NY * st + 1];
    x[NY * st] = ph;
    for (int j1 = NY - 1; j1 >= 2; j1 -= B) {
      double gq[B], uq[B], bq[B];
#pragma unroll
      for (int q = 0; q < B; q++) {
        const int j = j1 - q >= 2 ? j1 - q : 2;
        gq[q] = x[j * st];
        uq[q] = __ldg(rowc + 6 * L + j);
        bq[q] = RAd[j * st + 1];
      }
#pragma unroll
      for (int q = 0; q < B; q++) {
        if (j1 - q >= 2) {
          ph = (gq[q] - uq[q] * ph) * bq[q];
          gq[q] = ph;
        }
      }
#pragma unroll
      for (int q = 0; q < B; q++)
        if (j1 - q >= 2) x[(j1 - q) * st] = gq[q];
    }
    const double u1r = mean ? 0.0 : -1.0;
    ph = (x[1 * st] - u1r * ph) * RAd[1 * st + 1];
    x[1 * st] = ph;
  }
  __syncthreads();

  // ---- 4. projection, phi, CP += phi / h; every field's rows go out
  const double ihh = 1.0 / h;
  for (int i = tid; i < nitems; i += CS_THR) {
    const int f = i / (L * MT);
    const int rem = i - f * L * MT;
    const int j = rem / MT, m = rem - j * MT;
    if (m >= mt || j < pick_w(C.wlo, f)) continue;
    const long o = (long)j * ss + m0 + m;
    double2 v = R[i];
    if (f < 3 && j >= 1 && j <= NY) {
      const double2 ph = GX[rem];
      if (f == 0 || f == 2) {
        // U1 -= i kx phi, U3 -= i kz phi
        const double K = (f == 0) ? KXS[m] : KZS[m];
        v.x -= -K * ph.y;
        v.y -= K * ph.x;
      } else if (j >= 2) {
        // U2(j) -= (phi(j) - phi(j-1)) / DY(j)
        const double2 pm = GX[rem - MT];
        const double idy = rowc[4 * L + j];
        v.x -= (ph.x - pm.x) * idy;
        v.y -= (ph.y - pm.y) * idy;
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
    cc.cu[f][o] = v;
  }
}

template <int MT>
__global__ void __launch_bounds__(CS_THR) k_col_step(const __grid_constant__ ColCase cc,
                                                    int rk_step, long spin, unsigned extra_tx) {
  extern __shared__ __align__(128) unsigned char cs_raw[];
  unsigned char *sbase = cs_raw + ((128u - (dg_smem_addr(cs_raw) & 127u)) & 127u);
  col_body<MT>(cc, rk_step, (long)blockIdx.x * MT, spin, extra_tx, sbase);
}

// Ragged launch over several cases: CTA b takes tile work[b].y of case
// work[b].x (every case at substep rk_step; the cases' MT are all MT).
template <int MT>
__global__ void __launch_bounds__(CS_THR) k_col_step_ragged(const ColCase *__restrict__ cases,
                                                           const int2 *__restrict__ work,
                                                           int rk_step) {
  extern __shared__ __align__(128) unsigned char cs_raw[];
  unsigned char *sbase = cs_raw + ((128u - (dg_smem_addr(cs_raw) & 127u)) & 127u);
  const int2 w = work[blockIdx.x];
  col_body<MT>(cases[w.x], rk_step, (long)w.y * MT, DG_ASYNC_SPIN, 0u, sbase);
}

ColConst make_col_const(const dg_handle *h) {
  ColConst c;
  c.NY = h->NY; c.nf = h->nf; c.nth = h->NTH; c.nkxp = h->nkxp; c.ss = h->ss;
  c.JS = h->jstart; c.JE = h->jend;
  for (int f = 0; f < 3 + DG_MAX_TH; f++) c.wlo[f] = 1;
  for (int n = 0; n < DG_MAX_TH; n++) {
    c.JSt[n] = h->jstart_th[n]; c.JEt[n] = h->jend_th[n];
    c.ri[n] = h->p.ri[n]; c.pr[n] = h->p.pr[n];
    c.drhodx[n] = h->p.drhodx[n]; c.drhodz[n] = h->p.drhodz[n];
    if (n < h->NTH) c.wlo[3 + n] = h->jstart_th[n] - 1;
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

size_t dg_col_smem(const dg_handle *h, int mt, int *by_out, int *nbox_out) {
  const int L = h->NY + 2;
  // boxes of at most 256 planes; a multiple of 8 planes keeps every box's
  // shared-memory destination 128-byte aligned for any modes per CTA
  const int nbox = dg_cdiv(L, 256), by = (dg_cdiv(L, nbox) + 7) / 8 * 8;
  if (by_out) *by_out = by;
  if (nbox_out) *nbox_out = nbox;
  return sizeof(double2) * (size_t)h->nf * ((size_t)nbox * by * mt + (size_t)L * mt) +
         sizeof(double) * 3 * mt + 8 + 128;
}

// The column-kernel description of handle h for `mt` modes per CTA (builds
// the tensor maps of CU for that tile width).
static int fill_case(dg_handle *h, int mt, bool rd, ColCase *cc) {
  const int L = h->NY + 2;
  int by = 0, nbox = 0;
  dg_col_smem(h, mt, &by, &nbox);
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

// modes per CTA for handle h: the tuned value, halved until the tiles fit
static int col_mt(const dg_handle *h, int want) {
  int mt = want;
  while (mt > 2 && dg_col_smem(h, mt, nullptr, nullptr) > 220 * 1024) mt /= 2;
  return mt;
}

// One launch: the column stage of substep rk_step.  rd = false stops after
// the CN solves (the velocity goes out unprojected; COURANT and REM_DIV follow).
int dg_col_step_dev(dg_handle *h, int rk_step, bool rd) {
  if (h->tables_pending) {
    DG_CUDA(cudaStreamWaitEvent(h->st, h->ev_join, 0));
    h->tables_pending = false;
  }
  const int mt = col_mt(h, h->cn_mt);
  const size_t sm = dg_col_smem(h, mt, nullptr, nullptr);
  if (sm > 220 * 1024) {
    dg_set_error("column kernel: the y-columns of two modes do not fit in shared memory");
    return DG_ERR_DIMS;
  }
  ColCase cc;
  DG_TRY(fill_case(h, mt, rd, &cc));
  // the wait test (DG_TUNE_WAIT_TEST) applies to this one launch
  const long spin = h->wait_test > 0 ? (long)h->wait_test : DG_ASYNC_SPIN;
  const unsigned extra_tx = h->wait_test > 0 ? 16u : 0u;
  h->wait_test = 0;
  const dim3 grid(dg_cdiv(h->ss, mt));
#define CS_CASE(MTV)                                                                         \
  if (mt == MTV) {                                                                           \
    dg_big_smem((const void *)k_col_step<MTV>);                                              \
    dg_kt_begin(h, rd ? "k_col_step" : "k_col_step_cn", h->st);                              \
    DG_CUDA(dg_launch(h->pdl, k_col_step<MTV>, grid, dim3(CS_THR), sm, h->st, cc, rk_step,   \
                      spin, extra_tx));                                                      \
  }
  CS_CASE(2) CS_CASE(4) CS_CASE(8) CS_CASE(16)
#undef CS_CASE
  DG_LAUNCHED();
  return DG_OK;
}

// ---------------------------------------------------------- ragged launch
// The column stage of several cases at the same substep in one launch (the
// ensemble server's batches).  dg_col_batch_build fills, for the handles,
// the host images of the case table and the work list (one (case, tile)
// pair per CTA) with one MT for all, and returns the launch's shared memory;
// the caller copies them to device memory it owns and launches with
// dg_col_batch_launch.  Results do not depend on the batch: each mode's
// arithmetic is the single-case kernel's.
size_t dg_col_case_bytes() { return sizeof(ColCase); }

int dg_col_batch_build(dg_handle *const *hs, const int *rd, int n, int want_mt,
                       std::vector<unsigned char> &cases, std::vector<int2> &work, int *mt_out,
                       size_t *smem_out) {
  int mt = want_mt;
  for (int c = 0; c < n; c++) mt = std::min(mt, col_mt(hs[c], want_mt));
  size_t sm = 0;
  for (int c = 0; c < n; c++) sm = std::max(sm, dg_col_smem(hs[c], mt, nullptr, nullptr));
  if (sm > 220 * 1024) {
    dg_set_error("column kernel: the y-columns of two modes do not fit in shared memory");
    return DG_ERR_DIMS;
  }
  cases.assign(sizeof(ColCase) * n, 0);
  work.clear();
  for (int c = 0; c < n; c++) {
    ColCase cc;
    DG_TRY(fill_case(hs[c], mt, rd[c] != 0, &cc));
    memcpy(cases.data() + sizeof(ColCase) * c, &cc, sizeof(ColCase));
    const int tiles = dg_cdiv(hs[c]->ss, mt);
    for (int t = 0; t < tiles; t++) work.push_back(make_int2(c, t));
  }
  *mt_out = mt;
  *smem_out = sm;
  return DG_OK;
}

int dg_col_batch_launch(cudaStream_t st, int mt, size_t smem, const void *dev_cases,
                        const int2 *dev_work, int nwork, int rk_step) {
#define CR_CASE(MTV)                                                                              \
  if (mt == MTV) {                                                                                \
    dg_big_smem((const void *)k_col_step_ragged<MTV>);                                            \
    k_col_step_ragged<MTV><<<nwork, CS_THR, smem, st>>>((const ColCase *)dev_cases, dev_work,     \
                                                       rk_step);                                  \
  }
  CR_CASE(2) CR_CASE(4) CR_CASE(8) CR_CASE(16)
#undef CR_CASE
  DG_LAUNCHED();
  return DG_OK;
}
