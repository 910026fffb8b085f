// The per-mode column stage of RK_CHAN_1 before REM_DIV: explicit terms, the
// Crank-Nicolson right-hand side and the CN solve of one field, for a tile of
// MT retained (kx, kz) modes and their whole y-columns.
//
// Reference steps it replaces, per mode instead of per physical column (the
// operators are linear and the same for every column, so they commute with
// the x-z transform):
//   RHS assembly     for/channel.f:88-167   CR = CU + zeta h CF - h grad P
//   explicit terms   for/channel.f:175-290  CF = -nu k^2 CU + Coriolis,
//                                           buoyancy, GRAV, DRHODX/Z + NL
//   CN explicit half for/channel.f:580-626  R += beta h CF + (nu h/2) d2/dy2 CU
//   CN solves        for/channel.f:771-1029 (THOMAS_*_MPI, for/mpi.f:630-866)
// REM_DIV_CHAN and the pressure update follow as their own launch (k_rd_col).
//
// A work item is (case, mode tile, field); one thread per (mode, segment of
// SEG_K consecutive rows).  The CN system of a field is the same for every
// mode, and its elimination (the substep's table: multipliers a, reciprocal
// pivots 1/b, f = -c/b) turns the solve into two first-order linear
// recurrences, forward g(j) = r(j) + a(j) g(j-1) and backward
// x(j) = e(j) + f(j) x(j+1) with e = g/b.  A linear recurrence splits exactly
// over segments: each thread runs its segment from a zero start, keeping the
// product of the coefficients; one lane per mode then carries the segment
// ends across the column (one step per segment instead of one per row), and
// each thread adds carry x product to its rows.  The same algebra as
// THOMAS_FORWARD / THOMAS_BACKWARD, with the rounding of a different order
// of the same operations.  Segment boundaries depend only on NY, so a mode's
// arithmetic does not depend on the tile width.
//
// One CTA per work item.  One thread fetches the field's CU tile and the NL
// term the z-forward kernel left in the field's rhs array by bulk tensor
// copies (TMA, no multicast), and the table and grid-factor rows by bulk
// copies, all at once on one mbarrier with a bounded wait.  The right-hand
// side is formed in a flat loop over (row, mode) -- CF_old and CP read there
// in batches, each batch's loads issued before its stores -- and replaces
// NL in shared memory,
// the recurrences run there (each phase loads its rows before its chain),
// and the post-CN field goes to the field's rhs array.  CU is read-only in
// this kernel, so a field's right-hand side may read another field
// (rotation, buoyancy, GRAV, DRHODX/Z) without a race.  REM_DIV then reads
// the post-CN velocity from the rhs arrays and writes CU.  A scalar that no
// velocity right-hand side reads is written in place.
//
// The same kernel serves one case (a one-case table) and the ensemble
// server's groups (a ragged work list over every member), so a case
// computes with the same machine code either way.
#include <string.h>

#include <algorithm>
#include <vector>

#include "dg_internal.cuh"

namespace {

// rows per segment of the CN recurrences: 9 keeps a 129-plane column at 8
// modes per CTA within four warps (15 segments), so that at the 128
// registers a thread takes four CTAs share an SM (five warps fit three)
constexpr int SEG_K = 9;
constexpr int COL_MAX_THR = 256; // threads per CTA: MT x segments, rounded up to warps

struct ColConst {
  int NY, nf, nth, nkxp, JS, JE;
  int JSt[DG_MAX_TH], JEt[DG_MAX_TH];
  long ss;
  double nu, beta, nuv, i_ro, grav_x, grav_y, grav_z, px0, omega0, amp_omega0;
  int f_type;
  double ri[DG_MAX_TH], pr[DG_MAX_TH], drhodx[DG_MAX_TH], drhodz[DG_MAX_TH];
};

// Everything the column stage of one case needs, in device memory (tensor
// maps first: 64-byte aligned).  Maps are 2-D over [plane][2 ss doubles].
struct ColCase {
  CUtensorMap map_cu[3 + DG_MAX_TH], map_nl[3 + DG_MAX_TH];
  ColConst C;
  const double *dscal, *tab, *kxv, *kzv, *rowc;
  const double2 *cp;
  const double2 *cu[3 + DG_MAX_TH];
  double2 *cf[3 + DG_MAX_TH], *out[3 + DG_MAX_TH];  // out: the rhs arrays
  int *err;
  int by, nbox, nseg;
};

template <typename T>
__device__ __forceinline__ T pick(const T (&a)[DG_MAX_TH], int i) {
  T r = a[0];
#pragma unroll
  for (int k = 1; k < DG_MAX_TH; k++) r = (i == k) ? a[k] : r;
  return r;
}

__device__ __forceinline__ double2 z2() { return make_double2(0.0, 0.0); }

// rowc: per-row grid factors [8][LP] (LP = NY + 2 rounded up to even, so
// rows start on 16-byte boundaries for the bulk copies)
//   0 1/(DY(j+1) DYF(j))  1 1/(DY(j) DYF(j))       (GYF rows: U1, U3, TH)
//   2 1/(DYF(j) DY(j))    3 1/(DYF(j-1) DY(j))     (GY rows: U2)
//   4 1/DY(j)             5 DYF(j)                 (U2)
//   6 1/DYF(j)            7 REM_DIV upper diagonal

// The field's coefficients that do not change along the column.
// Everything the right-hand side of one field needs besides the tiles, read
// from the case table once per CTA into registers (the loop that uses them
// stores to global memory, after which the compiler would have to reload
// anything it reads from the table).
struct FieldCoef {
  double T3, T4, T5, aaU, NU, nup, ipr, ddx, ddz, sgn, time;
  double i_ro, px0, amp_omega0, omega0;
  double w[DG_MAX_TH];              // coupling weight of each scalar (0: none)
  const double2 *th[DG_MAX_TH];     // the scalars' CU
  const double2 *uo;                // the other horizontal velocity (rotation)
  const double2 *u1, *u3;           // U1, U3 (DRHODX/Z in a scalar's equation)
  long ss;
  int lo, hi, nth, f_type;
};

__device__ __forceinline__ FieldCoef field_coef(const ColCase &cc, int rk_step, int f) {
  const ColConst &C = cc.C;
  FieldCoef k;
  const double h = cc.dscal[1 + rk_step];
  const double zeta = (rk_step == 2) ? -17.0 / 8.0 : (rk_step == 3) ? -5.0 / 4.0 : 0.0;
  const double bbar = (rk_step == 2) ? 25.0 / 8.0 : (rk_step == 3) ? 9.0 / 4.0 : 1.0;
  const double T1 = C.nu * h / 2.0;
  k.T3 = zeta * h;
  k.T4 = h;
  k.T5 = bbar * h;
  k.aaU = T1 * C.nuv;
  k.NU = C.nu;
  k.time = cc.dscal[0];
  const int n = f - 3;
  k.nup = (f >= 3) ? C.nu / pick(C.pr, n) : C.nu;
  k.ipr = (f >= 3) ? 1.0 / pick(C.pr, n) : 1.0;
  k.ddx = (f >= 3) ? pick(C.drhodx, n) : 0.0;
  k.ddz = (f >= 3) ? pick(C.drhodz, n) : 0.0;
  k.sgn = (f == 0) ? 1.0 : -1.0;
  k.i_ro = C.i_ro;
  k.px0 = C.px0;
  k.amp_omega0 = C.amp_omega0;
  k.omega0 = C.omega0;
  k.f_type = C.f_type;
  k.nth = C.nth;
  k.ss = C.ss;
  // U1, U3: RI GRAV_x/z TH; U2: RI GRAV_y times the GY interpolation
  const double gr = (f == 0) ? C.grav_x : (f == 2) ? C.grav_z : C.grav_y;
#pragma unroll
  for (int q = 0; q < DG_MAX_TH; q++) {
    k.w[q] = (q < C.nth && f < 3) ? C.ri[q] * gr : 0.0;
    k.th[q] = cc.cu[3 + (q < C.nth ? q : 0)];
  }
  k.uo = cc.cu[(f == 0) ? 2 : 0];
  k.u1 = cc.cu[0];
  k.u3 = cc.cu[2];
  if (f == 0 || f == 2) { k.lo = C.JS; k.hi = C.JE; }
  else if (f == 1) { k.lo = 2; k.hi = C.NY; }
  else { k.lo = pick(C.JSt, n); k.hi = pick(C.JEt, n); }
  return k;
}

// The explicit terms fv (the new CF) and the CN right-hand side r of field f
// at row j, mode offset o: u, um, up = CU at j, j-1, j+1; nlv = NL;
// old = CF_old; p0, pm = CP at j, j-1.  RC: the field's grid-factor rows in
// shared memory, row stride ld: rows 0, 1 (U1, U3, TH) or 2, 3, 4, 5 (U2).
template <int FK>
__device__ __forceinline__ void rhs_row(const FieldCoef &k, int f, int j, long o, bool mean,
                                        double KX, double KZ, double kk, const double *RC, int ld,
                                        double2 u, double2 um, double2 up, double2 nlv,
                                        double2 old, double2 p0, double2 pm, double2 &fv,
                                        double2 &r) {
  if constexpr (FK == 0) {
    fv = make_double2(-k.NU * kk * u.x, -k.NU * kk * u.y);
    if (k.i_ro != 0.0) {
      const double2 uo = k.uo[o];
      fv.x += k.sgn * k.i_ro * uo.x;
      fv.y += k.sgn * k.i_ro * uo.y;
    }
#pragma unroll
    for (int q = 0; q < DG_MAX_TH; q++) {
      const double w = k.w[q];
      if (q >= k.nth || w == 0.0) continue;
      const double2 t = k.th[q][o];
      fv.x += w * t.x;
      fv.y += w * t.y;
    }
    fv.x += nlv.x;
    fv.y += nlv.y;
    r = u;
    r.x += k.T3 * old.x;
    r.y += k.T3 * old.y;
    const double K = (f == 0) ? KX : KZ;
    r.x -= k.T4 * (-K * p0.y);
    r.y -= k.T4 * (K * p0.x);
    if (f == 0 && mean) {
      if (k.f_type == 1) r.x -= k.T4 * k.px0;
      else if (k.f_type == 2) r.x -= k.T4 * (k.px0 + k.amp_omega0 * cos(k.omega0 * k.time));
    }
    r.x += k.T5 * fv.x;
    r.y += k.T5 * fv.y;
    const double cup = k.aaU * RC[0 * ld + j], cdn = k.aaU * RC[1 * ld + j];
    r.x += cup * (up.x - u.x) - cdn * (u.x - um.x);
    r.y += cup * (up.y - u.y) - cdn * (u.y - um.y);
  } else if constexpr (FK == 1) {
    fv = make_double2(-k.NU * kk * u.x, -k.NU * kk * u.y);
    if (!mean) {
      const double dyfj = RC[3 * ld + j], dyfm = RC[3 * ld + j - 1];
      const double bw2 = 0.5 * RC[2 * ld + j];
#pragma unroll
      for (int q = 0; q < DG_MAX_TH; q++) {
        if (q >= k.nth || k.w[q] == 0.0) continue;
        const double w = k.w[q] * bw2;
        const double2 t = k.th[q][o], tm = k.th[q][o - k.ss];
        fv.x += w * (t.x * dyfm + tm.x * dyfj);
        fv.y += w * (t.y * dyfm + tm.y * dyfj);
      }
    }
    fv.x += nlv.x;
    fv.y += nlv.y;
    r = u;
    r.x += k.T3 * old.x;
    r.y += k.T3 * old.y;
    const double idy = RC[2 * ld + j];
    r.x -= k.T4 * ((p0.x - pm.x) * idy);
    r.y -= k.T4 * ((p0.y - pm.y) * idy);
    r.x += k.T5 * fv.x;
    r.y += k.T5 * fv.y;
    const double cup2 = k.aaU * RC[0 * ld + j], cdn2 = k.aaU * RC[1 * ld + j];
    r.x += cup2 * (up.x - u.x) - cdn2 * (u.x - um.x);
    r.y += cup2 * (up.y - u.y) - cdn2 * (u.y - um.y);
  } else {
    fv = make_double2(-k.nup * kk * u.x, -k.nup * kk * u.y);
    if (k.ddx != 0.0 || k.ddz != 0.0) {
      const double2 u1 = k.u1[o], u3 = k.u3[o];
      fv.x = fv.x - u1.x * k.ddx - u3.x * k.ddz;
      fv.y = fv.y - u1.y * k.ddx - u3.y * k.ddz;
    }
    fv.x += nlv.x;
    fv.y += nlv.y;
    r = u;
    r.x += k.T3 * old.x;
    r.y += k.T3 * old.y;
    r.x += k.T5 * fv.x;
    r.y += k.T5 * fv.y;
    const double cup = k.aaU * RC[0 * ld + j], cdn = k.aaU * RC[1 * ld + j];
    r.x += k.ipr * (cup * (up.x - u.x) - cdn * (u.x - um.x));
    r.y += k.ipr * (cup * (up.y - u.y) - cdn * (u.y - um.y));
  }
}

// Launch-wide sizes: the largest item of the work list sets the layout.
struct ColLaunch {
  int tile;   // double2 per tile (nbox * by * MT of the largest case)
  int lp;     // table row length (the largest case's NY + 2, rounded up to even)
  int nseg;   // segments per column (the largest case)
  int nwork;  // work items (CTAs)
};

// Shared memory of one CTA (128-byte aligned): the tiles CU and NL (then R,
// g, e and x of the recurrences) [tile] double2; the CN table
// rows TB [5][lp] (a, 1/b, f = -c/b, kind, BC value); the field's grid
// factors RC [4][lp]; per (segment, mode) values SV [nseg][MT] double2
// (then carries); per segment products SP [nseg]; the modes' wavenumbers
// and k^2 (to the power BETA) KW [3][MT]; the mbarrier.
size_t col_smem_l(const ColLaunch &P, int mt) {
  return sizeof(double2) * (2 * (size_t)P.tile + (size_t)P.nseg * mt) +
         sizeof(double) * (9 * (size_t)P.lp + (size_t)P.nseg + 3 * (size_t)mt) + 8 + 128;
}

// The right-hand side of field f (kind FK: 0 U1/U3, 1 U2, 2 scalar) for the
// CTA's rows lo..hi: a flat loop over (row, mode) elements in batches of
// four per thread; CU and NL from the staged tiles, CF_old and CP read
// directly (each element once, coalesced).  CF_old is the array the loop
// writes CF into, so a batch's loads are all issued before its stores; CP
// is read-only here and goes through the read-only data path.  R replaces
// NL.  Everything else the loop reads is in registers or shared memory.
template <int MT, int FK>
__device__ __forceinline__ void rhs_tile(const FieldCoef &k, int rk_step, long m0, int f, int mt,
                                         double2 *cff, const double2 *cpp, const double2 *CUt,
                                         double2 *NLt, const double *RC, int LP,
                                         const double *KW) {
  const bool old_cf = rk_step > 1;
  const int nthr = blockDim.x;
  const int i0 = k.lo * MT + (int)threadIdx.x, iend = (k.hi + 1) * MT;
  constexpr int B = 4;
  for (int base = i0; base < iend; base += B * nthr) {
    double2 old[B], p0[B], pm[B];
#pragma unroll
    for (int u = 0; u < B; u++) {
      const int i = base + u * nthr;
      const int j = i / MT, m = i - j * MT;
      const bool ok = i < iend && m < mt;
      const long o = (long)j * k.ss + m0 + m;
      old[u] = (ok && old_cf) ? cff[o] : z2();
      p0[u] = (ok && FK < 2) ? __ldg(cpp + o) : z2();
      pm[u] = (ok && FK == 1) ? __ldg(cpp + o - k.ss) : z2();
    }
#pragma unroll
    for (int u = 0; u < B; u++) {
      const int i = base + u * nthr;
      const int j = i / MT, m = i - j * MT;
      if (i < iend && m < mt) {
        const long mg = m0 + m;
        const long o = (long)j * k.ss + mg;
        double2 fv, rr;
        rhs_row<FK>(k, f, j, o, mg == 0, KW[m], KW[MT + m], KW[2 * MT + m], RC, LP, CUt[i],
                    CUt[i - MT], CUt[i + MT], NLt[i], old[u], p0[u], pm[u], fv, rr);
        cff[o] = fv;
        NLt[i] = rr;
      }
    }
  }
}

// Carry the per-segment values e(t) through the segments in order
// t = t0, t0 + dt, ..., n steps: X(t) = e(t) + p(t) X(previous), storing the
// carry into each segment (its value before the segment) in place of e(t).
template <int MT>
__device__ __forceinline__ void carry_chain(double2 *SV, const double *SP, int t0, int dt, int n,
                                            int m) {
  double2 X = z2();
  for (int b = 0; b < n; b++) {
    const int t = t0 + dt * b;
    const double2 e = SV[t * MT + m];
    const double p = SP[t];
    SV[t * MT + m] = X;
    X = make_double2(e.x + p * X.x, e.y + p * X.y);
  }
}

// The column stage of field f for modes m0 .. m0+MT-1 of one case.  Every
// value the CTA needs from the case table is read before its first global
// store (after which the compiler would have to reload it).
template <int MT>
__device__ __forceinline__ void col_body(const ColCase &cc, int rk_step, long m0, int f,
                                         const ColLaunch &P, long spin, unsigned extra_tx,
                                         unsigned char *sbase) {
  const int NY = cc.C.NY, L = NY + 2, LP = (L + 1) & ~1;  // the case's own row length
  const int nseg = cc.nseg;
  const long ss = cc.C.ss;
  const int mt = (int)((ss - m0) < MT ? (ss - m0) : MT);
  const int wlo = (f >= 3) ? pick(cc.C.JSt, f - 3) - 1 : 1;  // first row solved
  double2 *const dst = cc.out[f];
  double2 *const cff = cc.cf[f];
  int *const err = cc.err;
  const FieldCoef k = field_coef(cc, rk_step, f);
  double2 *CUt = reinterpret_cast<double2 *>(sbase);
  double2 *NLt = CUt + P.tile;
  double *TB = reinterpret_cast<double *>(NLt + P.tile);
  const double2 *const cpp = cc.cp;
  double *RC = TB + 5 * P.lp;  // the slots are sized for the largest case
  double2 *SV = reinterpret_cast<double2 *>(RC + 4 * P.lp);
  double *SP = reinterpret_cast<double *>(SV + P.nseg * MT);
  double *KW = SP + P.nseg;
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(KW + 3 * MT);
  const int tid = threadIdx.x;
  if (tid < MT) {
    const long mg = (m0 + tid < ss) ? m0 + tid : 0;
    const double KX = cc.kxv[mg % cc.C.nkxp], KZ = cc.kzv[mg / cc.C.nkxp];
    const double k2 = KX * KX + KZ * KZ;
    KW[tid] = KX;
    KW[MT + tid] = KZ;
    KW[2 * MT + tid] = (cc.C.beta == 1.0) ? k2 : pow(k2, cc.C.beta);
  }

  // ---- 0. the field's tiles by bulk tensor copies, the table and grid-
  // factor rows by bulk copies, all in flight at once on one mbarrier
  if (tid == 0) dg_mbar_init(bar, 1);
  __syncthreads();
  dg_pdl_wait();  // NL comes from the z-forward kernel
  if (tid == 0) {
    const int ctile = cc.nbox * cc.by * MT;
    const unsigned ntiles = 2u;
    const int nrc = (f == 1) ? 4 : 2;  // grid-factor rows 2..5 (U2) or 0..1
    // extra_tx is 0 except in the wait test, where the barrier then never completes
    dg_mbar_expect_tx(bar, (unsigned)(sizeof(double2) * ctile) * ntiles +
                               (unsigned)(sizeof(double) * (5 + nrc) * LP) + extra_tx);
    // columns beyond ss and planes beyond L arrive as zeros
    for (int q = 0; q < cc.nbox; q++) {
      const long d = (long)q * cc.by * MT;
      const int x = (int)(2 * m0), y = q * cc.by;
      dg_tma_load_2d(CUt + d, &cc.map_cu[f], x, y, bar);
      dg_tma_load_2d(NLt + d, &cc.map_nl[f], x, y, bar);
    }
    dg_bulk_load(TB, cc.tab + ((long)(rk_step - 1) * (3 + DG_MAX_TH) + f) * 5 * LP,
                 (unsigned)(sizeof(double) * 5 * LP), bar);
    dg_bulk_load(RC, cc.rowc + (long)(f == 1 ? 2 : 0) * LP,
                 (unsigned)(sizeof(double) * nrc * LP), bar);
  }
  const bool landed = dg_mbar_wait(bar, 0, spin);
  if (__syncthreads_or(!landed)) {
    if (tid == 0) {
      atomicExch(err + 1, 1);
      dg_mbar_wait(bar, 0, spin);  // the copies in flight get one more bounded wait
    }
    return;
  }

  // ---- 1. explicit terms, CF and the right-hand side of rows lo..hi
  if (f == 1) rhs_tile<MT, 1>(k, rk_step, m0, f, mt, cff, cpp, CUt, NLt, RC, LP, KW);
  else if (f < 3) rhs_tile<MT, 0>(k, rk_step, m0, f, mt, cff, cpp, CUt, NLt, RC, LP, KW);
  else rhs_tile<MT, 2>(k, rk_step, m0, f, mt, cff, cpp, CUt, NLt, RC, LP, KW);
  __syncthreads();

  // ---- 2. forward recurrence g(j) = r(j) + a(j) g(j-1) over each segment
  // from zero (one thread per mode and segment); r is R on CN rows, the BC
  // value (the (0,0) mode's real part) or zero elsewhere; g replaces R.
  // Each phase loads its rows first, then runs its chain.
  const int m = tid % MT, s = tid / MT;
  const int j0 = s * SEG_K;
  const int nr = (s < nseg) ? min(SEG_K, L - j0) : 0;  // rows of this thread's segment
  const long mg = m0 + m;
  const bool live = m < mt;
  const bool mean = (mg == 0);
  double a[SEG_K];
  {
    double2 r[SEG_K];
#pragma unroll
    for (int q = 0; q < SEG_K; q++) {
      const int j = (q < nr) ? j0 + q : 0;
      const double kind = TB[3 * LP + j];
      const double2 rv = NLt[j * MT + m];
      const double bc = TB[4 * LP + j];
      r[q] = (kind == (double)ROW_RHS)
                 ? rv
                 : make_double2((kind == (double)ROW_BC && mean) ? bc : 0.0, 0.0);
      a[q] = TB[j];
    }
    double2 g = z2();
    double pa = 1.0;
#pragma unroll
    for (int q = 0; q < SEG_K; q++) {
      if (q < nr) {
        g.x = r[q].x + a[q] * g.x;
        g.y = r[q].y + a[q] * g.y;
        pa = a[q] * pa;
        NLt[(j0 + q) * MT + m] = g;
      }
    }
    if (nr > 0) {
      SV[s * MT + m] = g;
      if (m == 0) SP[s] = pa;
    }
  }
  __syncthreads();
  // ---- 3. the segment ends carried down the column, one lane per mode
  if (tid < MT) carry_chain<MT>(SV, SP, 0, 1, nseg, tid);
  __syncthreads();
  // ---- 4. g = local + product x carry, e = g / b; then the backward
  // recurrence x(j) = e(j) + f(j) x(j+1) over the segment (rows >= wlo)
  const int qb = wlo > j0 ? wlo - j0 : 0;  // first row of the segment to solve
  const bool solves = nr > 0 && qb < nr;
  double fc[SEG_K];
  {
    const double2 c = (nr > 0) ? SV[s * MT + m] : z2();
    double2 e[SEG_K];
    double rb[SEG_K];
#pragma unroll
    for (int q = 0; q < SEG_K; q++) {
      const int j = (q < nr) ? j0 + q : 0;
      e[q] = NLt[j * MT + m];
      rb[q] = TB[LP + j];
      fc[q] = TB[2 * LP + j];
    }
    double pi = 1.0;
#pragma unroll
    for (int q = 0; q < SEG_K; q++) {
      pi = a[q] * pi;
      e[q] = make_double2((e[q].x + pi * c.x) * rb[q], (e[q].y + pi * c.y) * rb[q]);
    }
    double2 xl = z2();
    double ps = 1.0;
#pragma unroll
    for (int q = SEG_K - 1; q >= 0; q--) {
      if (q < nr && q >= qb) {
        xl = make_double2(e[q].x + fc[q] * xl.x, e[q].y + fc[q] * xl.y);
        ps = fc[q] * ps;
        NLt[(j0 + q) * MT + m] = xl;
      }
    }
    // each thread overwrites only its own SV entry, read above by itself;
    // SP was last read in step 3, before the barrier
    if (solves) {
      SV[s * MT + m] = xl;
      if (m == 0) SP[s] = ps;
    }
  }
  __syncthreads();
  // ---- 5. the segment starts carried up the column, one lane per mode
  const int sw = wlo / SEG_K;  // lowest segment with rows to solve
  if (tid < MT) carry_chain<MT>(SV, SP, nseg - 1, -1, nseg - sw, tid);
  __syncthreads();
  // ---- 6. x = local + product x carry: the post-CN field, rows >= wlo
  if (solves && live) {
    const double2 c = SV[s * MT + m];
    double2 xl[SEG_K];
#pragma unroll
    for (int q = 0; q < SEG_K; q++) xl[q] = NLt[((q < nr) ? j0 + q : 0) * MT + m];
    double p2 = 1.0;
#pragma unroll
    for (int q = SEG_K - 1; q >= 0; q--) {
      if (q < nr && q >= qb) {
        p2 = fc[q] * p2;
        dst[(long)(j0 + q) * ss + mg] = make_double2(xl[q].x + p2 * c.x, xl[q].y + p2 * c.y);
      }
    }
  }
}

// The column kernel: CTA b takes work[b] = (case, mode tile, field) from
// the case table (every case at substep rk_step with MT modes per CTA).
template <int MT>
__global__ void __launch_bounds__(COL_MAX_THR, 2) k_col_cn(const ColCase *__restrict__ cases,
                                                       const int4 *__restrict__ work,
                                                       ColLaunch P, int rk_step, long spin,
                                                       unsigned extra_tx) {
  extern __shared__ __align__(128) unsigned char cs_raw[];
  unsigned char *sbase = cs_raw + ((128u - (dg_smem_addr(cs_raw) & 127u)) & 127u);
  const int4 w = work[blockIdx.x];
  col_body<MT>(cases[w.x], rk_step, (long)w.y * MT, w.z, P, spin, extra_tx, sbase);
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

// Whether the column stage leaves scalar n in its rhs array (for k_rd_col to
// copy into CU) rather than writing it in place: a velocity right-hand side
// of the same launch reads the scalar's CU when RI * GRAV_x/y/z is nonzero.
bool dg_col_th_to_rhs(const dg_handle *h, int n) {
  const double ri = h->p.ri[n];
  return ri * h->p.grav_x != 0.0 || ri * h->p.grav_y != 0.0 || ri * h->p.grav_z != 0.0;
}

// Per-row grid factors of the column kernel (once per handle, host side).
int dg_col_init(dg_handle *h) {
  const int L = h->NY + 2, LP = (L + 1) / 2 * 2;
  double *t = (double *)calloc((size_t)8 * LP, sizeof(double));
  if (!t) return DG_ERR_OOM;
  const double *dy = h->h_dy, *dyf = h->h_dyf;
  for (int j = 1; j <= h->NY; j++) {
    t[0 * LP + j] = 1.0 / (dy[j + 1] * dyf[j]);
    t[1 * LP + j] = 1.0 / (dy[j] * dyf[j]);
    t[2 * LP + j] = 1.0 / (dyf[j] * dy[j]);
    t[3 * LP + j] = 1.0 / (dyf[j - 1] * dy[j]);
    t[6 * LP + j] = 1.0 / dyf[j];
    t[7 * LP + j] = (j >= 2 && j < h->NY) ? 1.0 / (dy[j + 1] * dyf[j]) : 0.0;
  }
  for (int j = 1; j < L; j++) t[4 * LP + j] = 1.0 / dy[j];
  for (int j = 0; j < L; j++) t[5 * LP + j] = dyf[j];
  cudaError_t e = dg_malloc(h, (void **)&h->rowc, sizeof(double) * 8 * LP);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h->rowc, t, sizeof(double) * 8 * LP, cudaMemcpyHostToDevice, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  free(t);
  DG_CUDA(e);
  return DG_OK;
}

static void col_geometry(const dg_handle *h, int *by, int *nbox, int *nseg) {
  const int L = h->NY + 2;
  // boxes of at most 256 planes; a multiple of 8 planes keeps every box's
  // shared-memory destination 128-byte aligned for any modes per CTA
  *nbox = dg_cdiv(L, 256);
  *by = (dg_cdiv(L, *nbox) + 7) / 8 * 8;
  *nseg = dg_cdiv(L, SEG_K);
}

// launch sizes of handle h alone at mt modes per CTA (nwork left 0)
static ColLaunch col_sizes(const dg_handle *h, int mt) {
  int by, nbox, nseg;
  col_geometry(h, &by, &nbox, &nseg);
  ColLaunch P;
  P.tile = nbox * by * mt;
  P.lp = (h->NY + 2 + 1) / 2 * 2;
  P.nseg = nseg;
  P.nwork = 0;
  return P;
}

// threads of one CTA for handle h at mt modes: one per (mode, segment), and
// at least 128 for the flat right-hand-side loop
static int col_threads(const dg_handle *h, int mt) {
  return std::max(128, (mt * col_sizes(h, mt).nseg + 31) / 32 * 32);
}

size_t dg_col_smem(const dg_handle *h, int mt) { return col_smem_l(col_sizes(h, mt), mt); }

// The case description of handle h for `mt` modes per CTA (builds the
// tensor maps of its CU and rhs arrays for that tile width).
static int fill_case(dg_handle *h, int mt, ColCase *cc) {
  const int L = h->NY + 2;
  int by = 0, nbox = 0, nseg = 0;
  col_geometry(h, &by, &nbox, &nseg);
  memset(cc, 0, sizeof(*cc));
  for (int f = 0; f < h->nf; f++) {
    DG_TRY(dg_tmap_planes(h->cu[f], h->ss, L, mt, by, &cc->map_cu[f]));
    DG_TRY(dg_tmap_planes(h->rhs[f], h->ss, L, mt, by, &cc->map_nl[f]));
  }
  cc->cp = h->cp;
  cc->C = make_col_const(h);
  cc->dscal = h->dscal;
  cc->tab = h->cn_tab;
  cc->kxv = h->kx;
  cc->kzv = h->kz;
  cc->rowc = h->rowc;
  for (int f = 0; f < h->nf; f++) {
    cc->cu[f] = h->cu[f];
    cc->cf[f] = h->cf[f];
    cc->out[f] = (f < 3 || dg_col_th_to_rhs(h, f - 3)) ? h->rhs[f] : h->cu[f];
  }
  cc->err = h->dflag;
  cc->by = by;
  cc->nbox = nbox;
  cc->nseg = nseg;
  return DG_OK;
}

// modes per CTA for handle h: the tuned value, halved until the CTA fits
// (two stages in shared memory, one thread per mode and segment)
static int col_mt(const dg_handle *h, int want) {
  int mt = want;
  while (mt > 2 && (dg_col_smem(h, mt) > 220 * 1024 || col_threads(h, mt) > COL_MAX_THR)) mt /= 2;
  return mt;
}

static int col_fits(const dg_handle *h, int mt) {
  if (dg_col_smem(h, mt) > 220 * 1024 || col_threads(h, mt) > COL_MAX_THR) {
    dg_set_error("column kernel: NY too large for two modes per CTA (NY + 2 <= 1024)");
    return DG_ERR_DIMS;
  }
  return DG_OK;
}

int dg_col_mt_eff(const dg_handle *h) { return col_mt(h, h->cn_mt); }

// the work list of one case: (case c, tile, field, 0) per item
static void case_work(const dg_handle *h, int c, int mt, std::vector<int4> &work) {
  const int tiles = dg_cdiv(h->ss, mt);
  for (int f = 0; f < h->nf; f++)
    for (int t = 0; t < tiles; t++) work.push_back(make_int4(c, t, f, 0));
}

// The handle's device copy of its one-case table and work list for mt,
// rebuilt when mt changes.  The copies are synchronous, so they cannot run
// inside a stream capture: diablo_step's first step of a kind, which runs
// eagerly, builds them before any capture.
static int col_tables(dg_handle *h, int mt) {
  if (h->col_dcase && h->col_dmt == mt) return DG_OK;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(h->st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
    dg_set_error("the column kernel's case table must be built before a stream capture "
                 "(run one substep eagerly after changing the tuning)");
    return DG_ERR_ARG;
  }
  ColCase cc;
  DG_TRY(fill_case(h, mt, &cc));
  std::vector<int4> work;
  case_work(h, 0, mt, work);
  DG_CUDA(cudaStreamSynchronize(h->st));
  if (h->col_dcase) dg_free(h, h->col_dcase);
  if (h->col_dwork) dg_free(h, h->col_dwork);
  h->col_dcase = nullptr;
  h->col_dwork = nullptr;
  DG_CUDA(dg_malloc(h, &h->col_dcase, sizeof(cc)));
  DG_CUDA(dg_malloc(h, (void **)&h->col_dwork, sizeof(int4) * work.size()));
  DG_CUDA(cudaMemcpyAsync(h->col_dcase, &cc, sizeof(cc), cudaMemcpyHostToDevice, h->st));
  DG_CUDA(cudaMemcpyAsync(h->col_dwork, work.data(), sizeof(int4) * work.size(),
                          cudaMemcpyHostToDevice, h->st));
  DG_CUDA(cudaStreamSynchronize(h->st));
  h->col_dmt = mt;
  h->col_dnwork = (int)work.size();
  return DG_OK;
}

static int launch_col(cudaStream_t st, int pdl, const dg_col_launch &cl, const void *dev_cases,
                      const int4 *dev_work, int rk_step, long spin, unsigned extra_tx) {
  ColLaunch P;
  P.tile = cl.tile;
  P.lp = cl.lp;
  P.nseg = cl.nseg;
  P.nwork = cl.nwork;
#define CS_CASE(MTV)                                                                            \
  if (cl.mt == MTV) {                                                                           \
    dg_big_smem((const void *)k_col_cn<MTV>);                                                   \
    DG_CUDA(dg_launch(pdl, k_col_cn<MTV>, dim3(cl.grid), dim3(cl.thr), cl.smem, st,             \
                      (const ColCase *)dev_cases, dev_work, P, rk_step, spin, extra_tx));       \
  }
  CS_CASE(2) CS_CASE(4) CS_CASE(8) CS_CASE(16)
#undef CS_CASE
  DG_LAUNCHED();
  return DG_OK;
}

// launch sizes of handles hs together at `want` modes per CTA: the largest
// any of them needs (a case's CTAs leave threads beyond its own segments idle)
static int col_plan(dg_handle *const *hs, int n, int want, int nwork, dg_col_launch *cl) {
  int mt = want;
  for (int c = 0; c < n; c++) mt = std::min(mt, col_mt(hs[c], want));
  dg_col_launch r = {};
  r.mt = mt;
  for (int c = 0; c < n; c++) {
    DG_TRY(col_fits(hs[c], mt));
    const ColLaunch P = col_sizes(hs[c], mt);
    r.tile = std::max(r.tile, P.tile);
    r.lp = std::max(r.lp, P.lp);
    r.nseg = std::max(r.nseg, P.nseg);
    r.thr = std::max(r.thr, col_threads(hs[c], mt));
  }
  ColLaunch P;
  P.tile = r.tile;
  P.lp = r.lp;
  P.nseg = r.nseg;
  P.nwork = nwork;
  r.smem = col_smem_l(P, mt);
  if (r.smem > 220 * 1024) {
    dg_set_error("column kernel: the cases' tiles do not fit in shared memory together");
    return DG_ERR_DIMS;
  }
  r.nwork = nwork;
  r.grid = nwork;  // one CTA per work item
  *cl = r;
  return DG_OK;
}

// The column stage of substep rk_step: right-hand sides and CN solves of
// every field (k_col_cn; the post-CN fields land in the rhs arrays), then,
// when rd, REM_DIV and the pressure update from there into CU (k_rd_col).
// rd = false leaves REM_DIV to the caller (COURANT runs between them).
int dg_col_step_dev(dg_handle *h, int rk_step, bool rd) {
  if (h->tables_pending) {
    DG_CUDA(cudaStreamWaitEvent(h->st, h->ev_join, 0));
    h->tables_pending = false;
  }
  const int mt = col_mt(h, h->cn_mt);
  DG_TRY(col_fits(h, mt));
  DG_TRY(col_tables(h, mt));
  dg_col_launch cl;
  dg_handle *hs[1] = {h};
  DG_TRY(col_plan(hs, 1, mt, h->col_dnwork, &cl));
  // the wait test (DG_TUNE_WAIT_TEST) applies to this one launch
  const long spin = h->wait_test > 0 ? (long)h->wait_test : DG_ASYNC_SPIN;
  const unsigned extra_tx = h->wait_test > 0 ? 16u : 0u;
  h->wait_test = 0;
  dg_kt_begin(h, "k_col_cn", h->st);
  DG_TRY(launch_col(h->st, h->pdl, cl, h->col_dcase, h->col_dwork, rk_step, spin, extra_tx));
  if (rd) DG_TRY(dg_rem_div_dev(h, 1, rk_step, true));
  return DG_OK;
}

// ---------------------------------------------------------- ragged launch
// The column stage of several cases at the same substep in one launch (the
// ensemble server's groups).  dg_col_batch_build fills, for the handles, the
// host images of the case table and the work list (one (case, tile, field)
// entry per item) with one MT for all, and the launch sizes; the caller
// copies the images to device memory it owns and launches with
// dg_col_batch_launch.  Each case's REM_DIV follows on its own stream.
// Results do not depend on the batch: each mode's arithmetic is the
// single-case launch's, with the same kernel.
int dg_col_batch_build(dg_handle *const *hs, int n, int want_mt, std::vector<unsigned char> &cases,
                       std::vector<int4> &work, dg_col_launch *cl) {
  int mt = want_mt;
  for (int c = 0; c < n; c++) mt = std::min(mt, col_mt(hs[c], want_mt));
  cases.assign(sizeof(ColCase) * n, 0);
  work.clear();
  for (int c = 0; c < n; c++) {
    ColCase cc;
    DG_TRY(fill_case(hs[c], mt, &cc));
    memcpy(cases.data() + sizeof(ColCase) * c, &cc, sizeof(ColCase));
    case_work(hs[c], c, mt, work);
  }
  return col_plan(hs, n, mt, (int)work.size(), cl);
}

int dg_col_batch_launch(cudaStream_t st, const dg_col_launch &cl, const void *dev_cases,
                        const int4 *dev_work, int rk_step) {
  return launch_col(st, 0, cl, dev_cases, dev_work, rk_step, DG_ASYNC_SPIN, 0u);
}
