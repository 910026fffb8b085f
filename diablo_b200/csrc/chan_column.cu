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
// One CTA per (mode tile, field).  Every input tile of the field -- CU, the
// nonlinear term NL that the z-forward kernel left in the field's rhs array,
// CF_old (substeps 2, 3) and CP (velocity fields) -- arrives in shared
// memory by bulk tensor copies (TMA, no multicast), all issued at once by one
// thread and completed on one mbarrier with a bounded wait, so the CTA has
// its whole column in flight before it computes anything.  The right-hand
// side is formed in place of NL, the CN recurrences (one lane per mode, the
// real and imaginary parts interleaved) run in shared memory with the row
// tables staged there too, and the post-CN field goes to the field's rhs
// array: CU is read-only in this kernel, so a field's right-hand side may
// read another field (rotation, buoyancy, GRAV, DRHODX/Z) without a race.
// REM_DIV then reads the post-CN velocity from the rhs arrays and writes CU.
// A scalar that no velocity right-hand side reads is written in place.
//
// The same kernel serves one case (a one-case table) and the ensemble
// server's groups (a ragged (case, tile, field) work list over every member),
// so a case computes with the same machine code either way.
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

// Everything the column stage of one case needs, in device memory (tensor
// maps first: 64-byte aligned).  Maps are 2-D over [plane][2 ss doubles].
struct ColCase {
  CUtensorMap map_cu[3 + DG_MAX_TH], map_nl[3 + DG_MAX_TH], map_cf[3 + DG_MAX_TH];
  CUtensorMap map_cp;
  ColConst C;
  const double *dscal, *tab, *kxv, *kzv, *rowc;
  const double2 *cu[3 + DG_MAX_TH];
  double2 *cf[3 + DG_MAX_TH], *out[3 + DG_MAX_TH];  // out: the rhs arrays
  int *err;
  int by, nbox;
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
// The column stage of field f for modes m0 .. m0+MT-1 of one case.  sbase:
// the CTA's 128-byte aligned dynamic shared memory.
template <int MT>
__device__ __forceinline__ void col_body(const ColCase &cc, int rk_step, long m0, int f,
                                         long spin, unsigned extra_tx, unsigned char *sbase) {
  const ColConst &C = cc.C;
  const int NY = C.NY, L = NY + 2, nth = C.nth;
  const int by = cc.by, nbox = cc.nbox;
  const long ss = C.ss;
  const int mt = (int)((ss - m0) < MT ? (ss - m0) : MT);
  const bool vel = f < 3;
  const bool old_cf = rk_step > 1;
  const int tile = nbox * by * MT;                                 // double2 per tile
  double2 *CUt = reinterpret_cast<double2 *>(sbase);               // CU
  double2 *NLt = CUt + tile;                                       // NL -> R -> solution
  double2 *CFt = NLt + tile;                                       // CF_old
  double2 *CPt = CFt + tile;                                       // CP
  double *TB = reinterpret_cast<double *>(CPt + tile);             // [5][L] CN tables
  double *KXS = TB + 5 * L, *KZS = KXS + MT, *KKS = KZS + MT;      // [MT]
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(KKS + MT);
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
  const double *tab_f = cc.tab + ((long)(rk_step - 1) * (3 + DG_MAX_TH) + f) * 5 * L;
  for (int i = tid; i < 5 * L; i += CS_THR) TB[i] = tab_f[i];
  __syncthreads();
  dg_pdl_wait();  // NL comes from the z-forward kernel
  if (tid == 0) {
    // columns beyond ss and planes beyond L arrive as zeros (extra_tx is 0
    // except in the wait test, where the barrier can then never complete)
    const unsigned ntiles = 2u + (old_cf ? 1u : 0u) + (vel ? 1u : 0u);
    dg_mbar_expect_tx(bar, (unsigned)(sizeof(double2) * tile) * ntiles + extra_tx);
    for (int q = 0; q < nbox; q++) {
      const long d = (long)q * by * MT;
      dg_tma_load_2d(CUt + d, &cc.map_cu[f], (int)(2 * m0), q * by, bar);
      dg_tma_load_2d(NLt + d, &cc.map_nl[f], (int)(2 * m0), q * by, bar);
      if (old_cf) dg_tma_load_2d(CFt + d, &cc.map_cf[f], (int)(2 * m0), q * by, bar);
      if (vel) dg_tma_load_2d(CPt + d, &cc.map_cp, (int)(2 * m0), q * by, bar);
    }
  }
  const bool landed = dg_mbar_wait(bar, 0, spin);
  __syncthreads();
  if (!landed) {
    if (tid == 0) atomicExch(cc.err + 1, 1);
    dg_mbar_wait(bar, 0, spin);  // give the copies in flight one more bounded wait
    return;
  }

  // ---- 1. explicit terms, CF and the CN right-hand side (in place of NL)
  const double h = cc.dscal[1 + rk_step];
  const double time = cc.dscal[0];
  const double zeta = (rk_step == 2) ? -17.0 / 8.0 : (rk_step == 3) ? -5.0 / 4.0 : 0.0;
  const double bbar = (rk_step == 2) ? 25.0 / 8.0 : (rk_step == 3) ? 9.0 / 4.0 : 1.0;
  const double T1 = C.nu * h / 2.0, T3 = zeta * h, T4 = h, T5 = bbar * h;
  const double aaU = T1 * C.nuv;
  const double NU = C.nu;
  const double *__restrict__ rowc = cc.rowc;
  double2 *__restrict__ cff = cc.cf[f];
  int lo, hi;
  if (f == 0 || f == 2) { lo = C.JS; hi = C.JE; }
  else if (f == 1) { lo = 2; hi = NY; }
  else { lo = pick(C.JSt, f - 3); hi = pick(C.JEt, f - 3); }
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
    const double2 u = CUt[i], um = CUt[i - MT], up = CUt[i + MT];
    const double2 nlv = NLt[i];
    const double2 old = old_cf ? CFt[i] : make_double2(0.0, 0.0);
    const double kk = KKS[m];
    double2 fv, r;
    if (f == 0 || f == 2) {
      fv = make_double2(-NU * kk * u.x, -NU * kk * u.y);
      if (C.i_ro != 0.0) {
        const double2 uo = cc.cu[2 - f][o];
        fv.x += sgn * C.i_ro * uo.x;
        fv.y += sgn * C.i_ro * uo.y;
      }
      for (int q = 0; q < nth; q++) {
        const double w = C.ri[q] * gr;
        if (w == 0.0) continue;
        const double2 t = cc.cu[3 + q][o];
        fv.x += w * t.x;
        fv.y += w * t.y;
      }
      fv.x += nlv.x;
      fv.y += nlv.y;
      r = u;
      r.x += T3 * old.x;
      r.y += T3 * old.y;
      const double2 p0 = CPt[i];
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
          const double2 t = cc.cu[3 + q][o], tm = cc.cu[3 + q][o - ss];
          fv.x += w * (t.x * dyfm + tm.x * dyfj);
          fv.y += w * (t.y * dyfm + tm.y * dyfj);
        }
      }
      fv.x += nlv.x;
      fv.y += nlv.y;
      r = u;
      r.x += T3 * old.x;
      r.y += T3 * old.y;
      const double2 p0 = CPt[i], pm = CPt[i - MT];
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
        const double2 u1 = cc.cu[0][o], u3 = cc.cu[2][o];
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
    NLt[i] = r;
  }
  __syncthreads();

  // ---- 2. CN solve, one lane per mode, rows 0..NY+1.  The operator is real,
  // so the real and imaginary parts are two independent recurrences; one
  // lane runs both, interleaved, which hides half of each one's latency.
  const int wlo = (f >= 3) ? pick(C.JSt, f - 3) - 1 : 1;
  if (tid < MT) {
    const int m = tid;
    const double *Aa = TB, *Rb = TB + L, *Cc = TB + 2 * L, *K = TB + 3 * L, *V = TB + 4 * L;
    double2 *x = NLt + m;
    constexpr int B = 8;  // rows per register block: loads first, then the recurrences
    const bool mean = (m0 + m == 0);
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

  // ---- 3. the post-CN field goes to the field's rhs array (rows >= wlo)
  double2 *__restrict__ dst = cc.out[f];
  for (int i = wlo * MT + tid; i < L * MT; i += CS_THR) {
    const int j = i / MT, m = i - j * MT;
    if (m < mt) dst[(long)j * ss + m0 + m] = NLt[i];
  }
}

// dynamic shared memory of one CTA
size_t col_smem_l(int L, int mt, int by, int nbox) {
  return sizeof(double2) * 4 * (size_t)nbox * by * mt + sizeof(double) * (5 * (size_t)L + 3 * mt) +
         8 + 128;
}

// The column kernel: CTA b takes work[b] = (case, mode tile, field) from
// the case table (every case at substep rk_step with MT modes per CTA).
template <int MT>
__global__ void __launch_bounds__(CS_THR) k_col_cn(const ColCase *__restrict__ cases,
                                                  const int4 *__restrict__ work, int rk_step,
                                                  long spin, unsigned extra_tx) {
  extern __shared__ __align__(128) unsigned char cs_raw[];
  unsigned char *sbase = cs_raw + ((128u - (dg_smem_addr(cs_raw) & 127u)) & 127u);
  const int4 w = work[blockIdx.x];
  col_body<MT>(cases[w.x], rk_step, (long)w.y * MT, w.z, spin, extra_tx, sbase);
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

// Per-row grid factors of the column kernels (once per handle, host side).
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

size_t dg_col_smem(const dg_handle *h, int mt) {
  int by, nbox;
  col_geometry(h, &by, &nbox);
  return col_smem_l(h->NY + 2, mt, by, nbox);
}

// The case description of handle h for `mt` modes per CTA (builds the
// tensor maps of its CU, rhs and CF arrays and CP for that tile width).
static int fill_case(dg_handle *h, int mt, ColCase *cc) {
  const int L = h->NY + 2;
  int by = 0, nbox = 0;
  col_geometry(h, &by, &nbox);
  memset(cc, 0, sizeof(*cc));
  for (int f = 0; f < h->nf; f++) {
    DG_TRY(dg_tmap_planes(h->cu[f], h->ss, L, mt, by, &cc->map_cu[f]));
    DG_TRY(dg_tmap_planes(h->rhs[f], h->ss, L, mt, by, &cc->map_nl[f]));
    DG_TRY(dg_tmap_planes(h->cf[f], h->ss, L, mt, by, &cc->map_cf[f]));
  }
  DG_TRY(dg_tmap_planes(h->cp, h->ss, L, mt, by, &cc->map_cp));
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
  return DG_OK;
}

// modes per CTA for handle h: the tuned value, halved until the tiles fit
static int col_mt(const dg_handle *h, int want) {
  int mt = want;
  while (mt > 2 && dg_col_smem(h, mt) > 220 * 1024) mt /= 2;
  return mt;
}

// the work list of one case: (case c, tile, field, 0) per CTA
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

static int launch_col(cudaStream_t st, int pdl, int mt, size_t smem, const void *dev_cases,
                      const int4 *dev_work, int nwork, int rk_step, long spin,
                      unsigned extra_tx) {
#define CS_CASE(MTV)                                                                            \
  if (mt == MTV) {                                                                              \
    dg_big_smem((const void *)k_col_cn<MTV>);                                                   \
    DG_CUDA(dg_launch(pdl, k_col_cn<MTV>, dim3(nwork), dim3(CS_THR), smem, st,                  \
                      (const ColCase *)dev_cases, dev_work, rk_step, spin, extra_tx));          \
  }
  CS_CASE(2) CS_CASE(4) CS_CASE(8) CS_CASE(16)
#undef CS_CASE
  DG_LAUNCHED();
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
  const size_t sm = dg_col_smem(h, mt);
  if (sm > 220 * 1024) {
    dg_set_error("column kernel: the y-columns of two modes do not fit in shared memory");
    return DG_ERR_DIMS;
  }
  DG_TRY(col_tables(h, mt));
  // the wait test (DG_TUNE_WAIT_TEST) applies to this one launch
  const long spin = h->wait_test > 0 ? (long)h->wait_test : DG_ASYNC_SPIN;
  const unsigned extra_tx = h->wait_test > 0 ? 16u : 0u;
  h->wait_test = 0;
  dg_kt_begin(h, "k_col_cn", h->st);
  DG_TRY(launch_col(h->st, h->pdl, mt, sm, h->col_dcase, h->col_dwork, h->col_dnwork, rk_step,
                    spin, extra_tx));
  if (rd) DG_TRY(dg_rem_div_dev(h, 1, rk_step, true));
  return DG_OK;
}

// ---------------------------------------------------------- ragged launch
// The column stage of several cases at the same substep in one launch (the
// ensemble server's groups).  dg_col_batch_build fills, for the handles, the
// host images of the case table and the work list (one (case, tile, field)
// entry per CTA) with one MT for all, and returns the launch's shared
// memory; the caller copies them to device memory it owns and launches with
// dg_col_batch_launch.  Each case's REM_DIV follows on its own stream.
// Results do not depend on the batch: each mode's arithmetic is the
// single-case launch's, with the same kernel.
int dg_col_batch_build(dg_handle *const *hs, int n, int want_mt, std::vector<unsigned char> &cases,
                       std::vector<int4> &work, int *mt_out, size_t *smem_out) {
  int mt = want_mt;
  for (int c = 0; c < n; c++) mt = std::min(mt, col_mt(hs[c], want_mt));
  size_t sm = 0;
  for (int c = 0; c < n; c++) sm = std::max(sm, dg_col_smem(hs[c], mt));
  if (sm > 220 * 1024) {
    dg_set_error("column kernel: the y-columns of two modes do not fit in shared memory");
    return DG_ERR_DIMS;
  }
  cases.assign(sizeof(ColCase) * n, 0);
  work.clear();
  for (int c = 0; c < n; c++) {
    ColCase cc;
    DG_TRY(fill_case(hs[c], mt, &cc));
    memcpy(cases.data() + sizeof(ColCase) * c, &cc, sizeof(ColCase));
    case_work(hs[c], c, mt, work);
  }
  *mt_out = mt;
  *smem_out = sm;
  return DG_OK;
}

int dg_col_batch_launch(cudaStream_t st, int mt, size_t smem, const void *dev_cases,
                        const int4 *dev_work, int nwork, int rk_step) {
  return launch_col(st, 0, mt, smem, dev_cases, dev_work, nwork, rk_step, DG_ASYNC_SPIN, 0u);
}
