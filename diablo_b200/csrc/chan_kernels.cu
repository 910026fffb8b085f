// Channel substep kernels (RK_CHAN_1, for/channel.f:62-1073) on the
// retained-mode layout [j][kz][kx].
//
// One substep is five launches (plus COURANT's on the side stream when it
// runs):
//   zinv        spectral U1..U3, TH -> half-physical H (z inverse per kx)
//   k_xrow_w    per physical z-row, marching up in y: x c2r of every field,
//               all products/fluxes of for/channel.f:409-571,665-720, x r2c,
//               and the combination into 2 arrays per field
//               (A: to be multiplied by -i kz, B: the rest).  Row lengths
//               without a warp kernel take two launches instead: k_xc2r of
//               every plane into physical space, then k_xprod (products, x
//               r2c and the combination, one product pair per CTA).
//   k_zfwd_w    per plane: z forward of A/B -> the nonlinear term
//               NL = -i kz A + B of every retained mode (with LES, whose
//               solves need them, the epilogue also forms the explicit terms,
//               CF and the Crank-Nicolson right-hand side
//               R = CU + zeta h CF_old - h grad P + beta h CF_new
//                   + (nu h / 2) d2/dy2 CU,          for/channel.f:88-626)
//   k_col_cn    per (mode tile, field) (chan_column.cu): explicit terms, CF,
//               the CN right-hand side and solve.  The reference solves the
//               same x-z independent CN operator per physical column
//               (for/channel.f:767-1029); it is linear and identical for
//               every column, so it commutes with the x-z transform.
//   k_rd_col    per mode tile: REM_DIV_CHAN and CP += phi / h on the post-CN
//               velocity (for/channel.f:1037-1065, 1103-1214); with COURANT,
//               COURANT's transform and reduction run beside it.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <utility>
#include "dg_internal.cuh"
#include "fft.cuh"

using namespace dgfft;

namespace {

struct ChanConst {
  int NX, NY, NZ, NKX, NKZ, nkxp, nkzt, nf, nth;
  long ss;
  int JS, JE, JSt[DG_MAX_TH], JEt[DG_MAX_TH];
  double nu, beta, nuv, i_ro, grav_x, grav_y, grav_z, px0, omega0, amp_omega0;
  int f_type;
  double ri[DG_MAX_TH], pr[DG_MAX_TH], drhodx[DG_MAX_TH], drhodz[DG_MAX_TH];
};

// uniform selects from the parameter arrays (a run-time index into a kernel
// parameter array would copy the array to local memory)
template <typename T>
__device__ __forceinline__ T sel(const T (&a)[DG_MAX_TH], int i) {
  T r = a[0];
#pragma unroll
  for (int k = 1; k < DG_MAX_TH; k++) r = (i == k) ? a[k] : r;
  return r;
}

ChanConst make_const(const dg_handle *h) {
  ChanConst c;
  c.NX = h->NX; c.NY = h->NY; c.NZ = h->NZ; c.NKX = h->NKX; c.NKZ = h->NKZ;
  c.nkxp = h->nkxp; c.nkzt = h->nkzt; c.nf = h->nf; c.nth = h->NTH; c.ss = h->ss;
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

// ------------------------------------------------------------------ xrow
// Products per plane j (p = j+1, m = j-1), indices into the product list:
//  0 U1U3(j)  1 U1U1(j)  2 U3U3(j)  3 g(j) = (U2(j)+U2(j+1))^2/4
//  4 fl1(j+1) = (U1(j+1)+U1(j)) U2(j+1)   5 fl3(j+1)
//  6 Ubar1 U2(j)   7 Ubar3 U2(j)   (Ubar = (DYF(j) U(j) + DYF(j-1) U(j-1)) / (2 DY(j)))
//  8+3n TH U1(j)   9+3n TH U3(j)   10+3n flth(j+1) = (TH(j+1)+TH(j)) U2(j+1)
// Generic x-row stage (any NX, any N_TH).  The half-physical planes 0..NY+1
// are first taken to physical space by the x c2r kernel (into the work array,
// layout [field][plane][z][x]).  k_xprod then forms the products of output
// plane j for a batch of z-rows and x-transforms them in complex pairs.  The
// flux differences are taken in physical space (the x transform is linear),
// so each pair maps straight onto the A/B arrays of G:
//   pair 0          U1U3(j)       | fl3(j+1) - fl3(j)      -> G0, G5
//   pair 1          U1U1(j)       | fl1(j+1) - fl1(j)      -> G1
//   pair 2          Ubar1 U2(j)   | g(j) - g(j-1)          -> G3
//   pair 3          Ubar3 U2(j)   | U3U3(j)                -> G2, G4
//   pair 4+n        TH_n U1(j)    | flth_n(j+1) - flth_n(j) -> G(7+2n)
//   pair 4+N_TH+m   TH_2m U3(j)   | TH_2m+1 U3(j)          -> G(6+4m), G(8+4m)
// One CTA transforms one pair for `rz` z-rows of one plane (one z-row per
// warp for the compile-time lengths).  The pairs of a plane are adjacent in
// launch order, so the physical rows they share come from HBM once and from
// L2 after that.
constexpr int XP_THR = 128;

__host__ __device__ constexpr int xp_rows_max(int nx) {
  return nx <= 128 ? 16 : (nx <= 256 ? 8 : 4);
}
int xp_pairs(int nth) { return 4 + nth + (nth + 1) / 2; }
size_t xp_smem(int nx, int rz) {
  return sizeof(double2) * (nx + fft_bufs(nx) * (size_t)rz * padded_len(nx));
}
// z-rows per CTA: one per warp for the compile-time lengths; otherwise the
// batch for this length, halved until the shared memory fits
int xp_rows(int nx) {
  if (fft_bufs(nx) == 1) return XP_THR / 32;
  int rz = xp_rows_max(nx);
  while (rz > 1 && xp_smem(nx, rz) > 220 * 1024) rz >>= 1;
  return rz;
}

template <int NT>
__global__ void __launch_bounds__(XP_THR, 5) k_xprod(
    ChanConst C, const double *__restrict__ phys, long pfield, int rz, FftPlan pl,
    const double2 *__restrict__ tw, const double *__restrict__ dyf, const double *__restrict__ dy,
    const double *__restrict__ kxv, double2 *__restrict__ G, long Gfield) {
  extern __shared__ double2 sm[];
  const int NX = NT ? NT : C.NX;
  const int NZ = C.NZ, nkxp = C.nkxp, nth = C.nth;
  const int sstr = padded_len(NX);
  double2 *stw = sm;
  double2 *b0 = stw + NX;
  const int s = blockIdx.x;
  const int z0 = blockIdx.y * rz;
  const int j = 1 + blockIdx.z;
  const int tid = threadIdx.x;
  const long pplane = (long)NZ * NX;
  for (int i = tid; i < NX; i += XP_THR) stw[i] = tw[i];
  const double dyfj = dyf[j], dyfm = dyf[j - 1];
  const double wgy = 1.0 / (2.0 * dy[j]);
  const double *base = phys + (long)j * pplane + (long)z0 * NX;

  // the pair at element e = r NX + x of the CTA's rows
  auto pair_at = [&](int e) -> double2 {
    const double *pc = base + e;  // field 0, plane j
    auto U = [&](int f, int dj) { return __ldg(pc + f * pfield + dj * pplane); };
    double a, b = 0.0;
    if (s == 0) {
      const double u1 = U(0, 0), u2 = U(1, 0), u2p = U(1, 1);
      const double u3 = U(2, 0), u3p = U(2, 1), u3m = U(2, -1);
      a = u3 * u1;
      b = (u3p + u3) * u2p - (u3 + u3m) * u2;
    } else if (s == 1) {
      const double u1 = U(0, 0), u1p = U(0, 1), u1m = U(0, -1), u2 = U(1, 0), u2p = U(1, 1);
      a = u1 * u1;
      b = (u1p + u1) * u2p - (u1 + u1m) * u2;
    } else if (s == 2) {
      const double u1 = U(0, 0), u1m = U(0, -1);
      const double u2 = U(1, 0), u2p = U(1, 1), u2m = U(1, -1);
      a = ((dyfj * u1 + dyfm * u1m) * wgy) * u2;
      const double gp = u2 + u2p, gm = u2m + u2;
      b = 0.25 * (gp * gp) - 0.25 * (gm * gm);
    } else if (s == 3) {
      const double u3 = U(2, 0), u3m = U(2, -1), u2 = U(1, 0);
      a = ((dyfj * u3 + dyfm * u3m) * wgy) * u2;
      b = u3 * u3;
    } else if (s < 4 + nth) {
      const int f = 3 + (s - 4);
      const double t = U(f, 0), tp = U(f, 1), tm = U(f, -1);
      const double u1 = U(0, 0), u2 = U(1, 0), u2p = U(1, 1);
      a = t * u1;
      b = (tp + t) * u2p - (t + tm) * u2;
    } else {
      const int n = 2 * (s - 4 - nth);
      const double u3 = U(2, 0);
      a = U(3 + n, 0) * u3;
      if (n + 1 < nth) b = U(4 + n, 0) * u3;
    }
    return make_double2(a, b);
  };

  const bool pow2 = (NX & (NX - 1)) == 0;
  const double rnx = 1.0 / (double)NX;  // exact for a power of two
  const double id2 = 1.0 / (2.0 * dyfj), idyj = 1.0 / dy[j];
  const long jo = (long)j * NZ * nkxp;
  // mode k of row z from its transformed signal
  auto finish = [&](const double2 *sig, int z, int k) {
    const double2 zk = sig[pad(k)];
    const double2 zm = sig[pad((NX - k) % NX)];
    // the real and imaginary members of the pair: A = (Z_k + conj Z_{N-k})/2,
    // B = -i/2 (Z_k - conj Z_{N-k}), scaled by 1/NX
    double2 A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
    double2 B = make_double2(0.5 * (zk.y + zm.y), -0.5 * (zk.x - zm.x));
    if (pow2) {
      A = make_double2(A.x * rnx, A.y * rnx);
      B = make_double2(B.x * rnx, B.y * rnx);
    } else {
      A = make_double2(A.x / NX, A.y / NX);
      B = make_double2(B.x / NX, B.y / NX);
    }
    const double KX = kxv[k];
    // -i kx A - c B
    auto flux = [&](double c) { return make_double2(KX * A.y - B.x * c, -KX * A.x - B.y * c); };
    double2 *o = G + jo + (long)z * nkxp + k;
    if (s == 0) {
      o[0] = A;                       // U1: A = U1U3
      o[5 * Gfield] = flux(id2);      // U3: B = -ikx U1U3 - (fl3(j+1) - fl3(j)) / (2 DYF)
    } else if (s == 1) {
      o[Gfield] = flux(id2);          // U1: B = -ikx U1U1 - (fl1(j+1) - fl1(j)) / (2 DYF)
    } else if (s == 2) {
      o[3 * Gfield] = flux(idyj);     // U2: B = -ikx Ubar1 U2 - (g(j) - g(j-1)) / DY
    } else if (s == 3) {
      o[2 * Gfield] = A;              // U2: A = Ubar3 U2
      o[4 * Gfield] = B;              // U3: A = U3U3
    } else if (s < 4 + nth) {
      o[(7 + 2 * (s - 4)) * Gfield] = flux(id2);  // TH: B = -ikx TH U1 - dflth / (2 DYF)
    } else {
      const int n = 2 * (s - 4 - nth);
      o[(6 + 2 * n) * Gfield] = A;                // TH: A = TH U3
      if (n + 1 < nth) o[(8 + 2 * n) * Gfield] = B;
    }
  };

  if constexpr (NT != 0) {
    // one warp per z-row (rz = 4): past the twiddle staging, no CTA barrier
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31;
    const int z = z0 + warp;
    if (z >= NZ) return;
    double2 *sig = b0 + warp * sstr;
#pragma unroll 4
    for (int x = lane; x < NX; x += 32) sig[pad(x)] = pair_at(warp * NX + x);
    __syncwarp();
    wpasses_any<NT, -1, 0>(sig, 1, sstr, stw, lane);
    for (int k = lane; k < nkxp; k += 32) finish(sig, z, k);
  } else {
    double2 *b1 = b0 + rz * sstr;
    for (int idx = tid; idx < rz * NX; idx += XP_THR) {
      const int r = idx / NX, x = idx - r * NX;
      b0[r * sstr + pad(x)] = (z0 + r < NZ) ? pair_at(idx) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    double2 *res = fft<0>(b0, b1, pl, rz, sstr, stw, -1);
    for (int idx = tid; idx < rz * nkxp; idx += XP_THR) {
      const int r = idx / nkxp, k = idx - r * nkxp;
      if (z0 + r < NZ) finish(res + r * sstr, z0 + r, k);
    }
  }
}

// ------------------------------------------------- generic x-row stage, FP32
// The mixed form of the two launches above, for the compile-time row lengths
// without a warp x-row kernel (and for N_TH > 2).  As in k_xrow_w's FP32
// form, every x-row is split into its mean (FP64) and its fluctuation
// (FP32): k_xc2r_f takes the FP32 half-physical planes to physical
// fluctuation rows (the kx = 0 bin removed) and keeps each row's mean;
// k_xprod_f forms every product L1 L2 as D1 L2' + D2 L1' + L1' L2' in FP32
// (D the means, L' the fluctuations), transforms the pairs in FP32 and puts
// the FP64 row mean of the product, D1 D2 + <L1' L2'>, in the kx = 0 bin.

// c2r of two z-rows of one field per warp (4 warps, 8 rows per CTA)
template <int NT>
__global__ void __launch_bounds__(128) k_xc2r_f(const float2 *__restrict__ H, long Hfield,
                                               int NZ, int nkxp, const float2 *__restrict__ tw,
                                               float *__restrict__ out, long ofield,
                                               double *__restrict__ dc, long dfield) {
  extern __shared__ double2 sm_raw[];
  constexpr int NX = NT, SSTR = padded_len(NT);
  float2 *stw = reinterpret_cast<float2 *>(sm_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2 *sig = stw + NX + warp * SSTR;
  const int j = blockIdx.y, f = blockIdx.z;
  const int za = blockIdx.x * 8 + 2 * warp, zb = za + 1;
  for (int i = threadIdx.x; i < NX; i += 128) stw[i] = tw[i];
  dg_pdl_wait();  // H comes from the z inverse
  __syncthreads();
  if (za >= NZ) return;
  const float2 *ra = H + f * Hfield + ((long)j * NZ + za) * nkxp;
  const bool hb = zb < NZ;
  if (lane == 0) {
    dc[f * dfield + (long)j * NZ + za] = (double)ra[0].x;
    if (hb) dc[f * dfield + (long)j * NZ + zb] = (double)ra[nkxp].x;
  }
  for (int k = lane; k < NX; k += 32) {
    const int kk = (k <= NX / 2) ? k : NX - k;
    float2 v = make_float2(0.f, 0.f);
    if (kk > 0 && kk < nkxp && kk < NX / 2) {
      const float2 a = ra[kk];
      const float2 b = hb ? ra[nkxp + kk] : make_float2(0.f, 0.f);
      v = (k == kk) ? make_float2(a.x - b.y, a.y + b.x) : make_float2(a.x + b.y, -a.y + b.x);
    }
    sig[pad(k)] = v;
  }
  __syncwarp();
  wpasses_any<NT, +1, 0>(sig, 1, SSTR, stw, lane);
  float *oa = out + f * ofield + ((long)j * NZ + za) * NX;
  for (int x = lane; x < NX; x += 32) {
    const float2 v = sig[pad(x)];
    oa[x] = v.x;
    if (hb) oa[NX + x] = v.y;
  }
}

// c0 F(f0, j+d0) + c1 F(f1, j+d1) (f1 < 0: one term)
struct XLin {
  int f0, d0, f1, d1;
  double c0, c1;
};
struct XTerm {
  double sg;
  XLin l1, l2;
};

__device__ __forceinline__ XLin xl(int f, int d, double c = 1.0) { return {f, d, -1, 0, c, 0.0}; }
__device__ __forceinline__ XLin xl2(int f0, int d0, double c0, int f1, int d1, double c1) {
  return {f0, d0, f1, d1, c0, c1};
}

// the products of pair s (as listed before k_xprod), each a sum of +-L1 L2
__device__ __forceinline__ void xpair_terms(int s, int nth, double dyfj, double dyfm, double wgy,
                                            XTerm (&ta)[2], int &na, XTerm (&tb)[2], int &nb) {
  na = 1;
  nb = 2;
  if (s == 0) {
    ta[0] = {1.0, xl(2, 0), xl(0, 0)};
    tb[0] = {1.0, xl2(2, 1, 1.0, 2, 0, 1.0), xl(1, 1)};
    tb[1] = {-1.0, xl2(2, 0, 1.0, 2, -1, 1.0), xl(1, 0)};
  } else if (s == 1) {
    ta[0] = {1.0, xl(0, 0), xl(0, 0)};
    tb[0] = {1.0, xl2(0, 1, 1.0, 0, 0, 1.0), xl(1, 1)};
    tb[1] = {-1.0, xl2(0, 0, 1.0, 0, -1, 1.0), xl(1, 0)};
  } else if (s == 2) {
    ta[0] = {1.0, xl2(0, 0, dyfj * wgy, 0, -1, dyfm * wgy), xl(1, 0)};
    tb[0] = {1.0, xl2(1, 0, 0.5, 1, 1, 0.5), xl2(1, 0, 0.5, 1, 1, 0.5)};
    tb[1] = {-1.0, xl2(1, -1, 0.5, 1, 0, 0.5), xl2(1, -1, 0.5, 1, 0, 0.5)};
  } else if (s == 3) {
    ta[0] = {1.0, xl2(2, 0, dyfj * wgy, 2, -1, dyfm * wgy), xl(1, 0)};
    tb[0] = {1.0, xl(2, 0), xl(2, 0)};
    nb = 1;
  } else if (s < 4 + nth) {
    const int t = 3 + (s - 4);
    ta[0] = {1.0, xl(t, 0), xl(0, 0)};
    tb[0] = {1.0, xl2(t, 1, 1.0, t, 0, 1.0), xl(1, 1)};
    tb[1] = {-1.0, xl2(t, 0, 1.0, t, -1, 1.0), xl(1, 0)};
  } else {
    const int n = 2 * (s - 4 - nth);
    ta[0] = {1.0, xl(3 + n, 0), xl(2, 0)};
    tb[0] = {1.0, xl(4 + n, 0), xl(2, 0)};
    nb = (n + 1 < nth) ? 1 : 0;
  }
}

template <int NT>
__global__ void __launch_bounds__(XP_THR) k_xprod_f(
    ChanConst C, const float *__restrict__ ph, long pfield, const double *__restrict__ dc,
    long dfield, const float2 *__restrict__ tw, const double *__restrict__ dyf,
    const double *__restrict__ dy, const double *__restrict__ kxv, float2 *__restrict__ G,
    long Gfield) {
  extern __shared__ double2 sm_raw[];
  constexpr int NX = NT, SSTR = padded_len(NT);
  float2 *stw = reinterpret_cast<float2 *>(sm_raw);
  const int NZ = C.NZ, nkxp = C.nkxp, nth = C.nth;
  const int s = blockIdx.x, j = 1 + blockIdx.z;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int z = blockIdx.y * (XP_THR / 32) + warp;
  for (int i = threadIdx.x; i < NX; i += XP_THR) stw[i] = tw[i];
  dg_pdl_wait();  // the physical rows come from k_xc2r_f
  __syncthreads();
  if (z >= NZ) return;
  const long pplane = (long)NZ * NX;
  const double dyfj = dyf[j], dyfm = dyf[j - 1];
  const double wgy = 1.0 / (2.0 * dy[j]);
  XTerm ta[2], tb[2];
  int na, nb;
  xpair_terms(s, nth, dyfj, dyfm, wgy, ta, na, tb, nb);
  const float *row0 = ph + (long)j * pplane + (long)z * NX;
  auto Dm = [&](int f, int d) { return __ldg(dc + f * dfield + (long)(j + d) * NZ + z); };
  auto lin_d = [&](const XLin &l) {
    double v = l.c0 * Dm(l.f0, l.d0);
    if (l.f1 >= 0) v += l.c1 * Dm(l.f1, l.d1);
    return v;
  };
  auto lin_f = [&](const XLin &l, int x) {
    float v = (float)l.c0 * __ldg(row0 + l.f0 * pfield + l.d0 * pplane + x);
    if (l.f1 >= 0) v += (float)l.c1 * __ldg(row0 + l.f1 * pfield + l.d1 * pplane + x);
    return v;
  };
  // means of L1, L2 per term and the mean-mean part of the product means
  double Da[2][2], Db[2][2], dda = 0.0, ddb = 0.0;
#pragma unroll
  for (int t = 0; t < 2; t++) {
    if (t < na) {
      Da[t][0] = lin_d(ta[t].l1);
      Da[t][1] = lin_d(ta[t].l2);
      dda += ta[t].sg * Da[t][0] * Da[t][1];
    }
    if (t < nb) {
      Db[t][0] = lin_d(tb[t].l1);
      Db[t][1] = lin_d(tb[t].l2);
      ddb += tb[t].sg * Db[t][0] * Db[t][1];
    }
  }
  float2 *sig = stw + NX + warp * SSTR;
  double sa = 0.0, sb = 0.0;
  for (int x = lane; x < NX; x += 32) {
    float a = 0.f, b = 0.f;
#pragma unroll
    for (int t = 0; t < 2; t++) {
      // row means: exact products of the FP32 fluctuations, summed in FP64
      if (t < na) {
        const float l1 = lin_f(ta[t].l1, x), l2 = lin_f(ta[t].l2, x), ff = l1 * l2;
        a += (float)ta[t].sg * ((float)Da[t][0] * l2 + (float)Da[t][1] * l1 + ff);
        sa = fma(ta[t].sg * (double)l1, (double)l2, sa);
      }
      if (t < nb) {
        const float l1 = lin_f(tb[t].l1, x), l2 = lin_f(tb[t].l2, x), ff = l1 * l2;
        b += (float)tb[t].sg * ((float)Db[t][0] * l2 + (float)Db[t][1] * l1 + ff);
        sb = fma(tb[t].sg * (double)l1, (double)l2, sb);
      }
    }
    sig[pad(x)] = make_float2(a, b);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sa += __shfl_xor_sync(0xffffffffu, sa, o);
    sb += __shfl_xor_sync(0xffffffffu, sb, o);
  }
  const double dca = dda + sa / (double)NX, dcb = ddb + sb / (double)NX;
  __syncwarp();
  wpasses_any<NT, -1, 0>(sig, 1, SSTR, stw, lane);
  const double id2 = 1.0 / (2.0 * dyfj), idyj = 1.0 / dy[j];
  float2 *obase = G + (long)j * NZ * nkxp + (long)z * nkxp;
  for (int k = lane; k < nkxp; k += 32) {
    double2 A, B;
    if (k == 0) {
      A = make_double2(dca, 0.0);
      B = make_double2(dcb, 0.0);
    } else {
      const float2 zk = sig[pad(k)], zm = sig[pad(NX - k)];
      const double ax = 0.5 * ((double)zk.x + (double)zm.x), ay = 0.5 * ((double)zk.y - (double)zm.y);
      const double bx = 0.5 * ((double)zk.y + (double)zm.y), by = -0.5 * ((double)zk.x - (double)zm.x);
      A = make_double2(ax / NX, ay / NX);
      B = make_double2(bx / NX, by / NX);
    }
    const double KX = kxv[k];
    auto flux = [&](double c) {
      return make_float2((float)(KX * A.y - B.x * c), (float)(-KX * A.x - B.y * c));
    };
    const float2 Af = make_float2((float)A.x, (float)A.y), Bf = make_float2((float)B.x, (float)B.y);
    float2 *o = obase + k;
    if (s == 0) {
      o[0] = Af;
      o[5 * Gfield] = flux(id2);
    } else if (s == 1) {
      o[Gfield] = flux(id2);
    } else if (s == 2) {
      o[3 * Gfield] = flux(idyj);
    } else if (s == 3) {
      o[2 * Gfield] = Af;
      o[4 * Gfield] = Bf;
    } else if (s < 4 + nth) {
      o[(7 + 2 * (s - 4)) * Gfield] = flux(id2);
    } else {
      const int n = 2 * (s - 4 - nth);
      o[(6 + 2 * n) * Gfield] = Af;
      if (n + 1 < nth) o[(8 + 2 * n) * Gfield] = Bf;
    }
  }
}

// ------------------------------------------------------- xrow, one warp/row
// Same products as listed above, organised so a warp owns one physical z-row and
// marches up through its chunk of planes with no CTA-wide barrier: the two
// physical planes it needs (j and j+1) live in registers (lane l holds
// x = l + 32 i), the transforms run in a per-warp shared buffer with
// __syncwarp between passes, and the x-spectra carried from one plane to the
// next (fluxes at GY j, Ubar U2 at GY j, g at GYF j-1) live in registers
// (lane l holds kx = l + 32 s).  At step j it forms the GYF-j products and
// the GY-(j+1) products, so only planes j and j+1 are needed.
constexpr int XW_WARPS = 4;

__host__ __device__ constexpr bool xw_supported(int n) {
  return n == 16 || n == 32 || n == 48 || n == 64 || n == 96 || n == 128 || n == 256;
}

template <int NX, int NTH, typename CX = double2, int PV = 0>
__global__ void __launch_bounds__(32 * XW_WARPS, NTH == 0 ? (sizeof(CX) == 8 ? 4 : 3) : 2) k_xrow_w(
    ChanConst C, const CX *__restrict__ H, long Hfield, int chunk, int jbase, int jtop,
    const CX *__restrict__ tw, const double *__restrict__ dyf, const double *__restrict__ dy,
    const double *__restrict__ kxv, CX *__restrict__ G, long Gfield) {
  constexpr int NF = 3 + NTH;
  constexpr int NPIN = (NF + 1) / 2;
  constexpr int NPROD = 8 + 3 * NTH;
  constexpr int NPP = (NPROD + 1) / 2;
  constexpr int MAXP = NPIN > NPP ? NPIN : NPP;
  constexpr int XPL = (NX + 31) / 32;              // physical points per lane
  constexpr int NKXP = NX / 3 + 1;
  constexpr int KS = (NKXP + 31) / 32;             // kx slots per lane
  constexpr int SSTR = padded_len(NX);
  extern __shared__ double2 sm_raw[];
  using T = typename CT<CX>::T;
  CX *sm = reinterpret_cast<CX *>(sm_raw);
  CX *stw = sm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  CX *buf = stw + NX + warp * MAXP * SSTR;
  // carried x-spectra: 0 fl1, 1 fl3, 2 ubar1 u2, 3 ubar3 u2, 4 g, 5+n flth
  CX *pvs = stw + NX + XW_WARPS * MAXP * SSTR + warp * (5 + NTH) * NKXP;
  stage_tw<NX, PV, tp_ok(NX)>(stw, tw, NX, threadIdx.x, blockDim.x);
  dg_pdl_wait();  // H comes from the z inverse
  __syncthreads();
  const int z = blockIdx.x * XW_WARPS + warp;
  const int NZ = C.NZ;
  if (z >= NZ) return;
  const int j0 = jbase + blockIdx.y * chunk;
  int j1 = j0 + chunk - 1;
  if (j1 > jtop) j1 = jtop;
  const T rnx = (T)1 / (T)NX;            // exact: NX is 2^a 3^b ... see below
  const bool pow2 = (NX & (NX - 1)) == 0;
  const long plane = (long)NZ * NKXP;

  T cur[NF][XPL], nxt[NF][XPL];
#define PV(q, s) pvs[(q) * NKXP + lane + 32 * (s)]

  // FP32 form: each x-row is split into its x-mean (kept in FP64, uniform
  // across the row) and the fluctuation (FP32).  The transforms see only
  // fluctuations, so the two real rows packed into one complex transform
  // have comparable magnitude, and the row means of the products are formed
  // in FP64 from the means and the fluctuations.
  constexpr bool F32 = sizeof(T) == 4;
  double dcur[NF], dnxt[NF];
  auto load_plane = [&](int pl, T (&dst)[NF][XPL], double (&dcv)[NF]) {
    const CX *row = H + (long)pl * plane + (long)z * NKXP;
    if constexpr (F32) {
#pragma unroll
      for (int f = 0; f < NF; f++) dcv[f] = (double)row[f * Hfield].x;
    }
#pragma unroll
    for (int q = 0; q < NPIN; q++) {
      const int fa = 2 * q, fb = 2 * q + 1;
#pragma unroll
      for (int i = 0; i < (NX + 31) / 32; i++) {
        const int k = lane + 32 * i;
        const int kk = (k <= NX / 2) ? k : NX - k;
        // bins above NKX (the truncated band, the x-Nyquist bin among them)
        // are zero: the pruned first pass below does not read them
        if (k < NX && kk < NKXP && kk < NX / 2) {
          CX a = row[fa * Hfield + kk];
          CX bb = (fb < NF) ? row[fb * Hfield + kk] : CT<CX>::mk(0, 0);
          if (kk == 0) { a.y = 0.0; bb.y = 0.0; }
          if (F32 && kk == 0) { a.x = 0.0; bb.x = 0.0; }
          buf[q * SSTR + pad(k)] = (k == kk) ? CT<CX>::mk(a.x - bb.y, a.y + bb.x)
                                             : CT<CX>::mk(a.x + bb.y, -a.y + bb.x);
        }
      }
    }
    __syncwarp();
    static_assert(NKXP - 1 == NX / 3, "the truncated band of the pruned pass is NX/3 + 1 ..");
    wpasses_pz<NX, +1, PV, tp_ok(NX)>(buf, NPIN, SSTR, stw, lane);
#pragma unroll
    for (int q = 0; q < NPIN; q++)
#pragma unroll
      for (int i = 0; i < XPL; i++) {
        const int x = lane + 32 * i;
        const CX v = (x < NX) ? buf[q * SSTR + pad(x)] : CT<CX>::mk(0, 0);
        dst[2 * q][i] = v.x;
        if (2 * q + 1 < NF) dst[2 * q + 1][i] = v.y;
      }
    __syncwarp();
  };

  load_plane(j0 - 1, cur, dcur);
  for (int j = j0 - 1; j <= j1; j++) {
    load_plane(j + 1, nxt, dnxt);
    const T dyf_j = dyf[j], dyf_p = dyf[j + 1], dy_p = dy[j + 1];
    const T wgy = (T)1 / ((T)2 * dy_p);
    // products: GYF j (U1U3, U1U1, U3U3, g, TH U1, TH U3) and GY j+1 (fl1, fl3,
    // ubar1 u2, ubar3 u2, flth)
    // FP32 form: row means of the products, P = L1 L2 with L = D + L'
    double pdc[F32 ? NPROD : 1];
    if constexpr (F32) {
      double acc[NPROD];
#pragma unroll
      for (int p = 0; p < NPROD; p++) acc[p] = 0.0;
      const double wgyd = 1.0 / (2. * (double)dy[j + 1]);
      const double dfj = dyf[j], dfp = dyf[j + 1];
      double L1d[NPROD], L2d[NPROD];
      // (L1, L2) row means of each product, in the order of P[] below
      L1d[0] = dcur[2]; L2d[0] = dcur[0];
      L1d[1] = dcur[0]; L2d[1] = dcur[0];
      L1d[2] = dcur[2]; L2d[2] = dcur[2];
      L1d[3] = 0.5 * (dcur[1] + dnxt[1]); L2d[3] = L1d[3];
      L1d[4] = dnxt[0] + dcur[0]; L2d[4] = dnxt[1];
      L1d[5] = dnxt[2] + dcur[2]; L2d[5] = dnxt[1];
      L1d[6] = (dfp * dnxt[0] + dfj * dcur[0]) * wgyd; L2d[6] = dnxt[1];
      L1d[7] = (dfp * dnxt[2] + dfj * dcur[2]) * wgyd; L2d[7] = dnxt[1];
#pragma unroll
      for (int n = 0; n < NTH; n++) {
        L1d[8 + 3 * n] = dcur[3 + n]; L2d[8 + 3 * n] = dcur[0];
        L1d[9 + 3 * n] = dcur[3 + n]; L2d[9 + 3 * n] = dcur[2];
        L1d[10 + 3 * n] = dnxt[3 + n] + dcur[3 + n]; L2d[10 + 3 * n] = dnxt[1];
      }
#pragma unroll
      for (int i = 0; i < XPL; i++) {
        const int x = lane + 32 * i;
        if (x >= NX) continue;
        const float u1 = cur[0][i], u2 = cur[1][i], u3 = cur[2][i];
        const float u1p = nxt[0][i], u2p = nxt[1][i], u3p = nxt[2][i];
        float L1f[NPROD], L2f[NPROD];
        L1f[0] = u3; L2f[0] = u1;
        L1f[1] = u1; L2f[1] = u1;
        L1f[2] = u3; L2f[2] = u3;
        L1f[3] = 0.5f * (u2 + u2p); L2f[3] = L1f[3];
        L1f[4] = u1p + u1; L2f[4] = u2p;
        L1f[5] = u3p + u3; L2f[5] = u2p;
        L1f[6] = ((T)dyf_p * u1p + (T)dyf_j * u1) * wgy; L2f[6] = u2p;
        L1f[7] = ((T)dyf_p * u3p + (T)dyf_j * u3) * wgy; L2f[7] = u2p;
#pragma unroll
        for (int n = 0; n < NTH; n++) {
          const float t = cur[3 + n][i], tp = nxt[3 + n][i];
          L1f[8 + 3 * n] = t; L2f[8 + 3 * n] = u1;
          L1f[9 + 3 * n] = t; L2f[9 + 3 * n] = u3;
          L1f[10 + 3 * n] = tp + t; L2f[10 + 3 * n] = u2p;
        }
        T P[2 * NPP];
#pragma unroll
        for (int p = 0; p < NPROD; p++) {
          const float ff = L1f[p] * L2f[p];
          // the row mean takes the exact product of the FP32 fluctuations (48
          // significant bits fit FP64) and sums it in FP64: no FP32 rounding
          // enters the mean, whatever the row length
          acc[p] = fma((double)L1f[p], (double)L2f[p], acc[p]);
          P[p] = (float)L1d[p] * L2f[p] + (float)L2d[p] * L1f[p] + ff;
        }
        if (2 * NPP > NPROD) P[2 * NPP - 1] = 0.0f;
#pragma unroll
        for (int q = 0; q < NPP; q++) buf[q * SSTR + pad(x)] = CT<CX>::mk(P[2 * q], P[2 * q + 1]);
      }
#pragma unroll
      for (int p = 0; p < NPROD; p++) {
        double v = acc[p];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        pdc[p] = L1d[p] * L2d[p] + v / (double)NX;
      }
    } else {
#pragma unroll
    for (int i = 0; i < XPL; i++) {
      const int x = lane + 32 * i;
      if (x >= NX) continue;
      const T u1 = cur[0][i], u2 = cur[1][i], u3 = cur[2][i];
      const T u1p = nxt[0][i], u2p = nxt[1][i], u3p = nxt[2][i];
      T P[2 * NPP];
      P[0] = u3 * u1;
      P[1] = u1 * u1;
      P[2] = u3 * u3;
      { const T s = u2 + u2p; P[3] = (T)0.25 * (s * s); }
      P[4] = (u1p + u1) * u2p;
      P[5] = (u3p + u3) * u2p;
      P[6] = ((dyf_p * u1p + dyf_j * u1) * wgy) * u2p;
      P[7] = ((dyf_p * u3p + dyf_j * u3) * wgy) * u2p;
#pragma unroll
      for (int n = 0; n < NTH; n++) {
        const T t = cur[3 + n][i], tp = nxt[3 + n][i];
        P[8 + 3 * n] = t * u1;
        P[9 + 3 * n] = t * u3;
        P[10 + 3 * n] = (tp + t) * u2p;
      }
      if (2 * NPP > NPROD) P[2 * NPP - 1] = 0.0;
#pragma unroll
      for (int q = 0; q < NPP; q++) buf[q * SSTR + pad(x)] = CT<CX>::mk(P[2 * q], P[2 * q + 1]);
    }
    }
    __syncwarp();
    wpasses<NX, -1, 0, PV, tp_ok(NX)>(buf, NPP, SSTR, stw, lane);
    const bool out = (j >= j0);
    const T d2 = (T)2 * dyf_j, dyj = dy[j];
    const T id2 = (T)1 / d2, idyj = (T)1 / dyj;  // per plane: multiply in the row loop
#pragma unroll
    for (int s = 0; s < KS; s++) {
      const int k = lane + 32 * s;
      if (k >= NKXP) continue;
      auto X = [&](int p) -> CX {
        if constexpr (F32) {
          if (k == 0) return CT<CX>::mk((T)pdc[p], (T)0);
        }
        const int q = p >> 1;
        const CX zk = buf[q * SSTR + pad(k)];
        const CX zm = buf[q * SSTR + pad((NX - k) % NX)];
        CX v;
        if ((p & 1) == 0) v = CT<CX>::mk((T)0.5 * (zk.x + zm.x), (T)0.5 * (zk.y - zm.y));
        else v = CT<CX>::mk((T)0.5 * (zk.y + zm.y), -(T)0.5 * (zk.x - zm.x));
        if (pow2) return CT<CX>::mk(v.x * rnx, v.y * rnx);
        return CT<CX>::mk(v.x / (T)NX, v.y / (T)NX);
      };
      const T KX = kxv[k];
      auto mikx = [&](CX a) { return CT<CX>::mk(KX * a.y, -KX * a.x); };  // -i kx a
      const CX x3 = X(3), x4 = X(4), x5 = X(5), x6 = X(6), x7 = X(7);
      if (out) {
        const long off = (long)j * NZ * NKXP + (long)z * NKXP + k;
        const CX x0 = X(0), x1 = X(1), x2 = X(2);
        // U1: A = U1U3, B = -ikx U1U1 - (fl1(j+1) - fl1(j)) / (2 DYF(j))
        G[0 * Gfield + off] = x0;
        CX t = mikx(x1);
        G[1 * Gfield + off] = CT<CX>::mk(t.x - (x4.x - PV(0, s).x) * id2, t.y - (x4.y - PV(0, s).y) * id2);
        // U2 (GY j): A = ubar3 u2(j), B = -ikx ubar1 u2(j) - (g(j) - g(j-1)) / DY(j)
        G[2 * Gfield + off] = PV(3, s);
        t = mikx(PV(2, s));
        G[3 * Gfield + off] = CT<CX>::mk(t.x - (x3.x - PV(4, s).x) * idyj, t.y - (x3.y - PV(4, s).y) * idyj);
        // U3: A = U3U3, B = -ikx U1U3 - (fl3(j+1) - fl3(j)) / (2 DYF(j))
        G[4 * Gfield + off] = x2;
        t = mikx(x0);
        G[5 * Gfield + off] = CT<CX>::mk(t.x - (x5.x - PV(1, s).x) * id2, t.y - (x5.y - PV(1, s).y) * id2);
#pragma unroll
        for (int n = 0; n < NTH; n++) {
          const CX a = X(8 + 3 * n), b = X(9 + 3 * n), c = X(10 + 3 * n);
          G[(6 + 2 * n) * Gfield + off] = b;
          t = mikx(a);
          G[(7 + 2 * n) * Gfield + off] =
              CT<CX>::mk(t.x - (c.x - PV(5 + n, s).x) * id2, t.y - (c.y - PV(5 + n, s).y) * id2);
        }
      }
      PV(0, s) = x4;
      PV(1, s) = x5;
      PV(2, s) = x6;
      PV(3, s) = x7;
      PV(4, s) = x3;
#pragma unroll
      for (int n = 0; n < NTH; n++) PV(5 + n, s) = X(10 + 3 * n);
    }
    __syncwarp();
#pragma unroll
    for (int f = 0; f < NF; f++) {
#pragma unroll
      for (int i = 0; i < XPL; i++) cur[f][i] = nxt[f][i];
      dcur[f] = dnxt[f];
    }
  }
#undef PV
}

template <int NX, int NTH, typename CX = double2>
size_t xw_smem() {
  constexpr int NF = 3 + NTH, NPIN = (NF + 1) / 2, NPP = (8 + 3 * NTH + 1) / 2;
  constexpr int MAXP = NPIN > NPP ? NPIN : NPP;
  return sizeof(CX) * (NX + XW_WARPS * MAXP * padded_len(NX) + XW_WARPS * (5 + NTH) * (NX / 3 + 1));
}

// Planes one x-row CTA marches through when the tuning leaves it automatic
// (DG_TUNE_XROW_CHUNK = 0): the fewest (at least 3) that fit the whole grid
// into one wave of resident CTAs, so no SM waits out a partial last wave;
// grids too large for that take 32 planes per CTA.
int xrow_auto_chunk(int nplan, int NZ, const void *kern, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<const void *, size_t>, int> per_sm_cache;
  static int nsm = 0;
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!nsm) {
      int dev = 0;
      cudaGetDevice(&dev);
      if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        nsm = 148;
    }
    auto it = per_sm_cache.find({kern, smem});
    if (it != per_sm_cache.end()) {
      per_sm = it->second;
    } else {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * XW_WARPS, smem) !=
          cudaSuccess)
        per_sm = 1;
      per_sm_cache[{kern, smem}] = per_sm;
    }
  }
  const long slots = (long)(per_sm > 0 ? per_sm : 1) * nsm;
  const long zb = dg_cdiv(NZ, XW_WARPS);
  const long per_col = slots / zb > 0 ? slots / zb : 1;  // CTAs per z-block column in one wave
  int chunk = dg_cdiv(nplan, per_col);
  if (chunk < 3) chunk = 3;
  if (chunk > 32) chunk = 32;
  return chunk < nplan ? chunk : nplan;
}

// the plan variant of the handle's tuning, for lengths that have one
template <int NX, int NTH, typename CX>
auto xrow_kernel(int v) {
  if constexpr (plan_has_variant(NX))
    if (v) return k_xrow_w<NX, NTH, CX, 1>;
  return k_xrow_w<NX, NTH, CX, 0>;
}

// ------------------------------------------------------------- zfwd + rhs
constexpr int ZF_THR = 128;
__host__ __device__ constexpr int zf_kxg(int nz) { return nz <= 128 ? 8 : (nz <= 256 ? 4 : 2); }

// NLO: write only the nonlinear term -i kz A + B of every retained mode to
// rhs (the column kernel forms the explicit terms and the right-hand side);
// otherwise the epilogue below also forms CF and the CN right-hand side R.
template <int NT, bool NLO>
__global__ void __launch_bounds__(ZF_THR) k_zfwd_rhs(
    ChanConst C, const double2 *__restrict__ G, long Gfield, FftPlan pl,
    const double2 *__restrict__ tw, const double *__restrict__ dscal, int rk_step,
    const double *__restrict__ kxv, const double *__restrict__ kzv, const double *__restrict__ dy,
    const double *__restrict__ dyf, FieldPtrs cu, FieldPtrs cf, FieldPtrs rhs,
    const double2 *__restrict__ cp) {
  extern __shared__ double2 sm[];
  const int NZ = NT ? NT : C.NZ;
  const int nkxp = C.nkxp, nkzt = C.nkzt, nf = C.nf, NKZ = C.NKZ;
  const int ZF_KXG = zf_kxg(NZ);
  const int sstr = padded_len(NZ);
  double2 *stw = sm;
  double2 *b0 = stw + NZ;
  double2 *b1 = b0 + 2 * ZF_KXG * sstr;
  double2 *nl = b0 + fft_bufs(NZ) * 2 * ZF_KXG * sstr;  // [f][c][kp]
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int kx0 = blockIdx.x * ZF_KXG;
  const int j = 1 + blockIdx.y;
  for (int i = tid; i < NZ; i += nthr) stw[i] = tw[i];
  const double rnz = (double)NZ;

  for (int f = 0; f < nf; f++) {
    for (int idx = tid; idx < 2 * ZF_KXG * NZ; idx += nthr) {
      const int c = idx % ZF_KXG;
      const int z = (idx / ZF_KXG) % NZ;
      const int ab = idx / (ZF_KXG * NZ);
      double2 v = make_double2(0.0, 0.0);
      if (kx0 + c < nkxp)
        v = G[(2 * f + ab) * Gfield + (long)j * NZ * nkxp + (long)z * nkxp + kx0 + c];
      b0[(ab * ZF_KXG + c) * sstr + pad(z)] = v;
    }
    __syncthreads();
    double2 *res = fft<NT>(b0, b1, pl, 2 * ZF_KXG, sstr, stw, -1);
    for (int idx = tid; idx < ZF_KXG * nkzt; idx += nthr) {
      const int c = idx % ZF_KXG, kp = idx / ZF_KXG;
      const int z = (kp <= NKZ) ? kp : (NZ - 1 + (kp - NKZ) - NKZ);
      double2 a = res[(0 * ZF_KXG + c) * sstr + pad(z)];
      double2 b = res[(1 * ZF_KXG + c) * sstr + pad(z)];
      a = make_double2(a.x / rnz, a.y / rnz);
      b = make_double2(b.x / rnz, b.y / rnz);
      const double KZ = kzv[kp];
      // -i kz a + b
      nl[(f * ZF_KXG + c) * nkzt + kp] = make_double2(KZ * a.y + b.x, -KZ * a.x + b.y);
    }
    __syncthreads();
  }
  if constexpr (NLO) {
    for (int idx = tid; idx < ZF_KXG * nkzt; idx += nthr) {
      const int c = idx % ZF_KXG, kp = idx / ZF_KXG;
      const int kx = kx0 + c;
      if (kx >= nkxp) continue;
      const long o = (long)j * C.ss + (long)kp * nkxp + kx;
      if (j >= C.JS && j <= C.JE) {
        rhs(0)[o] = nl[(0 * ZF_KXG + c) * nkzt + kp];
        rhs(2)[o] = nl[(2 * ZF_KXG + c) * nkzt + kp];
      }
      if (j >= 2 && j <= C.NY) rhs(1)[o] = nl[(1 * ZF_KXG + c) * nkzt + kp];
      for (int n = 0; n < C.nth; n++)
        if (j >= C.JSt[n] && j <= C.JEt[n]) rhs(3 + n)[o] = nl[((3 + n) * ZF_KXG + c) * nkzt + kp];
    }
    return;
  }
  // explicit terms and CN right-hand side per retained mode of plane j
  const double h = dscal[1 + rk_step];
  const double time = dscal[0];
  const double zeta = (rk_step == 2) ? -17.0 / 8.0 : (rk_step == 3) ? -5.0 / 4.0 : 0.0;
  const double bbar = (rk_step == 2) ? 25.0 / 8.0 : (rk_step == 3) ? 9.0 / 4.0 : 1.0;
  const double T1 = C.nu * h / 2.0, T3 = zeta * h, T4 = h, T5 = bbar * h;
  const double NU = C.nu, NUV = C.nuv;
  const long ss = C.ss;
  const double dyj = dy[j], dyj1 = dy[j + 1], dyfj = dyf[j], dyfm = dyf[j - 1];
  for (int idx = tid; idx < ZF_KXG * nkzt; idx += nthr) {
    const int c = idx % ZF_KXG, kp = idx / ZF_KXG;
    const int kx = kx0 + c;
    if (kx >= nkxp) continue;
    const long o = (long)j * ss + (long)kp * nkxp + kx;
    const double KX = kxv[kx], KZ = kzv[kp];
    const double k2 = KX * KX + KZ * KZ;
    const double kk = (C.beta == 1.0) ? k2 : pow(k2, C.beta);
    const bool mean = (kx == 0 && kp == 0);
    const double2 u1 = cu(0)[o], u2 = cu(1)[o], u3 = cu(2)[o];
    const double2 p0 = cp[o];
    // ---- U1 and U3 (rows JSTART..JEND)
    if (j >= C.JS && j <= C.JE) {
      const double2 u1m = cu(0)[o - ss], u1p = cu(0)[o + ss];
      const double2 u3m = cu(2)[o - ss], u3p = cu(2)[o + ss];
      double2 f1 = make_double2(-NU * kk * u1.x + C.i_ro * u3.x, -NU * kk * u1.y + C.i_ro * u3.y);
      double2 f3 = make_double2(-NU * kk * u3.x - C.i_ro * u1.x, -NU * kk * u3.y - C.i_ro * u1.y);
      for (int n = 0; n < C.nth; n++) {
        const double2 t = cu(3 + n)[o];
        f1.x += C.ri[n] * C.grav_x * t.x; f1.y += C.ri[n] * C.grav_x * t.y;
        f3.x += C.ri[n] * C.grav_z * t.x; f3.y += C.ri[n] * C.grav_z * t.y;
      }
      const double2 n1 = nl[(0 * ZF_KXG + c) * nkzt + kp], n3 = nl[(2 * ZF_KXG + c) * nkzt + kp];
      f1.x += n1.x; f1.y += n1.y;
      f3.x += n3.x; f3.y += n3.y;
      double2 r1 = u1, r3 = u3;
      if (rk_step > 1) {
        const double2 o1 = cf(0)[o], o3 = cf(2)[o];
        r1.x += T3 * o1.x; r1.y += T3 * o1.y;
        r3.x += T3 * o3.x; r3.y += T3 * o3.y;
      }
      // - h (i kx P), - h (i kz P)
      r1.x -= T4 * (-KX * p0.y); r1.y -= T4 * (KX * p0.x);
      r3.x -= T4 * (-KZ * p0.y); r3.y -= T4 * (KZ * p0.x);
      if (mean) {
        if (C.f_type == 1) r1.x -= T4 * C.px0;
        else if (C.f_type == 2) r1.x -= T4 * (C.px0 + C.amp_omega0 * cos(C.omega0 * time));
      }
      r1.x += T5 * f1.x; r1.y += T5 * f1.y;
      r3.x += T5 * f3.x; r3.y += T5 * f3.y;
      const double a = T1 * NUV;
      r1.x += a * (((u1p.x - u1.x) / dyj1 - (u1.x - u1m.x) / dyj) / dyfj);
      r1.y += a * (((u1p.y - u1.y) / dyj1 - (u1.y - u1m.y) / dyj) / dyfj);
      r3.x += a * (((u3p.x - u3.x) / dyj1 - (u3.x - u3m.x) / dyj) / dyfj);
      r3.y += a * (((u3p.y - u3.y) / dyj1 - (u3.y - u3m.y) / dyj) / dyfj);
      cf(0)[o] = f1;
      cf(2)[o] = f3;
      rhs(0)[o] = r1;
      rhs(2)[o] = r3;
    }
    // ---- U2 (rows 2..NY)
    if (j >= 2 && j <= C.NY) {
      const double2 u2m = cu(1)[o - ss], u2p = cu(1)[o + ss];
      double2 f2 = make_double2(-NU * kk * u2.x, -NU * kk * u2.y);
      if (!mean) {
        for (int n = 0; n < C.nth; n++) {
          const double2 t = cu(3 + n)[o], tm = cu(3 + n)[o - ss];
          const double w = C.ri[n] * C.grav_y;
          f2.x += w * (t.x * dyfm + tm.x * dyfj) / (2.0 * dyj);
          f2.y += w * (t.y * dyfm + tm.y * dyfj) / (2.0 * dyj);
        }
      }
      const double2 n2 = nl[(1 * ZF_KXG + c) * nkzt + kp];
      f2.x += n2.x; f2.y += n2.y;
      double2 r2 = u2;
      if (rk_step > 1) {
        const double2 o2 = cf(1)[o];
        r2.x += T3 * o2.x; r2.y += T3 * o2.y;
      }
      const double2 pm = cp[o - ss];
      r2.x -= T4 * ((p0.x - pm.x) / dyj);
      r2.y -= T4 * ((p0.y - pm.y) / dyj);
      r2.x += T5 * f2.x; r2.y += T5 * f2.y;
      const double a = T1 * NUV;
      r2.x += a * (((u2p.x - u2.x) / dyfj - (u2.x - u2m.x) / dyfm) / dyj);
      r2.y += a * (((u2p.y - u2.y) / dyfj - (u2.y - u2m.y) / dyfm) / dyj);
      cf(1)[o] = f2;
      rhs(1)[o] = r2;
    }
    // ---- scalars (rows JSTART_TH..JEND_TH)
    for (int n = 0; n < C.nth; n++) {
      if (j < C.JSt[n] || j > C.JEt[n]) continue;
      const double2 t = cu(3 + n)[o], tm = cu(3 + n)[o - ss], tp = cu(3 + n)[o + ss];
      const double nup = NU / C.pr[n];
      double2 ft = make_double2(-nup * kk * t.x - u1.x * C.drhodx[n] - u3.x * C.drhodz[n],
                                -nup * kk * t.y - u1.y * C.drhodx[n] - u3.y * C.drhodz[n]);
      const double2 nt = nl[((3 + n) * ZF_KXG + c) * nkzt + kp];
      ft.x += nt.x; ft.y += nt.y;
      double2 rt = t;
      if (rk_step > 1) {
        const double2 ot = cf(3 + n)[o];
        rt.x += T3 * ot.x; rt.y += T3 * ot.y;
      }
      rt.x += T5 * ft.x; rt.y += T5 * ft.y;
      const double a = (T1 / C.pr[n]) * NUV;
      rt.x += a * (((tp.x - t.x) / dyj1 - (t.x - tm.x) / dyj) / dyfj);
      rt.y += a * (((tp.y - t.y) / dyj1 - (t.y - tm.y) / dyj) / dyfj);
      cf(3 + n)[o] = ft;
      rhs(3 + n)[o] = rt;
    }
  }
}

// Warp-per-column variant: a CTA of four warps takes 4 x zw_kpw kx columns of
// one field on one plane; the A and B columns are staged with one coalesced
// load, then each warp transforms its zw_kpw x (A, B) signals (warp passes;
// butterfly-parallel where a pass has more than 32 butterflies) and the CTA
// finishes those modes.  Two columns per warp up to NZ = 256, one above (the
// shared memory of a CTA grows with NZ).
__host__ __device__ constexpr int zw_kpw(int nz) { return nz <= 256 ? 2 : 1; }
__host__ __device__ constexpr int zw_kxg(int nz) { return 4 * zw_kpw(nz); }
__host__ __device__ constexpr int zw_minb(int nz, int esz) {
  return nz <= 256 ? (esz == 16 ? 6 : 5) : (nz <= 384 ? 3 : 2);
}
template <typename CX>
size_t zw_smem(int nz) {
  return sizeof(CX) * (nz + 4 * 2 * zw_kpw(nz) * (size_t)padded_len(nz));
}

// NLO as for k_zfwd_rhs: only -i kz A + B goes out, into rhs.
template <int NZ, typename CX = double2, bool NLO = false, int PV = 0>
__global__ void __launch_bounds__(128, zw_minb(NZ, sizeof(CX))) k_zfwd_w(
    ChanConst C, const CX *__restrict__ G, long Gfield, const CX *__restrict__ tw,
    const double *__restrict__ dscal, int rk_step, const double *__restrict__ kxv,
    const double *__restrict__ kzv, const double *__restrict__ dy, const double *__restrict__ dyf,
    FieldPtrs cu, FieldPtrs cf, FieldPtrs rhs, const double2 *__restrict__ cp, int jbase) {
  constexpr int SSTR = padded_len(NZ);
  constexpr int KPW = zw_kpw(NZ), KXG = zw_kxg(NZ);
  extern __shared__ double2 sm_raw[];
  CX *sm = reinterpret_cast<CX *>(sm_raw);
  CX *stw = sm;
  CX *buf = stw + NZ;                          // [warp][A_0..A_KPW-1 B_0..B_KPW-1][SSTR]
  const int nkxp = C.nkxp, nkzt = C.nkzt, NKZ = C.NKZ;
  const int kx0 = blockIdx.x * KXG;
  const int j = jbase + blockIdx.y;
  const int f = blockIdx.z;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // skip planes outside this field's rows
  const int jlo = (f == 0 || f == 2) ? C.JS : (f == 1 ? 2 : sel(C.JSt, f - 3));
  const int jhi = (f == 0 || f == 2) ? C.JE : (f == 1 ? C.NY : sel(C.JEt, f - 3));
  if (j < jlo || j > jhi) return;
  for (int i = threadIdx.x; i < NZ; i += blockDim.x) stw[i] = tw[i];
  dg_pdl_wait();  // G comes from the x-row kernel
  const CX *GA = G + (2 * f) * Gfield + (long)j * NZ * nkxp;
  const CX *GB = G + (2 * f + 1) * Gfield + (long)j * NZ * nkxp;
  for (int base = 0; base < 2 * KXG * NZ; base += 8 * 128) {
    CX v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int i = base + u * 128 + threadIdx.x;
      const int c = i % KXG, z = (i / KXG) % NZ, ab = i / (KXG * NZ);
      v[u] = (i < 2 * KXG * NZ && kx0 + c < nkxp) ? (ab ? GB : GA)[(long)z * nkxp + kx0 + c]
                                                 : CT<CX>::mk(0, 0);
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int i = base + u * 128 + threadIdx.x;
      if (i >= 2 * KXG * NZ) continue;
      const int c = i % KXG, z = (i / KXG) % NZ, ab = i / (KXG * NZ);
      const int w = c / KPW, s = ab * KPW + c % KPW;
      buf[(w * 2 * KPW + s) * SSTR + pad(z)] = v[u];
    }
  }
  __syncthreads();
  CX *wb = buf + warp * 2 * KPW * SSTR;
  wpasses_any<NZ, -1, 0, PV>(wb, 2 * KPW, SSTR, stw, lane);
  __syncthreads();  // the epilogue below reads every warp's columns

  const double h = dscal[1 + rk_step];
  const double time = dscal[0];
  const double zeta = (rk_step == 2) ? -17.0 / 8.0 : (rk_step == 3) ? -5.0 / 4.0 : 0.0;
  const double bbar = (rk_step == 2) ? 25.0 / 8.0 : (rk_step == 3) ? 9.0 / 4.0 : 1.0;
  const double T1 = C.nu * h / 2.0, T3 = zeta * h, T4 = h, T5 = bbar * h;
  const double NU = C.nu, NUV = C.nuv;
  const long ss = C.ss;
  const double dyj = dy[j], dyj1 = dy[j + 1], dyfj = dyf[j], dyfm = dyf[j - 1];
  // per-plane coefficients: the epilogue multiplies instead of dividing (FP64
  // division is a long instruction sequence on the FP64 pipe)
  const double inz = 1.0 / (double)NZ;
  const double aaU = T1 * NUV;
  const double cup = aaU / (dyj1 * dyfj), cdn = aaU / (dyj * dyfj);         // GYF rows
  const double cup2 = aaU / (dyfj * dyj), cdn2 = aaU / (dyfm * dyj);        // GY rows (U2)
  const double idy = 1.0 / dyj, bw2 = 1.0 / (2.0 * dyj);
  // all 128 threads over the CTA's (kz, kx) modes, kx fastest: consecutive
  // threads touch consecutive modes of a kz row
  for (int it = threadIdx.x; it < KXG * nkzt; it += 128) {
    const int c = it % KXG, kp = it / KXG;
    const int kx = kx0 + c;
    if (kx >= nkxp) continue;
    const int z = (kp <= NKZ) ? kp : (NZ - 1 + (kp - NKZ) - NKZ);
    // the transform's working precision ends here: everything below is FP64
    const CX *cb = buf + (c / KPW) * 2 * KPW * SSTR;
    const int cc = c % KPW;
    const CX aw = cb[cc * SSTR + pad(z)], bw = cb[(KPW + cc) * SSTR + pad(z)];
    const double2 a = make_double2((double)aw.x * inz, (double)aw.y * inz);
    const double2 b = make_double2((double)bw.x * inz, (double)bw.y * inz);
    const double KX = kxv[kx], KZ = kzv[kp];
    const double2 nlv = make_double2(KZ * a.y + b.x, -KZ * a.x + b.y);  // -i kz A + B
    const long o = (long)j * ss + (long)kp * nkxp + kx;
    if constexpr (NLO) {
      rhs(f)[o] = nlv;
      continue;
    }
    const double k2 = KX * KX + KZ * KZ;
    const double kk = (C.beta == 1.0) ? k2 : pow(k2, C.beta);
    const bool mean = (kx == 0 && kp == 0);
    if (f == 0 || f == 2) {
      // U1 / U3 (rows JSTART..JEND)
      const double2 u = __ldg(cu(f) + (o)), um = __ldg(cu(f) + (o - ss)), up = __ldg(cu(f) + (o + ss));
      // the other horizontal component (Coriolis), only with rotation
      const double2 uo = (C.i_ro != 0.0) ? __ldg(cu(2 - f) + (o)) : make_double2(0.0, 0.0);
      const double sgn = (f == 0) ? 1.0 : -1.0;
      const double gr = (f == 0) ? C.grav_x : C.grav_z;
      double2 fv = make_double2(-NU * kk * u.x + sgn * C.i_ro * uo.x, -NU * kk * u.y + sgn * C.i_ro * uo.y);
#pragma unroll
      for (int n = 0; n < DG_MAX_TH; n++) {
        if (n >= C.nth) break;
        const double2 t = __ldg(cu(3 + n) + (o));
        fv.x += C.ri[n] * gr * t.x;
        fv.y += C.ri[n] * gr * t.y;
      }
      fv.x += nlv.x;
      fv.y += nlv.y;
      double2 r = u;
      if (rk_step > 1) {
        const double2 old = __ldg(cf(f) + o);
        r.x += T3 * old.x;
        r.y += T3 * old.y;
      }
      const double2 p0 = __ldg(cp + o);
      const double K = (f == 0) ? KX : KZ;
      r.x -= T4 * (-K * p0.y);
      r.y -= T4 * (K * p0.x);
      if (mean && f == 0) {
        if (C.f_type == 1) r.x -= T4 * C.px0;
        else if (C.f_type == 2) r.x -= T4 * (C.px0 + C.amp_omega0 * cos(C.omega0 * time));
      }
      r.x += T5 * fv.x;
      r.y += T5 * fv.y;
      r.x += cup * (up.x - u.x) - cdn * (u.x - um.x);
      r.y += cup * (up.y - u.y) - cdn * (u.y - um.y);
      cf(f)[o] = fv;
      rhs(f)[o] = r;
    } else if (f == 1) {
      // U2 (rows 2..NY)
      const double2 u = __ldg(cu(1) + (o)), um = __ldg(cu(1) + (o - ss)), up = __ldg(cu(1) + (o + ss));
      double2 fv = make_double2(-NU * kk * u.x, -NU * kk * u.y);
      if (!mean) {
#pragma unroll
        for (int n = 0; n < DG_MAX_TH; n++) {
          if (n >= C.nth) break;
          const double2 t = __ldg(cu(3 + n) + (o)), tm = __ldg(cu(3 + n) + (o - ss));
          const double w = C.ri[n] * C.grav_y * bw2;
          fv.x += w * (t.x * dyfm + tm.x * dyfj);
          fv.y += w * (t.y * dyfm + tm.y * dyfj);
        }
      }
      fv.x += nlv.x;
      fv.y += nlv.y;
      double2 r = u;
      if (rk_step > 1) {
        const double2 old = __ldg(cf(1) + o);
        r.x += T3 * old.x;
        r.y += T3 * old.y;
      }
      const double2 p0 = __ldg(cp + o), pm = __ldg(cp + (o - ss));
      r.x -= T4 * ((p0.x - pm.x) * idy);
      r.y -= T4 * ((p0.y - pm.y) * idy);
      r.x += T5 * fv.x;
      r.y += T5 * fv.y;
      r.x += cup2 * (up.x - u.x) - cdn2 * (u.x - um.x);
      r.y += cup2 * (up.y - u.y) - cdn2 * (u.y - um.y);
      cf(1)[o] = fv;
      rhs(1)[o] = r;
    } else {
      // scalar n (rows JSTART_TH..JEND_TH)
      const int n = f - 3;
      const double2 t = __ldg(cu(f) + (o)), tm = __ldg(cu(f) + (o - ss)), tp = __ldg(cu(f) + (o + ss));
      const double nup = NU / sel(C.pr, n);  // once per item: scalar fields only
      double2 fv = make_double2(-nup * kk * t.x, -nup * kk * t.y);
      if (sel(C.drhodx, n) != 0.0 || sel(C.drhodz, n) != 0.0) {
        const double2 u1 = __ldg(cu(0) + (o)), u3 = __ldg(cu(2) + (o));
        fv.x = fv.x - u1.x * sel(C.drhodx, n) - u3.x * sel(C.drhodz, n);
        fv.y = fv.y - u1.y * sel(C.drhodx, n) - u3.y * sel(C.drhodz, n);
      }
      fv.x += nlv.x;
      fv.y += nlv.y;
      double2 r = t;
      if (rk_step > 1) {
        const double2 old = __ldg(cf(f) + o);
        r.x += T3 * old.x;
        r.y += T3 * old.y;
      }
      r.x += T5 * fv.x;
      r.y += T5 * fv.y;
      const double ipr = 1.0 / sel(C.pr, n);
      r.x += ipr * (cup * (tp.x - t.x) - cdn * (t.x - tm.x));
      r.y += ipr * (cup * (tp.y - t.y) - cdn * (t.y - tm.y));
      cf(f)[o] = fv;
      rhs(f)[o] = r;
    }
  }
}

template <int NZ, typename CX, bool NLO>
auto zfwd_kernel(int v) {
  if constexpr (plan_has_variant(NZ))
    if (v) return k_zfwd_w<NZ, CX, NLO, 1>;
  return k_zfwd_w<NZ, CX, NLO, 0>;
}

__host__ __device__ constexpr bool zw_supported(int n) {
  return n == 16 || n == 32 || n == 48 || n == 64 || n == 96 || n == 128 || n == 256;
}
// lengths with a compile-time plan above the warp-signal lengths (FP64 only)
__host__ __device__ constexpr bool zw_big(int n) { return n == 192 || n == 384 || n == 512; }

size_t zfwd_smem(const dg_handle *h) {
  const int kxg = zf_kxg(h->NZ);
  return sizeof(double2) * (h->NZ + fft_bufs(h->NZ) * 2 * kxg * padded_len(h->NZ) +
                            h->nf * kxg * h->nkzt);
}

// ------------------------------------------------------------ CN tables
// The reference builds, per physical column, identity rows, CN rows over the
// build range, then the lower and upper BC rows (for/channel.f:771-1029,
// 1660-2282), and eliminates forward (for/mpi.f:672-700):
// a(j) = -a(j)/b(j-1), b(j) += a(j) c(j-1).  The rows are the same for every
// column and linear in TEMP1 = NU H_BAR / 2, so the host stores per row
//   CN row : l = t l1, d = 1 + t d1, u = t u1   with t = TEMP1 (or TEMP1/PR)
//   fixed  : l0, d0, u0 and the BC value
// and one CTA per (substep, field) runs the elimination whenever DELTA_T
// changes.  Output per (rk, field): [5][LP] = a', 1/b', -c/b', kind, bc value
// (LP = NY + 2 rounded up to even).
struct CnRows {
  int NY, nfld;
  double nu, nuv, pr[3 + DG_MAX_TH];  // pr = 1 for velocity
};

// blockIdx.x = rk * nfld + field.  The CTA stages the field's row templates
// into shared memory with coalesced loads and forms every row's (l, d, u) in
// parallel.  The pivots b(j) = d(j) - l(j) u(j-1) / b(j-1) of the forward
// elimination are ratios b(j) = p(j) / p(j-1) of the continuants
//   p(j) = d(j) p(j-1) + w(j) p(j-2),   w(j) = -l(j) u(j-1),
//   p(-1) = 1, p(-2) = 0,
// so one thread runs that three-term recurrence, whose critical path per
// row is a single multiply-add (a zero pivot restarts it the way the
// elimination does: 1/b = 0, and the next row keeps its own diagonal), and
// rescales the pair by a power of two every 4 rows (exact, so the ratios
// are unchanged).  Every thread then forms its rows' reciprocal pivots
// p(j-1) / p(j), multipliers -l(j) / b(j-1) and -u(j) / b(j), and the CTA
// writes the table back with coalesced stores.
constexpr int CT_THR = 128;

__global__ void __launch_bounds__(CT_THR) k_cn_tables(CnRows P, const double *__restrict__ dscal,
                                                      const double *__restrict__ rows,
                                                      double *__restrict__ tab) {
  // rows: [field][8][L] = kind, l1, d1, u1, l0, d0, u0, v
  extern __shared__ double ct_sm[];
  const int L = P.NY + 2;
  const int rk = blockIdx.x / P.nfld, f = blockIdx.x % P.nfld;
  double *R = ct_sm;           // [8][L] templates, then the continuants [2][L]
  double *T = ct_sm + 8 * L;   // [5][L]: w, 1/b, u, kind, bc value
  double *W = T + 5 * L;       // [2][L] l, d of every row
  const double *Rg = rows + (long)f * 8 * L;
  for (int i = threadIdx.x; i < 8 * L; i += CT_THR) R[i] = Rg[i];
  __syncthreads();
  const double h = dscal[2 + rk];
  const double s = (P.nu * h / 2.0) / P.pr[f] * P.nuv;
  auto row_u = [&](int j) {
    return (R[j] == (double)ROW_RHS) ? s * R[3 * L + j] : R[6 * L + j];
  };
  for (int j = threadIdx.x; j < L; j += CT_THR) {
    const bool cn = R[j] == (double)ROW_RHS;
    const double l = cn ? s * R[1 * L + j] : R[4 * L + j];
    W[j] = l;
    W[L + j] = cn ? 1.0 + s * R[2 * L + j] : R[5 * L + j];     // d
    T[j] = (j > 0) ? -l * row_u(j - 1) : 0.0;                  // w
    T[2 * L + j] = row_u(j);                                   // u
    T[3 * L + j] = R[j];                                       // kind
    T[4 * L + j] = R[7 * L + j];                               // bc value
  }
  __syncthreads();
  double *Pc = R, *Qc = R + L;  // p(j) and p(j-1), one scale per row
  if (threadIdx.x == 0) {
    constexpr int B = 8;
    double pm = 0.0, pc = 1.0;  // p(j-2), p(j-1)
    for (int j0 = 0; j0 < L; j0 += B) {
      double d[B], w[B];
#pragma unroll
      for (int q = 0; q < B; q++) {
        const int j = j0 + q < L ? j0 + q : L - 1;
        d[q] = W[L + j];
        w[q] = T[j];
      }
#pragma unroll
      for (int q = 0; q < B; q++) {
        const int j = j0 + q;
        if (j < L) {
          double pn = fma(d[q], pc, w[q] * pm);
          const bool z = (pn == 0.0);
          const double pq = z ? 0.0 : pc;
          pn = z ? 1.0 : pn;
          Pc[j] = pn;
          Qc[j] = pq;
          pm = pq;
          pc = pn;
          if ((q & 3) == 3) {
            // 2^-e with e the exponent of p(j), clamped inside the normal range
            const int e = ((__double2hiint(pc) >> 20) & 0x7ff) - 1023;
            const int ec = e < -1000 ? -1000 : (e > 1000 ? 1000 : e);
            const double sc = __hiloint2double((1023 - ec) << 20, 0);
            pm *= sc;
            pc *= sc;
          }
        }
      }
    }
  }
  __syncthreads();
  for (int j = threadIdx.x; j < L; j += CT_THR) T[L + j] = Qc[j] / Pc[j];
  __syncthreads();
  // rows of LP = L rounded up to even doubles, so every row starts on a
  // 16-byte boundary (the column kernel fetches them by bulk copies)
  const int LP = (L + 1) & ~1;
  double *Tg = tab + (long)(rk * (3 + DG_MAX_TH) + f) * 5 * LP;
  for (int i = threadIdx.x; i < 5 * LP; i += CT_THR) {
    const int r = i / LP, j = i - r * LP;
    double v = 0.0;
    if (j < L) {
      // row 0: the multiplier -l / b(j-1) (0 on the first row); row 2: the
      // backward recurrence's coefficient -u / b (0 on the last row)
      if (r == 0) v = (j > 0) ? -W[j] * T[L + j - 1] : 0.0;
      else if (r == 2) v = (j < L - 1) ? -T[2 * L + j] * T[L + j] : 0.0;
      else v = T[r * L + j];
    }
    Tg[i] = v;
  }
}

// ------------------------------------------------------------- REM_DIV
// Multipliers and reciprocal pivots of REM_DIV_CHAN's system for every mode
// (rows 1..NY, APPLY_BC_REM_DIV_MPI rows 1 and NY, THOMAS_FORWARD_COMPLEX_MPI).
// The system depends only on the grid and kx^2 + kz^2, so it is built once.
__global__ void k_remdiv_init(int NY, long ss, int nkxp, const double *__restrict__ kxv,
                              const double *__restrict__ kzv, const double *__restrict__ dy,
                              const double *__restrict__ dyf, double *__restrict__ ra,
                              double *__restrict__ rrb) {
  const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= ss) return;
  const int kx = (int)(m % nkxp), kp = (int)(m / nkxp);
  const double kx2 = kxv[kx] * kxv[kx], kz2 = kzv[kp] * kzv[kp];
  const bool mean = (m == 0);
  double bprev = 1.0;
  double cprev = mean ? 0.0 : -1.0;
  ra[1 * ss + m] = 0.0;
  rrb[1 * ss + m] = 1.0;
  for (int j = 2; j <= NY; j++) {
    double l, d, u;
    if (j < NY) {
      l = 1. / (dy[j] * dyf[j]);
      d = -kx2 - kz2 - 1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]);
      u = 1. / (dy[j + 1] * dyf[j]);
    } else {
      l = 1.;
      d = -1.;
      u = 0.;
    }
    const double a = (bprev != 0.0) ? -l / bprev : 0.0;
    const double b = d + a * cprev;
    ra[(long)j * ss + m] = a;
    rrb[(long)j * ss + m] = (b != 0.0) ? 1.0 / b : 0.0;
    bprev = b;
    cprev = u;
  }
}

// ------------------------------------------------------- column kernels
// k_rd_col: REM_DIV_CHAN for MT modes and their whole y-columns -- the
// divergence of the velocity, the solve of the Poisson system for phi
// (multipliers and reciprocal pivots per mode from k_remdiv_init), the
// projection and CP += phi / H_BAR.  The solve is the two recurrences of
// THOMAS_FORWARD / THOMAS_BACKWARD, forward g(j) = r(j) + a(j) g(j-1) and
// backward phi(j) = e(j) + f(j) phi(j+1) with e = g / b and f = -c / b,
// split over segments of RD_K rows: one thread per (mode, segment) runs its
// segment from a zero start keeping the product of the coefficients, one
// lane per mode carries the segment ends across the column, and each thread
// adds carry x product to its rows (the same algebra as the sequential
// sweeps, with the rounding of a different order of the same operations;
// the segment boundaries depend only on NY).  The divergence and the
// projection are flat loops over (row, mode) across the CTA; the velocity
// and CP are read from global memory there (coalesced), the factors by the
// segment threads.
constexpr int RD_K = 8;        // rows per segment
constexpr int RD_MAX_THR = 256;

// The velocity is read from s1..s3 and written to u1..u3: the same arrays for
// REM_DIV_CHAN on its own (in place), the rhs arrays holding the column
// stage's post-CN velocity inside a substep.  In that case the rows the
// projection leaves alone (U1, U3 at NY+1; U2 at 1 and NY+1) and the scalars
// the column stage also left in the rhs arrays (RdCopy) are copied over too.
struct RdCopy {
  const double2 *src[DG_MAX_TH];
  double2 *dst[DG_MAX_TH];
  int lo[DG_MAX_TH];  // first row the column stage wrote
  int n;
};

struct RdArgs {
  int NY, nkxp, JS, JE, rk_step, nseg;
  long ss;
  const double *kxv, *kzv, *dy, *dyf, *ra, *rrb, *dscal;
  const double2 *s1, *s2, *s3;
  double2 *u1, *u2, *u3, *cp, *phi;
  RdCopy cpy;
};

// shared memory: PH [L][MT] double2 (r, g, e, phi), SV [nseg][MT] double2,
// SP [nseg][MT], UU, IDY, IDYF [L], KXS, KZS [MT]
size_t rd_smem(int L, int nseg, int mt) {
  return sizeof(double2) * ((size_t)L * mt + (size_t)nseg * mt) +
         sizeof(double) * ((size_t)nseg * mt + 3 * (size_t)L + 2 * (size_t)mt);
}

template <int MT>
__global__ void __launch_bounds__(RD_MAX_THR, 3) k_rd_col(RdArgs A) {
  extern __shared__ double2 rsm[];
  const int NY = A.NY, L = NY + 2, nseg = A.nseg;
  const long ss = A.ss;
  const long m0 = (long)blockIdx.x * MT;
  const int mt = (int)((ss - m0) < MT ? (ss - m0) : MT);
  double2 *PH = rsm;                                // [j][MT]
  double2 *SV = PH + (long)L * MT;                  // [seg][MT]
  double *SP = reinterpret_cast<double *>(SV + (long)nseg * MT);  // [seg][MT]
  double *UU = SP + (long)nseg * MT;                // [j] upper diagonal rows 2..NY-1
  double *IDY = UU + L;                             // [j] 1 / DY(j)
  double *IDYF = IDY + L;                           // [j] 1 / DYF(j)
  double *KXS = IDYF + L, *KZS = KXS + MT;          // wavenumbers of the CTA's modes
  const int tid = threadIdx.x, nthr = blockDim.x;
  if (tid < MT) {
    const int mi = (int)(m0 + tid) < (int)ss ? (int)(m0 + tid) : 0;
    KXS[tid] = A.kxv[mi % A.nkxp];
    KZS[tid] = A.kzv[mi / A.nkxp];
  }
  for (int j = tid; j < L; j += nthr) {
    UU[j] = (j >= 2 && j < NY) ? 1. / (A.dy[j + 1] * A.dyf[j]) : 0.0;
    IDY[j] = (j >= 1) ? 1. / A.dy[j] : 0.0;
    IDYF[j] = (j >= 1 && j <= NY) ? 1. / A.dyf[j] : 0.0;
  }
  dg_pdl_wait();  // the velocity comes from the CN solve
  __syncthreads();
  // The loops below read the velocity and CP and write the velocity, phi
  // and CP, in place when projecting on its own.  Every store depends on the
  // load of the same element in the same iteration, so the stores cannot move
  // above those loads, and the loads of later elements may be issued early:
  // the pointers are declared non-aliasing for that.
  const double2 *__restrict__ s1 = A.s1;
  const double2 *__restrict__ s2 = A.s2;
  const double2 *__restrict__ s3 = A.s3;
  double2 *__restrict__ u1 = A.u1;
  double2 *__restrict__ u2 = A.u2;
  double2 *__restrict__ u3 = A.u3;
  const double2 *__restrict__ cpin = A.cp;
  double2 *__restrict__ cpout = A.cp;
  double2 *__restrict__ phio = A.phi;
  // ---- 1. the divergence (rows 2..NY-1; rows 1 and NY have a zero
  // right-hand side)
  for (int i = MT + tid; i < (NY + 1) * MT; i += nthr) {
    const int j = i / MT, m = i - j * MT;
    double2 r = make_double2(0.0, 0.0);
    if (m < mt && j >= 2 && j < NY) {
      const long o = (long)j * ss + m0 + m;
      const double2 a1 = s1[o], a3 = s3[o], b2 = s2[o], b2p = s2[o + ss];
      const double KX = KXS[m], KZ = KZS[m];
      const double id = IDYF[j];
      r.x = (-KX * a1.y) + (b2p.x - b2.x) * id + (-KZ * a3.y);
      r.y = (KX * a1.x) + (b2p.y - b2.y) * id + (KZ * a3.x);
    }
    PH[i] = r;
  }
  __syncthreads();
  // ---- 2. forward recurrence over each segment of rows 1..NY from zero
  // (g(1) = 0: the multiplier of row 1 is taken as 0)
  const int m = tid % MT, s = tid / MT;
  const int j0 = 1 + s * RD_K;
  const int nr = (s < nseg) ? min(RD_K, NY + 1 - j0) : 0;
  const bool live = m < mt;
  const long mg = live ? m0 + m : m0;
  double a[RD_K], rb[RD_K];
#pragma unroll
  for (int q = 0; q < RD_K; q++) {
    const long o = (long)(j0 + q) * ss + mg;
    a[q] = (q < nr && j0 + q >= 2) ? A.ra[o] : 0.0;
    rb[q] = (q < nr) ? A.rrb[o] : 0.0;
  }
  {
    double2 g = make_double2(0.0, 0.0);
    double pa = 1.0;
#pragma unroll
    for (int q = 0; q < RD_K; q++) {
      if (q < nr) {
        const double2 r = PH[(j0 + q) * MT + m];
        g.x = r.x + a[q] * g.x;
        g.y = r.y + a[q] * g.y;
        pa = a[q] * pa;
        PH[(j0 + q) * MT + m] = g;
      }
    }
    if (nr > 0) {
      SV[s * MT + m] = g;
      SP[s * MT + m] = pa;
    }
  }
  __syncthreads();
  if (tid < MT) {
    double2 G = make_double2(0.0, 0.0);
    for (int t = 0; t < nseg; t++) {
      const double2 e = SV[t * MT + tid];
      const double p = SP[t * MT + tid];
      SV[t * MT + tid] = G;
      G = make_double2(e.x + p * G.x, e.y + p * G.y);
    }
  }
  __syncthreads();
  // ---- 3. g = local + product x carry, e = g / b; the backward recurrence
  // phi(j) = e(j) + f(j) phi(j+1), f = -c / b (row NY: f = 0; row 1: the
  // upper coefficient of APPLY_BC_REM_DIV_MPI, 0 for the mean mode, -1
  // otherwise)
  const bool mean = live && (m0 + m == 0);
  {
    const double2 c = (nr > 0) ? SV[s * MT + m] : make_double2(0.0, 0.0);
    double pi = 1.0;
    double2 e[RD_K];
#pragma unroll
    for (int q = 0; q < RD_K; q++) {
      e[q] = make_double2(0.0, 0.0);
      if (q < nr) {
        pi = a[q] * pi;
        const double2 gv = PH[(j0 + q) * MT + m];
        e[q] = make_double2((gv.x + pi * c.x) * rb[q], (gv.y + pi * c.y) * rb[q]);
      }
    }
    double2 xl = make_double2(0.0, 0.0);
    double ps = 1.0;
#pragma unroll
    for (int q = RD_K - 1; q >= 0; q--) {
      if (q < nr) {
        const int j = j0 + q;
        const double up = (j == NY) ? 0.0 : (j == 1) ? (mean ? 0.0 : -1.0) : UU[j];
        const double fj = -up * rb[q];
        xl = make_double2(e[q].x + fj * xl.x, e[q].y + fj * xl.y);
        ps = fj * ps;
        PH[j * MT + m] = xl;
      }
    }
    if (nr > 0) {
      SV[s * MT + m] = xl;
      SP[s * MT + m] = ps;
    }
  }
  __syncthreads();
  if (tid < MT) {
    double2 X = make_double2(0.0, 0.0);
    for (int t = nseg - 1; t >= 0; t--) {
      const double2 e = SV[t * MT + tid];
      const double p = SP[t * MT + tid];
      SV[t * MT + tid] = X;
      X = make_double2(e.x + p * X.x, e.y + p * X.y);
    }
  }
  __syncthreads();
  if (nr > 0) {
    const double2 c = SV[s * MT + m];
    double p2 = 1.0;
#pragma unroll
    for (int q = RD_K - 1; q >= 0; q--) {
      if (q < nr) {
        const int j = j0 + q;
        const double up = (j == NY) ? 0.0 : (j == 1) ? (mean ? 0.0 : -1.0) : UU[j];
        p2 = (-up * rb[q]) * p2;
        const double2 xl = PH[j * MT + m];
        PH[j * MT + m] = make_double2(xl.x + p2 * c.x, xl.y + p2 * c.y);
      }
    }
  }
  __syncthreads();
  // ---- 4. the projection, phi and CP += phi / H_BAR (rows 1..NY)
  const double ihh = (A.rk_step > 0) ? 1.0 / A.dscal[1 + A.rk_step] : 1.0;
  const bool rkc = A.rk_step > 0;
  const int JS = A.JS, JE = A.JE;
#pragma unroll 4
  for (int i = MT + tid; i < (NY + 1) * MT; i += nthr) {
    const int j = i / MT, mm = i - j * MT;
    if (mm >= mt) continue;
    const long o = (long)j * ss + m0 + mm;
    const double KX = KXS[mm], KZ = KZS[mm];
    const double2 ph = PH[i];
    double2 a1 = s1[o], a3 = s3[o];
    // U1 -= i kx phi, U3 -= i kz phi
    a1.x -= -KX * ph.y; a1.y -= KX * ph.x;
    a3.x -= -KZ * ph.y; a3.y -= KZ * ph.x;
    u1[o] = a1;
    u3[o] = a3;
    if (j >= 2) {
      // U2(j) -= (phi(j) - phi(j-1)) / DY(j)
      double2 b2 = s2[o];
      const double2 pm = PH[i - MT];
      b2.x -= (ph.x - pm.x) * IDY[j];
      b2.y -= (ph.y - pm.y) * IDY[j];
      u2[o] = b2;
    }
    phio[o] = ph;
    if (rkc && j >= JS && j <= JE) {
      double2 pc = cpin[o];
      pc.x = pc.x + ph.x * ihh;
      pc.y = pc.y + ph.y * ihh;
      cpout[o] = pc;
    }
  }
  if (A.s1 == A.u1) return;
  // rows the projection does not touch, and the scalars, from the rhs arrays
  for (int i = tid; i < 3 * MT; i += nthr) {
    const int q = i / MT, mm = i - q * MT;
    if (mm >= mt) continue;
    const long top = (long)(NY + 1) * ss + m0 + mm;
    if (q == 0) { A.u1[top] = A.s1[top]; A.u3[top] = A.s3[top]; }
    else if (q == 1) A.u2[top] = A.s2[top];
    else A.u2[ss + m0 + mm] = A.s2[ss + m0 + mm];
  }
  for (int c = 0; c < A.cpy.n; c++) {
    const double2 *src = A.cpy.src[c];
    double2 *dst = A.cpy.dst[c];
    for (int i = A.cpy.lo[c] * MT + tid; i < L * MT; i += nthr) {
      const int j = i / MT, mm = i - j * MT;
      if (mm < mt) dst[(long)j * ss + m0 + mm] = src[(long)j * ss + m0 + mm];
    }
  }
}

// -------------------------------------------------------- APPLY_BC_VEL
struct BcVel {
  int NY;
  int u0, v0, w0, u1, v1, w1;
  double cu0, cv0, cw0, cu1, cv1, cw1;
};

__global__ void k_bc_vel(BcVel B, long ss, const double *__restrict__ dy,
                         const double *__restrict__ dyf, double2 *__restrict__ U1,
                         double2 *__restrict__ U2, double2 *__restrict__ U3) {
  const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= ss) return;
  const bool mean = (m == 0);
  const int NY = B.NY;
  const double2 z = make_double2(0.0, 0.0);
#define AT(F, j) F[(long)(j) * ss + m]
  // lower wall (APPLY_BC_VEL_LOWER, for/channel.f:2285-2387)
  if (B.u0 == 0) {
    AT(U1, 0) = z; AT(U1, 1) = z;
    if (mean) { AT(U1, 1) = make_double2(B.cu0, 0.0); AT(U1, 0) = make_double2(B.cu0, 0.0); }
  } else {
    AT(U1, 1) = AT(U1, 2); AT(U1, 0) = AT(U1, 1);
    if (mean) {
      double2 t = AT(U1, 2); t.x = t.x - dy[2] * B.cu0; AT(U1, 1) = t;
      t.x = t.x - dy[1] * B.cu0; AT(U1, 0) = t;
    }
  }
  if (B.w0 == 0) {
    AT(U3, 0) = z; AT(U3, 1) = z;
    if (mean) { AT(U3, 1) = make_double2(B.cw0, 0.0); AT(U3, 0) = make_double2(B.cw0, 0.0); }
  } else {
    AT(U3, 1) = AT(U3, 2); AT(U3, 0) = AT(U3, 1);
    if (mean) {
      double2 t = AT(U3, 2); t.x = t.x - dy[2] * B.cw0; AT(U3, 1) = t;
      t.x = t.x - dy[1] * B.cw0; AT(U3, 0) = t;
    }
  }
  if (B.v0 == 0) {
    double2 t = AT(U2, 2);
    t = make_double2(2.0 * B.cv0 - t.x, -t.y);
    AT(U2, 1) = t; AT(U2, 0) = t;
  } else if (B.v0 == 1) {
    AT(U2, 1) = AT(U2, 2); AT(U2, 0) = AT(U2, 1);
    if (mean) {
      double2 t = AT(U2, 2); t.x = t.x - dyf[1] * B.cv0; AT(U2, 1) = t;
      t.x = t.x - dyf[1] * B.cv0; AT(U2, 0) = t;
    }
  } else if (B.v0 == 2) {
    if (mean) { double2 t = AT(U2, 2); AT(U2, 1) = make_double2(-t.x, -t.y); }
  }
  // upper wall (APPLY_BC_VEL_UPPER, for/channel.f:2390-2492)
  if (B.u1 == 0) {
    AT(U1, NY) = z; AT(U1, NY + 1) = z;
    if (mean) { AT(U1, NY) = make_double2(B.cu1, 0.0); AT(U1, NY + 1) = make_double2(B.cu1, 0.0); }
  } else {
    AT(U1, NY) = AT(U1, NY - 1); AT(U1, NY + 1) = AT(U1, NY);
    if (mean) {
      double2 t = AT(U1, NY - 1); t.x = t.x + dy[NY] * B.cu1; AT(U1, NY) = t;
      t.x = t.x + dy[NY] * B.cu1; AT(U1, NY + 1) = t;
    }
  }
  if (B.w1 == 0) {
    AT(U3, NY) = z; AT(U3, NY + 1) = z;
    if (mean) { AT(U3, NY) = make_double2(B.cw1, 0.0); AT(U3, NY + 1) = make_double2(B.cw1, 0.0); }
    if (mean) AT(U3, NY + 1) = z;  // "Ghost cell not used", for/channel.f:2445
  } else {
    AT(U3, NY) = AT(U3, NY - 1); AT(U3, NY + 1) = AT(U3, NY);
    if (mean) {
      double2 t = AT(U3, NY - 1); t.x = t.x + dy[NY] * B.cw1; AT(U3, NY) = t;
      t.x = t.x + dy[NY] * B.cw1; AT(U3, NY + 1) = t;
    }
  }
  if (B.v1 == 0) {
    if (mean) { double2 t = AT(U2, NY); AT(U2, NY + 1) = make_double2(2.0 * B.cv1 - t.x, -t.y); }
  } else if (B.v1 == 1) {
    AT(U2, NY) = AT(U2, NY - 1); AT(U2, NY + 1) = AT(U2, NY);
    if (mean) { double2 t = AT(U2, NY); t.x = t.x + dy[NY] * B.cv1; AT(U2, NY + 1) = t; }
  } else if (B.v1 == 2) {
    if (mean) { double2 t = AT(U2, NY); AT(U2, NY + 1) = make_double2(-t.x, -t.y); }
  }
#undef AT
}

// ------------------------------------------------------------- COURANT
__global__ void k_cfl_min(const double *__restrict__ phys, long pfield, int NY, int NZ, int NX,
                          double cfl, double dxv, double dzv, const double *__restrict__ dy,
                          unsigned long long *__restrict__ out) {
  // phys holds U1, U2, U3 for planes 1..NY, [f][j-1][z][x]
  const long np = (long)NZ * NX;
  const long total = (long)NY * np;
  double best = __longlong_as_double(0x7ff0000000000000LL);
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (long)gridDim.x * blockDim.x) {
    const int j = 1 + (int)(q / np);
    const double a = cfl * dxv / fabs(phys[q]);
    const double b = cfl * dy[j] / fabs(phys[pfield + q]);
    const double c = cfl * dzv / fabs(phys[2 * pfield + q]);
    best = fmin(best, fmin(a, fmin(b, c)));
  }
  for (int off = 16; off > 0; off >>= 1) best = fmin(best, __shfl_down_sync(0xffffffffu, best, off));
  if ((threadIdx.x & 31) == 0) dg_fold_min(out, best);
}

__global__ void k_dt_update(double *dscal, const unsigned long long *minbits, double dt0) {
  // for/courant.f:15-59: dt0 carries the velocity-independent limits.  The
  // new DELTA_T is parked in dscal[8]: the substep that called COURANT still
  // uses its own H_BAR for the pressure update (TEMP4 was set on entry).
  double dt = fmin(dt0, __longlong_as_double((long long)*minbits));
  double nd;
  if (dt <= 0) nd = 0.0001;
  else if (dt >= 999.) nd = 999.0;
  else nd = dt;
  dscal[8] = nd;
}

// DELTA_T = pending value; H_BAR from it (for/courant.f:60-62)
__global__ void k_dt_commit(double *dscal) {
  const double nd = dscal[8];
  dscal[1] = nd;
  dscal[2] = nd * (8.0 / 15.0);
  dscal[3] = nd * (2.0 / 15.0);
  dscal[4] = nd * (5.0 / 15.0);
}

// --------------------------------------------------------------- stats
// Per-plane Parseval sums (weights 1 for kx = 0, 2 for kx > 0):
// [0] sum|U1'|^2 [1] sum|U2'|^2 [2] sum|U3'|^2 [3] sum|U|^2 incl. mean (U1, U3)
// [4] sum|U2|^2 incl. mean  [5+n] sum|TH'|^2
__global__ void k_stats_planes(int nplanes, long ss, int nkxp, CFieldPtrs u, int nf,
                               double *__restrict__ out, int *__restrict__ flag) {
  const int j = blockIdx.x;
  __shared__ double red[8][256];
  double acc[8];
  for (int q = 0; q < 8; q++) acc[q] = 0.0;
  int bad = 0;
  for (long m = threadIdx.x; m < ss; m += blockDim.x) {
    const double w = ((m % nkxp) == 0) ? 1.0 : 2.0;
    const bool mean = (m == 0);
    for (int f = 0; f < nf; f++) {
      const double2 v = u(f)[(long)j * ss + m];
      if (!isfinite(v.x) || !isfinite(v.y)) bad = 1;
      const double e = w * (v.x * v.x + v.y * v.y);
      if (f < 3) {
        if (!mean) acc[f] += e;
        if (f == 1) acc[4] += e;
        else acc[3] += e;
      } else if (f - 3 + 5 < 8) {
        if (!mean) acc[5 + f - 3] += e;
      }
    }
  }
  if (bad) atomicOr(flag, 1);
  for (int q = 0; q < 8; q++) red[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int q = 0; q < 8; q++) red[q][threadIdx.x] += red[q][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 8) out[(long)j * 8 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_div_spec(int NY, long ss, int nkxp, const double *__restrict__ kxv,
                           const double *__restrict__ kzv, const double *__restrict__ dyf,
                           const double2 *__restrict__ u1, const double2 *__restrict__ u2,
                           const double2 *__restrict__ u3, double2 *__restrict__ d) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long tot = (long)(NY + 2) * ss;
  if (q >= tot) return;
  const int j = (int)(q / ss);
  const long m = q % ss;
  double2 r = make_double2(0.0, 0.0);
  if (j >= 2 && j <= NY - 1) {
    const double KX = kxv[m % nkxp], KZ = kzv[m / nkxp];
    const double2 a1 = u1[q], a3 = u3[q], b2 = u2[q], b2p = u2[q + ss];
    r.x = -KX * a1.y + (b2p.x - b2.x) / dyf[j] - KZ * a3.y;
    r.y = KX * a1.x + (b2p.y - b2.y) / dyf[j] + KZ * a3.x;
  }
  d[q] = r;
}

__global__ void k_absmax(const double *__restrict__ a, long n, unsigned long long *out) {
  double best = 0.0;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (long)gridDim.x * blockDim.x)
    best = fmax(best, fabs(a[q]));
  for (int off = 16; off > 0; off >>= 1) best = fmax(best, __shfl_down_sync(0xffffffffu, best, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

}  // namespace

// ================================================================ host side
// Row templates of the CN systems (host, once per handle).
static void cn_row_templates(const dg_handle *h, double *rows) {
  const int NY = h->NY, L = NY + 2, nfld = h->nf;
  const double *dy = h->h_dy, *dyf = h->h_dyf;
  for (int f = 0; f < nfld; f++) {
    double *K = rows + (long)f * 8 * L;
    double *l1 = K + L, *d1 = K + 2 * L, *u1 = K + 3 * L, *l0 = K + 4 * L, *d0 = K + 5 * L,
           *u0 = K + 6 * L, *v = K + 7 * L;
    for (int j = 0; j < L; j++) {
      K[j] = ROW_ZERO; l1[j] = d1[j] = u1[j] = 0.0; l0[j] = 0.0; d0[j] = 1.0; u0[j] = 0.0; v[j] = 0.0;
    }
    auto fixed = [&](int j, double l, double d, double u, double val) {
      K[j] = (val != 0.0) ? ROW_BC : ROW_ZERO; l0[j] = l; d0[j] = d; u0[j] = u; v[j] = val;
    };
    int lo, up;
    double clo, cup;
    if (f == F_U1) { lo = h->p.u_bc_ymin; up = h->p.u_bc_ymax; clo = h->p.u_bc_ymin_c1; cup = h->p.u_bc_ymax_c1; }
    else if (f == F_U2) { lo = h->p.v_bc_ymin; up = h->p.v_bc_ymax; clo = h->p.v_bc_ymin_c1; cup = h->p.v_bc_ymax_c1; }
    else if (f == F_U3) { lo = h->p.w_bc_ymin; up = h->p.w_bc_ymax; clo = h->p.w_bc_ymin_c1; cup = h->p.w_bc_ymax_c1; }
    else { const int n = f - 3; lo = h->p.th_bc_ymin[n]; up = h->p.th_bc_ymax[n]; clo = h->p.th_bc_ymin_c1[n]; cup = h->p.th_bc_ymax_c1[n]; }
    if (f == F_U2) {
      for (int j = 2; j <= NY; j++) {
        K[j] = ROW_RHS;
        l1[j] = -1.0 / (dyf[j - 1] * dy[j]);
        d1[j] = 1.0 / (dyf[j] * dy[j]) + 1.0 / (dyf[j - 1] * dy[j]);
        u1[j] = -1.0 / (dyf[j] * dy[j]);
      }
      if (lo == 0) { fixed(1, 0., 1., 0., clo); fixed(2, 0., 1., 0., clo); }
      else if (lo == 1) fixed(1, 0., -1., 1., dyf[1] * clo);
      fixed(0, 0., 1., 0., 0.);
      if (up == 0) { fixed(NY + 1, 0., 1., 0., cup); fixed(NY, 0., 1., 0., cup); }
      else if (up == 1) fixed(NY + 1, -1., 1., 0., dyf[NY] * cup);
    } else {
      const int j0 = (f < 3) ? h->jstart : h->jstart_th[f - 3];
      const int j1 = (f < 3) ? h->jend : h->jend_th[f - 3];
      for (int j = j0; j <= j1; j++) {
        K[j] = ROW_RHS;
        l1[j] = -1.0 / (dy[j] * dyf[j]);
        d1[j] = 1.0 / (dy[j + 1] * dyf[j]) + 1.0 / (dy[j] * dyf[j]);
        u1[j] = -1.0 / (dy[j + 1] * dyf[j]);
      }
      if (lo == 0) { fixed(0, 0., 1., 0., 0.); fixed(1, 0., 1., 0., clo); }
      else { fixed(0, 0., 1., 0., 0.); fixed(1, 0., -1., 1., dy[2] * clo); }
      if (up == 0) { fixed(NY + 1, 0., 1., 0., 0.); fixed(NY, 0., 1., 0., cup); }
      else { fixed(NY, -1., 1., 0., dy[NY] * cup); fixed(NY + 1, 0., 1., 0., 0.); }
    }
  }
}

int dg_cn_tables(dg_handle *h) {
  if (h->periodic) return DG_OK;
  const int L = h->NY + 2;
  if (!h->cn_rows) {
    double *rows = (double *)malloc(sizeof(double) * h->nf * 8 * L);
    cn_row_templates(h, rows);
    DG_CUDA(dg_malloc(h, (void **)&h->cn_rows, sizeof(double) * h->nf * 8 * L));
    cudaError_t e = cudaMemcpyAsync(h->cn_rows, rows, sizeof(double) * h->nf * 8 * L,
                                    cudaMemcpyHostToDevice, h->st);
    free(rows);
    DG_CUDA(e);
  }
  CnRows P;
  P.NY = h->NY; P.nfld = h->nf; P.nu = h->p.nu; P.nuv = h->p.nu_v_scale;
  for (int f = 0; f < 3 + DG_MAX_TH; f++) P.pr[f] = (f >= 3 && f - 3 < h->NTH) ? h->p.pr[f - 3] : 1.0;
  const size_t sm = sizeof(double) * 15 * (size_t)L;
  if (sm > 220 * 1024) {
    dg_set_error("NY too large for the Crank-Nicolson table kernel (NY + 2 <= 1877)");
    return DG_ERR_DIMS;
  }
  if (sm > 48 * 1024) dg_big_smem((const void *)k_cn_tables);
  dg_kt_begin(h, "k_cn_tables", h->st);
  k_cn_tables<<<3 * h->nf, CT_THR, sm, h->st>>>(P, h->dscal, h->cn_rows, h->cn_tab);
  DG_LAUNCHED();
  return DG_OK;
}

int dg_apply_bc_vel_dev(dg_handle *h) {
  BcVel B;
  B.NY = h->NY;
  B.u0 = h->p.u_bc_ymin; B.v0 = h->p.v_bc_ymin; B.w0 = h->p.w_bc_ymin;
  B.u1 = h->p.u_bc_ymax; B.v1 = h->p.v_bc_ymax; B.w1 = h->p.w_bc_ymax;
  B.cu0 = h->p.u_bc_ymin_c1; B.cv0 = h->p.v_bc_ymin_c1; B.cw0 = h->p.w_bc_ymin_c1;
  B.cu1 = h->p.u_bc_ymax_c1; B.cv1 = h->p.v_bc_ymax_c1; B.cw1 = h->p.w_bc_ymax_c1;
  dg_kt_begin(h, "k_bc_vel", h->st);
  k_bc_vel<<<dg_cdiv(h->ss, 128), 128, 0, h->st>>>(B, h->ss, h->dy, h->dyf, h->cu[0], h->cu[1],
                                                   h->cu[2]);
  DG_LAUNCHED();
  return DG_OK;
}

int dg_rem_div_dev(dg_handle *h, int update_cp, int rk_step, bool from_rhs) {
  const int L = h->NY + 2;
  const int nseg = dg_cdiv(h->NY, RD_K);
  // fewer modes per CTA where a tall column needs it
  int mt = h->col_mt;
  while (mt > 2 && ((mt * nseg + 31) / 32 * 32 > RD_MAX_THR || rd_smem(L, nseg, mt) > 220 * 1024))
    mt /= 2;
  const int thr = (mt * nseg + 31) / 32 * 32;
  const size_t sm = rd_smem(L, nseg, mt);
  if (thr > RD_MAX_THR || sm > 220 * 1024) {
    dg_set_error("REM_DIV column kernel: NY too large (NY <= 1016)");
    return DG_ERR_DIMS;
  }
  RdArgs A;
  memset(&A, 0, sizeof(A));
  A.NY = h->NY; A.nkxp = h->nkxp; A.JS = h->jstart; A.JE = h->jend;
  A.rk_step = update_cp ? rk_step : 0;
  A.nseg = nseg;
  A.ss = h->ss;
  A.kxv = h->kx; A.kzv = h->kz; A.dy = h->dy; A.dyf = h->dyf;
  A.ra = h->rem_a; A.rrb = h->rem_rb; A.dscal = h->dscal;
  // from_rhs: the column stage left the post-CN velocity (and the scalars a
  // velocity right-hand side reads) in the rhs arrays
  const double2 *const *src = from_rhs ? h->rhs : h->cu;
  A.s1 = src[0]; A.s2 = src[1]; A.s3 = src[2];
  A.u1 = h->cu[0]; A.u2 = h->cu[1]; A.u3 = h->cu[2];
  A.cp = h->cp; A.phi = h->cr1;
  if (from_rhs)
    for (int n = 0; n < h->NTH; n++)
      if (dg_col_th_to_rhs(h, n)) {
        A.cpy.src[A.cpy.n] = h->rhs[3 + n];
        A.cpy.dst[A.cpy.n] = h->cu[3 + n];
        A.cpy.lo[A.cpy.n] = h->jstart_th[n] - 1;
        A.cpy.n++;
      }
#define RD_CASE(MTV)                                                                          \
  if (mt == MTV) {                                                                            \
    dg_big_smem((const void *)k_rd_col<MTV>);                                                 \
    dg_kt_begin(h, "k_rd_col", h->st);                                                        \
    DG_CUDA(dg_launch(h->pdl && update_cp, k_rd_col<MTV>, dim3(dg_cdiv(h->ss, MTV)),           \
                      dim3(thr), sm, h->st, A));                                              \
  }
  RD_CASE(2) RD_CASE(4) RD_CASE(8) RD_CASE(16)
#undef RD_CASE
  DG_LAUNCHED();
  return DG_OK;
}

static double courant_dt0(const dg_handle *h) {
  // velocity-independent limits of for/courant.f:15-32
  const dg_params &p = h->p;
  double dt = 999.0;
  double dx = p.lx / h->NX;
  double dmin = dx < h->h_dy[1] ? dx : h->h_dy[1];
  double t = 0.5 * (dmin * dmin) / p.nu;
  dt = dt < t ? dt : t;
  for (int n = 0; n < h->NTH; n++) {
    t = dt * p.nu / (p.nu / p.pr[n]);
    dt = dt < t ? dt : t;
  }
  if (p.i_ro != 0.0) {
    t = 2.0 * h->pi / fabs(p.i_ro) / 20.0;
    dt = dt < t ? dt : t;
  }
  for (int n = 0; n < h->NTH; n++)
    if (p.ri[n] != 0.0) {
      double nmax = sqrt(fabs(p.ri[n] * p.th_bc_ymin_c1[n]));
      t = (double)0.1f * 2.0 * h->pi / nmax;  // 0.1 is a default-real literal
      dt = dt < t ? dt : t;
    }
  return dt;
}

// With `side`, the caller joins ev_cfl1 before the commit.
int dg_courant_dev(dg_handle *h, const double2 *const *u, bool side) {
  // physical U1..U3 on planes 1..NY, reduced to COURANT's minimum on the fly.
  // With `side`, all of it (the z inverse into H too) runs on the side
  // stream: it reads only u and writes H, dmin_bits and the parked DELTA_T,
  // so it overlaps REM_DIV on the main stream
  cudaStream_t keep = h->st;
  if (side) {
    DG_CUDA(cudaEventRecord(h->ev_cfl0, h->st));
    DG_CUDA(cudaStreamWaitEvent(h->st2, h->ev_cfl0, 0));
    h->st = h->st2;
  }
  auto run = [&]() -> int {
    h->pdl_zinv = 0;
    DG_TRY(dg_zinv(h, u, 3, 1, h->NY, h->H, 0));
    DG_CUDA(cudaMemsetAsync(h->dmin_bits, 0x7f, sizeof(unsigned long long), h->st));
    DG_TRY(dg_xc2r_cfl(h, h->H, 1, h->NY, h->dmin_bits));
    dg_kt_begin(h, "k_dt_update", h->st);
    k_dt_update<<<1, 1, 0, h->st>>>(h->dscal, h->dmin_bits, courant_dt0(h));
    DG_LAUNCHED();
    return DG_OK;
  };
  const int s = run();
  h->st = keep;
  DG_TRY(s);
  if (side) DG_CUDA(cudaEventRecord(h->ev_cfl1, h->st2));
  return DG_OK;
}

// COURANT on physical U1..U3 that already exist (planes 1..NY at u_plane1,
// u_plane1 + pfield, u_plane1 + 2 pfield; the LES path's post-solve velocity)
int dg_courant_phys(dg_handle *h, const double *u_plane1, long pfield) {
  DG_CUDA(cudaMemsetAsync(h->dmin_bits, 0x7f, sizeof(unsigned long long), h->st));
  dg_kt_begin(h, "k_cfl_min", h->st);
  k_cfl_min<<<4 * 148, 256, 0, h->st>>>(u_plane1, pfield, h->NY, h->NZ, h->NX, h->p.cfl,
                                         h->p.lx / h->NX, h->p.lz / h->NZ, h->dy, h->dmin_bits);
  DG_LAUNCHED();
  dg_kt_begin(h, "k_dt_update", h->st);
  k_dt_update<<<1, 1, 0, h->st>>>(h->dscal, h->dmin_bits, courant_dt0(h));
  DG_LAUNCHED();
  return DG_OK;
}

int dg_dt_commit(dg_handle *h) {
  dg_kt_begin(h, "k_dt_commit", h->st);
  k_dt_commit<<<1, 1, 0, h->st>>>(h->dscal);
  DG_LAUNCHED();
  if (h->defer_tables) return DG_OK;  // the next full step rebuilds them first
  if (h->p.les && h->les_nut) return DG_OK;  // the LES solves build their rows in place
  // the new tables are first needed by the next substep's CN solve: build them
  // on the side stream while the nonlinear terms of that substep run
  DG_CUDA(cudaEventRecord(h->ev_fork, h->st));
  DG_CUDA(cudaStreamWaitEvent(h->st2, h->ev_fork, 0));
  cudaStream_t keep = h->st;
  h->st = h->st2;
  int s = dg_cn_tables(h);
  h->st = keep;
  DG_TRY(s);
  DG_CUDA(cudaEventRecord(h->ev_join, h->st2));
  h->tables_pending = true;
  return DG_OK;
}

int dg_chan_init(dg_handle *h) {
  DG_TRY(dg_col_init(h));
  dg_kt_begin(h, "k_remdiv_init", h->st);
  k_remdiv_init<<<dg_cdiv(h->ss, 128), 128, 0, h->st>>>(h->NY, h->ss, h->nkxp, h->kx, h->kz, h->dy,
                                                        h->dyf, h->rem_a, h->rem_rb);
  DG_LAUNCHED();
  return dg_cn_tables(h);
}

// The mixed form needs a compile-time x length (the warp x-row kernel, or
// the FP32 two-launch stage) and a warp z-forward length.
bool dg_mixed_ok(int nx, int nz, int n_th) {
  (void)n_th;
  return fft_bufs(nx) == 1 && (zw_supported(nz) || zw_big(nz));
}

// Steps 1-3 of a substep in the mixed form: the z inverse converts the FP64
// state to FP32 half-physical planes, the x-row products and both x
// transforms run in FP32, the z forward runs in FP32 and its epilogue (the
// explicit terms, CF and the CN right-hand side) in FP64.
static int nl_chunk_mixed(dg_handle *h, const ChanConst &C, int rk_step, int a, int b, int &hdone,
                          const double2 *const *in, FieldPtrs cu, FieldPtrs cf, FieldPtrs rhs) {
  float2 *Hf = reinterpret_cast<float2 *>(h->H);
  float2 *Gf = reinterpret_cast<float2 *>(h->G);
  const long Hfield = (long)h->nplanes * h->NZ * h->nkxp;
  h->pdl_zinv = h->pdl;  // follows the previous substep's REM_DIV kernel
  const int zs = dg_cinv_gf(h, in, h->nf, hdone + 1, b + 1, h->ss, h->nkxp, h->NZ, h->NKZ, h->plz,
                            h->twz_f, Hf, Hfield);
  h->pdl_zinv = 0;
  DG_TRY(zs);
  hdone = b + 1;
  const int nplan = b - a + 1;
  bool done = false;
#define XW_CASE(NXV, NTHV)                                                                      \
  if (!done && h->NX == NXV && h->NTH == NTHV) {                                                \
    auto kern = xrow_kernel<NXV, NTHV, float2>(h->fft_plan);                                    \
    dg_big_smem((const void *)kern);                                                            \
    int chunk = h->xrow_chunk > 0 ? (h->xrow_chunk < nplan ? h->xrow_chunk : nplan)            \
                                  : xrow_auto_chunk(nplan, h->NZ, (const void *)kern,          \
                                                    xw_smem<NXV, NTHV, float2>());              \
    dim3 grid(dg_cdiv(h->NZ, XW_WARPS), dg_cdiv(nplan, chunk));                                 \
    dg_kt_begin(h, "k_xrow_w_f32", h->st);                                                      \
    DG_CUDA(dg_launch(h->pdl, kern, grid, dim3(32 * XW_WARPS),                                  \
                      xw_smem<NXV, NTHV, float2>(), h->st, C, Hf, Hfield, chunk, a, b,          \
                      h->twx_f, h->dyf, h->dy, h->kx, Gf, Hfield));                             \
    done = true;                                                                                \
  }
#define XW_ALL(NXV) XW_CASE(NXV, 0) XW_CASE(NXV, 1) XW_CASE(NXV, 2)
  XW_ALL(16) XW_ALL(32) XW_ALL(48) XW_ALL(64) XW_ALL(96) XW_ALL(128) XW_ALL(256)
#undef XW_ALL
#undef XW_CASE
  if (!done) {
    dg_set_error("mixed precision: no FP32 x-row kernel for this NX / N_TH");
    return DG_ERR_DIMS;
  }
  DG_LAUNCHED();
  dim3 zgrid(dg_cdiv(h->nkxp, zw_kxg(h->NZ)), nplan, h->nf);
  const size_t sm = zw_smem<float2>(h->NZ);
  done = false;
#define ZW_CASE(N)                                                                              \
  if (!done && h->NZ == N) {                                                                    \
    auto kern = h->zf_nlo ? zfwd_kernel<N, float2, true>(h->fft_plan)                           \
                          : zfwd_kernel<N, float2, false>(h->fft_plan);                         \
    dg_big_smem((const void *)kern);                                                            \
    dg_kt_begin(h, "k_zfwd_w_f32", h->st);                                                      \
    DG_CUDA(dg_launch(h->pdl, kern, zgrid, dim3(128), sm, h->st, C, Gf, Hfield,                 \
                      h->twz_f, h->dscal, rk_step, h->kx, h->kz, h->dy, h->dyf, cu, cf, rhs,    \
                      h->cp, a));                                                               \
    done = true;                                                                                \
  }
  ZW_CASE(16) ZW_CASE(32) ZW_CASE(48) ZW_CASE(64) ZW_CASE(96) ZW_CASE(128) ZW_CASE(192)
  ZW_CASE(256) ZW_CASE(384) ZW_CASE(512)
#undef ZW_CASE
  if (!done) {
    dg_set_error("mixed precision: no FP32 z-forward kernel for this NZ");
    return DG_ERR_DIMS;
  }
  DG_LAUNCHED();
  return DG_OK;
}

// Steps 1-3 in the mixed form for x lengths without an FP32 warp x-row
// kernel (or N_TH > 2): all planes at once through k_xc2r_f and k_xprod_f,
// then the FP32 warp z-forward with its FP64 epilogue.
static int nl_generic_mixed(dg_handle *h, const ChanConst &C, int rk_step,
                            const double2 *const *in, FieldPtrs cu, FieldPtrs cf, FieldPtrs rhs) {
  float2 *Hf = reinterpret_cast<float2 *>(h->H);
  float2 *Gf = reinterpret_cast<float2 *>(h->G);
  const long Hfield = (long)h->nplanes * h->NZ * h->nkxp;
  const int NX = h->NX, NY = h->NY, NZ = h->NZ;
  h->pdl_zinv = h->pdl;
  const int zs = dg_cinv_gf(h, in, h->nf, 0, NY + 1, h->ss, h->nkxp, NZ, h->NKZ, h->plz, h->twz_f,
                            Hf, Hfield);
  h->pdl_zinv = 0;
  DG_TRY(zs);
  // work: FP32 fluctuation rows [nf][NY+2][NZ][NX], then FP64 row means [nf][NY+2][NZ]
  const long pplane = (long)NZ * NX, pfield = (long)(NY + 2) * pplane;
  float *phys = reinterpret_cast<float *>(h->work);
  double *dc = reinterpret_cast<double *>(phys + h->nf * pfield);
  const long dfield = (long)(NY + 2) * NZ;
  bool done = false;
  {
    dim3 grid(dg_cdiv(NZ, 8), NY + 2, h->nf);
    const size_t sm = sizeof(float2) * (NX + 4 * (size_t)padded_len(NX));
#define XC_CASE(N)                                                                              \
  if (!done && NX == N) {                                                                       \
    dg_big_smem((const void *)k_xc2r_f<N>);                                                     \
    dg_kt_begin(h, "k_xc2r_f32", h->st);                                                        \
    DG_CUDA(dg_launch(h->pdl, k_xc2r_f<N>, grid, dim3(128), sm, h->st, Hf, Hfield, NZ, h->nkxp, \
                      h->twx_f, phys, pfield, dc, dfield));                                     \
    done = true;                                                                                \
  }
    DG_FOR_EACH_N(XC_CASE)
#undef XC_CASE
  }
  if (!done) {
    dg_set_error("mixed precision: no FP32 x-row kernel for this NX");
    return DG_ERR_DIMS;
  }
  DG_LAUNCHED();
  done = false;
  {
    dim3 grid(xp_pairs(h->NTH), dg_cdiv(NZ, XP_THR / 32), NY);
    const size_t sm = sizeof(float2) * (NX + (XP_THR / 32) * (size_t)padded_len(NX));
#define XP_CASE(N)                                                                              \
  if (!done && NX == N) {                                                                       \
    dg_big_smem((const void *)k_xprod_f<N>);                                                    \
    dg_kt_begin(h, "k_xprod_f32", h->st);                                                       \
    DG_CUDA(dg_launch(h->pdl, k_xprod_f<N>, grid, dim3(XP_THR), sm, h->st, C, phys, pfield, dc, \
                      dfield, h->twx_f, h->dyf, h->dy, h->kx, Gf, Hfield));                     \
    done = true;                                                                                \
  }
    DG_FOR_EACH_N(XP_CASE)
#undef XP_CASE
  }
  DG_LAUNCHED();
  done = false;
  dim3 zgrid(dg_cdiv(h->nkxp, zw_kxg(NZ)), NY, h->nf);
  const size_t sm = zw_smem<float2>(NZ);
#define ZW_CASE(N)                                                                              \
  if (!done && NZ == N) {                                                                       \
    auto kern = h->zf_nlo ? zfwd_kernel<N, float2, true>(h->fft_plan)                           \
                          : zfwd_kernel<N, float2, false>(h->fft_plan);                         \
    dg_big_smem((const void *)kern);                                                            \
    dg_kt_begin(h, "k_zfwd_w_f32", h->st);                                                      \
    DG_CUDA(dg_launch(h->pdl, kern, zgrid, dim3(128), sm, h->st, C, Gf, Hfield,                 \
                      h->twz_f, h->dscal, rk_step, h->kx, h->kz, h->dy, h->dyf, cu, cf, rhs,    \
                      h->cp, 1));                                                               \
    done = true;                                                                                \
  }
  ZW_CASE(16) ZW_CASE(32) ZW_CASE(48) ZW_CASE(64) ZW_CASE(96) ZW_CASE(128) ZW_CASE(192)
  ZW_CASE(256) ZW_CASE(384) ZW_CASE(512)
#undef ZW_CASE
  if (!done) {
    dg_set_error("mixed precision: no FP32 z-forward kernel for this NZ");
    return DG_ERR_DIMS;
  }
  DG_LAUNCHED();
  return DG_OK;
}

// Steps 1-3 of RK_CHAN_1 (and, with LES, the subgrid model and the LES
// solves): everything before the per-mode column stage.  *column_next says
// whether the column stage (dg_chan_column) must follow; LES substeps finish
// here.
int dg_chan_nonlinear(dg_handle *h, int time_step, int rk_step, bool *column_next) {
  *column_next = false;
  const ChanConst C = make_const(h);
  // Steps 1-3 run over y-chunks of planes so the half-physical (H) and
  // product (G) planes a chunk produces are consumed while still in L2.
  const double2 *in[3 + DG_MAX_TH];
  for (int f = 0; f < h->nf; f++) in[f] = h->cu[f];
  const long Hfield = (long)h->nplanes * h->NZ * h->nkxp;
  // planes per y-chunk (tunable DG_TUNE_YCHUNK; 0 = all planes in one chunk,
  // the measured default on B200 for the grids benchmarked)
  int cj = h->NY;
  if (h->ychunk >= 4 && h->ychunk < h->NY) cj = h->ychunk;
  FieldPtrs cu, cf, rhs;
  for (int f = 0; f < h->nf; f++) { cu.p[f] = h->cu[f]; cf.p[f] = h->cf[f]; rhs.p[f] = h->rhs[f]; }
  int hdone = -1;  // last H plane already produced
  int a0 = 1;
  // LES: the subgrid model wraps the nonlinear stage; once NU_T exists the
  // Crank-Nicolson solves run on physical columns (for/channel.f:303,631)
  const bool sgs = dg_les_active(h, time_step);
  const bool les_solve = h->p.les && (sgs || h->les_nut);
  // the z forward writes only the nonlinear terms unless the LES solves need
  // the assembled right-hand side R and CF from it
  h->zf_nlo = les_solve ? 0 : 1;
  if (sgs) DG_TRY(dg_les_pre(h, rk_step));
  if (h->mixed && !(xw_supported(h->NX) && h->NTH <= 2)) {
    DG_TRY(nl_generic_mixed(h, C, rk_step, in, cu, cf, rhs));
    a0 = h->NY + 1;  // every plane done: no chunk loop
  }
  for (int a = a0; a <= h->NY; a += cj) {
    const int b = (a + cj - 1 < h->NY) ? a + cj - 1 : h->NY;
    if (h->mixed) {
      DG_TRY(nl_chunk_mixed(h, C, rk_step, a, b, hdone, in, cu, cf, rhs));
      continue;
    }
    // 1. z inverse of the planes this chunk's x-rows need (a-1 .. b+1)
    h->pdl_zinv = h->pdl;
    const int zs = dg_zinv(h, in, h->nf, hdone + 1, b + 1, h->H, 0);
    h->pdl_zinv = 0;
    DG_TRY(zs);
    hdone = b + 1;
    // 2. x-row nonlinear products for output planes a..b
    bool done = false;
    if (xw_supported(h->NX) && h->NTH <= 2) {
      const int nplan = b - a + 1;
      // planes marched by one CTA (tunable DG_TUNE_XROW_CHUNK; 0 = the one-wave
      // choice of xrow_auto_chunk)
#define XW_CASE(NXV, NTHV)                                                                         \
  if (h->NX == NXV && h->NTH == NTHV) {                                                          \
    auto kern = xrow_kernel<NXV, NTHV, double2>(h->fft_plan);                                    \
    dg_big_smem((const void *)kern);                                                             \
    int chunk = h->xrow_chunk > 0 ? (h->xrow_chunk < nplan ? h->xrow_chunk : nplan)             \
                                  : xrow_auto_chunk(nplan, h->NZ, (const void *)kern,           \
                                                    xw_smem<NXV, NTHV>());                       \
    dim3 grid(dg_cdiv(h->NZ, XW_WARPS), dg_cdiv(nplan, chunk));                                  \
    dg_kt_begin(h, "k_xrow_w", h->st);                                                             \
    DG_CUDA(dg_launch(h->pdl, kern, grid, dim3(32 * XW_WARPS),                                   \
                      xw_smem<NXV, NTHV>(), h->st, C, h->H, Hfield, chunk, a, b, h->twx,        \
                      h->dyf, h->dy, h->kx, h->G, Hfield));                                     \
    done = true;                                                                                 \
  }
#define XW_ALL(NXV) XW_CASE(NXV, 0) XW_CASE(NXV, 1) XW_CASE(NXV, 2)
      XW_ALL(16) XW_ALL(32) XW_ALL(48) XW_ALL(64) XW_ALL(96) XW_ALL(128) XW_ALL(256)
#undef XW_ALL
#undef XW_CASE
      if (done) DG_LAUNCHED();
    }
    if (!done) {
      // generic CTA kernel covers all planes 1..NY in one launch
      if (a == 1) {
        DG_TRY(dg_zinv(h, in, h->nf, hdone + 1, h->NY + 1, h->H, 0));
        hdone = h->NY + 1;
        // every plane to physical space (the work array holds nf stacks of
        // NY+2 planes), then the products of planes 1..NY
        const long pplane = (long)h->NZ * h->NX, pfield = (long)(h->NY + 2) * pplane;
        double *phys = (double *)h->work;
        DG_TRY(dg_xc2r_planes(h, h->H, h->nf, 0, h->NY + 1, phys, pplane, h->NX, pfield));
        const int rz = xp_rows(h->NX);
        dim3 grid(xp_pairs(h->NTH), dg_cdiv(h->NZ, rz), h->NY);
        const size_t sm = xp_smem(h->NX, rz);
#define KERNEL_BODY(N)                                                                          \
  dg_big_smem((const void *)k_xprod<N>);                                                        \
  dg_kt_begin(h, "k_xprod", h->st);                                                             \
  k_xprod<N><<<grid, XP_THR, sm, h->st>>>(C, phys, pfield, rz, h->plx, h->twx, h->dyf, h->dy,   \
                                          h->kx, h->G, Hfield)
        switch (h->NX) {
          DG_FOR_EACH_N(DG_CASE_N)
          default: KERNEL_BODY(0); break;
        }
#undef KERNEL_BODY
        DG_LAUNCHED();
      }
    }
    // 3. z forward, explicit terms, CN right-hand side for planes a..b (all
    //    planes 1..NY after the generic x-row stage)
    const int za = done ? a : 1, zb = done ? b : h->NY;
    bool zdone = false;
    if (zw_supported(h->NZ) || zw_big(h->NZ)) {
      dim3 grid(dg_cdiv(h->nkxp, zw_kxg(h->NZ)), zb - za + 1, h->nf);
      const size_t sm = zw_smem<double2>(h->NZ);
#define ZW_CASE(N)                                                                             \
  if (h->NZ == N) {                                                                            \
    auto kern = h->zf_nlo ? zfwd_kernel<N, double2, true>(h->fft_plan)                         \
                          : zfwd_kernel<N, double2, false>(h->fft_plan);                       \
    dg_big_smem((const void *)kern);                                                           \
    dg_kt_begin(h, "k_zfwd_w", h->st);                                                          \
    DG_CUDA(dg_launch(h->pdl, kern, grid, dim3(128), sm, h->st, C, h->G, Hfield, h->twz,       \
                      h->dscal, rk_step, h->kx, h->kz, h->dy, h->dyf, cu, cf, rhs, h->cp, za)); \
    zdone = true;                                                                              \
  }
      ZW_CASE(16) ZW_CASE(32) ZW_CASE(48) ZW_CASE(64) ZW_CASE(96) ZW_CASE(128) ZW_CASE(192)
      ZW_CASE(256) ZW_CASE(384) ZW_CASE(512)
#undef ZW_CASE
      if (zdone) DG_LAUNCHED();
    }
    // generic path: one launch over all planes after all products exist
    if (!zdone && (!done || b == h->NY)) {
      dim3 grid(dg_cdiv(h->nkxp, zf_kxg(h->NZ)), h->NY);
      const size_t sm = zfwd_smem(h);
#define KERNEL_BODY(N)                                                                          \
  {                                                                                             \
    auto kern = h->zf_nlo ? k_zfwd_rhs<N, true> : k_zfwd_rhs<N, false>;                         \
    dg_big_smem((const void *)kern);                                                            \
    dg_kt_begin(h, "k_zfwd_rhs", h->st);                                                        \
    kern<<<grid, ZF_THR, sm, h->st>>>(C, h->G, Hfield, h->plz, h->twz, h->dscal, rk_step,       \
                                      h->kx, h->kz, h->dy, h->dyf, cu, cf, rhs, h->cp);         \
  }
      switch (h->NZ) {
        DG_FOR_EACH_N(DG_CASE_N)
        default: KERNEL_BODY(0); break;
      }
#undef KERNEL_BODY
      DG_LAUNCHED();
    }
    if (!done) break;  // the generic kernels covered every plane
  }
  if (les_solve) return dg_les_post(h, time_step, rk_step, sgs);
  *column_next = true;
  return DG_OK;
}

// COURANT runs in substep 3 at the UPDATE_DT cadence with variable DELTA_T
bool dg_chan_cfl(const dg_handle *h, int time_step, int rk_step) {
  return h->p.variable_dt && rk_step == 3 && h->p.update_dt > 0 &&
         (time_step % h->p.update_dt) == 0;
}

// After the column stage of a substep that runs COURANT: COURANT on the
// post-CN velocity (for/channel.f:1037-1040) on the side stream, REM_DIV_CHAN
// and CP += phi / H_BAR on the main stream meanwhile, then the new DELTA_T
// is committed.
int dg_chan_cfl_tail(dg_handle *h, int rk_step) {
  // the column stage left the post-CN velocity in the rhs arrays
  const double2 *u[3] = {h->rhs[0], h->rhs[1], h->rhs[2]};
  DG_TRY(dg_courant_dev(h, u, true));
  DG_TRY(dg_rem_div_dev(h, 1, rk_step, true));
  DG_CUDA(cudaStreamWaitEvent(h->st, h->ev_cfl1, 0));
  return dg_dt_commit(h);
}

extern "C" int diablo_rk_chan_1(dg_handle *h, int time_step, int rk_step) {
  if (!h || h->periodic || rk_step < 1 || rk_step > 3) return DG_ERR_ARG;
  bool column = false;
  DG_TRY(dg_chan_nonlinear(h, time_step, rk_step, &column));
  if (!column) return DG_OK;
  // 4. per-mode column stage: explicit terms, right-hand sides and CN solves
  //    (k_col_cn), then REM_DIV_CHAN and CP += phi / H_BAR (k_rd_col); with
  //    COURANT the tail above runs between them
  const bool cfl = dg_chan_cfl(h, time_step, rk_step);
  DG_TRY(dg_col_step_dev(h, rk_step, !cfl));
  if (cfl) DG_TRY(dg_chan_cfl_tail(h, rk_step));
  return DG_OK;
}

extern "C" int diablo_rem_div_chan(dg_handle *h) {
  if (!h || h->periodic) return DG_ERR_ARG;
  return dg_rem_div_dev(h, 0, 0, false);
}

extern "C" int diablo_apply_bc_vel(dg_handle *h) {
  if (!h || h->periodic) return DG_ERR_ARG;
  return dg_apply_bc_vel_dev(h);
}

extern "C" int diablo_courant(dg_handle *h) {
  if (!h || h->periodic) return DG_ERR_ARG;
  const double2 *u[3] = {h->cu[0], h->cu[1], h->cu[2]};
  DG_TRY(dg_courant_dev(h, u));
  return dg_dt_commit(h);
}

int dg_stats_dev(dg_handle *h, dg_stats *s) {
  if (h->periodic) return dg_per_stats(h, s);
  const int NP = h->nplanes;
  double *dsum = (double *)h->work;
  CFieldPtrs u;
  for (int f = 0; f < h->nf; f++) u.p[f] = h->cu[f];
  DG_CUDA(cudaMemsetAsync(h->dflag, 0, sizeof(int), h->st));
  dg_kt_begin(h, "k_stats_planes", h->st);
  k_stats_planes<<<NP, 256, 0, h->st>>>(NP, h->ss, h->nkxp, u, h->nf, dsum, h->dflag);
  DG_LAUNCHED();
  double *hs = (double *)malloc(sizeof(double) * 8 * NP);
  int flag = 0;
  cudaError_t e1 = cudaMemcpyAsync(hs, dsum, sizeof(double) * 8 * NP, cudaMemcpyDeviceToHost, h->st);
  cudaError_t e2 = cudaMemcpyAsync(&flag, h->dflag, sizeof(int), cudaMemcpyDeviceToHost, h->st);
  cudaError_t e3 = cudaStreamSynchronize(h->st);
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
    free(hs);
    dg_set_error("stats copy failed");
    return DG_ERR_CUDA;
  }
  memset(s, 0, sizeof(*s));
  if (h->periodic) {
    free(hs);
    return DG_ERR_ARG;
  }
  const int NY = h->NY;
  const double *DY = h->h_dy;
  auto integ = [&](const double *v) {
    double r = 0.;
    for (int j = 2; j <= NY; j++) r = r + 0.5 * (v[j] + v[j - 1]) * DY[j];
    return r / h->p.ly;
  };
  double *ume = (double *)calloc(NY + 2, sizeof(double));
  double *tmp = (double *)calloc(4 * (NY + 2), sizeof(double));
  double *urms = tmp, *vrms = tmp + (NY + 2), *wrms = tmp + 2 * (NY + 2), *ke = tmp + 3 * (NY + 2);
  // the mean U1 of every plane: one strided copy on the handle's stream
  double2 *c0 = (double2 *)malloc(sizeof(double2) * (NY + 2));
  cudaError_t ce = cudaMemcpy2DAsync(c0, sizeof(double2), h->cu[0], sizeof(double2) * h->ss,
                                     sizeof(double2), NY + 2, cudaMemcpyDeviceToHost, h->st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->st);
  for (int j = 0; j <= NY + 1; j++) ume[j] = (ce == cudaSuccess) ? c0[j].x : 0.0;
  free(c0);
  if (ce != cudaSuccess) {
    free(ume);
    free(tmp);
    free(hs);
    DG_CUDA(ce);
  }
  s->ubulk = integ(ume);
  for (int j = 1; j <= NY; j++) {
    const double *a = hs + 8 * j, *b = hs + 8 * (j + 1);
    urms[j] = sqrt(a[0]);
    vrms[j] = sqrt(0.5 * (a[1] + b[1]));
    wrms[j] = sqrt(a[2]);
    ke[j] = 0.5 * (a[3] + 0.5 * (a[4] + b[4]));
  }
  s->urms_b = integ(urms);
  s->vrms_b = integ(vrms);
  s->wrms_b = integ(wrms);
  s->ke = integ(ke);
  for (int n = 0; n < h->NTH && n < 3; n++) {
    for (int j = 1; j <= NY; j++) {
      urms[j] = sqrt(hs[8 * j + 5 + n]);
      vrms[j] = hs[8 * j + 5 + n];
    }
    s->thrms_b[n] = integ(urms);
    s->th_var[n] = integ(vrms);
  }
  free(ume);
  free(tmp);
  free(hs);
  // max |div u| on rows 2..NY-1 in physical space
  double2 *dspec = h->rhs[0];
  dg_kt_begin(h, "k_div_spec", h->st);
  k_div_spec<<<dg_cdiv((long)(NY + 2) * h->ss, 256), 256, 0, h->st>>>(
      NY, h->ss, h->nkxp, h->kx, h->kz, h->dyf, h->cu[0], h->cu[1], h->cu[2], dspec);
  DG_LAUNCHED();
  const double2 *dd[1] = {dspec};
  DG_TRY(dg_zinv(h, dd, 1, 2, NY - 1, h->H, 0));
  const long pplane = (long)h->NZ * h->NX;
  double *phys = (double *)h->work;
  DG_TRY(dg_xc2r_planes(h, h->H, 1, 2, NY - 1, phys - 2 * pplane, pplane, h->NX, 0));
  DG_CUDA(cudaMemsetAsync(h->dmin_bits, 0, sizeof(unsigned long long), h->st));
  dg_kt_begin(h, "k_absmax", h->st);
  k_absmax<<<4 * 148, 256, 0, h->st>>>(phys, (long)(NY - 2) * pplane, h->dmin_bits);
  DG_LAUNCHED();
  unsigned long long bits = 0;
  DG_CUDA(cudaMemcpyAsync(&bits, h->dmin_bits, sizeof(bits), cudaMemcpyDeviceToHost, h->st));
  DG_CUDA(cudaStreamSynchronize(h->st));
  double dmax;
  memcpy(&dmax, &bits, sizeof(double));
  s->div_max = dmax;
  return flag ? DG_ERR_NAN : DG_OK;
}
