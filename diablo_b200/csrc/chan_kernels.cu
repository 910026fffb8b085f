// Channel substep kernels (RK_CHAN_1, for/channel.f:62-1073) on the
// retained-mode layout [j][kz][kx].
//
// One substep is five launches:
//   zinv        spectral U1..U3, TH -> half-physical H (z inverse per kx)
//   k_xrow_nl   per physical z-row, marching up in y: x c2r of every field,
//               all products/fluxes of for/channel.f:409-571,665-720, x r2c,
//               and the combination into 2 arrays per field
//               (A: to be multiplied by -i kz, B: the rest)
//   k_zfwd_rhs  per plane: z forward of A/B, nonlinear + explicit linear
//               terms -> CF (new), and the Crank-Nicolson right-hand side
//               R = CU + zeta h CF_old - h grad P + beta h CF_new
//                   + (nu h / 2) d2/dy2 CU           (for/channel.f:88-626)
//   k_cn_solve  per (mode, field): tridiagonal CN solve in Fourier space
//               (the reference solves the same x-z independent operator per
//               physical column, for/channel.f:767-1029; the operator is linear
//               and identical for every column, so it commutes with the FFT)
//   k_remdiv    per mode: REM_DIV_CHAN's complex tridiagonal, projection and
//               CP += phi / h (for/channel.f:1103-1214, 1059-1065)
#include <math.h>
#include "dg_internal.cuh"
#include "fft.cuh"

using namespace dgfft;

namespace {

constexpr int XR_ROWS = 2;     // physical z-rows per CTA in k_xrow_nl
constexpr int ZF_KXG = 4;      // kx columns per CTA in k_zfwd_rhs

struct ChanConst {
  int NX, NY, NZ, NKX, NKZ, nkxp, nkzt, nf, nth;
  long ss;
  int JS, JE, JSt[DG_MAX_TH], JEt[DG_MAX_TH];
  double nu, beta, nuv, i_ro, grav_x, grav_y, grav_z, px0, omega0, amp_omega0;
  int f_type;
  double ri[DG_MAX_TH], pr[DG_MAX_TH], drhodx[DG_MAX_TH], drhodz[DG_MAX_TH];
};

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
// The y-flux terms of for/channel.f:511-571,704-720 are differences of these
// fluxes between neighbouring planes; they are differenced after the x
// transform (linearity), so each flux is transformed once.
__global__ void __launch_bounds__(256) k_xrow_nl(
    ChanConst C, const double2 *__restrict__ H, long Hfield, int chunk, FftPlan pl,
    const double2 *__restrict__ tw, const double *__restrict__ dyf, const double *__restrict__ dy,
    const double *__restrict__ kxv, double2 *__restrict__ G, long Gfield) {
  extern __shared__ double2 sm[];
  const int NX = C.NX, nkxp = C.nkxp, nf = C.nf, nth = C.nth;
  const int npin = (nf + 1) / 2;            // c2r signals per row
  const int nprod = 8 + 3 * nth;
  const int npp = (nprod + 1) / 2;          // r2c signals per row
  const int maxp = npin > npp ? npin : npp;
  const int sstr = NX + 1;
  double2 *stw = sm;
  double2 *b0 = stw + NX;
  double2 *b1 = b0 + XR_ROWS * maxp * sstr;
  double2 *prev = b1 + XR_ROWS * maxp * sstr;               // [row][3+nth][nkxp]
  double *ring = (double *)(prev + XR_ROWS * (3 + nth) * nkxp);  // [3][row][nf][NX]
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int z0 = blockIdx.x * XR_ROWS;
  const int j0 = 1 + blockIdx.y * chunk;
  int j1 = j0 + chunk - 1;
  if (j1 > C.NY) j1 = C.NY;
  const int NZ = C.NZ;

  for (int i = tid; i < NX; i += nthr) stw[i] = tw[i];
  // plane j0-2 may be -1: zero the whole ring once
  for (int i = tid; i < 3 * XR_ROWS * nf * NX; i += nthr) ring[i] = 0.0;
  __syncthreads();

  auto ringp = [&](int plane, int r, int f) -> double * {
    int s = (plane + 3) % 3;
    return ring + (((long)s * XR_ROWS + r) * nf + f) * NX;
  };

  // load + c2r of one plane into its ring slot
  auto load_plane = [&](int plane) {
    for (int idx = tid; idx < XR_ROWS * npin * NX; idx += nthr) {
      const int k = idx % NX;
      const int q = (idx / NX) % npin;
      const int r = idx / (NX * npin);
      const int z = z0 + r;
      const int fa = 2 * q, fb = 2 * q + 1;
      const int kk = (k <= NX / 2) ? k : NX - k;
      double2 v = make_double2(0.0, 0.0);
      if (z < NZ && kk <= C.NKX && kk < NX / 2) {
        const long off = (long)plane * NZ * nkxp + (long)z * nkxp + kk;
        double2 a = H[fa * Hfield + off];
        double2 b = (fb < nf) ? H[fb * Hfield + off] : make_double2(0.0, 0.0);
        if (kk == 0) { a.y = 0.0; b.y = 0.0; }
        v = (k == kk) ? make_double2(a.x - b.y, a.y + b.x) : make_double2(a.x + b.y, -a.y + b.x);
      }
      b0[(r * maxp + q) * sstr + k] = v;
    }
    __syncthreads();
    double2 *res = run(b0, b1, pl, XR_ROWS * maxp, sstr, stw, +1);
    for (int idx = tid; idx < XR_ROWS * npin * NX; idx += nthr) {
      const int x = idx % NX;
      const int q = (idx / NX) % npin;
      const int r = idx / (NX * npin);
      const double2 v = res[(r * maxp + q) * sstr + x];
      ringp(plane, r, 2 * q)[x] = v.x;
      if (2 * q + 1 < nf) ringp(plane, r, 2 * q + 1)[x] = v.y;
    }
    __syncthreads();
  };

  if (j0 - 2 >= 0) load_plane(j0 - 2);
  load_plane(j0 - 1);

  for (int j = j0 - 1; j <= j1; j++) {
    load_plane(j + 1);
    // products of plane j into complex pairs
    const double dyfj = (j >= 1) ? dyf[j] : 0.0, dyfm = (j >= 1) ? dyf[j - 1] : 0.0;
    const double dyj = (j >= 1) ? dy[j] : 1.0;
    for (int idx = tid; idx < XR_ROWS * npp * NX; idx += nthr) {
      const int x = idx % NX;
      const int q = (idx / NX) % npp;
      const int r = idx / (NX * npp);
      double pv[2];
#pragma unroll
      for (int h2 = 0; h2 < 2; h2++) {
        const int p = 2 * q + h2;
        double v = 0.0;
        if (p < nprod) {
          const double *U1c = ringp(j, r, 0), *U2c = ringp(j, r, 1), *U3c = ringp(j, r, 2);
          const double *U1p = ringp(j + 1, r, 0), *U2p = ringp(j + 1, r, 1), *U3p = ringp(j + 1, r, 2);
          const double *U1m = ringp(j - 1, r, 0), *U3m = ringp(j - 1, r, 2);
          switch (p) {
            case 0: v = U3c[x] * U1c[x]; break;
            case 1: v = U1c[x] * U1c[x]; break;
            case 2: v = U3c[x] * U3c[x]; break;
            case 3: { double s = U2c[x] + U2p[x]; v = 0.25 * (s * s); } break;
            case 4: v = (U1p[x] + U1c[x]) * U2p[x]; break;
            case 5: v = (U3p[x] + U3c[x]) * U2p[x]; break;
            case 6: v = ((dyfj * U1c[x] + dyfm * U1m[x]) / (2. * dyj)) * U2c[x]; break;
            case 7: v = ((dyfj * U3c[x] + dyfm * U3m[x]) / (2. * dyj)) * U2c[x]; break;
            default: {
              const int n = (p - 8) / 3, w = (p - 8) % 3;
              const double *Tc = ringp(j, r, 3 + n), *Tp = ringp(j + 1, r, 3 + n);
              if (w == 0) v = Tc[x] * U1c[x];
              else if (w == 1) v = Tc[x] * U3c[x];
              else v = (Tp[x] + Tc[x]) * U2p[x];
            }
          }
        }
        pv[h2] = v;
      }
      b0[(r * maxp + q) * sstr + x] = make_double2(pv[0], pv[1]);
    }
    __syncthreads();
    double2 *res = run(b0, b1, pl, XR_ROWS * maxp, sstr, stw, -1);
    // separate, scale by 1/NX, combine, write
    const double rnx = (double)NX;
    const bool out = (j >= j0);
    for (int idx = tid; idx < XR_ROWS * nkxp; idx += nthr) {
      const int k = idx % nkxp;
      const int r = idx / nkxp;
      const int z = z0 + r;
      if (z >= NZ) continue;
      auto X = [&](int p) -> double2 {
        const int q = p >> 1;
        const double2 zk = res[(r * maxp + q) * sstr + k];
        const double2 zm = res[(r * maxp + q) * sstr + ((NX - k) % NX)];
        double2 v;
        if ((p & 1) == 0) v = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
        else v = make_double2(0.5 * (zk.y + zm.y), -0.5 * (zk.x - zm.x));
        return make_double2(v.x / rnx, v.y / rnx);
      };
      double2 *pv = prev + (r * (3 + nth)) * nkxp;  // [0]=fl1 [1]=fl3 [2]=g [3+n]=flth
      const double KX = kxv[k];
      auto mikx = [&](double2 a) { return make_double2(KX * a.y, -KX * a.x); };  // -i kx a
      const double2 x3 = X(3), x4 = X(4), x5 = X(5);
      if (out) {
        const long off = (long)j * NZ * nkxp + (long)z * nkxp + k;
        const double2 x0 = X(0), x1 = X(1), x2 = X(2), x6 = X(6), x7 = X(7);
        const double2 f1p = pv[0 * nkxp + k], f3p = pv[1 * nkxp + k], gp = pv[2 * nkxp + k];
        const double d2 = 2.0 * dyfj;
        // U1: A = U1U3, B = -ikx U1U1 - (fl1(j+1) - fl1(j)) / (2 DYF)
        G[0 * Gfield + off] = x0;
        double2 t = mikx(x1);
        G[1 * Gfield + off] = make_double2(t.x - (x4.x - f1p.x) / d2, t.y - (x4.y - f1p.y) / d2);
        // U2: A = Ubar3 U2, B = -ikx Ubar1 U2 - (g(j) - g(j-1)) / DY
        G[2 * Gfield + off] = x7;
        t = mikx(x6);
        G[3 * Gfield + off] = make_double2(t.x - (x3.x - gp.x) / dyj, t.y - (x3.y - gp.y) / dyj);
        // U3: A = U3U3, B = -ikx U1U3 - (fl3(j+1) - fl3(j)) / (2 DYF)
        G[4 * Gfield + off] = x2;
        t = mikx(x0);
        G[5 * Gfield + off] = make_double2(t.x - (x5.x - f3p.x) / d2, t.y - (x5.y - f3p.y) / d2);
        for (int n = 0; n < nth; n++) {
          const double2 a = X(8 + 3 * n), b = X(9 + 3 * n), c = X(10 + 3 * n);
          const double2 fp = pv[(3 + n) * nkxp + k];
          G[(6 + 2 * n) * Gfield + off] = b;
          t = mikx(a);
          G[(7 + 2 * n) * Gfield + off] = make_double2(t.x - (c.x - fp.x) / d2, t.y - (c.y - fp.y) / d2);
        }
      }
      pv[0 * nkxp + k] = x4;
      pv[1 * nkxp + k] = x5;
      pv[2 * nkxp + k] = x3;
      for (int n = 0; n < nth; n++) pv[(3 + n) * nkxp + k] = X(10 + 3 * n);
    }
    __syncthreads();
  }
}

size_t xrow_smem(const dg_handle *h) {
  const int nf = h->nf, nth = h->NTH, NX = h->NX;
  const int npin = (nf + 1) / 2, npp = (8 + 3 * nth + 1) / 2;
  const int maxp = npin > npp ? npin : npp;
  return sizeof(double2) * (NX + 2 * XR_ROWS * maxp * (NX + 1) + XR_ROWS * (3 + nth) * h->nkxp) +
         sizeof(double) * 3 * XR_ROWS * nf * NX;
}

// ------------------------------------------------------------- zfwd + rhs
__global__ void __launch_bounds__(256) k_zfwd_rhs(
    ChanConst C, const double2 *__restrict__ G, long Gfield, FftPlan pl,
    const double2 *__restrict__ tw, const double *__restrict__ dscal, int rk_step,
    const double *__restrict__ kxv, const double *__restrict__ kzv, const double *__restrict__ dy,
    const double *__restrict__ dyf, FieldPtrs cu, FieldPtrs cf, FieldPtrs rhs,
    const double2 *__restrict__ cp) {
  extern __shared__ double2 sm[];
  const int NZ = C.NZ, nkxp = C.nkxp, nkzt = C.nkzt, nf = C.nf, NKZ = C.NKZ;
  const int sstr = NZ + 1;
  double2 *stw = sm;
  double2 *b0 = stw + NZ;
  double2 *b1 = b0 + 2 * ZF_KXG * sstr;
  double2 *nl = b1 + 2 * ZF_KXG * sstr;  // [f][c][kp]
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
      b0[(ab * ZF_KXG + c) * sstr + z] = v;
    }
    __syncthreads();
    double2 *res = run(b0, b1, pl, 2 * ZF_KXG, sstr, stw, -1);
    for (int idx = tid; idx < ZF_KXG * nkzt; idx += nthr) {
      const int c = idx % ZF_KXG, kp = idx / ZF_KXG;
      const int z = (kp <= NKZ) ? kp : (NZ - 1 + (kp - NKZ) - NKZ);
      double2 a = res[(0 * ZF_KXG + c) * sstr + z];
      double2 b = res[(1 * ZF_KXG + c) * sstr + z];
      a = make_double2(a.x / rnz, a.y / rnz);
      b = make_double2(b.x / rnz, b.y / rnz);
      const double KZ = kzv[kp];
      // -i kz a + b
      nl[(f * ZF_KXG + c) * nkzt + kp] = make_double2(KZ * a.y + b.x, -KZ * a.x + b.y);
    }
    __syncthreads();
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
    const double2 u1 = cu.p[0][o], u2 = cu.p[1][o], u3 = cu.p[2][o];
    const double2 p0 = cp[o];
    // ---- U1 and U3 (rows JSTART..JEND)
    if (j >= C.JS && j <= C.JE) {
      const double2 u1m = cu.p[0][o - ss], u1p = cu.p[0][o + ss];
      const double2 u3m = cu.p[2][o - ss], u3p = cu.p[2][o + ss];
      double2 f1 = make_double2(-NU * kk * u1.x + C.i_ro * u3.x, -NU * kk * u1.y + C.i_ro * u3.y);
      double2 f3 = make_double2(-NU * kk * u3.x - C.i_ro * u1.x, -NU * kk * u3.y - C.i_ro * u1.y);
      for (int n = 0; n < C.nth; n++) {
        const double2 t = cu.p[3 + n][o];
        f1.x += C.ri[n] * C.grav_x * t.x; f1.y += C.ri[n] * C.grav_x * t.y;
        f3.x += C.ri[n] * C.grav_z * t.x; f3.y += C.ri[n] * C.grav_z * t.y;
      }
      const double2 n1 = nl[(0 * ZF_KXG + c) * nkzt + kp], n3 = nl[(2 * ZF_KXG + c) * nkzt + kp];
      f1.x += n1.x; f1.y += n1.y;
      f3.x += n3.x; f3.y += n3.y;
      double2 r1 = u1, r3 = u3;
      if (rk_step > 1) {
        const double2 o1 = cf.p[0][o], o3 = cf.p[2][o];
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
      cf.p[0][o] = f1;
      cf.p[2][o] = f3;
      rhs.p[0][o] = r1;
      rhs.p[2][o] = r3;
    }
    // ---- U2 (rows 2..NY)
    if (j >= 2 && j <= C.NY) {
      const double2 u2m = cu.p[1][o - ss], u2p = cu.p[1][o + ss];
      double2 f2 = make_double2(-NU * kk * u2.x, -NU * kk * u2.y);
      if (!mean) {
        for (int n = 0; n < C.nth; n++) {
          const double2 t = cu.p[3 + n][o], tm = cu.p[3 + n][o - ss];
          const double w = C.ri[n] * C.grav_y;
          f2.x += w * (t.x * dyfm + tm.x * dyfj) / (2.0 * dyj);
          f2.y += w * (t.y * dyfm + tm.y * dyfj) / (2.0 * dyj);
        }
      }
      const double2 n2 = nl[(1 * ZF_KXG + c) * nkzt + kp];
      f2.x += n2.x; f2.y += n2.y;
      double2 r2 = u2;
      if (rk_step > 1) {
        const double2 o2 = cf.p[1][o];
        r2.x += T3 * o2.x; r2.y += T3 * o2.y;
      }
      const double2 pm = cp[o - ss];
      r2.x -= T4 * ((p0.x - pm.x) / dyj);
      r2.y -= T4 * ((p0.y - pm.y) / dyj);
      r2.x += T5 * f2.x; r2.y += T5 * f2.y;
      const double a = T1 * NUV;
      r2.x += a * (((u2p.x - u2.x) / dyfj - (u2.x - u2m.x) / dyfm) / dyj);
      r2.y += a * (((u2p.y - u2.y) / dyfj - (u2.y - u2m.y) / dyfm) / dyj);
      cf.p[1][o] = f2;
      rhs.p[1][o] = r2;
    }
    // ---- scalars (rows JSTART_TH..JEND_TH)
    for (int n = 0; n < C.nth; n++) {
      if (j < C.JSt[n] || j > C.JEt[n]) continue;
      const double2 t = cu.p[3 + n][o], tm = cu.p[3 + n][o - ss], tp = cu.p[3 + n][o + ss];
      const double nup = NU / C.pr[n];
      double2 ft = make_double2(-nup * kk * t.x - u1.x * C.drhodx[n] - u3.x * C.drhodz[n],
                                -nup * kk * t.y - u1.y * C.drhodx[n] - u3.y * C.drhodz[n]);
      const double2 nt = nl[((3 + n) * ZF_KXG + c) * nkzt + kp];
      ft.x += nt.x; ft.y += nt.y;
      double2 rt = t;
      if (rk_step > 1) {
        const double2 ot = cf.p[3 + n][o];
        rt.x += T3 * ot.x; rt.y += T3 * ot.y;
      }
      rt.x += T5 * ft.x; rt.y += T5 * ft.y;
      const double a = (T1 / C.pr[n]) * NUV;
      rt.x += a * (((tp.x - t.x) / dyj1 - (t.x - tm.x) / dyj) / dyfj);
      rt.y += a * (((tp.y - t.y) / dyj1 - (t.y - tm.y) / dyj) / dyfj);
      cf.p[3 + n][o] = ft;
      rhs.p[3 + n][o] = rt;
    }
  }
}

size_t zfwd_smem(const dg_handle *h) {
  return sizeof(double2) * (h->NZ + 4 * ZF_KXG * (h->NZ + 1) + h->nf * ZF_KXG * h->nkzt);
}

// ------------------------------------------------------------ CN tables
// One thread per field builds the reference's physical-space system exactly
// (identity init, CN rows over the build range, lower then upper BC rows,
// for/channel.f:771-1029 and 1660-2282) and runs the MPI forward elimination
// (for/mpi.f:672-700): a(j) = -a(j)/b(j-1), b(j) += a(j) c(j-1).
struct CnParams {
  int NY, nth, JS, JE, JSt[DG_MAX_TH], JEt[DG_MAX_TH];
  int bct[3 + DG_MAX_TH][2];        // BC types lower/upper per field
  double bcc[3 + DG_MAX_TH][2];     // BC values
  double nu, nuv, pr[DG_MAX_TH];
};

__global__ void k_cn_tables(CnParams P, const double *__restrict__ dscal, int rk_step,
                            const double *__restrict__ dy, const double *__restrict__ dyf,
                            double *__restrict__ tab, int *__restrict__ kind,
                            double *__restrict__ bcv) {
  const int f = threadIdx.x;
  if (f >= 3 + P.nth) return;
  const int NY = P.NY, L = NY + 2;
  double *A = tab + (long)(f * 4 + 0) * L;   // becomes the multiplier
  double *B = tab + (long)(f * 4 + 1) * L;   // becomes 1/b'
  double *Cc = tab + (long)(f * 4 + 2) * L;
  int *K = kind + f * L;
  double *V = bcv + f * L;
  const double h = dscal[1 + rk_step];
  const double T1 = P.nu * h / 2.0, NUV = P.nuv;
  for (int j = 0; j < L; j++) { A[j] = 0.; B[j] = 1.; Cc[j] = 0.; K[j] = ROW_ZERO; V[j] = 0.; }
  auto row = [&](int j, double l, double d, double u, double v) {
    A[j] = l; B[j] = d; Cc[j] = u; V[j] = v; K[j] = (v != 0.0) ? ROW_BC : ROW_ZERO;
  };
  const int lo = P.bct[f][0], up = P.bct[f][1];
  const double clo = P.bcc[f][0], cup = P.bcc[f][1];
  if (f == F_U2) {
    for (int j = 2; j <= NY; j++) {
      A[j] = -T1 * NUV / (dyf[j - 1] * dy[j]);
      B[j] = 1. + T1 * NUV / (dyf[j] * dy[j]) + T1 * NUV / (dyf[j - 1] * dy[j]);
      Cc[j] = -T1 * NUV / (dyf[j] * dy[j]);
      K[j] = ROW_RHS;
    }
    // APPLY_BC_2_LOWER / _UPPER (for/channel.f:1822-1933)
    if (lo == 0) { row(1, 0., 1., 0., clo); row(2, 0., 1., 0., clo); }
    else if (lo == 1) row(1, 0., -1., 1., dyf[1] * clo);
    row(0, 0., 1., 0., 0.);
    if (up == 0) { row(NY + 1, 0., 1., 0., cup); row(NY, 0., 1., 0., cup); }
    else if (up == 1) row(NY + 1, -1., 1., 0., dyf[NY] * cup);
  } else {
    int j0, j1;
    double a;
    if (f < 3) { j0 = P.JS; j1 = P.JE; a = T1 * NUV; }
    else { j0 = P.JSt[f - 3]; j1 = P.JEt[f - 3]; a = T1 / P.pr[f - 3] * NUV; }
    for (int j = j0; j <= j1; j++) {
      if (f < 3) {
        A[j] = -T1 * NUV / (dy[j] * dyf[j]);
        B[j] = 1. - T1 * NUV * (-1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]));
        Cc[j] = -T1 * NUV / (dy[j + 1] * dyf[j]);
      } else {
        A[j] = -(a) / (dy[j] * dyf[j]);
        B[j] = 1. + (a) / (dy[j + 1] * dyf[j]) + (a) / (dy[j] * dyf[j]);
        Cc[j] = -(a) / (dy[j + 1] * dyf[j]);
      }
      K[j] = ROW_RHS;
    }
    // APPLY_BC_1/3/TH_LOWER and _UPPER share one form
    if (lo == 0) { row(0, 0., 1., 0., 0.); row(1, 0., 1., 0., clo); }
    else { row(0, 0., 1., 0., 0.); row(1, 0., -1., 1., dy[2] * clo); }
    if (up == 0) { row(NY + 1, 0., 1., 0., 0.); row(NY, 0., 1., 0., cup); }
    else { row(NY, -1., 1., 0., dy[NY] * cup); row(NY + 1, 0., 1., 0., 0.); }
  }
  // forward elimination (THOMAS_FORWARD_REAL_MPI, single rank)
  for (int j = 1; j < L; j++) {
    A[j] = -A[j] / B[j - 1];
    B[j] = B[j] + A[j] * Cc[j - 1];
  }
  for (int j = 0; j < L; j++) B[j] = (B[j] != 0.0) ? 1.0 / B[j] : 0.0;
}

// --------------------------------------------------------------- CN solve
__global__ void __launch_bounds__(128) k_cn_solve(
    int NY, long ss, int nf, const double *__restrict__ tab, const int *__restrict__ kind,
    const double *__restrict__ bcv, FieldPtrs rhs, FieldPtrs cu, int wlo0, int wlo1, int wlo2,
    int wlo3, int wlo4, int wlo5, int wlo6) {
  const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (m >= ss || f >= nf) return;
  const int L = NY + 2;
  const double *A = tab + (long)(f * 4 + 0) * L;
  const double *RB = tab + (long)(f * 4 + 1) * L;
  const double *Cc = tab + (long)(f * 4 + 2) * L;
  const int *K = kind + f * L;
  const double *V = bcv + f * L;
  const double2 *R = rhs.p[f];
  double2 *U = cu.p[f];
  const int wl[7] = {wlo0, wlo1, wlo2, wlo3, wlo4, wlo5, wlo6};
  const int wlo = wl[f];
  const bool mean = (m == 0);
  // forward sweep; g(j) is parked in U(j) for j >= wlo
  double2 g = make_double2(0.0, 0.0);
  for (int j = 0; j < L; j++) {
    double2 r = make_double2(0.0, 0.0);
    const int k = K[j];
    if (k == ROW_RHS) r = R[(long)j * ss + m];
    else if (k == ROW_BC && mean) r = make_double2(V[j], 0.0);
    if (j > 0) {
      const double a = A[j];
      r.x += a * g.x;
      r.y += a * g.y;
    }
    g = r;
    if (j >= wlo) U[(long)j * ss + m] = g;
  }
  // backward sweep (THOMAS_BACKWARD_REAL_MPI, single rank)
  double2 x = make_double2(g.x * RB[L - 1], g.y * RB[L - 1]);
  U[(long)(L - 1) * ss + m] = x;
  for (int j = L - 2; j >= wlo; j--) {
    const double2 gj = U[(long)j * ss + m];
    const double c = Cc[j], rb = RB[j];
    x = make_double2((gj.x - c * x.x) * rb, (gj.y - c * x.y) * rb);
    U[(long)j * ss + m] = x;
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
  // row 1
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

__global__ void __launch_bounds__(128) k_remdiv(
    int NY, long ss, int nkxp, int JS, int JE, const double *__restrict__ kxv,
    const double *__restrict__ kzv, const double *__restrict__ dy, const double *__restrict__ dyf,
    const double *__restrict__ ra, const double *__restrict__ rrb, double2 *__restrict__ u1,
    double2 *__restrict__ u2, double2 *__restrict__ u3, double2 *__restrict__ cp,
    double2 *__restrict__ phi_out, double2 *__restrict__ gs, const double *__restrict__ dscal,
    int rk_step) {
  const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= ss) return;
  const int kx = (int)(m % nkxp), kp = (int)(m / nkxp);
  const double KX = kxv[kx], KZ = kzv[kp];
  const bool mean = (m == 0);
  // forward sweep rows 2..NY; RHS = i kx U1 + (U2(j+1)-U2(j))/DYF(j) + i kz U3
  double2 g = make_double2(0.0, 0.0);  // g(1) = 0
  for (int j = 2; j <= NY; j++) {
    double2 r = make_double2(0.0, 0.0);
    if (j < NY) {
      const long o = (long)j * ss + m;
      const double2 a1 = u1[o], a3 = u3[o], b2 = u2[o], b2p = u2[o + ss];
      const double d = dyf[j];
      r.x = (-KX * a1.y) + (b2p.x - b2.x) / d + (-KZ * a3.y);
      r.y = (KX * a1.x) + (b2p.y - b2.y) / d + (KZ * a3.x);
    }
    const double a = ra[(long)j * ss + m];
    g = make_double2(r.x + a * g.x, r.y + a * g.y);
    gs[(long)j * ss + m] = g;
  }
  const double hh = (rk_step > 0) ? dscal[1 + rk_step] : 1.0;
  // backward sweep with projection
  double2 phin = make_double2(g.x * rrb[(long)NY * ss + m], g.y * rrb[(long)NY * ss + m]);
  auto project = [&](int j, double2 ph) {
    const long o = (long)j * ss + m;
    double2 a1 = u1[o], a3 = u3[o];
    // U1 -= i kx phi, U3 -= i kz phi
    a1.x -= -KX * ph.y; a1.y -= KX * ph.x;
    a3.x -= -KZ * ph.y; a3.y -= KZ * ph.x;
    u1[o] = a1;
    u3[o] = a3;
    phi_out[o] = ph;
    if (rk_step > 0 && j >= JS && j <= JE) {
      double2 p = cp[o];
      p.x = p.x + ph.x / hh;
      p.y = p.y + ph.y / hh;
      cp[o] = p;
    }
  };
  project(NY, phin);
  for (int j = NY - 1; j >= 1; j--) {
    double u;
    if (j == 1) u = mean ? 0.0 : -1.0;
    else u = 1. / (dy[j + 1] * dyf[j]);
    const double2 gj = (j >= 2) ? gs[(long)j * ss + m] : make_double2(0.0, 0.0);
    const double rb = rrb[(long)j * ss + m];
    const double2 ph = make_double2((gj.x - u * phin.x) * rb, (gj.y - u * phin.y) * rb);
    project(j, ph);
    // U2(j+1) -= (phi(j+1) - phi(j)) / DY(j+1)
    const long o = (long)(j + 1) * ss + m;
    double2 b = u2[o];
    b.x -= (phin.x - ph.x) / dy[j + 1];
    b.y -= (phin.y - ph.y) / dy[j + 1];
    u2[o] = b;
    phin = ph;
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
__device__ __forceinline__ void atomic_min_pos(unsigned long long *addr, double v) {
  // v >= 0 or +inf: the IEEE bit patterns order like unsigned integers
  atomicMin(addr, (unsigned long long)__double_as_longlong(v));
}

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
  if ((threadIdx.x & 31) == 0) atomic_min_pos(out, best);
}

__global__ void k_dt_update(double *dscal, const unsigned long long *minbits, double dt0) {
  // for/courant.f:15-62: dt0 carries the velocity-independent limits
  double dt = fmin(dt0, __longlong_as_double((long long)*minbits));
  double nd;
  if (dt <= 0) nd = 0.0001;
  else if (dt >= 999.) nd = 999.0;
  else nd = dt;
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
      const double2 v = u.p[f][(long)j * ss + m];
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
static int cn_tables(dg_handle *h, int rk_step) {
  CnParams P;
  P.NY = h->NY; P.nth = h->NTH; P.JS = h->jstart; P.JE = h->jend;
  P.nu = h->p.nu; P.nuv = h->p.nu_v_scale;
  for (int n = 0; n < DG_MAX_TH; n++) { P.JSt[n] = h->jstart_th[n]; P.JEt[n] = h->jend_th[n]; P.pr[n] = h->p.pr[n]; }
  P.bct[0][0] = h->p.u_bc_ymin; P.bct[0][1] = h->p.u_bc_ymax;
  P.bcc[0][0] = h->p.u_bc_ymin_c1; P.bcc[0][1] = h->p.u_bc_ymax_c1;
  P.bct[1][0] = h->p.v_bc_ymin; P.bct[1][1] = h->p.v_bc_ymax;
  P.bcc[1][0] = h->p.v_bc_ymin_c1; P.bcc[1][1] = h->p.v_bc_ymax_c1;
  P.bct[2][0] = h->p.w_bc_ymin; P.bct[2][1] = h->p.w_bc_ymax;
  P.bcc[2][0] = h->p.w_bc_ymin_c1; P.bcc[2][1] = h->p.w_bc_ymax_c1;
  for (int n = 0; n < h->NTH; n++) {
    P.bct[3 + n][0] = h->p.th_bc_ymin[n]; P.bct[3 + n][1] = h->p.th_bc_ymax[n];
    P.bcc[3 + n][0] = h->p.th_bc_ymin_c1[n]; P.bcc[3 + n][1] = h->p.th_bc_ymax_c1[n];
  }
  k_cn_tables<<<1, 32, 0, h->st>>>(P, h->dscal, rk_step, h->dy, h->dyf, h->cn_tab, h->cn_kind,
                                   h->cn_bc);
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
  k_bc_vel<<<dg_cdiv(h->ss, 128), 128, 0, h->st>>>(B, h->ss, h->dy, h->dyf, h->cu[0], h->cu[1],
                                                   h->cu[2]);
  DG_LAUNCHED();
  return DG_OK;
}

int dg_rem_div_dev(dg_handle *h, int update_cp, int rk_step) {
  k_remdiv<<<dg_cdiv(h->ss, 128), 128, 0, h->st>>>(
      h->NY, h->ss, h->nkxp, h->jstart, h->jend, h->kx, h->kz, h->dy, h->dyf, h->rem_a,
      h->rem_rb, h->cu[0], h->cu[1], h->cu[2], h->cp, h->cr1, h->gphi, h->dscal,
      update_cp ? rk_step : 0);
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

int dg_courant_dev(dg_handle *h, const double2 *const *u) {
  // physical U1..U3 on planes 1..NY into the work array
  DG_TRY(dg_zinv(h, u, 3, 1, h->NY, h->H, 0));
  const long pplane = (long)h->NZ * h->NX;
  const long pfield = (long)h->NY * pplane;
  double *phys = (double *)h->work;
  // dg_xc2r_planes addresses phys + f*pfield + j*pplane; shift so plane 1 lands at 0
  DG_TRY(dg_xc2r_planes(h, h->H, 3, 1, h->NY, phys - pplane, pplane, h->NX, pfield));
  DG_CUDA(cudaMemsetAsync(h->dmin_bits, 0x7f, sizeof(unsigned long long), h->st));
  k_cfl_min<<<4 * 148, 256, 0, h->st>>>(phys, pfield, h->NY, h->NZ, h->NX, h->p.cfl,
                                        h->p.lx / h->NX, h->p.lz / h->NZ, h->dy, h->dmin_bits);
  DG_LAUNCHED();
  k_dt_update<<<1, 1, 0, h->st>>>(h->dscal, h->dmin_bits, courant_dt0(h));
  DG_LAUNCHED();
  return DG_OK;
}

int dg_chan_init(dg_handle *h) {
  k_remdiv_init<<<dg_cdiv(h->ss, 128), 128, 0, h->st>>>(h->NY, h->ss, h->nkxp, h->kx, h->kz, h->dy,
                                                        h->dyf, h->rem_a, h->rem_rb);
  DG_LAUNCHED();
  cudaFuncSetAttribute(k_xrow_nl, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_zfwd_rhs, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  return DG_OK;
}

extern "C" int diablo_rk_chan_1(dg_handle *h, int time_step, int rk_step) {
  if (!h || h->periodic || rk_step < 1 || rk_step > 3) return DG_ERR_ARG;
  const ChanConst C = make_const(h);
  // 1. z inverse of every prognostic field, all planes
  const double2 *in[3 + DG_MAX_TH];
  for (int f = 0; f < h->nf; f++) in[f] = h->cu[f];
  DG_TRY(dg_zinv(h, in, h->nf, 0, h->NY + 1, h->H, 0));
  // 2. x-row nonlinear products, y-marching chunks
  const int chunk = 16;
  const long Hfield = (long)h->nplanes * h->NZ * h->nkxp;
  {
    dim3 grid(dg_cdiv(h->NZ, XR_ROWS), dg_cdiv(h->NY, chunk));
    k_xrow_nl<<<grid, 256, xrow_smem(h), h->st>>>(C, h->H, Hfield, chunk, h->plx, h->twx, h->dyf,
                                                  h->dy, h->kx, h->G, Hfield);
    DG_LAUNCHED();
  }
  // 3. z forward, explicit terms, CN right-hand side
  {
    FieldPtrs cu, cf, rhs;
    for (int f = 0; f < h->nf; f++) { cu.p[f] = h->cu[f]; cf.p[f] = h->cf[f]; rhs.p[f] = h->rhs[f]; }
    dim3 grid(dg_cdiv(h->nkxp, ZF_KXG), h->NY);
    k_zfwd_rhs<<<grid, 256, zfwd_smem(h), h->st>>>(C, h->G, Hfield, h->plz, h->twz, h->dscal,
                                                   rk_step, h->kx, h->kz, h->dy, h->dyf, cu, cf,
                                                   rhs, h->cp);
    DG_LAUNCHED();
  }
  // 4. CN tables for this substep and the per-mode solves
  DG_TRY(cn_tables(h, rk_step));
  {
    FieldPtrs cu, rhs;
    for (int f = 0; f < h->nf; f++) { cu.p[f] = h->cu[f]; rhs.p[f] = h->rhs[f]; }
    int wl[7] = {1, 1, 1, 1, 1, 1, 1};
    for (int n = 0; n < h->NTH; n++) wl[3 + n] = h->jstart_th[n] - 1;
    dim3 grid(dg_cdiv(h->ss, 128), h->nf);
    k_cn_solve<<<grid, 128, 0, h->st>>>(h->NY, h->ss, h->nf, h->cn_tab, h->cn_kind, h->cn_bc, rhs,
                                        cu, wl[0], wl[1], wl[2], wl[3], wl[4], wl[5], wl[6]);
    DG_LAUNCHED();
  }
  // 5. COURANT on the post-CN velocity (for/channel.f:1037-1040)
  if (h->p.variable_dt && rk_step == 3 && h->p.update_dt > 0 &&
      (time_step % h->p.update_dt) == 0) {
    const double2 *u[3] = {h->cu[0], h->cu[1], h->cu[2]};
    DG_TRY(dg_courant_dev(h, u));
  }
  // 6. REM_DIV_CHAN + CP update
  DG_TRY(dg_rem_div_dev(h, 1, rk_step));
  return DG_OK;
}

extern "C" int diablo_rem_div_chan(dg_handle *h) {
  if (!h || h->periodic) return DG_ERR_ARG;
  return dg_rem_div_dev(h, 0, 0);
}

extern "C" int diablo_apply_bc_vel(dg_handle *h) {
  if (!h || h->periodic) return DG_ERR_ARG;
  return dg_apply_bc_vel_dev(h);
}

extern "C" int diablo_courant(dg_handle *h) {
  if (!h || h->periodic) return DG_ERR_ARG;
  const double2 *u[3] = {h->cu[0], h->cu[1], h->cu[2]};
  return dg_courant_dev(h, u);
}

int dg_stats_dev(dg_handle *h, dg_stats *s) {
  const int NP = h->nplanes;
  double *dsum = (double *)h->work;
  CFieldPtrs u;
  for (int f = 0; f < h->nf; f++) u.p[f] = h->cu[f];
  DG_CUDA(cudaMemsetAsync(h->dflag, 0, sizeof(int), h->st));
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
  double2 c0;
  for (int j = 0; j <= NY + 1; j++) {
    cudaMemcpy(&c0, h->cu[0] + (long)j * h->ss, sizeof(double2), cudaMemcpyDeviceToHost);
    ume[j] = c0.x;
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
  k_div_spec<<<dg_cdiv((long)(NY + 2) * h->ss, 256), 256, 0, h->st>>>(
      NY, h->ss, h->nkxp, h->kx, h->kz, h->dyf, h->cu[0], h->cu[1], h->cu[2], dspec);
  DG_LAUNCHED();
  const double2 *dd[1] = {dspec};
  DG_TRY(dg_zinv(h, dd, 1, 2, NY - 1, h->H, 0));
  const long pplane = (long)h->NZ * h->NX;
  double *phys = (double *)h->work;
  DG_TRY(dg_xc2r_planes(h, h->H, 1, 2, NY - 1, phys - 2 * pplane, pplane, h->NX, 0));
  DG_CUDA(cudaMemsetAsync(h->dmin_bits, 0, sizeof(unsigned long long), h->st));
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
