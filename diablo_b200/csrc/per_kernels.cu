// Triply periodic substep (RK_PER_1, for/periodic.f:23-285) and its helpers
// REM_DIV_PER (:299-326) and POISSON_P_PER (:329-393).
//
// Spectral fields are [ky][kz][kx] (TNKY+1 planes of the retained (kz, kx)
// modes, packed like kz).  One substep:
//   yinv   spectral -> Hy [y][kz][kx]       (c2c along y per (kz, kx) column)
//   zinv   Hy -> H [y][z][kx]               (c2c along z per kx column)
//   k_prod_per_w  per physical (y, z) row: x c2r of U1..U3 (and TH), the 6
//          (+3 per scalar) products u_i u_j, x r2c -> Hp [p][y][z][kx] / NX
//   zfwd   Hp -> Qz [p][y][kz][kx] / NZ
//   yfwd   Qz -> Fy [p][ky][kz][kx] / NY
//   k_per_final  per mode: CF = -i k . (products), forcing and buoyancy,
//          RK3 + diagonal Crank-Nicolson, REM_DIV_PER, CP += phi / h.
// Everything after the transforms is local in spectral space.
//
// Deviation from the shipped reference, by design: FFT_XZ_TO_PHYSICAL in
// for/mpi.f does not zero kx = NKX+1..NX/2-1 before the c2r
// (for/mpi.f:1652-1655), and RK_PER_1 leaves physical-space values in those
// slots of CU between substeps, so the shipped periodic path would feed them
// back into the next transform.  This implementation (and the CPU oracle)
// follows the packing contract documented in for/fft.f:48-50: modes beyond
// the retained set are zero on every inverse transform.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dg_internal.cuh"
#include "fft.cuh"

using namespace dgfft;

namespace {

struct PerConst {
  int NX, NY, NZ, NKX, NKY, NKZ, nkxp, nkzt, nkyt, nf, nth, np;
  long ss;
  double nu, eps, ri[DG_MAX_TH], pr[DG_MAX_TH];
  int bg[DG_MAX_TH];
};

PerConst make_pc(const dg_handle *h) {
  PerConst c;
  c.NX = h->NX; c.NY = h->NY; c.NZ = h->NZ; c.NKX = h->NKX; c.NKY = h->NKY; c.NKZ = h->NKZ;
  c.nkxp = h->nkxp; c.nkzt = h->nkzt; c.nkyt = h->nkyt; c.nf = h->nf; c.nth = h->NTH;
  c.np = 6 + 3 * h->NTH; c.ss = h->ss;
  c.nu = h->p.nu; c.eps = h->eps;
  for (int n = 0; n < DG_MAX_TH; n++) {
    c.ri[n] = h->p.ri[n]; c.pr[n] = h->p.pr[n]; c.bg[n] = h->p.background_grad[n];
  }
  return c;
}

// ----------------------------------------------------------- products (warp)
// One warp per physical (y, z) row: c2r of the fields, products, r2c.
template <int NX, int NTH, typename CX = double2>
__global__ void __launch_bounds__(128) k_prod_per_w(PerConst C, const CX *__restrict__ H,
                                                    long Hfield, const CX *__restrict__ tw,
                                                    CX *__restrict__ Hp, long Pfield) {
  constexpr int NF = 3 + NTH;
  constexpr int NPIN = (NF + 1) / 2;
  constexpr int NPROD = 6 + 3 * NTH;
  constexpr int NPP = (NPROD + 1) / 2;
  constexpr int MAXP = NPIN > NPP ? NPIN : NPP;
  constexpr int XPL = (NX + 31) / 32;
  constexpr int NKXP = NX / 3 + 1;
  constexpr int KS = (NKXP + 31) / 32;
  constexpr int SSTR = padded_len(NX);
  extern __shared__ double2 sm_raw[];
  using T = typename CT<CX>::T;
  CX *sm = reinterpret_cast<CX *>(sm_raw);
  CX *stw = sm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  CX *buf = stw + NX + warp * MAXP * SSTR;
  for (int i = threadIdx.x; i < NX; i += blockDim.x) stw[i] = tw[i];
  __syncthreads();
  const long row = (long)blockIdx.x * 4 + warp;  // row = y * NZ + z
  if (row >= (long)C.NY * C.NZ) return;
  const CX *src = H + row * NKXP;
  // c2r of field pairs
#pragma unroll
  for (int q = 0; q < NPIN; q++) {
    const int fa = 2 * q, fb = 2 * q + 1;
#pragma unroll
    for (int i = 0; i < (NX + 31) / 32; i++) {
      const int k = lane + 32 * i;
      if (k < NX) {
        const int kk = (k <= NX / 2) ? k : NX - k;
        CX v = CT<CX>::mk(0, 0);
        if (kk < NKXP && kk < NX / 2) {
          CX a = src[fa * Hfield + kk];
          CX b = (fb < NF) ? src[fb * Hfield + kk] : CT<CX>::mk(0, 0);
          if (kk == 0) { a.y = 0.0; b.y = 0.0; }
          v = (k == kk) ? CT<CX>::mk(a.x - b.y, a.y + b.x) : CT<CX>::mk(a.x + b.y, -a.y + b.x);
        }
        buf[q * SSTR + pad(k)] = v;
      }
    }
  }
  __syncwarp();
  wpasses<NX, +1, 0>(buf, NPIN, SSTR, stw, lane);
  T u[NF][XPL];
#pragma unroll
  for (int q = 0; q < NPIN; q++)
#pragma unroll
    for (int i = 0; i < XPL; i++) {
      const int x = lane + 32 * i;
      const CX v = (x < NX) ? buf[q * SSTR + pad(x)] : CT<CX>::mk(0, 0);
      u[2 * q][i] = v.x;
      if (2 * q + 1 < NF) u[2 * q + 1][i] = v.y;
    }
  __syncwarp();
#pragma unroll
  for (int i = 0; i < XPL; i++) {
    const int x = lane + 32 * i;
    if (x >= NX) continue;
    const T u1 = u[0][i], u2 = u[1][i], u3 = u[2][i];
    T P[2 * NPP];
    P[0] = u1 * u1;
    P[1] = u1 * u2;
    P[2] = u1 * u3;
    P[3] = u2 * u2;
    P[4] = u2 * u3;
    P[5] = u3 * u3;
#pragma unroll
    for (int n = 0; n < NTH; n++) {
      const T t = u[3 + n][i];
      P[6 + 3 * n] = u1 * t;
      P[7 + 3 * n] = u2 * t;
      P[8 + 3 * n] = u3 * t;
    }
    if (2 * NPP > NPROD) P[2 * NPP - 1] = 0.0;
#pragma unroll
    for (int q = 0; q < NPP; q++) buf[q * SSTR + pad(x)] = CT<CX>::mk(P[2 * q], P[2 * q + 1]);
  }
  __syncwarp();
  wpasses<NX, -1, 0>(buf, NPP, SSTR, stw, lane);
  CX *dst = Hp + row * NKXP;
#pragma unroll
  for (int s = 0; s < KS; s++) {
    const int k = lane + 32 * s;
    if (k >= NKXP) continue;
#pragma unroll
    for (int p = 0; p < NPROD; p++) {
      const int q = p >> 1;
      const CX zk = buf[q * SSTR + pad(k)];
      const CX zm = buf[q * SSTR + pad((NX - k) % NX)];
      CX v;
      if ((p & 1) == 0) v = CT<CX>::mk((T)0.5 * (zk.x + zm.x), (T)0.5 * (zk.y - zm.y));
      else v = CT<CX>::mk((T)0.5 * (zk.y + zm.y), -(T)0.5 * (zk.x - zm.x));
      dst[p * Pfield + k] = CT<CX>::mk(v.x / (T)NX, v.y / (T)NX);
    }
  }
}

template <int NX, int NTH, typename CX = double2>
size_t prod_smem() {
  constexpr int NF = 3 + NTH, NPIN = (NF + 1) / 2, NPP = (6 + 3 * NTH + 1) / 2;
  constexpr int MAXP = NPIN > NPP ? NPIN : NPP;
  return sizeof(CX) * (NX + 4 * MAXP * padded_len(NX));
}

// generic products from physical fields (any NX): phys [f][y][z][x] -> prod [p][y][z][x]
__global__ void k_prod_phys(const double *__restrict__ phys, long pf, int nth, long n,
                            double *__restrict__ prod) {
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x) {
    const double u1 = phys[q], u2 = phys[pf + q], u3 = phys[2 * pf + q];
    prod[0 * pf + q] = u1 * u1;
    prod[1 * pf + q] = u1 * u2;
    prod[2 * pf + q] = u1 * u3;
    prod[3 * pf + q] = u2 * u2;
    prod[4 * pf + q] = u2 * u3;
    prod[5 * pf + q] = u3 * u3;
    for (int s = 0; s < nth; s++) {
      const double t = phys[(3 + s) * pf + q];
      prod[(6 + 3 * s) * pf + q] = u1 * t;
      prod[(7 + 3 * s) * pf + q] = u2 * t;
      prod[(8 + 3 * s) * pf + q] = u3 * t;
    }
  }
}

// --------------------------------------------------------------- final
// RK_PER_1 (for/periodic.f:36-281) per retained mode, after the transforms.
// product spectra in the working precision, widened to FP64
__device__ __forceinline__ double2 ldF(const double2 *p) { return __ldg(p); }
__device__ __forceinline__ double2 ldF(const float2 *p) {
  const float2 v = __ldg(p);
  return make_double2((double)v.x, (double)v.y);
}

template <int NTHM, typename CF = double2>
__global__ void __launch_bounds__(256) k_per_final(
    PerConst C, int rk_step, const double *__restrict__ dscal, const double *__restrict__ kxv,
    const double *__restrict__ kyv, const double *__restrict__ kzv,
    const CF *__restrict__ Fy, long Ffield, FieldPtrs cu, FieldPtrs cf,
    double2 *__restrict__ cp, double2 *__restrict__ phi, double forcing) {
  // grid: x over the modes of a ky plane, y over the ky planes
  const int jy = blockIdx.y;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= (int)C.ss) return;
  const long q = (long)jy * C.ss + m;
  const int kz = m / C.nkxp, kx = m - kz * C.nkxp;
  // every load of the mode first (the stores below could alias them, so a
  // load placed after a store would wait for the previous load's latency)
  double2 Fp[6 + 3 * (NTHM > 0 ? NTHM : 1)], u[3], old[3], t[NTHM > 0 ? NTHM : 1],
      oldt[NTHM > 0 ? NTHM : 1];
#pragma unroll
  for (int p = 0; p < 6; p++) Fp[p] = ldF(Fy + p * Ffield + q);
#pragma unroll
  for (int d = 0; d < 3; d++) u[d] = __ldg(cu(d) + q);
  const bool hist = rk_step > 1;
#pragma unroll
  for (int d = 0; d < 3; d++) old[d] = hist ? __ldg(cf(d) + q) : make_double2(0.0, 0.0);
#pragma unroll
  for (int n = 0; n < NTHM; n++) {
    if (n < C.nth) {
      t[n] = __ldg(cu(3 + n) + q);
      oldt[n] = hist ? __ldg(cf(3 + n) + q) : make_double2(0.0, 0.0);
#pragma unroll
      for (int r = 0; r < 3; r++) Fp[6 + 3 * n + r] = ldF(Fy + (6 + 3 * n + r) * Ffield + q);
    }
  }
  const double2 p0 = __ldg(cp + q);
  const double KX = kxv[kx], KY = kyv[jy], KZ = kzv[kz];
  const double k2 = KX * KX + KY * KY + KZ * KZ;
  const double h = dscal[1 + rk_step];
  const double zeta = (rk_step == 2) ? -17.0 / 8.0 : (rk_step == 3) ? -5.0 / 4.0 : 0.0;
  const double bbar = (rk_step == 2) ? 25.0 / 8.0 : (rk_step == 3) ? 9.0 / 4.0 : 1.0;
  const double T1 = C.nu * h / 2.0, T2 = bbar * h, T3 = zeta * h, T4 = h;
  // -i k . (f_a, f_b, f_c) = (KX Im a + KY Im b + KZ Im c, -(KX Re a + KY Re b + KZ Re c))
  auto mdiv = [&](double2 a, double2 b, double2 c) {
    return make_double2(KX * a.y + KY * b.y + KZ * c.y, -(KX * a.x + KY * b.x + KZ * c.x));
  };
  double2 nf[3] = {mdiv(Fp[0], Fp[1], Fp[2]), mdiv(Fp[1], Fp[3], Fp[4]),
                   mdiv(Fp[2], Fp[4], Fp[5])};
  // USER_RHS_PER_PHYSICAL: CF_i += (EPSILON_TARGET / EK) U_i (exact in
  // spectral space for band-limited U)
  if (forcing != 0.0) {
#pragma unroll
    for (int d = 0; d < 3; d++) { nf[d].x += forcing * u[d].x; nf[d].y += forcing * u[d].y; }
  }
#pragma unroll
  for (int n = 0; n < NTHM; n++) {
    if (n < C.nth) {
      nf[1].x += C.ri[n] * t[n].x;
      nf[1].y += C.ri[n] * t[n].y;
    }
  }
  // one reciprocal per mode instead of a division per component
  const double t5 = 1 - T1 * k2, it5 = 1.0 / (1 + T1 * k2);
  const double Kd[3] = {KX, KY, KZ};
  double2 un[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    // CR = (1 - T1 k^2) CU - h (i k_d CP) [+ zeta h CF_old] + beta h CF
    double2 r = make_double2(t5 * u[d].x - T4 * (-Kd[d] * p0.y), t5 * u[d].y - T4 * (Kd[d] * p0.x));
    if (hist) {
      r.x += T3 * old[d].x;
      r.y += T3 * old[d].y;
    }
    r.x += T2 * nf[d].x;
    r.y += T2 * nf[d].y;
    un[d] = make_double2(r.x * it5, r.y * it5);
  }
#pragma unroll
  for (int n = 0; n < NTHM; n++) {
    if (n < C.nth) {
      double2 ft = C.bg[n] ? make_double2(-u[1].x, -u[1].y) : make_double2(0.0, 0.0);
      const double2 g = mdiv(Fp[6 + 3 * n], Fp[7 + 3 * n], Fp[8 + 3 * n]);
      ft.x += g.x;
      ft.y += g.y;
      const double t6 = 1 - (T1 / C.pr[n]) * k2, it6 = 1.0 / (1 + (T1 / C.pr[n]) * k2);
      double2 r = make_double2(t6 * t[n].x, t6 * t[n].y);
      if (hist) {
        r.x += T3 * oldt[n].x;
        r.y += T3 * oldt[n].y;
      }
      r.x += T2 * ft.x;
      r.y += T2 * ft.y;
      cu(3 + n)[q] = make_double2(r.x * it6, r.y * it6);
      cf(3 + n)[q] = ft;
    }
  }
  // REM_DIV_PER: phi = (i k . U) / -(k^2 + EPS); U -= i k phi; CP += phi / h
  const double iden = 1.0 / -(KX * KX + KY * KY + KZ * KZ + C.eps);
  const double2 dv = make_double2(-(KX * un[0].y + KY * un[1].y + KZ * un[2].y),
                                  KX * un[0].x + KY * un[1].x + KZ * un[2].x);
  const double2 ph = make_double2(dv.x * iden, dv.y * iden);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    un[d].x -= -Kd[d] * ph.y;
    un[d].y -= Kd[d] * ph.x;
    cu(d)[q] = un[d];
    cf(d)[q] = nf[d];
  }
  phi[q] = ph;
  const double iT4 = 1.0 / T4;
  cp[q] = make_double2(p0.x + ph.x * iT4, p0.y + ph.y * iT4);
}

__global__ void k_rem_div_per(PerConst C, const double *__restrict__ kxv,
                              const double *__restrict__ kyv, const double *__restrict__ kzv,
                              double2 *__restrict__ u1, double2 *__restrict__ u2,
                              double2 *__restrict__ u3, double2 *__restrict__ phi) {
  const int jy = blockIdx.y;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= (int)C.ss) return;
  const long q = (long)jy * C.ss + m;
  const double KX = kxv[m % C.nkxp], KY = kyv[jy], KZ = kzv[m / C.nkxp];
  const double den = -(KX * KX + KY * KY + KZ * KZ + C.eps);
  double2 a = u1[q], b = u2[q], c = u3[q];
  const double2 dv = make_double2(-(KX * a.y + KY * b.y + KZ * c.y), KX * a.x + KY * b.x + KZ * c.x);
  const double2 ph = make_double2(dv.x / den, dv.y / den);
  a.x -= -KX * ph.y; a.y -= KX * ph.x;
  b.x -= -KY * ph.y; b.y -= KY * ph.x;
  c.x -= -KZ * ph.y; c.y -= KZ * ph.x;
  u1[q] = a;
  u2[q] = b;
  u3[q] = c;
  phi[q] = ph;
}

// dst = i k_axis * src (axis 0 = x, 1 = y, 2 = z)
__global__ void k_ik(PerConst C, const double *__restrict__ kxv, const double *__restrict__ kyv,
                     const double *__restrict__ kzv, const double2 *__restrict__ src, int axis,
                     double2 *__restrict__ dst) {
  const int jy = blockIdx.y;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= (int)C.ss) return;
  const long q = (long)jy * C.ss + m;
  const double K = axis == 0 ? kxv[m % C.nkxp] : (axis == 1 ? kyv[jy] : kzv[m / C.nkxp]);
  const double2 v = src[q];
  dst[q] = make_double2(-K * v.y, K * v.x);
}

__global__ void k_pp_first(long n, const double *__restrict__ r1, const double *__restrict__ r2,
                           double *__restrict__ P) {
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    P[q] = r1[q] * r1[q] + r1[q] * r2[q] + r2[q] * r2[q];
}

__global__ void k_pp_second(long n, const double *__restrict__ A, double *__restrict__ P) {
  // A holds F1 F2 F3 R1 R2 R3 (n each)
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    P[q] = 2 * (P[q] + A[q] * A[n + q] + A[2 * n + q] * A[3 * n + q] + A[4 * n + q] * A[5 * n + q]);
}

__global__ void k_pp_solve(PerConst C, const double *__restrict__ kxv, const double *__restrict__ kyv,
                           const double *__restrict__ kzv, double2 *__restrict__ cp) {
  const int jy = blockIdx.y;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= (int)C.ss) return;
  const long q = (long)jy * C.ss + m;
  const double KX = kxv[m % C.nkxp], KY = kyv[jy], KZ = kzv[m / C.nkxp];
  const double d = KX * KX + KY * KY + KZ * KZ + C.eps;
  double2 v = cp[q];
  v = make_double2(v.x / d, v.y / d);
  if (q == 0) v = make_double2(0.0, 0.0);
  cp[q] = v;
}

// Parseval sums per ky plane: [0..2] sum w |U_d|^2, [3+n] sum w |TH_n'|^2
__global__ void k_per_sums(PerConst C, CFieldPtrs u, double *__restrict__ out, int *__restrict__ flag) {
  const int jy = blockIdx.x;
  __shared__ double red[8][256];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int bad = 0;
  for (long m = threadIdx.x; m < C.ss; m += blockDim.x) {
    const double w = (((int)m % C.nkxp) == 0) ? 1.0 : 2.0;
    const long q = (long)jy * C.ss + m;
    for (int f = 0; f < C.nf && f < 8; f++) {
      const double2 v = u(f)[q];
      if (!isfinite(v.x) || !isfinite(v.y)) bad = 1;
      if (f >= 3 && q == 0) continue;
      acc[f] += w * (v.x * v.x + v.y * v.y);
    }
  }
  if (bad) atomicOr(flag, 1);
  for (int k = 0; k < 8; k++) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 8; k++) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 8) out[jy * 8 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_absmax_p(const double *__restrict__ a, long n, unsigned long long *out) {
  double best = 0.0;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
    best = fmax(best, fabs(a[q]));
  for (int off = 16; off > 0; off >>= 1) best = fmax(best, __shfl_down_sync(0xffffffffu, best, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

__global__ void k_div_per(PerConst C, const double *__restrict__ kxv, const double *__restrict__ kyv,
                          const double *__restrict__ kzv, const double2 *__restrict__ u1,
                          const double2 *__restrict__ u2, const double2 *__restrict__ u3,
                          double2 *__restrict__ d) {
  const int jy = blockIdx.y;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= (int)C.ss) return;
  const long q = (long)jy * C.ss + m;
  const double KX = kxv[m % C.nkxp], KY = kyv[jy], KZ = kzv[m / C.nkxp];
  const double2 a = u1[q], b = u2[q], c = u3[q];
  d[q] = make_double2(-(KX * a.y + KY * b.y + KZ * c.y), KX * a.x + KY * b.x + KZ * c.x);
}

}  // namespace

// ================================================================ host side
namespace {

// sizes of the periodic work arrays
long hy_field(const dg_handle *h) { return (long)h->NY * h->ss; }
long h_field(const dg_handle *h) { return (long)h->NY * h->NZ * h->nkxp; }
long fy_field(const dg_handle *h) { return (long)h->nkyt * h->ss; }
long phys_field(const dg_handle *h) { return (long)h->NY * h->NZ * h->NX; }

// Spectral fields (nf of them) -> physical values dst[f][y][z][x] with
// strides (pfield, pplane, prow); y inverse into Hy, z inverse into H, x c2r.
int per_to_physical(dg_handle *h, const double2 *const *fields, int nf, double *dst, long pfield,
                    long pplane, long prow) {
  DG_TRY(dg_cinv_g(h, fields, nf, 0, 0, 0, (int)h->ss, h->NY, h->NKY, h->ply, h->twy, h->Hy,
                   hy_field(h)));
  const double2 *hy[3 + DG_MAX_TH + 1];
  for (int f = 0; f < nf; f++) hy[f] = h->Hy + f * hy_field(h);
  DG_TRY(dg_cinv_g(h, hy, nf, 0, h->NY - 1, h->ss, h->nkxp, h->NZ, h->NKZ, h->plz, h->twz, h->H,
                   h_field(h)));
  // the x kernels address H planes of NZ rows; one field per call
  dg_handle tmp = *h;
  tmp.nplanes = h->NY;
  for (int f = 0; f < nf; f++)
    DG_TRY(dg_xc2r_planes(&tmp, h->H + f * h_field(h), 1, 0, h->NY - 1, dst + f * pfield, pplane,
                          prow, 0));
  return DG_OK;
}

// Physical values src[f][y][z][x] (strides as above) -> spectral fields.
int per_to_fourier(dg_handle *h, const double *src, int nf, long pfield, long pplane, long prow,
                   double2 *const *fields) {
  dg_handle tmp = *h;
  tmp.nplanes = h->NY;
  for (int f = 0; f < nf; f++)
    DG_TRY(dg_xr2c_planes(&tmp, src + f * pfield, 1, 0, h->NY - 1, pplane, prow, 0,
                          h->P + f * h_field(h)));
  double2 *qz[3 + DG_MAX_TH + 1];
  for (int f = 0; f < nf; f++) qz[f] = h->Hy + f * hy_field(h);
  DG_TRY(dg_cfwd_g(h, h->P, h_field(h), nf, 0, h->NY - 1, h->nkxp, h->nkzt, h->NZ, h->NKZ, h->plz,
                   h->twz, qz, h->ss));
  DG_TRY(dg_cfwd_g(h, h->Hy, hy_field(h), nf, 0, 0, (int)h->ss, h->nkyt, h->NY, h->NKY, h->ply,
                   h->twy, fields, 0));
  return DG_OK;
}

int per_to_physical(dg_handle *h, const double2 *const *fields, int nf, double *dst) {
  return per_to_physical(h, fields, nf, dst, phys_field(h), (long)h->NZ * h->NX, h->NX);
}

int per_to_fourier(dg_handle *h, const double *src, int nf, double2 *const *fields) {
  return per_to_fourier(h, src, nf, phys_field(h), (long)h->NZ * h->NX, h->NX, fields);
}

// whether k_prod_per_w has a specialisation for this NX and N_TH
bool prod_warp_ok(const dg_handle *h) {
  const int n = h->NX;
  return h->NTH <= 2 && (n == 16 || n == 32 || n == 48 || n == 64 || n == 96 || n == 128 || n == 256);
}

}  // namespace

int dg_per_init(dg_handle *h) {
  const int np = 6 + 3 * h->NTH;
  const int nmax = np > h->nf ? np : h->nf;
  auto al = [&](double2 **p, size_t n) -> int {
    cudaError_t e = dg_malloc(h, (void **)p, n * sizeof(double2));
    if (e != cudaSuccess) {
      dg_set_error("device allocation failed (periodic work arrays)");
      return e == cudaErrorMemoryAllocation ? DG_ERR_OOM : DG_ERR_CUDA;
    }
    return DG_OK;
  };
  DG_TRY(al(&h->Hy, (size_t)nmax * hy_field(h)));      // Hy, then Qz
  DG_TRY(al(&h->H, (size_t)h->nf * h_field(h)));       // H
  DG_TRY(al(&h->P, (size_t)nmax * h_field(h)));        // Hp
  DG_TRY(al(&h->Q, (size_t)np * fy_field(h)));         // Fy
  // physical scratch: 6 fields for POISSON_P_PER; the generic product path
  // (lengths or scalar counts without a warp specialisation) needs nf + np
  const int nphys = prod_warp_ok(h) ? 6 : (h->nf + np > 6 ? h->nf + np : 6);
  h->work_bytes = sizeof(double) * (size_t)phys_field(h) * nphys;
  if (h->work_bytes < sizeof(double) * 8 * (size_t)h->nkyt)
    h->work_bytes = sizeof(double) * 8 * (size_t)h->nkyt;
  cudaError_t e = dg_malloc(h, (void **)&h->work, h->work_bytes);
  if (e != cudaSuccess) {
    dg_set_error("device allocation failed (periodic physical scratch)");
    return DG_ERR_OOM;
  }
  return DG_OK;
}

static int per_sums(dg_handle *h, double tot[8]);

// USER_RHS_PER_PHYSICAL (for/user_rhs.f:124-194) forcing coefficient
// EPSILON_TARGET / EK with EK = 0.8 <u.u>, from Parseval on the retained modes
static int per_forcing(dg_handle *h, double *coef) {
  *coef = 0.0;
  if (h->p.epsilon_target == 0.0) return DG_OK;
  double tot[8];
  DG_TRY(per_sums(h, tot));
  *coef = h->p.epsilon_target / (0.8 * (tot[0] + tot[1] + tot[2]));
  return DG_OK;
}

// Mixed form of the transforms and products of a periodic substep: the y
// inverse converts the FP64 state to FP32, everything up to the product
// spectra Fy runs in FP32, and the completion kernel widens Fy to FP64.
static int per_nonlinear_mixed(dg_handle *h, const PerConst &C) {
  const int nf = h->nf, np = C.np;
  float2 *Hyf = reinterpret_cast<float2 *>(h->Hy), *Hf = reinterpret_cast<float2 *>(h->H);
  float2 *Pf = reinterpret_cast<float2 *>(h->P), *Qf = reinterpret_cast<float2 *>(h->Q);
  const double2 *in[3 + DG_MAX_TH];
  for (int f = 0; f < nf; f++) in[f] = h->cu[f];
  DG_TRY(dg_cinv_gf(h, in, nf, 0, 0, 0, (int)h->ss, h->NY, h->NKY, h->ply, h->twy_f, Hyf,
                    hy_field(h)));
  const float2 *hy[3 + DG_MAX_TH];
  for (int f = 0; f < nf; f++) hy[f] = Hyf + f * hy_field(h);
  DG_TRY(dg_cinv_ff(h, hy, nf, 0, h->NY - 1, h->ss, h->nkxp, h->NZ, h->NKZ, h->plz, h->twz_f, Hf,
                    h_field(h)));
  bool done = false;
  const long rows = (long)h->NY * h->NZ;
#define PW_CASE(NXV, NTHV)                                                                      \
  if (!done && h->NX == NXV && h->NTH == NTHV) {                                                \
    dg_big_smem((const void *)k_prod_per_w<NXV, NTHV, float2>);                                 \
    dg_kt_begin(h, "k_prod_per_w_f32", h->st);                                                  \
    k_prod_per_w<NXV, NTHV, float2><<<dg_cdiv(rows, 4), 128, prod_smem<NXV, NTHV, float2>(),    \
                                      h->st>>>(C, Hf, h_field(h), h->twx_f, Pf, h_field(h));    \
    done = true;                                                                                \
  }
#define PW_ALL(NXV) PW_CASE(NXV, 0) PW_CASE(NXV, 1) PW_CASE(NXV, 2)
  PW_ALL(16) PW_ALL(32) PW_ALL(48) PW_ALL(64) PW_ALL(96) PW_ALL(128) PW_ALL(256)
#undef PW_ALL
#undef PW_CASE
  if (!done) {
    dg_set_error("mixed precision: no FP32 product kernel for this NX / N_TH");
    return DG_ERR_DIMS;
  }
  DG_LAUNCHED();
  float2 *qz[6 + 3 * DG_MAX_TH], *fy[6 + 3 * DG_MAX_TH];
  for (int p = 0; p < np; p++) {
    qz[p] = Hyf + p * hy_field(h);
    fy[p] = Qf + p * fy_field(h);
  }
  for (int p0 = 0; p0 < np; p0 += 3 + DG_MAX_TH) {
    const int cnt = (np - p0) < 3 + DG_MAX_TH ? (np - p0) : 3 + DG_MAX_TH;
    DG_TRY(dg_cfwd_ff(h, Pf + p0 * h_field(h), h_field(h), cnt, 0, h->NY - 1, h->nkxp, h->nkzt,
                      h->NZ, h->NKZ, h->plz, h->twz_f, qz + p0, h->ss));
  }
  for (int p0 = 0; p0 < np; p0 += 3 + DG_MAX_TH) {
    const int cnt = (np - p0) < 3 + DG_MAX_TH ? (np - p0) : 3 + DG_MAX_TH;
    DG_TRY(dg_cfwd_ff(h, Hyf + p0 * hy_field(h), hy_field(h), cnt, 0, 0, (int)h->ss, h->nkyt,
                      h->NY, h->NKY, h->ply, h->twy_f, fy + p0, 0));
  }
  return DG_OK;
}

bool dg_per_mixed_ok(int nx, int n_th) {
  return n_th <= 2 && (nx == 16 || nx == 32 || nx == 48 || nx == 64 || nx == 96 || nx == 128 ||
                       nx == 256);
}

extern "C" int diablo_rk_per_1(dg_handle *h, int rk_step) {
  if (!h || !h->periodic || rk_step < 1 || rk_step > 3) return DG_ERR_ARG;
  const PerConst C = make_pc(h);
  const int nf = h->nf, np = C.np;
  double forcing = 0.0;
  DG_TRY(per_forcing(h, &forcing));
  if (h->mixed) {
    DG_TRY(per_nonlinear_mixed(h, C));
    FieldPtrs cu, cf;
    for (int f = 0; f < nf; f++) { cu.p[f] = h->cu[f]; cf.p[f] = h->cf[f]; }
    const float2 *Qf = reinterpret_cast<const float2 *>(h->Q);
    const int nthm = h->NTH == 0 ? 0 : (h->NTH == 1 ? 1 : 2);
    dg_kt_begin(h, "k_per_final", h->st);
#define PF_CASE(NM)                                                                             \
  if (nthm == NM)                                                                               \
    k_per_final<NM, float2><<<dim3(dg_cdiv(h->ss, 256), h->nkyt), 256, 0, h->st>>>(             \
        C, rk_step, h->dscal, h->kx, h->ky, h->kz, Qf, fy_field(h), cu, cf, h->cp, h->cr1,      \
        forcing);
    PF_CASE(0) PF_CASE(1) PF_CASE(2)
#undef PF_CASE
    DG_LAUNCHED();
    return DG_OK;
  }
  // y inverse, z inverse
  const double2 *in[3 + DG_MAX_TH];
  for (int f = 0; f < nf; f++) in[f] = h->cu[f];
  DG_TRY(dg_cinv_g(h, in, nf, 0, 0, 0, (int)h->ss, h->NY, h->NKY, h->ply, h->twy, h->Hy,
                   hy_field(h)));
  const double2 *hy[3 + DG_MAX_TH];
  for (int f = 0; f < nf; f++) hy[f] = h->Hy + f * hy_field(h);
  DG_TRY(dg_cinv_g(h, hy, nf, 0, h->NY - 1, h->ss, h->nkxp, h->NZ, h->NKZ, h->plz, h->twz, h->H,
                   h_field(h)));
  // x rows: products
  bool done = false;
  const long rows = (long)h->NY * h->NZ;
#define PW_CASE(NXV, NTHV)                                                                     \
  if (!done && h->NX == NXV && h->NTH == NTHV) {                                               \
    dg_big_smem((const void *)k_prod_per_w<NXV, NTHV>);                                        \
    dg_kt_begin(h, "k_prod_per_w", h->st);                                                       \
    k_prod_per_w<NXV, NTHV><<<dg_cdiv(rows, 4), 128, prod_smem<NXV, NTHV>(), h->st>>>(          \
        C, h->H, h_field(h), h->twx, h->P, h_field(h));                                       \
    done = true;                                                                               \
  }
#define PW_ALL(NXV) PW_CASE(NXV, 0) PW_CASE(NXV, 1) PW_CASE(NXV, 2)
  PW_ALL(16) PW_ALL(32) PW_ALL(48) PW_ALL(64) PW_ALL(96) PW_ALL(128) PW_ALL(256)
#undef PW_ALL
#undef PW_CASE
  if (done) {
    DG_LAUNCHED();
  } else {
    // generic: physical fields, pointwise products, r2c of each product
    double *phys = (double *)h->work;
    dg_handle tmp = *h;
    tmp.nplanes = h->NY;
    for (int f = 0; f < nf; f++)
      DG_TRY(dg_xc2r_planes(&tmp, h->H + f * h_field(h), 1, 0, h->NY - 1, phys + f * phys_field(h),
                            (long)h->NZ * h->NX, h->NX, 0));
    double *prod = phys + (long)nf * phys_field(h);
    dg_kt_begin(h, "k_prod_phys", h->st);
    k_prod_phys<<<4 * 148, 256, 0, h->st>>>(phys, phys_field(h), h->NTH, phys_field(h), prod);
    DG_LAUNCHED();
    for (int p = 0; p < np; p++)
      DG_TRY(dg_xr2c_planes(&tmp, prod + p * phys_field(h), 1, 0, h->NY - 1, (long)h->NZ * h->NX,
                            h->NX, 0, h->P + p * h_field(h)));
  }
  // z forward, y forward of the products
  double2 *qz[6 + 3 * DG_MAX_TH];
  for (int p = 0; p < np; p++) qz[p] = h->Hy + p * hy_field(h);
  for (int p0 = 0; p0 < np; p0 += 3 + DG_MAX_TH) {
    const int cnt = (np - p0) < 3 + DG_MAX_TH ? (np - p0) : 3 + DG_MAX_TH;
    DG_TRY(dg_cfwd_g(h, h->P + p0 * h_field(h), h_field(h), cnt, 0, h->NY - 1, h->nkxp, h->nkzt,
                     h->NZ, h->NKZ, h->plz, h->twz, qz + p0, h->ss));
  }
  double2 *fy[6 + 3 * DG_MAX_TH];
  for (int p = 0; p < np; p++) fy[p] = h->Q + p * fy_field(h);
  for (int p0 = 0; p0 < np; p0 += 3 + DG_MAX_TH) {
    const int cnt = (np - p0) < 3 + DG_MAX_TH ? (np - p0) : 3 + DG_MAX_TH;
    DG_TRY(dg_cfwd_g(h, h->Hy + p0 * hy_field(h), hy_field(h), cnt, 0, 0, (int)h->ss, h->nkyt,
                     h->NY, h->NKY, h->ply, h->twy, fy + p0, 0));
  }
  // per-mode completion
  FieldPtrs cu, cf;
  for (int f = 0; f < nf; f++) { cu.p[f] = h->cu[f]; cf.p[f] = h->cf[f]; }
  const long tot = (long)h->nkyt * h->ss;
  dg_kt_begin(h, "k_per_final", h->st);
  const int nthm = h->NTH == 0 ? 0 : (h->NTH == 1 ? 1 : (h->NTH == 2 ? 2 : 4));
#define PF_CASE(NM)                                                                             \
  if (nthm == NM)                                                                               \
    k_per_final<NM><<<dim3(dg_cdiv(h->ss, 256), h->nkyt), 256, 0, h->st>>>(                     \
        C, rk_step, h->dscal, h->kx, h->ky, h->kz, h->Q, fy_field(h), cu, cf, h->cp, h->cr1,    \
        forcing);
  PF_CASE(0) PF_CASE(1) PF_CASE(2) PF_CASE(4)
#undef PF_CASE
  DG_LAUNCHED();
  return DG_OK;
}

extern "C" int diablo_rem_div_per(dg_handle *h) {
  if (!h || !h->periodic) return DG_ERR_ARG;
  const PerConst C = make_pc(h);
  const long tot = (long)h->nkyt * h->ss;
  dg_kt_begin(h, "k_rem_div_per", h->st);
  k_rem_div_per<<<dim3(dg_cdiv(h->ss, 256), h->nkyt), 256, 0, h->st>>>(C, h->kx, h->ky, h->kz, h->cu[0], h->cu[1],
                                                      h->cu[2], h->cr1);
  DG_LAUNCHED();
  return DG_OK;
}

extern "C" int diablo_poisson_p_per(dg_handle *h) {
  if (!h || !h->periodic) return DG_ERR_ARG;
  const PerConst C = make_pc(h);
  const long tot = (long)h->nkyt * h->ss;
  const long n = phys_field(h);
  double *W = (double *)h->work;  // 6 physical fields
  double2 *s0 = h->rhs[0], *s1 = h->rhs[1];
  // R1 = IFFT(i kx U1), R2 = IFFT(i kz U3); P = R1^2 + R1 R2 + R2^2
  dg_kt_begin(h, "k_ik", h->st);
  k_ik<<<dim3(dg_cdiv(h->ss, 256), h->nkyt), 256, 0, h->st>>>(C, h->kx, h->ky, h->kz, h->cu[0], 0, s0);
  DG_LAUNCHED();
  dg_kt_begin(h, "k_ik", h->st);
  k_ik<<<dim3(dg_cdiv(h->ss, 256), h->nkyt), 256, 0, h->st>>>(C, h->kx, h->ky, h->kz, h->cu[2], 2, s1);
  DG_LAUNCHED();
  const double2 *pr[2] = {s0, s1};
  DG_TRY(per_to_physical(h, pr, 2, W));
  double *P = W + 2 * n;
  dg_kt_begin(h, "k_pp_first", h->st);
  k_pp_first<<<4 * 148, 256, 0, h->st>>>(n, W, W + n, P);
  DG_LAUNCHED();
  // copy P aside (W is reused), then the six gradient products
  double *Psave = (double *)h->P;  // enough room: P holds nmax * h_field complex values
  DG_CUDA(cudaMemcpyAsync(Psave, P, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->st));
  struct G { int src, axis; } g[6] = {{0, 1}, {1, 0}, {0, 2}, {2, 0}, {1, 2}, {2, 1}};
  for (int k = 0; k < 6; k += 2) {
    dg_kt_begin(h, "k_ik", h->st);
    k_ik<<<dim3(dg_cdiv(h->ss, 256), h->nkyt), 256, 0, h->st>>>(C, h->kx, h->ky, h->kz, h->cu[g[k].src], g[k].axis, s0);
    DG_LAUNCHED();
    dg_kt_begin(h, "k_ik", h->st);
    k_ik<<<dim3(dg_cdiv(h->ss, 256), h->nkyt), 256, 0, h->st>>>(C, h->kx, h->ky, h->kz, h->cu[g[k + 1].src],
                                               g[k + 1].axis, s1);
    DG_LAUNCHED();
    DG_TRY(per_to_physical(h, pr, 2, W + k * n));
  }
  dg_kt_begin(h, "k_pp_second", h->st);
  k_pp_second<<<4 * 148, 256, 0, h->st>>>(n, W, Psave);
  DG_LAUNCHED();
  DG_CUDA(cudaMemcpyAsync(W, Psave, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->st));
  double2 *out[1] = {h->cp};
  DG_TRY(per_to_fourier(h, W, 1, out));
  dg_kt_begin(h, "k_pp_solve", h->st);
  k_pp_solve<<<dim3(dg_cdiv(h->ss, 256), h->nkyt), 256, 0, h->st>>>(C, h->kx, h->ky, h->kz, h->cp);
  DG_LAUNCHED();
  return DG_OK;
}

// Parseval sums over the retained modes: tot[0..2] = <U_d^2>, tot[3+n] =
// variance of TH_n; returns DG_ERR_NAN if the state holds a non-finite value.
static int per_sums(dg_handle *h, double tot[8]) {
  const PerConst C = make_pc(h);
  double *dsum = (double *)h->work;
  CFieldPtrs u;
  for (int f = 0; f < h->nf; f++) u.p[f] = h->cu[f];
  DG_CUDA(cudaMemsetAsync(h->dflag, 0, sizeof(int), h->st));
  dg_kt_begin(h, "k_per_sums", h->st);
  k_per_sums<<<h->nkyt, 256, 0, h->st>>>(C, u, dsum, h->dflag);
  DG_LAUNCHED();
  double *hs = (double *)malloc(sizeof(double) * 8 * h->nkyt);
  int flag = 0;
  cudaMemcpyAsync(hs, dsum, sizeof(double) * 8 * h->nkyt, cudaMemcpyDeviceToHost, h->st);
  cudaMemcpyAsync(&flag, h->dflag, sizeof(int), cudaMemcpyDeviceToHost, h->st);
  cudaError_t e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) {
    free(hs);
    DG_CUDA(e);
  }
  for (int k = 0; k < 8; k++) tot[k] = 0.0;
  for (int j = 0; j < h->nkyt; j++)
    for (int k = 0; k < 8; k++) tot[k] += hs[8 * j + k];
  free(hs);
  if (flag) {
    dg_set_error("non-finite value in the periodic state");
    return DG_ERR_NAN;
  }
  return DG_OK;
}

int dg_per_stats(dg_handle *h, dg_stats *s) {
  const PerConst C = make_pc(h);
  double tot[8];
  const int rc = per_sums(h, tot);
  if (rc != DG_OK && rc != DG_ERR_NAN) return rc;
  const int flag = (rc == DG_ERR_NAN);
  memset(s, 0, sizeof(*s));
  s->urms_b = sqrt(tot[0]);
  s->vrms_b = sqrt(tot[1]);
  s->wrms_b = sqrt(tot[2]);
  s->ke = 0.5 * (tot[0] + tot[1] + tot[2]);
  for (int n = 0; n < h->NTH && n < DG_MAX_TH; n++) {
    s->th_var[n] = tot[3 + n];
    s->thrms_b[n] = sqrt(tot[3 + n]);
  }
  // max |div u| in physical space
  const long tot_m = (long)h->nkyt * h->ss;
  dg_kt_begin(h, "k_div_per", h->st);
  k_div_per<<<dim3(dg_cdiv(h->ss, 256), h->nkyt), 256, 0, h->st>>>(C, h->kx, h->ky, h->kz, h->cu[0], h->cu[1],
                                                    h->cu[2], h->rhs[0]);
  DG_LAUNCHED();
  const double2 *d[1] = {h->rhs[0]};
  double *W = (double *)h->work;
  DG_TRY(per_to_physical(h, d, 1, W));
  DG_CUDA(cudaMemsetAsync(h->dmin_bits, 0, sizeof(unsigned long long), h->st));
  dg_kt_begin(h, "k_absmax_p", h->st);
  k_absmax_p<<<4 * 148, 256, 0, h->st>>>(W, phys_field(h), h->dmin_bits);
  DG_LAUNCHED();
  unsigned long long bits = 0;
  DG_CUDA(cudaMemcpyAsync(&bits, h->dmin_bits, sizeof(bits), cudaMemcpyDeviceToHost, h->st));
  DG_CUDA(cudaStreamSynchronize(h->st));
  memcpy(&s->div_max, &bits, sizeof(double));
  return flag ? DG_ERR_NAN : DG_OK;
}

namespace {

// retained modes [nkyt][nkzt][nkxp] <-> reference array CU(0:NX/2,0:NZ+1,0:NY+1)
__global__ void k_xzy_compact_to_ref(const double2 *__restrict__ cmp, double2 *__restrict__ ref,
                                     int nky2, int nkyt, int nzt, int nkxp, int nxp1, int nz2) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)nky2 * nz2 * nxp1) return;
  const int i = (int)(q % nxp1);
  const int k = (int)((q / nxp1) % nz2);
  const int j = (int)(q / ((long)nxp1 * nz2));
  double2 v = make_double2(0.0, 0.0);
  if (i < nkxp && k < nzt && j < nkyt) v = cmp[((long)j * nzt + k) * nkxp + i];
  ref[q] = v;
}

__global__ void k_xzy_ref_to_compact(const double2 *__restrict__ ref, double2 *__restrict__ cmp,
                                     int nkyt, int nzt, int nkxp, int nxp1, int nz2) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)nkyt * nzt * nkxp) return;
  const int i = (int)(q % nkxp);
  const int k = (int)((q / nkxp) % nzt);
  const int j = (int)(q / ((long)nkxp * nzt));
  cmp[q] = ref[((long)j * nz2 + k) * nxp1 + i];
}

// one reference-layout array on the device: the caller's, or a staged copy
struct RefBuf {
  double *d = nullptr;
  bool owned = false;
};

int ref_acquire(dg_handle *h, const double *src, int where, size_t bytes, RefBuf *b) {
  if (where == DG_DEVICE) {
    b->d = (double *)src;
    return DG_OK;
  }
  DG_CUDA(cudaMallocAsync((void **)&b->d, bytes, h->st));
  b->owned = true;
  DG_CUDA(cudaMemcpyAsync(b->d, src, bytes, cudaMemcpyHostToDevice, h->st));
  return DG_OK;
}

int ref_release(dg_handle *h, RefBuf *b, double *dst, int where, size_t bytes) {
  if (where == DG_HOST) {
    cudaError_t e = cudaMemcpyAsync(dst, b->d, bytes, cudaMemcpyDeviceToHost, h->st);
    cudaFreeAsync(b->d, h->st);
    DG_CUDA(e);
    DG_CUDA(cudaStreamSynchronize(h->st));
  }
  return DG_OK;
}

}  // namespace

// FFT_XZY_TO_FOURIER(U, CU) (for/fft.f:223-258) on reference-layout arrays
// U(0:NX+1,0:NZ+1,0:NY+1) and CU(0:NX/2,0:NZ+1,0:NY+1); U and CU may alias.
// Retained modes land at CU(0:NKX,0:TNKZ,0:TNKY); every other slot is zeroed.
extern "C" int diablo_fft_xzy_to_fourier(dg_handle *h, const double *U, double *CU, int where) {
  if (!h || !h->periodic || !U || !CU || (where != DG_HOST && where != DG_DEVICE)) return DG_ERR_ARG;
  const int nxp2 = h->NX + 2, nz2 = h->NZ + 2, ny2 = h->NY + 2;
  const size_t bytes = sizeof(double) * (size_t)nxp2 * nz2 * ny2;
  RefBuf b;
  DG_TRY(ref_acquire(h, U, where, bytes, &b));
  double2 *tmp[1] = {h->rhs[0]};
  int s = per_to_fourier(h, b.d, 1, 0, (long)nz2 * nxp2, nxp2, tmp);
  double *out = (where == DG_DEVICE) ? CU : b.d;
  if (s == DG_OK) {
    const long tot = (long)ny2 * nz2 * (nxp2 / 2);
    dg_kt_begin(h, "k_xzy_compact_to_ref", h->st);
    k_xzy_compact_to_ref<<<dg_cdiv(tot, 256), 256, 0, h->st>>>(h->rhs[0], (double2 *)out, ny2,
                                                                h->nkyt, h->nkzt, h->nkxp,
                                                                nxp2 / 2, nz2);
    dg_count_launch();
    if (cudaGetLastError() != cudaSuccess) s = DG_ERR_CUDA;
  }
  if (b.owned) {
    const int r = ref_release(h, &b, CU, where, bytes);
    if (s == DG_OK) s = r;
  }
  return s;
}

// FFT_XZY_TO_PHYSICAL(CU, U) (for/fft.f:261-299), same layouts; CU and U may
// alias.  Points outside 0:NX-1, 0:NZ-1, 0:NY-1 are zeroed.
extern "C" int diablo_fft_xzy_to_physical(dg_handle *h, const double *CU, double *U, int where) {
  if (!h || !h->periodic || !U || !CU || (where != DG_HOST && where != DG_DEVICE)) return DG_ERR_ARG;
  const int nxp2 = h->NX + 2, nz2 = h->NZ + 2, ny2 = h->NY + 2;
  const size_t bytes = sizeof(double) * (size_t)nxp2 * nz2 * ny2;
  RefBuf b;
  DG_TRY(ref_acquire(h, CU, where, bytes, &b));
  const long tot = (long)h->nkyt * h->ss;
  dg_kt_begin(h, "k_xzy_ref_to_compact", h->st);
  k_xzy_ref_to_compact<<<dg_cdiv(tot, 256), 256, 0, h->st>>>((const double2 *)b.d, h->rhs[0],
                                                              h->nkyt, h->nkzt, h->nkxp, nxp2 / 2,
                                                              nz2);
  dg_count_launch();
  int s = (cudaGetLastError() == cudaSuccess) ? DG_OK : DG_ERR_CUDA;
  double *out = (where == DG_DEVICE) ? U : b.d;
  if (s == DG_OK && cudaMemsetAsync(out, 0, bytes, h->st) != cudaSuccess) s = DG_ERR_CUDA;
  if (s == DG_OK) {
    const double2 *in[1] = {h->rhs[0]};
    s = per_to_physical(h, in, 1, out, 0, (long)nz2 * nxp2, nxp2);
  }
  if (b.owned) {
    const int r = ref_release(h, &b, U, where, bytes);
    if (s == DG_OK) s = r;
  }
  return s;
}
