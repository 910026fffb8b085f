// SAVE_STATS_CHAN (for/save_stats.f:4-690) and tkebudget_chan
// (for/save_stats.f:963-1173) on the device, channel only.
//
// Every statistic of those routines is a plane mean of a product of two
// fields that are x-z Fourier series over the retained modes: the velocity,
// the scalars, their x and z derivatives and their finite-difference y
// derivatives.  By the discrete Parseval identity, the mean of a.b over the
// NX x NZ points equals sum_k w_k Re(a_k conj(b_k)) over the retained modes
// (w = 1 for kx = 0, 2 for kx > 0; a physical field sees only the real part
// of its (0,0) coefficient).  So instead of the reference's 12 + 4 N_TH
// inverse transforms of the whole field, one kernel makes a single pass over
// the spectral state and forms every plane sum; the host turns the sums into
// the profiles (square roots, grid factors, the interpolation onto GY).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dg_internal.cuh"

namespace {

// raw plane sums (rows of the [NR][NY+2] output)
enum {
  R_UME, R_VME, R_WME, R_CP,  // Re of the (0,0) mode
  R_A11, R_A22, R_A33,        // |u_i'|^2
  R_X12, R_X12M, R_X32, R_X32M, R_X13,  // u1'(j) u2'(j), u1'(j-1) u2'(j), ..., u1' u3'
  R_SH,                       // |u1(j+1)-u1(j-1)|^2 + |u3(j+1)-u3(j-1)|^2
  R_OX, R_OY, R_OZ,           // |omega_i|^2
  R_EUX, R_EVX, R_EWX, R_EUZ, R_EVZ, R_EWZ,  // kx^2 |u_i|^2, kz^2 |u_i|^2
  R_EUY, R_EWY,               // |u'(j) - u'(j-1)|^2 (u1, u3)
  R_EVY,                      // |u2(j+1) - u2(j-1)|^2 with the reference's mean shift
  R_NV
};
// per scalar n, from row R_NV + 5 n: THME, |th'|^2, th' v', (kx^2+kz^2)|th|^2,
// |th(j+1) - th(j-1)|^2
enum { T_ME, T_A, T_V, T_K, T_Y, T_N };

constexpr int ST_THR = 256;
constexpr int ST_MAXR = R_NV + T_N * DG_MAX_TH;

struct c2 {
  double x, y;
};
__device__ __forceinline__ c2 ld(const double2 *p) {
  const double2 v = __ldg(p);
  return {v.x, v.y};
}
__device__ __forceinline__ c2 sub(c2 a, c2 b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ c2 add(c2 a, c2 b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ c2 scl(c2 a, double s) { return {a.x * s, a.y * s}; }
__device__ __forceinline__ c2 mul_i(c2 a, double k) { return {-k * a.y, k * a.x}; }  // i k a
__device__ __forceinline__ double n2(c2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double dotr(c2 a, c2 b) { return a.x * b.x + a.y * b.y; }  // Re(a conj b)

// One CTA per plane j = 0..NY+1.  Planes 0 and NY+1 form only what the
// host reads there (the means; |u2'|^2 on NY+1 for vrms on NY).
__global__ void __launch_bounds__(ST_THR) k_stats_prof(int NY, long ss, int nkxp, int nth,
                                                      CFieldPtrs u, const double2 *__restrict__ cp,
                                                      const double *__restrict__ kxv,
                                                      const double *__restrict__ kzv,
                                                      const double *__restrict__ dyf,
                                                      double *__restrict__ raw) {
  const int j = blockIdx.x;
  const int L = NY + 2;
  const int nr = R_NV + T_N * nth;
  const bool inner = (j >= 1 && j <= NY);
  double acc[ST_MAXR];
#pragma unroll
  for (int r = 0; r < ST_MAXR; r++) acc[r] = 0.0;
  const double i2f = inner ? 1.0 / (2.0 * dyf[j]) : 0.0;
  const double2 *U1 = u(0), *U2 = u(1), *U3 = u(2);
  for (long m = threadIdx.x; m < ss; m += ST_THR) {
    const int i = (int)(m % nkxp), k = (int)(m / nkxp);
    const double w = (i == 0) ? 1.0 : 2.0;
    const bool mean = (m == 0);
    const long o = (long)j * ss + m;
    // the physical fields see only the real part of the (0,0) coefficient
    auto val = [&](const double2 *f, long q) {
      c2 v = ld(f + q);
      if (mean) v.y = 0.0;
      return v;
    };
    auto fl = [&](c2 v) { return mean ? c2{0.0, 0.0} : v; };  // mean removed
    const c2 a2 = val(U2, o);
    if (mean) {
      acc[R_UME] = ld(U1 + o).x;
      acc[R_VME] = a2.x;
      acc[R_WME] = ld(U3 + o).x;
      acc[R_CP] = ld(cp + o).x;
#pragma unroll
      for (int n = 0; n < DG_MAX_TH; n++)
        if (n < nth) acc[R_NV + T_N * n + T_ME] = ld(u(3 + n) + o).x;
    }
    acc[R_A22] += w * n2(fl(a2));
    if (!inner) continue;
    const double KX = kxv[i], KZ = kzv[k];
    const c2 a1 = val(U1, o), a3 = val(U3, o);
    const c2 a1m = val(U1, o - ss), a1p = val(U1, o + ss);
    const c2 a2m = val(U2, o - ss), a2p = val(U2, o + ss);
    const c2 a3m = val(U3, o - ss), a3p = val(U3, o + ss);
    const c2 f1 = fl(a1), f2 = fl(a2), f3 = fl(a3), f1m = fl(a1m), f3m = fl(a3m);
    acc[R_A11] += w * n2(f1);
    acc[R_A33] += w * n2(f3);
    acc[R_X12] += w * dotr(f1, f2);
    acc[R_X12M] += w * dotr(f1m, f2);
    acc[R_X32] += w * dotr(f3, f2);
    acc[R_X32M] += w * dotr(f3m, f2);
    acc[R_X13] += w * dotr(f1, f3);
    acc[R_SH] += w * (n2(sub(a1p, a1m)) + n2(sub(a3p, a3m)));
    // omega_x = d(u3)/dy - d(u2)/dz, omega_y = du1/dz - du3/dx,
    // omega_z = du2/dx - du1/dy, with u2 averaged onto GYF
    // (for/save_stats.f:268-272,296-300,324-329)
    const c2 v2 = scl(add(a2p, a2), 0.5);
    acc[R_OX] += w * n2(sub(scl(sub(a3p, a3m), i2f), mul_i(v2, KZ)));
    acc[R_OY] += w * n2(sub(mul_i(a1, KZ), mul_i(a3, KX)));
    acc[R_OZ] += w * n2(sub(mul_i(v2, KX), scl(sub(a1p, a1m), i2f)));
    const double kx2 = KX * KX, kz2 = KZ * KZ;
    acc[R_EUX] += w * kx2 * n2(a1);
    acc[R_EVX] += w * kx2 * n2(a2);
    acc[R_EWX] += w * kx2 * n2(a3);
    acc[R_EUZ] += w * kz2 * n2(a1);
    acc[R_EVZ] += w * kz2 * n2(a2);
    acc[R_EWZ] += w * kz2 * n2(a3);
    acc[R_EUY] += w * n2(sub(f1, f1m));
    acc[R_EWY] += w * n2(sub(f3, f3m));
    // tkebudget_chan's dv/dy subtracts VME(j) from U2(j+1) and VME(j-1) from
    // U2(j-1) (for/save_stats.f:1094-1097): its mean is VME(j+1) - VME(j)
    const c2 dv = mean ? c2{a2p.x - a2.x, 0.0} : sub(a2p, a2m);
    acc[R_EVY] += w * n2(dv);
    const c2 v2f = scl(add(f2, fl(a2p)), 0.5);
#pragma unroll
    for (int n = 0; n < DG_MAX_TH; n++) {
      if (n >= nth) break;
      const double2 *T = u(3 + n);
      const c2 t = val(T, o), tm = val(T, o - ss), tp = val(T, o + ss);
      acc[R_NV + T_N * n + T_A] += w * n2(fl(t));
      acc[R_NV + T_N * n + T_V] += w * dotr(fl(t), v2f);
      acc[R_NV + T_N * n + T_K] += w * (kx2 + kz2) * n2(t);
      acc[R_NV + T_N * n + T_Y] += w * n2(sub(tp, tm));
    }
  }
  // block reduction: warp shuffles, then one row of partial sums per warp
  __shared__ double part[ST_THR / 32][ST_MAXR];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int r = 0; r < ST_MAXR; r++) {
    double v = acc[r];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) part[wid][r] = v;
  }
  __syncthreads();
  if (threadIdx.x < nr) {
    double v = 0.0;
    for (int q = 0; q < ST_THR / 32; q++) v += part[q][threadIdx.x];
    raw[(long)threadIdx.x * L + j] = v;
  }
}

double integ_y(const dg_handle *h, const double *v) {
  // INTEGRATE_Y_VAR (for/mpi.f:1676-1698)
  double res = 0.;
  for (int j = 2; j <= h->NY; j++) res = res + 0.5 * (v[j] + v[j - 1]) * h->h_dy[j];
  return res / h->p.ly;
}

}  // namespace

extern "C" int diablo_save_stats_chan(dg_handle *h, double *prof, double *prof_th, double *bulk) {
  if (!h || h->periodic || !prof || !bulk || (h->NTH > 0 && !prof_th)) return DG_ERR_ARG;
  const int NY = h->NY, L = NY + 2, NTH = h->NTH;
  const int nr = R_NV + T_N * NTH;
  DG_TRY(dg_apply_bc_vel_dev(h));
  double *raw = nullptr;
  DG_CUDA(dg_malloc(h, (void **)&raw, sizeof(double) * nr * L));
  CFieldPtrs u;
  for (int f = 0; f < h->nf; f++) u.p[f] = h->cu[f];
  dg_kt_begin(h, "k_stats_prof", h->st);
  k_stats_prof<<<L, ST_THR, 0, h->st>>>(NY, h->ss, h->nkxp, NTH, u, h->cp, h->kx, h->kz, h->dyf,
                                        raw);
  cudaError_t e = cudaGetLastError();
  dg_count_launch();
  double *R = (double *)malloc(sizeof(double) * nr * L);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(R, raw, sizeof(double) * nr * L, cudaMemcpyDeviceToHost, h->st);
  dg_free(h, raw);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  if (e != cudaSuccess) {
    free(R);
    dg_set_error((std::string("statistics: ") + cudaGetErrorString(e)).c_str());
    return DG_ERR_CUDA;
  }
  const double *DY = h->h_dy, *DYF = h->h_dyf, *GYF = h->h_gyf, *GY = h->h_gy;
#define RW(r, j) R[(long)(r) * L + (j)]
#define PR(q, j) prof[(long)(q) * L + (j)]
  memset(prof, 0, sizeof(double) * DG_PR_COUNT * L);
  for (int j = 0; j < L; j++) {
    PR(DG_PR_UME, j) = RW(R_UME, j);
    PR(DG_PR_VME, j) = RW(R_VME, j);
    PR(DG_PR_WME, j) = RW(R_WME, j);
    PR(DG_PR_CP, j) = RW(R_CP, j);
  }
  for (int j = 1; j <= NY; j++) {
    PR(DG_PR_URMS, j) = sqrt(RW(R_A11, j));
    PR(DG_PR_VRMS, j) = sqrt(0.5 * (RW(R_A22, j) + RW(R_A22, j + 1)));
    PR(DG_PR_WRMS, j) = sqrt(RW(R_A33, j));
    PR(DG_PR_UV, j) = (DYF[j - 1] * RW(R_X12, j) + DYF[j] * RW(R_X12M, j)) / (2.0 * DY[j]);
    PR(DG_PR_WV, j) = (DYF[j - 1] * RW(R_X32, j) + DYF[j] * RW(R_X32M, j)) / (2.0 * DY[j]);
    PR(DG_PR_UW, j) = RW(R_X13, j);
    PR(DG_PR_DUDY, j) = (RW(R_UME, j) - RW(R_UME, j - 1)) / (GYF[j] - GYF[j - 1]);
    PR(DG_PR_DWDY, j) = (RW(R_WME, j) - RW(R_WME, j - 1)) / (GYF[j] - GYF[j - 1]);
    PR(DG_PR_SHEAR, j) = RW(R_SH, j) / ((2.0 * DYF[j]) * (2.0 * DYF[j]));
    PR(DG_PR_OMEGA_X, j) = sqrt(RW(R_OX, j));
    PR(DG_PR_OMEGA_Y, j) = sqrt(RW(R_OY, j));
    PR(DG_PR_OMEGA_Z, j) = sqrt(RW(R_OZ, j));
  }
  // pseudo-dissipation on GY, rows the reference writes (tke.txt)
  auto interp = [&](int r, int j) {
    return (DYF[j - 1] * RW(r, j) + DYF[j] * RW(r, j - 1)) / (2.0 * DY[j]);
  };
  for (int j = 2; j <= NY - 1; j++) {
    const double gy2 = (GY[j + 1] - GY[j - 1]) * (GY[j + 1] - GY[j - 1]);
    double e = interp(R_EUX, j) + RW(R_EVX, j) + RW(R_EUY, j) / (DY[j] * DY[j]) +
               interp(R_EWX, j) + interp(R_EUZ, j) + RW(R_EVY, j) / gy2 +
               RW(R_EWY, j) / (DY[j] * DY[j]) + RW(R_EVZ, j) + interp(R_EWZ, j);
    PR(DG_PR_EPSILON, j) = h->p.nu * e;
  }
  double *tmp = (double *)calloc(L, sizeof(double));
  for (int j = 0; j < L; j++) tmp[j] = PR(DG_PR_UME, j);
  bulk[0] = integ_y(h, tmp);
  const int jh = NY / 2;
  bulk[1] = (NY % 2 == 0) ? RW(R_UME, jh) : 0.5 * (RW(R_UME, jh - 1) + RW(R_UME, jh));
  for (int c = 0; c < 3; c++) {
    for (int j = 0; j < L; j++) tmp[j] = PR(DG_PR_URMS + c, j);
    bulk[2 + c] = integ_y(h, tmp);
  }
  free(tmp);
  for (int n = 0; n < NTH; n++) {
    double *T = prof_th + (long)n * DG_PRT_COUNT * L;
    memset(T, 0, sizeof(double) * DG_PRT_COUNT * L);
    const int b = R_NV + T_N * n;
    for (int j = 0; j < L; j++) T[DG_PRT_THME * L + j] = RW(b + T_ME, j);
    for (int j = 1; j <= NY; j++) {
      T[DG_PRT_THRMS * L + j] = sqrt(RW(b + T_A, j));
      T[DG_PRT_THV * L + j] = RW(b + T_V, j);
      T[DG_PRT_DTHDY * L + j] = (RW(b + T_ME, j) - RW(b + T_ME, j - 1)) / (GYF[j] - GYF[j - 1]);
      const double g = GYF[j + 1] - GYF[j - 1];
      T[DG_PRT_PE_DISS * L + j] = RW(b + T_K, j) + RW(b + T_Y, j) / (g * g);
    }
  }
  // running means (for/save_stats.f:99-114); the weights are REAL*4
  // expressions: 1./FLOAT(NSAMPLES) and (FLOAT(NSAMPLES)-1.)/FLOAT(NSAMPLES)
  if (!h->h_ubar) h->h_ubar = (double *)calloc((size_t)(3 + NTH) * L, sizeof(double));
  h->nsamples++;
  const float fn = (float)h->nsamples;
  const double w1 = (double)(1.0f / fn), w2 = (double)((fn - 1.0f) / fn);
  for (int j = 1; j <= NY; j++) {
    for (int c = 0; c < 3; c++)
      h->h_ubar[c * L + j] = w1 * RW(R_UME + c, j) + w2 * h->h_ubar[c * L + j];
    for (int n = 0; n < NTH; n++)
      h->h_ubar[(3 + n) * L + j] = w1 * RW(R_NV + T_N * n + T_ME, j) + w2 * h->h_ubar[(3 + n) * L + j];
  }
#undef RW
#undef PR
  free(R);
  return DG_OK;
}

extern "C" int diablo_stats_means(dg_handle *h, double *ubar, double *vbar, double *wbar,
                                  double *thbar, int *nsamples) {
  if (!h || h->periodic) return DG_ERR_ARG;
  const int L = h->NY + 2;
  double *src[3] = {ubar, vbar, wbar};
  for (int c = 0; c < 3; c++)
    if (src[c]) {
      if (h->h_ubar) memcpy(src[c], h->h_ubar + (long)c * L, sizeof(double) * L);
      else memset(src[c], 0, sizeof(double) * L);
    }
  if (thbar && h->NTH > 0) {
    if (h->h_ubar) memcpy(thbar, h->h_ubar + 3L * L, sizeof(double) * h->NTH * L);
    else memset(thbar, 0, sizeof(double) * h->NTH * L);
  }
  if (nsamples) *nsamples = h->nsamples;
  return DG_OK;
}
