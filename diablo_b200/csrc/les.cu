// Channel LES: constant Smagorinsky subgrid model (LES_MODEL_TYPE = 1, the
// only model the MPI build runs) inside RK_CHAN_1.
//
// The reference (for/les.f:1-275, for/channel.f:299-372,631-659,748-1029)
// computes S_ij in physical space, the eddy viscosity NU_T = C_S^2 DELTA^2 |S|
// at GY points, the SGS stress divergence (explicit, into CF), and moves the
// Crank-Nicolson solves to physical columns because NU_T varies in x and z.
// Here the substep keeps its fused spectral stages for everything the DNS
// does, and wraps them:
//   pre  : APPLY_BC_VEL + APPLY_BC_LES on CU, strain rates (spectral) -> S_ij
//          and U (physical), APPLY_BC_VEL_PHYS, one column pass for |S|, NU_T,
//          |S| S_ij and the NU_T dU/dy cross terms, forward transforms, the SGS
//          forcing G per field, the scalar eddy diffusion; the boundary planes
//          of CU get APPLY_BC_VEL_PHYS stated on the retained modes, so the
//          nonlinear stage sees what the reference's physical U holds;
//   (the fused z inverse / x-row products / z forward write CF and the
//    spectral right-hand side R as in the DNS)
//   post : CF += G, R += BETA_BAR H_BAR G; R, TH to physical; one thread per
//          physical column builds the CN rows with the eddy-viscosity terms and
//          the BC rows, runs the MPI Thomas sweeps and writes U / TH; COURANT on
//          that velocity; forward transforms to CU / CTH; REM_DIV_CHAN.
// Slots (physical): 0-5 S_ij (then R), 6-10 the |S| S_ij products, 11-12
// cross terms (products and cross terms adjacent: one transform batch), 13
// NU_T, 14-16 U1-U3, 17.. TH(n) (U and TH adjacent: one transform batch), then
// nf Thomas scratch (pivots b').
// Slots (spectral): 0-5 CS_ij (then the products, then scalar temporaries),
// 6-7 cross terms, 8.. G(f).
#include "dg_internal.cuh"

namespace {

constexpr int PS_S = 0, PS_P = 6, PS_X = 11, PS_NUT = 13, PS_U = 14, PS_TH = 17;
constexpr int SS_S = 0, SS_X = 6, SS_G = 8;
constexpr int LES_HF = 8;  // fields per transform launch (the pointer-array capacity)

inline int phys_slots(const dg_handle *h) { return PS_TH + h->NTH + h->nf; }
inline int spec_slots(const dg_handle *h) { return SS_G + h->nf; }
inline long pfield_of(const dg_handle *h) { return (long)(h->NY + 2) * h->NZ * h->NX; }
inline double *pslot(dg_handle *h, int s) { return h->les_phys + (long)s * pfield_of(h); }
inline double2 *sslot(dg_handle *h, int s) { return h->les_spec + (long)s * h->nspec; }

struct LesBc {
  int u_lo, w_lo, v_lo, u_hi, w_hi, v_hi;
  double u_lo_c1, w_lo_c1, v_lo_c1, u_hi_c1, w_hi_c1, v_hi_c1;
};

LesBc make_bc(const dg_params &p) {
  return {p.u_bc_ymin, p.w_bc_ymin, p.v_bc_ymin, p.u_bc_ymax, p.w_bc_ymax, p.v_bc_ymax,
          p.u_bc_ymin_c1, p.w_bc_ymin_c1, p.v_bc_ymin_c1, p.u_bc_ymax_c1, p.w_bc_ymax_c1,
          p.v_bc_ymax_c1};
}

// APPLY_BC_LES (for/les.f:805-865): Neumann walls copy the first interior
// plane of CU1 / CU3 into the wall and ghost planes.
__global__ void k_les_bc_spec(LesBc B, int NY, long ss, double2 *u1, double2 *u3) {
  const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= ss) return;
  if (B.u_hi == 1) {
    u1[NY * ss + m] = u1[(NY - 1) * ss + m];
    u1[(NY + 1) * ss + m] = u1[NY * ss + m];
  }
  if (B.w_hi == 1) {
    u3[NY * ss + m] = u3[(NY - 1) * ss + m];
    u3[(NY + 1) * ss + m] = u3[NY * ss + m];
  }
  if (B.u_lo == 1) {
    u1[ss + m] = u1[2 * ss + m];
    u1[m] = u1[ss + m];
  }
  if (B.w_lo == 1) {
    u3[ss + m] = u3[2 * ss + m];
    u3[m] = u3[ss + m];
  }
}

// APPLY_BC_VEL_PHYS_LOWER / _UPPER (for/channel.f:2495-2652) stated on the
// retained modes: the physical boundary planes are the neighbouring planes
// plus constants, so their transforms are the neighbouring modes plus the
// constants on the (0,0) mode.  This is the transform of what
// k_les_bc_phys leaves in the physical velocity, without a transform.
__global__ void k_les_bc_spec_phys(LesBc B, int NY, long ss, const double *__restrict__ dy,
                                   const double *__restrict__ dyf, double2 *u1, double2 *u2,
                                   double2 *u3) {
  const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= ss) return;
  const double on = (m == 0) ? 1.0 : 0.0;  // constants live on the (0,0) mode
  const long p0 = m, p1 = ss + m, p2 = 2 * ss + m;
  const long pm = (long)(NY - 1) * ss + m, pn = (long)NY * ss + m, pn1 = (long)(NY + 1) * ss + m;
  auto sh = [](double2 a, double c) { return make_double2(a.x + c, a.y); };
  if (B.u_lo == 0) {
    u1[p0] = make_double2(on * B.u_lo_c1, 0.0);
    u1[p1] = u1[p0];
  } else {
    u1[p1] = sh(u1[p2], -on * dy[2] * B.u_lo_c1);
    u1[p0] = sh(u1[p1], -on * dy[1] * B.u_lo_c1);
  }
  if (B.w_lo == 0) {
    u3[p0] = make_double2(on * B.w_lo_c1, 0.0);
    u3[p1] = u3[p0];
  } else {
    u3[p1] = sh(u3[p2], -on * dy[2] * B.w_lo_c1);
    u3[p0] = sh(u3[p1], -on * dy[1] * B.w_lo_c1);
  }
  if (B.v_lo == 0) {
    const double2 a = u2[p2];
    u2[p1] = make_double2(on * 2.0 * B.v_lo_c1 - a.x, -a.y);
    u2[p0] = u2[p1];
  } else {
    u2[p1] = sh(u2[p2], -on * dyf[1] * B.v_lo_c1);
    u2[p0] = sh(u2[p1], -on * dyf[1] * B.v_lo_c1);
  }
  if (B.u_hi == 0) {
    u1[pn] = make_double2(on * B.u_hi_c1, 0.0);
    u1[pn1] = u1[pn];
  } else {
    u1[pn] = sh(u1[pm], on * dy[NY] * B.u_hi_c1);
    u1[pn1] = sh(u1[pn], on * dy[NY] * B.u_hi_c1);
  }
  if (B.w_hi == 0) {
    u3[pn] = make_double2(on * B.w_hi_c1, 0.0);
    u3[pn1] = u3[pn];
  } else {
    u3[pn] = sh(u3[pm], on * dy[NY] * B.w_hi_c1);
    u3[pn1] = sh(u3[pn], on * dy[NY] * B.w_hi_c1);
  }
  if (B.v_hi == 0) {
    const double2 a = u2[pn];
    u2[pn1] = make_double2(on * 2.0 * B.v_hi_c1 - a.x, -a.y);
  } else {
    u2[pn1] = sh(u2[pn], on * dy[NY] * B.v_hi_c1);
  }
}

__device__ __forceinline__ double2 cmul_i(double k, double2 a) {  // (i k) a
  return make_double2(-k * a.y, k * a.x);
}

// compute_strain_chan (for/les.f:526-569) into six spectral slots, zero on
// the planes it does not write; the mean U1, U3 per plane for les_chan.
__global__ void k_les_strain(int NY, long ss, int nkxp, const double *__restrict__ kxv,
                             const double *__restrict__ kzv, const double *__restrict__ dy,
                             const double *__restrict__ dyf, const double2 *__restrict__ u1,
                             const double2 *__restrict__ u2, const double2 *__restrict__ u3,
                             double2 *__restrict__ cs, long nspec, double *__restrict__ ubar) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)(NY + 2) * ss) return;
  const int j = (int)(q / ss);
  const long m = q % ss;
  const double KX = kxv[m % nkxp], KZ = kzv[m / nkxp];
  const double2 z = make_double2(0.0, 0.0);
  double2 s0 = z, s1 = z, s2 = z, s3 = z, s4 = z, s5 = z;
  if (j >= 1 && j <= NY) {
    const double2 a1 = u1[q], a3 = u3[q], b2 = u2[q], b2p = u2[q + ss];
    s0 = cmul_i(KX, a1);
    s1 = make_double2((b2p.x - b2.x) / dyf[j], (b2p.y - b2.y) / dyf[j]);
    s2 = cmul_i(KZ, a3);
    const double2 t1 = cmul_i(KZ, a1), t3 = cmul_i(KX, a3);
    s4 = make_double2(0.5 * (t1.x + t3.x), 0.5 * (t1.y + t3.y));
  }
  if (j >= 1) {
    const double2 a1 = u1[q], a1m = u1[q - ss], a3 = u3[q], a3m = u3[q - ss], b2 = u2[q];
    const double2 k2 = cmul_i(KX, b2), k2z = cmul_i(KZ, b2);
    s3 = make_double2(0.5 * ((a1.x - a1m.x) / dy[j] + k2.x), 0.5 * ((a1.y - a1m.y) / dy[j] + k2.y));
    s5 = make_double2(0.5 * (k2z.x + (a3.x - a3m.x) / dy[j]), 0.5 * (k2z.y + (a3.y - a3m.y) / dy[j]));
  }
  cs[q] = s0;
  cs[nspec + q] = s1;
  cs[2 * nspec + q] = s2;
  cs[3 * nspec + q] = s3;
  cs[4 * nspec + q] = s4;
  cs[5 * nspec + q] = s5;
  if (m == 0) {
    ubar[j] = u1[q].x;
    ubar[NY + 2 + j] = u3[q].x;
  }
}

// APPLY_BC_VEL_PHYS_LOWER / _UPPER (for/channel.f:2495-2652) on the physical
// U1..U3 (slots at stride pfield).
__global__ void k_les_bc_phys(LesBc B, int NY, long np, long pfield, const double *__restrict__ dy,
                              const double *__restrict__ dyf, double *__restrict__ U) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  double *U1 = U, *U2 = U + pfield, *U3 = U + 2 * pfield;
  const long j0 = q, j1 = np + q, j2 = 2 * np + q;
  const long jm = (long)(NY - 1) * np + q, jn = (long)NY * np + q, jn1 = (long)(NY + 1) * np + q;
  if (B.u_lo == 0) {
    U1[j0] = B.u_lo_c1;
    U1[j1] = B.u_lo_c1;
  } else {
    U1[j1] = U1[j2] - dy[2] * B.u_lo_c1;
    U1[j0] = U1[j1] - dy[1] * B.u_lo_c1;
  }
  if (B.w_lo == 0) {
    U3[j0] = B.w_lo_c1;
    U3[j1] = B.w_lo_c1;
  } else {
    U3[j1] = U3[j2] - dy[2] * B.w_lo_c1;
    U3[j0] = U3[j1] - dy[1] * B.w_lo_c1;
  }
  if (B.v_lo == 0) {
    U2[j1] = 2.0 * B.v_lo_c1 - U2[j2];
    U2[j0] = U2[j1];
  } else {
    U2[j1] = U2[j2] - dyf[1] * B.v_lo_c1;
    U2[j0] = U2[j1] - dyf[1] * B.v_lo_c1;
  }
  if (B.u_hi == 0) {
    U1[jn] = B.u_hi_c1;
    U1[jn1] = B.u_hi_c1;
  } else {
    U1[jn] = U1[jm] + dy[NY] * B.u_hi_c1;
    U1[jn1] = U1[jn] + dy[NY] * B.u_hi_c1;
  }
  if (B.w_hi == 0) {
    U3[jn] = B.w_hi_c1;
    U3[jn1] = B.w_hi_c1;
  } else {
    U3[jn] = U3[jm] + dy[NY] * B.w_hi_c1;
    U3[jn1] = U3[jn] + dy[NY] * B.w_hi_c1;
  }
  if (B.v_hi == 0)
    U2[jn1] = 2.0 * B.v_hi_c1 - U2[jn];
  else
    U2[jn1] = U2[jn] + dy[NY] * B.v_hi_c1;
}

// The model, one thread per physical point (for/les.f:114-227): |S| at GYF
// for JSTART..JEND and at GY for 2..NY+1 from the raw S_ij of planes j-1,
// j, j+1; the products |S| S_ij written out of place (P: S11, S33, S12 at
// GY, S13, S23 at GY; raw where the reference leaves S_ij unscaled), NU_T at
// GY (zero on planes 1, 2, NY, NY+1: GHOST_LES_MPI for one rank) and the
// cross terms NU_T dU1/dy, NU_T dU3/dy on planes 2..NY.
__global__ void __launch_bounds__(256, 4)
    k_les_model(int NY, long np, long pfield, int JS, int JE, const double *__restrict__ dy,
                const double *__restrict__ dyf, const double *__restrict__ dfac,
                const double *__restrict__ ubar, const double *__restrict__ S,
                double *__restrict__ P, double *__restrict__ X, const double *__restrict__ U,
                double *__restrict__ NUT) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)(NY + 2) * np) return;
  const int j = (int)(t / np);
  const long o = t;
  const double *u1b = ubar, *u3b = ubar + NY + 2;
  const double *U1 = U, *U3 = U + 2 * pfield;
  // every load the point needs, issued together (the neighbouring planes
  // clamped to the point's own where the branches below do not use them),
  // so the thread waits on memory once
  const long m = (j >= 1) ? o - np : o, pn = (j <= NY) ? o + np : o;
  const double r0 = S[o], r1 = S[pfield + o], r2 = S[2 * pfield + o], r3 = S[3 * pfield + o];
  const double r4 = S[4 * pfield + o], r5 = S[5 * pfield + o];
  const double s0m = S[m], s1m = S[pfield + m], s2m = S[2 * pfield + m], s4m = S[4 * pfield + m];
  const double n3 = S[3 * pfield + pn], n5 = S[5 * pfield + pn];
  const double u1o = U1[o], u1m = U1[m], u3o = U3[o], u3m = U3[m];
  double p0 = r0, p2 = r2, p3 = r3, p4 = r4, p5 = r5;
  double tg = 0.0;  // |S| at GY
  if (j >= 2) {
    const double w = 2.0 * dy[j];
    const double b1 = (r0 * dyf[j - 1] + s0m * dyf[j]) / w;
    const double b4 = r3 - 0.5 * (u1b[j] - u1b[j - 1]) / dy[j];
    const double b5 = (r4 * dyf[j - 1] + s4m * dyf[j]) / w;
    const double b2 = (r1 * dyf[j - 1] + s1m * dyf[j]) / w;
    const double b6 = r5 - 0.5 * (u3b[j] - u3b[j - 1]) / dy[j];
    const double b3 = (r2 * dyf[j - 1] + s2m * dyf[j]) / w;
    tg = sqrt(2.0 * (b1 * b1) + 4.0 * (b4 * b4) + 4.0 * (b5 * b5) + 2.0 * (b2 * b2) +
              4.0 * (b6 * b6) + 2.0 * (b3 * b3));
    const double du1 = 0.5 * (u1o - u1m) / dy[j];
    const double du3 = 0.5 * (u3o - u3m) / dy[j];
    p3 = tg * (r3 - du1);
    p5 = tg * (r5 - du3);
  }
  if (j >= JS && j <= JE) {
    const double a4 = 0.5 * (n3 + r3 - 0.5 * (u1b[j] - u1b[j - 1]) / dy[j] -
                             0.5 * (u1b[j + 1] - u1b[j]) / dy[j + 1]);
    const double a6 = 0.5 * (n5 + r5 - 0.5 * (u3b[j] - u3b[j - 1]) / dy[j] -
                             0.5 * (u3b[j + 1] - u3b[j]) / dy[j + 1]);
    const double sf = sqrt(2.0 * (r0 * r0) + 4.0 * (a4 * a4) + 4.0 * (r4 * r4) +
                           2.0 * (r1 * r1) + 4.0 * (a6 * a6) + 2.0 * (r2 * r2));
    p0 = sf * r0;
    p4 = sf * r4;
    p2 = sf * r2;
  }
  P[o] = p0;
  P[pfield + o] = p2;
  P[2 * pfield + o] = p3;
  P[3 * pfield + o] = p4;
  P[4 * pfield + o] = p5;
  if (j >= 1) {
    const double nut = (j >= 3 && j <= NY - 1) ? -0.5 * dfac[NY + 2 + j] * tg : 0.0;
    NUT[o] = nut;
    if (j >= 2 && j <= NY) {
      X[o] = nut * (u1o - u1m) / dy[j];
      X[pfield + o] = nut * (u3o - u3m) / dy[j];
    }
  }
}

// SGS stress divergence per field (for/les.f:236-333) from the transformed
// |S| S_ij (slots 0, 2-5) and cross terms (slots 6-7), with the filter-width
// factors applied as the reference scales CS_ij.  G1, G3 on J1..J2 = JSTART..
// NY-1, G2 on 2..NY, zero elsewhere.
__global__ void k_les_force(int NY, long ss, int nkxp, int JS, const double *__restrict__ kxv,
                            const double *__restrict__ kzv, const double *__restrict__ dyf,
                            const double *__restrict__ dfac, const double2 *__restrict__ cs,
                            long nspec, double2 *__restrict__ g) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)(NY + 2) * ss) return;
  const int j = (int)(q / ss);
  const long m = q % ss;
  const double KX = kxv[m % nkxp], KZ = kzv[m / nkxp];
  const double *ff = dfac, *fy = dfac + NY + 2;
  const double2 *C0 = cs, *C2 = cs + 2 * nspec, *C3 = cs + 3 * nspec, *C4 = cs + 4 * nspec;
  const double2 *C5 = cs + 5 * nspec, *X1 = cs + 6 * nspec, *X3 = cs + 7 * nspec;
  auto sc = [](double f, double2 a) { return make_double2(f * a.x, f * a.y); };
  double2 g1 = make_double2(0.0, 0.0), g2 = g1, g3 = g1;
  if (j >= JS && j <= NY - 1) {
    const double2 t1 = sc(ff[j], C0[q]), t5 = sc(ff[j], C4[q]), t3 = sc(ff[j], C2[q]);
    const double2 t4 = sc(fy[j], C3[q]), t4p = sc(fy[j + 1], C3[q + ss]);
    const double2 t6 = sc(fy[j], C5[q]), t6p = sc(fy[j + 1], C5[q + ss]);
    const double2 a = cmul_i(KX, t1), b = cmul_i(KZ, t5);
    g1.x = -a.x - (t4p.x - t4.x) / dyf[j] - b.x;
    g1.y = -a.y - (t4p.y - t4.y) / dyf[j] - b.y;
    const double2 c = cmul_i(KX, t5), d = cmul_i(KZ, t3);
    g3.x = -c.x - (t6p.x - t6.x) / dyf[j] - d.x;
    g3.y = -c.y - (t6p.y - t6.y) / dyf[j] - d.y;
  }
  if (j >= 2 && j <= NY) {
    const double2 a = cmul_i(KX, sc(fy[j], C3[q])), b = cmul_i(KZ, sc(fy[j], C5[q]));
    const double2 c = cmul_i(KX, X1[q]), d = cmul_i(KZ, X3[q]);
    g2.x = -a.x - b.x + c.x + d.x;
    g2.y = -a.y - b.y + c.y + d.y;
  }
  g[q] = g1;
  g[nspec + q] = g2;
  g[2 * nspec + q] = g3;
}

// Plane means for mean_les (for/les.f:336-459), one block per plane:
// NU_T_MEAN and EPS_SGS1_MEAN = <F1 U1 + F3 U3 + F2 U2>, F the SGS stress
// divergence in physical space (slots at stride pfield, U likewise).
__global__ void k_les_means(long np, long pfield, const double *__restrict__ F,
                            const double *__restrict__ U, const double *__restrict__ nut,
                            double *__restrict__ out, int L) {
  const int j = blockIdx.x;
  const long base = (long)j * np;
  double a = 0.0, b = 0.0;
  for (long q = threadIdx.x; q < np; q += blockDim.x) {
    const long o = base + q;
    a += F[o] * U[o] + F[2 * pfield + o] * U[2 * pfield + o] + F[pfield + o] * U[pfield + o];
    b += nut[o];
  }
  __shared__ double sa[256], sb[256];
  sa[threadIdx.x] = a;
  sb[threadIdx.x] = b;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      sa[threadIdx.x] += sa[threadIdx.x + w];
      sb[threadIdx.x] += sb[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[j] = sb[0] / (double)np;
    out[L + j] = sa[0] / (double)np;
  }
}

// tkebudget_chan_les (for/save_stats.f:887-964): per plane J = 1..NY the sum
// over its points of U1 d(NU_T dU1/dy)/dy + U3 (same) + U2 d(NU_T dU2/dy)/dy
// on GY, one block per plane.  DYF(0) is 0 as in the reference (never set),
// so plane 1's U2 term is 0/0 there and here.
__global__ void k_les_tke(int NY, long np, long pfield, const double *__restrict__ dy,
                          const double *__restrict__ dyf, const double *__restrict__ U,
                          const double *__restrict__ nut, double *__restrict__ out) {
  const int j = 1 + blockIdx.x;
  const double *U1 = U, *U2 = U + pfield, *U3 = U + 2 * pfield;
  double a = 0.0;
  for (long q = threadIdx.x; q < np; q += blockDim.x) {
    const long c = (long)j * np + q, p = c + np, m = c - np;
    a += U1[c] * ((nut[p] * (U1[p] - U1[c]) / dy[j + 1] - nut[c] * (U1[c] - U1[m]) / dy[j]) /
                  dyf[j]) +
         U3[c] * ((nut[p] * (U3[p] - U3[c]) / dy[j + 1] - nut[c] * (U3[c] - U3[m]) / dy[j]) /
                  dyf[j]) +
         U2[c] * ((0.5 * (nut[c] + nut[p]) * (U2[p] - U2[c]) / dyf[j] -
                   0.5 * (nut[c] + nut[m]) * (U2[c] - U2[m]) / dyf[j - 1]) /
                  dy[j]);
  }
  __shared__ double sa[256];
  sa[threadIdx.x] = a;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) sa[threadIdx.x] += sa[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[j] = sa[0];
}

// i kx CTH and i kz CTH on planes 1..NY+1 (for/channel.f:326-355)
__global__ void k_les_th_grad(int NY, long ss, int nkxp, const double *__restrict__ kxv,
                              const double *__restrict__ kzv, const double2 *__restrict__ th,
                              double2 *__restrict__ out, long nspec) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)(NY + 2) * ss) return;
  const int j = (int)(q / ss);
  const long m = q % ss;
  double2 a = make_double2(0.0, 0.0), b = a;
  if (j >= 1) {
    a = cmul_i(kxv[m % nkxp], th[q]);
    b = cmul_i(kzv[m / nkxp], th[q]);
  }
  out[q] = a;
  out[nspec + q] = b;
}

// KAPPA_T = NU_T times both physical gradients on planes 1..NY+1
__global__ void k_les_th_scale(int NY, long np, long pfield, const double *__restrict__ nut,
                               double *__restrict__ a) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)NY * np + np) return;
  const long o = np + q;  // planes 1..NY+1
  a[o] = nut[o] * a[o];
  a[pfield + o] = nut[o] * a[pfield + o];
}

// G(TH) = i kx F(K_T dTH/dx) + i kz F(K_T dTH/dz) on JSTART_TH..JEND_TH
__global__ void k_les_th_force(int NY, long ss, int nkxp, int jlo, int jhi,
                               const double *__restrict__ kxv, const double *__restrict__ kzv,
                               const double2 *__restrict__ c, long nspec, double2 *__restrict__ g) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)(NY + 2) * ss) return;
  const int j = (int)(q / ss);
  const long m = q % ss;
  double2 r = make_double2(0.0, 0.0);
  if (j >= jlo && j <= jhi) {
    const double2 a = cmul_i(kxv[m % nkxp], c[q]), b = cmul_i(kzv[m / nkxp], c[nspec + q]);
    r = make_double2(a.x + b.x, a.y + b.y);
  }
  g[q] = r;
}

// CF += G, R += BETA_BAR H_BAR G for every field (G is zero outside its rows)
__global__ void k_les_add(int nf, long nspec, const double *__restrict__ dscal, int rk_step,
                          const double2 *__restrict__ g, FieldPtrs cf, FieldPtrs rhs) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (q >= nspec || f >= nf) return;
  const double h = dscal[1 + rk_step];
  const double bbar = (rk_step == 2) ? 25.0 / 8.0 : (rk_step == 3) ? 9.0 / 4.0 : 1.0;
  const double T5 = bbar * h;
  const double2 a = g[(long)f * nspec + q];
  double2 *c = cf(f) + q, *r = rhs(f) + q;
  const double2 cv = *c, rv = *r;
  *c = make_double2(cv.x + a.x, cv.y + a.y);
  *r = make_double2(rv.x + T5 * a.x, rv.y + T5 * a.y);
}

// ------------------------------------------------ physical-column CN solve
struct LesCn {
  int NY, nf, JS, JE, jst[DG_MAX_TH], jet[DG_MAX_TH];
  int bc_lo[3 + DG_MAX_TH], bc_hi[3 + DG_MAX_TH];
  double c1_lo[3 + DG_MAX_TH], c1_hi[3 + DG_MAX_TH];
  double nu, nuv, pr[DG_MAX_TH];
  double dy2, dyn, dyf1, dyfn;  // DY(2), DY(NY), DYF(1), DYF(NY) for the Neumann BC rows
};

// Row j of field f (0 U1, 1 U2, 2 U3, 3+n TH(n)) as the reference builds it:
// identity, then CN rows with the eddy-viscosity terms over the update range,
// then the lower and upper BC rows (APPLY_BC_*_MPI, for/mpi.f:1137-1291 with
// for/channel.f:1660-2241).  The right-hand side of a CN row is R plus the
// explicit eddy-viscosity half.  um, uj, up: the field on planes j-1, j, j+1;
// nm, nj, np1: NU_T on the same planes; r: R on plane j.  The grid factors
// come as reciprocals (T, [6][L] in shared memory): 1/(DY_j DYF_j),
// 1/(DY_j+1 DYF_j), 1/(DYF_j-1 DY_j), 1/(DYF_j DY_j), 1/DY_j, 1/DYF_j; the
// reference divides by the products, which differs in the last bit only.
__device__ __forceinline__ void les_row(const LesCn &P, int f, int j, double T1, double T2,
                                        const double *T, int L, double um, double uj, double up,
                                        double nm_, double nj, double np1, double r, double &l,
                                        double &d, double &u, double &v) {
  const int NY = P.NY;
  const double *g0 = T, *g1 = T + L, *h0 = T + 2 * L, *h1 = T + 3 * L, *idy = T + 4 * L,
               *idyf = T + 5 * L;
  l = 0.0, d = 1.0, u = 0.0, v = 0.0;
  if (f == 1) {
    if (j >= 2 && j <= NY) {
      const double a = T1 * P.nuv;
      const double nm = 0.5 * (nj + nm_), npl = 0.5 * (nj + np1);
      l = -a * h0[j] - T2 * nm * h0[j];
      d = 1. + a * h1[j] + a * h0[j] + T2 * npl * h1[j] + T2 * nm * h0[j];
      u = -a * h1[j] - T2 * npl * h1[j];
      v = r + T2 * ((npl * (up - uj) * idyf[j] - nm * (uj - um) * idyf[j - 1]) * idy[j]);
    }
    // APPLY_BC_2_LOWER / _UPPER
    const int lo = P.bc_lo[1], hi = P.bc_hi[1];
    if (j == 0) { l = 0.; d = 1.; u = 0.; v = 0.; }
    if (lo == 0 && (j == 1 || j == 2)) { l = 0.; d = 1.; u = 0.; v = P.c1_lo[1]; }
    if (lo == 1 && j == 1) { l = 0.; d = -1.; u = 1.; v = P.dyf1 * P.c1_lo[1]; }
    if (hi == 0 && (j == NY || j == NY + 1)) { l = 0.; d = 1.; u = 0.; v = P.c1_hi[1]; }
    if (hi == 1 && j == NY + 1) { l = -1.; d = 1.; u = 0.; v = P.dyfn * P.c1_hi[1]; }
    return;
  }
  const bool th = f >= 3;
  const int js = th ? P.jst[f - 3] : P.JS, je = th ? P.jet[f - 3] : P.JE;
  if (j >= js && j <= je) {
    const double a = th ? T1 / P.pr[f - 3] * P.nuv : T1 * P.nuv;
    l = -a * g0[j] - T2 * nj * g0[j];
    d = 1. + a * g1[j] + a * g0[j] + T2 * np1 * g1[j] + T2 * nj * g0[j];
    u = -a * g1[j] - T2 * np1 * g1[j];
    v = r + T2 * ((np1 * (up - uj) * idy[j + 1] - nj * (uj - um) * idy[j]) * idyf[j]);
  }
  // APPLY_BC_1/3/TH_LOWER / _UPPER
  const int lo = P.bc_lo[f], hi = P.bc_hi[f];
  if (j == 0) { l = 0.; d = 1.; u = 0.; v = 0.; }
  if (j == 1) {
    if (lo == 0) { l = 0.; d = 1.; u = 0.; v = P.c1_lo[f]; }
    else { l = 0.; d = -1.; u = 1.; v = P.dy2 * P.c1_lo[f]; }
  }
  if (j == NY + 1) { l = 0.; d = 1.; u = 0.; v = 0.; }
  if (j == NY) {
    if (hi == 0) { l = 0.; d = 1.; u = 0.; v = P.c1_hi[f]; }
    else { l = -1.; d = 1.; u = 0.; v = P.dyn * P.c1_hi[f]; }
  }
}

// One thread per physical column of one field: rows, THOMAS_FORWARD_REAL_MPI
// and THOMAS_BACKWARD_REAL_MPI for the only rank (for/mpi.f:630-703,767-809),
// the solution written back over the reference's ranges.  The forward sweep
// stores per row the two coefficients of the back substitution
// x(j) = e(j) + f(j) x(j+1), e = g / b and f = -c / b (R's slot takes e,
// the scratch slot B takes f; both 0 for a zero pivot, so the backward
// sweep writes 0 there, as the reference's guard does); the backward sweep
// then reads only those two.  Both sweeps load CB rows at a time before
// their recurrence so the loads overlap.
constexpr int CB = 12;

__global__ void __launch_bounds__(128) k_les_cn(LesCn P, long np, long pfield,
                                                const double *__restrict__ dscal, int rk_step,
                                                const double *__restrict__ rowtab,
                                                const double *__restrict__ nut,
                                                double *__restrict__ Rbase,
                                                double *__restrict__ Ubase,
                                                double *__restrict__ THbase,
                                                double *__restrict__ Bbase) {
  extern __shared__ double tab[];
  const int NY = P.NY, L = NY + 2;
  for (int i = threadIdx.x; i < 6 * L; i += blockDim.x) tab[i] = rowtab[i];
  __syncthreads();
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (q >= np || f >= P.nf) return;
  const double h = dscal[1 + rk_step];
  const double T1 = P.nu * h / 2.0, T2 = h / 2.0;
  double *R = Rbase + (long)f * pfield + q;
  double *U = (f < 3 ? Ubase + (long)f * pfield : THbase + (long)(f - 3) * pfield) + q;
  double *B = Bbase + (long)f * pfield + q;
  const double *nq = nut + q;
  double l, d, u, v;
  les_row(P, f, 0, T1, T2, tab, L, 0., 0., 0., 0., 0., 0., 0., l, d, u, v);
  double rbprev = (d != 0.0) ? 1.0 / d : 0.0, cprev = u, gprev = v;
  B[0] = -u * rbprev;
  R[0] = v * rbprev;
  for (int j0 = 1; j0 < L; j0 += CB) {
    double uu[CB + 2], nn[CB + 2], rr[CB];
#pragma unroll
    for (int k = 0; k < CB + 2; k++) {
      const int j = j0 - 1 + k;
      const bool ok = j < L;
      uu[k] = ok ? U[(long)j * np] : 0.0;
      nn[k] = ok ? nq[(long)j * np] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < CB; k++) {
      const int j = j0 + k;
      rr[k] = j < L ? R[(long)j * np] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < CB; k++) {
      const int j = j0 + k;
      if (j < L) {
        les_row(P, f, j, T1, T2, tab, L, uu[k], uu[k + 1], uu[k + 2], nn[k], nn[k + 1],
                nn[k + 2], rr[k], l, d, u, v);
        const double a = -l * rbprev;
        const double b = d + a * cprev;
        const double g = v + a * gprev;
        const double rb = (b != 0.0) ? 1.0 / b : 0.0;
        const long o = (long)j * np;
        B[o] = -u * rb;
        R[o] = g * rb;
        rbprev = rb;
        cprev = u;
        gprev = g;
      }
    }
  }
  // back substitution; rows written back: U1/U3 JSTART-1..JEND+1, U2
  // 1..NY+1, TH(n) JSTART_TH-1..JEND_TH+1
  int wlo, whi;
  if (f == 1) { wlo = 1; whi = NY + 1; }
  else if (f >= 3) { wlo = P.jst[f - 3] - 1; whi = P.jet[f - 3] + 1; }
  else { wlo = P.JS - 1; whi = P.JE + 1; }
  double x = 0.0;
  for (int j1 = NY + 1; j1 >= 0; j1 -= CB) {
    double ff[CB], ee[CB];
#pragma unroll
    for (int k = 0; k < CB; k++) {
      const int j = j1 - k;
      const long o = (long)(j >= 0 ? j : 0) * np;
      ff[k] = B[o];
      ee[k] = R[o];
    }
#pragma unroll
    for (int k = 0; k < CB; k++) {
      const int j = j1 - k;
      if (j >= 0) {
        x = ee[k] + ff[k] * x;
        if (j >= wlo && j <= whi) U[(long)j * np] = x;
      }
    }
  }
}

// n spectral fields (planes jmin..jmax) to physical slots at stride pfield,
// and back, LES_HF fields per launch through the LES staging buffer
int to_physical(dg_handle *h, const double2 *const *in, int n, int jmin, int jmax, double *out) {
  const long pplane = (long)h->NZ * h->NX, pf = pfield_of(h);
  for (int b = 0; b < n; b += LES_HF) {
    const int k = (n - b < LES_HF) ? n - b : LES_HF;
    const int r = dg_plane_c2r(h, in + b, k, jmin, jmax, out + (long)b * pf, pplane, h->NX, pf);
    if (r != 1) {
      DG_TRY(r);
      continue;
    }
    DG_TRY(dg_zinv(h, in + b, k, jmin, jmax, h->les_H, 0));
    DG_TRY(dg_xc2r_planes(h, h->les_H, k, jmin, jmax, out + (long)b * pf, pplane, h->NX, pf));
  }
  return DG_OK;
}

int to_fourier(dg_handle *h, const double *in, int n, int jmin, int jmax, double2 *const *out) {
  const long pplane = (long)h->NZ * h->NX, pf = pfield_of(h);
  for (int b = 0; b < n; b += LES_HF) {
    const int k = (n - b < LES_HF) ? n - b : LES_HF;
    const int r = dg_plane_r2c(h, in + (long)b * pf, k, jmin, jmax, pplane, h->NX, pf, out + b);
    if (r != 1) {
      DG_TRY(r);
      continue;
    }
    DG_TRY(dg_xr2c_planes(h, in + (long)b * pf, k, jmin, jmax, pplane, h->NX, pf, h->les_H));
    DG_TRY(dg_zfwd_planes(h, h->les_H, k, jmin, jmax, out + b, nullptr, 0));
  }
  return DG_OK;
}

}  // namespace

int dg_les_init(dg_handle *h) {
  const int NY = h->NY;
  const size_t pf = (size_t)pfield_of(h), ns = (size_t)h->nspec;
  DG_CUDA(dg_malloc(h, (void **)&h->les_phys, sizeof(double) * pf * phys_slots(h)));
  DG_CUDA(dg_malloc(h, (void **)&h->les_spec, sizeof(double2) * ns * spec_slots(h)));
  DG_CUDA(dg_malloc(h, (void **)&h->les_dfac, sizeof(double) * 2 * (NY + 2)));
  DG_CUDA(dg_malloc(h, (void **)&h->les_ubar, sizeof(double) * 2 * (NY + 2)));
  DG_CUDA(dg_malloc(h, (void **)&h->les_means, sizeof(double) * 2 * (NY + 2)));
  DG_CUDA(dg_malloc(h, (void **)&h->les_H,
                    sizeof(double2) * LES_HF * (size_t)h->nplanes * h->NZ * h->nkxp));
  DG_CUDA(cudaMemsetAsync(h->les_phys, 0, sizeof(double) * pf * phys_slots(h), h->st));
  DG_CUDA(cudaMemsetAsync(h->les_spec, 0, sizeof(double2) * ns * spec_slots(h), h->st));
  // -2 C_S^2 (DX BETA DY 2 DZ BETA)^(2/3), C_S = 0.13, BETA = 1 (for/les.f:194-217),
  // on GYF (DYF) and GY (DY) spacings, planes 1..NY+1
  double *t = (double *)calloc(2 * (NY + 2), sizeof(double));
  const double dx = h->p.lx / h->NX, dz = h->p.lz / h->NZ, cs = 0.13, beta_sgs = 1.0;
  for (int j = 1; j <= NY + 1; j++) {
    t[j] = -2.0 * cs * cs * pow(dx * beta_sgs * h->h_dyf[j] * 2.0 * dz * beta_sgs, 2.0 / 3.0);
    t[NY + 2 + j] = -2.0 * cs * cs * pow(dx * beta_sgs * h->h_dy[j] * 2.0 * dz * beta_sgs, 2.0 / 3.0);
  }
  // reciprocal grid factors of the CN rows, planes 0..NY+1 (zero where a
  // factor would reach outside the grid; those rows are BC or identity rows)
  const int L = NY + 2;
  double *rt = (double *)calloc(6 * L, sizeof(double));
  const double *DY = h->h_dy, *DYF = h->h_dyf;
  for (int j = 1; j <= NY; j++) {
    rt[j] = 1.0 / (DY[j] * DYF[j]);
    rt[L + j] = 1.0 / (DY[j + 1] * DYF[j]);
    if (j >= 2) rt[2 * L + j] = 1.0 / (DYF[j - 1] * DY[j]);
    rt[3 * L + j] = 1.0 / (DYF[j] * DY[j]);
  }
  for (int j = 1; j <= NY + 1; j++) {
    rt[4 * L + j] = 1.0 / DY[j];
    rt[5 * L + j] = 1.0 / DYF[j];
  }
  cudaError_t e0 = dg_malloc(h, (void **)&h->les_rowtab, sizeof(double) * 6 * L);
  if (e0 != cudaSuccess) {
    free(t);
    free(rt);
    DG_CUDA(e0);
  }
  cudaError_t e = cudaMemcpyAsync(h->les_dfac, t, sizeof(double) * 2 * (NY + 2),
                                  cudaMemcpyHostToDevice, h->st);
  cudaError_t e1 = cudaMemcpyAsync(h->les_rowtab, rt, sizeof(double) * 6 * L,
                                   cudaMemcpyHostToDevice, h->st);
  cudaError_t e2 = cudaStreamSynchronize(h->st);
  free(t);
  free(rt);
  DG_CUDA(e);
  DG_CUDA(e1);
  DG_CUDA(e2);
  h->les_nut = false;
  return DG_OK;
}

// The subgrid model runs from the first step, or after 100 steps of a new
// flow (for/channel.f:303).
bool dg_les_active(const dg_handle *h, int time_step) {
  return h->p.les && !h->periodic && (!h->p.create_new_flow || time_step > 100);
}

int dg_les_pre(dg_handle *h, int rk_step) {
  (void)rk_step;
  const int NY = h->NY;
  const long ss = h->ss, ns = h->nspec, np = (long)h->NZ * h->NX, pf = pfield_of(h);
  const LesBc B = make_bc(h->p);
  // APPLY_BC_VEL_MPI, APPLY_BC_LES
  DG_TRY(dg_apply_bc_vel_dev(h));
  dg_kt_begin(h, "k_les_bc_spec", h->st);
  k_les_bc_spec<<<dg_cdiv(ss, 256), 256, 0, h->st>>>(B, NY, ss, h->cu[0], h->cu[2]);
  DG_LAUNCHED();
  // strain rates and the plane means, then S_ij and U in physical space
  dg_kt_begin(h, "k_les_strain", h->st);
  k_les_strain<<<dg_cdiv((long)(NY + 2) * ss, 256), 256, 0, h->st>>>(
      NY, ss, h->nkxp, h->kx, h->kz, h->dy, h->dyf, h->cu[0], h->cu[1], h->cu[2], sslot(h, SS_S),
      ns, h->les_ubar);
  DG_LAUNCHED();
  const double2 *cs[6];
  for (int c = 0; c < 6; c++) cs[c] = sslot(h, SS_S + c);
  DG_TRY(to_physical(h, cs, 6, 0, NY + 1, pslot(h, PS_S)));
  const double2 *cu[3] = {h->cu[0], h->cu[1], h->cu[2]};
  DG_TRY(to_physical(h, cu, 3, 0, NY + 1, pslot(h, PS_U)));
  dg_kt_begin(h, "k_les_bc_phys", h->st);
  k_les_bc_phys<<<dg_cdiv(np, 256), 256, 0, h->st>>>(B, NY, np, pf, h->dy, h->dyf, pslot(h, PS_U));
  DG_LAUNCHED();
  double *prod = pslot(h, PS_P);
  dg_kt_begin(h, "k_les_model", h->st);
  k_les_model<<<dg_cdiv((long)(NY + 2) * np, 256), 256, 0, h->st>>>(
      NY, np, pf, h->jstart, h->jend, h->dy, h->dyf, h->les_dfac, h->les_ubar, pslot(h, PS_S),
      prod, pslot(h, PS_X), pslot(h, PS_U), pslot(h, PS_NUT));
  DG_LAUNCHED();
  h->les_nut = true;
  // |S| S_ij (S_22 excluded) and the cross terms to Fourier space
  // (the cross-term slots are zero outside planes 2..NY, which is all the
  // forcing reads of them)
  double2 *op[7] = {sslot(h, SS_S),     sslot(h, SS_S + 2), sslot(h, SS_S + 3), sslot(h, SS_S + 4),
                    sslot(h, SS_S + 5), sslot(h, SS_X),     sslot(h, SS_X + 1)};
  DG_TRY(to_fourier(h, prod, 7, 0, NY + 1, op));
  dg_kt_begin(h, "k_les_force", h->st);
  k_les_force<<<dg_cdiv((long)(NY + 2) * ss, 256), 256, 0, h->st>>>(
      NY, ss, h->nkxp, h->jstart, h->kx, h->kz, h->dyf, h->les_dfac, sslot(h, SS_S), ns,
      sslot(h, SS_G));
  DG_LAUNCHED();
  if (h->les_stats_req) {
    // the velocity here has APPLY_BC_VEL_PHYS applied; les_chan's own is the
    // one before it, which differs on planes 1 and NY only for non-zero BC
    // constants
    const double2 *g[3] = {sslot(h, SS_G), sslot(h, SS_G + 1), sslot(h, SS_G + 2)};
    DG_TRY(to_physical(h, g, 3, 0, NY + 1, pslot(h, PS_S)));
    dg_kt_begin(h, "k_les_means", h->st);
    k_les_means<<<NY + 2, 256, 0, h->st>>>(np, pf, pslot(h, PS_S), pslot(h, PS_U),
                                           pslot(h, PS_NUT), h->les_means, NY + 2);
    DG_LAUNCHED();
    h->les_stats_req = false;
    h->les_stats_valid = true;
  }
  // scalar eddy diffusion, KAPPA_T = NU_T
  for (int n = 0; n < h->NTH; n++) {
    dg_kt_begin(h, "k_les_th_grad", h->st);
    k_les_th_grad<<<dg_cdiv((long)(NY + 2) * ss, 256), 256, 0, h->st>>>(
        NY, ss, h->nkxp, h->kx, h->kz, h->cu[3 + n], sslot(h, SS_S), ns);
    DG_LAUNCHED();
    const double2 *tg[2] = {sslot(h, SS_S), sslot(h, SS_S + 1)};
    DG_TRY(to_physical(h, tg, 2, 0, NY + 1, pslot(h, PS_S)));
    dg_kt_begin(h, "k_les_th_scale", h->st);
    k_les_th_scale<<<dg_cdiv((long)(NY + 1) * np, 256), 256, 0, h->st>>>(NY, np, pf,
                                                                       pslot(h, PS_NUT),
                                                                       pslot(h, PS_S));
    DG_LAUNCHED();
    double2 *tf[2] = {sslot(h, SS_S), sslot(h, SS_S + 1)};
    DG_TRY(to_fourier(h, pslot(h, PS_S), 2, 0, NY + 1, tf));
    dg_kt_begin(h, "k_les_th_force", h->st);
    k_les_th_force<<<dg_cdiv((long)(NY + 2) * ss, 256), 256, 0, h->st>>>(
        NY, ss, h->nkxp, h->jstart_th[n], h->jend_th[n], h->kx, h->kz, sslot(h, SS_S), ns,
        sslot(h, SS_G + 3 + n));
    DG_LAUNCHED();
  }
  // the nonlinear stage reads the velocity from CU: give its boundary planes
  // the values APPLY_BC_VEL_PHYS left in the physical velocity
  dg_kt_begin(h, "k_les_bc_spec_phys", h->st);
  k_les_bc_spec_phys<<<dg_cdiv(ss, 256), 256, 0, h->st>>>(B, NY, ss, h->dy, h->dyf, h->cu[0],
                                                          h->cu[1], h->cu[2]);
  DG_LAUNCHED();
  return DG_OK;
}

int dg_les_post(dg_handle *h, int time_step, int rk_step, bool sgs) {
  const int NY = h->NY;
  const long ns = h->nspec, np = (long)h->NZ * h->NX, pf = pfield_of(h);
  FieldPtrs cf, rhs;
  for (int f = 0; f < h->nf; f++) {
    cf.p[f] = h->cf[f];
    rhs.p[f] = h->rhs[f];
  }
  if (sgs) {
    dg_kt_begin(h, "k_les_add", h->st);
    k_les_add<<<dim3(dg_cdiv(ns, 256), h->nf), 256, 0, h->st>>>(h->nf, ns, h->dscal, rk_step,
                                                                sslot(h, SS_G), cf, rhs);
    DG_LAUNCHED();
  } else {
    // the model is idle this substep but NU_T stays in the solves; the
    // velocity enters them as the plain transform of CU
    const double2 *cu[3] = {h->cu[0], h->cu[1], h->cu[2]};
    DG_TRY(to_physical(h, cu, 3, 0, NY + 1, pslot(h, PS_U)));
  }
  // right-hand sides and scalars to physical space
  const double2 *r[3 + DG_MAX_TH];
  for (int f = 0; f < h->nf; f++) r[f] = h->rhs[f];
  DG_TRY(to_physical(h, r, h->nf, 1, NY, pslot(h, PS_S)));
  if (h->NTH > 0) {
    const double2 *th[DG_MAX_TH];
    for (int n = 0; n < h->NTH; n++) th[n] = h->cu[3 + n];
    DG_TRY(to_physical(h, th, h->NTH, 0, NY + 1, pslot(h, PS_TH)));
  }
  LesCn P;
  memset(&P, 0, sizeof(P));
  const dg_params &p = h->p;
  P.NY = NY;
  P.nf = h->nf;
  P.JS = h->jstart;
  P.JE = h->jend;
  P.nu = p.nu;
  P.nuv = p.nu_v_scale;
  const int lo[3] = {p.u_bc_ymin, p.v_bc_ymin, p.w_bc_ymin}, hi[3] = {p.u_bc_ymax, p.v_bc_ymax, p.w_bc_ymax};
  const double clo[3] = {p.u_bc_ymin_c1, p.v_bc_ymin_c1, p.w_bc_ymin_c1};
  const double chi[3] = {p.u_bc_ymax_c1, p.v_bc_ymax_c1, p.w_bc_ymax_c1};
  for (int f = 0; f < 3; f++) {
    P.bc_lo[f] = lo[f];
    P.bc_hi[f] = hi[f];
    P.c1_lo[f] = clo[f];
    P.c1_hi[f] = chi[f];
  }
  for (int n = 0; n < h->NTH; n++) {
    P.jst[n] = h->jstart_th[n];
    P.jet[n] = h->jend_th[n];
    P.pr[n] = p.pr[n];
    P.bc_lo[3 + n] = p.th_bc_ymin[n];
    P.bc_hi[3 + n] = p.th_bc_ymax[n];
    P.c1_lo[3 + n] = p.th_bc_ymin_c1[n];
    P.c1_hi[3 + n] = p.th_bc_ymax_c1[n];
  }
  P.dy2 = h->h_dy[2];
  P.dyn = h->h_dy[NY];
  P.dyf1 = h->h_dyf[1];
  P.dyfn = h->h_dyf[NY];
  const size_t tsm = sizeof(double) * 6 * (NY + 2);
  if (tsm > 48 * 1024)
    DG_CUDA(cudaFuncSetAttribute(k_les_cn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm));
  dg_kt_begin(h, "k_les_cn", h->st);
  k_les_cn<<<dim3(dg_cdiv(np, 128), h->nf), 128, tsm, h->st>>>(
      P, np, pf, h->dscal, rk_step, h->les_rowtab, pslot(h, PS_NUT), pslot(h, PS_S),
      pslot(h, PS_U), pslot(h, PS_TH), pslot(h, PS_TH + h->NTH));
  DG_LAUNCHED();
  // COURANT on the solved velocity (for/channel.f:1037-1040)
  const bool cfl = p.variable_dt && rk_step == 3 && p.update_dt > 0 &&
                   (time_step % p.update_dt) == 0;
  if (cfl) DG_TRY(dg_courant_phys(h, pslot(h, PS_U) + np, pf));
  double2 *v[3 + DG_MAX_TH];
  for (int f = 0; f < h->nf; f++) v[f] = h->cu[f];
  DG_TRY(to_fourier(h, pslot(h, PS_U), h->nf, 0, NY + 1, v));
  DG_TRY(dg_rem_div_dev(h, 1, rk_step, false));
  if (cfl) DG_TRY(dg_dt_commit(h));
  return DG_OK;
}

// NU_T (COMMON /LES_VARS/, for/header:166) of the last LES substep, physical
// layout [NY+2][NZ][NX].
extern "C" int diablo_les_nu_t(dg_handle *h, double *dst, int where) {
  if (!h || h->periodic || !dst) return DG_ERR_ARG;
  if (!h->p.les || !h->les_phys) {
    dg_set_error("the handle was created without LES");
    return DG_ERR_ARG;
  }
  const size_t bytes = sizeof(double) * (size_t)pfield_of(h);
  DG_CUDA(cudaMemcpyAsync(dst, pslot(h, PS_NUT), bytes,
                          where == DG_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                          h->st));
  DG_CUDA(cudaStreamSynchronize(h->st));
  return DG_OK;
}

// les_chan's plane means at the SAVE_STATS cadence (MOD(TIME_STEP,
// SAVE_STATS_INT) = 0 and RK_STEP = 1, for/les.f:336): the request makes the
// next LES substep record NU_T_MEAN and EPS_SGS1_MEAN (rows 0..NY+1), which
// diablo_les_stats returns.
extern "C" int diablo_les_stats_request(dg_handle *h) {
  if (!h || h->periodic || !h->p.les) return DG_ERR_ARG;
  h->les_stats_req = true;
  return DG_OK;
}

extern "C" int diablo_les_stats(dg_handle *h, double *nu_t_mean, double *eps_sgs1_mean) {
  if (!h || h->periodic || !h->p.les || !nu_t_mean || !eps_sgs1_mean) return DG_ERR_ARG;
  if (!h->les_stats_valid) {
    dg_set_error("no LES substep has recorded statistics since the request");
    return DG_ERR_ARG;
  }
  const size_t n = sizeof(double) * (h->NY + 2);
  DG_CUDA(cudaMemcpyAsync(nu_t_mean, h->les_means, n, cudaMemcpyDeviceToHost, h->st));
  DG_CUDA(cudaMemcpyAsync(eps_sgs1_mean, h->les_means + h->NY + 2, n, cudaMemcpyDeviceToHost,
                          h->st));
  DG_CUDA(cudaStreamSynchronize(h->st));
  return DG_OK;
}

// tkebudget_chan_les as SAVE_STATS_CHAN runs it when LES is on
// (for/save_stats.f:30-36,164-170): APPLY_BC_VEL on the state, the velocity to
// physical space, epsilon_sgs (rows 1..NY of NY+2) with the NU_T of the last
// LES substep.
extern "C" int diablo_les_tke(dg_handle *h, double *epsilon_sgs) {
  if (!h || h->periodic || !h->p.les || !epsilon_sgs) return DG_ERR_ARG;
  const int NY = h->NY;
  const long np = (long)h->NZ * h->NX, pf = pfield_of(h);
  DG_TRY(dg_apply_bc_vel_dev(h));
  const double2 *cu[3] = {h->cu[0], h->cu[1], h->cu[2]};
  DG_TRY(to_physical(h, cu, 3, 0, NY + 1, pslot(h, PS_U)));
  DG_CUDA(cudaMemsetAsync(h->les_means, 0, sizeof(double) * (NY + 2), h->st));
  dg_kt_begin(h, "k_les_tke", h->st);
  k_les_tke<<<NY, 256, 0, h->st>>>(NY, np, pf, h->dy, h->dyf, pslot(h, PS_U), pslot(h, PS_NUT),
                                   h->les_means);
  DG_LAUNCHED();
  DG_CUDA(cudaMemcpyAsync(epsilon_sgs, h->les_means, sizeof(double) * (NY + 2),
                          cudaMemcpyDeviceToHost, h->st));
  DG_CUDA(cudaStreamSynchronize(h->st));
  h->les_stats_valid = false;  // the means buffer now holds epsilon_sgs
  return DG_OK;
}
