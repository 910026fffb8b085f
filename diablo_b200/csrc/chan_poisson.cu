// POISSON_P_CHAN (for/channel.f:1217-1453): the pressure of the current
// velocity (and buoyancy) field, solved mode by mode in y.
//
// Source term, rows J = 2..NY (the reference's order of operations):
//   S = F(u_x^2) + F(v_y^2) + F(w_z^2)
//     + F(2 u_y v_x) + F(2 w_y v_z) + F(2 u_z w_x)   (all in physical space)
//     + sum_n RI_n d(TH_n)/dy                          (modes other than (0,0))
// with u_x = IFFT(i kx CU1), v_y = IFFT((CU2(J+1) - CU2(J)) / DYF(J)), ...
// Here the four groups of physical products are accumulated into one
// physical plane stack and transformed forward once (the transform is
// linear; the reference transforms each group and adds in Fourier space).
// The tridiagonal operator is REM_DIV_CHAN's (same rows, same boundary rows),
// so its elimination factors, computed once at set-up, are reused; the
// right-hand side is -S on rows 2..NY-1 and zero on the boundary rows.
//
// The reference uses CF1..CF3 as scratch here and leaves products in them;
// this implementation uses its own scratch and leaves CF1..CF3 unchanged.
// Nothing reads CF before RK substep 1 overwrites it.
#include "dg_internal.cuh"

namespace {

// spectral inputs of one product group, rows 2..NY, into s0, s1, s2
__global__ void k_ppc_prep(int stage, int NY, long ss, int nkxp, const double *__restrict__ kxv,
                           const double *__restrict__ kzv, const double *__restrict__ dyf,
                           const double2 *__restrict__ u1, const double2 *__restrict__ u2,
                           const double2 *__restrict__ u3, double2 *__restrict__ s0,
                           double2 *__restrict__ s1, double2 *__restrict__ s2) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x + 2 * ss;
  if (q >= (long)(NY + 1) * ss) return;
  const int j = (int)(q / ss);
  const long m = q % ss;
  const double KX = kxv[m % nkxp], KZ = kzv[m / nkxp];
  auto ik = [](double k, double2 v) { return make_double2(-k * v.y, k * v.x); };
  auto sc = [](double a, double2 v) { return make_double2(a * v.x, a * v.y); };
  auto sub = [](double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); };
  auto add = [](double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); };
  if (stage == 0) {
    s0[q] = ik(KX, u1[q]);
    const double2 d = sub(u2[q + ss], u2[q]);
    s1[q] = make_double2(d.x / dyf[j], d.y / dyf[j]);
    s2[q] = ik(KZ, u3[q]);
  } else if (stage == 1) {
    const double2 d = sub(u1[q + ss], u1[q - ss]);
    s0[q] = make_double2(d.x / (2. * dyf[j]), d.y / (2. * dyf[j]));
    s1[q] = ik(KX, sc(0.5, add(u2[q], u2[q + ss])));
  } else if (stage == 2) {
    const double2 d = sub(u3[q + ss], u3[q - ss]);
    s0[q] = make_double2(d.x / (2. * dyf[j]), d.y / (2. * dyf[j]));
    s1[q] = ik(KZ, sc(0.5, add(u2[q], u2[q + ss])));
  } else {
    s0[q] = ik(KZ, u1[q]);
    s1[q] = ik(KX, u3[q]);
  }
}

// physical accumulation over planes 2..NY: stage 0 W0 = W0^2 + W1^2 + W2^2,
// later stages W0 += 2 W1 W2
__global__ void k_ppc_accum(int stage, long n, double *__restrict__ w0,
                            const double *__restrict__ w1, const double *__restrict__ w2) {
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
       q += (long)gridDim.x * blockDim.x) {
    if (stage == 0)
      w0[q] = w0[q] * w0[q] + w1[q] * w1[q] + w2[q] * w2[q];
    else
      w0[q] = w0[q] + 2. * w1[q] * w2[q];
  }
}

// Per mode: buoyancy term, then the y solve with REM_DIV_CHAN's factors
// (MPI Thomas, rows 1..NY); CP rows 1..NY.
struct RiVals {
  double v[DG_MAX_TH];
};

__global__ void k_ppc_col(int NY, long ss, int nth, RiVals ri,
                          const double *__restrict__ gyf, const double *__restrict__ dy,
                          const double *__restrict__ dyf, const double *__restrict__ ra,
                          const double *__restrict__ rrb, const double2 *__restrict__ S,
                          CFieldPtrs th, double2 *__restrict__ cp) {
  const long m = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= ss) return;
  const bool mean = (m == 0);
  // forward sweep: G(1) = 0; G(j) = V(j) + a(j) G(j-1)
  double2 g = make_double2(0.0, 0.0);
  cp[ss + m] = g;
  for (int j = 2; j <= NY; j++) {
    const long q = (long)j * ss + m;
    double2 v = make_double2(0.0, 0.0);
    if (j < NY) {
      double2 s = S[q];
      if (!mean)
        for (int n = 0; n < nth; n++) {
          const double r = ri.v[n] / (gyf[j + 1] - gyf[j - 1]);
          const double2 a = th(n)[q + ss], b = th(n)[q - ss];
          s.x += r * (a.x - b.x);
          s.y += r * (a.y - b.y);
        }
      v = make_double2(-s.x, -s.y);
    }
    const double a = ra[q];
    g = make_double2(v.x + a * g.x, v.y + a * g.y);
    cp[q] = g;
  }
  // backward sweep: G(NY) /= B(NY); G(j) = (G(j) - C(j) G(j+1)) / B(j)
  double2 up = make_double2(g.x * rrb[(long)NY * ss + m], g.y * rrb[(long)NY * ss + m]);
  cp[(long)NY * ss + m] = up;
  for (int j = NY - 1; j >= 1; j--) {
    const long q = (long)j * ss + m;
    const double c = (j == 1) ? (mean ? 0.0 : -1.0) : 1. / (dy[j + 1] * dyf[j]);
    const double2 gj = cp[q];
    const double rb = rrb[q];
    up = make_double2((gj.x - c * up.x) * rb, (gj.y - c * up.y) * rb);
    cp[q] = up;
  }
}

}  // namespace

extern "C" int diablo_poisson_p_chan(dg_handle *h) {
  if (!h || h->periodic) return DG_ERR_ARG;
  const int NY = h->NY;
  const long ss = h->ss;
  const long pplane = (long)h->NZ * h->NX;
  const long pfield = (long)(NY + 2) * pplane;
  double *W = (double *)h->work;  // three physical plane stacks
  double2 *s[3] = {h->rhs[0], h->rhs[1], h->rhs[2]};
  const long nint = (long)(NY - 1) * ss;  // rows 2..NY
  const long nphys = (long)(NY - 1) * pplane;
  for (int stage = 0; stage < 4; stage++) {
    dg_kt_begin(h, "k_ppc_prep", h->st);
    k_ppc_prep<<<dg_cdiv(nint, 256), 256, 0, h->st>>>(stage, NY, ss, h->nkxp, h->kx, h->kz,
                                                      h->dyf, h->cu[0], h->cu[1], h->cu[2], s[0],
                                                      s[1], s[2]);
    DG_LAUNCHED();
    const int nf = (stage == 0) ? 3 : 2;
    const double2 *in[3] = {s[0], s[1], s[2]};
    DG_TRY(dg_zinv(h, in, nf, 2, NY, h->H, 0));
    // stage 0 fills W0..W2, later stages W1..W2
    double *dst = (stage == 0) ? W : W + pfield;
    DG_TRY(dg_xc2r_planes(h, h->H, nf, 2, NY, dst, pplane, h->NX, pfield));
    dg_kt_begin(h, "k_ppc_accum", h->st);
    k_ppc_accum<<<4 * 148, 256, 0, h->st>>>(stage, nphys, W + 2 * pplane,
                                            W + pfield + 2 * pplane, W + 2 * pfield + 2 * pplane);
    DG_LAUNCHED();
  }
  DG_TRY(dg_xr2c_planes(h, W, 1, 2, NY, pplane, h->NX, 0, h->H));
  double2 *out[1] = {s[0]};
  DG_TRY(dg_zfwd_planes(h, h->H, 1, 2, NY, out, nullptr, 0));
  CFieldPtrs th;
  for (int n = 0; n < h->NTH; n++) th.p[n] = h->cu[3 + n];
  RiVals ri;
  for (int n = 0; n < DG_MAX_TH; n++) ri.v[n] = (n < h->NTH) ? h->p.ri[n] : 0.0;
  dg_kt_begin(h, "k_ppc_col", h->st);
  k_ppc_col<<<dg_cdiv(ss, 128), 128, 0, h->st>>>(NY, ss, h->NTH, ri, h->gyf, h->dy, h->dyf,
                                                 h->rem_a, h->rem_rb, s[0], th, h->cp);
  DG_LAUNCHED();
  return DG_OK;
}
