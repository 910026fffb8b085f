// Shared-memory mixed-radix Stockham FFT used by all transform kernels.
//
// A batch of `nsig` complex signals of length N lives in shared memory, one
// signal per `sig_stride` double2.  Every thread of the CTA takes butterflies
// of every signal in turn; one __syncthreads() separates passes.  The
// autosorting (Stockham) form needs a second buffer of the same size and
// gives naturally ordered output.  Pass with radix R and running span Ns:
//   butterfly b in [0, N/R): k = b mod Ns,
//   v[r] = src[b + r N/R] * W_N^(r k N/(Ns R)),  v = DFT_R(v),
//   dst[(b/Ns) Ns R + k + r Ns] = v[r];   Ns <- Ns R.
// W_N = exp(sign 2 pi i / N); the table holds exp(-2 pi i m / N) and the
// inverse direction conjugates it.  Unnormalised in both directions, which
// is FFTW's convention (forward sign -1).
#pragma once

#include <cuda_runtime.h>
#include "dg_internal.cuh"

namespace dgfft {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 conjg(double2 a) { return make_double2(a.x, -a.y); }
// multiply by sign*i
__device__ __forceinline__ double2 mul_si(double2 a, int sign) {
  return sign < 0 ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
}

template <int R>
__device__ __forceinline__ void dft(double2 *v, int sign);

template <>
__device__ __forceinline__ void dft<2>(double2 *v, int) {
  double2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <>
__device__ __forceinline__ void dft<3>(double2 *v, int sign) {
  const double s3 = 0.86602540378443864676;  // sqrt(3)/2
  double2 t1 = cadd(v[1], v[2]);
  double2 t2 = make_double2(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
  double2 d = csub(v[1], v[2]);
  double2 t3 = mul_si(cscale(d, s3), sign);
  v[0] = cadd(v[0], t1);
  v[1] = cadd(t2, t3);
  v[2] = csub(t2, t3);
}

template <>
__device__ __forceinline__ void dft<4>(double2 *v, int sign) {
  double2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
  double2 s13 = cadd(v[1], v[3]), d13 = mul_si(csub(v[1], v[3]), sign);
  v[0] = cadd(s02, s13);
  v[1] = cadd(d02, d13);
  v[2] = csub(s02, s13);
  v[3] = csub(d02, d13);
}

template <>
__device__ __forceinline__ void dft<8>(double2 *v, int sign) {
  const double h = 0.70710678118654752440;  // 1/sqrt(2)
  double2 e[4] = {v[0], v[2], v[4], v[6]};
  double2 o[4] = {v[1], v[3], v[5], v[7]};
  dft<4>(e, sign);
  dft<4>(o, sign);
  // twiddles w8^t, w8 = exp(sign 2 pi i / 8) = (1 + sign i)/sqrt(2)
  double2 o1 = o[1], o2 = o[2], o3 = o[3];
  double2 t1 = make_double2(h * (o1.x - sign * o1.y), h * (o1.y + sign * o1.x));
  double2 t2 = mul_si(o2, sign);
  double2 t3 = make_double2(h * (-o3.x - sign * o3.y), h * (-o3.y + sign * o3.x));
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], t1);
  v[5] = csub(e[1], t1);
  v[2] = cadd(e[2], t2);
  v[6] = csub(e[2], t2);
  v[3] = cadd(e[3], t3);
  v[7] = csub(e[3], t3);
}

template <int R>
__device__ __forceinline__ void pass(const double2 *__restrict__ src, double2 *__restrict__ dst,
                                     int N, int Ns, int nsig, int sig_stride,
                                     const double2 *__restrict__ tw, int sign, int tid, int nthr) {
  const int nb = N / R;
  const int tmul = N / (Ns * R);
  const int total = nsig * nb;
  for (int w = tid; w < total; w += nthr) {
    const int s = w / nb;
    const int b = w - s * nb;
    const double2 *in = src + (long)s * sig_stride;
    double2 *out = dst + (long)s * sig_stride;
    const int k = b % Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      double2 x = in[b + r * nb];
      if (r > 0 && k > 0) {
        double2 t = tw[r * k * tmul];
        if (sign > 0) t.y = -t.y;
        x = cmul(x, t);
      }
      v[r] = x;
    }
    dft<R>(v, sign);
    const int idx = (b / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) out[idx + r * Ns] = v[r];
  }
}

// Runs the whole plan; returns the buffer holding the result (buf0 or buf1).
// Must be called by every thread of the CTA.
__device__ inline double2 *run(double2 *buf0, double2 *buf1, const FftPlan &pl, int nsig,
                               int sig_stride, const double2 *tw, int sign) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  double2 *src = buf0, *dst = buf1;
  int Ns = 1;
  for (int p = 0; p < pl.np; p++) {
    const int R = pl.r[p];
    switch (R) {
      case 8: pass<8>(src, dst, pl.n, Ns, nsig, sig_stride, tw, sign, tid, nthr); break;
      case 4: pass<4>(src, dst, pl.n, Ns, nsig, sig_stride, tw, sign, tid, nthr); break;
      case 3: pass<3>(src, dst, pl.n, Ns, nsig, sig_stride, tw, sign, tid, nthr); break;
      default: pass<2>(src, dst, pl.n, Ns, nsig, sig_stride, tw, sign, tid, nthr); break;
    }
    __syncthreads();
    double2 *t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  return src;
}

}  // namespace dgfft
