// Shared-memory mixed-radix Stockham FFT used by all transform kernels.
//
// A batch of `nsig` complex signals of length N lives in shared memory, one
// signal per `sig_stride` double2, element i of a signal stored at pad(i) =
// i + i/16 (one spare slot per 16 keeps the strided stores of the early
// passes off a single bank).  Every thread of the CTA takes butterflies of
// every signal in turn; one __syncthreads() separates passes.  The
// autosorting (Stockham) form needs a second buffer of the same size and
// gives naturally ordered output.  Pass with radix R and running span Ns:
//   butterfly b in [0, N/R): k = b mod Ns,
//   v[r] = src[b + r N/R] * W_N^(r k N/(Ns R)),  v = DFT_R(v),
//   dst[(b/Ns) Ns R + k + r Ns] = v[r];   Ns <- Ns R.
// W_N = exp(sign 2 pi i / N); the table holds exp(-2 pi i m / N) and the
// inverse direction conjugates it.  Unnormalised in both directions, which
// is FFTW's convention (forward sign -1).
//
// Two front ends: run<N>() with the transform length and radix plan fixed at
// compile time (all index arithmetic folds), and run() with a runtime plan
// for lengths without a specialisation.
#pragma once

#include <cuda_runtime.h>
#include "dg_internal.cuh"

namespace dgfft {

// Complex helpers for double2 (FP64 path) and float2 (mixed path); CT<C>
// gives the real type and a constructor.
template <typename C> struct CT;
template <> struct CT<double2> {
  using T = double;
  static __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
};
template <> struct CT<float2> {
  using T = float;
  static __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
};

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return CT<C>::mk(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return CT<C>::mk(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return CT<C>::mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cscale(C a, typename CT<C>::T s) {
  return CT<C>::mk(a.x * s, a.y * s);
}
template <typename C> __device__ __forceinline__ C conjg(C a) { return CT<C>::mk(a.x, -a.y); }
// multiply by sign*i
template <typename C> __device__ __forceinline__ C mul_si(C a, int sign) {
  return sign < 0 ? CT<C>::mk(a.y, -a.x) : CT<C>::mk(-a.y, a.x);
}

__host__ __device__ constexpr int pad(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded_len(int n) { return n + (n >> 4) + 1; }

template <int R> struct DFT;

template <> struct DFT<2> {
  template <typename C> static __device__ __forceinline__ void run(C *v, int) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <> struct DFT<3> {
  template <typename C> static __device__ __forceinline__ void run(C *v, int sign) {
    using T = typename CT<C>::T;
    const T s3 = (T)0.86602540378443864676;  // sqrt(3)/2
    C t1 = cadd(v[1], v[2]);
    C t2 = CT<C>::mk(v[0].x - (T)0.5 * t1.x, v[0].y - (T)0.5 * t1.y);
    C d = csub(v[1], v[2]);
    C t3 = mul_si(cscale(d, s3), sign);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
  }
};

// 5-point DFT: with W = exp(sign 2 pi i / 5), c_m = cos(2 pi m / 5) and
// s_m = sin(2 pi m / 5), X_1,4 = x0 + c1 (x1 + x4) + c2 (x2 + x3)
// +- sign i (s1 (x1 - x4) + s2 (x2 - x3)) and X_2,3 = x0 + c2 (x1 + x4)
// + c1 (x2 + x3) +- sign i (s2 (x1 - x4) - s1 (x2 - x3)).
template <> struct DFT<5> {
  template <typename C> static __device__ __forceinline__ void run(C *v, int sign) {
    using T = typename CT<C>::T;
    const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
    const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;
    const C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    const C t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    const C a1 = CT<C>::mk(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    const C a2 = CT<C>::mk(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    // b = s-weighted differences, then times sign * i
    const C b1 = mul_si(CT<C>::mk(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y), sign);
    const C b2 = mul_si(CT<C>::mk(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y), sign);
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, b1);
    v[4] = csub(a1, b1);
    v[2] = cadd(a2, b2);
    v[3] = csub(a2, b2);
  }
};

template <> struct DFT<4> {
  template <typename C> static __device__ __forceinline__ void run(C *v, int sign) {
    C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    C s13 = cadd(v[1], v[3]), d13 = mul_si(csub(v[1], v[3]), sign);
    v[0] = cadd(s02, s13);
    v[1] = cadd(d02, d13);
    v[2] = csub(s02, s13);
    v[3] = csub(d02, d13);
  }
};

template <> struct DFT<8> {
  template <typename C> static __device__ __forceinline__ void run(C *v, int sign) {
    using T = typename CT<C>::T;
    const T h = (T)0.70710678118654752440;  // 1/sqrt(2)
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    DFT<4>::run(e, sign);
    DFT<4>::run(o, sign);
    // twiddles w8^t, w8 = exp(sign 2 pi i / 8) = (1 + sign i)/sqrt(2)
    C o1 = o[1], o2 = o[2], o3 = o[3];
    C t1 = CT<C>::mk(h * (o1.x - sign * o1.y), h * (o1.y + sign * o1.x));
    C t2 = mul_si(o2, sign);
    C t3 = CT<C>::mk(h * (-o3.x - sign * o3.y), h * (-o3.y + sign * o3.x));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], t1);
    v[5] = csub(e[1], t1);
    v[2] = cadd(e[2], t2);
    v[6] = csub(e[2], t2);
    v[3] = cadd(e[3], t3);
    v[7] = csub(e[3], t3);
  }
};

// 16-point DFT as 4 x 4: n = 4 n1 + n2, k = k1 + 4 k2
template <> struct DFT<16> {
  template <typename C> static __device__ __forceinline__ void run(C *v, int sign) {
    using T = typename CT<C>::T;
    // cos and sin of 2 pi m / 16, m = 0..9
    const T Cs[10] = {(T)1.0, (T)0.92387953251128675613, (T)0.70710678118654752440,
                      (T)0.38268343236508977173, (T)0.0, (T)-0.38268343236508977173,
                      (T)-0.70710678118654752440, (T)-0.92387953251128675613, (T)-1.0,
                      (T)-0.92387953251128675613};
    const T Sn[10] = {(T)0.0, (T)0.38268343236508977173, (T)0.70710678118654752440,
                      (T)0.92387953251128675613, (T)1.0, (T)0.92387953251128675613,
                      (T)0.70710678118654752440, (T)0.38268343236508977173, (T)0.0,
                      (T)-0.38268343236508977173};
    C a[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
      C t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
      DFT<4>::run(t, sign);
#pragma unroll
      for (int k1 = 0; k1 < 4; k1++) {
        const int m = n2 * k1;
        C x = t[k1];
        if (m != 0) {
          const C w = CT<C>::mk(Cs[m], sign * Sn[m]);
          x = cmul(x, w);
        }
        a[n2][k1] = x;
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
      C t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
      DFT<4>::run(t, sign);
#pragma unroll
      for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = t[k2];
    }
  }
};

template <int R, typename C>
__device__ __forceinline__ void dft(C *v, int sign) {
  DFT<R>::run(v, sign);
}

// -------------------------------------------------------- runtime-plan pass
template <int R, typename C>
__device__ __forceinline__ void pass(const C *__restrict__ src, C *__restrict__ dst,
                                     int N, int Ns, int nsig, int sig_stride,
                                     const C *__restrict__ tw, int sign, int tid, int nthr) {
  const int nb = N / R;
  const int tmul = N / (Ns * R);
  const int total = nsig * nb;
  for (int w = tid; w < total; w += nthr) {
    const int s = w / nb;
    const int b = w - s * nb;
    const C *in = src + (long)s * sig_stride;
    C *out = dst + (long)s * sig_stride;
    const int k = b % Ns;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      C x = in[pad(b + r * nb)];
      if (r > 0 && k > 0) {
        C t = tw[r * k * tmul];
        if (sign > 0) t.y = -t.y;
        x = cmul(x, t);
      }
      v[r] = x;
    }
    dft<R>(v, sign);
    const int idx = (b / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) out[pad(idx + r * Ns)] = v[r];
  }
}

// Runs a runtime plan; returns the buffer holding the result (buf0 or buf1).
// Must be called by every thread of the CTA.
template <typename C>
__device__ inline C *run(C *buf0, C *buf1, const FftPlan &pl, int nsig,
                               int sig_stride, const C *tw, int sign) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  C *src = buf0, *dst = buf1;
  int Ns = 1;
  for (int p = 0; p < pl.np; p++) {
    const int R = pl.r[p];
    switch (R) {
      case 16: pass<16>(src, dst, pl.n, Ns, nsig, sig_stride, tw, sign, tid, nthr); break;
      case 8: pass<8>(src, dst, pl.n, Ns, nsig, sig_stride, tw, sign, tid, nthr); break;
      case 4: pass<4>(src, dst, pl.n, Ns, nsig, sig_stride, tw, sign, tid, nthr); break;
      case 3: pass<3>(src, dst, pl.n, Ns, nsig, sig_stride, tw, sign, tid, nthr); break;
      case 5: pass<5>(src, dst, pl.n, Ns, nsig, sig_stride, tw, sign, tid, nthr); break;
      default: pass<2>(src, dst, pl.n, Ns, nsig, sig_stride, tw, sign, tid, nthr); break;
    }
    __syncthreads();
    C *t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  return src;
}

// ----------------------------------------------------- compile-time plans
// radix of pass p for length N (0 = no pass).  Lengths 2^a 3^b; every pass
// keeps N/R <= 128 so a 128-thread CTA holds whole signals per round.
__host__ __device__ constexpr int plan_radix0(int N, int p) {
  int m = N, r = 0;
  for (int q = 0; q <= p; q++) {
    if (m == 1) return 0;
    if (m == 512 || m == 64 || m == 8 * 3 || m == 96) r = 8;
    else if (m % 16 == 0) r = 16;
    else if (m % 8 == 0) r = 8;
    else if (m % 4 == 0) r = 4;
    else if (m % 2 == 0) r = 2;
    else if (m % 3 == 0) r = 3;
    else return 0;
    m /= r;
  }
  return r;
}

__host__ __device__ constexpr int plan_passes(int N) {
  int p = 0;
  while (p < DG_MAX_PASSES && plan_radix0(N, p) != 0) p++;
  return p;
}

// Plan variant V: 0 as above (largest radix first), 1 the same radices in
// reverse order.  Both are the same transform (a Stockham pass sequence is
// valid for any order of the factors); they differ in shared-memory strides,
// twiddle reuse and register use, so the autotuner picks per grid shape.
__host__ __device__ constexpr int plan_radix(int N, int p, int V = 0) {
  return V == 0 ? plan_radix0(N, p)
                : (p < plan_passes(N) ? plan_radix0(N, plan_passes(N) - 1 - p) : 0);
}

// lengths whose two plan variants differ
__host__ __device__ constexpr bool plan_has_variant(int N) {
  bool differ = false;
  for (int p = 0; p < plan_passes(N); p++)
    if (plan_radix(N, p, 0) != plan_radix(N, p, 1)) differ = true;
  return differ;
}

__host__ __device__ constexpr int plan_ns(int N, int p, int V = 0) {
  int ns = 1;
  for (int q = 0; q < p; q++) ns *= plan_radix(N, q, V);
  return ns;
}

template <int N, int R, int NS, int SIGN, typename C>
__device__ __forceinline__ void cpass(const C *__restrict__ src, C *__restrict__ dst,
                                      int nsig, int sig_stride, const C *__restrict__ tw,
                                      int tid, int nthr) {
  constexpr int NB = N / R;
  constexpr int TMUL = N / (NS * R);
  const int total = nsig * NB;
  for (int w = tid; w < total; w += nthr) {
    const int s = w / NB;
    const int b = w - s * NB;
    const C *in = src + (long)s * sig_stride;
    C *out = dst + (long)s * sig_stride;
    const int k = b % NS;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      C x = in[pad(b + r * NB)];
      if (NS > 1 && r > 0) {
        C t = tw[r * k * TMUL];
        if (SIGN > 0) t.y = -t.y;
        x = cmul(x, t);
      }
      v[r] = x;
    }
    dft<R>(v, SIGN);
    const int idx = (b / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) out[pad(idx + r * NS)] = v[r];
  }
}

template <int N, int SIGN, int P, int V = 0, typename C>
__device__ __forceinline__ void cpasses(C *&src, C *&dst, int nsig, int sig_stride,
                                        const C *tw, int tid, int nthr) {
  constexpr int R = plan_radix(N, P, V);
  if constexpr (R != 0) {
    constexpr int NS = plan_ns(N, P, V);
    cpass<N, R, NS, SIGN>(src, dst, nsig, sig_stride, tw, tid, nthr);
    __syncthreads();
    C *t = src;
    src = dst;
    dst = t;
    cpasses<N, SIGN, P + 1, V>(src, dst, nsig, sig_stride, tw, tid, nthr);
  }
}

// In-place variant: each round covers whole signals (nthr / (N/R) of them);
// every thread of the round loads its butterfly, the CTA syncs, then stores.
template <int N, int R, int NS, int SIGN, typename C>
__device__ __forceinline__ void ippass(C *__restrict__ buf, int nsig, int sig_stride,
                                       const C *__restrict__ tw, int tid, int nthr) {
  constexpr int NB = N / R;
  constexpr int TMUL = N / (NS * R);
  const int spr = nthr / NB;
  const int nrounds = (nsig + spr - 1) / spr;
  const int sl = tid / NB, b = tid % NB, k = b % NS;
  const int idx = (b / NS) * NS * R + k;
  for (int rd = 0; rd < nrounds; rd++) {
    const int s = rd * spr + sl;
    const bool act = (sl < spr) && (s < nsig);
    C v[R];
    if (act) {
      const C *in = buf + (long)s * sig_stride;
#pragma unroll
      for (int r = 0; r < R; r++) {
        C x = in[pad(b + r * NB)];
        if (NS > 1 && r > 0) {
          C t = tw[r * k * TMUL];
          if (SIGN > 0) t.y = -t.y;
          x = cmul(x, t);
        }
        v[r] = x;
      }
      dft<R>(v, SIGN);
    }
    __syncthreads();
    if (act) {
      C *out = buf + (long)s * sig_stride;
#pragma unroll
      for (int r = 0; r < R; r++) out[pad(idx + r * NS)] = v[r];
    }
    __syncthreads();
  }
}

template <int N, int SIGN, int P, int V = 0, typename C>
__device__ __forceinline__ void ippasses(C *buf, int nsig, int sig_stride, const C *tw,
                                         int tid, int nthr) {
  constexpr int R = plan_radix(N, P, V);
  if constexpr (R != 0) {
    constexpr int NS = plan_ns(N, P, V);
    ippass<N, R, NS, SIGN>(buf, nsig, sig_stride, tw, tid, nthr);
    ippasses<N, SIGN, P + 1, V>(buf, nsig, sig_stride, tw, tid, nthr);
  }
}

template <int N, int SIGN, typename C>
__device__ __forceinline__ C *run_ct(C *buf0, C *buf1, int nsig, int sig_stride,
                                           const C *tw) {
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  C *src = buf0, *dst = buf1;
  cpasses<N, SIGN, 0>(src, dst, nsig, sig_stride, tw, tid, nthr);
  return src;
}

// Dispatch helper: N == 0 selects the runtime plan.
// ---------------------------------------------------------- warp-level passes
// One warp transforms `nsig` signals in place with __syncwarp between the
// load and store halves of every pass (needs N/R <= 32 in every pass).
__host__ __device__ constexpr bool warp_fft_ok(int n) {
  return n == 16 || n == 32 || n == 48 || n == 64 || n == 96 || n == 128 || n == 256;
}

// TP: tw is this pass's slice of the per-pass twiddle table (build_twp),
// indexed r NS + k, instead of the plain table indexed r k N/(NS R).
template <int N, int R, int NS, int SIGN, bool TP = false, typename C>
__device__ __forceinline__ void wpass(C *__restrict__ buf, int nsig, int sstr,
                                      const C *__restrict__ tw, int lane) {
  constexpr int NB = N / R;
  static_assert(NB <= 32, "warp pass needs N/R <= 32");
  constexpr int TMUL = N / (NS * R);
  constexpr int SPR = 32 / NB;
  const int sl = lane / NB, b = lane % NB, k = b % NS;
  const int idx = (b / NS) * NS * R + k;
  for (int s0 = 0; s0 < nsig; s0 += SPR) {
    const int s = s0 + sl;
    const bool act = (sl < SPR) && (s < nsig);
    C v[R];
    if (act) {
      const C *in = buf + s * sstr;
#pragma unroll
      for (int r = 0; r < R; r++) {
        C x = in[pad(b + r * NB)];
        if (NS > 1 && r > 0) {
          C t = TP ? tw[r * NS + k] : tw[r * k * TMUL];
          if (SIGN > 0) t.y = -t.y;
          x = cmul(x, t);
        }
        v[r] = x;
      }
      dft<R>(v, SIGN);
    }
    __syncwarp();
    if (act) {
      C *out = buf + s * sstr;
#pragma unroll
      for (int r = 0; r < R; r++) out[pad(idx + r * NS)] = v[r];
    }
    __syncwarp();
  }
}

// Per-pass twiddle table of a compile-time plan: for every pass p >= 1
// (radix R_p, running span NS_p) the R_p x NS_p factors W^(r k N/(NS_p R_p)),
// k fastest.  The lanes of a warp pass take consecutive k, so they read
// consecutive entries; indexing the plain table by r k N/(NS R) strides it
// and conflicts in the shared-memory banks.  Same values as the plain
// table: results do not change.
template <int N, int V>
__host__ __device__ constexpr int twp_off(int p) {
  int o = 0;
  for (int q = 1; q < p; q++) o += plan_radix(N, q, V) * plan_ns(N, q, V);
  return o;
}
template <int N, int V>
__host__ __device__ constexpr int twp_len() { return twp_off<N, V>(plan_passes(N)); }
// lengths whose warp passes take the per-pass table in the space of the plain one
__host__ __device__ constexpr bool tp_ok(int N) {
  return N == 16 || N == 32 || N == 48 || N == 64 || N == 128 || N == 256;
}
template <int N, int V = 0, typename C>
__device__ __forceinline__ void build_twp(C *twp, const C *__restrict__ tw, int tid, int nthr) {
  static_assert(twp_len<N, V>() <= N, "per-pass table longer than the plain one");
  for (int i = tid; i < twp_len<N, V>(); i += nthr) {
    int p = 1;
    while (i >= twp_off<N, V>(p + 1)) p++;
    const int R = plan_radix(N, p, V), NS = plan_ns(N, p, V);
    const int e = i - twp_off<N, V>(p);
    const int r = e / NS, k = e - r * NS;
    twp[i] = tw[r * k * (N / (NS * R))];
  }
}
// the twiddles a kernel stages: the per-pass table where its warp passes
// take one (TP), the plain table otherwise
template <int N, int V, bool TP, typename C>
__device__ __forceinline__ void stage_tw(C *stw, const C *__restrict__ tw, int n, int tid,
                                         int nthr) {
  if constexpr (TP) build_twp<N, V>(stw, tw, tid, nthr);
  else
    for (int i = tid; i < n; i += nthr) stw[i] = tw[i];
}

template <int N, int SIGN, int P, int V = 0, bool TP = false, typename C>
__device__ __forceinline__ void wpasses(C *buf, int nsig, int sstr, const C *tw,
                                        int lane) {
  constexpr int R = plan_radix(N, P, V);
  if constexpr (R != 0) {
    wpass<N, R, plan_ns(N, P, V), SIGN, TP>(buf, nsig, sstr, TP ? tw + twp_off<N, V>(P) : tw,
                                            lane);
    wpasses<N, SIGN, P + 1, V, TP>(buf, nsig, sstr, tw, lane);
  }
}

// Warp pass with more butterflies than lanes (N/R > 32): lane l takes
// butterflies l, l + 32, ... of one signal at a time, all loaded before the
// __syncwarp and stored after it.  Same butterflies and twiddles as the CTA
// passes, so the results are identical.
template <int N, int R, int NS, int SIGN, bool TP = false, typename C>
__device__ __forceinline__ void wpass_m(C *__restrict__ buf, int nsig, int sstr,
                                        const C *__restrict__ tw, int lane) {
  constexpr int NB = N / R;
  constexpr int M = (NB + 31) / 32;
  constexpr int TMUL = N / (NS * R);
  for (int s = 0; s < nsig; s++) {
    C v[M][R];
    const C *in = buf + s * sstr;
#pragma unroll
    for (int m = 0; m < M; m++) {
      const int b = lane + 32 * m;
      if (NB % 32 == 0 || b < NB) {
        const int k = b % NS;
#pragma unroll
        for (int r = 0; r < R; r++) {
          C x = in[pad(b + r * NB)];
          if (NS > 1 && r > 0) {
            C t = TP ? tw[r * NS + k] : tw[r * k * TMUL];
            if (SIGN > 0) t.y = -t.y;
            x = cmul(x, t);
          }
          v[m][r] = x;
        }
        dft<R>(v[m], SIGN);
      }
    }
    __syncwarp();
    C *out = buf + s * sstr;
#pragma unroll
    for (int m = 0; m < M; m++) {
      const int b = lane + 32 * m;
      if (NB % 32 == 0 || b < NB) {
        const int k = b % NS;
        const int idx = (b / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) out[pad(idx + r * NS)] = v[m][r];
      }
    }
    __syncwarp();
  }
}

// warp passes for any compile-time length: signal-parallel where N/R <= 32,
// butterfly-parallel above
template <int N, int SIGN, int P, int V = 0, bool TP = false, typename C>
__device__ __forceinline__ void wpasses_any(C *buf, int nsig, int sstr, const C *tw, int lane) {
  constexpr int R = plan_radix(N, P, V);
  if constexpr (R != 0) {
    const C *twp = TP ? tw + twp_off<N, V>(P) : tw;
    if constexpr (N / R <= 32) wpass<N, R, plan_ns(N, P, V), SIGN, TP>(buf, nsig, sstr, twp, lane);
    else wpass_m<N, R, plan_ns(N, P, V), SIGN, TP>(buf, nsig, sstr, twp, lane);
    wpasses_any<N, SIGN, P + 1, V, TP>(buf, nsig, sstr, tw, lane);
  }
}

// First pass of an inverse transform whose input is zero in the truncated
// band [N/3 + 1, N - N/3 - 1] (the 2/3-rule modes the reference zeroes
// before FFT_XZ_TO_PHYSICAL, for/mpi.f:1640-1655): the pass reads nothing
// there, so the band of the buffer need not be written beforehand.  NS = 1:
// no twiddles; the output index of butterfly b is b R + r.
template <int N, int R, int SIGN, typename C>
__device__ __forceinline__ void wpass_first_pz(C *__restrict__ buf, int nsig, int sstr,
                                               int lane) {
  constexpr int NB = N / R;
  static_assert(NB <= 32, "warp pass needs N/R <= 32");
  constexpr int SPR = 32 / NB;
  constexpr int ZLO = N / 3 + 1, ZHI = N - N / 3 - 1;
  const int sl = lane / NB, b = lane % NB;
  for (int s0 = 0; s0 < nsig; s0 += SPR) {
    const int s = s0 + sl;
    const bool act = (sl < SPR) && (s < nsig);
    C v[R];
    if (act) {
      const C *in = buf + s * sstr;
#pragma unroll
      for (int r = 0; r < R; r++) {
        const int e = b + r * NB;
        v[r] = (e >= ZLO && e <= ZHI) ? CT<C>::mk(0, 0) : in[pad(e)];
      }
      dft<R>(v, SIGN);
    }
    __syncwarp();
    if (act) {
      C *out = buf + s * sstr;
#pragma unroll
      for (int r = 0; r < R; r++) out[pad(b * R + r)] = v[r];
    }
    __syncwarp();
  }
}

// whole transform with the pruned first pass (lengths whose first pass has
// at most 32 butterflies; others take wpasses_any)
template <int N, int SIGN, int V = 0, bool TP = false, typename C>
__device__ __forceinline__ void wpasses_pz(C *buf, int nsig, int sstr, const C *tw, int lane) {
  constexpr int R0 = plan_radix(N, 0, V);
  if constexpr (N / R0 <= 32) {
    wpass_first_pz<N, R0, SIGN>(buf, nsig, sstr, lane);
    wpasses_any<N, SIGN, 1, V, TP>(buf, nsig, sstr, tw, lane);
  } else {
    wpasses_any<N, SIGN, 0, V, TP>(buf, nsig, sstr, tw, lane);
  }
}

// Compile-time lengths run in place in buf0 (buf1 unused); the runtime plan
// ping-pongs between buf0 and buf1.
template <int N, int V = 0, typename C>
__device__ __forceinline__ C *fft(C *buf0, C *buf1, const FftPlan &pl, int nsig,
                                        int sig_stride, const C *tw, int sign) {
  if constexpr (N == 0) {
    return run(buf0, buf1, pl, nsig, sig_stride, tw, sign);
  } else {
    const int tid = threadIdx.x, nthr = blockDim.x;
    if (sign < 0) ippasses<N, -1, 0, V>(buf0, nsig, sig_stride, tw, tid, nthr);
    else ippasses<N, +1, 0, V>(buf0, nsig, sig_stride, tw, tid, nthr);
    return buf0;
  }
}

// CTA front end: with a warp-capable length the signals are dealt out to the
// warps (no CTA barrier between passes), otherwise the CTA-wide passes run.
// (For 192, 384 and 512 the CTA-wide passes measured faster here than
// butterfly-parallel warp passes: fewer registers, more resident CTAs.)
template <int N, int V = 0, bool TP = false, typename C>
__device__ __forceinline__ C *fft_cta(C *buf0, C *buf1, const FftPlan &pl,
                                            int nsig, int sig_stride, const C *tw,
                                            int sign) {
  if constexpr (N != 0 && warp_fft_ok(N)) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int per = (nsig + nw - 1) / nw;
    const int s0 = warp * per;
    const int ns = (nsig - s0) < per ? (nsig - s0) : per;
    if (ns > 0) {
      if (sign < 0)
        wpasses_any<N, -1, 0, V, TP>(buf0 + (long)s0 * sig_stride, ns, sig_stride, tw, lane);
      else
        wpasses_any<N, +1, 0, V, TP>(buf0 + (long)s0 * sig_stride, ns, sig_stride, tw, lane);
    }
    __syncthreads();
    return buf0;
  } else {
    return fft<N, V>(buf0, buf1, pl, nsig, sig_stride, tw, sign);
  }
}

// CTA front end of an inverse transform with the truncated band unread
// (wpass_first_pz); warp-capable lengths only
template <int N, int V = 0, bool TP = false, typename C>
__device__ __forceinline__ C *fft_cta_inv_pz(C *buf0, int nsig, int sig_stride, const C *tw) {
  static_assert(N != 0 && warp_fft_ok(N), "pruned transforms need a warp-capable length");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int per = (nsig + nw - 1) / nw;
  const int s0 = warp * per;
  const int ns = (nsig - s0) < per ? (nsig - s0) : per;
  if (ns > 0) wpasses_pz<N, +1, V, TP>(buf0 + (long)s0 * sig_stride, ns, sig_stride, tw, lane);
  __syncthreads();
  return buf0;
}

// shared buffers a transform of length n needs (1 in place, 2 ping-pong)
__host__ __device__ constexpr int fft_bufs(int n) {
  return (n == 16 || n == 32 || n == 48 || n == 64 || n == 96 || n == 128 || n == 192 ||
          n == 256 || n == 384 || n == 512) ? 1 : 2;
}

}  // namespace dgfft

// Supported compile-time lengths; anything else takes the runtime plan.
#define DG_FOR_EACH_N(X) X(16) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512)
