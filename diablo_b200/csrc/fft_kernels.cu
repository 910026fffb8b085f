// Plane transforms between the retained-mode spectral layout and physical
// space, built from the shared-memory Stockham FFT in fft.cuh.
//
//   zinv : spectral [j][kz][kx] -> half-physical H [j][z][kx]   (c2c along z, +1)
//   xc2r : H [j][z][kx]         -> physical rows                  (c2r along x)
//   xr2c : physical rows        -> H [j][z][kx] / NX              (r2c along x)
//   zfwd : H [j][z][kx]         -> spectral [j][kz][kx] / NZ      (c2c along z, -1)
//
// Packing follows FFT_XZ_TO_FOURIER / FFT_XZ_TO_PHYSICAL (for/mpi.f:1530-1674):
// kz = 0..NKZ at 0..NKZ, kz = -NKZ..-1 at NKZ+1..TNKZ; |kz| > NKZ, kx > NKX
// and the x-Nyquist bin are zero on the way to physical space.  Real
// transforms use the two-real-rows-per-complex-transform identity; the
// imaginary parts of the x-DC and x-Nyquist bins are ignored by the c2r, as in
// FFTW's complex-to-real.
#include <mutex>
#include <type_traits>
#include <unordered_set>

#include "dg_internal.cuh"
#include "fft.cuh"

using namespace dgfft;

namespace {

// signals per CTA: 16 for lengths <= 128, fewer for longer transforms so the
// two shared buffers stay near 70 KB
__host__ __device__ constexpr int batch_for(int n) {
  return n <= 128 ? 16 : (n <= 256 ? 8 : 4);
}
constexpr int NTHR = 128;

__device__ __forceinline__ int packed_index(int z, int NZ, int NKZ) {
  // physical-order z bin -> packed kz slot, or -1 if not retained
  if (z <= NKZ) return z;
  if (z >= NZ - NKZ) return z - NZ + 1 + 2 * NKZ;
  return -1;
}

template <int NT, typename CX, typename PA = CFieldPtrs, int PV = 0>
__global__ void __launch_bounds__(NTHR) k_zinv(PA fields, int jmin, long ss, int nkxp,
                                              int NZr, int NKZ, FftPlan pl,
                                              const CX *__restrict__ tw,
                                              CX *__restrict__ H, long Hfield) {
  extern __shared__ double2 sm_raw[];
  CX *sm = reinterpret_cast<CX *>(sm_raw);
  const int NZ = NT ? NT : NZr;
  const int KXG = batch_for(NZ);
  const int sstr = padded_len(NZ);
  CX *stw = sm;
  CX *b0 = stw + NZ;
  CX *b1 = b0 + KXG * sstr;
  const int kx0 = blockIdx.x * KXG;
  const int j = jmin + blockIdx.y;
  const int f = blockIdx.z;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const auto *in = fields(f) + (long)j * ss;
  for (int i = tid; i < NZ; i += nthr) stw[i] = tw[i];
  dg_pdl_wait();
  for (int base = 0; base < KXG * NZ; base += 8 * nthr) {
    using CI = typename std::remove_const<typename std::remove_pointer<decltype(in)>::type>::type;
    CI v[8];
    const CI zero{};
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * nthr + tid;
      const int c = idx % KXG, z = idx / KXG;
      const int kp = packed_index(z, NZ, NKZ);
      v[u] = (idx < KXG * NZ && kp >= 0 && kx0 + c < nkxp) ? in[(long)kp * nkxp + kx0 + c] : zero;
    }
    // with a compile-time length the first pass skips the truncated band
    // (NK = N/3), so its zeros are not stored
    constexpr bool PRUNED = NT != 0 && warp_fft_ok(NT);
    const bool pz = PRUNED && NKZ == NZ / 3;
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * nthr + tid;
      const int z = idx / KXG;
      if (idx < KXG * NZ && !(pz && z > NKZ && z < NZ - NKZ))
        b0[(idx % KXG) * sstr + pad(z)] =
            CT<CX>::mk((typename CT<CX>::T)v[u].x, (typename CT<CX>::T)v[u].y);
    }
  }
  __syncthreads();
  CX *res;
  if constexpr (NT != 0 && warp_fft_ok(NT)) {
    if (NKZ == NZ / 3) res = fft_cta_inv_pz<NT, PV>(b0, KXG, sstr, stw);
    else res = fft_cta<NT, PV>(b0, b1, pl, KXG, sstr, stw, +1);
  } else {
    res = fft_cta<NT, PV>(b0, b1, pl, KXG, sstr, stw, +1);
  }
  CX *out = H + f * Hfield + (long)j * NZ * nkxp;
  for (int idx = tid; idx < KXG * NZ; idx += nthr) {
    const int c = idx % KXG, z = idx / KXG;
    if (kx0 + c < nkxp) out[(long)z * nkxp + kx0 + c] = res[c * sstr + pad(z)];
  }
}

template <int NT, typename CX = double2, typename PO = FieldPtrs>
__global__ void __launch_bounds__(NTHR) k_zfwd(const CX *__restrict__ H, long Hfield, int jmin,
                                              int nkxp, int nkzt, int NZr, int NKZ, FftPlan pl,
                                              const CX *__restrict__ tw, PO fields,
                                              long ss) {
  extern __shared__ double2 sm_raw[];
  CX *sm = reinterpret_cast<CX *>(sm_raw);
  const int NZ = NT ? NT : NZr;
  const int KXG = batch_for(NZ);
  const int sstr = padded_len(NZ);
  CX *stw = sm;
  CX *b0 = stw + NZ;
  CX *b1 = b0 + KXG * sstr;
  const int kx0 = blockIdx.x * KXG;
  const int j = jmin + blockIdx.y;
  const int f = blockIdx.z;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const CX *in = H + f * Hfield + (long)j * NZ * nkxp;
  for (int i = tid; i < NZ; i += nthr) stw[i] = tw[i];
  for (int base = 0; base < KXG * NZ; base += 8 * nthr) {
    CX v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * nthr + tid;
      const int c = idx % KXG, z = idx / KXG;
      v[u] = (idx < KXG * NZ && kx0 + c < nkxp) ? in[(long)z * nkxp + kx0 + c] : CT<CX>::mk(0, 0);
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int idx = base + u * nthr + tid;
      if (idx < KXG * NZ) b0[(idx % KXG) * sstr + pad(idx / KXG)] = v[u];
    }
  }
  __syncthreads();
  CX *res = fft_cta<NT>(b0, b1, pl, KXG, sstr, stw, -1);
  auto *out = fields(f) + (long)j * ss;
  using CO = typename std::remove_pointer<decltype(out)>::type;
  using TO = typename CT<CO>::T;
  const double rnz = (double)NZ;
  for (int idx = tid; idx < KXG * nkzt; idx += nthr) {
    const int c = idx % KXG, kp = idx / KXG;
    if (kx0 + c >= nkxp) continue;
    const int z = (kp <= NKZ) ? kp : (NZ - 1 + (kp - NKZ) - NKZ);
    const CX v = res[c * sstr + pad(z)];
    out[(long)kp * nkxp + kx0 + c] = CT<CO>::mk((TO)((double)v.x / rnz), (TO)((double)v.y / rnz));
  }
}

// c2r of RPAIR row pairs of one plane of one field.
template <int NT>
__global__ void __launch_bounds__(NTHR) k_xc2r(const double2 *__restrict__ H, long Hfield, int jmin,
                                              int nkxp, int NXr, int NZ, FftPlan pl,
                                              const double2 *__restrict__ tw,
                                              double *__restrict__ phys, long pplane, long prow,
                                              long pfield) {
  extern __shared__ double2 sm[];
  const int NX = NT ? NT : NXr;
  const int RPAIR = batch_for(NX);
  const int sstr = padded_len(NX);
  double2 *stw = sm;
  double2 *b0 = stw + NX;
  double2 *b1 = b0 + RPAIR * sstr;
  const int z0 = blockIdx.x * 2 * RPAIR;
  const int j = jmin + blockIdx.y;
  const int f = blockIdx.z;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const double2 *in = H + f * Hfield + (long)j * NZ * nkxp;
  const int NKX = nkxp - 1;
  for (int i = tid; i < NX; i += nthr) stw[i] = tw[i];
  // bin k of Z = A + iB with the Hermitian extension of A and B (A_k + i B_k
  // for k <= NX/2, conj(A_k) + i conj(B_k) above); loads four bins at a time
  for (int base = 0; base < RPAIR * NX; base += 4 * nthr) {
    double2 av[4], bv[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int idx = base + u * nthr + tid;
      const int q = idx / NX, k = idx % NX;
      const int za = z0 + 2 * q, zb = za + 1;
      const int kk = (k <= NX / 2) ? k : NX - k;
      const bool ok = idx < RPAIR * NX && za < NZ && kk <= NKX && kk < NX / 2;
      av[u] = ok ? in[(long)za * nkxp + kk] : make_double2(0.0, 0.0);
      bv[u] = (ok && zb < NZ) ? in[(long)zb * nkxp + kk] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int idx = base + u * nthr + tid;
      if (idx >= RPAIR * NX) continue;
      const int q = idx / NX, k = idx % NX;
      const int kk = (k <= NX / 2) ? k : NX - k;
      double2 a = av[u], b = bv[u];
      if (kk == 0) {
        a.y = 0.0;
        b.y = 0.0;
      }
      b0[q * sstr + pad(k)] =
          (k == kk) ? make_double2(a.x - b.y, a.y + b.x) : make_double2(a.x + b.y, -a.y + b.x);
    }
  }
  __syncthreads();
  double2 *res = fft_cta<NT>(b0, b1, pl, RPAIR, sstr, stw, +1);
  double *out = phys + f * pfield + (long)j * pplane;
  for (int idx = tid; idx < RPAIR * NX; idx += nthr) {
    const int q = idx / NX, x = idx % NX;
    const int za = z0 + 2 * q, zb = za + 1;
    const double2 v = res[q * sstr + pad(x)];
    if (za < NZ) out[(long)za * prow + x] = v.x;
    if (zb < NZ) out[(long)zb * prow + x] = v.y;
  }
}

// c2r of RPAIR row pairs followed by COURANT's per-point limit
// min(CFL d / |u|) (for/courant.f:35-44) instead of a store: field 0 uses DX,
// field 1 DY(j), field 2 DZ.  The minimum goes to *out as ordered bits.
template <int NT, int PV = 0>
__global__ void __launch_bounds__(NTHR) k_xc2r_cfl(const double2 *__restrict__ H, long Hfield,
                                                   int jmin, int nkxp, int NXr, int NZ, FftPlan pl,
                                                   const double2 *__restrict__ tw, double cfl,
                                                   double dxv, double dzv,
                                                   const double *__restrict__ dy,
                                                   unsigned long long *__restrict__ out) {
  extern __shared__ double2 sm[];
  const int NX = NT ? NT : NXr;
  const int RPAIR = batch_for(NX);
  const int sstr = padded_len(NX);
  double2 *stw = sm;
  double2 *b0 = stw + NX;
  double2 *b1 = b0 + RPAIR * sstr;
  const int z0 = blockIdx.x * 2 * RPAIR;
  const int j = jmin + blockIdx.y;
  const int f = blockIdx.z;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const double2 *in = H + f * Hfield + (long)j * NZ * nkxp;
  const int NKX = nkxp - 1;
  for (int i = tid; i < NX; i += nthr) stw[i] = tw[i];
  dg_pdl_wait();
  // bin k of Z = A + iB with the Hermitian extension of A and B; the row-pair
  // loads are issued four bins at a time per thread
  for (int base = 0; base < RPAIR * NX; base += 4 * nthr) {
    double2 av[4], bv[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int idx = base + u * nthr + tid;
      const int q = idx / NX, k = idx % NX;
      const int za = z0 + 2 * q, zb = za + 1;
      const int kk = (k <= NX / 2) ? k : NX - k;
      const bool ok = idx < RPAIR * NX && za < NZ && kk <= NKX && kk < NX / 2;
      av[u] = ok ? in[(long)za * nkxp + kk] : make_double2(0.0, 0.0);
      bv[u] = (ok && zb < NZ) ? in[(long)zb * nkxp + kk] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int idx = base + u * nthr + tid;
      if (idx >= RPAIR * NX) continue;
      const int q = idx / NX, k = idx % NX;
      const int kk = (k <= NX / 2) ? k : NX - k;
      double2 a = av[u], b = bv[u];
      if (kk == 0) {
        a.y = 0.0;
        b.y = 0.0;
      }
      b0[q * sstr + pad(k)] =
          (k == kk) ? make_double2(a.x - b.y, a.y + b.x) : make_double2(a.x + b.y, -a.y + b.x);
    }
  }
  __syncthreads();
  double2 *res = fft_cta<NT, PV>(b0, b1, pl, RPAIR, sstr, stw, +1);
  const double d = (f == 0) ? dxv : (f == 1 ? dy[j] : dzv);
  // min over points of CFL d / |u| is CFL d / max |u| (division is correctly
  // rounded and monotone), so only the largest |u| of the CTA is divided
  double big = 0.0;
  for (int idx = tid; idx < RPAIR * NX; idx += nthr) {
    const int q = idx / NX, x = idx % NX;
    const int za = z0 + 2 * q, zb = za + 1;
    const double2 v = res[q * sstr + pad(x)];
    if (za < NZ) big = fmax(big, fabs(v.x));
    if (zb < NZ) big = fmax(big, fabs(v.y));
  }
  for (int off = 16; off > 0; off >>= 1) big = fmax(big, __shfl_down_sync(0xffffffffu, big, off));
  // the CTA's warps reduced in shared memory, folded into the minimum once
  __shared__ double wbig[NTHR / 32];
  if ((tid & 31) == 0) wbig[tid >> 5] = big;
  __syncthreads();
  if (tid == 0) {
    double m = wbig[0];
#pragma unroll
    for (int w = 1; w < NTHR / 32; w++) m = fmax(m, wbig[w]);
    dg_fold_min(out, cfl * d / m);  // +inf for an all-zero slab, as before
  }
}

// r2c of RPAIR row pairs of one plane of one field; keeps kx = 0..NKX, / NX.
template <int NT>
__global__ void __launch_bounds__(NTHR) k_xr2c(const double *__restrict__ phys, long pplane,
                                              long prow, long pfield, int jmin, int nkxp, int NXr,
                                              int NZ, FftPlan pl, const double2 *__restrict__ tw,
                                              double2 *__restrict__ H, long Hfield) {
  extern __shared__ double2 sm[];
  const int NX = NT ? NT : NXr;
  const int RPAIR = batch_for(NX);
  const int sstr = padded_len(NX);
  double2 *stw = sm;
  double2 *b0 = stw + NX;
  double2 *b1 = b0 + RPAIR * sstr;
  const int z0 = blockIdx.x * 2 * RPAIR;
  const int j = jmin + blockIdx.y;
  const int f = blockIdx.z;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const double *in = phys + f * pfield + (long)j * pplane;
  for (int i = tid; i < NX; i += nthr) stw[i] = tw[i];
  for (int idx = tid; idx < RPAIR * NX; idx += nthr) {
    const int q = idx / NX, x = idx % NX;
    const int za = z0 + 2 * q, zb = za + 1;
    double a = (za < NZ) ? in[(long)za * prow + x] : 0.0;
    double b = (zb < NZ) ? in[(long)zb * prow + x] : 0.0;
    b0[q * sstr + pad(x)] = make_double2(a, b);
  }
  __syncthreads();
  double2 *res = fft_cta<NT>(b0, b1, pl, RPAIR, sstr, stw, -1);
  double2 *out = H + f * Hfield + (long)j * NZ * nkxp;
  const double rnx = (double)NX;
  for (int idx = tid; idx < RPAIR * nkxp; idx += nthr) {
    const int q = idx / nkxp, k = idx % nkxp;
    const int za = z0 + 2 * q, zb = za + 1;
    const double2 zk = res[q * sstr + pad(k)];
    const double2 zm = res[q * sstr + pad((NX - k) % NX)];
    // A = (Z_k + conj Z_{N-k})/2, B = -i/2 (Z_k - conj Z_{N-k})
    const double2 A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
    const double2 B = make_double2(0.5 * (zk.y + zm.y), -0.5 * (zk.x - zm.x));
    if (za < NZ) out[(long)za * nkxp + k] = make_double2(A.x / rnx, A.y / rnx);
    if (zb < NZ) out[(long)zb * nkxp + k] = make_double2(B.x / rnx, B.y / rnx);
  }
}

// ------------------------------------------- whole-plane transforms (x-z)
// One CTA per (plane, field) moves a plane between the retained-mode layout
// and physical rows without the half-physical staging array: the plane's
// NKX+1 z columns (NZ bins each) stay in shared memory between the z and
// the x transform.  Same passes, plans and twiddles as k_zinv + k_xc2r and
// k_xr2c + k_zfwd (the plan variant 0), so the results are the same.
// Requires NKX = NX/3 and NKZ = NZ/3 (the truncated bands the pruned first
// passes skip).  Shared memory: the columns [NKX+1][SZ] (SZ odd, so the x
// stage's reads across the columns hit distinct banks) and two row-pair
// signals per warp.
constexpr int PL_THR = 128;

// 16-byte asynchronous copy global -> shared (both addresses 16-byte aligned)
__device__ __forceinline__ void pl_cp16(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
// wait for every copy this thread issued
__device__ __forceinline__ void pl_cp_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

__host__ __device__ constexpr int pl_sz(int nz) { return padded_len(nz) | 1; }
__host__ __device__ constexpr size_t pl_smem(int nx, int nz) {
  return sizeof(double2) * ((size_t)(nx / 3 + 1) * pl_sz(nz) + (PL_THR / 32) * 2 * padded_len(nx));
}

template <int NXT, int NZT>
__global__ void __launch_bounds__(PL_THR, 2) k_plane_c2r(CFieldPtrs fields, int jmin, long ss,
                                                         const double2 *__restrict__ twz,
                                                         const double2 *__restrict__ twx,
                                                         double *__restrict__ phys, long pplane,
                                                         long prow, long pfield) {
  constexpr int NKXP = NXT / 3 + 1, NKZ = NZT / 3, NKZT = 2 * NKZ + 1;
  constexpr int SZ = pl_sz(NZT), SX = padded_len(NXT);
  extern __shared__ double2 sm[];
  double2 *Hs = sm;                   // [NKXP][SZ]: the z bins of every kx column
  double2 *xb = Hs + NKXP * SZ;       // [warp][2][SX]: row-pair signals
  const int j = jmin + blockIdx.x, f = blockIdx.y;
  const int tid = threadIdx.x;
  const double2 *in = fields(f) + (long)j * ss;
  // 1. retained modes into their z bins (the band stays unwritten: the
  // pruned first pass does not read it); eight loads in flight per thread
  // by asynchronous 16-byte copies, all of the plane's in flight at once
  for (int i = tid; i < NKZT * NKXP; i += PL_THR) {
    const int kp = i / NKXP, kx = i - kp * NKXP;
    const int z = (kp <= NKZ) ? kp : kp + NZT - NKZT;
    pl_cp16(Hs + kx * SZ + pad(z), in + i);
  }
  pl_cp_wait_all();
  __syncthreads();
  // 2. z inverse of every column
  fft_cta_inv_pz<NZT, 0>(Hs, NKXP, SZ, twz);
  // 3. x c2r of row pairs (za, za + 1), two pairs per warp at a time: bin k
  // of Z = A + iB with the Hermitian extension above NX/2 (as k_xc2r)
  const int warp = tid >> 5, lane = tid & 31;
  double2 *xw = xb + warp * 2 * SX;
  double *out = phys + f * pfield + (long)j * pplane;
  for (int p0 = 2 * warp; p0 < NZT / 2; p0 += 2 * (PL_THR / 32)) {
    const int np = (NZT / 2 - p0) < 2 ? (NZT / 2 - p0) : 2;
    for (int q = 0; q < np; q++) {
      const int za = 2 * (p0 + q), zb = za + 1;
#pragma unroll
      for (int i = 0; i < (NXT + 31) / 32; i++) {
        const int k = lane + 32 * i;
        const int kk = (k <= NXT / 2) ? k : NXT - k;
        if (k < NXT && kk < NKXP && kk < NXT / 2) {
          double2 a = Hs[kk * SZ + pad(za)], b = Hs[kk * SZ + pad(zb)];
          if (kk == 0) {
            a.y = 0.0;
            b.y = 0.0;
          }
          xw[q * SX + pad(k)] = (k == kk) ? make_double2(a.x - b.y, a.y + b.x)
                                          : make_double2(a.x + b.y, -a.y + b.x);
        }
      }
    }
    __syncwarp();
    wpasses_pz<NXT, +1, 0, false>(xw, np, SX, twx, lane);
    for (int q = 0; q < np; q++) {
      const int za = 2 * (p0 + q), zb = za + 1;
#pragma unroll
      for (int i = 0; i < (NXT + 31) / 32; i++) {
        const int x = lane + 32 * i;
        if (x < NXT) {
          const double2 v = xw[q * SX + pad(x)];
          out[(long)za * prow + x] = v.x;
          out[(long)zb * prow + x] = v.y;
        }
      }
    }
    __syncwarp();
  }
}

template <int NXT, int NZT>
__global__ void __launch_bounds__(PL_THR, 2) k_plane_r2c(const double *__restrict__ phys,
                                                         long pplane, long prow, long pfield,
                                                         int jmin,
                                                         const double2 *__restrict__ twx,
                                                         const double2 *__restrict__ twz,
                                                         FieldPtrs fields, long ss) {
  constexpr int NKXP = NXT / 3 + 1, NKZ = NZT / 3, NKZT = 2 * NKZ + 1;
  constexpr int SZ = pl_sz(NZT), SX = padded_len(NXT);
  extern __shared__ double2 sm[];
  double2 *Hs = sm;
  double2 *xb = Hs + NKXP * SZ;
  const int j = jmin + blockIdx.x, f = blockIdx.y;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  double2 *xw = xb + warp * 2 * SX;
  const double *in = phys + f * pfield + (long)j * pplane;
  const double rnx = (double)NXT;
  // 1. x r2c of row pairs into the kx columns, kx = 0..NKX, / NX (as k_xr2c);
  // a round's rows are loaded while the previous round transforms
  constexpr int XPL = (NXT + 31) / 32;
  constexpr int PSTEP = 2 * (PL_THR / 32);
  double va[2][XPL], vb[2][XPL];
  auto fetch = [&](int p) {
#pragma unroll
    for (int q = 0; q < 2; q++)
#pragma unroll
      for (int i = 0; i < XPL; i++) {
        const int x = lane + 32 * i, za = 2 * (p + q);
        const bool ok = p + q < NZT / 2 && x < NXT;
        va[q][i] = ok ? in[(long)za * prow + x] : 0.0;
        vb[q][i] = ok ? in[(long)(za + 1) * prow + x] : 0.0;
      }
  };
  if (2 * warp < NZT / 2) fetch(2 * warp);
  for (int p0 = 2 * warp; p0 < NZT / 2; p0 += PSTEP) {
    const int np = (NZT / 2 - p0) < 2 ? (NZT / 2 - p0) : 2;
#pragma unroll
    for (int q = 0; q < 2; q++)
#pragma unroll
      for (int i = 0; i < XPL; i++) {
        const int x = lane + 32 * i;
        if (q < np && x < NXT) xw[q * SX + pad(x)] = make_double2(va[q][i], vb[q][i]);
      }
    __syncwarp();
    if (p0 + PSTEP < NZT / 2) fetch(p0 + PSTEP);
    wpasses_any<NXT, -1, 0, 0, false>(xw, np, SX, twx, lane);
    for (int q = 0; q < np; q++) {
      const int za = 2 * (p0 + q), zb = za + 1;
      for (int k = lane; k < NKXP; k += 32) {
        const double2 zk = xw[q * SX + pad(k)];
        const double2 zm = xw[q * SX + pad((NXT - k) % NXT)];
        const double2 A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
        const double2 B = make_double2(0.5 * (zk.y + zm.y), -0.5 * (zk.x - zm.x));
        Hs[k * SZ + pad(za)] = make_double2(A.x / rnx, A.y / rnx);
        Hs[k * SZ + pad(zb)] = make_double2(B.x / rnx, B.y / rnx);
      }
    }
    __syncwarp();
  }
  __syncthreads();
  // 2. z forward of every column
  FftPlan none{};
  fft_cta<NZT>(Hs, Hs, none, NKXP, SZ, twz, -1);
  // 3. retained modes out, / NZ (as k_zfwd)
  double2 *out = fields(f) + (long)j * ss;
  const double rnz = (double)NZT;
  for (int i = tid; i < NKZT * NKXP; i += PL_THR) {
    const int kp = i / NKXP, kx = i - kp * NKXP;
    const int z = (kp <= NKZ) ? kp : kp + NZT - NKZT;
    const double2 v = Hs[kx * SZ + pad(z)];
    out[i] = make_double2(v.x / rnz, v.y / rnz);
  }
}

size_t zsmem(int NZ, size_t esz = sizeof(double2)) {
  return esz * (NZ + fft_bufs(NZ) * batch_for(NZ) * padded_len(NZ));
}
size_t xsmem(int NX) { return sizeof(double2) * (NX + fft_bufs(NX) * batch_for(NX) * padded_len(NX)); }

}  // namespace

void dg_big_smem(const void *kern) {
  static std::mutex mu;
  static std::unordered_set<const void *> done;
  std::lock_guard<std::mutex> lk(mu);
  if (done.insert(kern).second)
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
}

namespace {
template <typename K>
void big_smem(K kern) {
  dg_big_smem((const void *)kern);
}

// the plan variant the handle's tuning chose, for lengths that have one
template <int NN, typename CX, typename PA>
auto zinv_kernel(int v) {
  if constexpr (NN != 0 && plan_has_variant(NN))
    if (v) return k_zinv<NN, CX, PA, 1>;
  return k_zinv<NN, CX, PA, 0>;
}
template <int NN>
auto xc2r_cfl_kernel(int v) {
  if constexpr (NN != 0 && plan_has_variant(NN))
    if (v) return k_xc2r_cfl<NN, 1>;
  return k_xc2r_cfl<NN, 0>;
}

}  // namespace

// ------------------------------------------------------------- host wrappers

// Column transforms along one axis for a batch of planes.  Geometry (per
// field): input plane j at fields[f] + j*in_plane, packed slot kp of column c
// at + kp*rowlen + c; output plane j at H + f*out_field + j*N*rowlen, bin z of
// column c at + z*rowlen + c.  z transforms: rowlen = NKX+1, planes = y;
// y transforms (periodic): rowlen = modes per ky-plane, one plane.
template <typename CI, typename CX>
static int cinv_t(dg_handle *h, const CI *const *fields, int nf, int jmin, int jmax,
                  long in_plane, int rowlen, int N, int NK, const FftPlan &pl, const CX *tw, CX *H,
                  long out_field) {
  using PA = PtrArray<const CI>;
  if (jmax < jmin || nf <= 0) return DG_OK;
  PA fp;
  for (int f = 0; f < nf; f++) fp.p[f] = fields[f];
  dim3 grid(dg_cdiv(rowlen, batch_for(N)), jmax - jmin + 1, nf);
  const size_t sm = zsmem(N, sizeof(CX));
#define KERNEL_BODY(NN)                                                                       \
  {                                                                                           \
    auto kern = zinv_kernel<NN, CX, PA>(h->fft_plan);                                         \
    big_smem(kern);                                                                           \
    dg_kt_begin(h, "k_zinv", h->st);                                                          \
    DG_CUDA(dg_launch(h->pdl_zinv, kern, grid, dim3(NTHR), sm, h->st, fp, jmin, in_plane,     \
                      rowlen, N, NK, pl, tw, H, out_field));                                  \
  }
  switch (N) {
    DG_FOR_EACH_N(DG_CASE_N)
    default: KERNEL_BODY(0); break;
  }
#undef KERNEL_BODY
  DG_LAUNCHED();
  return DG_OK;
}

int dg_cinv_g(dg_handle *h, const double2 *const *fields, int nf, int jmin, int jmax,
              long in_plane, int rowlen, int N, int NK, const FftPlan &pl, const double2 *tw,
              double2 *H, long out_field) {
  return cinv_t(h, fields, nf, jmin, jmax, in_plane, rowlen, N, NK, pl, tw, H, out_field);
}

int dg_cinv_gf(dg_handle *h, const double2 *const *fields, int nf, int jmin, int jmax,
               long in_plane, int rowlen, int N, int NK, const FftPlan &pl, const float2 *tw,
               float2 *H, long out_field) {
  return cinv_t(h, fields, nf, jmin, jmax, in_plane, rowlen, N, NK, pl, tw, H, out_field);
}

int dg_cinv_ff(dg_handle *h, const float2 *const *fields, int nf, int jmin, int jmax,
               long in_plane, int rowlen, int N, int NK, const FftPlan &pl, const float2 *tw,
               float2 *H, long out_field) {
  return cinv_t(h, fields, nf, jmin, jmax, in_plane, rowlen, N, NK, pl, tw, H, out_field);
}

template <typename CX, typename PO, typename OUT>
static int cfwd_t(dg_handle *h, const CX *H, long in_field, int nf, int jmin, int jmax, int rowlen,
                  int nkt, int N, int NK, const FftPlan &pl, const CX *tw, OUT *const *fields,
                  long out_plane) {
  if (jmax < jmin || nf <= 0) return DG_OK;
  PO fp;
  for (int f = 0; f < nf; f++) fp.p[f] = fields[f];
  dim3 grid(dg_cdiv(rowlen, batch_for(N)), jmax - jmin + 1, nf);
  const size_t sm = zsmem(N, sizeof(CX));
#define KERNEL_BODY(NN)                                                                        \
  big_smem(k_zfwd<NN, CX, PO>);                                                                \
  dg_kt_begin(h, "k_zfwd", h->st);                                                             \
  k_zfwd<NN, CX, PO><<<grid, NTHR, sm, h->st>>>(H, in_field, jmin, rowlen, nkt, N, NK, pl, tw, fp, \
                                               out_plane)
  switch (N) {
    DG_FOR_EACH_N(DG_CASE_N)
    default: KERNEL_BODY(0); break;
  }
#undef KERNEL_BODY
  DG_LAUNCHED();
  return DG_OK;
}

int dg_cfwd_g(dg_handle *h, const double2 *H, long in_field, int nf, int jmin, int jmax,
              int rowlen, int nkt, int N, int NK, const FftPlan &pl, const double2 *tw,
              double2 *const *fields, long out_plane) {
  return cfwd_t<double2, FieldPtrs>(h, H, in_field, nf, jmin, jmax, rowlen, nkt, N, NK, pl, tw,
                                    fields, out_plane);
}

int dg_cfwd_ff(dg_handle *h, const float2 *H, long in_field, int nf, int jmin, int jmax,
               int rowlen, int nkt, int N, int NK, const FftPlan &pl, const float2 *tw,
               float2 *const *fields, long out_plane) {
  return cfwd_t<float2, PtrArray<float2>>(h, H, in_field, nf, jmin, jmax, rowlen, nkt, N, NK, pl,
                                          tw, fields, out_plane);
}

int dg_zinv(dg_handle *h, const double2 *const *fields, int nf, int jmin, int jmax, double2 *H,
            int) {
  return dg_cinv_g(h, fields, nf, jmin, jmax, h->ss, h->nkxp, h->NZ, h->NKZ, h->plz, h->twz, H,
                   (long)h->nplanes * h->NZ * h->nkxp);
}

int dg_zfwd_planes(dg_handle *h, const double2 *H, int nf, int jmin, int jmax,
                   double2 *const *fields, double2 *, long) {
  return dg_cfwd_g(h, H, (long)h->nplanes * h->NZ * h->nkxp, nf, jmin, jmax, h->nkxp, h->nkzt,
                   h->NZ, h->NKZ, h->plz, h->twz, fields, h->ss);
}

int dg_xc2r_planes(dg_handle *h, const double2 *H, int nf, int jmin, int jmax, double *phys,
                   long pplane, long prow, long pfield) {
  if (jmax < jmin || nf <= 0) return DG_OK;
  dim3 grid(dg_cdiv(h->NZ, 2 * batch_for(h->NX)), jmax - jmin + 1, nf);
  const size_t sm = xsmem(h->NX);
  const long Hf = (long)h->nplanes * h->NZ * h->nkxp;
#define KERNEL_BODY(N)                                                                     \
  big_smem(k_xc2r<N>);                                                                     \
  dg_kt_begin(h, "k_xc2r", h->st);                                                                \
  k_xc2r<N><<<grid, NTHR, sm, h->st>>>(H, Hf, jmin, h->nkxp, h->NX, h->NZ, h->plx, h->twx, phys, \
                                      pplane, prow, pfield)
  switch (h->NX) {
    DG_FOR_EACH_N(DG_CASE_N)
    default: KERNEL_BODY(0); break;
  }
#undef KERNEL_BODY
  DG_LAUNCHED();
  return DG_OK;
}

int dg_xr2c_planes(dg_handle *h, const double *phys, int nf, int jmin, int jmax, long pplane,
                   long prow, long pfield, double2 *H) {
  if (jmax < jmin || nf <= 0) return DG_OK;
  dim3 grid(dg_cdiv(h->NZ, 2 * batch_for(h->NX)), jmax - jmin + 1, nf);
  const size_t sm = xsmem(h->NX);
  const long Hf = (long)h->nplanes * h->NZ * h->nkxp;
#define KERNEL_BODY(N)                                                                        \
  big_smem(k_xr2c<N>);                                                                        \
  dg_kt_begin(h, "k_xr2c", h->st);                                                                 \
  k_xr2c<N><<<grid, NTHR, sm, h->st>>>(phys, pplane, prow, pfield, jmin, h->nkxp, h->NX, h->NZ,   \
                                      h->plx, h->twx, H, Hf)
  switch (h->NX) {
    DG_FOR_EACH_N(DG_CASE_N)
    default: KERNEL_BODY(0); break;
  }
#undef KERNEL_BODY
  DG_LAUNCHED();
  return DG_OK;
}

// ------------------------------------------------- whole-plane transforms
// Lengths of the whole-plane kernels: x and z lengths with a compile-time
// warp plan up to 128 (the z columns of a plane then fit two CTAs per SM).
#define DG_PLANE_NX(X) X(16) X(32) X(48) X(64) X(96) X(128)

bool dg_plane_ok(const dg_handle *h) {
  auto len_ok = [](int n) {
    return n == 16 || n == 32 || n == 48 || n == 64 || n == 96 || n == 128;
  };
  return h->plane_xz && !h->periodic && len_ok(h->NX) && len_ok(h->NZ) &&
         h->nkxp == h->NX / 3 + 1 && h->NKZ == h->NZ / 3 &&
         h->ss == (long)h->nkxp * (2 * h->NKZ + 1);
}

namespace {
// the whole-plane kernels run two CTAs per SM at the largest sizes only with
// the shared-memory carveout at its maximum
void plane_attrs(const void *kern) {
  static std::mutex mu;
  static std::unordered_set<const void *> done;
  std::lock_guard<std::mutex> lk(mu);
  if (done.insert(kern).second) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
  }
}

template <int NXT, int NZT>
int plane_c2r_t(dg_handle *h, const double2 *const *in, int nf, int jmin, int jmax, double *phys,
                long pplane, long prow, long pfield) {
  CFieldPtrs fp;
  for (int f = 0; f < nf; f++) fp.p[f] = in[f];
  auto kern = k_plane_c2r<NXT, NZT>;
  plane_attrs((const void *)kern);
  dg_kt_begin(h, "k_plane_c2r", h->st);
  kern<<<dim3(jmax - jmin + 1, nf), PL_THR, pl_smem(NXT, NZT), h->st>>>(
      fp, jmin, h->ss, h->twz, h->twx, phys, pplane, prow, pfield);
  DG_LAUNCHED();
  return DG_OK;
}
template <int NXT, int NZT>
int plane_r2c_t(dg_handle *h, const double *phys, int nf, int jmin, int jmax, long pplane,
                long prow, long pfield, double2 *const *out) {
  FieldPtrs fp;
  for (int f = 0; f < nf; f++) fp.p[f] = out[f];
  auto kern = k_plane_r2c<NXT, NZT>;
  plane_attrs((const void *)kern);
  dg_kt_begin(h, "k_plane_r2c", h->st);
  kern<<<dim3(jmax - jmin + 1, nf), PL_THR, pl_smem(NXT, NZT), h->st>>>(
      phys, pplane, prow, pfield, jmin, h->twx, h->twz, fp, h->ss);
  DG_LAUNCHED();
  return DG_OK;
}
template <int NXT>
int plane_c2r_z(dg_handle *h, const double2 *const *in, int nf, int jmin, int jmax, double *phys,
                long pplane, long prow, long pfield) {
#define KERNEL_BODY(NZT) return plane_c2r_t<NXT, NZT>(h, in, nf, jmin, jmax, phys, pplane, prow, pfield)
  switch (h->NZ) {
    DG_PLANE_NX(DG_CASE_N)
    default: break;
  }
#undef KERNEL_BODY
  return 1;
}
template <int NXT>
int plane_r2c_z(dg_handle *h, const double *phys, int nf, int jmin, int jmax, long pplane,
                long prow, long pfield, double2 *const *out) {
#define KERNEL_BODY(NZT) return plane_r2c_t<NXT, NZT>(h, phys, nf, jmin, jmax, pplane, prow, pfield, out)
  switch (h->NZ) {
    DG_PLANE_NX(DG_CASE_N)
    default: break;
  }
#undef KERNEL_BODY
  return 1;
}
}  // namespace

int dg_plane_c2r(dg_handle *h, const double2 *const *in, int nf, int jmin, int jmax, double *phys,
                 long pplane, long prow, long pfield) {
  if (!dg_plane_ok(h)) return 1;
  if (jmax < jmin || nf <= 0) return DG_OK;
#define KERNEL_BODY(NXT) return plane_c2r_z<NXT>(h, in, nf, jmin, jmax, phys, pplane, prow, pfield)
  switch (h->NX) {
    DG_PLANE_NX(DG_CASE_N)
    default: break;
  }
#undef KERNEL_BODY
  return 1;
}

int dg_plane_r2c(dg_handle *h, const double *phys, int nf, int jmin, int jmax, long pplane,
                 long prow, long pfield, double2 *const *out) {
  if (!dg_plane_ok(h)) return 1;
  if (jmax < jmin || nf <= 0) return DG_OK;
#define KERNEL_BODY(NXT) return plane_r2c_z<NXT>(h, phys, nf, jmin, jmax, pplane, prow, pfield, out)
  switch (h->NX) {
    DG_PLANE_NX(DG_CASE_N)
    default: break;
  }
#undef KERNEL_BODY
  return 1;
}

int dg_xc2r_cfl(dg_handle *h, const double2 *H, int jmin, int jmax, unsigned long long *out) {
  dim3 grid(dg_cdiv(h->NZ, 2 * batch_for(h->NX)), jmax - jmin + 1, 3);
  const size_t sm = xsmem(h->NX);
  const long Hf = (long)h->nplanes * h->NZ * h->nkxp;
  const double dxv = h->p.lx / h->NX, dzv = h->p.lz / h->NZ;
#define KERNEL_BODY(N)                                                                          \
  {                                                                                             \
    auto kern = xc2r_cfl_kernel<N>(h->fft_plan);                                                \
    big_smem(kern);                                                                             \
    dg_kt_begin(h, "k_xc2r_cfl", h->st);                                                        \
    DG_CUDA(dg_launch(0, kern, grid, dim3(NTHR), sm, h->st, H, Hf, jmin, h->nkxp, h->NX, h->NZ,  \
                      h->plx, h->twx, h->p.cfl, dxv, dzv, h->dy, out));                        \
  }
  switch (h->NX) {
    DG_FOR_EACH_N(DG_CASE_N)
    default: KERNEL_BODY(0); break;
  }
#undef KERNEL_BODY
  DG_LAUNCHED();
  return DG_OK;
}

bool dg_make_plan(int n, FftPlan *pl) {
  pl->n = n;
  pl->np = 0;
  int m = n;
  while (m > 1) {
    int r;
    if (m % 16 == 0) r = 16;
    else if (m % 8 == 0) r = 8;
    else if (m % 4 == 0) r = 4;
    else if (m % 2 == 0) r = 2;
    else if (m % 3 == 0) r = 3;
    else if (m % 5 == 0) r = 5;
    else return false;
    if (pl->np >= DG_MAX_PASSES) return false;
    pl->r[pl->np++] = r;
    m /= r;
  }
  return true;
}
