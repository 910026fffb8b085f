// Reference-layout entry points: FFT_XZ_TO_FOURIER / FFT_XZ_TO_PHYSICAL and the
// batched THOMAS_REAL / THOMAS_COMPLEX solvers.
#include <string.h>
#include "dg_internal.cuh"

namespace {

__global__ void k_compact_to_ref_planes(const double2 *__restrict__ cmp, double2 *__restrict__ ref,
                                        int nj, int nzt, int nkxp, int nxp1, int nz2) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long tot = (long)nj * nz2 * nxp1;
  if (q >= tot) return;
  const int i = (int)(q % nxp1);
  const int k = (int)((q / nxp1) % nz2);
  const int j = (int)(q / ((long)nxp1 * nz2));
  double2 v = make_double2(0.0, 0.0);
  if (i < nkxp && k < nzt) v = cmp[((long)j * nzt + k) * nkxp + i];
  ref[q] = v;
}

__global__ void k_ref_to_compact_planes(const double2 *__restrict__ ref, double2 *__restrict__ cmp,
                                        int nj, int nzt, int nkxp, int nxp1, int nz2) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long tot = (long)nj * nzt * nkxp;
  if (q >= tot) return;
  const int i = (int)(q % nkxp);
  const int k = (int)((q / nkxp) % nzt);
  const int j = (int)(q / ((long)nkxp * nzt));
  cmp[q] = ref[((long)j * nz2 + k) * nxp1 + i];
}

// THOMAS_REAL, for/channel.f:2653-2684 (one thread per column i)
__global__ void k_thomas_real(double *A, double *B, const double *C, double *G, int ny, int nx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int ld = nx + 1;
  if (i > nx) return;
  for (int j = 0; j < ny; j++) {
    const long c = (long)(j + 1) * ld + i, p = (long)j * ld + i;
    A[c] = -A[c] / B[p];
    B[c] = B[c] + A[c] * C[p];
    G[c] = G[c] + A[c] * G[p];
  }
  const long t = (long)ny * ld + i;
  G[t] = G[t] / B[t];
  for (int j = ny - 1; j >= 0; j--) {
    const long c = (long)j * ld + i;
    G[c] = (G[c] - C[c] * G[c + ld]) / B[c];
  }
}

// THOMAS_COMPLEX, for/channel.f:2687-2720
__global__ void k_thomas_complex(double *A, double *B, const double *C, double2 *G, int ny, int nx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int ld = nx + 1;
  if (i > nx) return;
  for (int j = 0; j < ny; j++) {
    const long c = (long)(j + 1) * ld + i, p = (long)j * ld + i;
    A[c] = -A[c] / B[p];
    B[c] = B[c] + A[c] * C[p];
    const double2 gp = G[p];
    double2 gc = G[c];
    gc.x = gc.x + A[c] * gp.x;
    gc.y = gc.y + A[c] * gp.y;
    G[c] = gc;
  }
  const long t = (long)ny * ld + i;
  G[t] = make_double2(G[t].x / B[t], G[t].y / B[t]);
  for (int j = ny - 1; j >= 0; j--) {
    const long c = (long)j * ld + i;
    const double2 g1 = G[c + ld];
    double2 g = G[c];
    g.x = (g.x - C[c] * g1.x) / B[c];
    g.y = (g.y - C[c] * g1.y) / B[c];
    G[c] = g;
  }
}

int check_planes(dg_handle *h, int jmin, int jmax) {
  if (!h || h->periodic) return DG_ERR_ARG;
  if (jmin < 0 || jmax > h->NY + 1 || jmax < jmin) {
    dg_set_error("JMIN/JMAX outside 0..NY+1");
    return DG_ERR_ARG;
  }
  return DG_OK;
}

}  // namespace

extern "C" int diablo_fft_xz_to_fourier(dg_handle *h, const double *V, double *VV, int jmin,
                                        int jmax, int where) {
  DG_TRY(check_planes(h, jmin, jmax));
  if (!V || !VV) return DG_ERR_ARG;
  const int nj = jmax - jmin + 1;
  const long pplane = (long)(h->NX + 2) * (h->NZ + 2);  // doubles per physical plane
  const int nxp1 = h->NX / 2 + 1, nz2 = h->NZ + 2;      // complex per spectral plane
  const size_t bytes = sizeof(double) * pplane * nj;
  const double *vin = V + (long)jmin * pplane;
  double *vout = VV + (long)jmin * pplane;
  double *tin = nullptr;
  if (where == DG_HOST) {
    DG_CUDA(cudaMallocAsync((void **)&tin, bytes, h->st));
    DG_CUDA(cudaMemcpyAsync(tin, vin, bytes, cudaMemcpyHostToDevice, h->st));
    vin = tin;
  }
  DG_TRY(dg_xr2c_planes(h, vin - (long)jmin * pplane, 1, jmin, jmax, pplane, h->NX + 2, 0, h->H));
  double2 *cmp = h->rhs[0];
  double2 *flds[1] = {cmp};
  DG_TRY(dg_zfwd_planes(h, h->H, 1, jmin, jmax, flds, nullptr, 0));
  double2 *dref = (double2 *)(where == DG_HOST ? tin : vout);
  k_compact_to_ref_planes<<<dg_cdiv((long)nj * nz2 * nxp1, 256), 256, 0, h->st>>>(
      cmp + (long)jmin * h->ss, dref, nj, h->nkzt, h->nkxp, nxp1, nz2);
  DG_LAUNCHED();
  if (where == DG_HOST) {
    DG_CUDA(cudaMemcpyAsync(vout, tin, bytes, cudaMemcpyDeviceToHost, h->st));
    DG_CUDA(cudaFreeAsync(tin, h->st));
  }
  DG_CUDA(cudaStreamSynchronize(h->st));
  return DG_OK;
}

extern "C" int diablo_fft_xz_to_physical(dg_handle *h, const double *VV, double *V, int jmin,
                                         int jmax, int where) {
  DG_TRY(check_planes(h, jmin, jmax));
  if (!V || !VV) return DG_ERR_ARG;
  const int nj = jmax - jmin + 1;
  const long pplane = (long)(h->NX + 2) * (h->NZ + 2);
  const int nxp1 = h->NX / 2 + 1, nz2 = h->NZ + 2;
  const size_t bytes = sizeof(double) * pplane * nj;
  const double *sin_ = VV + (long)jmin * pplane;
  double *pout = V + (long)jmin * pplane;
  double *tin = nullptr, *tout = nullptr;
  if (where == DG_HOST) {
    DG_CUDA(cudaMallocAsync((void **)&tin, bytes, h->st));
    DG_CUDA(cudaMallocAsync((void **)&tout, bytes, h->st));
    DG_CUDA(cudaMemcpyAsync(tin, sin_, bytes, cudaMemcpyHostToDevice, h->st));
    // rows the transform does not write keep the caller's values
    DG_CUDA(cudaMemcpyAsync(tout, pout, bytes, cudaMemcpyHostToDevice, h->st));
    sin_ = tin;
    pout = tout;
  }
  double2 *cmp = h->rhs[0];
  k_ref_to_compact_planes<<<dg_cdiv((long)nj * h->ss, 256), 256, 0, h->st>>>(
      (const double2 *)sin_, cmp + (long)jmin * h->ss, nj, h->nkzt, h->nkxp, nxp1, nz2);
  DG_LAUNCHED();
  const double2 *flds[1] = {cmp};
  DG_TRY(dg_zinv(h, flds, 1, jmin, jmax, h->H, 0));
  DG_TRY(dg_xc2r_planes(h, h->H, 1, jmin, jmax, pout - (long)jmin * pplane, pplane, h->NX + 2, 0));
  if (where == DG_HOST) {
    DG_CUDA(cudaMemcpyAsync(V + (long)jmin * pplane, tout, bytes, cudaMemcpyDeviceToHost, h->st));
    DG_CUDA(cudaFreeAsync(tin, h->st));
    DG_CUDA(cudaFreeAsync(tout, h->st));
  }
  DG_CUDA(cudaStreamSynchronize(h->st));
  return DG_OK;
}

static int thomas_common(double *A, double *B, double *C, double *G, int ny, int nx, int where,
                         int cplx) {
  if (!A || !B || !C || !G || ny < 0 || nx < 0) return DG_ERR_ARG;
  const size_t n = (size_t)(nx + 1) * (ny + 1);
  const size_t gb = n * sizeof(double) * (cplx ? 2 : 1);
  cudaStream_t st = 0;
  double *dA = A, *dB = B, *dC = C, *dG = G;
  if (where == DG_HOST) {
    DG_CUDA(cudaMallocAsync((void **)&dA, n * sizeof(double), st));
    DG_CUDA(cudaMallocAsync((void **)&dB, n * sizeof(double), st));
    DG_CUDA(cudaMallocAsync((void **)&dC, n * sizeof(double), st));
    DG_CUDA(cudaMallocAsync((void **)&dG, gb, st));
    DG_CUDA(cudaMemcpyAsync(dA, A, n * sizeof(double), cudaMemcpyHostToDevice, st));
    DG_CUDA(cudaMemcpyAsync(dB, B, n * sizeof(double), cudaMemcpyHostToDevice, st));
    DG_CUDA(cudaMemcpyAsync(dC, C, n * sizeof(double), cudaMemcpyHostToDevice, st));
    DG_CUDA(cudaMemcpyAsync(dG, G, gb, cudaMemcpyHostToDevice, st));
  }
  if (cplx)
    k_thomas_complex<<<dg_cdiv(nx + 1, 128), 128, 0, st>>>(dA, dB, dC, (double2 *)dG, ny, nx);
  else
    k_thomas_real<<<dg_cdiv(nx + 1, 128), 128, 0, st>>>(dA, dB, dC, dG, ny, nx);
  DG_LAUNCHED();
  if (where == DG_HOST) {
    DG_CUDA(cudaMemcpyAsync(A, dA, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    DG_CUDA(cudaMemcpyAsync(B, dB, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    DG_CUDA(cudaMemcpyAsync(G, dG, gb, cudaMemcpyDeviceToHost, st));
    DG_CUDA(cudaFreeAsync(dA, st));
    DG_CUDA(cudaFreeAsync(dB, st));
    DG_CUDA(cudaFreeAsync(dC, st));
    DG_CUDA(cudaFreeAsync(dG, st));
  }
  DG_CUDA(cudaStreamSynchronize(st));
  return DG_OK;
}

extern "C" int diablo_thomas_real(double *A, double *B, double *C, double *G, int ny, int nx,
                                  int where) {
  return thomas_common(A, B, C, G, ny, nx, where, 0);
}

extern "C" int diablo_thomas_complex(double *A, double *B, double *C, double *G, int ny, int nx,
                                     int where) {
  return thomas_common(A, B, C, G, ny, nx, where, 1);
}
