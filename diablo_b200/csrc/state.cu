// Handle lifecycle, device-resident state, tables and field I/O.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <mutex>
#include <string>

#include <stddef.h>

#include "dg_internal.cuh"

namespace {
thread_local std::string g_err;
std::atomic<long long> g_launches{0};

// exp(-2 pi i m / n) for m = 0..n-1, evaluated in long double
void twiddles(int n, double2 *out) {
  const long double tp = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < n; m++) {
    long double a = tp * (long double)m / (long double)n;
    out[m] = make_double2((double)cosl(a), -(double)sinl(a));
  }
}

template <typename T>
int dalloc(dg_handle *h, T **p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = dg_malloc(h, (void **)p, count * sizeof(T));
  if (e != cudaSuccess) {
    dg_set_error((std::string("device allocation: ") + cudaGetErrorString(e)).c_str());
    return e == cudaErrorMemoryAllocation ? DG_ERR_OOM : DG_ERR_CUDA;
  }
  return DG_OK;
}

__global__ void k_compact_to_ref(const double2 *__restrict__ cmp, double2 *__restrict__ ref,
                                 int nplanes, int nzt, int nkxp, int nxp1, int nz2) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long tot = (long)nplanes * nz2 * nxp1;
  if (q >= tot) return;
  const int i = (int)(q % nxp1);
  const int k = (int)((q / nxp1) % nz2);
  const int j = (int)(q / ((long)nxp1 * nz2));
  double2 v = make_double2(0.0, 0.0);
  if (i < nkxp && k < nzt) v = cmp[((long)j * nzt + k) * nkxp + i];
  ref[q] = v;
}

__global__ void k_advance_time(double *dscal) { dscal[0] = dscal[0] + dscal[1]; }
}  // namespace

// Device memory of a handle comes from the device's default stream-ordered
// pool (cudaMallocAsync / cudaFreeAsync on the handle's stream).  Freeing a
// handle then does not synchronise the device, so a process that creates and
// destroys handles while others run (the ensemble server) does not stall
// them; the pool keeps freed blocks for reuse (release threshold raised once
// per device, for this process's pool only).
cudaError_t dg_malloc(dg_handle *h, void **p, size_t bytes) {
  static std::mutex mu;
  static bool raised[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev >= 0 && dev < 64 && !raised[dev]) {
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
      }
      raised[dev] = true;
    }
  }
  // ordered on the handle's stream: every first use of a block is queued on
  // that stream too (set-up copies included), or comes after a join with it
  return cudaMallocAsync(p, bytes, h->st);
}

void dg_free(dg_handle *h, void *p) {
  if (p) cudaFreeAsync(p, h->st);
}

void dg_set_error(const char *msg) { g_err = msg ? msg : ""; }
void dg_count_launch(int n) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
  dg_kt_end();
}

extern "C" int dg_version(void) { return 100; }

// The layout of the ABI structs as this build compiled them, for binding
// checks: sizeof(dg_params), sizeof(dg_stats), then the byte offsets of
// dg_params' fields nx, nu, f_type, ubulk0, th_bc_ymin, epsilon_target, les,
// les_model_type, create_new_flow.  Returns the number of values written
// (at most n).
extern "C" int dg_abi_layout(int64_t *out, int n) {
  const int64_t v[] = {(int64_t)sizeof(dg_params), (int64_t)sizeof(dg_stats),
                       (int64_t)offsetof(dg_params, nx), (int64_t)offsetof(dg_params, nu),
                       (int64_t)offsetof(dg_params, f_type), (int64_t)offsetof(dg_params, ubulk0),
                       (int64_t)offsetof(dg_params, th_bc_ymin),
                       (int64_t)offsetof(dg_params, epsilon_target),
                       (int64_t)offsetof(dg_params, les), (int64_t)offsetof(dg_params, les_model_type),
                       (int64_t)offsetof(dg_params, create_new_flow)};
  const int k = (int)(sizeof(v) / sizeof(v[0]));
  if (!out) return k;
  for (int i = 0; i < k && i < n; i++) out[i] = v[i];
  return k < n ? k : n;
}
extern "C" const char *dg_last_error(void) { return g_err.c_str(); }
extern "C" int64_t dg_kernel_launches(void) { return (int64_t)g_launches.load(); }

static int validate(const dg_params *p, const double *gy) {
  if (!p) return DG_ERR_ARG;
  if (p->num_per_dir != 2 && p->num_per_dir != 3) {
    dg_set_error("num_per_dir must be 2 (channel) or 3 (periodic)");
    return DG_ERR_ARG;
  }
  if (p->n_th < 0 || p->n_th > DG_MAX_TH) {
    dg_set_error("n_th out of range");
    return DG_ERR_ARG;
  }
  if (p->nx < 8 || p->nz < 8 || (p->nx & 1) || (p->nz & 1) || p->nx > 4096 || p->nz > 4096) {
    dg_set_error("NX and NZ must be even, 8..4096");
    return DG_ERR_DIMS;
  }
  FftPlan t;
  if (!dg_make_plan(p->nx, &t) || !dg_make_plan(p->nz, &t)) {
    dg_set_error("NX and NZ must factor into 2, 3 and 5");
    return DG_ERR_DIMS;
  }
  if (p->num_per_dir == 2) {
    if (p->ny < 4 || !gy) {
      dg_set_error("channel needs NY >= 4 and a GY grid");
      return DG_ERR_DIMS;
    }
    int bcs[6] = {p->u_bc_ymin, p->w_bc_ymin, p->u_bc_ymax, p->w_bc_ymax, p->v_bc_ymin, p->v_bc_ymax};
    for (int i = 0; i < 4; i++)
      if (bcs[i] != 0 && bcs[i] != 1) {
        dg_set_error("Error: U/W_BC_Y* must be 0, or 1");
        return DG_ERR_ARG;
      }
    for (int i = 4; i < 6; i++)
      if (bcs[i] < 0 || bcs[i] > 2) {
        dg_set_error("Error: V_BC_Y* must be 0, 1, or 2");
        return DG_ERR_ARG;
      }
    if (p->les) {
      // for/les.f:269-272 and APPLY_BC_VEL_PHYS (for/channel.f:2537,2633)
      if (p->les_model_type != 1) {
        dg_set_error("ERROR: LES_MODEL_TYPE=2, 3 not supported yet in MPI");
        return DG_ERR_ARG;
      }
      if (p->v_bc_ymin > 1 || p->v_bc_ymax > 1) {
        dg_set_error("Error: V_BC_YMIN/V_BC_YMAX must be 0, 1 with LES");
        return DG_ERR_ARG;
      }
      if (p->v_bc_ymax == 1) {
        dg_set_error("LES with a Neumann V at the upper wall is not supported: APPLY_BC_VEL "
                     "rewrites CU2(NY) after CR2(NY) was formed, which the fused stage cannot "
                     "reproduce");
        return DG_ERR_ARG;
      }
    }
    if (p->precision != 0 && p->precision != 1) {
      dg_set_error("precision must be 0 (FP64) or 1 (mixed)");
      return DG_ERR_ARG;
    }
    if (p->precision == 1 && !dg_mixed_ok(p->nx, p->nz, p->n_th)) {
      dg_set_error("mixed precision needs NX and NZ in {16, 32, 48, 64, 96, 128, 256} and "
                   "N_TH <= 2");
      return DG_ERR_DIMS;
    }
  } else {
    if (p->precision != 0 && p->precision != 1) {
      dg_set_error("precision must be 0 (FP64) or 1 (mixed)");
      return DG_ERR_ARG;
    }
    if (p->precision == 1 && !dg_per_mixed_ok(p->nx, p->n_th)) {
      dg_set_error("periodic mixed precision needs NX in {16, 32, 48, 64, 96, 128, 256} and "
                   "N_TH <= 2");
      return DG_ERR_DIMS;
    }
    if (!dg_make_plan(p->ny, &t) || p->ny < 8) {
      dg_set_error("periodic NY must be >= 8 and factor into 2, 3 and 5");
      return DG_ERR_DIMS;
    }
  }
  return DG_OK;
}

// Device bytes diablo_gpu_init allocates for these parameters (the sum of
// the allocations below and in dg_per_init), for admission against a budget.
extern "C" int64_t dg_state_bytes(const dg_params *p) {
  if (!p || p->nx <= 0 || p->ny <= 0 || p->nz <= 0) return -1;
  const int64_t nkxp = p->nx / 3 + 1, nkzt = 2 * (p->nz / 3) + 1, nkyt = 2 * (p->ny / 3) + 1;
  const int64_t nf = 3 + p->n_th, L = p->ny + 2;
  const bool per = p->num_per_dir == 3;
  const int64_t planes = per ? nkyt : L;
  const int64_t ns = nkxp * nkzt * planes;
  int64_t b = 16 * ns * (3 * nf + 2);                      // cu, cf, rhs, cp, cr1
  b += 8 * (3 * L + nkxp + nkzt + nkyt) + 16 * (p->nx + p->nz + p->ny) + 8 * 16 + 256;
  if (!per) {
    const int64_t hsz = planes * p->nz * nkxp;
    b += 16 * ns + 8 * 2 * ns;                              // gphi, rem_a, rem_rb
    const int64_t LP = (L + 1) / 2 * 2;                     // 16-byte table rows
    b += 8 * 3 * (3 + DG_MAX_TH) * 5 * LP + 8 * nf * 8 * L; // cn_tab, cn_rows
    b += 8 * 8 * LP;                                         // rowc
    b += 16 * hsz * nf + 16 * hsz * 2 * nf;                 // H, G
    int64_t w = 8 * L * p->nz * p->nx * (nf > 3 ? nf : 3);
    if (w < 8 * 8 * L) w = 8 * 8 * L;
    b += w;
  } else {
    const int64_t np = 6 + 3 * p->n_th, nmax = np > nf ? np : nf;
    const int64_t hy = (int64_t)p->ny * nkxp * nkzt, hf = (int64_t)p->ny * p->nz * nkxp;
    b += 16 * (nmax * hy + nf * hf + nmax * hf + np * nkyt * nkxp * nkzt);
    b += 8 * (int64_t)p->ny * p->nz * p->nx * (nf + np > 6 ? nf + np : 6);
  }
  return b;
}

extern "C" int diablo_gpu_init(const dg_params *p, const double *gy, void *stream,
                               dg_handle **out) {
  if (!out) return DG_ERR_ARG;
  *out = nullptr;
  DG_TRY(validate(p, gy));
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    dg_set_error("no CUDA device");
    return DG_ERR_NODEV;
  }
  int dev = 0, major = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10) {
    dg_set_error("this build targets sm_100a (B200)");
    return DG_ERR_NODEV;
  }
  dg_handle *h = (dg_handle *)calloc(1, sizeof(dg_handle));
  h->p = *p;
  h->NX = p->nx; h->NY = p->ny; h->NZ = p->nz; h->NTH = p->n_th;
  h->NKX = p->nx / 3; h->NKZ = p->nz / 3; h->TNKZ = 2 * h->NKZ;
  h->NKY = p->ny / 3; h->TNKY = 2 * h->NKY;
  h->nkxp = h->NKX + 1; h->nkzt = h->TNKZ + 1; h->nkyt = h->TNKY + 1;
  h->periodic = (p->num_per_dir == 3);
  h->nplanes = h->periodic ? h->nkyt : h->NY + 2;
  h->ss = (long)h->nkxp * h->nkzt;
  h->nspec = h->ss * h->nplanes;
  h->nf = 3 + h->NTH;
  h->col_mt = dg_default_col_mt(h);
  h->cn_mt = 4;
  h->zf_nlo = 1;
  h->pdl = 1;
  h->plane_xz = 1;
  h->pi = 4.0 * atan(1.0);
  h->eps = (double)(float)0.000000001;  // default-real literal, for/fft.f:74
  // INIT_CHAN_MPI with NPROCY = 1 (for/mpi.f:1080-1100)
  h->jstart = 2;
  h->jend = h->NY;
  for (int n = 0; n < DG_MAX_TH; n++) {
    h->jend_th[n] = h->NY;
    h->jstart_th[n] = (n < h->NTH && p->th_bc_ymin[n] == 1) ? 1 : 2;
  }
  if (stream) {
    h->st = (cudaStream_t)stream;
    h->own_stream = false;
  } else {
    if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
      free(h);
      dg_set_error("stream creation failed");
      return DG_ERR_CUDA;
    }
    h->own_stream = true;
  }
  if (cudaStreamCreateWithFlags(&h->st2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_cfl0, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_cfl1, cudaEventDisableTiming) != cudaSuccess) {
    dg_set_error("side stream creation failed");
    if (h->own_stream) cudaStreamDestroy(h->st);
    free(h);
    return DG_ERR_CUDA;
  }
  *out = h;
  const int NY = h->NY, L = NY + 2;

  // ---- host tables
  h->h_gy = (double *)calloc(L, sizeof(double));
  h->h_gyf = (double *)calloc(L, sizeof(double));
  h->h_dy = (double *)calloc(L, sizeof(double));
  h->h_dyf = (double *)calloc(L, sizeof(double));
  h->h_kx = (double *)calloc(h->nkxp, sizeof(double));
  h->h_kz = (double *)calloc(h->nkzt, sizeof(double));
  h->h_ky = (double *)calloc(h->nkyt, sizeof(double));
  const double pi = h->pi;
  for (int i = 0; i <= h->NKX; i++) h->h_kx[i] = (double)i * (2.0 * pi) / p->lx;
  for (int k = 0; k <= h->NKZ; k++) h->h_kz[k] = (double)k * (2.0 * pi) / p->lz;
  for (int k = 1; k <= h->NKZ; k++) h->h_kz[h->TNKZ + 1 - k] = -((double)k * (2.0 * pi) / p->lz);
  if (h->periodic) {
    for (int j = 1; j <= h->NKY; j++) h->h_ky[j] = (double)j * (2.0 * pi) / p->ly;
    for (int j = 1; j <= h->NKY; j++) h->h_ky[h->TNKY + 1 - j] = -((double)j * (2.0 * pi) / p->ly);
    for (int j = 0; j <= NY && j < L; j++) h->h_dy[j] = p->ly / NY;
  } else {
    // ReadGridHDF5 (for/hdf5.f:676-703) and metrics (for/channel.f:1646-1652)
    for (int j = 1; j <= NY + 1; j++) h->h_gy[j] = gy[j - 1];
    for (int j = 1; j <= NY; j++) h->h_gyf[j] = 0.5 * (h->h_gy[j] + h->h_gy[j + 1]);
    h->h_gyf[0] = 2.0 * h->h_gyf[1] - h->h_gyf[2];
    h->h_gyf[NY + 1] = 2.0 * h->h_gyf[NY] - h->h_gyf[NY - 1];
    for (int j = 1; j <= NY + 1; j++) h->h_dy[j] = h->h_gyf[j] - h->h_gyf[j - 1];
    for (int j = 1; j <= NY; j++) h->h_dyf[j] = h->h_gy[j + 1] - h->h_gy[j];
    h->h_dyf[NY + 1] = h->h_dyf[NY];
  }

  // ---- device allocations
  DG_TRY(dalloc(h, &h->gyf, L));
  DG_TRY(dalloc(h, &h->dy, L));
  DG_TRY(dalloc(h, &h->dyf, L));
  DG_TRY(dalloc(h, &h->kx, h->nkxp));
  DG_TRY(dalloc(h, &h->kz, h->nkzt));
  DG_TRY(dalloc(h, &h->ky, h->nkyt));
  DG_CUDA(cudaMemcpyAsync(h->gyf, h->h_gyf, sizeof(double) * L, cudaMemcpyHostToDevice, h->st));
  DG_CUDA(cudaMemcpyAsync(h->dy, h->h_dy, sizeof(double) * L, cudaMemcpyHostToDevice, h->st));
  DG_CUDA(cudaMemcpyAsync(h->dyf, h->h_dyf, sizeof(double) * L, cudaMemcpyHostToDevice, h->st));
  DG_CUDA(cudaMemcpyAsync(h->kx, h->h_kx, sizeof(double) * h->nkxp, cudaMemcpyHostToDevice, h->st));
  DG_CUDA(cudaMemcpyAsync(h->kz, h->h_kz, sizeof(double) * h->nkzt, cudaMemcpyHostToDevice, h->st));
  DG_CUDA(cudaMemcpyAsync(h->ky, h->h_ky, sizeof(double) * h->nkyt, cudaMemcpyHostToDevice, h->st));

  dg_make_plan(h->NX, &h->plx);
  dg_make_plan(h->NZ, &h->plz);
  if (h->periodic) dg_make_plan(h->NY, &h->ply);
  {
    int nmax = h->NX > h->NZ ? h->NX : h->NZ;
    if (h->NY > nmax) nmax = h->NY;
    double2 *tmp = (double2 *)malloc(sizeof(double2) * nmax);
    DG_TRY(dalloc(h, &h->twx, h->NX));
    twiddles(h->NX, tmp);
    DG_CUDA(cudaMemcpyAsync(h->twx, tmp, sizeof(double2) * h->NX, cudaMemcpyHostToDevice, h->st));
    DG_TRY(dalloc(h, &h->twz, h->NZ));
    twiddles(h->NZ, tmp);
    DG_CUDA(cudaMemcpyAsync(h->twz, tmp, sizeof(double2) * h->NZ, cudaMemcpyHostToDevice, h->st));
    if (p->precision == 1) {
      h->mixed = 1;
      float2 *tf = (float2 *)malloc(sizeof(float2) * nmax);
      twiddles(h->NX, tmp);
      for (int m = 0; m < h->NX; m++) tf[m] = make_float2((float)tmp[m].x, (float)tmp[m].y);
      DG_CUDA(dg_malloc(h, (void **)&h->twx_f, sizeof(float2) * h->NX));
      DG_CUDA(cudaMemcpyAsync(h->twx_f, tf, sizeof(float2) * h->NX, cudaMemcpyHostToDevice, h->st));
      twiddles(h->NZ, tmp);
      for (int m = 0; m < h->NZ; m++) tf[m] = make_float2((float)tmp[m].x, (float)tmp[m].y);
      DG_CUDA(dg_malloc(h, (void **)&h->twz_f, sizeof(float2) * h->NZ));
      DG_CUDA(cudaMemcpyAsync(h->twz_f, tf, sizeof(float2) * h->NZ, cudaMemcpyHostToDevice, h->st));
      free(tf);
    }
    if (h->periodic && p->precision == 1) {
      float2 *tf = (float2 *)malloc(sizeof(float2) * nmax);
      twiddles(h->NY, tmp);
      for (int m = 0; m < h->NY; m++) tf[m] = make_float2((float)tmp[m].x, (float)tmp[m].y);
      DG_CUDA(dg_malloc(h, (void **)&h->twy_f, sizeof(float2) * h->NY));
      DG_CUDA(cudaMemcpyAsync(h->twy_f, tf, sizeof(float2) * h->NY, cudaMemcpyHostToDevice, h->st));
      free(tf);
    }
    if (h->periodic) {
      DG_TRY(dalloc(h, &h->twy, h->NY));
      twiddles(h->NY, tmp);
      DG_CUDA(cudaMemcpyAsync(h->twy, tmp, sizeof(double2) * h->NY, cudaMemcpyHostToDevice, h->st));
    }
    free(tmp);
  }

  DG_TRY(dalloc(h, &h->dscal, 16));
  DG_TRY(dalloc(h, &h->dmin_bits, 32));
  DG_TRY(dalloc(h, &h->dflag, 4));
  DG_CUDA(cudaMemsetAsync(h->dflag, 0, 4 * sizeof(int), h->st));
  const size_t ns = (size_t)h->nspec;
  for (int f = 0; f < h->nf; f++) {
    DG_TRY(dalloc(h, &h->cu[f], ns));
    DG_TRY(dalloc(h, &h->cf[f], ns));
    DG_TRY(dalloc(h, &h->rhs[f], ns));
    // on the handle's stream: a legacy-stream memset is not ordered with the
    // handle's non-blocking stream, and could land after the first state upload
    DG_CUDA(cudaMemsetAsync(h->cu[f], 0, ns * sizeof(double2), h->st));
    DG_CUDA(cudaMemsetAsync(h->cf[f], 0, ns * sizeof(double2), h->st));
    DG_CUDA(cudaMemsetAsync(h->rhs[f], 0, ns * sizeof(double2), h->st));
  }
  DG_TRY(dalloc(h, &h->cp, ns));
  DG_TRY(dalloc(h, &h->cr1, ns));
  DG_CUDA(cudaMemsetAsync(h->cp, 0, ns * sizeof(double2), h->st));
  DG_CUDA(cudaMemsetAsync(h->cr1, 0, ns * sizeof(double2), h->st));

  if (!h->periodic) {
    DG_TRY(dalloc(h, &h->gphi, ns));
    DG_TRY(dalloc(h, &h->rem_a, ns));
    DG_TRY(dalloc(h, &h->rem_rb, ns));
    DG_TRY(dalloc(h, &h->cn_tab, (size_t)3 * (3 + DG_MAX_TH) * 5 * ((L + 1) / 2 * 2)));
    const size_t hsz = (size_t)h->nplanes * h->NZ * h->nkxp;
    DG_TRY(dalloc(h, &h->H, hsz * h->nf));
    DG_TRY(dalloc(h, &h->G, hsz * 2 * h->nf));
    const size_t phys = (size_t)(NY + 2) * h->NZ * h->NX;
    h->work_bytes = sizeof(double) * phys * (h->nf > 3 ? h->nf : 3);
    if (h->work_bytes < sizeof(double) * 8 * L) h->work_bytes = sizeof(double) * 8 * L;
    DG_TRY(dalloc(h, (double **)&h->work, h->work_bytes / sizeof(double)));
  } else {
    DG_TRY(dg_per_init(h));
  }
  DG_TRY(diablo_set_time(h, 0.0, p->delta_t));
  if (!h->periodic) DG_TRY(dg_chan_init(h));
  if (!h->periodic && p->les) DG_TRY(dg_les_init(h));
  DG_CUDA(cudaStreamSynchronize(h->st));
  return DG_OK;
}

extern "C" int diablo_gpu_finalize(dg_handle *h) {
  if (!h) return DG_OK;
  cudaStreamSynchronize(h->st);
  cudaStreamSynchronize(h->st2);
  void *dp[] = {h->gyf, h->dy, h->dyf, h->kx, h->kz, h->ky, h->kx2, h->kz2, h->ky2, h->twx, h->twz,
                h->twy, h->twx_f, h->twz_f, h->twy_f, h->dscal, h->cp, h->cr1, h->gphi, h->rem_a, h->rem_rb, h->cn_tab, h->cn_rows, h->rowc, h->col_dcase, h->col_dwork, h->H, h->G, h->work, h->dmin_bits, h->dflag, h->Hy, h->P,
                h->Q};
  for (void *q : dp) dg_free(h, q);
  dg_free(h, h->les_phys);
  dg_free(h, h->les_spec);
  dg_free(h, h->les_dfac);
  dg_free(h, h->les_ubar);
  dg_free(h, h->les_H);
  dg_free(h, h->les_means);
  dg_free(h, h->les_rowtab);
  for (int f = 0; f < 3 + DG_MAX_TH; f++) {
    dg_free(h, h->cu[f]);
    dg_free(h, h->cf[f]);
    dg_free(h, h->rhs[f]);
  }
  cudaStreamSynchronize(h->st2);
  dg_kt_free(h);
  dg_graphs_free(h);
  free(h->h_ubar);
  cudaEventDestroy(h->ev_fork);
  cudaEventDestroy(h->ev_join);
  cudaEventDestroy(h->ev_cfl0);
  cudaEventDestroy(h->ev_cfl1);
  cudaStreamDestroy(h->st2);
  if (h->own_stream) cudaStreamDestroy(h->st);
  free(h->h_gy); free(h->h_gyf); free(h->h_dy); free(h->h_dyf);
  free(h->h_kx); free(h->h_kz); free(h->h_ky);
  free(h);
  return DG_OK;
}

// dflag[1] is set by a kernel whose bulk tensor copies did not land within
// its bounded wait (the kernel then skipped its work).  Reported once: the
// flag is cleared, so the next call reports only a new failure.
static int check_async_flag(dg_handle *h) {
  int f = 0;
  DG_CUDA(cudaMemcpyAsync(&f, h->dflag + 1, sizeof(int), cudaMemcpyDeviceToHost, h->st));
  DG_CUDA(cudaStreamSynchronize(h->st));
  if (f) {
    DG_CUDA(cudaMemsetAsync(h->dflag + 1, 0, sizeof(int), h->st));
    DG_CUDA(cudaStreamSynchronize(h->st));
    dg_set_error("a bulk tensor copy did not complete within its wait limit; the substep's "
                 "results are invalid");
    return DG_ERR_TIMEOUT;
  }
  return DG_OK;
}

extern "C" int diablo_synchronize(dg_handle *h) {
  if (!h) return DG_ERR_ARG;
  DG_CUDA(cudaStreamSynchronize(h->st2));
  DG_CUDA(cudaStreamSynchronize(h->st));
  return check_async_flag(h);
}

extern "C" int diablo_set_time(dg_handle *h, double time, double delta_t) {
  if (!h) return DG_ERR_ARG;
  double s[5] = {time, delta_t, delta_t * (8.0 / 15.0), delta_t * (2.0 / 15.0),
                 delta_t * (5.0 / 15.0)};
  if (h->tables_pending) {
    DG_CUDA(cudaStreamWaitEvent(h->st, h->ev_join, 0));
    h->tables_pending = false;
  }
  DG_CUDA(cudaMemcpyAsync(h->dscal, s, sizeof(s), cudaMemcpyHostToDevice, h->st));
  if (h->cn_tab) DG_TRY(dg_cn_tables(h));
  DG_CUDA(cudaStreamSynchronize(h->st));
  return DG_OK;
}

extern "C" int diablo_get_time(dg_handle *h, double *time, double *delta_t) {
  if (!h) return DG_ERR_ARG;
  double s[2];
  DG_CUDA(cudaMemcpyAsync(s, h->dscal, sizeof(s), cudaMemcpyDeviceToHost, h->st));
  DG_CUDA(cudaStreamSynchronize(h->st));
  if (time) *time = s[0];
  if (delta_t) *delta_t = s[1];
  return DG_OK;
}

extern "C" int diablo_advance_time(dg_handle *h) {
  if (!h) return DG_ERR_ARG;
  k_advance_time<<<1, 1, 0, h->st>>>(h->dscal);
  DG_LAUNCHED();
  return DG_OK;
}

static double2 *field_ptr(dg_handle *h, int id) {
  if (id >= DG_CFTH && id < DG_CFTH + h->NTH) return h->cf[3 + id - DG_CFTH];
  if (id >= DG_CTH && id < DG_CTH + h->NTH) return h->cu[3 + id - DG_CTH];
  switch (id) {
    case DG_CU1: return h->cu[0];
    case DG_CU2: return h->cu[1];
    case DG_CU3: return h->cu[2];
    case DG_CP: return h->cp;
    case DG_CF1: return h->cf[0];
    case DG_CF2: return h->cf[1];
    case DG_CF3: return h->cf[2];
    case DG_CR1: return h->cr1;
    default: return nullptr;
  }
}

// reference layout sizes: (NX/2+1) x (NZ+2) x planes complex
static void ref_dims(const dg_handle *h, int *nxp1, int *nz2) {
  *nxp1 = h->NX / 2 + 1;
  *nz2 = h->NZ + 2;
}

extern "C" int diablo_set_field(dg_handle *h, int field, const double *src, int layout, int where) {
  if (!h || !src) return DG_ERR_ARG;
  double2 *dst = field_ptr(h, field);
  if (!dst) return DG_ERR_ARG;
  const size_t nc = (size_t)h->nspec;
  if (layout != DG_LAYOUT_COMPACT && layout != DG_LAYOUT_REFERENCE &&
      layout != DG_LAYOUT_REFERENCE_RETAINED)
    return DG_ERR_ARG;
  if (layout == DG_LAYOUT_COMPACT) {
    DG_CUDA(cudaMemcpyAsync(dst, src, nc * sizeof(double2),
                            where == DG_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                            h->st));
  } else {
    // the retained block of the reference array -- kx 0..NKX of kz slots
    // 0..TNKZ of every plane -- is the compact array with a wider row and
    // plane pitch: one strided copy, and the padding never crosses the bus
    int nxp1, nz2;
    ref_dims(h, &nxp1, &nz2);
    cudaMemcpy3DParms prm = {};
    prm.srcPtr = make_cudaPitchedPtr((void *)src, sizeof(double2) * nxp1, nxp1, nz2);
    prm.dstPtr = make_cudaPitchedPtr(dst, sizeof(double2) * h->nkxp, h->nkxp, h->nkzt);
    prm.extent = make_cudaExtent(sizeof(double2) * h->nkxp, h->nkzt, h->nplanes);
    prm.kind = where == DG_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    DG_CUDA(cudaMemcpy3DAsync(&prm, h->st));
  }
  DG_CUDA(cudaStreamSynchronize(h->st));
  return DG_OK;
}

extern "C" int diablo_get_field(dg_handle *h, int field, double *dst, int layout, int where) {
  if (!h || !dst) return DG_ERR_ARG;
  double2 *src = field_ptr(h, field);
  if (!src) return DG_ERR_ARG;
  const size_t nc = (size_t)h->nspec;
  if (layout == DG_LAYOUT_COMPACT) {
    DG_CUDA(cudaMemcpyAsync(dst, src, nc * sizeof(double2),
                            where == DG_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                            h->st));
  } else if (layout == DG_LAYOUT_REFERENCE_RETAINED) {
    // the compact array into the retained block of the reference array: one
    // strided copy, the caller's other entries untouched
    int nxp1, nz2;
    ref_dims(h, &nxp1, &nz2);
    cudaMemcpy3DParms prm = {};
    prm.srcPtr = make_cudaPitchedPtr(src, sizeof(double2) * h->nkxp, h->nkxp, h->nkzt);
    prm.dstPtr = make_cudaPitchedPtr(dst, sizeof(double2) * nxp1, nxp1, nz2);
    prm.extent = make_cudaExtent(sizeof(double2) * h->nkxp, h->nkzt, h->nplanes);
    prm.kind = where == DG_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    DG_CUDA(cudaMemcpy3DAsync(&prm, h->st));
  } else if (layout == DG_LAYOUT_REFERENCE) {
    int nxp1, nz2;
    ref_dims(h, &nxp1, &nz2);
    const size_t nr = (size_t)h->nplanes * nz2 * nxp1;
    double2 *dref = (double2 *)dst;
    double2 *tmp = nullptr;
    if (where == DG_HOST) {
      DG_CUDA(cudaMallocAsync((void **)&tmp, nr * sizeof(double2), h->st));
      dref = tmp;
    }
    k_compact_to_ref<<<dg_cdiv(nr, 256), 256, 0, h->st>>>(src, dref, h->nplanes, h->nkzt, h->nkxp,
                                                         nxp1, nz2);
    DG_LAUNCHED();
    if (tmp) {
      DG_CUDA(cudaMemcpyAsync(dst, tmp, nr * sizeof(double2), cudaMemcpyDeviceToHost, h->st));
      DG_CUDA(cudaFreeAsync(tmp, h->st));
    }
  } else {
    return DG_ERR_ARG;
  }
  DG_CUDA(cudaStreamSynchronize(h->st));
  return DG_OK;
}

// One strided or contiguous copy between a field and a caller's array on
// stream st, no synchronisation (the layouts that need no staging kernel).
static int copy_field_async(dg_handle *h, double2 *dev, double *arr, int layout, int where,
                            bool to_device, cudaStream_t st) {
  const size_t nc = (size_t)h->nspec;
  if (layout == DG_LAYOUT_COMPACT) {
    const cudaMemcpyKind k = where == DG_HOST
                                 ? (to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost)
                                 : cudaMemcpyDeviceToDevice;
    DG_CUDA(to_device ? cudaMemcpyAsync(dev, arr, nc * sizeof(double2), k, st)
                      : cudaMemcpyAsync(arr, dev, nc * sizeof(double2), k, st));
    return DG_OK;
  }
  int nxp1, nz2;
  ref_dims(h, &nxp1, &nz2);
  cudaMemcpy3DParms prm = {};
  cudaPitchedPtr a = make_cudaPitchedPtr(arr, sizeof(double2) * nxp1, nxp1, nz2);
  cudaPitchedPtr d = make_cudaPitchedPtr(dev, sizeof(double2) * h->nkxp, h->nkxp, h->nkzt);
  prm.srcPtr = to_device ? a : d;
  prm.dstPtr = to_device ? d : a;
  prm.extent = make_cudaExtent(sizeof(double2) * h->nkxp, h->nkzt, h->nplanes);
  prm.kind = where == DG_HOST ? (to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost)
                              : cudaMemcpyDeviceToDevice;
  DG_CUDA(cudaMemcpy3DAsync(&prm, st));
  return DG_OK;
}

// Several fields in one call: the copies alternate between the handle's two
// streams (two copy engines work at once) and the call synchronises once.
static int copy_fields(dg_handle *h, int n, const int *fields, double *const *arrs, int layout,
                       int where, bool to_device) {
  if (!h || n < 0 || (n > 0 && (!fields || !arrs))) return DG_ERR_ARG;
  if (layout != DG_LAYOUT_COMPACT && layout != DG_LAYOUT_REFERENCE_RETAINED &&
      !(to_device && layout == DG_LAYOUT_REFERENCE))
    return DG_ERR_ARG;
  for (int i = 0; i < n; i++)
    if (!arrs[i] || !field_ptr(h, fields[i])) return DG_ERR_ARG;
  // the side stream starts after the work queued so far on the main stream
  DG_CUDA(cudaEventRecord(h->ev_fork, h->st));
  DG_CUDA(cudaStreamWaitEvent(h->st2, h->ev_fork, 0));
  int status = DG_OK;
  for (int i = 0; i < n && status == DG_OK; i++)
    status = copy_field_async(h, field_ptr(h, fields[i]), arrs[i], layout, where, to_device,
                              (i & 1) ? h->st2 : h->st);
  // join and synchronise whatever was queued, also after a failed copy
  DG_CUDA(cudaEventRecord(h->ev_join, h->st2));
  DG_CUDA(cudaStreamWaitEvent(h->st, h->ev_join, 0));
  h->tables_pending = false;  // anything pending on the side stream is joined now
  DG_CUDA(cudaStreamSynchronize(h->st));
  return status;
}

extern "C" int diablo_set_fields(dg_handle *h, int n, const int *fields, const double *const *src,
                                 int layout, int where) {
  return copy_fields(h, n, fields, const_cast<double *const *>(src), layout, where, true);
}

extern "C" int diablo_get_fields(dg_handle *h, int n, const int *fields, double *const *dst,
                                 int layout, int where) {
  return copy_fields(h, n, fields, dst, layout, where, false);
}

extern "C" int diablo_stats(dg_handle *h, dg_stats *s) {
  if (!h || !s) return DG_ERR_ARG;
  DG_TRY(check_async_flag(h));
  return dg_stats_dev(h, s);
}
