// FFT_XZ_TO_FOURIER without any device allocation.
//
// Some host codes cannot let a library allocate device memory: a solver that
// reserves nearly all of HBM for its own fields at start-up (large ensembles
// sized to fill the GPU) has nothing left for a library's cudaMalloc; a
// process whose device memory belongs to another runtime's caching
// allocator cannot have a second allocator carve pieces out of the same
// pool; and cudaFree (and often cudaMalloc) synchronises the whole device,
// which stalls a caller that keeps several streams busy.  Such callers pass
// their own input and output arrays to diablo_fft_xz_to_fourier_noalloc and
// need no dg_handle (whose set-up allocates the solver state).
//
// The only working storage is g_noalloc_scratch below, a fixed array in the
// library's device image: every GPU that loads the library holds its
// DG_NOALLOC_SCRATCH_BYTES until the process exits.  It is laid out as the
// x and z twiddle tables followed by a chunk of planes (the half-spectral
// planes after the x transform, then their retained modes after the z
// transform); the planes jmin..jmax are processed in chunks that fit.
// Every byte a call reads from the scratch was written earlier in the same
// call, so nothing needs clearing between calls.  All calls on all streams
// of one device share the array: calls that overlap on the GPU race.
#include <string.h>

#include <map>
#include <mutex>
#include <utility>

#include "dg_internal.cuh"

static __device__ __align__(256) unsigned char g_noalloc_scratch[DG_NOALLOC_SCRATCH_BYTES];

namespace {

// The scratch array's device address per CUDA context.  A module is loaded
// per context, so the address belongs to the context current at the call
// (the device's primary context for runtime-API callers; another context
// made current, or the primary context after cudaDeviceReset, gets its own
// entry).  The first call in a context looks it up with cudaGetSymbolAddress
// -- in host code the array's name is only a host-side stand-in -- and later
// calls reuse it while it is still mapped.  That first call may load the
// module, so it belongs before any stream capture.
typedef int (*CtxGetCurrent)(void **);

CtxGetCurrent ctx_getter() {
  static CtxGetCurrent fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrent>(p);
  });
  return fn;
}

std::mutex g_mu;
std::map<std::pair<int, void *>, void *> g_addr;  // (device, context) -> address

int scratch_address(void **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    dg_set_error((std::string("no current CUDA device: ") + cudaGetErrorString(e)).c_str());
    return DG_ERR_NODEV;
  }
  CtxGetCurrent get = ctx_getter();
  if (!get) {
    dg_set_error("cuCtxGetCurrent is not available from the driver");
    return DG_ERR_CUDA;
  }
  auto lookup = [&](void **p) -> int {
    e = cudaGetSymbolAddress(p, g_noalloc_scratch);
    if (e != cudaSuccess || !*p) {
      dg_set_error((std::string("cudaGetSymbolAddress of the scratch array: ") +
                    cudaGetErrorString(e)).c_str());
      return DG_ERR_CUDA;
    }
    return DG_OK;
  };
  std::lock_guard<std::mutex> lk(g_mu);
  void *ctx = nullptr;
  if (get(&ctx) != 0) {
    dg_set_error("cuCtxGetCurrent failed");
    return DG_ERR_CUDA;
  }
  void *p = nullptr;
  if (!ctx) {
    // no context bound to this thread yet: the lookup binds the device's
    // primary context (the runtime does that lazily), which then identifies
    DG_TRY(lookup(&p));
    if (get(&ctx) != 0 || !ctx) {
      dg_set_error("no CUDA context is current after the scratch lookup");
      return DG_ERR_CUDA;
    }
    g_addr[{dev, ctx}] = p;
    *out = p;
    return DG_OK;
  }
  auto it = g_addr.find({dev, ctx});
  if (it != g_addr.end()) {
    // a context handle can come back with the same value after a reset, with
    // the module reloaded elsewhere: keep the cached address only while it
    // is still mapped device memory of this device
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, it->second) == cudaSuccess &&
        a.type == cudaMemoryTypeDevice && a.device == dev) {
      *out = it->second;
      return DG_OK;
    }
    cudaGetLastError();
  }
  DG_TRY(lookup(&p));
  g_addr[{dev, ctx}] = p;
  *out = p;
  return DG_OK;
}

// V and VV must be memory this device can address as device memory:
// anything else would fault inside a kernel and poison the caller's context
int check_device_pointer(const void *ptr, const char *name) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return DG_ERR_NODEV;
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();  // clear the query's error so the next launch check does not see it
    dg_set_error((std::string(name) + " is not a device pointer: " + cudaGetErrorString(e)).c_str());
    return DG_ERR_ARG;
  }
  if ((a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) || a.device != dev) {
    dg_set_error((std::string(name) + " must be device (or managed) memory of the current "
                  "device").c_str());
    return DG_ERR_ARG;
  }
  return DG_OK;
}

// exp(-2 pi i m / n) for the x and z lengths
__global__ void k_na_twiddles(double2 *twx, int nx, double2 *twz, int nz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nx + nz) {
    const int n = (i < nx) ? nx : nz;
    const int m = (i < nx) ? i : i - nx;
    double s, c;
    sincospi(2.0 * (double)m / (double)n, &s, &c);
    ((i < nx) ? twx : twz)[m] = make_double2(c, -s);
  }
}

// retained modes [nj][nkzt][nkxp] -> reference planes VV(0:NX/2,0:NZ+1), zero
// outside the retained block
__global__ void k_na_expand(const double2 *__restrict__ cmp, double2 *__restrict__ ref, int nj,
                            int nkzt, int nkxp, int nxp1, int nz2) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)nj * nz2 * nxp1) return;
  const int i = (int)(q % nxp1);
  const int k = (int)((q / nxp1) % nz2);
  const int j = (int)(q / ((long)nxp1 * nz2));
  double2 v = make_double2(0.0, 0.0);
  if (i < nkxp && k < nkzt) v = cmp[((long)j * nkzt + k) * nkxp + i];
  ref[q] = v;
}

size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" int diablo_fft_xz_to_fourier_noalloc(const double *V, double *VV, int nx, int nz,
                                                int ny, int jmin, int jmax, void *stream) {
  if (!V || !VV) {
    dg_set_error("V and VV must be device pointers");
    return DG_ERR_ARG;
  }
  DG_TRY(check_device_pointer(V, "V"));
  DG_TRY(check_device_pointer(VV, "VV"));
  if (ny < 1 || jmin < 0 || jmax > ny + 1 || jmax < jmin) {
    dg_set_error("need NY >= 1 and 0 <= JMIN <= JMAX <= NY+1");
    return DG_ERR_ARG;
  }
  FftPlan plx, plz;
  if (nx < 8 || nz < 8 || (nx & 1) || (nz & 1) || nx > 4096 || nz > 4096 ||
      !dg_make_plan(nx, &plx) || !dg_make_plan(nz, &plz)) {
    dg_set_error("NX and NZ must be even, 8..4096, and factor into 2, 3 and 5");
    return DG_ERR_DIMS;
  }
  const int nkx = nx / 3, nkz = nz / 3;
  const int nkxp = nkx + 1, nkzt = 2 * nkz + 1;
  const int nxp1 = nx / 2 + 1, nz2 = nz + 2;
  const size_t tw_bytes = up256(sizeof(double2) * nx) + up256(sizeof(double2) * nz);
  const size_t h_plane = sizeof(double2) * (size_t)nz * nkxp;     // after the x transform
  const size_t c_plane = sizeof(double2) * (size_t)nkzt * nkxp;   // retained modes
  const size_t per_plane = h_plane + c_plane;
  if (tw_bytes + up256(h_plane) + up256(c_plane) > (size_t)DG_NOALLOC_SCRATCH_BYTES) {
    dg_set_error("one NX x NZ plane needs more than the allocation-free entry point's "
                 "DG_NOALLOC_SCRATCH_BYTES of scratch");
    return DG_ERR_DIMS;
  }
  // planes per chunk
  int chunk = (int)((DG_NOALLOC_SCRATCH_BYTES - tw_bytes - 512) / per_plane);
  const int nj_all = jmax - jmin + 1;
  if (chunk > nj_all) chunk = nj_all;
  if (chunk < 1) chunk = 1;

  void *base = nullptr;
  DG_TRY(scratch_address(&base));
  unsigned char *b = (unsigned char *)base;
  double2 *twx = (double2 *)b;
  double2 *twz = (double2 *)(b + up256(sizeof(double2) * nx));
  double2 *H = (double2 *)(b + tw_bytes);
  double2 *cmp = (double2 *)(b + tw_bytes + up256(h_plane * chunk));

  // a handle on the stack carrying only what the transform launchers read
  dg_handle hh;
  memset(&hh, 0, sizeof(hh));
  hh.NX = nx;
  hh.NZ = nz;
  hh.NKX = nkx;
  hh.NKZ = nkz;
  hh.TNKZ = 2 * nkz;
  hh.nkxp = nkxp;
  hh.nkzt = nkzt;
  hh.ss = (long)nkzt * nkxp;
  hh.nplanes = chunk;
  hh.st = (cudaStream_t)stream;
  hh.plx = plx;
  hh.plz = plz;
  hh.twx = twx;
  hh.twz = twz;

  k_na_twiddles<<<dg_cdiv(nx + nz, 128), 128, 0, hh.st>>>(twx, nx, twz, nz);
  DG_LAUNCHED();
  const long pplane = (long)(nx + 2) * nz2;  // doubles per reference plane
  for (int j0 = jmin; j0 <= jmax; j0 += chunk) {
    const int nj = (jmax - j0 + 1 < chunk) ? jmax - j0 + 1 : chunk;
    DG_TRY(dg_xr2c_planes(&hh, V + (long)j0 * pplane, 1, 0, nj - 1, pplane, nx + 2, 0, H));
    double2 *flds[1] = {cmp};
    DG_TRY(dg_zfwd_planes(&hh, H, 1, 0, nj - 1, flds, nullptr, 0));
    k_na_expand<<<dg_cdiv((long)nj * nz2 * nxp1, 256), 256, 0, hh.st>>>(
        cmp, (double2 *)(VV + (long)j0 * pplane), nj, nkzt, nkxp, nxp1, nz2);
    DG_LAUNCHED();
  }
  return DG_OK;
}
