// Tensor maps for the bulk tensor copies (TMA) of the column kernels.
//
// cuTensorMapEncodeTiled is a driver entry point; it is looked up once
// through the runtime (cudaGetDriverEntryPoint) so the library needs no
// direct link to the driver library.
#include <mutex>

#include "dg_internal.cuh"

namespace {

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}

}  // namespace

int dg_tmap_planes(const void *base, long ss, int rows, int mt, int by, CUtensorMap *out) {
  EncodeTiled fn = encoder();
  if (!fn) {
    dg_set_error("cuTensorMapEncodeTiled is not available from the driver");
    return DG_ERR_CUDA;
  }
  // x: the 2 ss doubles of a plane (16-byte row pitch; a box starts at
  // x = 2 m0, a 16-byte boundary), y: planes
  const cuuint64_t gdim[2] = {(cuuint64_t)(2 * ss), (cuuint64_t)rows};
  const cuuint64_t gstride[1] = {(cuuint64_t)ss * sizeof(double2)};
  const cuuint32_t box[2] = {(cuuint32_t)(2 * mt), (cuuint32_t)by};
  const cuuint32_t estride[2] = {1, 1};
  const CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void *>(base), gdim,
                        gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    dg_set_error("cuTensorMapEncodeTiled rejected a column tile map");
    return DG_ERR_CUDA;
  }
  return DG_OK;
}
