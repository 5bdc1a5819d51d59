// pip_tma.cu -- host side of the TMA tile staging: the tensor-map encoder, reached through
// the runtime's driver entry point (no link against the driver library).
#include <cudaTypedefs.h>

#include <mutex>

#include "pip_tma.cuh"

namespace pip {

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

}  // namespace

bool tma_encode(CUtensorMap *map, const void *base, int ix, int jx, int nv, int esize, int rx,
                int ry) {
  PFN_cuTensorMapEncodeTiled_v12000 fn = encoder();
  if (!fn || (esize != 4 && esize != 8)) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)ix, (cuuint64_t)jx, (cuuint64_t)nv};
  const cuuint64_t strides[2] = {(cuuint64_t)ix * esize, (cuuint64_t)ix * jx * esize};
  const cuuint32_t box[3] = {(cuuint32_t)rx, (cuuint32_t)ry, (cuuint32_t)nv};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r =
      fn(map, esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
         const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace pip
