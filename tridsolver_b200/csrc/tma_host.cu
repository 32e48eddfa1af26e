// Host side of the TMA helpers: tensor-map encoding through the driver entry
// point cuTensorMapEncodeTiled, looked up once through the runtime.
#include <cudaTypedefs.h>

#include <mutex>

#include "tma.cuh"

namespace tridb200 {

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static std::once_flag g_encode_once;

static void load_encode() {
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault,
                                       &q) == cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  else
    cudaGetLastError();
}

bool encode_tensor_map(CUtensorMap *map, const void *base, int elem_bytes, int rank,
                       const uint64_t *dims, const uint64_t *strides_bytes, const uint32_t *box,
                       bool swizzle128) {
  std::call_once(g_encode_once, load_encode);
  if (!g_encode || rank < 1 || rank > 5) return false;
  cuuint64_t gdim[5], gstride[4];
  cuuint32_t bdim[5], estride[5];
  for (int i = 0; i < rank; ++i) {
    gdim[i] = dims[i];
    bdim[i] = box[i];
    estride[i] = 1;
    if (i + 1 < rank) gstride[i] = strides_bytes[i];
  }
  const CUtensorMapDataType dt =
      elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const CUresult r =
      g_encode(map, dt, (cuuint32_t)rank, const_cast<void *>(base), gdim, gstride, bdim, estride,
               CU_TENSOR_MAP_INTERLEAVE_NONE,
               swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace tridb200
