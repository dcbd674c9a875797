// tma.cu -- host side of the tiled TMA copies: tensor maps encoded through the driver entry point
// cuTensorMapEncodeTiled (reached through the runtime, so the library links no driver library).
#include <mutex>

#include "tma.cuh"

namespace ofc {
namespace {

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static std::once_flag once;
  static EncodeTiled fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
    (void)cudaGetLastError();
  });
  return fn;
}

}  // namespace

bool tma_map_f32(CUtensorMap* m, const void* base, int rank, const uint64_t* dims, const uint64_t* strides_bytes,
                 const uint32_t* box) {
  if (rank < 1 || rank > 3 || ((uintptr_t)base & 15) != 0) return false;
  if ((box[0] * sizeof(float)) % 16 != 0) return false;
  for (int i = 0; i < rank; i++)
    if (box[i] < 1 || box[i] > 256 || dims[i] < 1) return false;
  for (int i = 0; i + 1 < rank; i++)
    if (strides_bytes[i] % 16 != 0) return false;
  EncodeTiled enc = encode_fn();
  if (!enc) return false;
  cuuint64_t d[3], s[2];
  cuuint32_t b[3], e[3];
  for (int i = 0; i < rank; i++) {
    d[i] = dims[i];
    b[i] = box[i];
    e[i] = 1;
  }
  for (int i = 0; i + 1 < rank; i++) s[i] = strides_bytes[i];
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank, const_cast<void*>(base), d, s, b, e,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace ofc
