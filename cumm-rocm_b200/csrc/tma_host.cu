// tma_host.cu - host-side TMA tensor-map encoding (cuTensorMapEncodeTiled,
// fetched through the runtime's driver entry point so the library does not
// link libcuda directly).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "kernels.h"

namespace scb {
namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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

bool encode_tmap_2d(void *out_map, int dtype, const void *base, uint64_t inner, uint64_t outer,
                    uint64_t row_stride_bytes, uint32_t box_inner, uint32_t box_outer,
                    int swizzle_bytes) {
  auto fn = encode_fn();
  if (fn == nullptr) return false;
  if (reinterpret_cast<uintptr_t>(base) % 16 || row_stride_bytes % 16) return false;
  if (inner == 0 || outer == 0 || box_inner == 0 || box_outer == 0) return false;
  if (box_inner > 256 || box_outer > 256) return false;
  if (outer >= (1ull << 32) || inner >= (1ull << 32)) return false;
  CUtensorMapDataType t;
  uint32_t es;
  switch (dtype) {
    case 12: t = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; es = 2; break;
    case 7: t = CU_TENSOR_MAP_DATA_TYPE_FLOAT16; es = 2; break;
    case 14: t = CU_TENSOR_MAP_DATA_TYPE_UINT8; es = 1; break;
    default: return false;
  }
  // one swizzle line per box row: SWIZZLE_128B or SWIZZLE_64B
  if (swizzle_bytes != 128 && swizzle_bytes != 64) return false;
  if (box_inner * es != static_cast<uint32_t>(swizzle_bytes)) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {row_stride_bytes};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t elem_strides[2] = {1, 1};
  CUresult r = fn(reinterpret_cast<CUtensorMap *>(out_map), t, 2, const_cast<void *>(base), dims,
                  strides, box, elem_strides, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  swizzle_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace scb
