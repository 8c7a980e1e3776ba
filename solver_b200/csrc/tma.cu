// Host side of tma.cuh: tensor-map encoding through the driver entry point
// (no link-time dependency on libcuda).
#include "tma.cuh"

#include <mutex>

namespace ofb {
namespace tma {

namespace {

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                              CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                              CUtensorMapFloatOOBfill);

EncodeFn encoder() {
  static std::once_flag once;
  static EncodeFn fn = nullptr;
  static cudaError_t err = cudaSuccess;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    err = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
    if(err == cudaSuccess && q == cudaDriverEntryPointSuccess) fn = reinterpret_cast<EncodeFn>(p);
  });
  if(fn == nullptr) throw std::runtime_error("cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

}  // namespace

CUtensorMap make_map_3d(const void* base, int elem_bytes, int nx, int ny, int nz, int bx, int by) {
  if(reinterpret_cast<uintptr_t>(base) % 16 != 0)
    throw std::invalid_argument("tensor map base must be 16-byte aligned");
  if((static_cast<long long>(nx) * elem_bytes) % 16 != 0)
    throw std::invalid_argument("tensor map row pitch must be a multiple of 16 bytes");
  if((static_cast<long long>(bx) * elem_bytes) % 16 != 0 || bx > 256 || by > 256 || bx < 1 || by < 1)
    throw std::invalid_argument("tensor map box must be 16-byte wide and at most 256 elements per axis");
  CUtensorMap map;
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(nx), static_cast<cuuint64_t>(ny),
                              static_cast<cuuint64_t>(nz)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(nx) * elem_bytes,
                                 static_cast<cuuint64_t>(nx) * ny * elem_bytes};
  const cuuint32_t box[3] = {static_cast<cuuint32_t>(bx), static_cast<cuuint32_t>(by), 1u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  const CUresult r = encoder()(&map, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                                     : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                               3, const_cast<void*>(base), dims, strides, box, estr,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if(r != CUDA_SUCCESS)
    throw std::runtime_error("cuTensorMapEncodeTiled failed (" + std::to_string(static_cast<int>(r)) + ")");
  return map;
}

}  // namespace tma
}  // namespace ofb
