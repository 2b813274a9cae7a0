// Host-side TMA descriptors for row-major BF16 matrices, encoded through the
// driver entry point fetched by the runtime (no link-time libcuda dependency).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"

namespace mm {

using TensorMapEncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                       const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                       CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline int tensor_map_encoder(TensorMapEncodeFn* out) {
  static TensorMapEncodeFn fn = nullptr;
  static cudaError_t status = cudaSuccess;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q{};
    status = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", reinterpret_cast<void**>(&fn), cudaEnableDefault, &q);
    if (status == cudaSuccess && q != cudaDriverEntryPointSuccess) fn = nullptr;
  });
  if (status != cudaSuccess) return cuda_status(status, "cudaGetDriverEntryPoint(cuTensorMapEncodeTiled)");
  if (!fn) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return MM_ERR_CUDA;
  }
  *out = fn;
  return MM_OK;
}

// Box of 64 columns (128 bytes, one swizzle row) x box_rows rows with the
// 128-byte swizzle; reads outside [rows x cols] return zeros.
inline int bf16_map(CUtensorMap* m, const void* ptr, long long rows, long long cols, int box_rows) {
  MM_CHECK_ARG(ptr != nullptr, "tensor map over a NULL matrix");
  MM_CHECK_ARG(reinterpret_cast<uintptr_t>(ptr) % 16 == 0, "BF16 matrix must be 16-byte aligned");
  MM_CHECK_ARG(rows >= 1 && cols >= 8 && cols % 8 == 0, "BF16 matrix %lld x %lld: columns must be a multiple of 8",
               rows, cols);
  MM_CHECK_ARG(box_rows >= 8 && box_rows <= 256, "box rows %d", box_rows);
  TensorMapEncodeFn fn;
  if (int rc = tensor_map_encoder(&fn)) return rc;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  const cuuint32_t box[2] = {64u, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d) for a %lld x %lld BF16 matrix, box %d rows", (int)r, rows, cols,
              box_rows);
    return MM_ERR_CUDA;
  }
  return MM_OK;
}

}  // namespace mm
