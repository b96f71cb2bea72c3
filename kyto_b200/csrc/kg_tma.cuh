// Host-side TMA descriptors for 2D row-major operands (tensor maps for
// cp.async.bulk.tensor loads into 128-byte-swizzled shared-memory tiles).
#pragma once

#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>
#include <string>

#include "kg_internal.cuh"

namespace kg {

inline PFN_cuTensorMapEncodeTiled_v12000 tma_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  if (!fn) fail(KG_ERR_DEVICE, "cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

// A rows x cols matrix of 16-bit elements (row stride row_bytes, a multiple of 16; base
// 16-byte aligned), boxes of box_rows x box_cols (box_cols * 2 = 128 bytes: one swizzle
// row), 128-byte swizzle, zero fill past the edges.
inline CUtensorMap tma_map_2d_16bit(const void* base, CUtensorMapDataType type, uint64_t cols,
                                    uint64_t rows, uint64_t row_bytes, uint32_t box_cols,
                                    uint32_t box_rows) {
  if (row_bytes % 16 != 0 || (reinterpret_cast<uintptr_t>(base) & 15u) != 0)
    fail(KG_ERR_INVALID, "tensor map: base and row stride must be 16-byte aligned");
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)row_bytes};
  cuuint32_t box[2] = {box_cols, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = tma_encode_fn()(&m, type, 2, const_cast<void*>(base), dims, strides, box, estr,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(KG_ERR_DEVICE, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return m;
}

}  // namespace kg
