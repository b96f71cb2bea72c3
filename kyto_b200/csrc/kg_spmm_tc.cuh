// The tensor-core sparse x dense product of the PCA (kg_spmm_tc.cu).
#pragma once

#include <cstdint>

#include "kg_internal.cuh"

namespace kg {

enum : int { kOutRows = 0, kOutPartial = 1 };

// Where C = S D goes.
struct SpmmOut {
  int mode = kOutRows;
  uint32_t width = 64;             // columns of C that carry data (<= 64)
  // kOutRows (one K segment): row r of C minus `offsets` (width f64 values) ...
  const double* offsets = nullptr;
  float* t_hi = nullptr;           // ... as C^T split in two tf32 parts (64 x ld_t f32),
  float* t_lo = nullptr;
  uint64_t ld_t = 0;
  float* rows_f32 = nullptr;       // ... as f32 rows (rows x width),
  double* colsum_partial = nullptr;  // ... and the column sums of t_hi + t_lo per tile
                                     // of 128 rows (n_tiles x 64 f64).
  // kOutPartial: each K segment's C as f64 (segments x rows x 64).
  double* partial = nullptr;
};

struct SpmmArgs {
  const uint64_t* ptr = nullptr;   // CSR row pointers (rows + 1)
  const uint16_t* col16 = nullptr; // column indices, 16-bit ...
  const uint32_t* col32 = nullptr; // ... or 32-bit
  const float* val = nullptr;
  uint64_t rows = 0, K = 0;
  uint64_t seg_len = 0;            // K per work item (a multiple of 32)
  const float* dt_hi = nullptr;    // D^T, 64 x K, tf32 parts, row stride ld_t floats
  const float* dt_lo = nullptr;
  uint64_t ld_t = 0;
  SpmmOut out;
  int sm_count = 148;
};

void spmm_tc(const SpmmArgs& a, cudaStream_t s);

}  // namespace kg
