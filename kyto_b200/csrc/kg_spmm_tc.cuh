// The tensor-core sparse x dense product of the PCA (kg_spmm_tc.cu) and the blocked
// sparse layout it reads.
#pragma once

#include <cstdint>

#include "kg_internal.cuh"

namespace kg {

// A sparse matrix (rows x K) cut into blocks of 128 rows x 32 columns. Block
// b = tile * n_chunks + chunk starts at byte 16 * off[b] of `data` and is empty
// (off[b + 1] == off[b]) or holds 128 mask words (bit c of word r: a value at row r,
// column c of the block) followed by its values, rows in order and columns in order
// inside a row, padded to a multiple of 4 floats: 16-byte aligned, one bulk copy each.
// At the benchmark's 30% density that is 512 + 4 nnz bytes a block, against 6 nnz for
// 16-bit positions beside the values.
struct Blocked {
  uint64_t rows = 0, K = 0;
  uint32_t n_tiles = 0, n_chunks = 0;
  uint64_t bytes = 0;
  DeviceBuffer<uint64_t> off;   // n_tiles * n_chunks + 1 offsets, 16-byte units
  DeviceBuffer<uint8_t> data;
};

// The blocked layout of a CSR matrix (n_rows x n_cols, u32 column indices, each row's
// columns strictly increasing), or of its transpose (rows = the CSR's columns).
void build_blocked(const uint64_t* ptr, const uint32_t* col, const float* val, uint64_t n_rows,
                   uint64_t n_cols, uint64_t nnz, bool transpose, Blocked& out, cudaStream_t s);

// The blocked layout of X^T from X's (bit-transposed blocks, values moved by rank): the
// same bytes build_blocked(..., transpose = true) writes.
void transpose_blocked(const Blocked& x, Blocked& out, cudaStream_t s);

enum : int { kOutRows = 0, kOutPartial = 1 };
enum : int { kValuePlain = 0, kValueCentredSquare = 1, kValueOne = 2 };

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
  const Blocked* s = nullptr;      // the sparse operand
  int value_mode = kValuePlain;    // kValueCentredSquare: (v - row_means[row])^2;
                                   // kValueOne: 1 for every stored value
  const double* row_means = nullptr;
  uint64_t seg_chunks = 0;         // K-chunks (32 columns) per work item
  const float* dt_hi = nullptr;    // D^T, 64 x K, tf32 parts, row stride ld_t floats
  const float* dt_lo = nullptr;
  uint64_t ld_t = 0;
  SpmmOut out;
  int sm_count = 148;
};

void spmm_tc(const SpmmArgs& a, cudaStream_t s);

}  // namespace kg
