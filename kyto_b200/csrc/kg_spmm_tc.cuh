// The tensor-core sparse x dense product of the PCA (kg_spmm_tc.cu), the blocked sparse
// layout it reads and the dense operand layout it takes.
#pragma once

#include <cstdint>

#include "kg_internal.cuh"

namespace kg {

// A sparse matrix (rows x K) cut into blocks of 128 rows x 32 columns, each column pair
// (2p, 2p + 1) stored as one entry per row that holds a value in either column. Block
// b = tile * n_chunks + chunk starts at byte 16 * off[b] of `data` and is empty
// (off[b + 1] == off[b]) or holds a header of 64 (mask, base) words followed by its
// entries:
//  - header word q * 16 + p (rows 32 q .. 32 q + 31, pair p): bit l of the mask is set
//    where row 32 q + l has an entry for pair p; base is the rank of the first such entry
//    (entries ordered by row quarter, then pair, then row);
//  - an entry is two 32-bit words: the fp16 high parts of the pair's two values
//    (column 2p in bits 0-15, 2p + 1 in bits 16-31), then their fp16 low parts, where a
//    value's parts are hi = fp16(x) and lo = fp16(x - hi) of x = value * 2^scale (about
//    22 bits of x); a column without a value holds hi = 0x8000 (fp16 -0, which adds
//    nothing to a product) and lo = 0, so that a stored zero (hi = +0) stays a value;
//  - the whole block is a multiple of 16 bytes (one bulk copy).
// A warp of the product reads one (mask, base) word per pair and, in its lanes that hold
// an entry, consecutive 8-byte entries: two words of the tensor-core operand per pair
// with no unpacking. At the benchmark's 33% density a block is 512 + 8 x ~1,130 bytes.
struct Blocked {
  uint64_t rows = 0, K = 0;
  uint32_t n_tiles = 0, n_chunks = 0;
  uint64_t bytes = 0;
  int scale = 0;            // values stored times 2^scale (largest |x| in [2^14, 2^15))
  double max_abs = 0.0;     // the largest |value| and the smallest nonzero one
  double min_abs = 0.0;
  double max_row_norm = 0.0;  // the largest row's Euclidean norm (rows of the CSR)
  DeviceBuffer<uint64_t> off;  // n_tiles * n_chunks + 1 offsets, 16-byte units
  DeviceBuffer<uint8_t> data;
};

// The blocked layout of a CSR matrix (n_rows x n_cols, u32 column indices, each row's
// columns strictly increasing).
void build_blocked(const uint64_t* ptr, const uint32_t* col, const float* val, uint64_t n_rows,
                   uint64_t n_cols, uint64_t nnz, Blocked& out, cudaStream_t s);

// The blocked layout of the same CSR's transpose (n_cols x n_rows), with x's scale and
// value range (x = build_blocked of that CSR).
void transpose_blocked(const uint64_t* ptr, const uint32_t* col, const float* val,
                       uint64_t n_rows, uint64_t n_cols, uint64_t nnz, const Blocked& x,
                       Blocked& out, cudaStream_t s);

// The dense operand D (K x 64) as the products read it: D^T, 64 rows of fp16 parts of
// each value times 2^scale, interleaved by chunk: for chunk c, row j holds the 32 high
// parts of D[32c .. 32c+31][j] and then their 32 low parts (128 bytes, one TMA box row).
// Rows are `ld` halves long (ld = 64 * chunks, chunks = ceil(K / 32)).
inline uint64_t dense_ld(uint64_t K) { return (K + 31) / 32 * 64; }

// The exponent that puts the largest magnitude `bound` in [2^14, 2^15) (0 for 0).
int part_scale(double bound);

enum : int { kOutRows = 0, kOutPartial = 1 };
enum : int { kValuePlain = 0, kValueCentredSquare = 1, kValueOne = 2 };

// Where C = S D goes.
struct SpmmOut {
  int mode = kOutRows;
  uint32_t width = 64;             // columns of C that carry data (<= 64)
  // kOutRows (one K segment): row r of C minus `offsets` (width f64 values) ...
  const double* offsets = nullptr;
  uint16_t* t = nullptr;           // ... as the next product's D^T (dense layout above,
  uint64_t ld_t = 0;               //     row length ld_t halves, values times 2^t_scale),
  int t_scale = 0;
  float* rows_f32 = nullptr;       // ... as f32 rows (rows x width),
  double* colsum_partial = nullptr;  // ... and the column sums of the rounded rows (as
                                     // the next product sees them) per tile of 128 rows
                                     // (n_tiles x 64 f64).
  // kOutPartial: each K segment's C as f64 (segments x rows x 64).
  double* partial = nullptr;
};

struct SpmmArgs {
  const Blocked* s = nullptr;      // the sparse operand
  int value_mode = kValuePlain;    // kValueCentredSquare: (v - row_means[row])^2;
                                   // kValueOne: 1 for every stored value
  const double* row_means = nullptr;
  uint64_t seg_chunks = 0;         // K-chunks (32 columns) per work item
  const uint16_t* dt = nullptr;    // D^T in the dense layout, row length ld_t halves,
  uint64_t ld_t = 0;               // values times 2^dt_scale
  int dt_scale = 0;
  SpmmOut out;
  int sm_count = 148;
  int* error = nullptr;            // set to 1 if a bounded wait ran out (device flag)
};

// Launches the product on stream s (no host synchronisation; `error` reports a pipeline
// that gave up waiting).
void spmm_tc(const SpmmArgs& a, cudaStream_t s);

}  // namespace kg
