// The tensor-core candidate filter of the exact kNN (kg_knn_tc.cu).
#pragma once

#include <cstdint>

#include "kg_internal.cuh"

namespace kg {

constexpr uint32_t kTcCap = 512;             // candidate slots per query (a query
                                             // overflows when more than half stay after
                                             // a compaction)
constexpr uint32_t kTcRetryCap = 8192;       // slots per query in the overflow retry
constexpr uint64_t kTcRetryChunk = 65536;    // queries per retry pass
constexpr uint32_t kTcRetrySplitCap = 4096;  // slots per query copy when a retry's tiles
                                             // are split between copies of its queries
constexpr uint64_t kTcRetrySplitSlots = 32768;  // query slots over all copies, at most
constexpr uint32_t kTcQueryBlock = 256;      // query slots per block of the fp16/bf16 filter

// The filter's operands: fp16 or bf16 (one 64-wide row: the components and the norm), or
// split (fp16 hi and lo parts, three products; a slack 2^5 times smaller than fp16's).
enum class FilterKind { Fp16, Bf16, Split };

// Where the filter's MMAs read the query operand and how its accumulators are cut (the
// same keys every way): shared memory, two slots of both query halves; tensor memory,
// three half slots; shared memory, four half slots.
enum : int { kTcAmSmem = 0, kTcAmTmem = 1, kTcAmHalf = 2 };

// Query slots per block of the filter of this kind (the blocks tile lists are built for).
uint32_t filter_query_block(FilterKind kind);

// What one filter launch scans. Query slot q is row qrows[q] of x, point slot p row
// prows[p]; each block of query slots (filter_query_block) scans its list of point tiles (128 slots) in
// order, or every tile from its own when list_tiles is NULL, skipping a listed tile whose
// bound (list_lb2, a lower bound of the scaled squared distance between the tile's rows and
// the block's) exceeds every live query's threshold + s^2 |q|^2 + its slack.
struct FilterScan {
  uint64_t n_q = 0, n_p = 0;
  const uint32_t* q_point = nullptr;     // query slot -> point slot of the same row (NULL:
                                         // the same slot)
  const uint32_t* list_tiles = nullptr;  // the blocks' tile lists
  const float* list_lb2 = nullptr;       // their bounds (or NULL: none skipped)
  const uint64_t* list_off = nullptr;    // block qb's entries start at list_off[qb] and end
                                         // at list_off[qb + 1] (or NULL: qb * list_stride,
                                         // list_stride entries each)
  uint64_t list_stride = 0;
  bool list_sorted = false;              // each block's bounds ascend: the first skipped
                                         // tile ends the block's scan
  const uint32_t* slot_sample = nullptr;  // per query slot its sample (NULL: one sample):
  const uint64_t* sample_first = nullptr; // a query takes only the point slots
                                          // [sample_first[s], sample_first[s + 1]) of its
                                          // sample s (a batch of samples searched at once)
  unsigned long long* tiles_scanned = nullptr;  // when set: += tiles the launch multiplied
  unsigned int* block_counter = nullptr;  // query blocks handed out past the first wave
                                          // (zero before the launch; set by tc_filter)
  int a_mode = -1;                       // the query operand's mode (kTcAmSmem, kTcAmTmem,
                                         // kTcAmHalf), or -1: shared memory;
                                         // KYTO_GPU_FILTER_A overrides either
  const double* qn2 = nullptr;           // per query slot |q - mean|^2 (set by tc_filter)
  double s2 = 1.0;                       // scale^2 (set by tc_filter)
};

// The power-of-two scale of the filter's operands (the largest centred row norm of x's
// n rows scaled to at most 2^7), and that largest squared norm on the device (max_sq).
double tc_scale(const float* x, uint64_t n, uint32_t width, uint32_t d, const double* mean,
                double* max_sq, cudaStream_t s);

// Fills cand_key/cand_row (n_q x cap), cand_count and threshold (n_q) for every query
// slot, and per query slot qn2 (the centred squared norm) and slack_d (the bound of
// |approximate - exact| key in squared-distance units). Keys are in units scaled by
// scale^2: the approximate squared distance is key / scale^2 + qn2.
void tc_filter(kg_ctx* ctx, cudaStream_t s, const float* x, uint32_t width, uint32_t d,
               const uint32_t* qrows, const uint32_t* prows, FilterScan scan,
               const double* mean, double scale, const double* max_sq, FilterKind kind,
               uint32_t k, uint32_t cap, float* cand_key, uint32_t* cand_row,
               uint32_t* cand_count, float* threshold, double* qn2, double* slack_d,
               Trace* trace = nullptr, DeviceBuffer<uint16_t>* point_ops = nullptr);

void max_kernel_launch(const double* v, uint64_t n, double* out, cudaStream_t s);

}  // namespace kg
