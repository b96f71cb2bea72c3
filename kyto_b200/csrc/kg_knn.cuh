// Sizes of the exact-kNN kernels.
#pragma once

#include <cstdint>
#include <functional>
#include <vector>

#include "kg_internal.cuh"

namespace kg {

constexpr int kDim = 64;                  // components a row is padded to
constexpr uint32_t kTile = 128;           // points per shared-memory tile (filter)
constexpr int kFilterThreads = 128;       // queries per filter CTA
constexpr int kMaxK = 128;                // largest n_neighbors - 1
constexpr uint32_t kCandidateCap = 1024;  // candidate slots per query
constexpr uint32_t kCandidateLimit = 512; // candidates kept after a compaction, at most
constexpr uint32_t kOverflow = 0xFFFFFFFFu;
constexpr uint64_t kQueryChunk = 1ull << 18;  // queries per filter launch
constexpr int kRankWarps = 4;
constexpr int kFullWarps = 8;

// Every row's k nearest other rows (device), with the search's counters.
struct KnnResult {
  DeviceBuffer<double> key;    // n x k, ascending by (key, row)
  DeviceBuffer<uint32_t> row;
  uint64_t candidates = 0, rows_full = 0, retried = 0;
  uint64_t tiles_scanned = 0, tiles_total = 0;  // the filter's block-tile products
  double filter_ms = 0, rank_ms = 0;
};

// The tensor-core filter's scan: query slot q is row qrows[q], point slot p row prows[p]
// (prows empty: qrows), q_point (or empty) maps a query slot to the point slot of the
// same row; each block of 256 query slots scans its list of point tiles (list_off CSR, or
// list_stride entries a block; no list: every tile from the block's own), skipping
// tiles on their list_lb2 bounds when given.
// A batch of samples searched at once: sample s is rows [first[s], first[s + 1]) of x,
// and a row's neighbours come from its own sample only.
struct KnnBatch {
  std::vector<uint64_t> first;         // n_samples + 1 row offsets (host)
  DeviceBuffer<uint64_t> d_first;      // the same on the device
  DeviceBuffer<uint32_t> row_sample;   // per row: its sample
};

struct ScanPlan {
  DeviceBuffer<uint32_t> qrows, prows, q_point;
  DeviceBuffer<uint32_t> list_tiles;
  DeviceBuffer<float> list_lb2;
  DeviceBuffer<uint64_t> list_off;
  uint64_t list_stride = 0;
  bool list_sorted = false;  // each block's list ascending by bound  // Per query slot (or empty): 1 where the slot's list does not cover its row, which is
  // then searched over every tile with the overflowed queries.
  DeviceBuffer<uint8_t> q_full;
};
// Builds the filter's scan for query blocks of qblock slots.
using PlanBuilder = std::function<void(const float* x, uint64_t n, uint32_t width, uint32_t d,
                                       double scale, uint32_t qblock, ScanPlan& plan,
                                       Trace& trace)>;

void knn_core(kg_ctx* ctx, const float* x, uint64_t n, uint32_t width, uint32_t d, uint32_t k,
              const PlanBuilder* plan, KnnResult& out, Trace& trace,
              const KnnBatch* batch = nullptr);
void knn_batch_run(kg_ctx* ctx, const float* x, uint64_t n, uint32_t width, uint32_t d,
                   uint32_t k, const std::vector<uint64_t>& first, uint64_t* indptr,
                   uint32_t* indices, float* distances, kg_knn_stats* stats);
void check_search_args(uint64_t n, uint32_t width, uint32_t n_components, uint32_t n_neighbors,
                       uint32_t& k, uint32_t& d);
void check_finite(const float* x, uint64_t n, uint32_t width, uint32_t d, cudaStream_t s);
void write_graph(const KnnResult& r, uint64_t n, uint32_t k, uint64_t* indptr, uint32_t* indices,
                 float* distances, cudaStream_t s);

}  // namespace kg
