// The tensor-core candidate filter of the exact kNN (kg_knn_tc.cu).
#pragma once

#include <cstdint>

#include "kg_internal.cuh"

namespace kg {

constexpr uint32_t kTcCap = 512;             // candidate slots per query
constexpr uint32_t kTcCandidateLimit = 256;  // candidates kept after a compaction, at most

// Fills cand_key/cand_row (n x cap), cand_count and threshold (n) for every query, and
// per row qn2 (the centred squared norm) and slack_d (the bound of |approximate -
// exact| key in squared-distance units). Keys are in units scaled by out_scale^2:
// the approximate squared distance is key / out_scale^2 + qn2.
// perm: the rows in scan order (row i of the operands is row perm[i] of x), or NULL.
void tc_filter(kg_ctx* ctx, cudaStream_t s, const float* x, uint64_t n, uint32_t width,
               uint32_t d, const uint32_t* perm, const double* mean, bool bf16, uint32_t k,
               uint32_t cap,
               float* cand_key, uint32_t* cand_row, uint32_t* cand_count, float* threshold,
               double* qn2, double* slack_d, double* out_scale);

void max_kernel_launch(const double* v, uint64_t n, double* out, cudaStream_t s);

}  // namespace kg
