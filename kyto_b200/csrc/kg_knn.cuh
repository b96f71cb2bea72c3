// Sizes of the exact-kNN kernels.
#pragma once

#include <cstdint>

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

}  // namespace kg
