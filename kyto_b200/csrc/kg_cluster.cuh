// Clusters of an embedding's rows: Lloyd's k-means on the device, the rows ordered by
// cluster (then by their first component), for the learned partitioner's parts and as
// a scan order of the exact kNN filter.
#pragma once

#include <cstdint>

#include "kg_internal.cuh"

namespace kg {

constexpr uint32_t kClusterDim = 64;  // components a centre is padded to

struct Clusters {
  uint32_t K = 0;
  DeviceBuffer<uint32_t> label;   // n: the row's cluster
  DeviceBuffer<double> centre;    // K x kClusterDim: the mean of the cluster's rows
  DeviceBuffer<uint32_t> perm;    // n: slot -> row, rows by cluster then first component
  DeviceBuffer<uint32_t> start;   // K + 1: first slot of each cluster
};

// Lloyd's k-means on the leading d components of x (n x width f32): K centres fitted on
// an evenly strided sample of at most `sample` rows for `iters` rounds (seeded with
// evenly strided sample rows), then every row assigned and the centres recomputed from
// all rows. Deterministic: fixed-order sums, ties to the lower centre.
void cluster_rows(const float* x, uint64_t n, uint32_t width, uint32_t d, uint32_t K,
                  uint32_t iters, uint64_t sample, Clusters& out, cudaStream_t s);

// labels[r] = the centre (of K, K x kClusterDim f32, squared norms cn) nearest to row r
// of x (f32 distances; ties to the lower centre).
void nearest_centres(const float* x, uint64_t n, uint32_t width, uint32_t d,
                     const float* centres, const float* cn, uint32_t K, uint32_t* labels,
                     cudaStream_t s);

}  // namespace kg
