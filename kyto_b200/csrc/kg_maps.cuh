// Device steps of kyto's per-cell maps (normalize_total, log1p), shared by the map
// entry points and the PCA's pack kernel.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace kg {

// A stored value as kyto's KernelValue reads it (crates/kyto-exec/src/kernels.rs:48-90).
__device__ __forceinline__ float value_f32(const uint32_t* v, uint64_t i) {
  return __uint2float_rn(v[i]);  // Rust `as f32`: round to nearest even
}
__device__ __forceinline__ float value_f32(const float* v, uint64_t i) { return v[i]; }
__device__ __forceinline__ double value_wide(const uint32_t* v, uint64_t i, bool round32) {
  return round32 ? (double)__uint2float_rn(v[i]) : (double)v[i];
}
__device__ __forceinline__ double value_wide(const float* v, uint64_t i, bool) {
  return (double)v[i];
}

// The normalize divisor of one row, computed by the 8 threads of an aligned group of 8
// lanes (lane class c = lane % 8 sums values c, c+8, ... of the row in order, as kyto's
// SUM_LANES accumulators; the classes combine in kyto's fixed tree
// ((a0+a4)+(a2+a6))+((a1+a5)+(a3+a7)), kernels.rs:281-292). Every thread of the group
// gets the divisor: f32(total) / f32(target), 0 -> 1 (elementwise.rs:262-269).
// All 32 lanes of the warp must call it together.
// round32: the block holds a u32 count that is not a float32 (elementwise.rs:241-257).
template <class V>
__device__ __forceinline__ float row_divisor(const V* values, uint64_t s, uint64_t e,
                                             float target32, bool round32) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned c = lane & 7u;
  double acc = 0.0;
  for (uint64_t i = s + c; i < e; i += 8) acc = __dadd_rn(acc, value_wide(values, i, round32));
  const unsigned mask = 0xFFFFFFFFu;  // the whole warp calls this (rows past the end
                                      // pass s == e)
  // h_c = a_c + a_{c+4} (c < 4); q_c = h_c + h_{c+2} (c < 2); total = q_0 + q_1.
  double other = __shfl_down_sync(mask, acc, 4, 8);
  double h = __dadd_rn(acc, other);
  other = __shfl_down_sync(mask, h, 2, 8);
  double q = __dadd_rn(h, other);
  other = __shfl_down_sync(mask, q, 1, 8);
  double total = __dadd_rn(q, other);
  total = __shfl_sync(mask, total, 0, 8);
  float divisor = __fdiv_rn((float)total, target32);
  return divisor == 0.0f ? 1.0f : divisor;
}

// kyto's log1p (crates/kyto-exec/src/kernels/log1p.rs:49-75): ln(1 + x) evaluated in f64
// and rounded once to f32. CUDA's f64 log1p is within an ulp of f64, so the f32
// rounding is the correctly rounded one except within ~1e-16 of a halfway point.
__device__ __forceinline__ float log1p_f32(float x) { return (float)log1p((double)x); }

// One stored value after the maps: f32(v) / divisor (IEEE division), then log1p.
template <class V>
__device__ __forceinline__ float mapped_value(const V* values, uint64_t i, bool normalize,
                                              float divisor, bool do_log1p) {
  float v = value_f32(values, i);
  if (normalize) v = __fdiv_rn(v, divisor);
  if (do_log1p) v = log1p_f32(v);
  return v;
}

}  // namespace kg
