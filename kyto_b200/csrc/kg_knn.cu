// Exact Euclidean kNN (kyto's neighbors.rs + neighbors_exact.rs) on the device.
//
// Three steps, each one kernel family:
//  1. filter: every query against every point by an approximate key with a proven
//     error bound; each query keeps its k smallest approximate keys and every point
//     whose approximate key is at most the k-th plus twice its slack (kyto's
//     neighbors_exact.rs:50-356 algorithm, one query per thread, the point tile in
//     shared memory);
//  2. rank: the candidates' exact keys (f64, kyto's 8-lane order, no FMA: the same bits
//     as the CPU) ranked by (key, row); a row whose candidates are not proven complete
//     (too many, or an approximate key outside its slack) is flagged;
//  3. full rows: flagged rows searched against every row with exact keys.
// So every row is the CPU's brute-force row, bit for bit.
#include <cub/device/device_select.cuh>
#include <cub/iterator/counting_input_iterator.cuh>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_radix_sort.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>
#include <tuple>
#include <mutex>
#include <map>

#include <cstdlib>
#include <string>

#include "kg_cluster.cuh"
#include "kg_internal.cuh"
#include "kg_knn.cuh"
#include "kg_knn_tc.cuh"
#include "kg_tune.cuh"

namespace kg {

// ------------------------------------------------------------------ prepare --------

__global__ void finite_check_kernel(const float* x, uint64_t n, uint32_t width, uint32_t d,
                                    unsigned long long* first_bad) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n * d;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t r = i / d, j = i % d;
    if (!isfinite(x[r * width + j])) atomicMin(first_bad, (unsigned long long)(r * width + j));
  }
}

// Column sums, minima and maxima of the leading d components, per chunk of kMeanRows
// rows (4 row classes of 64 column threads, combined in a fixed order), then over the
// chunks in order (column_finish_kernel): the same bits on every run.
constexpr uint32_t kMeanRows = 2048;

__global__ void __launch_bounds__(256)
column_partial_kernel(const float* x, uint64_t n, uint32_t width, uint32_t d, double* part_sum,
                      float* part_lo, float* part_hi) {
  __shared__ double ss[4][64];
  __shared__ float sl[4][64], sh[4][64];
  const uint32_t j = threadIdx.x & 63u, g = threadIdx.x >> 6;
  const uint64_t r0 = blockIdx.x * (uint64_t)kMeanRows;
  const uint64_t r1 = r0 + kMeanRows < n ? r0 + kMeanRows : n;
  double sum = 0.0;
  float lo = INFINITY, hi = -INFINITY;
  if (j < d)
    for (uint64_t r = r0 + g; r < r1; r += 4) {
      const float v = x[r * width + j];
      sum = __dadd_rn(sum, (double)v);
      lo = fminf(lo, v);
      hi = fmaxf(hi, v);
    }
  ss[g][j] = sum;
  sl[g][j] = lo;
  sh[g][j] = hi;
  __syncthreads();
  if (g == 0 && j < d) {
    part_sum[blockIdx.x * 64ull + j] =
        __dadd_rn(__dadd_rn(ss[0][j], ss[1][j]), __dadd_rn(ss[2][j], ss[3][j]));
    part_lo[blockIdx.x * 64ull + j] = fminf(fminf(sl[0][j], sl[1][j]), fminf(sl[2][j], sl[3][j]));
    part_hi[blockIdx.x * 64ull + j] = fmaxf(fmaxf(sh[0][j], sh[1][j]), fmaxf(sh[2][j], sh[3][j]));
  }
}

// mean[j] (f64) and, for the first three components, the range of the centred values
// f32(x - mean) (that map is monotonic, so the range is the centred raw range).
__global__ void column_finish_kernel(const double* part_sum, const float* part_lo,
                                     const float* part_hi, uint32_t n_parts, uint64_t n,
                                     uint32_t d, double* mean, float* lo_hi) {
  const uint32_t j = threadIdx.x;
  if (j >= d) return;
  double sum = 0.0;
  float lo = INFINITY, hi = -INFINITY;
  for (uint32_t b = 0; b < n_parts; ++b) {
    sum = __dadd_rn(sum, part_sum[b * 64ull + j]);
    lo = fminf(lo, part_lo[b * 64ull + j]);
    hi = fmaxf(hi, part_hi[b * 64ull + j]);
  }
  const double m = sum / (double)n;
  mean[j] = m;
  if (j < 3) {
    lo_hi[2 * j] = (float)((double)lo - m);
    lo_hi[2 * j + 1] = (float)((double)hi - m);
  }
}

void column_stats(const float* x, uint64_t n, uint32_t width, uint32_t d, double* mean,
                  float* lo_hi, cudaStream_t s) {
  const uint32_t parts = (uint32_t)((n + kMeanRows - 1) / kMeanRows);
  DeviceBuffer<double> sum(parts * 64ull, s);
  DeviceBuffer<float> lo(parts * 64ull, s), hi(parts * 64ull, s);
  column_partial_kernel<<<parts, 256, 0, s>>>(x, n, width, d, sum.ptr, lo.ptr, hi.ptr);
  KG_LAUNCH_CHECK();
  column_finish_kernel<<<1, 64, 0, s>>>(sum.ptr, lo.ptr, hi.ptr, parts, n, d, mean, lo_hi);
  KG_LAUNCH_CHECK();
}

// Centred f32 rows padded to kDim (zeros), their f32 squared norms and f64 squares.
__global__ void centre_kernel(const float* x, uint64_t n, uint32_t width, uint32_t d,
                              const double* mean, float* rows, float* offsets,
                              double* squares) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  double s = 0.0;
  for (uint32_t j = 0; j < kDim; ++j) {
    float c = 0.0f;
    if (j < d) c = (float)__dadd_rn((double)x[r * width + j], -mean[j]);
    rows[r * kDim + j] = c;
    s = __dadd_rn(s, __dmul_rn((double)c, (double)c));
  }
  squares[r] = s;
  offsets[r] = (float)s;
}

// *out = max(*out, max of v): v >= 0 (squared norms), so the f64 bit patterns order as
// the values do and one atomicMax per warp combines the blocks (*out starts at 0).
__global__ void max_kernel(const double* v, uint64_t n, unsigned long long* out) {
  unsigned long long m = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v[i]);
    m = b > m ? b : m;
  }
  for (int o = 16; o; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xFFFFFFFFu, m, o);
    m = t > m ? t : m;
  }
  if ((threadIdx.x & 31u) == 0) atomicMax(out, m);
}

__device__ __forceinline__ uint32_t spread3(uint32_t v) {  // 10 bits -> every third bit
  v &= 0x3FFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__device__ __forceinline__ uint32_t morton_code(const float* xr, uint32_t dims,
                                                const double* mean, const float* lo_hi) {
  uint32_t code = 0;
  for (uint32_t j = 0; j < dims; ++j) {
    float v = (float)((double)xr[j] - mean[j]);
    float span = lo_hi[2 * j + 1] - lo_hi[2 * j];
    float t = span > 0.0f ? (v - lo_hi[2 * j]) / span : 0.0f;
    uint32_t q = (uint32_t)fminf(fmaxf(t * 1023.0f, 0.0f), 1023.0f);
    code |= spread3(q) << j;
  }
  return code;
}

__global__ void morton_kernel(const float* x, uint64_t n, uint32_t width, uint32_t dims,
                              const double* mean, const float* lo_hi, uint32_t* key,
                              uint32_t* row) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  key[r] = morton_code(x + r * width, dims, mean, lo_hi);
  row[r] = (uint32_t)r;
}

// The batch's order key: the row's sample, then its Morton code.
__global__ void batch_morton_kernel(const float* x, uint64_t n, uint32_t width, uint32_t dims,
                                    const double* mean, const float* lo_hi,
                                    const uint32_t* row_sample, unsigned long long* key,
                                    uint32_t* row) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  key[r] = ((unsigned long long)row_sample[r] << 32) | morton_code(x + r * width, dims, mean, lo_hi);
  row[r] = (uint32_t)r;
}

// Per query slot its sample (the batch's order is sample-major).
__global__ void slot_sample_kernel(const uint32_t* qrows, const uint32_t* row_sample, uint64_t n,
                                  uint32_t* slot_sample) {
  uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (q < n) slot_sample[q] = row_sample[qrows[q]];
}

// A batch's tile lists: the block of query slots [qb * block, ...) scans the point tiles
// of the samples it holds (a contiguous range, the samples being contiguous in slot
// order), from its own tile on, wrapping inside the range. len pass (list NULL) or fill.
__global__ void batch_lists_kernel(const uint32_t* slot_sample, const uint64_t* sample_first,
                                   uint64_t n, uint32_t block, uint64_t n_blocks,
                                   uint64_t* len, const uint64_t* off, uint32_t* list) {
  const uint64_t qb = blockIdx.x;
  if (qb >= n_blocks) return;
  const uint64_t q0 = qb * block, q1 = (q0 + block < n ? q0 + block : n) - 1;
  const uint64_t p0 = sample_first[slot_sample[q0]], p1 = sample_first[slot_sample[q1] + 1];
  const uint32_t t0 = (uint32_t)(p0 / 128), t1 = (uint32_t)((p1 - 1) / 128);
  const uint32_t count = t1 - t0 + 1;
  if (!list) {
    if (threadIdx.x == 0) len[qb] = count;
    return;
  }
  const uint32_t own = min(max((uint32_t)(q0 / 128), t0), t1);
  for (uint32_t i = threadIdx.x; i < count; i += blockDim.x)
    list[off[qb] + i] = t0 + (own - t0 + i) % count;
}

// The rows in Morton order of their first (up to) three centred components: nearby rows
// end up in nearby tiles. Any order gives the same graph; this one makes the filter's
// threshold tight early.
void spatial_order(const float* x, uint64_t n, uint32_t width, uint32_t d, const double* mean,
                   const float* lo_hi, DeviceBuffer<uint32_t>& perm, cudaStream_t s) {
  uint32_t dims = d < 3 ? d : 3;
  DeviceBuffer<uint32_t> key(n, s), key_sorted(n, s), rows(n, s);
  morton_kernel<<<blocks_for(n, 256), 256, 0, s>>>(x, n, width, dims, mean, lo_hi, key.ptr,
                                                   rows.ptr);
  KG_LAUNCH_CHECK();
  perm.alloc(n, s);
  size_t temp = 0;
  KG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, key.ptr, key_sorted.ptr, rows.ptr,
                                          perm.ptr, (int)n, 0, 30, s));
  DeviceBuffer<unsigned char> scratch(temp, s);
  KG_CUDA(cub::DeviceRadixSort::SortPairs(scratch.ptr, temp, key.ptr, key_sorted.ptr, rows.ptr,
                                          perm.ptr, (int)n, 0, 30, s));
}

// ------------------------------------------------------ bounded scan lists ---------
// The rows ordered by k-means part, so a block of query slots and a tile of point slots
// each hold rows close together in all d components; every query block's list holds every
// tile, nearest first, each with a lower bound on the distance between its rows and the
// block's (two balls). The filter skips a tile whose bound exceeds every query's threshold:
// no row in it can pass, so the graph is the same as the full scan's.

// Centre (the f64 mean of the group's centred rows), radius (the largest distance of a
// group row from it, rounded up) and box (each component's smallest and largest centred
// value) of each group of `size` consecutive slots; component j of group g is written at
// g * g_stride + j * j_stride of each per-component array (component-major: g_stride 1,
// j_stride n_groups; group-major: 64 and 1). One 64-thread block per group.
__global__ void __launch_bounds__(64)
group_balls_kernel(const float* x, uint32_t width, uint32_t d, const double* mean,
                   const uint32_t* rows, uint64_t n, uint32_t size, uint64_t g_stride,
                   uint64_t j_stride, double* centre_t, double* lo_t, double* hi_t,
                   double* radius) {
  const uint64_t g = blockIdx.x;
  const uint64_t s0 = g * size, s1 = min(s0 + size, n);
  __shared__ double c[kDim];
  __shared__ double red[64];
  const uint32_t j = threadIdx.x;
  double lo = 0.0, hi = 0.0;
  if (j < d) {
    double sum = 0.0;
    lo = INFINITY;
    hi = -INFINITY;
    for (uint64_t sl = s0; sl < s1; ++sl) {
      const double v = (double)x[(uint64_t)rows[sl] * width + j] - mean[j];
      sum += v;
      lo = fmin(lo, v);
      hi = fmax(hi, v);
    }
    c[j] = sum / (double)(s1 - s0);
  }
  __syncthreads();
  double worst = 0.0;
  for (uint64_t sl = s0 + threadIdx.x; sl < s1; sl += blockDim.x) {
    const float* xr = x + (uint64_t)rows[sl] * width;
    double acc = 0.0;
    for (uint32_t jj = 0; jj < d; ++jj) {
      const double t = ((double)xr[jj] - mean[jj]) - c[jj];
      acc += t * t;
    }
    worst = fmax(worst, acc);
  }
  red[threadIdx.x] = worst;
  __syncthreads();
  for (int o = 32; o; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) radius[g] = sqrt(red[0]) * (1.0 + 0x1p-40);
  const uint64_t at = g * g_stride + (uint64_t)j * j_stride;
  centre_t[at] = j < d ? c[j] : 0.0;
  lo_t[at] = lo;
  hi_t[at] = hi;
}

// Per (query block, tile), two lower bounds on the distance between a row of the block
// and a row of the tile: the balls' |c_b - c_t| - r_b - r_t (triangle inequality) and the
// boxes' sqrt(sum_j gap_j^2) (gap_j: how far apart the two boxes are in component j). The
// larger, less a margin for the rounding of the centred rows and at least 0, is kept as a
// scaled squared distance rounded down, packed with the centre distance into the sort key
// (bound, then centre distance); the tile as the value. kBoundBlocks query blocks per CTA
// share each tile's reads.
constexpr int kBoundBlocks = 8;
__global__ void __launch_bounds__(256)
ball_bounds_kernel(const double* bc_t, const double* blo_t, const double* bhi_t,
                   const double* br, uint64_t n_blocks, const double* tc_t, const double* tlo_t,
                   const double* thi_t, const double* tr, uint32_t n_tiles, uint32_t d,
                   double s2, double margin, unsigned long long* key, uint32_t* tile) {
  __shared__ double cb[kBoundBlocks][kDim], lb_[kBoundBlocks][kDim], hb[kBoundBlocks][kDim];
  const uint64_t b0 = (uint64_t)blockIdx.x * kBoundBlocks;
  for (uint32_t i = threadIdx.x; i < kBoundBlocks * kDim; i += blockDim.x) {
    const uint32_t bb = i / kDim, j = i % kDim;
    const bool in = b0 + bb < n_blocks && j < d;
    const uint64_t at = (uint64_t)j * n_blocks + b0 + bb;
    cb[bb][j] = in ? bc_t[at] : 0.0;
    lb_[bb][j] = in ? blo_t[at] : 0.0;
    hb[bb][j] = in ? bhi_t[at] : 0.0;
  }
  __syncthreads();
  double rb[kBoundBlocks];
#pragma unroll
  for (int bb = 0; bb < kBoundBlocks; ++bb) rb[bb] = b0 + bb < n_blocks ? br[b0 + bb] : 0.0;
  for (uint32_t t = threadIdx.x; t < n_tiles; t += blockDim.x) {
    double acc[kBoundBlocks], box[kBoundBlocks];
#pragma unroll
    for (int bb = 0; bb < kBoundBlocks; ++bb) acc[bb] = box[bb] = 0.0;
    for (uint32_t j = 0; j < d; ++j) {
      const uint64_t at = (uint64_t)j * n_tiles + t;
      const double v = tc_t[at], tl = tlo_t[at], th = thi_t[at];
#pragma unroll
      for (int bb = 0; bb < kBoundBlocks; ++bb) {
        const double u = cb[bb][j] - v;
        acc[bb] = fma(u, u, acc[bb]);
        const double gap = fmax(fmax(tl - hb[bb][j], lb_[bb][j] - th), 0.0);
        box[bb] = fma(gap, gap, box[bb]);
      }
    }
    const double rt = tr[t];
#pragma unroll
    for (int bb = 0; bb < kBoundBlocks; ++bb) {
      if (b0 + bb >= n_blocks) break;
      const double dist = sqrt(acc[bb]);
      const double ball = dist * (1.0 - 0x1p-40) - rb[bb] - rt;
      const double boxd = sqrt(box[bb]) * (1.0 - 0x1p-40);
      const double lb = fmax(fmax(ball, boxd) - margin, 0.0);
      const float lb2 = __double2float_rd(s2 * lb * lb * (1.0 - 0x1p-40));
      const float near = __double2float_rn(dist);
      const uint64_t at = (b0 + bb) * (uint64_t)n_tiles + t;
      key[at] = ((unsigned long long)__float_as_uint(lb2) << 32) | __float_as_uint(near);
      tile[at] = t;
    }
  }
}

__global__ void key_bounds_kernel(const unsigned long long* key, uint64_t count, float* lb2) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
       i += (uint64_t)gridDim.x * blockDim.x)
    lb2[i] = __uint_as_float((uint32_t)(key[i] >> 32));
}

// The bounded scan of the exact search (qrows, list_tiles, list_lb2, list_stride,
// list_sorted of sp): rows by k-means part (about 1,024 rows a part); bounds with
// skipping when `skip`, else the same lists without bounds. Returns false (sp untouched)
// when the lists would not fit the sort's 32-bit sizes or `max_bytes` of scratch.
bool bounded_scan(const float* x, uint64_t n, uint32_t width, uint32_t d, const double* mean,
                  double scale, double max_norm, uint32_t qblock, bool skip, uint64_t max_bytes,
                  ScanPlan& sp, cudaStream_t s, Trace& trace) {
  const uint64_t n_blocks = (n + qblock - 1) / qblock;
  const uint32_t n_tiles = (uint32_t)((n + kTile - 1) / kTile);
  const uint64_t entries = n_blocks * n_tiles;
  if (entries > (uint64_t)INT32_MAX || entries * 28 > max_bytes) return false;
  Clusters cl;
  const uint32_t parts = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(n / 1024, 1), 4096);
  cluster_rows(x, n, width, d, parts, 5, 131072, cl, s);
  trace.mark("scan parts");
  DeviceBuffer<double> bc((uint64_t)kDim * n_blocks, s), blo((uint64_t)kDim * n_blocks, s),
      bhi((uint64_t)kDim * n_blocks, s), br(n_blocks, s);
  DeviceBuffer<double> tc((uint64_t)kDim * n_tiles, s), tlo((uint64_t)kDim * n_tiles, s),
      thi((uint64_t)kDim * n_tiles, s), tr(n_tiles, s);
  group_balls_kernel<<<(unsigned)n_blocks, 64, 0, s>>>(x, width, d, mean, cl.perm.ptr, n, qblock,
                                                       1, n_blocks, bc.ptr, blo.ptr, bhi.ptr,
                                                       br.ptr);
  KG_LAUNCH_CHECK();
  group_balls_kernel<<<n_tiles, 64, 0, s>>>(x, width, d, mean, cl.perm.ptr, n, kTile, 1, n_tiles,
                                            tc.ptr, tlo.ptr, thi.ptr, tr.ptr);
  KG_LAUNCH_CHECK();
  DeviceBuffer<unsigned long long> key(entries, s), key_sorted(entries, s);
  DeviceBuffer<uint32_t> tile(entries, s);
  sp.list_tiles.alloc(entries, s);
  // Margin: the centred rows' f64 rounding, far below any bound that prunes.
  const double margin = 0x1p-30 * max_norm;
  ball_bounds_kernel<<<(unsigned)((n_blocks + kBoundBlocks - 1) / kBoundBlocks), 256, 0, s>>>(
      bc.ptr, blo.ptr, bhi.ptr, br.ptr, n_blocks, tc.ptr, tlo.ptr, thi.ptr, tr.ptr, n_tiles, d,
      scale * scale, margin, key.ptr, tile.ptr);
  KG_LAUNCH_CHECK();
  trace.mark("scan bounds");
  DeviceBuffer<int> off(n_blocks + 1, s);
  std::vector<int> h_off(n_blocks + 1);
  for (uint64_t b = 0; b <= n_blocks; ++b) h_off[b] = (int)(b * n_tiles);
  KG_CUDA(cudaMemcpyAsync(off.ptr, h_off.data(), (n_blocks + 1) * sizeof(int),
                          cudaMemcpyHostToDevice, s));
  size_t temp = 0;
  KG_CUDA(cub::DeviceSegmentedSort::StableSortPairs(
      nullptr, temp, key.ptr, key_sorted.ptr, tile.ptr, sp.list_tiles.ptr, (int)entries,
      (int)n_blocks, off.ptr, off.ptr + 1, s));
  DeviceBuffer<unsigned char> scratch(temp, s);
  KG_CUDA(cub::DeviceSegmentedSort::StableSortPairs(
      scratch.ptr, temp, key.ptr, key_sorted.ptr, tile.ptr, sp.list_tiles.ptr, (int)entries,
      (int)n_blocks, off.ptr, off.ptr + 1, s));
  if (skip) {
    sp.list_lb2.alloc(entries, s);
    key_bounds_kernel<<<std::min<uint64_t>(blocks_for(entries, 256), 8192), 256, 0, s>>>(
        key_sorted.ptr, entries, sp.list_lb2.ptr);
    KG_LAUNCH_CHECK();
  }
  // The host offsets must outlive the copy.
  KG_CUDA(cudaStreamSynchronize(s));
  sp.qrows = std::move(cl.perm);
  sp.list_stride = n_tiles;
  sp.list_sorted = true;
  return true;
}

// The bounds of a given CSR of lists (block b's tiles at list_tiles[off[b] .. off[b + 1])):
// one CTA per block (its ball and box in shared memory), a warp per entry reading the
// tile's group-major ball and box; the same bound and sort key as ball_bounds_kernel.
__global__ void __launch_bounds__(256)
list_bounds_kernel(const uint64_t* off, const uint32_t* list_tiles, const double* bc,
                   const double* blo, const double* bhi, const double* br, const double* tc,
                   const double* tlo, const double* thi, const double* tr, uint32_t d, double s2,
                   double margin, unsigned long long* key) {
  __shared__ double cb[kDim], lb_[kDim], hb[kDim];
  const uint64_t b = blockIdx.x;
  for (uint32_t j = threadIdx.x; j < kDim; j += blockDim.x) {
    const bool in = j < d;
    cb[j] = in ? bc[b * kDim + j] : 0.0;
    lb_[j] = in ? blo[b * kDim + j] : 0.0;
    hb[j] = in ? bhi[b * kDim + j] : 0.0;
  }
  __syncthreads();
  const double rb = br[b];
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  for (uint64_t i = off[b] + warp; i < off[b + 1]; i += warps) {
    const uint32_t t = list_tiles[i];
    double acc = 0.0, box = 0.0;
    for (uint32_t j = lane; j < d; j += 32) {
      const uint64_t at = (uint64_t)t * kDim + j;
      const double u = cb[j] - tc[at];
      acc = fma(u, u, acc);
      const double gap = fmax(fmax(tlo[at] - hb[j], lb_[j] - thi[at]), 0.0);
      box = fma(gap, gap, box);
    }
    for (int o = 16; o; o >>= 1) {
      acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
      box += __shfl_xor_sync(0xFFFFFFFFu, box, o);
    }
    if (lane == 0) {
      const double dist = sqrt(acc);
      const double ball = dist * (1.0 - 0x1p-40) - rb - tr[t];
      const double boxd = sqrt(box) * (1.0 - 0x1p-40);
      const double lb = fmax(fmax(ball, boxd) - margin, 0.0);
      const float lb2 = __double2float_rd(s2 * lb * lb * (1.0 - 0x1p-40));
      key[i] = ((unsigned long long)__float_as_uint(lb2) << 32) |
               __float_as_uint(__double2float_rn(dist));
    }
  }
}

// Bounds for a plan's own CSR lists (the learned form's probe lists): each entry's bound
// as in bounded_scan, each block's list sorted by (bound, centre distance), skipping on.
// Leaves sp untouched when the lists exceed the sort's 32-bit sizes.
void bound_lists(const float* x, uint64_t n_q, uint64_t n_p, uint32_t width, uint32_t d,
                 const double* mean, double scale, double max_norm, uint32_t qblock,
                 ScanPlan& sp, cudaStream_t s) {
  const uint64_t n_blocks = (n_q + qblock - 1) / qblock;
  const uint32_t n_tiles = (uint32_t)((n_p + kTile - 1) / kTile);
  uint64_t entries = 0;
  KG_CUDA(cudaMemcpyAsync(&entries, sp.list_off.ptr + n_blocks, 8, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  if (!entries || entries > (uint64_t)INT32_MAX) return;
  const uint32_t* prows = sp.prows.ptr ? sp.prows.ptr : sp.qrows.ptr;
  DeviceBuffer<double> bc((uint64_t)kDim * n_blocks, s), blo((uint64_t)kDim * n_blocks, s),
      bhi((uint64_t)kDim * n_blocks, s), br(n_blocks, s);
  DeviceBuffer<double> tc((uint64_t)kDim * n_tiles, s), tlo((uint64_t)kDim * n_tiles, s),
      thi((uint64_t)kDim * n_tiles, s), tr(n_tiles, s);
  group_balls_kernel<<<(unsigned)n_blocks, 64, 0, s>>>(x, width, d, mean, sp.qrows.ptr, n_q,
                                                       qblock, kDim, 1, bc.ptr, blo.ptr, bhi.ptr,
                                                       br.ptr);
  KG_LAUNCH_CHECK();
  group_balls_kernel<<<n_tiles, 64, 0, s>>>(x, width, d, mean, prows, n_p, kTile, kDim, 1, tc.ptr,
                                            tlo.ptr, thi.ptr, tr.ptr);
  KG_LAUNCH_CHECK();
  DeviceBuffer<unsigned long long> key(entries, s), key_sorted(entries, s);
  list_bounds_kernel<<<(unsigned)n_blocks, 256, 0, s>>>(
      sp.list_off.ptr, sp.list_tiles.ptr, bc.ptr, blo.ptr, bhi.ptr, br.ptr, tc.ptr, tlo.ptr,
      thi.ptr, tr.ptr, d, scale * scale, 0x1p-30 * max_norm, key.ptr);
  KG_LAUNCH_CHECK();
  std::vector<uint64_t> h_off(n_blocks + 1);
  KG_CUDA(cudaMemcpyAsync(h_off.data(), sp.list_off.ptr, (n_blocks + 1) * 8,
                          cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  std::vector<int> h_ioff(n_blocks + 1);
  for (uint64_t b = 0; b <= n_blocks; ++b) h_ioff[b] = (int)h_off[b];
  DeviceBuffer<int> ioff(n_blocks + 1, s);
  KG_CUDA(cudaMemcpyAsync(ioff.ptr, h_ioff.data(), (n_blocks + 1) * sizeof(int),
                          cudaMemcpyHostToDevice, s));
  DeviceBuffer<uint32_t> tiles_sorted(entries, s);
  size_t temp = 0;
  KG_CUDA(cub::DeviceSegmentedSort::StableSortPairs(
      nullptr, temp, key.ptr, key_sorted.ptr, sp.list_tiles.ptr, tiles_sorted.ptr, (int)entries,
      (int)n_blocks, ioff.ptr, ioff.ptr + 1, s));
  DeviceBuffer<unsigned char> scratch(temp, s);
  KG_CUDA(cub::DeviceSegmentedSort::StableSortPairs(
      scratch.ptr, temp, key.ptr, key_sorted.ptr, sp.list_tiles.ptr, tiles_sorted.ptr,
      (int)entries, (int)n_blocks, ioff.ptr, ioff.ptr + 1, s));
  sp.list_lb2.alloc(entries, s);
  key_bounds_kernel<<<std::min<uint64_t>(blocks_for(entries, 256), 8192), 256, 0, s>>>(
      key_sorted.ptr, entries, sp.list_lb2.ptr);
  KG_LAUNCH_CHECK();
  // The host offsets must outlive the copy.
  KG_CUDA(cudaStreamSynchronize(s));
  sp.list_tiles = std::move(tiles_sorted);
  sp.list_sorted = true;
}

// The batch's rows sample by sample, each sample in Morton order: a query block's own
// tiles hold its nearest points, and each sample's rows are one contiguous slot range.
void batch_order(const float* x, uint64_t n, uint32_t width, uint32_t d, const double* mean,
                 const float* lo_hi, const KnnBatch& batch, DeviceBuffer<uint32_t>& perm,
                 cudaStream_t s) {
  uint32_t dims = d < 3 ? d : 3;
  DeviceBuffer<unsigned long long> key(n, s), key_sorted(n, s);
  DeviceBuffer<uint32_t> rows(n, s);
  batch_morton_kernel<<<blocks_for(n, 256), 256, 0, s>>>(x, n, width, dims, mean, lo_hi,
                                                         batch.row_sample.ptr, key.ptr, rows.ptr);
  KG_LAUNCH_CHECK();
  perm.alloc(n, s);
  int end_bit = 32;
  while (end_bit < 64 && (1ull << (end_bit - 32)) < batch.first.size()) ++end_bit;
  size_t temp = 0;
  KG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, key.ptr, key_sorted.ptr, rows.ptr,
                                          perm.ptr, (int)n, 0, end_bit, s));
  DeviceBuffer<unsigned char> scratch(temp, s);
  KG_CUDA(cub::DeviceRadixSort::SortPairs(scratch.ptr, temp, key.ptr, key_sorted.ptr, rows.ptr,
                                          perm.ptr, (int)n, 0, end_bit, s));
}

// *out = the largest of v[0..n) (all >= 0), on the stream.
void max_kernel_launch(const double* v, uint64_t n, double* out, cudaStream_t s) {
  KG_CUDA(cudaMemsetAsync(out, 0, sizeof(double), s));
  unsigned blocks = std::min<unsigned>(blocks_for(n, 256), 1184);
  max_kernel<<<blocks, 256, 0, s>>>(v, n, reinterpret_cast<unsigned long long*>(out));
  KG_LAUNCH_CHECK();
}

// kyto's slack E_q = 2 (w + 8) u (|a_q| + max |a|)^2 + 4 (w + 8) FLT_MIN
// (neighbors_exact.rs:80-95, 114-136).
__global__ void slack_kernel(const double* squares, uint64_t n, uint32_t d,
                             const double* largest_sq, double* slack) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  double u = 1.0 / 16777216.0;
  double factor = 2.0 * ((double)d + 8.0) * u;
  double underflow = 4.0 * ((double)d + 8.0) * (double)FLT_MIN;
  double a = sqrt(squares[r]) + sqrt(*largest_sq);
  slack[r] = factor * a * a + underflow;
}

// ------------------------------------------------------------------ filter ---------

__device__ __forceinline__ float round_up_f32(double v) {
  float r = (float)v;
  if ((double)r < v) r = nextafterf(r, INFINITY);
  return r;
}

// One thread per query: its centred row in registers, point tiles of kTile rows
// staged in shared memory. Each query's k smallest approximate keys live in local
// memory; candidates go to its own slice of the candidate buffer (kyto's Query::offer,
// neighbors_exact.rs:216-255), compacted against the falling threshold when full.
__global__ void __launch_bounds__(kFilterThreads)
filter_kernel(const float* __restrict__ rows, const float* __restrict__ offsets,
              const double* __restrict__ slack, uint64_t n, uint64_t q_begin,
              uint64_t q_end, uint32_t k, uint32_t cap, float* cand_key, uint32_t* cand_row,
              uint32_t* cand_count, float* threshold_out) {
  __shared__ float tile[kTile * kDim];
  __shared__ float tile_off[kTile];
  uint64_t q = q_begin + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  bool active = q < q_end;
  float qv[kDim];
#pragma unroll
  for (int j = 0; j < kDim; ++j) qv[j] = active ? rows[q * kDim + j] : 0.0f;
  float off_q = active ? offsets[q] : 0.0f;
  double sl = active ? slack[q] : 0.0;
  float smallest[kMaxK];
  uint32_t n_small = 0;
  float threshold = INFINITY;
  uint64_t slot = (q - q_begin) * (uint64_t)cap;
  uint32_t count = 0, compact_at = 64;
  bool overflowed = false;
  for (uint64_t p0 = 0; p0 < n; p0 += kTile) {
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kTile * kDim; i += blockDim.x) {
      uint64_t p = p0 + i / kDim;
      tile[i] = p < n ? rows[p0 * kDim + i] : 0.0f;
    }
    for (uint32_t i = threadIdx.x; i < kTile; i += blockDim.x)
      tile_off[i] = p0 + i < n ? offsets[p0 + i] : INFINITY;
    __syncthreads();
    if (!active || overflowed) continue;
    uint32_t span = (uint32_t)((n - p0) < kTile ? (n - p0) : kTile);
    for (uint32_t c = 0; c < span; ++c) {
      const float* pv = &tile[c * kDim];
      float dot = 0.0f;
#pragma unroll
      for (int j = 0; j < kDim; ++j) dot = fmaf(qv[j], pv[j], dot);
      float key = __fsub_rn(__fadd_rn(off_q, tile_off[c]), 2.0f * dot);
      uint64_t p = p0 + c;
      if (!(key <= threshold) || p == q) continue;
      if (n_small < k || key < smallest[k - 1]) {
        if (n_small < k) ++n_small;
        uint32_t at = n_small - 1;
        while (at > 0 && smallest[at - 1] > key) {
          smallest[at] = smallest[at - 1];
          --at;
        }
        smallest[at] = key;
        if (n_small == k) threshold = round_up_f32((double)smallest[k - 1] + 2.0 * sl);
      }
      if (key <= threshold) {
        if (count == cap) {
          overflowed = true;
          break;
        }
        cand_key[slot + count] = key;
        cand_row[slot + count] = (uint32_t)p;
        ++count;
        if (count >= compact_at) {
          uint32_t kept = 0;
          for (uint32_t i = 0; i < count; ++i) {
            float ck = cand_key[slot + i];
            if (ck <= threshold) {
              cand_key[slot + kept] = ck;
              cand_row[slot + kept] = cand_row[slot + i];
              ++kept;
            }
          }
          count = kept;
          if (count > kCandidateLimit) {
            overflowed = true;
            break;
          }
          compact_at = min(max(2 * count, 64u), cap);
        }
      }
    }
  }
  if (active) {
    cand_count[q - q_begin] = overflowed ? kOverflow : count;
    threshold_out[q - q_begin] = threshold;
  }
}

// ------------------------------------------------------------------ exact keys -----

// kyto's exact key (kernels.rs:420-448): component j's difference and square in f64
// into lane j % 8 (no FMA), the lanes combined by the fixed tree.
__device__ __forceinline__ double exact_key(const float* a, const float* b, uint32_t d) {
  double lanes[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (uint32_t j = 0; j < d; ++j) {
    double diff = __dsub_rn((double)a[j], (double)b[j]);
    lanes[j & 7] = __dadd_rn(lanes[j & 7], __dmul_rn(diff, diff));
  }
  double h0 = __dadd_rn(lanes[0], lanes[4]);
  double h1 = __dadd_rn(lanes[1], lanes[5]);
  double h2 = __dadd_rn(lanes[2], lanes[6]);
  double h3 = __dadd_rn(lanes[3], lanes[7]);
  return __dadd_rn(__dadd_rn(h0, h2), __dadd_rn(h1, h3));
}

__device__ __forceinline__ bool before(double ka, uint32_t ia, double kb, uint32_t ib) {
  return ka < kb || (ka == kb && ia < ib);
}

// Offer (key, row) to a ranked list of at most k entries (kyto's Nearest::offer).
__device__ __forceinline__ void offer(double* keys, uint32_t* idx, uint32_t& len, uint32_t k,
                                      double key, uint32_t row) {
  if (len == k) {
    if (before(keys[k - 1], idx[k - 1], key, row)) return;
    --len;
  }
  uint32_t at = len;
  while (at > 0 && before(key, row, keys[at - 1], idx[at - 1])) {
    keys[at] = keys[at - 1];
    idx[at] = idx[at - 1];
    --at;
  }
  keys[at] = key;
  idx[at] = row;
  ++len;
}

// Merge the warp's per-lane ranked lists into the first k of all: k rounds of a warp
// arg-min over the lanes' heads.
__device__ void warp_merge(const double* keys, const uint32_t* idx, uint32_t len, uint32_t k,
                           double* out_key, uint32_t* out_row, uint32_t* out_len) {
  unsigned lane = threadIdx.x & 31u;
  uint32_t head = 0;
  uint32_t produced = 0;
  for (uint32_t r = 0; r < k; ++r) {
    double hk = head < len ? keys[head] : INFINITY;
    uint32_t hi = head < len ? idx[head] : 0xFFFFFFFFu;
    bool has = head < len;
    double bk = hk;
    uint32_t bi = hi;
    unsigned bl = has ? lane : 32u;
    for (int o = 16; o; o >>= 1) {
      double ok = __shfl_xor_sync(0xFFFFFFFFu, bk, o);
      uint32_t oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
      unsigned ol = __shfl_xor_sync(0xFFFFFFFFu, bl, o);
      bool take = (ol < 32u) && (bl == 32u || before(ok, oi, bk, bi));
      if (take) {
        bk = ok;
        bi = oi;
        bl = ol;
      }
    }
    if (bl == 32u) break;
    if (lane == bl) ++head;
    if (lane == 0) {
      out_key[r] = bk;
      out_row[r] = bi;
    }
    ++produced;
  }
  if (lane == 0) *out_len = produced;
}

// One warp per query: exact keys of its candidates, the k best by (key, row). A row
// that overflowed, holds fewer than k candidates or has a candidate outside its slack
// is flagged for a full search (kyto's rank, neighbors_exact.rs:318-340).
// An approximate key a stands for the squared distance a * inv_s2 + qn2[q] (the
// tensor-core filter's keys are scaled and shifted by the query's norm; the SIMT
// filter's are distances already: inv_s2 = 1, qn2 = NULL).
// With `perm`, the filter ran on the rows in scan order: its query position qp and its
// candidates' rows are positions there, row perm[.] of x (ranks and outputs use x's).
__global__ void rank_kernel(const float* __restrict__ x, uint32_t width, uint32_t d,
                            uint64_t q_begin, uint64_t q_end, uint32_t k, uint32_t cap,
                            const float* cand_key, const uint32_t* cand_row,
                            const uint32_t* cand_count, const float* threshold,
                            const double* slack, double inv_s2, const double* qn2,
                            const uint32_t* qperm, const uint32_t* pperm, double* out_key,
                            uint32_t* out_row, uint32_t* full_flag,
                            unsigned long long* n_candidates) {
  uint64_t qi = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  uint64_t qp = q_begin + qi;
  if (qp >= q_end) return;
  uint64_t q = qperm ? qperm[qp] : qp;
  uint32_t count = cand_count[qi];
  if (count == kOverflow) {
    if (lane == 0) full_flag[q] = 1;
    return;
  }
  float th = threshold[qi];
  double sl = slack[qp];
  double shift = qn2 ? qn2[qp] : 0.0;
  const float* qrow = x + q * width;
  double keys[kMaxK];
  uint32_t idx[kMaxK];
  uint32_t len = 0;
  bool bad = false;
  uint32_t used = 0;
  for (uint32_t c = lane; c < count; c += 32) {
    float ak = cand_key[qi * (uint64_t)cap + c];
    if (ak > th) continue;
    uint32_t p = cand_row[qi * (uint64_t)cap + c];
    if (pperm) p = pperm[p];
    double e = exact_key(qrow, x + (uint64_t)p * width, d);
    if (fabs(e - ((double)ak * inv_s2 + shift)) > sl) bad = true;
    offer(keys, idx, len, k, e, p);
    ++used;
  }
  for (int o = 16; o; o >>= 1) used += __shfl_xor_sync(0xFFFFFFFFu, used, o);
  bool any_bad = __any_sync(0xFFFFFFFFu, bad);
  __shared__ uint32_t merged_len[kRankWarps];
  unsigned w = threadIdx.x >> 5;
  double* ok = out_key + q * (uint64_t)k;
  uint32_t* orow = out_row + q * (uint64_t)k;
  warp_merge(keys, idx, len, k, ok, orow, &merged_len[w]);
  __syncwarp();
  if (lane == 0) {
    atomicAdd(n_candidates, (unsigned long long)used);
    full_flag[q] = (any_bad || merged_len[w] != k) ? 1u : 0u;
  }
}

// One CTA per flagged row: every other row's exact key, the k best by (key, row).
// With a batch (row_sample), only the rows of the row's own sample.
__global__ void full_rows_kernel(const float* __restrict__ x, uint64_t n, uint32_t width,
                                 uint32_t d, uint32_t k, const uint32_t* rows_list,
                                 const uint32_t* row_sample, const uint64_t* sample_first,
                                 double* out_key, uint32_t* out_row) {
  uint64_t q = rows_list[blockIdx.x];
  const float* qrow = x + q * width;
  double keys[kMaxK];
  uint32_t idx[kMaxK];
  uint32_t len = 0;
  uint64_t lo = 0, hi = n;
  if (row_sample) {
    lo = sample_first[row_sample[q]];
    hi = sample_first[row_sample[q] + 1];
  }
  for (uint64_t p = lo + threadIdx.x; p < hi; p += blockDim.x) {
    if (p == q) continue;
    offer(keys, idx, len, k, exact_key(qrow, x + p * width, d), (uint32_t)p);
  }
  // Each warp merges its lanes; warp 0 then merges the warps' lists.
  __shared__ double wkeys[kFullWarps][kMaxK];
  __shared__ uint32_t wrow[kFullWarps][kMaxK];
  __shared__ uint32_t wlen[kFullWarps];
  unsigned w = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  warp_merge(keys, idx, len, k, wkeys[w], wrow[w], &wlen[w]);
  __syncthreads();
  if (w == 0) {
    uint32_t l2 = 0;
    if (lane < kFullWarps) {
      for (uint32_t i = 0; i < wlen[lane]; ++i) {
        keys[i] = wkeys[lane][i];
        idx[i] = wrow[lane][i];
      }
      l2 = wlen[lane];
    }
    __shared__ uint32_t final_len;
    warp_merge(keys, idx, l2, k, out_key + q * (uint64_t)k, out_row + q * (uint64_t)k,
               &final_len);
  }
}

// Each row's ranked entries sorted by row index, distances f32(sqrt(key))
// (neighbors.rs:412-435).
__global__ void graph_kernel(const double* keys, const uint32_t* rows, uint64_t n,
                             uint32_t k, uint64_t* indptr, uint32_t* indices,
                             float* distances) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r == 0) indptr[0] = 0;
  if (r >= n) return;
  indptr[r + 1] = (r + 1) * (uint64_t)k;
  const double* kr = keys + r * k;
  const uint32_t* rr = rows + r * k;
  uint32_t* oi = indices + r * k;
  float* od = distances + r * k;
  // Insertion by row index (k is small; rows are distinct).
  for (uint32_t i = 0; i < k; ++i) {
    uint32_t row = rr[i];
    float dist = (float)sqrt(kr[i]);
    uint32_t at = i;
    while (at > 0 && oi[at - 1] > row) {
      oi[at] = oi[at - 1];
      od[at] = od[at - 1];
      --at;
    }
    oi[at] = row;
    od[at] = dist;
  }
}

__global__ void compact_flags_kernel(const uint32_t* flag, uint64_t n, uint32_t* list,
                                     unsigned int* count) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r < n && flag[r]) list[atomicAdd(count, 1u)] = (uint32_t)r;
}

// Whether each query slot's candidates overflowed (1) or not (0).
__global__ void overflow_flags_kernel(const uint32_t* cand_count, uint64_t n, uint8_t* flag) {
  uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (q < n) flag[q] = cand_count[q] == kOverflow ? 1 : 0;
}

// Slots whose list does not cover their row: marked overflowed, so they are searched
// over every tile with the overflowed queries.
__global__ void force_overflow_kernel(const uint8_t* q_full, uint64_t n, uint32_t* cand_count) {
  const uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (q < n && q_full[q]) cand_count[q] = kOverflow;
}

// The retry's query slots: retry slot j is slot slots[j] of the first pass.
// The retry's query slots: `copies` copies of the m overflowed slots, each padded to mq
// slots (a whole number of query blocks) by repeating the last; copy c scans its own
// range of the point tiles.
__global__ void retry_slots_kernel(const uint32_t* slots, uint64_t m, uint64_t mq,
                                   uint32_t copies, const uint32_t* qrows,
                                   const uint32_t* q_point, const uint32_t* slot_sample,
                                   uint32_t* r_qrows, uint32_t* r_qpoint, uint32_t* r_sample) {
  uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (v >= mq * copies) return;
  const uint64_t j = v % mq;
  const uint32_t q = slots[j < m ? j : m - 1];
  r_qrows[v] = qrows[q];
  r_qpoint[v] = q_point ? q_point[q] : q;
  if (slot_sample) r_sample[v] = slot_sample[q];
}

// The retry's tile lists: block b = c * nb + j (copy c, query block j) scans the tiles
// [c * n_tiles / copies, (c + 1) * n_tiles / copies). One CTA per block.
__global__ void retry_lists_kernel(uint64_t nb, uint32_t copies, uint32_t n_tiles,
                                   uint64_t* off, uint32_t* list) {
  const uint64_t b = blockIdx.x;
  const uint64_t c = b / nb, j = b % nb;
  const uint32_t t0 = (uint32_t)(c * n_tiles / copies), t1 = (uint32_t)((c + 1) * n_tiles / copies);
  // The copies before c hold nb blocks of their own range each: nb * t0 entries.
  const uint64_t o = nb * (uint64_t)t0 + j * (uint64_t)(t1 - t0);
  if (threadIdx.x == 0) {
    off[b] = o;
    if (b + 1 == nb * copies) off[b + 1] = nb * (uint64_t)n_tiles;
  }
  for (uint32_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) list[o + (t - t0)] = t;
}

// One warp per overflowed query j: its copies' candidates merged into one slice of `cap`
// slots. The merged threshold is the smallest copy's: every copy kept each of its points
// whose key is at most its own threshold (at least the smallest), and the copy with the
// smallest threshold holds k keys below it; so the keys at most the smallest threshold,
// over all copies, are what one pass over every tile would keep. Any copy overflowed, or
// more than `cap` merged keys: the query overflows again.
__global__ void retry_merge_kernel(uint64_t m, uint64_t mq, uint32_t copies, uint32_t copy_cap,
                                   const float* key, const uint32_t* row, const uint32_t* count,
                                   const float* thr, uint32_t cap, float* m_key,
                                   uint32_t* m_row, uint32_t* m_count, float* m_thr) {
  const uint64_t j = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (j >= m) return;
  float th = INFINITY;
  bool over = false;
  for (uint32_t c = 0; c < copies; ++c) {
    const uint64_t v = c * mq + j;
    over |= count[v] == kOverflow;
    th = fminf(th, thr[v]);
  }
  uint32_t n_out = 0;
  const unsigned lt = (1u << lane) - 1u;
  for (uint32_t c = 0; c < copies && !over; ++c) {
    const uint64_t v = c * mq + j;
    const uint32_t cnt = count[v];
    for (uint32_t i0 = 0; i0 < cnt; i0 += 32) {
      const uint32_t i = i0 + lane;
      const float kk = i < cnt ? key[v * copy_cap + i] : INFINITY;
      const bool pass = i < cnt && kk <= th;
      const unsigned b = __ballot_sync(0xFFFFFFFFu, pass);
      const uint32_t at = n_out + (uint32_t)__popc(b & lt);
      if (pass && at < cap) {
        m_key[j * cap + at] = kk;
        m_row[j * cap + at] = row[v * copy_cap + i];
      }
      n_out += (uint32_t)__popc(b);
    }
  }
  if (lane == 0) {
    m_count[j] = over || n_out > cap ? kOverflow : n_out;
    m_thr[j] = th;
  }
}

namespace {

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s;
  explicit Timer(cudaStream_t st) : s(st) {
    KG_CUDA(cudaEventCreate(&a));
    KG_CUDA(cudaEventCreate(&b));
    KG_CUDA(cudaEventRecord(a, s));
  }
  double stop_ms() {
    KG_CUDA(cudaEventRecord(b, s));
    KG_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    KG_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
  }
  ~Timer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
  Timer(const Timer&) = delete;
  Timer& operator=(const Timer&) = delete;
};

}  // namespace

// ---------------------------------------------------------------- filter tuning ----

// The pilot's scan: pilot block i is block blocks[i] of the plan (its query slots, its
// tile list, or every tile from its own when the plan has none). len pass (list NULL)
// then fill; pilot query slot j of block i is plan slot blocks[i] * block + j.
__global__ void pilot_plan_kernel(const uint64_t* blocks, uint64_t n_pilot, uint32_t block,
                                  uint64_t n, const uint32_t* qrows, const uint32_t* q_point,
                                  const uint32_t* slot_sample, const uint32_t* list_tiles,
                                  const uint64_t* list_off, uint64_t list_stride,
                                  uint32_t n_tiles, uint64_t* len, const uint64_t* off,
                                  uint32_t* p_qrows, uint32_t* p_qpoint, uint32_t* p_sample,
                                  uint32_t* p_list) {
  const uint64_t i = blockIdx.x;
  if (i >= n_pilot) return;
  const uint64_t qb = blocks[i];
  uint64_t l0 = 0, count = n_tiles;
  if (list_tiles) {
    l0 = list_off ? list_off[qb] : qb * list_stride;
    count = list_off ? list_off[qb + 1] - l0 : list_stride;
  }
  if (!p_list) {
    if (threadIdx.x == 0) len[i] = count;
    return;
  }
  for (uint32_t j = threadIdx.x; j < block; j += blockDim.x) {
    const uint64_t src = qb * block + j, dst = i * block + j;
    if (src >= n) continue;
    p_qrows[dst] = qrows[src];
    p_qpoint[dst] = q_point ? q_point[src] : (uint32_t)src;
    if (slot_sample) p_sample[dst] = slot_sample[src];
  }
  const uint32_t own = (uint32_t)((qb * block / 128) % n_tiles);
  for (uint64_t t = threadIdx.x; t < count; t += blockDim.x)
    p_list[off[i] + t] = list_tiles ? list_tiles[l0 + t] : (uint32_t)((own + t) % n_tiles);
}

// The filter kind (fp16 or split operands) that ends the search soonest on this data,
// measured: each kind filters up to one query block per SM (blocks spread over the
// scan) against every point, and the estimate is its time scaled to all blocks plus its
// overflowed queries' full-row searches (1.65e-10 s per point and 50 components, as
// measured on B200). The kinds return the same graph, so the choice only moves time;
// it is kept per (rows, components, k) class for later calls in the process.
// The filter's tuned operand kind and query-operand mode (neither changes a result).
struct FilterChoice {
  FilterKind kind = FilterKind::Fp16;
  int a_mode = kTcAmSmem;
};

FilterChoice tune_filter_kind(kg_ctx* ctx, cudaStream_t s, const float* x, uint64_t n,
                              uint32_t width, uint32_t d, uint32_t k, const ScanPlan& sp,
                              const FilterScan& scan, const uint32_t* prows, const double* mean,
                              double scale, const double* max_sq) {
  // Two levels: this process's choices, then the cache file (kg_tune.cuh), keyed by the
  // GPU and the shape class (rows to the next power of two, components, k, and whether
  // the scan is a batch of samples).
  static std::mutex mu;
  static std::map<std::string, FilterChoice> cache;
  int n_bits = 0;
  while (n_bits < 63 && (1ull << n_bits) < n) ++n_bits;
  const std::string gpu = tune_gpu_name();
  const std::string cls = "knn_filter/n2^" + std::to_string(n_bits) + "/d" + std::to_string(d) +
                          "/k" + std::to_string(k) + (scan.slot_sample ? "/batch" : "");
  const std::string key = gpu + "|" + cls;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  const std::string path = tune_cache_path();
  const char* retune = std::getenv("KYTO_GPU_TUNE");
  TuneChoice tc;
  if (!(retune && std::string(retune) == "retune") && tune_lookup(path, gpu, cls, tc)) {
    FilterChoice c;
    c.kind = tc["kind"] == "split" ? FilterKind::Split
             : tc["kind"] == "bf16" ? FilterKind::Bf16 : FilterKind::Fp16;
    c.a_mode = tc["a_mode"] == "tmem" ? kTcAmTmem : tc["a_mode"] == "half" ? kTcAmHalf
                                                                           : kTcAmSmem;
    if (trace_on())
      std::fprintf(stderr, "[kyto_gpu trace] filter choice from %s: %s, %s\n", path.c_str(),
                   tc["kind"].c_str(), tc["a_mode"].c_str());
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = c;
    return c;
  }
  const uint32_t block = kTcQueryBlock;
  const uint64_t n_blocks = (n + block - 1) / block;
  const uint32_t n_tiles = (uint32_t)((n + 127) / 128);
  const uint64_t n_pilot = std::min<uint64_t>(n_blocks, (uint64_t)ctx->sm_count);
  std::vector<uint64_t> h_blocks(n_pilot);
  for (uint64_t i = 0; i < n_pilot; ++i) h_blocks[i] = i * n_blocks / n_pilot;
  DeviceBuffer<uint64_t> blocks(n_pilot, s), len(n_pilot + 1, s), off(n_pilot + 1, s);
  KG_CUDA(cudaMemcpyAsync(blocks.ptr, h_blocks.data(), n_pilot * 8, cudaMemcpyHostToDevice, s));
  pilot_plan_kernel<<<(unsigned)n_pilot, 256, 0, s>>>(
      blocks.ptr, n_pilot, block, n, sp.qrows.ptr, scan.q_point, scan.slot_sample,
      scan.list_tiles, scan.list_off, scan.list_stride, n_tiles, len.ptr, nullptr, nullptr,
      nullptr, nullptr, nullptr);
  KG_LAUNCH_CHECK();
  std::vector<uint64_t> h_off(n_pilot + 1, 0);
  KG_CUDA(cudaMemcpyAsync(h_off.data() + 1, len.ptr, n_pilot * 8, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  for (uint64_t i = 0; i < n_pilot; ++i) h_off[i + 1] += h_off[i];
  KG_CUDA(cudaMemcpyAsync(off.ptr, h_off.data(), (n_pilot + 1) * 8, cudaMemcpyHostToDevice, s));
  // Pilot slots past the last row (a partial last block) stay inactive: n_q stops there.
  const uint64_t last = h_blocks[n_pilot - 1];
  const uint64_t n_q = std::min<uint64_t>(n_pilot * block, (n_pilot - 1) * block + (n - last * block));
  DeviceBuffer<uint32_t> p_qrows(n_pilot * block, s), p_qpoint(n_pilot * block, s);
  DeviceBuffer<uint32_t> p_sample(scan.slot_sample ? n_pilot * block : 0, s);
  DeviceBuffer<uint32_t> p_list(std::max<uint64_t>(h_off[n_pilot], 1), s);
  pilot_plan_kernel<<<(unsigned)n_pilot, 256, 0, s>>>(
      blocks.ptr, n_pilot, block, n, sp.qrows.ptr, scan.q_point, scan.slot_sample,
      scan.list_tiles, scan.list_off, scan.list_stride, n_tiles, len.ptr, off.ptr, p_qrows.ptr,
      p_qpoint.ptr, p_sample.ptr, p_list.ptr);
  KG_LAUNCH_CHECK();
  FilterScan ps = scan;
  ps.n_q = n_q;
  ps.q_point = p_qpoint.ptr;
  ps.slot_sample = scan.slot_sample ? p_sample.ptr : nullptr;
  ps.list_tiles = p_list.ptr;
  ps.list_lb2 = nullptr;
  ps.list_sorted = false;
  ps.tiles_scanned = nullptr;
  ps.list_off = off.ptr;
  ps.list_stride = 0;
  const uint32_t cap = kTcCap;
  DeviceBuffer<float> ck(n_q * cap, s), th(n_q, s);
  DeviceBuffer<uint32_t> cr(n_q * cap, s), cc(n_q, s);
  DeviceBuffer<double> qn2(n_q, s), sl(n_q, s);
  const double per_point = 1.65e-10 * std::max<double>(d, 1) / 50.0;
  FilterChoice best;
  double best_cost = INFINITY;
  const std::pair<FilterKind, int> tries[] = {
      {FilterKind::Fp16, kTcAmSmem}, {FilterKind::Fp16, kTcAmHalf}, {FilterKind::Fp16, kTcAmTmem},
      {FilterKind::Split, kTcAmSmem}, {FilterKind::Split, kTcAmHalf}, {FilterKind::Split, kTcAmTmem}};
  for (const auto& tr : tries) {
    const FilterKind kind = tr.first;
    ps.a_mode = tr.second;
    cudaEvent_t a, b;
    KG_CUDA(cudaEventCreate(&a));
    KG_CUDA(cudaEventCreate(&b));
    KG_CUDA(cudaEventRecord(a, s));
    tc_filter(ctx, s, x, width, d, p_qrows.ptr, prows, ps, mean, scale, max_sq, kind, k, cap,
              ck.ptr, cr.ptr, cc.ptr, th.ptr, qn2.ptr, sl.ptr, nullptr);
    KG_CUDA(cudaEventRecord(b, s));
    KG_CUDA(cudaEventSynchronize(b));
    float ms = 0.0f;
    KG_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    std::vector<uint32_t> h_cc(n_q);
    KG_CUDA(cudaMemcpyAsync(h_cc.data(), cc.ptr, n_q * 4, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    uint64_t over = 0;
    for (uint32_t c : h_cc) over += c == kOverflow;
    const double cost = ms * 1e-3 * (double)n_blocks / (double)n_pilot +
                        (double)over / (double)n_q * (double)n * (double)n * per_point;
    if (trace_on())
      std::fprintf(stderr,
                   "[kyto_gpu trace] filter pilot %s/%s: %.3f ms for %llu blocks, %llu of %llu "
                   "queries overflowed, estimate %.1f ms\n",
                   kind == FilterKind::Split ? "split" : "fp16",
                   tr.second == kTcAmTmem ? "tmem" : tr.second == kTcAmHalf ? "half" : "smem", ms,
                   (unsigned long long)n_pilot, (unsigned long long)over,
                   (unsigned long long)n_q, cost * 1e3);
    if (cost < best_cost) {
      best_cost = cost;
      best.kind = kind;
      best.a_mode = tr.second;
    }
  }
  tune_store(path, gpu, cls,
             TuneChoice{{"kind", best.kind == FilterKind::Split ? "split" : "fp16"},
                        {"a_mode", best.a_mode == kTcAmTmem ? "tmem"
                                   : best.a_mode == kTcAmHalf ? "half" : "smem"}},
             best_cost * 1e3);
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = best;
  return best;
}

// The exact search on device rows: every row's k nearest other rows by (kyto key, row)
// into out.key / out.row (n x k). `plan` chooses the tensor-core filter's scan (NULL:
// the rows in a spatial order, each query block scanning every tile from its own).
void knn_core(kg_ctx* ctx, const float* x, uint64_t n, uint32_t width, uint32_t d, uint32_t k,
              const PlanBuilder* plan, KnnResult& out, Trace& trace, const KnnBatch* batch) {
  cudaStream_t s = ctx->stream;
  DeviceBuffer<double> mean(d, s), squares(n, s), slack(n, s), largest(1, s);
  DeviceBuffer<float> rows(n * kDim, s), offsets(n, s), lo_hi(6, s);
  column_stats(x, n, width, d, mean.ptr, lo_hi.ptr, s);
  centre_kernel<<<blocks_for(n, 128), 128, 0, s>>>(x, n, width, d, mean.ptr, rows.ptr,
                                                   offsets.ptr, squares.ptr);
  max_kernel_launch(squares.ptr, n, largest.ptr, s);
  slack_kernel<<<blocks_for(n, 256), 256, 0, s>>>(squares.ptr, n, d, largest.ptr, slack.ptr);
  KG_LAUNCH_CHECK();
  double h_largest = 0;
  KG_CUDA(cudaMemcpyAsync(&h_largest, largest.ptr, 8, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  bool brute = !std::isfinite(h_largest) || std::sqrt(h_largest) > 1e15;

  out.key.alloc(n * k, s);
  out.row.alloc(n * k, s);
  DeviceBuffer<uint32_t> full_flag(n, s);
  DeviceBuffer<unsigned long long> n_cand(1, s);
  n_cand.zero();
  double filter_ms = 0, rank_ms = 0;
  // The filter: the tensor-core GEMM (fp16, split fp16 hi/lo, or bf16 on request) when
  // the components and the three norm columns fit one 64-wide operand row; the SIMT
  // filter otherwise or on request (KYTO_GPU_KNN_FILTER=simt|fp16|split|bf16). All give
  // the same graph.
  const char* choice = std::getenv("KYTO_GPU_KNN_FILTER");
  std::string filter = choice ? choice : "auto";
  bool tc = !brute && d + 3 <= 64 &&
            (filter == "auto" || filter == "fp16" || filter == "bf16" || filter == "split");
  if (batch && !brute && !tc)
    fail(KG_ERR_INVALID, "batched neighbors: the tensor-core filter (at most 61 components)");
  FilterKind kind = filter == "bf16"    ? FilterKind::Bf16
                          : filter == "split" ? FilterKind::Split
                                              : FilterKind::Fp16;
  if (brute) {
    uint32_t one = 1;
    std::vector<uint32_t> all(n, one);
    KG_CUDA(cudaMemcpyAsync(full_flag.ptr, all.data(), n * 4, cudaMemcpyHostToDevice, s));
  } else if (tc) {
    check_cancel(ctx);
    const uint32_t cap = kTcCap;
    const size_t slice = (size_t)n * cap * 4;
    if (ctx->knn_ws.count < 2 * slice) {
      ctx->knn_ws.reset();
      ctx->knn_ws.alloc(2 * slice, s);
    }
    float* cand_key = reinterpret_cast<float*>(ctx->knn_ws.ptr);
    uint32_t* cand_row = reinterpret_cast<uint32_t*>(ctx->knn_ws.ptr + slice);
    DeviceBuffer<float> thr(n, s);
    DeviceBuffer<uint32_t> cand_count(n, s);
    DeviceBuffer<double> qn2(n, s), slack_d(n, s), max_sq(1, s);
    Timer tf(s);
    const double scale = tc_scale(x, n, width, d, mean.ptr, max_sq.ptr, s);
    ScanPlan sp;
    DeviceBuffer<uint32_t> slot_sample;
    if (plan) {
      (*plan)(x, n, width, d, scale, filter_query_block(kind), sp, trace);
      // Bounds for the plan's lists too (unless KYTO_GPU_KNN_ORDER=cluster or morton
      // asks for scans without skipping).
      const char* ord = std::getenv("KYTO_GPU_KNN_ORDER");
      if (sp.list_tiles.ptr && sp.list_off.ptr && !sp.list_lb2.ptr &&
          (!ord || std::string(ord) == "bounded")) {
        bound_lists(x, n, n, width, d, mean.ptr, scale, std::sqrt(h_largest),
                    filter_query_block(kind), sp, s);
        trace.mark("scan bounds");
      }
    } else if (batch) {
      // Samples one after another, each in Morton order; each query block scans the
      // tiles of the samples it holds.
      batch_order(x, n, width, d, mean.ptr, lo_hi.ptr, *batch, sp.qrows, s);
      slot_sample.alloc(n, s);
      slot_sample_kernel<<<blocks_for(n, 256), 256, 0, s>>>(sp.qrows.ptr, batch->row_sample.ptr,
                                                            n, slot_sample.ptr);
      KG_LAUNCH_CHECK();
      const uint32_t qblock = filter_query_block(kind);
      const uint64_t n_blocks = (n + qblock - 1) / qblock;
      DeviceBuffer<uint64_t> len(n_blocks + 1, s);
      len.zero();
      batch_lists_kernel<<<(unsigned)n_blocks, 128, 0, s>>>(
          slot_sample.ptr, batch->d_first.ptr, n, qblock, n_blocks, len.ptr, nullptr, nullptr);
      KG_LAUNCH_CHECK();
      sp.list_off.alloc(n_blocks + 1, s);
      size_t temp = 0;
      KG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, len.ptr, sp.list_off.ptr,
                                            n_blocks + 1, s));
      DeviceBuffer<unsigned char> scratch(temp, s);
      KG_CUDA(cub::DeviceScan::ExclusiveSum(scratch.ptr, temp, len.ptr, sp.list_off.ptr,
                                            n_blocks + 1, s));
      uint64_t total = 0;
      KG_CUDA(cudaMemcpyAsync(&total, sp.list_off.ptr + n_blocks, 8, cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaStreamSynchronize(s));
      sp.list_tiles.alloc(std::max<uint64_t>(total, 1), s);
      batch_lists_kernel<<<(unsigned)n_blocks, 128, 0, s>>>(slot_sample.ptr, batch->d_first.ptr,
                                                            n, qblock, n_blocks, len.ptr,
                                                            sp.list_off.ptr, sp.list_tiles.ptr);
      KG_LAUNCH_CHECK();
      trace.mark("scan order");
    } else {
      // By default the bounded scan (rows by k-means part, nearest tiles first, far tiles
      // skipped on their bounds); KYTO_GPU_KNN_ORDER=cluster keeps its order and lists
      // without skipping, =morton the rows sorted by a Morton code of their first three
      // centred components, each query block scanning every tile from its own (also
      // when the lists would not fit).
      const char* ord = std::getenv("KYTO_GPU_KNN_ORDER");
      const std::string order = ord ? ord : "bounded";
      bool listed = false;
      if (order != "morton") {
        size_t free_b = 0, total_b = 0;
        KG_CUDA(cudaMemGetInfo(&free_b, &total_b));
        listed = bounded_scan(x, n, width, d, mean.ptr, scale, std::sqrt(h_largest),
                              filter_query_block(kind), order != "cluster", free_b / 3, sp, s,
                              trace);
      }
      if (!listed) spatial_order(x, n, width, d, mean.ptr, lo_hi.ptr, sp.qrows, s);
      trace.mark("scan order");
    }
    FilterScan scan;
    scan.n_q = n;
    scan.n_p = n;
    scan.q_point = sp.q_point.ptr;
    scan.list_tiles = sp.list_tiles.ptr;
    scan.list_lb2 = sp.list_lb2.ptr;
    scan.list_off = sp.list_off.ptr;
    scan.list_stride = sp.list_stride;
    scan.list_sorted = sp.list_sorted;
    if (batch) {
      scan.slot_sample = slot_sample.ptr;
      scan.sample_first = batch->d_first.ptr;
    }
    const uint32_t* prows = sp.prows.ptr ? sp.prows.ptr : sp.qrows.ptr;
    if (filter == "auto") {
      const FilterChoice fc = tune_filter_kind(ctx, s, x, n, width, d, k, sp, scan, prows,
                                               mean.ptr, scale, max_sq.ptr);
      kind = fc.kind;
      scan.a_mode = fc.a_mode;
      trace.mark("filter tuning");
    }
    DeviceBuffer<uint16_t> point_ops;  // kept for the overflow retry
    DeviceBuffer<unsigned long long> tiles(1, s);
    tiles.zero();
    scan.tiles_scanned = tiles.ptr;
    tc_filter(ctx, s, x, width, d, sp.qrows.ptr, prows, scan, mean.ptr, scale, max_sq.ptr,
              kind, k, cap, cand_key, cand_row, cand_count.ptr, thr.ptr,
              qn2.ptr, slack_d.ptr, &trace, &point_ops);
    if (sp.q_full.ptr) {
      force_overflow_kernel<<<blocks_for(n, 256), 256, 0, s>>>(sp.q_full.ptr, n,
                                                               cand_count.ptr);
      KG_LAUNCH_CHECK();
    }
    filter_ms += tf.stop_ms();
    {
      unsigned long long h_tiles = 0;
      KG_CUDA(cudaMemcpyAsync(&h_tiles, tiles.ptr, 8, cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaStreamSynchronize(s));
      out.tiles_scanned = h_tiles;
      out.tiles_total = ((n + kTcQueryBlock - 1) / kTcQueryBlock) * ((n + kTile - 1) / kTile);
    }
    check_cancel(ctx);
    Timer tr(s);
    rank_kernel<<<blocks_for(n * 32, kRankWarps * 32), kRankWarps * 32, 0, s>>>(
        x, width, d, 0, n, k, cap, cand_key, cand_row, cand_count.ptr, thr.ptr,
        slack_d.ptr, 1.0 / (scale * scale), qn2.ptr, sp.qrows.ptr, prows, out.key.ptr,
        out.row.ptr, full_flag.ptr, n_cand.ptr);
    KG_LAUNCH_CHECK();
    rank_ms += tr.stop_ms();
    // Queries whose candidates overflowed (more than the slots hold within the slack of
    // their k-th: dense regions) get a second filter pass with room for kTcRetryCap
    // candidates, scanning every point tile; only those that overflow again are searched
    // in full below. The retry's rank overwrites their entries and flags.
    DeviceBuffer<uint32_t> over(n, s);
    DeviceBuffer<unsigned int> n_over(1, s);
    n_over.zero();
    {
      // The overflowed slots in slot order (a stable compaction: the retry's blocks, and
      // with them every count the search reports, are the same run to run).
      DeviceBuffer<uint8_t> oflag(n, s);
      overflow_flags_kernel<<<blocks_for(n, 256), 256, 0, s>>>(cand_count.ptr, n, oflag.ptr);
      KG_LAUNCH_CHECK();
      cub::CountingInputIterator<uint32_t> slots(0);
      size_t tb = 0;
      KG_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, slots, oflag.ptr, over.ptr, n_over.ptr,
                                         (int64_t)n, s));
      DeviceBuffer<unsigned char> tmp(tb, s);
      KG_CUDA(cub::DeviceSelect::Flagged(tmp.ptr, tb, slots, oflag.ptr, over.ptr, n_over.ptr,
                                         (int64_t)n, s));
    }
    unsigned int h_over = 0;
    KG_CUDA(cudaMemcpyAsync(&h_over, n_over.ptr, 4, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    if (trace_on())
      std::fprintf(stderr, "[kyto_gpu trace] filter: %u of %llu queries overflowed (retried)\n",
                   h_over, (unsigned long long)n);
    // A few overflowed queries would keep a few CTAs busy over every tile while the rest
    // idle: the tiles are split into ranges, each range searched by its own copy of the
    // queries (query blocks x copies about twice the SMs), and the copies merged.
    const uint32_t qblock = filter_query_block(kind);
    const uint32_t n_tiles_all = (uint32_t)((n + kTile - 1) / kTile);
    for (uint64_t r0 = 0; r0 < h_over; r0 += kTcRetryChunk) {
      check_cancel(ctx);
      const uint64_t m = std::min<uint64_t>(kTcRetryChunk, h_over - r0);
      const uint64_t nb = (m + qblock - 1) / qblock, mq = nb * qblock;
      uint64_t copies = std::max<uint64_t>(1, (2 * (uint64_t)ctx->sm_count + nb - 1) / nb);
      copies = std::min<uint64_t>(copies, std::max<uint64_t>(1, kTcRetrySplitSlots / mq));
      copies = std::min<uint64_t>(copies, n_tiles_all);
      const uint32_t nc = (uint32_t)copies;
      const uint32_t copy_cap = nc > 1 ? kTcRetrySplitCap : kTcRetryCap;
      const uint64_t mv = mq * nc;
      DeviceBuffer<uint32_t> r_qrows(mv, s), r_qpoint(mv, s), r_sample(batch ? mv : 0, s);
      retry_slots_kernel<<<blocks_for(mv, 256), 256, 0, s>>>(
          over.ptr + r0, m, mq, nc, sp.qrows.ptr, sp.q_point.ptr,
          batch ? slot_sample.ptr : nullptr, r_qrows.ptr, r_qpoint.ptr, r_sample.ptr);
      KG_LAUNCH_CHECK();
      FilterScan rs = scan;
      rs.n_q = mv;
      rs.q_point = r_qpoint.ptr;
      rs.slot_sample = batch ? r_sample.ptr : nullptr;
      rs.list_tiles = nullptr;
      rs.list_lb2 = nullptr;
      rs.list_off = nullptr;
      rs.list_stride = 0;
      rs.list_sorted = false;
      rs.tiles_scanned = nullptr;
      DeviceBuffer<uint64_t> r_off;
      DeviceBuffer<uint32_t> r_list;
      if (nc > 1) {
        r_off.alloc(nb * nc + 1, s);
        r_list.alloc(nb * (uint64_t)n_tiles_all, s);
        retry_lists_kernel<<<(unsigned)(nb * nc), 256, 0, s>>>(nb, nc, n_tiles_all, r_off.ptr,
                                                               r_list.ptr);
        KG_LAUNCH_CHECK();
        rs.list_tiles = r_list.ptr;
        rs.list_off = r_off.ptr;
      }
      DeviceBuffer<float> r_key(mv * copy_cap, s), r_thr(mv, s);
      DeviceBuffer<uint32_t> r_row(mv * copy_cap, s), r_count(mv, s);
      DeviceBuffer<double> r_qn2(mv, s), r_slack(mv, s);
      Timer trf(s);
      tc_filter(ctx, s, x, width, d, r_qrows.ptr, prows, rs, mean.ptr, scale, max_sq.ptr, kind,
                k, copy_cap, r_key.ptr, r_row.ptr, r_count.ptr, r_thr.ptr, r_qn2.ptr,
                r_slack.ptr, nullptr, &point_ops);
      filter_ms += trf.stop_ms();
      Timer trr(s);
      // Copy 0's slots 0..m-1 are the overflowed queries in order (their rows, norms and
      // slacks); the merged candidates replace the copies'.
      DeviceBuffer<float> m_key, m_thr;
      DeviceBuffer<uint32_t> m_row, m_count;
      const float* use_key = r_key.ptr;
      const uint32_t* use_row = r_row.ptr;
      const uint32_t* use_count = r_count.ptr;
      const float* use_thr = r_thr.ptr;
      if (nc > 1) {
        m_key.alloc(m * kTcRetryCap, s);
        m_row.alloc(m * kTcRetryCap, s);
        m_count.alloc(m, s);
        m_thr.alloc(m, s);
        retry_merge_kernel<<<blocks_for(m * 32, 256), 256, 0, s>>>(
            m, mq, nc, copy_cap, r_key.ptr, r_row.ptr, r_count.ptr, r_thr.ptr, kTcRetryCap,
            m_key.ptr, m_row.ptr, m_count.ptr, m_thr.ptr);
        KG_LAUNCH_CHECK();
        use_key = m_key.ptr;
        use_row = m_row.ptr;
        use_count = m_count.ptr;
        use_thr = m_thr.ptr;
      }
      rank_kernel<<<blocks_for(m * 32, kRankWarps * 32), kRankWarps * 32, 0, s>>>(
          x, width, d, 0, m, k, nc > 1 ? kTcRetryCap : copy_cap, use_key, use_row, use_count,
          use_thr, r_slack.ptr, 1.0 / (scale * scale), r_qn2.ptr, r_qrows.ptr, prows,
          out.key.ptr, out.row.ptr, full_flag.ptr, n_cand.ptr);
      KG_LAUNCH_CHECK();
      rank_ms += trr.stop_ms();
    }
    out.retried = h_over;
    trace.mark("overflow retry");
    ctx->done = n;
  } else {
    const uint32_t cap = kCandidateCap;
    uint64_t chunk = std::min<uint64_t>(n, kQueryChunk);
    DeviceBuffer<float> cand_key(chunk * cap, s), thr(chunk, s);
    DeviceBuffer<uint32_t> cand_row(chunk * cap, s), cand_count(chunk, s);
    for (uint64_t q0 = 0; q0 < n; q0 += chunk) {
      check_cancel(ctx);
      uint64_t q1 = std::min(n, q0 + chunk);
      Timer tf(s);
      filter_kernel<<<blocks_for(q1 - q0, kFilterThreads), kFilterThreads, 0, s>>>(
          rows.ptr, offsets.ptr, slack.ptr, n, q0, q1, k, cap, cand_key.ptr, cand_row.ptr,
          cand_count.ptr, thr.ptr);
      KG_LAUNCH_CHECK();
      filter_ms += tf.stop_ms();
      Timer tr(s);
      rank_kernel<<<blocks_for((q1 - q0) * 32, kRankWarps * 32), kRankWarps * 32, 0, s>>>(
          x, width, d, q0, q1, k, cap, cand_key.ptr, cand_row.ptr, cand_count.ptr, thr.ptr,
          slack.ptr, 1.0, nullptr, nullptr, nullptr, out.key.ptr, out.row.ptr, full_flag.ptr,
          n_cand.ptr);
      KG_LAUNCH_CHECK();
      rank_ms += tr.stop_ms();
      ctx->done = q1;
    }
  }
  trace.mark("rank");
  // Rows that need a full search.
  DeviceBuffer<uint32_t> list(n, s);
  DeviceBuffer<unsigned int> n_full(1, s);
  n_full.zero();
  compact_flags_kernel<<<blocks_for(n, 256), 256, 0, s>>>(full_flag.ptr, n, list.ptr,
                                                          n_full.ptr);
  KG_LAUNCH_CHECK();
  unsigned int h_full = 0;
  KG_CUDA(cudaMemcpyAsync(&h_full, n_full.ptr, 4, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  if (h_full) {
    // The list's order does not matter: each CTA writes its own row.
    Timer tr(s);
    for (uint64_t a = 0; a < h_full; a += 65535) {
      check_cancel(ctx);
      unsigned blocks = (unsigned)std::min<uint64_t>(65535, h_full - a);
      full_rows_kernel<<<blocks, kFullWarps * 32, 0, s>>>(
          x, n, width, d, k, list.ptr + a, batch ? batch->row_sample.ptr : nullptr,
          batch ? batch->d_first.ptr : nullptr, out.key.ptr, out.row.ptr);
      KG_LAUNCH_CHECK();
    }
    rank_ms += tr.stop_ms();
  }
  trace.mark("full rows");
  unsigned long long h_cand = 0;
  KG_CUDA(cudaMemcpyAsync(&h_cand, n_cand.ptr, 8, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  out.candidates = h_cand;
  out.rows_full = h_full;
  out.filter_ms = filter_ms;
  out.rank_ms = rank_ms;
}

// n_neighbors and n_components checked as neighbors::search does (neighbors.rs:226-312);
// returns k and d.
void check_search_args(uint64_t n, uint32_t width, uint32_t n_components, uint32_t n_neighbors,
                       uint32_t& k, uint32_t& d) {
  if (width == 0) fail(KG_ERR_INVALID, "neighbors: an embedding of 0 components");
  d = n_components ? n_components : width;
  if (d > width)
    fail(KG_ERR_INVALID, "neighbors: n_components " + std::to_string(n_components) +
                             " is more than the embedding's " + std::to_string(width));
  if (d > (uint32_t)kDim)
    fail(KG_ERR_INVALID, "neighbors: more than " + std::to_string(kDim) + " components");
  if (n_neighbors < 2 || n_neighbors > n)
    fail(KG_ERR_INVALID, "neighbors: n_neighbors " + std::to_string(n_neighbors) +
                             " (it counts the cell itself; " + std::to_string(n) +
                             " cells): an int from 2 to " + std::to_string(std::max<uint64_t>(n, 2)));
  if (n - 1 >= (1ull << 32)) fail(KG_ERR_INVALID, "neighbors: at most 2^32 cells");
  k = n_neighbors - 1;
  if (k > (uint32_t)kMaxK)
    fail(KG_ERR_INVALID, "neighbors: n_neighbors above " + std::to_string(kMaxK + 1));
}

// Finite values only (neighbors.rs:279-291).
void check_finite(const float* x, uint64_t n, uint32_t width, uint32_t d, cudaStream_t s) {
  DeviceBuffer<unsigned long long> bad(1, s);
  unsigned long long init = ~0ull;
  KG_CUDA(cudaMemcpyAsync(bad.ptr, &init, 8, cudaMemcpyHostToDevice, s));
  finite_check_kernel<<<std::min<unsigned>(blocks_for(n * d, 256), 8192), 256, 0, s>>>(
      x, n, width, d, bad.ptr);
  KG_LAUNCH_CHECK();
  unsigned long long first = 0;
  KG_CUDA(cudaMemcpyAsync(&first, bad.ptr, 8, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  if (first != ~0ull)
    fail(KG_ERR_INVALID, "neighbors: row " + std::to_string(first / width) + ", component " +
                             std::to_string(first % width) + " is not finite");
}

// A batch's graphs: sample s's CSR (indptr of n_s + 1 entries at indptr + first[s] + s,
// columns relative to its first row) and entries at first[s] * k, rows sorted by column.
__global__ void batch_graph_kernel(const double* keys, const uint32_t* rows, uint64_t n,
                                   uint32_t k, const uint32_t* row_sample,
                                   const uint64_t* first, uint64_t* indptr, uint32_t* indices,
                                   float* distances) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  const uint32_t smp = row_sample[r];
  const uint64_t f = first[smp];
  uint64_t* ip = indptr + f + smp;
  if (r == f) ip[0] = 0;
  ip[r - f + 1] = (r - f + 1) * (uint64_t)k;
  const double* kr = keys + r * k;
  const uint32_t* rr = rows + r * k;
  uint32_t* oi = indices + r * k;
  float* od = distances + r * k;
  for (uint32_t i = 0; i < k; ++i) {
    const uint32_t row = rr[i] - (uint32_t)f;
    const float dist = (float)sqrt(kr[i]);
    uint32_t at = i;
    while (at > 0 && oi[at - 1] > row) {
      oi[at] = oi[at - 1];
      od[at] = od[at - 1];
      --at;
    }
    oi[at] = row;
    od[at] = dist;
  }
}

// The CSR graph (rows sorted by column, f32 sqrt of the key) into host or device memory.
void write_graph(const KnnResult& r, uint64_t n, uint32_t k, uint64_t* indptr, uint32_t* indices,
                 float* distances, cudaStream_t s) {
  DeviceBuffer<uint64_t> g_indptr;
  DeviceBuffer<uint32_t> g_idx;
  DeviceBuffer<float> g_dist;
  bool dev_out = is_device_pointer(indptr);
  uint64_t* gi = indptr;
  uint32_t* gx = indices;
  float* gd = distances;
  if (!dev_out) {
    g_indptr.alloc(n + 1, s);
    g_idx.alloc(n * k, s);
    g_dist.alloc(n * k, s);
    gi = g_indptr.ptr;
    gx = g_idx.ptr;
    gd = g_dist.ptr;
  }
  graph_kernel<<<blocks_for(n, 128), 128, 0, s>>>(r.key.ptr, r.row.ptr, n, k, gi, gx, gd);
  KG_LAUNCH_CHECK();
  if (!dev_out) {
    KG_CUDA(cudaMemcpyAsync(indptr, gi, (n + 1) * 8, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaMemcpyAsync(indices, gx, n * k * 4, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaMemcpyAsync(distances, gd, n * k * 4, cudaMemcpyDeviceToHost, s));
  }
  KG_CUDA(cudaStreamSynchronize(s));
}

// The batch's search and graphs (kg_knn_batch after its checks; x on the device).
void knn_batch_run(kg_ctx* ctx, const float* x, uint64_t n, uint32_t width, uint32_t d,
                   uint32_t k, const std::vector<uint64_t>& first, uint64_t* indptr,
                   uint32_t* indices, float* distances, kg_knn_stats* stats) {
  cudaStream_t s = ctx->stream;
  const uint32_t n_samples = (uint32_t)first.size() - 1;
  ctx->total = n;
  ctx->done = 0;
  Trace trace(s, "knn_batch");
  KnnBatch batch;
  batch.first = first;
  batch.d_first.alloc(n_samples + 1, s);
  KG_CUDA(cudaMemcpyAsync(batch.d_first.ptr, batch.first.data(), (n_samples + 1) * 8ull,
                          cudaMemcpyHostToDevice, s));
  std::vector<uint32_t> rs(n);
  for (uint32_t smp = 0; smp < n_samples; ++smp)
    std::fill(rs.begin() + batch.first[smp], rs.begin() + batch.first[smp + 1], smp);
  batch.row_sample.alloc(n, s);
  KG_CUDA(cudaMemcpyAsync(batch.row_sample.ptr, rs.data(), n * 4, cudaMemcpyHostToDevice, s));
  KnnResult r;
  knn_core(ctx, x, n, width, d, k, nullptr, r, trace, &batch);
  // The graphs (host or device outputs).
  const bool dev_out = is_device_pointer(indptr);
  DeviceBuffer<uint64_t> g_indptr;
  DeviceBuffer<uint32_t> g_idx;
  DeviceBuffer<float> g_dist;
  uint64_t* gi = indptr;
  uint32_t* gx = indices;
  float* gd = distances;
  if (!dev_out) {
    g_indptr.alloc(n + n_samples, s);
    g_idx.alloc(n * k, s);
    g_dist.alloc(n * k, s);
    gi = g_indptr.ptr;
    gx = g_idx.ptr;
    gd = g_dist.ptr;
  }
  batch_graph_kernel<<<blocks_for(n, 128), 128, 0, s>>>(r.key.ptr, r.row.ptr, n, k,
                                                        batch.row_sample.ptr, batch.d_first.ptr,
                                                        gi, gx, gd);
  KG_LAUNCH_CHECK();
  if (!dev_out) {
    KG_CUDA(cudaMemcpyAsync(indptr, gi, (n + n_samples) * 8, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaMemcpyAsync(indices, gx, n * k * 4, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaMemcpyAsync(distances, gd, n * k * 4, cudaMemcpyDeviceToHost, s));
  }
  trace.mark("graph");
  wait_stream(ctx, s);
  ctx->done = n;
  if (stats) {
    stats->candidates = r.candidates;
    stats->rows_full = r.rows_full;
    stats->filter_ms = r.filter_ms;
    stats->rank_ms = r.rank_ms;
    stats->tiles_scanned = r.tiles_scanned;
    stats->tiles_total = r.tiles_total;
  }
}

}  // namespace kg

using namespace kg;

extern "C" kg_status kg_knn_batch(kg_ctx* ctx, const float* embedding, uint64_t n,
                                  uint32_t width, uint32_t n_components, uint32_t n_neighbors,
                                  const uint64_t* sample_rows, uint32_t n_samples,
                                  uint64_t* indptr, uint32_t* indices, float* distances,
                                  kg_knn_stats* stats) {
  return guarded([&] {
    if (!ctx || !embedding || !sample_rows || !indptr || !indices || !distances)
      fail(KG_ERR_INVALID, "kg_knn_batch: NULL argument");
    if (n_samples == 0) fail(KG_ERR_INVALID, "kg_knn_batch: no samples");
    KnnBatch batch;
    batch.first.assign(sample_rows, sample_rows + n_samples + 1);
    if (batch.first[0] != 0 || batch.first[n_samples] != n)
      fail(KG_ERR_INVALID, "kg_knn_batch: sample_rows must run from 0 to n_rows");
    uint32_t k = 0, d = 0;
    for (uint32_t smp = 0; smp < n_samples; ++smp) {
      if (batch.first[smp + 1] < batch.first[smp])
        fail(KG_ERR_INVALID, "kg_knn_batch: sample_rows must not decrease");
      const uint64_t ns = batch.first[smp + 1] - batch.first[smp];
      try {
        check_search_args(ns, width, n_components, n_neighbors, k, d);
      } catch (const Error& e) {
        fail(e.status, "sample " + std::to_string(smp) + ": " + e.message);
      }
    }
    use_device(ctx);
    cudaStream_t s = ctx->stream;
    DeviceBuffer<float> hold;
    const float* x = device_view(embedding, n * width, hold, s);
    check_finite(x, n, width, d, s);
    knn_batch_run(ctx, x, n, width, d, k, batch.first, indptr, indices, distances, stats);
  });
}

extern "C" kg_status kg_knn_exact(kg_ctx* ctx, const float* embedding, uint64_t n,
                                  uint32_t width, uint32_t n_components,
                                  uint32_t n_neighbors, uint64_t* indptr, uint32_t* indices,
                                  float* distances, kg_knn_stats* stats) {
  return guarded([&] {
    if (!ctx || !embedding || !indptr || !indices || !distances)
      fail(KG_ERR_INVALID, "kg_knn_exact: NULL argument");
    uint32_t k = 0, d = 0;
    check_search_args(n, width, n_components, n_neighbors, k, d);
    use_device(ctx);
    cudaStream_t s = ctx->stream;
    ctx->total = n;
    ctx->done = 0;
    DeviceBuffer<float> hold;
    const float* x = device_view(embedding, n * width, hold, s);
    check_finite(x, n, width, d, s);
    Trace trace(s, "knn_exact");
    KnnResult r;
    knn_core(ctx, x, n, width, d, k, nullptr, r, trace);
    write_graph(r, n, k, indptr, indices, distances, s);
    trace.mark("graph");
    wait_stream(ctx, s);
    ctx->done = n;
    if (stats) {
      stats->candidates = r.candidates;
      stats->rows_full = r.rows_full;
      stats->filter_ms = r.filter_ms;
      stats->rank_ms = r.rank_ms;
      stats->tiles_scanned = r.tiles_scanned;
      stats->tiles_total = r.tiles_total;
    }
  });
}
