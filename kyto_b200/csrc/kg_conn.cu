// UMAP connectivities of a kNN graph on the device: kyto's `connectivities`
// (crates/kyto-exec/src/connectivities.rs:84-131, scanpy's pp.neighbors(method="umap")
// weights). One thread per row ranks the row's distances and bisects its sigma in f64; one
// thread per entry weighs it in f32; the fuzzy union w + w^T - w o w^T pairs each row's own
// entries with the transposed ones (a radix sort of (column, row) keys) in a two-pointer
// merge, counted then written, so the output rows come out with increasing columns and no
// stored zeros. The f32 arithmetic is IEEE without contraction (explicit _rn intrinsics),
// the sums run in kyto's order, and the one f32 exponential is evaluated in f64 and
// rounded once.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cfloat>
#include <cmath>
#include <vector>

#include "kg_internal.cuh"

namespace kg {

namespace {

constexpr int kConnIterations = 64;        // SMOOTH_K_ITERATIONS (connectivities.rs:26)
constexpr double kConnTolerance = 1e-5;    // SMOOTH_K_TOLERANCE (:28)
constexpr double kMinKDistScale = 1e-3;    // MIN_K_DIST_SCALE (:30)
constexpr uint32_t kConnMaxK = 255;        // stored neighbours a row, at most

// f32 bits as an int in IEEE total order (Rust's f32::total_cmp).
__device__ __forceinline__ int32_t total_order(float v) {
  const int32_t b = __float_as_int(v);
  return b ^ (int32_t)((uint32_t)(b >> 31) >> 1);
}

// The graph's shape: row r holds entries [r k, (r + 1) k), columns strictly increasing and
// below n. Sets *bad on the first violation seen.
__global__ void check_graph_kernel(const uint64_t* indptr, const uint32_t* indices, uint64_t n,
                                   uint32_t k, int* bad) {
  const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r > n) return;
  if (indptr[r] != r * k) {
    atomicExch(bad, 1);
    return;
  }
  if (r == n) return;
  const uint32_t* c = indices + r * k;
  for (uint32_t j = 0; j < k; ++j)
    if (c[j] >= n || (j > 0 && c[j] <= c[j - 1])) {
      atomicExch(bad, 2);
      return;
    }
}

// Per row (connectivities.rs:90-104, 133-176): the k distances ranked by (distance, column)
// into ranked; rho = the first ranked distance above 0; sigma by the 64-step bisection on
// sum_j [d_j > 0 ? exp(-(d_j / mid)) : 1] = target (d_j = f32(ranked_j - rho) widened),
// floored at 1e-3 of the row's mean (a sequential f32 sum over n_neighbors) when rho > 0.
__global__ void smooth_knn_kernel(const float* distances, uint64_t n, uint32_t k,
                                  uint32_t n_neighbors, double target, float* ranked,
                                  float* sigma_out, float* rho_out, int* any_zero_rho) {
  const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  float* row = ranked + r * k;
  const float* d = distances + r * k;
  // A stable insertion sort on the f32 total order into the row's slice of `ranked`: equal
  // distances keep the input order, which is the order of their (increasing) columns.
  for (uint32_t j = 0; j < k; ++j) {
    const float v = d[j];
    const int32_t kv = total_order(v);
    uint32_t at = j;
    while (at > 0 && total_order(row[at - 1]) > kv) {
      row[at] = row[at - 1];
      --at;
    }
    row[at] = v;
  }
  float rho = 0.0f;
  for (uint32_t j = 0; j < k; ++j)
    if (row[j] > 0.0f) {
      rho = row[j];
      break;
    }
  const double ceiling = (double)FLT_MAX;
  double lo = 0.0, hi = ceiling, mid = 1.0;
  for (int it = 0; it < kConnIterations; ++it) {
    double sum = 0.0;
    for (uint32_t j = 0; j < k; ++j) {
      const double dj = (double)__fsub_rn(row[j], rho);
      sum = __dadd_rn(sum, dj > 0.0 ? exp(-__ddiv_rn(dj, mid)) : 1.0);
    }
    if (fabs(sum - target) < kConnTolerance) break;
    if (sum > target) {
      hi = mid;
      mid = __dmul_rn(__dadd_rn(lo, hi), 0.5);
    } else {
      lo = mid;
      mid = hi >= ceiling ? __dmul_rn(mid, 2.0) : __dmul_rn(__dadd_rn(lo, hi), 0.5);
    }
  }
  float sigma = __double2float_rn(mid);
  if (rho > 0.0f) {
    float s = 0.0f;
    for (uint32_t j = 0; j < k; ++j) s = __fadd_rn(s, row[j]);
    const double floor_v = kMinKDistScale * ((double)s / (double)n_neighbors);
    if ((double)sigma < floor_v) sigma = __double2float_rn(floor_v);
  } else {
    atomicExch(any_zero_rho, 1);
  }
  sigma_out[r] = sigma;
  rho_out[r] = rho;
}

// The sequential f32 sum of every ranked distance, rows in order (connectivities.rs:108-
// 116, only when some row has rho == 0), then the floor applied to those rows.
__global__ void global_floor_kernel(const float* ranked, uint64_t count, uint64_t n,
                                    uint32_t n_neighbors, const float* rho, float* sigma) {
  __shared__ double floor_v;
  if (threadIdx.x == 0) {
    float s = 0.0f;
    for (uint64_t i = 0; i < count; ++i) s = __fadd_rn(s, ranked[i]);
    floor_v = kMinKDistScale * ((double)s / ((double)n * (double)n_neighbors));
  }
  __syncthreads();
  for (uint64_t r = threadIdx.x; r < n; r += blockDim.x)
    if (rho[r] == 0.0f && (double)sigma[r] < floor_v) sigma[r] = __double2float_rn(floor_v);
}

// Each entry's membership (connectivities.rs:189-198) and its transpose key
// (column << 32 | row).
__global__ void membership_kernel(const float* distances, const uint32_t* indices, uint64_t n,
                                  uint32_t k, const float* sigma, const float* rho, float* w,
                                  unsigned long long* tkey, float* tval) {
  const uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (e >= n * k) return;
  const uint64_t r = e / k;
  const uint32_t c = indices[e];
  const float s = sigma[r], t = __fsub_rn(distances[e], rho[r]);
  float v;
  if (c == r)
    v = 0.0f;
  else if (t <= 0.0f || s == 0.0f)
    v = 1.0f;
  else
    v = __double2float_rn(exp(-(double)__fdiv_rn(t, s)));
  w[e] = v;
  tkey[e] = ((unsigned long long)c << 32) | (unsigned long long)r;
  tval[e] = v;
}

// tstart[c] = the first sorted transposed entry of column (= transposed row) c.
__global__ void transposed_starts_kernel(const unsigned long long* sorted, uint64_t m,
                                         uint64_t n, uint64_t* tstart) {
  const uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (c > n) return;
  uint64_t lo = 0, hi = m;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if ((sorted[mid] >> 32) < c) lo = mid + 1; else hi = mid;
  }
  tstart[c] = lo;
}

// The union of row r (connectivities.rs:221-255): its own entries (increasing columns) and
// its transposed ones (increasing rows), merged; weight (w + wT) - w wT in f32, zeros
// dropped. Count pass (out NULL: counts[r]) or write pass (at out_ptr[r]).
__global__ void union_kernel(const uint32_t* indices, const float* w, uint64_t n, uint32_t k,
                             const unsigned long long* tkeys, const float* tvals,
                             const uint64_t* tstart, uint64_t* counts, const uint64_t* out_ptr,
                             uint32_t* out_idx, float* out_w) {
  const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  uint64_t f = r * k;
  const uint64_t f_end = f + k;
  uint64_t b = tstart[r];
  const uint64_t b_end = tstart[r + 1];
  uint64_t at = out_ptr ? out_ptr[r] : 0, count = 0;
  while (f < f_end || b < b_end) {
    uint32_t col;
    float wf = 0.0f, wt = 0.0f;
    const uint32_t fc = f < f_end ? indices[f] : 0xFFFFFFFFu;
    const uint32_t bc = b < b_end ? (uint32_t)(tkeys[b] & 0xFFFFFFFFull) : 0xFFFFFFFFu;
    if (f < f_end && (b >= b_end || fc < bc)) {
      col = fc;
      wf = w[f++];
    } else if (b < b_end && (f >= f_end || bc < fc)) {
      col = bc;
      wt = tvals[b++];
    } else {
      col = fc;
      wf = w[f++];
      wt = tvals[b++];
    }
    const float weight = __fsub_rn(__fadd_rn(wf, wt), __fmul_rn(wf, wt));
    if (weight != 0.0f) {
      if (out_ptr) {
        out_idx[at] = col;
        out_w[at] = weight;
        ++at;
      }
      ++count;
    }
  }
  if (!out_ptr) counts[r] = count;
}

}  // namespace

}  // namespace kg

using namespace kg;

extern "C" kg_status kg_connectivities(kg_ctx* ctx, const uint64_t* indptr,
                                       const uint32_t* indices, const float* distances,
                                       uint64_t n_rows, uint32_t n_neighbors,
                                       uint64_t* out_indptr, uint32_t* out_indices,
                                       float* out_weights, uint64_t* out_nnz) {
  return guarded([&] {
    if (!ctx || !indptr || !indices || !distances || !out_indptr || !out_indices ||
        !out_weights || !out_nnz)
      fail(KG_ERR_INVALID, "kg_connectivities: NULL argument");
    if (n_neighbors < 2 || n_neighbors - 1 > kConnMaxK)
      fail(KG_ERR_INVALID, "kg_connectivities: n_neighbors must be 2.." +
                               std::to_string(kConnMaxK + 1));
    if (n_rows == 0 || n_rows >= 0xFFFFFFFFull ||
        n_rows * (uint64_t)(n_neighbors - 1) > (uint64_t)INT32_MAX)
      fail(KG_ERR_INVALID,
           "kg_connectivities: n_rows must be at least 1 and n_rows x (n_neighbors - 1) below 2^31");
    use_device(ctx);
    cudaStream_t s = ctx->stream;
    Trace trace(s, "connectivities");
    const uint32_t k = n_neighbors - 1;
    const uint64_t m = n_rows * k;
    DeviceBuffer<uint64_t> hp;
    DeviceBuffer<uint32_t> hi;
    DeviceBuffer<float> hd;
    const uint64_t* d_ptr = device_view(indptr, n_rows + 1, hp, s);
    const uint32_t* d_idx = device_view(indices, m, hi, s);
    const float* d_dist = device_view(distances, m, hd, s);
    DeviceBuffer<int> flags(2, s);
    flags.zero();
    check_graph_kernel<<<blocks_for(n_rows + 1, 256), 256, 0, s>>>(d_ptr, d_idx, n_rows, k,
                                                                   flags.ptr);
    KG_LAUNCH_CHECK();
    int h_bad = 0;
    KG_CUDA(cudaMemcpyAsync(&h_bad, flags.ptr, 4, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    if (h_bad == 1)
      fail(KG_ERR_INVALID, "kg_connectivities: every row must hold n_neighbors - 1 entries");
    if (h_bad == 2)
      fail(KG_ERR_INVALID,
           "kg_connectivities: a row's columns must increase strictly and be below n_rows");
    // Rows: ranked distances, rho, sigma.
    DeviceBuffer<float> ranked(m, s), sigma(n_rows, s), rho(n_rows, s);
    smooth_knn_kernel<<<blocks_for(n_rows, 128), 128, 0, s>>>(
        d_dist, n_rows, k, n_neighbors, std::log2((double)n_neighbors), ranked.ptr, sigma.ptr,
        rho.ptr, flags.ptr + 1);
    KG_LAUNCH_CHECK();
    int h_zero = 0;
    KG_CUDA(cudaMemcpyAsync(&h_zero, flags.ptr + 1, 4, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    if (h_zero) {
      global_floor_kernel<<<1, 256, 0, s>>>(ranked.ptr, m, n_rows, n_neighbors, rho.ptr,
                                            sigma.ptr);
      KG_LAUNCH_CHECK();
    }
    trace.mark("sigma");
    // Entries: memberships and the transpose.
    DeviceBuffer<float> w(m, s), tval(m, s), tval_sorted(m, s);
    DeviceBuffer<unsigned long long> tkey(m, s), tkey_sorted(m, s);
    membership_kernel<<<blocks_for(m, 256), 256, 0, s>>>(d_dist, d_idx, n_rows, k, sigma.ptr,
                                                         rho.ptr, w.ptr, tkey.ptr, tval.ptr);
    KG_LAUNCH_CHECK();
    int bits = 32;
    while (bits < 64 && (1ull << (bits - 32)) <= n_rows) ++bits;
    size_t temp = 0;
    KG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, tkey.ptr, tkey_sorted.ptr, tval.ptr,
                                            tval_sorted.ptr, (int)m, 0, bits, s));
    DeviceBuffer<unsigned char> scratch(temp, s);
    KG_CUDA(cub::DeviceRadixSort::SortPairs(scratch.ptr, temp, tkey.ptr, tkey_sorted.ptr,
                                            tval.ptr, tval_sorted.ptr, (int)m, 0, bits, s));
    DeviceBuffer<uint64_t> tstart(n_rows + 1, s);
    transposed_starts_kernel<<<blocks_for(n_rows + 1, 256), 256, 0, s>>>(tkey_sorted.ptr, m,
                                                                         n_rows, tstart.ptr);
    KG_LAUNCH_CHECK();
    trace.mark("memberships");
    // The union: counts, offsets, entries.
    DeviceBuffer<uint64_t> ptr(n_rows + 1, s);
    ptr.zero();
    union_kernel<<<blocks_for(n_rows, 128), 128, 0, s>>>(d_idx, w.ptr, n_rows, k,
                                                         tkey_sorted.ptr, tval_sorted.ptr,
                                                         tstart.ptr, ptr.ptr, nullptr, nullptr,
                                                         nullptr);
    KG_LAUNCH_CHECK();
    size_t temp2 = 0;
    KG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp2, ptr.ptr, ptr.ptr, n_rows + 1, s));
    DeviceBuffer<unsigned char> scratch2(temp2, s);
    KG_CUDA(cub::DeviceScan::ExclusiveSum(scratch2.ptr, temp2, ptr.ptr, ptr.ptr, n_rows + 1, s));
    uint64_t nnz = 0;
    KG_CUDA(cudaMemcpyAsync(&nnz, ptr.ptr + n_rows, 8, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    DeviceBuffer<uint32_t> oi(std::max<uint64_t>(nnz, 1), s);
    DeviceBuffer<float> ow(std::max<uint64_t>(nnz, 1), s);
    union_kernel<<<blocks_for(n_rows, 128), 128, 0, s>>>(d_idx, w.ptr, n_rows, k,
                                                         tkey_sorted.ptr, tval_sorted.ptr,
                                                         tstart.ptr, nullptr, ptr.ptr, oi.ptr,
                                                         ow.ptr);
    KG_LAUNCH_CHECK();
    KG_CUDA(cudaMemcpyAsync(out_indptr, ptr.ptr, (n_rows + 1) * 8, cudaMemcpyDefault, s));
    if (nnz) {
      KG_CUDA(cudaMemcpyAsync(out_indices, oi.ptr, nnz * 4, cudaMemcpyDefault, s));
      KG_CUDA(cudaMemcpyAsync(out_weights, ow.ptr, nnz * 4, cudaMemcpyDefault, s));
    }
    trace.mark("union");
    wait_stream(ctx, s);
    *out_nnz = nnz;
  });
}
