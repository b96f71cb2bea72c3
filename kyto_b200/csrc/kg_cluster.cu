// k-means on the device (kg_cluster.cuh). Every sum runs in a fixed order; ties go to
// the lower index: the same clusters on every run.
#include "kg_cluster.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>

namespace kg {

namespace {

constexpr int kNcRows = 64;   // rows per nearest-centre block
constexpr int kNcChunk = 64;  // centres per shared-memory chunk

// 256 threads: thread (ty, tx) holds rows ty*4.. and centres tx*4.. of each chunk.
__global__ void __launch_bounds__(256)
nearest_centres_kernel(const float* __restrict__ x, uint64_t n, uint32_t width, uint32_t d,
                       const float* __restrict__ centres, const float* __restrict__ cn,
                       uint32_t K, uint32_t* labels) {
  __shared__ float xs[kClusterDim][kNcRows + 1];
  __shared__ float cs[kClusterDim][kNcChunk + 1];
  __shared__ float cb[kNcChunk];
  const uint32_t tx = threadIdx.x & 15u, ty = threadIdx.x >> 4;
  const uint64_t r0 = blockIdx.x * (uint64_t)kNcRows;
  for (uint32_t e = threadIdx.x; e < kClusterDim * kNcRows; e += 256) {
    const uint32_t rr = e / kClusterDim, j = e % kClusterDim;
    const uint64_t row = r0 + rr;
    xs[j][rr] = (row < n && j < d) ? x[row * width + j] : 0.0f;
  }
  float best[4];
  uint32_t arg[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    best[i] = INFINITY;
    arg[i] = 0xFFFFFFFFu;
  }
  for (uint32_t c0 = 0; c0 < K; c0 += kNcChunk) {
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < kClusterDim * kNcChunk; e += 256) {
      const uint32_t cc = e / kClusterDim, j = e % kClusterDim;
      cs[j][cc] = (c0 + cc < K) ? centres[(uint64_t)(c0 + cc) * kClusterDim + j] : 0.0f;
    }
    if (threadIdx.x < kNcChunk) {
      const uint32_t c = c0 + threadIdx.x;
      cb[threadIdx.x] = c < K ? cn[c] : INFINITY;
    }
    __syncthreads();
    float dot[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dot[i][j] = 0.0f;
    for (uint32_t j = 0; j < d; ++j) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = xs[j][ty * 4 + i];
#pragma unroll
      for (int i = 0; i < 4; ++i) b[i] = cs[j][tx * 4 + i];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) dot[i][jj] = fmaf(a[i], b[jj], dot[i][jj]);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const uint32_t c = c0 + tx * 4 + jj;
        const float dist = cb[tx * 4 + jj] - 2.0f * dot[i][jj];
        if (c < K && (dist < best[i] || (dist == best[i] && c < arg[i]))) {
          best[i] = dist;
          arg[i] = c;
        }
      }
  }
  // The 16 threads of a row group (lanes sharing ty) combine.
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float bv = best[i];
    uint32_t ba = arg[i];
    for (int o = 8; o; o >>= 1) {
      const float ov = __shfl_xor_sync(0xFFFFFFFFu, bv, o);
      const uint32_t oa = __shfl_xor_sync(0xFFFFFFFFu, ba, o);
      if (ov < bv || (ov == bv && oa < ba)) {
        bv = ov;
        ba = oa;
      }
    }
    const uint64_t row = r0 + ty * 4 + i;
    if (tx == 0 && row < n) labels[row] = ba;
  }
}

__global__ void gather_rows_kernel(const float* x, uint64_t n, uint32_t width, uint32_t d,
                                   uint64_t m, float* out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= m * d) return;
  const uint64_t r = i / d, j = i % d;
  const uint64_t row = r * n / m;  // evenly strided
  out[r * d + j] = x[row * width + j];
}

// centre[c] = row (c * m / K) of the sample (d columns, padded with zeros).
__global__ void seed_centres_kernel(const float* sample, uint64_t m, uint32_t d, uint32_t K,
                                    double* centre) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (uint64_t)K * kClusterDim) return;
  const uint64_t c = i / kClusterDim, j = i % kClusterDim;
  centre[i] = j < d ? (double)sample[(c * m / K) * d + j] : 0.0;
}

__global__ void centres_f32_kernel(const double* centre, uint32_t K, float* cf, float* cn) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= K) return;
  float s = 0.0f;
  for (uint32_t j = 0; j < kClusterDim; ++j) {
    const float v = (float)centre[(uint64_t)c * kClusterDim + j];
    cf[(uint64_t)c * kClusterDim + j] = v;
    s = fmaf(v, v, s);
  }
  cn[c] = s;
}

// key = (label << 32) | the first component's f32 bits mapped to an unsigned order.
__global__ void order_key_kernel(const float* x, uint64_t n, uint32_t width, const uint32_t* label,
                                 unsigned long long* key, uint32_t* iota) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  uint32_t b = __float_as_uint(x[r * width]);
  b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  key[r] = ((unsigned long long)label[r] << 32) | b;
  iota[r] = (uint32_t)r;
}

// starts[c] = the first position whose key's label is >= c (c = 0..K).
__global__ void key_starts_kernel(const unsigned long long* sorted, uint64_t n, uint32_t K,
                                  uint32_t* starts) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > K) return;
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if ((uint32_t)(sorted[mid] >> 32) < c) lo = mid + 1; else hi = mid;
  }
  starts[c] = (uint32_t)lo;
}

// centre[c] = the mean (f64, members in slot order) of cluster c's rows; an empty
// cluster keeps its centre. One block per cluster, one thread per component.
__global__ void update_centres_kernel(const float* x, uint32_t width, uint32_t d,
                                      const uint32_t* order, const uint32_t* starts,
                                      double* centre) {
  const uint32_t c = blockIdx.x, j = threadIdx.x;
  const uint32_t b = starts[c], e = starts[c + 1];
  if (b == e || j >= d) return;
  double s = 0.0;
  for (uint32_t i = b; i < e; ++i) s += (double)x[(uint64_t)order[i] * width + j];
  centre[(uint64_t)c * kClusterDim + j] = s / (double)(e - b);
}

// The rows by (cluster, first component): perm and the clusters' starts.
void order_by_cluster(const float* x, uint64_t n, uint32_t width, const uint32_t* label,
                      uint32_t K, DeviceBuffer<uint32_t>& perm, DeviceBuffer<uint32_t>& start,
                      cudaStream_t s) {
  DeviceBuffer<unsigned long long> key(n, s), key_sorted(n, s);
  DeviceBuffer<uint32_t> iota(n, s);
  order_key_kernel<<<blocks_for(n, 256), 256, 0, s>>>(x, n, width, label, key.ptr, iota.ptr);
  KG_LAUNCH_CHECK();
  perm.alloc(n, s);
  int bits = 33;
  while (bits < 64 && (1ull << (bits - 32)) <= (uint64_t)K) ++bits;
  size_t temp = 0;
  KG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, key.ptr, key_sorted.ptr, iota.ptr,
                                          perm.ptr, (int)n, 0, bits, s));
  DeviceBuffer<unsigned char> scratch(temp, s);
  KG_CUDA(cub::DeviceRadixSort::SortPairs(scratch.ptr, temp, key.ptr, key_sorted.ptr, iota.ptr,
                                          perm.ptr, (int)n, 0, bits, s));
  start.alloc((uint64_t)K + 1, s);
  key_starts_kernel<<<blocks_for((uint64_t)K + 1, 256), 256, 0, s>>>(key_sorted.ptr, n, K,
                                                                    start.ptr);
  KG_LAUNCH_CHECK();
}

}  // namespace

void nearest_centres(const float* x, uint64_t n, uint32_t width, uint32_t d,
                     const float* centres, const float* cn, uint32_t K, uint32_t* labels,
                     cudaStream_t s) {
  if (!n) return;
  if (d > kClusterDim) fail(KG_ERR_INVALID, "clusters: more than 64 components");
  nearest_centres_kernel<<<(unsigned)((n + kNcRows - 1) / kNcRows), 256, 0, s>>>(
      x, n, width, d, centres, cn, K, labels);
  KG_LAUNCH_CHECK();
}

void cluster_rows(const float* x, uint64_t n, uint32_t width, uint32_t d, uint32_t K,
                  uint32_t iters, uint64_t sample, Clusters& out, cudaStream_t s) {
  if (d > kClusterDim) fail(KG_ERR_INVALID, "clusters: more than 64 components");
  K = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(K, n));
  out.K = K;
  const uint64_t m = std::max<uint64_t>(std::min<uint64_t>(sample, n), K);
  DeviceBuffer<float> xs(m * d, s), cf((uint64_t)K * kClusterDim, s), cn(K, s);
  gather_rows_kernel<<<blocks_for(m * d, 256), 256, 0, s>>>(x, n, width, d, m, xs.ptr);
  KG_LAUNCH_CHECK();
  out.centre.alloc((uint64_t)K * kClusterDim, s);
  seed_centres_kernel<<<blocks_for((uint64_t)K * kClusterDim, 256), 256, 0, s>>>(
      xs.ptr, m, d, K, out.centre.ptr);
  KG_LAUNCH_CHECK();
  DeviceBuffer<uint32_t> lab(m, s);
  for (uint32_t it = 0; it < iters; ++it) {
    centres_f32_kernel<<<blocks_for(K, 128), 128, 0, s>>>(out.centre.ptr, K, cf.ptr, cn.ptr);
    KG_LAUNCH_CHECK();
    nearest_centres(xs.ptr, m, d, d, cf.ptr, cn.ptr, K, lab.ptr, s);
    DeviceBuffer<uint32_t> order, starts;
    order_by_cluster(xs.ptr, m, d, lab.ptr, K, order, starts, s);
    update_centres_kernel<<<K, kClusterDim, 0, s>>>(xs.ptr, d, d, order.ptr, starts.ptr,
                                                    out.centre.ptr);
    KG_LAUNCH_CHECK();
  }
  centres_f32_kernel<<<blocks_for(K, 128), 128, 0, s>>>(out.centre.ptr, K, cf.ptr, cn.ptr);
  KG_LAUNCH_CHECK();
  out.label.alloc(n, s);
  nearest_centres(x, n, width, d, cf.ptr, cn.ptr, K, out.label.ptr, s);
  order_by_cluster(x, n, width, out.label.ptr, K, out.perm, out.start, s);
  update_centres_kernel<<<K, kClusterDim, 0, s>>>(x, width, d, out.perm.ptr, out.start.ptr,
                                                  out.centre.ptr);
  KG_LAUNCH_CHECK();
}

}  // namespace kg
