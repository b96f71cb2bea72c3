// normalize_total / log1p and the seurat HVG statistics pass on the device, and the
// seurat flags on the host (kyto computes them on the host too).
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

#include "kg_internal.cuh"
#include "kg_maps.cuh"

namespace kg {

// Sets *flag when a u32 count is above 2^24 and not a float32 (elementwise.rs:241-257:
// then every value of the block is rounded to float32 before the row sums).
__global__ void inexact_counts_kernel(const uint32_t* values, uint64_t nnz, int* flag) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nnz;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t c = values[i];
    if (c > (1u << 24) && (uint32_t)__uint2float_rn(c) != c) *flag = 1;
  }
}

// The largest gene index of a block (a block's indices must be below its genes).
__global__ void max_index_kernel(const uint32_t* idx, uint64_t nnz, unsigned int* out) {
  unsigned int m = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nnz;
       i += (uint64_t)gridDim.x * blockDim.x)
    m = max(m, idx[i]);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
  if ((threadIdx.x & 31u) == 0) atomicMax(out, m);
}

void check_indices(const uint32_t* d_idx, uint64_t nnz, uint32_t n_genes, cudaStream_t s) {
  if (!nnz) return;
  DeviceBuffer<unsigned int> m(1, s);
  m.zero();
  unsigned blocks = std::min<unsigned>(blocks_for(nnz, 256), 4096);
  max_index_kernel<<<blocks, 256, 0, s>>>(d_idx, nnz, m.ptr);
  KG_LAUNCH_CHECK();
  unsigned int h = 0;
  KG_CUDA(cudaMemcpyAsync(&h, m.ptr, 4, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  if (h >= n_genes)
    fail(KG_ERR_INVALID, "a block holds gene index " + std::to_string(h) + " but has " +
                             std::to_string(n_genes) + " genes");
}

// 8 threads per row: the row's divisor (kg_maps.cuh) then its mapped values.
template <class V>
__global__ void normalize_log1p_kernel(const uint64_t* indptr, const V* values,
                                       uint64_t n_rows, float target32, int normalize,
                                       int do_log1p, const int* inexact, float* out) {
  uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint64_t row = t >> 3;
  unsigned c = threadIdx.x & 7u;
  uint64_t s = 0, e = 0;
  if (row < n_rows) {
    s = indptr[row];
    e = indptr[row + 1];
  }
  float divisor = 1.0f;
  if (normalize) divisor = row_divisor(values, s, e, target32, inexact && *inexact);
  for (uint64_t i = s + c; i < e; i += 8)
    out[i] = mapped_value(values, i, normalize != 0, divisor, do_log1p != 0);
}

template <class V>
void launch_normalize(const uint64_t* indptr, const void* values, uint64_t n_rows,
                      double target_sum, int do_log1p, const int* inexact, float* out,
                      cudaStream_t stream) {
  bool normalize = !std::isnan(target_sum);
  unsigned threads = 256;
  normalize_log1p_kernel<V><<<blocks_for(n_rows * 8, threads), threads, 0, stream>>>(
      indptr, (const V*)values, n_rows, (float)target_sum, normalize ? 1 : 0, do_log1p,
      inexact, out);
  KG_LAUNCH_CHECK();
}

// The device flag of inexact_counts_kernel for a block about to be normalized (left
// unallocated, NULL, when no u32 count of the block can need rounding).
void inexact_flag(const void* d_values, kg_dtype dtype, uint64_t nnz, double target_sum,
                  DeviceBuffer<int>& flag, cudaStream_t stream) {
  if (dtype != KG_U32 || std::isnan(target_sum) || !nnz) return;
  flag.alloc(1, stream);
  flag.zero();
  unsigned threads = 256;
  unsigned blocks = std::min<unsigned>(blocks_for(nnz, threads), 4096);
  inexact_counts_kernel<<<blocks, threads, 0, stream>>>((const uint32_t*)d_values, nnz,
                                                        flag.ptr);
  KG_LAUNCH_CHECK();
}

// Device f32 map outputs of a (device) CSR block.
void map_block(const uint64_t* d_indptr, const void* d_values, kg_dtype dtype,
               uint64_t n_rows, uint64_t nnz, double target_sum, int do_log1p,
               float* d_out, cudaStream_t stream) {
  DeviceBuffer<int> inexact;
  inexact_flag(d_values, dtype, nnz, target_sum, inexact, stream);
  if (dtype == KG_U32)
    launch_normalize<uint32_t>(d_indptr, d_values, n_rows, target_sum, do_log1p, inexact.ptr,
                               d_out, stream);
  else
    launch_normalize<float>(d_indptr, d_values, n_rows, target_sum, do_log1p, inexact.ptr,
                            d_out, stream);
}

// seurat's transformed value and its f32 square (hvg_pass.rs:189-206).
__global__ void expm1_kernel(const float* v, uint64_t nnz, float* t) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nnz;
       i += (uint64_t)gridDim.x * blockDim.x)
    t[i] = (float)expm1((double)v[i]);
}

// colptr[g] = first sorted entry of gene >= g.
__global__ void column_starts_kernel(const uint32_t* sorted_genes, uint64_t nnz,
                                     uint32_t n_genes, uint64_t* colptr) {
  uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (g > n_genes) return;
  uint64_t lo = 0, hi = nnz;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (sorted_genes[mid] < g) lo = mid + 1; else hi = mid;
  }
  colptr[g] = lo;
}

// One warp per gene, its cells in cell order: the bits of kyto's single-leaf fold (two
// f64 sums in one fixed sequential order, made by lane 0). The other lanes keep the next
// 128 values on their way while lane 0 folds the current 128 from shared memory, so the
// fold's dependent adds, not the loads, set the pace; many genes' warps share an SM.
constexpr int kMomentWarps = 4;
constexpr int kMomentChunk = 128;

__global__ void __launch_bounds__(kMomentWarps * 32)
gene_moments_kernel(const uint64_t* colptr, const float* t, uint32_t n_genes, double* sums,
                    double* squares, uint64_t* positives) {
  __shared__ float buf[kMomentWarps][2][kMomentChunk];
  const unsigned lane = threadIdx.x & 31u, wi = threadIdx.x >> 5;
  const uint32_t g = blockIdx.x * kMomentWarps + wi;
  if (g >= n_genes) return;
  const uint64_t a = colptr[g], e = colptr[g + 1];
  float nxt[kMomentChunk / 32];
  auto load = [&](uint64_t c0) {
#pragma unroll
    for (int m = 0; m < kMomentChunk / 32; ++m) {
      const uint64_t i = c0 + m * 32 + lane;
      nxt[m] = i < e ? __ldg(t + i) : 0.0f;
    }
  };
  auto stash = [&](int half) {
#pragma unroll
    for (int m = 0; m < kMomentChunk / 32; ++m) buf[wi][half][m * 32 + lane] = nxt[m];
  };
  double s = 0.0, q = 0.0;
  uint64_t p = 0;
  load(a);
  stash(0);
  __syncwarp();
  int half = 0;
  for (uint64_t c0 = a; c0 < e; c0 += kMomentChunk, half ^= 1) {
    if (c0 + kMomentChunk < e) load(c0 + kMomentChunk);
    if (lane == 0) {
      const uint32_t n = e - c0 < (uint64_t)kMomentChunk ? (uint32_t)(e - c0) : (uint32_t)kMomentChunk;
      const float* v = buf[wi][half];
#pragma unroll 8
      for (uint32_t j = 0; j < n; ++j) {
        const float x = v[j];
        if (x > 0.0f) ++p;  // t > 0 exactly when the log1p value > 0 (expm1 keeps sign)
        s = __dadd_rn(s, (double)x);
        q = __dadd_rn(q, (double)__fmul_rn(x, x));
      }
    }
    __syncwarp();
    if (c0 + kMomentChunk < e) stash(half ^ 1);
    __syncwarp();
  }
  if (lane == 0) {
    sums[g] = s;
    squares[g] = q;
    positives[g] = p;
  }
}

int bits_for(uint32_t n) {
  int b = 1;
  while (b < 32 && (1ull << b) < (uint64_t)n) ++b;
  return b;
}

// Stable sort of (gene, payload) by gene: each gene's payloads stay in cell order.
template <class P>
void sort_by_gene(const uint32_t* genes, const P* payload, uint64_t nnz, uint32_t n_genes,
                  DeviceBuffer<uint32_t>& genes_out, DeviceBuffer<P>& payload_out,
                  cudaStream_t stream) {
  if (nnz > (uint64_t)std::numeric_limits<int>::max())
    fail(KG_ERR_INVALID, "a block of more than 2^31 stored values");
  genes_out.alloc(nnz, stream);
  payload_out.alloc(nnz, stream);
  size_t temp = 0;
  int end_bit = bits_for(n_genes + 1);
  KG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, genes, genes_out.ptr, payload,
                                          payload_out.ptr, (int)nnz, 0, end_bit, stream));
  DeviceBuffer<unsigned char> scratch(temp, stream);
  KG_CUDA(cub::DeviceRadixSort::SortPairs(scratch.ptr, temp, genes, genes_out.ptr, payload,
                                          payload_out.ptr, (int)nnz, 0, end_bit, stream));
}

template void sort_by_gene<uint32_t>(const uint32_t*, const uint32_t*, uint64_t, uint32_t,
                                     DeviceBuffer<uint32_t>&, DeviceBuffer<uint32_t>&,
                                     cudaStream_t);
template void sort_by_gene<uint64_t>(const uint32_t*, const uint64_t*, uint64_t, uint32_t,
                                     DeviceBuffer<uint32_t>&, DeviceBuffer<uint64_t>&,
                                     cudaStream_t);

void column_starts(const uint32_t* sorted_genes, uint64_t nnz, uint32_t n_genes,
                   uint64_t* colptr, cudaStream_t stream) {
  column_starts_kernel<<<blocks_for((uint64_t)n_genes + 1, 256), 256, 0, stream>>>(
      sorted_genes, nnz, n_genes, colptr);
  KG_LAUNCH_CHECK();
}

// ------------------------------------------------------------------ seurat (host) ----

double kahan_mean(const std::vector<double>& values) {
  double sum = 0.0, comp = 0.0;
  uint64_t count = 0;
  for (double v : values) {
    if (std::isnan(v)) continue;
    ++count;
    double y = v - comp;
    double t = sum + y;
    comp = t - sum - y;
    if (std::isnan(comp)) comp = 0.0;
    sum = t;
  }
  return count == 0 ? NAN : sum / (double)count;
}

double welford_std(const std::vector<double>& values) {
  uint64_t count = 0;
  double mean = 0.0, squared = 0.0;
  for (double v : values) {
    if (std::isnan(v)) continue;
    ++count;
    double prev = mean;
    mean += (v - prev) / (double)count;
    squared += (v - mean) * (v - prev);
  }
  return count <= 1 ? NAN : std::sqrt(squared / (double)(count - 1));
}

}  // namespace kg

using namespace kg;

extern "C" {

kg_status kg_normalize_log1p(kg_ctx* ctx, const uint64_t* indptr, const void* values,
                             kg_dtype dtype, uint64_t n_rows, double target_sum,
                             int32_t log1p, float* out) {
  return guarded([&] {
    if (!ctx || !indptr || (!values && n_rows) || !out)
      fail(KG_ERR_INVALID, "kg_normalize_log1p: NULL argument");
    if (dtype != KG_U32 && dtype != KG_F32) fail(KG_ERR_INVALID, "unknown dtype");
    use_device(ctx);
    cudaStream_t s = ctx->stream;
    DeviceBuffer<uint64_t> hp;
    const uint64_t* d_indptr = device_view(indptr, n_rows + 1, hp, s);
    uint64_t nnz = 0;
    KG_CUDA(cudaMemcpyAsync(&nnz, d_indptr + n_rows, 8, cudaMemcpyDefault, s));
    KG_CUDA(cudaStreamSynchronize(s));
    DeviceBuffer<uint32_t> hv;
    const void* d_values = device_view((const uint32_t*)values, nnz, hv, s);
    DeviceBuffer<float> ho;
    bool out_dev = is_device_pointer(out);
    float* d_out = out;
    if (!out_dev) {
      ho.alloc(nnz, s);
      d_out = ho.ptr;
    }
    map_block(d_indptr, d_values, dtype, n_rows, nnz, target_sum, log1p, d_out, s);
    if (!out_dev && nnz)
      KG_CUDA(cudaMemcpyAsync(out, d_out, nnz * 4, cudaMemcpyDeviceToHost, s));
    wait_stream(ctx, s);
  });
}

kg_status kg_hvg_moments(kg_ctx* ctx, const uint64_t* indptr, const uint32_t* indices,
                         const void* values, kg_dtype dtype, uint64_t n_rows,
                         uint32_t n_genes, double target_sum, int32_t log1p,
                         double* sums, double* sums_of_squares, uint64_t* positives) {
  return guarded([&] {
    if (!ctx || !indptr || !sums || !sums_of_squares || !positives)
      fail(KG_ERR_INVALID, "kg_hvg_moments: NULL argument");
    if (dtype != KG_U32 && dtype != KG_F32) fail(KG_ERR_INVALID, "unknown dtype");
    use_device(ctx);
    cudaStream_t s = ctx->stream;
    DeviceBuffer<uint64_t> hp;
    const uint64_t* d_indptr = device_view(indptr, n_rows + 1, hp, s);
    uint64_t nnz = 0;
    KG_CUDA(cudaMemcpyAsync(&nnz, d_indptr + n_rows, 8, cudaMemcpyDefault, s));
    KG_CUDA(cudaStreamSynchronize(s));
    DeviceBuffer<uint32_t> hi, hv;
    const uint32_t* d_idx = device_view(indices, nnz, hi, s);
    const void* d_values = device_view((const uint32_t*)values, nnz, hv, s);
    check_indices(d_idx, nnz, n_genes, s);
    DeviceBuffer<float> mapped(nnz, s), t(nnz, s);
    map_block(d_indptr, d_values, dtype, n_rows, nnz, target_sum, log1p, mapped.ptr, s);
    if (nnz) {
      unsigned blocks = std::min<unsigned>(blocks_for(nnz, 256), 8192);
      expm1_kernel<<<blocks, 256, 0, s>>>(mapped.ptr, nnz, t.ptr);
      KG_LAUNCH_CHECK();
    }
    mapped.reset();
    DeviceBuffer<uint32_t> genes_sorted, t_sorted;
    sort_by_gene<uint32_t>(d_idx, (const uint32_t*)t.ptr, nnz, n_genes, genes_sorted,
                           t_sorted, s);
    t.reset();
    DeviceBuffer<uint64_t> colptr((uint64_t)n_genes + 1, s);
    column_starts(genes_sorted.ptr, nnz, n_genes, colptr.ptr, s);
    DeviceBuffer<double> dsum(n_genes, s), dsq(n_genes, s);
    DeviceBuffer<uint64_t> dpos(n_genes, s);
    gene_moments_kernel<<<(n_genes + kMomentWarps - 1) / kMomentWarps, kMomentWarps * 32, 0,
                          s>>>(colptr.ptr, (const float*)t_sorted.ptr, n_genes, dsum.ptr,
                               dsq.ptr, dpos.ptr);
    KG_LAUNCH_CHECK();
    KG_CUDA(cudaMemcpyAsync(sums, dsum.ptr, n_genes * 8ull, cudaMemcpyDefault, s));
    KG_CUDA(cudaMemcpyAsync(sums_of_squares, dsq.ptr, n_genes * 8ull, cudaMemcpyDefault, s));
    KG_CUDA(cudaMemcpyAsync(positives, dpos.ptr, n_genes * 8ull, cudaMemcpyDefault, s));
    wait_stream(ctx, s);
  });
}

kg_status kg_hvg_seurat(const double* sums, const double* sums_of_squares,
                        const uint64_t* positives, uint64_t n_cells, uint32_t n_genes,
                        int64_t n_top_genes, double* means_out, double* dispersions_out,
                        double* normalized_out, uint8_t* flags_out) {
  (void)positives;  // seurat without batches keeps every gene (hvg.rs:290-293)
  return guarded([&] {
    if (!sums || !sums_of_squares || !means_out || !dispersions_out || !normalized_out ||
        !flags_out)
      fail(KG_ERR_INVALID, "kg_hvg_seurat: NULL argument");
    const int kBins = 20;  // hvg.rs:34
    double n = (double)n_cells;
    std::vector<double> mean(n_genes), disp(n_genes), norm(n_genes, NAN);
    for (uint32_t g = 0; g < n_genes; ++g) {
      // statistics.rs:153-168 (variances with ddof=1), hvg.rs:295-308.
      double m = sums[g] / n;
      double var = sums_of_squares[g] / n - m * m;
      if (n_cells != 1) var = var * (n / (n - 1.0));
      if (m == 0.0) m = 1e-12;
      double d = var / m;
      if (d == 0.0) d = NAN;
      d = std::log(d);
      mean[g] = std::log1p(m);
      disp[g] = d;
    }
    // hvg.rs:393-425: 20 equal-width bins (pd.cut).
    double lo = INFINITY, hi = -INFINITY;
    bool any = false;
    for (double m : mean)
      if (!std::isnan(m)) {
        lo = std::min(lo, m);
        hi = std::max(hi, m);
        any = true;
      }
    std::vector<int> bins(n_genes, -1);
    if (any) {
      std::vector<double> edges(kBins + 1);
      auto linspace = [&](double a, double b) {
        double step = (b - a) / (double)kBins;
        for (int i = 0; i <= kBins; ++i) edges[i] = (double)i * step + a;
        edges[kBins] = b;
      };
      if (lo == hi) {
        linspace(lo - (lo == 0.0 ? 0.001 : 0.001 * std::fabs(lo)),
                 hi + (hi == 0.0 ? 0.001 : 0.001 * std::fabs(hi)));
      } else {
        linspace(lo, hi);
        edges[0] -= (hi - lo) * 0.001;
      }
      for (uint32_t g = 0; g < n_genes; ++g) {
        if (std::isnan(mean[g])) continue;
        int index = (int)(std::lower_bound(edges.begin(), edges.end(), mean[g]) -
                          edges.begin());
        index = std::max(index, 1);
        if (index < (int)edges.size()) bins[g] = index - 1;
      }
    }
    // hvg.rs:501-535: z-score of the dispersion in its bin.
    std::vector<std::vector<double>> members(kBins);
    for (uint32_t g = 0; g < n_genes; ++g)
      if (bins[g] >= 0) members[bins[g]].push_back(disp[g]);
    std::vector<std::pair<double, double>> stats(kBins);
    for (int b = 0; b < kBins; ++b) {
      double avg = kahan_mean(members[b]);
      double dev = welford_std(members[b]);
      stats[b] = std::isnan(dev) ? std::make_pair(0.0, avg) : std::make_pair(avg, dev);
    }
    for (uint32_t g = 0; g < n_genes; ++g)
      if (bins[g] >= 0) norm[g] = (disp[g] - stats[bins[g]].first) / stats[bins[g]].second;
    // hvg.rs:320-349: top n by >= cutoff, or scanpy's cutoffs.
    auto nan_to_num = [](double v, double nan) {
      if (std::isnan(v)) return nan;
      if (v == INFINITY) return std::numeric_limits<double>::max();
      if (v == -INFINITY) return std::numeric_limits<double>::lowest();
      return v;
    };
    if (n_top_genes >= 0) {
      std::vector<double> finite;
      for (double v : norm)
        if (!std::isnan(v)) finite.push_back(v);
      uint64_t count = std::min<uint64_t>((uint64_t)n_top_genes,
                                          std::min<uint64_t>(n_genes, finite.size()));
      if (count == 0) {
        for (uint32_t g = 0; g < n_genes; ++g) flags_out[g] = 0;
      } else {
        std::sort(finite.begin(), finite.end(), [](double a, double b) { return a > b; });
        double cutoff = finite[count - 1];
        for (uint32_t g = 0; g < n_genes; ++g)
          flags_out[g] = nan_to_num(norm[g], -INFINITY) >= cutoff ? 1 : 0;
      }
    } else {
      for (uint32_t g = 0; g < n_genes; ++g) {
        double z = nan_to_num(norm[g], 0.0);
        flags_out[g] = (mean[g] > 0.0125 && mean[g] < 3.0 && z > 0.5 && z < INFINITY) ? 1 : 0;
      }
    }
    for (uint32_t g = 0; g < n_genes; ++g) {
      means_out[g] = mean[g];
      dispersions_out[g] = disp[g];
      normalized_out[g] = norm[g];
    }
  });
}

}  // extern "C"

// ------------------------------------------ seurat moments in fixed scratch ----------

namespace kg {

constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// The limits of kg_hvg_moments_noalloc and the layout of its scratch (byte offsets):
// two flags, the sort's key and payload double buffers, the per-gene arrays, the radix
// sort's temporary storage. 22.1 MB in all.
constexpr uint64_t kNoAllocMaxValues = 1ull << 20;  // stored values of one block
constexpr uint32_t kNoAllocMaxGenes = 1u << 16;
constexpr size_t kNoAllocValues = align256(kNoAllocMaxValues * 4);
constexpr size_t kNoAllocGenes = align256(((size_t)kNoAllocMaxGenes + 1) * 8);
constexpr size_t kNoAllocKeys0 = 256;
constexpr size_t kNoAllocKeys1 = kNoAllocKeys0 + kNoAllocValues;
constexpr size_t kNoAllocVals0 = kNoAllocKeys1 + kNoAllocValues;
constexpr size_t kNoAllocVals1 = kNoAllocVals0 + kNoAllocValues;
constexpr size_t kNoAllocColptr = kNoAllocVals1 + kNoAllocValues;
constexpr size_t kNoAllocSums = kNoAllocColptr + kNoAllocGenes;
constexpr size_t kNoAllocSquares = kNoAllocSums + kNoAllocGenes;
constexpr size_t kNoAllocPositives = kNoAllocSquares + kNoAllocGenes;
constexpr size_t kNoAllocSort = kNoAllocPositives + kNoAllocGenes;
constexpr size_t kNoAllocSortBytes = 4u << 20;
constexpr size_t kNoAllocBytes = kNoAllocSort + kNoAllocSortBytes;

// One array per device (this module's static device memory), shared by every call on
// that device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocDevices = 64;

// The scratch's device address on `device` (which must be current). The first call on
// a device resolves it with cudaGetSymbolAddress, which loads this module there, and
// checks that the radix sort's storage for the largest block fits its slot.
unsigned char* noalloc_scratch(int device) {
  static std::mutex mu;
  static unsigned char* resolved[kNoAllocDevices] = {};
  if (device < 0 || device >= kNoAllocDevices)
    fail(KG_ERR_INVALID, "kg_hvg_moments_noalloc: device ordinal above 63");
  std::lock_guard<std::mutex> lock(mu);
  if (resolved[device]) return resolved[device];
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) fail_cuda(e, "cudaGetSymbolAddress (fixed scratch)", __FILE__, __LINE__);
  size_t temp = 0;
  cub::DoubleBuffer<uint32_t> keys(nullptr, nullptr), vals(nullptr, nullptr);
  KG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, keys, vals, (int)kNoAllocMaxValues, 0,
                                          bits_for(kNoAllocMaxGenes + 1)));
  if (temp > kNoAllocSortBytes)
    fail(KG_ERR_DEVICE, "kg_hvg_moments_noalloc: the radix sort wants " +
                            std::to_string(temp) + " bytes, above its fixed slot");
  resolved[device] = (unsigned char*)p;
  return resolved[device];
}

}  // namespace kg

extern "C" {

kg_status kg_hvg_moments_noalloc(kg_ctx* ctx, const uint64_t* indptr, const uint32_t* indices,
                                 const void* values, kg_dtype dtype, uint64_t n_rows,
                                 uint32_t n_genes, double target_sum, int32_t log1p,
                                 double* sums, double* sums_of_squares, uint64_t* positives) {
  return guarded([&] {
    if (!ctx || !indptr || !sums || !sums_of_squares || !positives)
      fail(KG_ERR_INVALID, "kg_hvg_moments_noalloc: NULL argument");
    if (dtype != KG_U32 && dtype != KG_F32) fail(KG_ERR_INVALID, "unknown dtype");
    if (n_genes > kNoAllocMaxGenes)
      fail(KG_ERR_INVALID, "kg_hvg_moments_noalloc: " + std::to_string(n_genes) +
                               " genes, above its limit of " +
                               std::to_string(kNoAllocMaxGenes) + " (use kg_hvg_moments)");
    use_device(ctx);
    if (!is_device_pointer(indptr))
      fail(KG_ERR_INVALID, "kg_hvg_moments_noalloc: indptr must be device memory");
    unsigned char* base = noalloc_scratch(ctx->device);
    cudaStream_t s = ctx->stream;
    uint64_t nnz = 0;
    KG_CUDA(cudaMemcpyAsync(&nnz, indptr + n_rows, 8, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    if (nnz > kNoAllocMaxValues)
      fail(KG_ERR_INVALID, "kg_hvg_moments_noalloc: a block of " + std::to_string(nnz) +
                               " stored values, above its limit of " +
                               std::to_string(kNoAllocMaxValues) + " (use kg_hvg_moments)");
    if (nnz && (!is_device_pointer(indices) || !is_device_pointer(values)))
      fail(KG_ERR_INVALID, "kg_hvg_moments_noalloc: indices and values must be device memory");
    int* inexact = (int*)base;
    unsigned int* max_index = (unsigned int*)(base + 4);
    uint32_t* keys0 = (uint32_t*)(base + kNoAllocKeys0);
    uint32_t* keys1 = (uint32_t*)(base + kNoAllocKeys1);
    float* vals0 = (float*)(base + kNoAllocVals0);
    float* vals1 = (float*)(base + kNoAllocVals1);
    uint64_t* colptr = (uint64_t*)(base + kNoAllocColptr);
    double* dsum = (double*)(base + kNoAllocSums);
    double* dsq = (double*)(base + kNoAllocSquares);
    uint64_t* dpos = (uint64_t*)(base + kNoAllocPositives);
    KG_CUDA(cudaMemsetAsync(base, 0, 8, s));  // both flags start at zero
    cub::DoubleBuffer<uint32_t> keys(keys0, keys1), vals((uint32_t*)vals0, (uint32_t*)vals1);
    if (nnz) {
      unsigned blocks = std::min<unsigned>(blocks_for(nnz, 256), 4096);
      max_index_kernel<<<blocks, 256, 0, s>>>(indices, nnz, max_index);
      KG_LAUNCH_CHECK();
      unsigned int h = 0;
      KG_CUDA(cudaMemcpyAsync(&h, max_index, 4, cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaStreamSynchronize(s));
      if (h >= n_genes)
        fail(KG_ERR_INVALID, "a block holds gene index " + std::to_string(h) + " but has " +
                                 std::to_string(n_genes) + " genes");
      const int* flag = nullptr;
      if (dtype == KG_U32 && !std::isnan(target_sum)) {
        inexact_counts_kernel<<<blocks, 256, 0, s>>>((const uint32_t*)values, nnz, inexact);
        KG_LAUNCH_CHECK();
        flag = inexact;
      }
      if (dtype == KG_U32)
        launch_normalize<uint32_t>(indptr, values, n_rows, target_sum, log1p, flag, vals0, s);
      else
        launch_normalize<float>(indptr, values, n_rows, target_sum, log1p, flag, vals0, s);
      expm1_kernel<<<std::min<unsigned>(blocks_for(nnz, 256), 8192), 256, 0, s>>>(vals0, nnz,
                                                                                 vals0);
      KG_LAUNCH_CHECK();
      // The sort may write either half of each double buffer: the keys start as a copy.
      KG_CUDA(cudaMemcpyAsync(keys0, indices, nnz * 4, cudaMemcpyDeviceToDevice, s));
      size_t temp = 0;
      int end_bit = bits_for(n_genes + 1);
      KG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, keys, vals, (int)nnz, 0, end_bit,
                                              s));
      if (temp > kNoAllocSortBytes)
        fail(KG_ERR_DEVICE, "kg_hvg_moments_noalloc: the radix sort wants " +
                                std::to_string(temp) + " bytes, above its fixed slot");
      temp = kNoAllocSortBytes;
      KG_CUDA(cub::DeviceRadixSort::SortPairs(base + kNoAllocSort, temp, keys, vals, (int)nnz,
                                              0, end_bit, s));
    }
    if (n_genes) {
      column_starts(keys.Current(), nnz, n_genes, colptr, s);
      gene_moments_kernel<<<(n_genes + kMomentWarps - 1) / kMomentWarps, kMomentWarps * 32, 0,
                            s>>>(colptr, (const float*)vals.Current(), n_genes, dsum, dsq, dpos);
      KG_LAUNCH_CHECK();
      KG_CUDA(cudaMemcpyAsync(sums, dsum, n_genes * 8ull, cudaMemcpyDefault, s));
      KG_CUDA(cudaMemcpyAsync(sums_of_squares, dsq, n_genes * 8ull, cudaMemcpyDefault, s));
      KG_CUDA(cudaMemcpyAsync(positives, dpos, n_genes * 8ull, cudaMemcpyDefault, s));
    }
    wait_stream(ctx, s);
  });
}

}  // extern "C"
