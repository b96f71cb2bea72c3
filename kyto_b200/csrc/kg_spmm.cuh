// The PCA's sparse x dense products over the held input (first, general version:
// f64 accumulation on the SIMT pipes).
//   row_product:         out = X M - 1 offsets^T   (CSR, one warp per row)
//   transposed_product:  out = X^T D               (gene-major segments, fixed order)
#pragma once

#include <algorithm>
#include <vector>

#include "kg_internal.cuh"

namespace kg {

constexpr uint64_t kSegment = 2048;  // gene-major entries one CTA sums in order

__global__ void iota_kernel(uint32_t* p, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = (uint32_t)i;
}

inline void iota_fill(uint32_t* p, uint64_t n, cudaStream_t s) {
  if (!n) return;
  iota_kernel<<<std::min<unsigned>(blocks_for(n, 256), 16384), 256, 0, s>>>(p, n);
  KG_LAUNCH_CHECK();
}

// out[r, j] = -offsets[j] + sum over row r's entries (in gene order) v * m[gene, j]
// (kyto's `project`, pca.rs:548-586). m: g x w row-major. One warp per row, each lane
// up to 4 columns per sweep over the row.
__global__ void row_product_kernel(const uint64_t* indptr, const uint32_t* col,
                                   const float* val, uint64_t n, const double* m,
                                   const double* offsets, uint32_t w, double* out) {
  uint64_t row = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  if (row >= n) return;
  uint64_t s = indptr[row], e = indptr[row + 1];
  for (uint32_t j0 = 0; j0 < w; j0 += 128) {
    double acc[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      uint32_t j = j0 + lane + 32 * t;
      acc[t] = j < w ? -offsets[j] : 0.0;
    }
    for (uint64_t i = s; i < e; ++i) {
      uint32_t c = col[i];
      double v = (double)val[i];
      const double* mr = m + (uint64_t)c * w;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        uint32_t j = j0 + lane + 32 * t;
        if (j < w) acc[t] = fma(v, mr[j], acc[t]);
      }
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      uint32_t j = j0 + lane + 32 * t;
      if (j < w) out[row * w + j] = acc[t];
    }
  }
}

inline void row_product(const uint64_t* indptr, const uint32_t* col, const float* val,
                        uint64_t n, const double* m, const double* offsets, uint32_t w,
                        double* out, cudaStream_t s) {
  row_product_kernel<<<blocks_for(n * 32, 256), 256, 0, s>>>(indptr, col, val, n, m,
                                                             offsets, w, out);
  KG_LAUNCH_CHECK();
}

// One segment's sum of v * d[row, j] over its entries, in order.
__global__ void segment_product_kernel(const uint64_t* seg_begin, const uint64_t* seg_end,
                                       const uint32_t* row, const float* val,
                                       const double* d, uint32_t w, double* partial) {
  uint64_t seg = blockIdx.x;
  uint64_t a = seg_begin[seg], b = seg_end[seg];
  for (uint32_t j = threadIdx.x; j < w; j += blockDim.x) {
    double acc = 0.0;
    for (uint64_t i = a; i < b; ++i) acc = fma((double)val[i], d[(uint64_t)row[i] * w + j], acc);
    partial[seg * w + j] = acc;
  }
}

// out[j * g + gene] = the gene's segments summed in order (column-major g x w).
__global__ void segment_reduce_kernel(const uint64_t* gene_seg, const double* partial,
                                      uint32_t g, uint32_t w, double* out) {
  uint32_t gene = blockIdx.x;
  uint64_t a = gene_seg[gene], b = gene_seg[gene + 1];
  for (uint32_t j = threadIdx.x; j < w; j += blockDim.x) {
    double acc = 0.0;
    for (uint64_t sg = a; sg < b; ++sg) acc = __dadd_rn(acc, partial[sg * w + j]);
    out[(uint64_t)j * g + gene] = acc;
  }
}

// One segment's sum of (v - mean)^2.
__global__ void segment_squares_kernel(const uint64_t* seg_begin, const uint64_t* seg_end,
                                       const uint32_t* seg_gene, const float* val,
                                       const double* means, uint64_t n_segs,
                                       double* partial) {
  uint64_t seg = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (seg >= n_segs) return;
  double mu = means[seg_gene[seg]];
  double acc = 0.0;
  for (uint64_t i = seg_begin[seg]; i < seg_end[seg]; ++i) {
    double c = (double)val[i] - mu;
    acc = fma(c, c, acc);
  }
  partial[seg] = acc;
}

// The held input gene by gene: each gene's entries in cell order, cut into segments of
// at most kSegment entries (a gene's segments are consecutive).
struct GeneMajor {
  DeviceBuffer<uint64_t> colptr;
  DeviceBuffer<uint32_t> row;
  DeviceBuffer<float> val;
  DeviceBuffer<uint64_t> seg_begin, seg_end, gene_seg;
  DeviceBuffer<uint32_t> seg_gene;
  uint64_t n_segs = 0;

  void build_segments(uint32_t g, uint64_t nnz, cudaStream_t s) {
    (void)nnz;
    std::vector<uint64_t> cp(g + 1);
    KG_CUDA(cudaMemcpyAsync(cp.data(), colptr.ptr, (g + 1) * 8ull, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    std::vector<uint64_t> b, e, gs(g + 1);
    std::vector<uint32_t> sg;
    for (uint32_t gene = 0; gene < g; ++gene) {
      gs[gene] = b.size();
      for (uint64_t a = cp[gene]; a < cp[gene + 1]; a += kSegment) {
        b.push_back(a);
        e.push_back(std::min(cp[gene + 1], a + kSegment));
        sg.push_back(gene);
      }
    }
    gs[g] = b.size();
    n_segs = b.size();
    seg_begin.alloc(n_segs, s);
    seg_end.alloc(n_segs, s);
    seg_gene.alloc(n_segs, s);
    gene_seg.alloc(g + 1, s);
    if (n_segs) {
      KG_CUDA(cudaMemcpyAsync(seg_begin.ptr, b.data(), n_segs * 8, cudaMemcpyHostToDevice, s));
      KG_CUDA(cudaMemcpyAsync(seg_end.ptr, e.data(), n_segs * 8, cudaMemcpyHostToDevice, s));
      KG_CUDA(cudaMemcpyAsync(seg_gene.ptr, sg.data(), n_segs * 4, cudaMemcpyHostToDevice, s));
    }
    KG_CUDA(cudaMemcpyAsync(gene_seg.ptr, gs.data(), (g + 1) * 8ull, cudaMemcpyHostToDevice, s));
    KG_CUDA(cudaStreamSynchronize(s));
  }

  // out (g x w column-major) = X^T d, d n x w row-major.
  void transposed_product(const double* d, uint32_t w, uint32_t g, double* out,
                          cudaStream_t s) {
    DeviceBuffer<double> partial(std::max<uint64_t>(n_segs, 1) * w, s);
    unsigned threads = std::min<unsigned>(256, ((w + 31) / 32) * 32);
    if (n_segs) {
      segment_product_kernel<<<(unsigned)n_segs, threads, 0, s>>>(
          seg_begin.ptr, seg_end.ptr, row.ptr, val.ptr, d, w, partial.ptr);
      KG_LAUNCH_CHECK();
    }
    segment_reduce_kernel<<<g, threads, 0, s>>>(gene_seg.ptr, partial.ptr, g, w, out);
    KG_LAUNCH_CHECK();
  }

  void centred_squares(const double* means, uint32_t g, double* out, cudaStream_t s) {
    DeviceBuffer<double> partial(std::max<uint64_t>(n_segs, 1), s);
    if (n_segs) {
      segment_squares_kernel<<<blocks_for(n_segs, 128), 128, 0, s>>>(
          seg_begin.ptr, seg_end.ptr, seg_gene.ptr, val.ptr, means, n_segs, partial.ptr);
      KG_LAUNCH_CHECK();
    }
    segment_reduce_kernel<<<g, 32, 0, s>>>(gene_seg.ptr, partial.ptr, g, 1, out);
    KG_LAUNCH_CHECK();
  }
};

}  // namespace kg
