// The PCA session: kyto's streamed randomized block Krylov PCA
// (crates/kyto-exec/src/pca.rs, pca_dense.rs) with the input held in HBM.
//
// Layout in HBM: the held input is a CSR (u64 row pointers, u32 PCA-gene positions,
// f32 values after normalize/log1p) plus, built once per run, its gene-major twin
// (CSC: u32 rows, f32 values) cut into fixed segments so that X^T D runs as
// independent, deterministic per-segment sums. Dense g x w matrices (the basis, the
// products, the blocks) are f64 column-major for cuBLAS/cuSOLVER; per-cell matrices
// (Omega, W, the embedding rows) are row-major n x w.
#include <cub/device/device_scan.cuh>
#include <cuda_fp16.h>

#include <cstdlib>
#include <string>

#include <algorithm>
#include <atomic>
#include <memory>
#include <exception>
#include <thread>
#include <cmath>
#include <vector>

#include "kg_internal.cuh"
#include "kg_knn.cuh"
#include "kg_maps.cuh"
#include "kg_spmm.cuh"
#include "kg_spmm_tc.cuh"
#include "kg_tiles.cuh"

namespace kg {

// Declared in kg_maps.cu.
void inexact_flag(const void* d_values, kg_dtype dtype, uint64_t nnz, double target_sum,
                  DeviceBuffer<int>& flag, cudaStream_t stream);
template <class P>
void sort_by_gene(const uint32_t* genes, const P* payload, uint64_t nnz, uint32_t n_genes,
                  DeviceBuffer<uint32_t>& genes_out, DeviceBuffer<P>& payload_out,
                  cudaStream_t stream);
void column_starts(const uint32_t* sorted_genes, uint64_t nnz, uint32_t n_genes,
                   uint64_t* colptr, cudaStream_t stream);
void check_indices(const uint32_t* d_idx, uint64_t nnz, uint32_t n_genes, cudaStream_t s);

constexpr uint32_t kNoGene = 0xFFFFFFFFu;
constexpr int kPasses = 11;            // 2 + PCA_POWER_ITERATIONS (pca.rs:123)
constexpr uint32_t kOversamples = 10;  // PCA_OVERSAMPLES (estimate.rs:153)
constexpr double kDropTolerance = 1e-10;  // pca_dense.rs:30

// ----------------------------------------------------------------- pack kernels ----

// Kept entries per row (genes mapped into the PCA's set), one warp per row, and the
// row's normalize divisor (kg_maps.cuh: every 8-lane group of the warp sums the row in
// kyto's lane order and gets the same divisor) when divisor is not NULL.
// A gene index at or past the stream's genes is never kept and sets *bad (an
// asynchronous push checks the indices only when the run starts).
template <class V>
__global__ void count_kept_kernel(const uint64_t* indptr, const uint32_t* idx, const V* values,
                                  uint64_t n_rows, const uint32_t* gene_map, uint32_t n_genes,
                                  float target32, const int* inexact, uint64_t* kept,
                                  float* divisor, unsigned int* bad) {
  uint64_t row = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  if (row >= n_rows) return;  // whole warps leave together
  uint64_t s = indptr[row], e = indptr[row + 1];
  uint64_t count = 0;
  for (uint64_t i = s + lane; i < e; i += 32) {
    const uint32_t gi = idx[i];
    if (gi >= n_genes) {
      atomicOr(bad, 1u);
      continue;
    }
    count += (gene_map == nullptr || gene_map[gi] != kNoGene);
  }
  for (int o = 16; o; o >>= 1) count += __shfl_down_sync(0xFFFFFFFFu, count, o);
  if (lane == 0) kept[row] = count;
  if (divisor) {
    float d = row_divisor(values, s, e, target32, inexact && *inexact);
    if (lane == 0) divisor[row] = d;
  }
}

// Writes each row's kept entries in order at out_ptr[row] (warp per row, ballot
// compaction keeps the row's gene order), each value mapped on the way: f32(v) / the
// row's divisor (when divisor is not NULL), then log1p (kg_maps.cuh).
template <class V>
__global__ void write_kept_kernel(const uint64_t* indptr, const uint32_t* idx, const V* values,
                                  const float* divisor, int do_log1p, uint64_t n_rows,
                                  const uint32_t* gene_map, uint32_t n_genes,
                                  const uint64_t* out_ptr, uint32_t* col, float* val) {
  uint64_t row = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  if (row >= n_rows) return;
  uint64_t s = indptr[row], e = indptr[row + 1];
  uint64_t base = out_ptr[row];
  const float d = divisor ? divisor[row] : 1.0f;
  for (uint64_t i0 = s; i0 < e; i0 += 32) {
    uint64_t i = i0 + lane;
    bool in = i < e;
    uint32_t p = kNoGene;
    if (in && idx[i] < n_genes) p = gene_map ? gene_map[idx[i]] : idx[i];
    bool keep = in && p != kNoGene;
    unsigned ballot = __ballot_sync(0xFFFFFFFFu, keep);
    if (keep) {
      uint64_t at = base + __popc(ballot & ((1u << lane) - 1u));
      col[at] = p;
      val[at] = mapped_value(values, i, divisor != nullptr, d, do_log1p != 0);
    }
    base += __popc(ballot);
  }
}

// The row of each held entry (for the gene-major twin).
__global__ void row_of_kernel(const uint64_t* indptr, uint64_t n_rows, uint32_t* row_of) {
  uint64_t row = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  if (row >= n_rows) return;
  for (uint64_t i = indptr[row] + lane; i < indptr[row + 1]; i += 32) row_of[i] = (uint32_t)row;
}

__global__ void gather_csc_kernel(const uint32_t* perm, const uint32_t* row_of,
                                  const float* val, uint64_t nnz, uint32_t* csc_row,
                                  float* csc_val) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nnz;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t e = perm[i];
    csc_row[i] = row_of[e];
    csc_val[i] = val[e];
  }
}

// Cell positions first, first + 1, ... (a block pushed without its cells' positions).
__global__ void iota64_kernel(uint64_t* out, uint64_t n, uint64_t first) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = first + i;
}

__global__ void add_offset_kernel(uint64_t* p, uint64_t n, uint64_t offset) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) p[i] += offset;
}

// --------------------------------------------------------------- small kernels -----

// Omega's rows (pca.rs:936-950): out is n x width row-major.
__device__ __forceinline__ uint64_t splitmix_mix(uint64_t v) {
  v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
  v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
  return v ^ (v >> 31);
}

// A cell's Omega stream: seeded from (seed, the cell's table position), then one
// value in [-1, 1) per column (pca.rs:936-950). Every kernel that needs Omega draws it
// from these two functions.
__device__ __forceinline__ uint64_t omega_state(uint64_t seed, uint64_t cell) {
  return splitmix_mix(seed ^ splitmix_mix(cell + 0x9E3779B97F4A7C15ull));
}
__device__ __forceinline__ double omega_next(uint64_t& state) {
  state += 0x9E3779B97F4A7C15ull;
  return __dadd_rn((double)(splitmix_mix(state) >> 11) * 0x1p-52, -1.0);
}

__global__ void omega_kernel(const uint64_t* cells, uint64_t n, uint32_t width,
                             uint64_t seed, double* out) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  uint64_t state = omega_state(seed, cells[r]);
  double* row = out + r * (uint64_t)width;
  for (uint32_t j = 0; j < width; ++j) row[j] = omega_next(state);
}

// D^T = [1 ... 1; 0 ...] in the dense layout (row 0: ones over the n cells, scale 0; all
// else zero).
__global__ void fill_rows_kernel(uint16_t* t, uint64_t n, uint64_t ld) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= 64 * ld) return;
  const uint64_t k = i % 64, r = (i / 64) * 32 + k;  // row 0's column r (hi parts)
  t[i] = (i < ld && k < 32 && r < n) ? (uint16_t)0x3C00u : (uint16_t)0;
}

__global__ void fill_kernel(double* p, uint64_t n, double v) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// Column sums of an n x w row-major matrix, stage 1: block b sums rows
// [b*rows_per, ...) in row order per column.
__global__ void colsum_partial_kernel(const double* m, uint64_t n, uint32_t w,
                                      uint32_t ld, uint64_t rows_per, double* partial) {
  uint64_t r0 = blockIdx.x * rows_per;
  uint64_t r1 = min(n, r0 + rows_per);
  for (uint32_t j = threadIdx.x; j < w; j += blockDim.x) {
    double acc = 0.0;
    for (uint64_t r = r0; r < r1; ++r) acc = __dadd_rn(acc, m[r * ld + j]);
    partial[blockIdx.x * (uint64_t)w + j] = acc;
  }
}

__global__ void colsum_final_kernel(const double* partial, uint32_t nb, uint32_t w,
                                    double* out) {
  for (uint32_t j = threadIdx.x; j < w; j += blockDim.x) {
    double acc = 0.0;
    for (uint32_t b = 0; b < nb; ++b) acc = __dadd_rn(acc, partial[b * (uint64_t)w + j]);
    out[j] = acc;
  }
}

// m[:, j] -= means * sums[j]  (g x w column-major).
__global__ void subtract_outer_kernel(double* m, const double* means, const double* sums,
                                      uint32_t g, uint32_t w) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (uint64_t)g * w) return;
  uint32_t j = (uint32_t)(i / g), r = (uint32_t)(i % g);
  m[i] = __dadd_rn(m[i], -__dmul_rn(means[r], sums[j]));
}

// out[j] = sum_g means[g] * m[g, j], genes in order (set_block / finish_basis).
__global__ void mean_dot_kernel(const double* m, const double* means, uint32_t g,
                                uint32_t w, double* out) {
  uint32_t j = blockIdx.x;
  if (j >= w) return;
  __shared__ double part[256];
  double acc = 0.0;
  uint32_t chunk = (g + blockDim.x - 1) / blockDim.x;
  uint32_t a = threadIdx.x * chunk, b = min(g, a + chunk);
  for (uint32_t r = a; r < b; ++r) acc = __dadd_rn(acc, __dmul_rn(means[r], m[(uint64_t)j * g + r]));
  part[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (unsigned t = 0; t < blockDim.x; ++t) s = __dadd_rn(s, part[t]);
    out[j] = s;
  }
}

// Column-major g x w -> row-major g x w.
__global__ void to_row_major_kernel(const double* cm, uint32_t g, uint32_t w, double* rm) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (uint64_t)g * w) return;
  uint32_t r = (uint32_t)(i / w), j = (uint32_t)(i % w);
  rm[i] = cm[(uint64_t)j * g + r];
}

// sym = (B + B^T) / 2.
__global__ void symmetrize_kernel(const double* b, uint32_t m, double* sym) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (uint64_t)m * m) return;
  uint32_t r = (uint32_t)(i % m), c = (uint32_t)(i / m);
  sym[i] = 0.5 * __dadd_rn(b[i], b[(uint64_t)r * m + c]);
}

// chosen[:, c] = vectors[:, m - 1 - c] (largest eigenvalue first).
__global__ void pick_columns_kernel(const double* vectors, uint32_t m, uint32_t taken,
                                    double* chosen) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (uint64_t)m * taken) return;
  uint32_t r = (uint32_t)(i % m), c = (uint32_t)(i / m);
  chosen[i] = vectors[(uint64_t)(m - 1 - c) * m + r];
}

// pca_dense.rs:225-253 (complement): `count` unit vectors of the least-covered genes
// (first on ties), projected off the columns twice, appended after column `have`.
// One CTA; l is g x k column-major with columns [0, have) filled.
__global__ void complement_kernel(double* l, uint32_t g, uint32_t have, uint32_t k,
                                  double* coeff, double* vec) {
  __shared__ double red[256];
  __shared__ uint32_t red_i[256];
  for (uint32_t col = have; col < k; ++col) {
    // The least covered gene.
    double best = INFINITY;
    uint32_t best_i = 0;
    for (uint32_t r = threadIdx.x; r < g; r += blockDim.x) {
      double c = 0.0;
      for (uint32_t j = 0; j < col; ++j) {
        double v = l[(uint64_t)j * g + r];
        c += v * v;
      }
      if (c < best || (c == best && r < best_i)) {
        best = c;
        best_i = r;
      }
    }
    red[threadIdx.x] = best;
    red_i[threadIdx.x] = best_i;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (unsigned t = 1; t < blockDim.x; ++t)
        if (red[t] < red[0] || (red[t] == red[0] && red_i[t] < red_i[0])) {
          red[0] = red[t];
          red_i[0] = red_i[t];
        }
    }
    __syncthreads();
    uint32_t gene = red_i[0];
    for (uint32_t r = threadIdx.x; r < g; r += blockDim.x) vec[r] = (r == gene) ? 1.0 : 0.0;
    __syncthreads();
    for (int pass = 0; pass < 2; ++pass) {
      for (uint32_t j = threadIdx.x; j < col; j += blockDim.x) {
        double s = 0.0;
        for (uint32_t r = 0; r < g; ++r) s += l[(uint64_t)j * g + r] * vec[r];
        coeff[j] = s;
      }
      __syncthreads();
      for (uint32_t r = threadIdx.x; r < g; r += blockDim.x) {
        double s = 0.0;
        for (uint32_t j = 0; j < col; ++j) s += l[(uint64_t)j * g + r] * coeff[j];
        vec[r] -= s;
      }
      __syncthreads();
    }
    double part = 0.0;
    for (uint32_t r = threadIdx.x; r < g; r += blockDim.x) part += vec[r] * vec[r];
    red[threadIdx.x] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (unsigned t = 0; t < blockDim.x; ++t) s += red[t];
      red[0] = sqrt(s);
    }
    __syncthreads();
    double norm = red[0];
    for (uint32_t r = threadIdx.x; r < g; r += blockDim.x) l[(uint64_t)col * g + r] = vec[r] / norm;
    __syncthreads();
  }
}

// pca_dense.rs:257-275 (flip_signs): one CTA per column; the first largest |v| made
// positive.
__global__ void flip_signs_kernel(double* l, uint32_t g) {
  uint32_t j = blockIdx.x;
  __shared__ double best_v[256];
  __shared__ uint32_t best_i[256];
  double bv = 0.0;
  uint32_t bi = 0xFFFFFFFFu;
  double sign = 1.0;
  for (uint32_t r = threadIdx.x; r < g; r += blockDim.x) {
    double v = l[(uint64_t)j * g + r];
    if (fabs(v) > bv) {
      bv = fabs(v);
      bi = r;
    }
  }
  best_v[threadIdx.x] = bv;
  best_i[threadIdx.x] = bi;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (unsigned t = 1; t < blockDim.x; ++t)
      if (best_v[t] > best_v[0] || (best_v[t] == best_v[0] && best_i[t] < best_i[0])) {
        best_v[0] = best_v[t];
        best_i[0] = best_i[t];
      }
    if (best_i[0] != 0xFFFFFFFFu && l[(uint64_t)j * g + best_i[0]] < 0.0) sign = -1.0;
    best_v[0] = sign;
  }
  __syncthreads();
  if (best_v[0] < 0.0)
    for (uint32_t r = threadIdx.x; r < g; r += blockDim.x) l[(uint64_t)j * g + r] = -l[(uint64_t)j * g + r];
}

// Loadings over the stream's genes (zeros outside the set), f32, row-major.
__global__ void scatter_loadings_kernel(const double* l, uint32_t g, uint32_t k,
                                        const uint32_t* set_genes, uint32_t stream_genes,
                                        float* out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (uint64_t)g * k) return;
  uint32_t r = (uint32_t)(i / k), c = (uint32_t)(i % k);
  uint32_t sg = set_genes ? set_genes[r] : r;
  out[(uint64_t)sg * k + c] = (float)l[(uint64_t)c * g + r];
}

__global__ void to_f32_kernel(const double* in, uint64_t n, float* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

__global__ void divide_kernel(const double* in, uint32_t n, double d, double* out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i] / d;
}

// ------------------------------------------------ thin SVD (one-sided Jacobi) -------

constexpr uint32_t kJacobiMaxCols = 256;

// Hestenes' one-sided Jacobi SVD of the g x w column-major f64 matrix `a` (w <= 256),
// one CTA of 32 warps: columns are rotated pairwise (round-robin tournament, one warp
// per pair, dot products by a fixed shuffle tree) until every pair is orthogonal to
// 1e-15 of its norms. Then a = U diag(sigma) column by column; sigma[c] is the c-th
// largest column norm and order[c] its column (ties to the lower column). Relative
// accuracy for small singular values, as the drop rule (1e-10 of the block's norm)
// needs. status: 0, or 1 if 60 sweeps did not converge.
__global__ void __launch_bounds__(1024)
jacobi_svd_kernel(double* a, uint32_t g, uint32_t w, double* sigma, uint32_t* order,
                  int* status) {
  __shared__ int rotated;
  __shared__ double norms[kJacobiMaxCols];
  const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const unsigned warps = blockDim.x >> 5;
  const uint32_t players = (w + 1) & ~1u;
  int sweep = 0;
  for (; sweep < 60; ++sweep) {
    if (threadIdx.x == 0) rotated = 0;
    __syncthreads();
    for (uint32_t r = 0; r + 1 < players; ++r) {
      for (uint32_t pr = warp; pr < players / 2; pr += warps) {
        auto at = [&](uint32_t pos) {
          return pos == 0 ? 0u : ((pos - 1 + r) % (players - 1)) + 1;
        };
        uint32_t i = at(pr), j = at(players - 1 - pr);
        if (i > j) {
          uint32_t t = i;
          i = j;
          j = t;
        }
        if (j >= w) continue;
        double* ai = a + (uint64_t)i * g;
        double* aj = a + (uint64_t)j * g;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (uint32_t x = lane; x < g; x += 32) {
          double u = ai[x], v = aj[x];
          al = fma(u, u, al);
          be = fma(v, v, be);
          ga = fma(u, v, ga);
        }
        for (int o = 16; o; o >>= 1) {
          al += __shfl_xor_sync(0xFFFFFFFFu, al, o);
          be += __shfl_xor_sync(0xFFFFFFFFu, be, o);
          ga += __shfl_xor_sync(0xFFFFFFFFu, ga, o);
        }
        if (!(al > 0.0) || !(be > 0.0) || !(fabs(ga) > 1e-15 * sqrt(al) * sqrt(be))) continue;
        double zeta = (be - al) / (2.0 * ga);
        double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + hypot(1.0, zeta));
        double c = 1.0 / sqrt(1.0 + t * t), sn = c * t;
        for (uint32_t x = lane; x < g; x += 32) {
          double u = ai[x], v = aj[x];
          ai[x] = c * u - sn * v;
          aj[x] = sn * u + c * v;
        }
        if (lane == 0) rotated = 1;
      }
      __syncthreads();
    }
    bool again = rotated != 0;
    __syncthreads();
    if (!again) break;
  }
  // Column norms, then the order by norm (descending, ties to the lower column).
  for (uint32_t col = warp; col < w; col += warps) {
    const double* ac = a + (uint64_t)col * g;
    double ss = 0.0;
    for (uint32_t x = lane; x < g; x += 32) ss = fma(ac[x], ac[x], ss);
    for (int o = 16; o; o >>= 1) ss += __shfl_xor_sync(0xFFFFFFFFu, ss, o);
    if (lane == 0) norms[col] = sqrt(ss);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t idx[kJacobiMaxCols];
    for (uint32_t c = 0; c < w; ++c) idx[c] = c;
    for (uint32_t c = 1; c < w; ++c) {
      uint32_t v = idx[c], at = c;
      while (at > 0 && norms[idx[at - 1]] < norms[v]) {
        idx[at] = idx[at - 1];
        --at;
      }
      idx[at] = v;
    }
    for (uint32_t c = 0; c < w; ++c) {
      order[c] = idx[c];
      sigma[c] = norms[idx[c]];
    }
    *status = sweep >= 60 ? 1 : 0;
  }
}

constexpr uint32_t kQrMaxCols = 64;

// Hestenes' one-sided Jacobi on the w columns of the w x w matrix in shared memory `rs`
// (by column; round-robin tournament, one warp per pair, pairs orthogonal to 1e-15 of
// their norms): rs becomes U_R diag(sigma). Then norms[c] = sigma of column c, order =
// the columns by descending sigma (ties to the lower column), sigma[] (global) in that
// order and *status = 0, or 1 if 60 sweeps did not converge. All threads call it.
__device__ void jacobi_square(double (*rs)[kQrMaxCols + 1], uint32_t w, double* norms,
                              uint32_t* order, int* rotated_flag, double* sigma, int* status) {
  const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const unsigned warps = blockDim.x >> 5;
  int& rotated = *rotated_flag;
  const uint32_t players = (w + 1) & ~1u;
  int sweep = 0;
  for (; sweep < 60; ++sweep) {
    if (threadIdx.x == 0) rotated = 0;
    __syncthreads();
    for (uint32_t r = 0; r + 1 < players; ++r) {
      for (uint32_t pr = warp; pr < players / 2; pr += warps) {
        auto at = [&](uint32_t pos) {
          return pos == 0 ? 0u : ((pos - 1 + r) % (players - 1)) + 1;
        };
        uint32_t i = at(pr), j2 = at(players - 1 - pr);
        if (i > j2) {
          uint32_t tt = i;
          i = j2;
          j2 = tt;
        }
        if (j2 >= w) continue;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (uint32_t x = lane; x < w; x += 32) {
          double p = rs[i][x], q = rs[j2][x];
          al = fma(p, p, al);
          be = fma(q, q, be);
          ga = fma(p, q, ga);
        }
        for (int o = 16; o; o >>= 1) {
          al += __shfl_xor_sync(0xFFFFFFFFu, al, o);
          be += __shfl_xor_sync(0xFFFFFFFFu, be, o);
          ga += __shfl_xor_sync(0xFFFFFFFFu, ga, o);
        }
        if (!(al > 0.0) || !(be > 0.0) || !(fabs(ga) > 1e-15 * sqrt(al) * sqrt(be))) continue;
        double zeta = (be - al) / (2.0 * ga);
        double tn = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + hypot(1.0, zeta));
        double cs = 1.0 / sqrt(1.0 + tn * tn), sn = cs * tn;
        for (uint32_t x = lane; x < w; x += 32) {
          double p = rs[i][x], q = rs[j2][x];
          rs[i][x] = cs * p - sn * q;
          rs[j2][x] = sn * p + cs * q;
        }
        if (lane == 0) rotated = 1;
      }
      __syncthreads();
    }
    bool again = rotated != 0;
    __syncthreads();
    if (!again) break;
  }
  // Column norms = singular values; the order (descending, ties to the lower column).
  for (uint32_t c = warp; c < w; c += warps) {
    double ss = 0.0;
    for (uint32_t x = lane; x < w; x += 32) ss = fma(rs[c][x], rs[c][x], ss);
    for (int o = 16; o; o >>= 1) ss += __shfl_xor_sync(0xFFFFFFFFu, ss, o);
    if (lane == 0) norms[c] = sqrt(ss);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t c = 0; c < w; ++c) order[c] = c;
    for (uint32_t c = 1; c < w; ++c) {
      uint32_t v = order[c], pos = c;
      while (pos > 0 && norms[order[pos - 1]] < norms[v]) {
        order[pos] = order[pos - 1];
        --pos;
      }
      order[pos] = v;
    }
    for (uint32_t c = 0; c < w; ++c) sigma[c] = norms[order[c]];
    *status = sweep >= 60 ? 1 : 0;
  }
  __syncthreads();
}

// The thin SVD's left singular vectors of the g x w column-major block `b` (w <= 64,
// overwritten), one CTA of 32 warps: Householder QR in place (b = Q R, the reflectors
// below the diagonal, LAPACK's dlarfg convention v_j = 1), then Hestenes' one-sided
// Jacobi on R in shared memory (R V = U_R diag(sigma); pairs orthogonal to 1e-15 of
// their norms), then U = Q [U_R; 0] by applying the reflectors backwards. QR is
// backward stable, so sigma carries an absolute error of about 1e-16 |b|: the drop rule
// (sigma > 1e-10 |b|_F) sees rank deficiency as an SVD of b would.
// Outputs: sigma (w, descending; ties to the lower column), u (g x w: column c the
// unit vector of sigma[c]). status: 0, or 1 if 60 sweeps did not converge.
__global__ void __launch_bounds__(1024)
qr_svd_kernel(double* b, uint32_t g, uint32_t w, double* sigma, double* u, int* status) {
  __shared__ double rs[kQrMaxCols][kQrMaxCols + 1];  // R, then U_R diag(sigma), by column
  __shared__ double tau[kQrMaxCols];
  __shared__ double norms[kQrMaxCols];
  __shared__ uint32_t order[kQrMaxCols];
  __shared__ int rotated;
  const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const unsigned warps = blockDim.x >> 5;
  auto colp = [&](uint32_t c) { return b + (uint64_t)c * g; };

  // Householder QR.
  for (uint32_t j = 0; j < w; ++j) {
    if (warp == 0) {
      const double* bj = colp(j);
      double ss = 0.0;
      for (uint32_t i = j + 1 + lane; i < g; i += 32) ss = fma(bj[i], bj[i], ss);
      for (int o = 16; o; o >>= 1) ss += __shfl_xor_sync(0xFFFFFFFFu, ss, o);
      if (lane == 0) {
        double alpha = bj[j];
        double normx = sqrt(fma(alpha, alpha, ss));
        if (ss == 0.0) {
          tau[j] = 0.0;  // already upper triangular in this column
        } else {
          double beta = alpha >= 0.0 ? -normx : normx;
          tau[j] = (beta - alpha) / beta;
          norms[j] = 1.0 / (alpha - beta);  // scale of v below the diagonal
          colp(j)[j] = beta;
        }
      }
    }
    __syncthreads();
    const double t = tau[j];
    if (t != 0.0) {
      double* bj = colp(j);
      const double sc = norms[j];
      for (uint32_t i = j + 1 + threadIdx.x; i < g; i += blockDim.x) bj[i] *= sc;
      __syncthreads();
      for (uint32_t c = j + 1 + warp; c < w; c += warps) {
        double* bc = colp(c);
        double d = (lane == 0) ? bc[j] : 0.0;
        for (uint32_t i = j + 1 + lane; i < g; i += 32) d = fma(bj[i], bc[i], d);
        for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xFFFFFFFFu, d, o);
        const double f = t * d;
        if (lane == 0) bc[j] -= f;
        for (uint32_t i = j + 1 + lane; i < g; i += 32) bc[i] = fma(-f, bj[i], bc[i]);
      }
    }
    __syncthreads();
  }
  // R into shared memory.
  for (uint32_t x = threadIdx.x; x < w * w; x += blockDim.x) {
    uint32_t c = x / w, r = x % w;
    rs[c][r] = r <= c ? colp(c)[r] : 0.0;
  }
  __syncthreads();
  jacobi_square(rs, w, norms, order, &rotated, sigma, status);
  // U = Q [U_R; 0]: start from U_R's unit columns, apply H_{w-1}, ..., H_0.
  for (uint64_t x = threadIdx.x; x < (uint64_t)g * w; x += blockDim.x) {
    uint32_t c = (uint32_t)(x / g), r = (uint32_t)(x % g);
    double nv = norms[order[c]];
    u[x] = (r < w && nv > 0.0) ? rs[order[c]][r] / nv : 0.0;
  }
  __syncthreads();
  for (int j = (int)w - 1; j >= 0; --j) {
    const double t = tau[j];
    if (t == 0.0) continue;
    const double* v = colp(j);
    for (uint32_t c = warp; c < w; c += warps) {
      double* uc = u + (uint64_t)c * g;
      double d = (lane == 0) ? uc[j] : 0.0;
      for (uint32_t i = j + 1 + lane; i < g; i += 32) d = fma(v[i], uc[i], d);
      for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xFFFFFFFFu, d, o);
      const double f = t * d;
      if (lane == 0) uc[j] -= f;
      for (uint32_t i = j + 1 + lane; i < g; i += 32) uc[i] = fma(-f, v[i], uc[i]);
    }
    __syncthreads();
  }
}

// One step of shifted CholeskyQR3 (Fukaya, Kannan, Nakatsukasa, Yamamoto and Yanagisawa,
// "Shifted Cholesky QR for computing the QR factorization of ill-conditioned
// matrices", SIAM J. Sci. Comput. 2020), one CTA, w <= 64: the upper Cholesky factor R
// of the Gram matrix G (w x w, column-major) plus shift * trace(G) on the diagonal
// (trace(G) = |A|_F^2 >= |A|_2^2), into r (w x w column-major, zeros below), and the
// running product r_total = R r_total (R itself when first). *status = 1 if a pivot is
// not positive (the caller then uses Householder QR).
__global__ void __launch_bounds__(1024)
cholesky_step_kernel(const double* gram, uint32_t w, double shift, int first, double* r,
                     double* r_total, int* status) {
  __shared__ double a[kQrMaxCols][kQrMaxCols + 1];  // a[row][col]
  __shared__ double trace;
  __shared__ int bad;
  for (uint32_t x = threadIdx.x; x < w * w; x += blockDim.x) a[x % w][x / w] = gram[x];
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tr = 0.0;
    for (uint32_t j = 0; j < w; ++j) tr += a[j][j];
    trace = tr;
  }
  __syncthreads();
  if (threadIdx.x < w) a[threadIdx.x][threadIdx.x] += shift * trace;
  __syncthreads();
  for (uint32_t j = 0; j < w; ++j) {
    const double d = a[j][j];
    if (!(d > 0.0)) {
      if (threadIdx.x == 0) bad = 1;
      break;  // every thread reads the same d and leaves together
    }
    const double piv = sqrt(d);
    __syncthreads();
    // Row j of R: a[j][c] / piv for c > j (the diagonal written after the reads).
    for (uint32_t c = j + 1 + threadIdx.x; c < w; c += blockDim.x) a[j][c] /= piv;
    __syncthreads();
    if (threadIdx.x == 0) a[j][j] = piv;
    // Trailing update: a[i][c] -= R[j][i] R[j][c] for j < i <= c.
    const uint32_t m = w - j - 1;
    for (uint32_t x = threadIdx.x; x < m * m; x += blockDim.x) {
      uint32_t i = j + 1 + x / m, c = j + 1 + x % m;
      if (i <= c) a[i][c] -= a[j][i] * a[j][c];
    }
    __syncthreads();
  }
  __syncthreads();
  if (bad) {
    if (threadIdx.x == 0) *status = 1;
    return;
  }
  for (uint32_t x = threadIdx.x; x < w * w; x += blockDim.x) {
    uint32_t c = x / w, i = x % w;
    r[x] = i <= c ? a[i][c] : 0.0;
  }
  // r_total = R r_total (both upper triangular): every thread computes its (at most 4,
  // w <= 64 with 1024 threads) entries from the old r_total before any is written.
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (uint32_t x = threadIdx.x, e = 0; x < w * w; x += blockDim.x, ++e) {
    uint32_t c = x / w, i = x % w;
    if (i > c) continue;
    if (first) {
      v[e] = a[i][c];
    } else {
      double acc = 0.0;
      for (uint32_t q = i; q <= c; ++q) acc = fma(a[i][q], r_total[(uint64_t)c * w + q], acc);
      v[e] = acc;
    }
  }
  __syncthreads();
  for (uint32_t x = threadIdx.x, e = 0; x < w * w; x += blockDim.x, ++e) r_total[x] = v[e];
}

// The SVD of the w x w upper-triangular r (column-major, w <= 64): sigma (descending,
// ties to the lower column) and u_r (w x w: column c the unit left singular vector of
// sigma[c]; zero for sigma 0). *status |= 1 if Jacobi did not converge.
__global__ void __launch_bounds__(1024)
small_svd_kernel(const double* r, uint32_t w, double* sigma, double* u_r, int* status) {
  __shared__ double rs[kQrMaxCols][kQrMaxCols + 1];
  __shared__ double norms[kQrMaxCols];
  __shared__ uint32_t order[kQrMaxCols];
  __shared__ int rotated;
  __shared__ int jstatus;
  for (uint32_t x = threadIdx.x; x < w * w; x += blockDim.x) rs[x / w][x % w] = r[x];
  __syncthreads();
  jacobi_square(rs, w, norms, order, &rotated, sigma, &jstatus);
  __syncthreads();
  for (uint32_t x = threadIdx.x; x < w * w; x += blockDim.x) {
    uint32_t c = x / w, i = x % w;
    double nv = norms[order[c]];
    u_r[x] = nv > 0.0 ? rs[order[c]][i] / nv : 0.0;
  }
  if (threadIdx.x == 0 && jstatus) *status = 1;
}

// out[:, c] = a[:, order[c]] / sigma[c] (the left singular vectors kept).
__global__ void gather_unit_columns_kernel(const double* a, uint32_t g, uint32_t keep,
                                           const double* sigma, const uint32_t* order,
                                           double* out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (uint64_t)g * keep) return;
  uint32_t c = (uint32_t)(i / g), r = (uint32_t)(i % g);
  out[i] = a[(uint64_t)order[c] * g + r] / sigma[c];
}

// ------------------------------------------------ tensor-core product support -------

// A value times 2^scale as the two fp16 parts of the products' dense operand
// (kg_spmm_tc.cuh): hi = fp16(y), lo = fp16(y - hi).
__device__ __forceinline__ void split_half(double v, double mul, uint16_t& hi, uint16_t& lo) {
  const double y = v * mul;
  const __half h = __double2half(y);
  hi = __half_as_ushort(h);
  lo = __half_as_ushort(__double2half(y - (double)__half2float(h)));
}

// The value the products see for a split value (hi + lo, unscaled).
__device__ __forceinline__ double joined(uint16_t hi, uint16_t lo, double inv) {
  return ((double)__half2float(__ushort_as_half(hi)) +
          (double)__half2float(__ushort_as_half(lo))) * inv;
}

// D^T in the dense layout (row length ld halves, values times 2^scale) from a g x w
// column-major f64 matrix: thread per (j, r), r < ld / 2 (zero past w columns and g
// rows).
__global__ void split_t_kernel(const double* cm, uint32_t g, uint32_t w, uint64_t ld,
                               int scale, uint16_t* t) {
  const uint64_t half = ld / 2;
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= 64 * half) return;
  uint32_t j = (uint32_t)(i / half);
  uint64_t r = i % half;
  double v = (j < w && r < g) ? cm[(uint64_t)j * g + r] : 0.0;
  uint16_t hi, lo;
  split_half(v, ldexp(1.0, scale), hi, lo);
  uint16_t* at = t + (uint64_t)j * ld + (r / 32) * 64 + (r % 32);
  at[0] = hi;
  at[32] = lo;
}

// Omega^T in the dense layout (values times 2^scale; rows past width zero), and each
// block's Omega column sums of the split values (as the products see them; f64, a fixed
// tree) for the centring.
__global__ void omega_t_kernel(const uint64_t* cells, uint64_t n, uint32_t width,
                               uint64_t seed, uint64_t ld, int scale, uint16_t* t,
                               double* block_sums) {
  __shared__ double red[8][64];
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  bool live = r < n;
  uint64_t state = live ? omega_state(seed, cells[r]) : 0;
  const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const double mul = ldexp(1.0, scale), inv = ldexp(1.0, -scale);
  for (uint32_t j = 0; j < 64; ++j) {
    uint16_t hi = 0, lo = 0;
    if (live && j < width) split_half(omega_next(state), mul, hi, lo);
    if (r < ld / 2) {
      uint16_t* at = t + (uint64_t)j * ld + (r / 32) * 64 + (r % 32);
      at[0] = hi;
      at[32] = lo;
    }
    if (j < width) {
      double sv = joined(hi, lo, inv);
      for (int o = 16; o; o >>= 1) sv += __shfl_xor_sync(0xFFFFFFFFu, sv, o);
      if (lane == 0) red[warp][j] = sv;
    }
  }
  __syncthreads();
  if (threadIdx.x < width) {
    double t = 0.0;
    for (unsigned w8 = 0; w8 < blockDim.x / 32; ++w8) t += red[w8][threadIdx.x];
    block_sums[blockIdx.x * (uint64_t)64 + threadIdx.x] = t;
  }
}

// out[j] = sum over blocks (in order) of partial[b][j], j < w.
// out[j] = the sum over b of partial[b * 64 + j] (j < w): one CTA of 1024 threads, 16
// row classes per column summed in order, then the classes in order (a fixed tree).
__global__ void __launch_bounds__(1024)
sum_blocks_kernel(const double* partial, uint64_t nb, uint32_t w, double* out) {
  __shared__ double part[16][64];
  const uint32_t j = threadIdx.x & 63u, cls = threadIdx.x >> 6;
  double t = 0.0;
  if (j < w)
    for (uint64_t b = cls; b < nb; b += 16) t += partial[b * 64 + j];
  part[cls][j] = t;
  __syncthreads();
  if (cls == 0 && j < w) {
    double u = 0.0;
    for (int c = 0; c < 16; ++c) u += part[c][j];
    out[j] = u;
  }
}

// out (g x w column-major) = sum over segments (in order) of partial[seg][gene][j].
__global__ void reduce_segments_kernel(const double* partial, uint32_t segs, uint32_t g,
                                       uint32_t w, double* out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (uint64_t)g * w) return;
  uint32_t gene = (uint32_t)(i / w), j = (uint32_t)(i % w);
  double t = 0.0;
  for (uint32_t sg = 0; sg < segs; ++sg) t += partial[((uint64_t)sg * g + gene) * 64 + j];
  out[(uint64_t)j * g + gene] = t;
}

// Each gene's sum of (x - mean)^2 over its stored values: a warp per gene, lanes over
// the gene's entries in order, then a fixed shuffle tree.
__global__ void gene_squares_kernel(const uint64_t* ptr, const float* val, const double* means,
                                    uint32_t g, double* out) {
  uint64_t gene = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  if (gene >= g) return;
  double mu = means[gene], acc = 0.0;
  for (uint64_t i = ptr[gene] + lane; i < ptr[gene + 1]; i += 32) {
    double c = (double)val[i] - mu;
    acc = fma(c, c, acc);
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
  if (lane == 0) out[gene] = acc;
}

__global__ void to_u16_kernel(const uint32_t* in, uint64_t n, uint16_t* out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (uint16_t)in[i];
}

// (row << 32) | value bits, for the gene-major sort.
__global__ void pack_rows_kernel(const uint64_t* indptr, const float* val, uint64_t n_rows,
                                 uint64_t* packed) {
  uint64_t row = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  if (row >= n_rows) return;
  for (uint64_t i = indptr[row] + lane; i < indptr[row + 1]; i += 32)
    packed[i] = (row << 32) | (uint64_t)__float_as_uint(val[i]);
}

__global__ void unpack_rows_kernel(const uint64_t* packed, uint64_t n, uint32_t* row,
                                   float* val) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t p = packed[i];
    row[i] = (uint32_t)(p >> 32);
    val[i] = __uint_as_float((uint32_t)p);
  }
}

// The held input for the tensor-core products: X and X^T in the blocked layout
// (kg_spmm_tc.cuh), and the D^T buffers the passes fill.
// Device time and algorithmic bytes of a session's sparse x dense products: a CUDA event
// pair around each launch on the session's stream, read once the run has finished.
struct ProductClock {
  struct Launch {
    cudaEvent_t a = nullptr, b = nullptr;
    double bytes = 0.0;
  };
  std::vector<Launch> launches;
  cudaStream_t s = nullptr;
  void begin(cudaStream_t st, double bytes) {
    s = st;
    Launch l;
    l.bytes = bytes;
    if (cudaEventCreate(&l.a) != cudaSuccess || cudaEventCreate(&l.b) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    cudaEventRecord(l.a, s);
    launches.push_back(l);
  }
  void end() {
    if (!launches.empty()) cudaEventRecord(launches.back().b, s);
  }
  // Sums over the launches (after the stream finished); releases the events.
  void collect(uint32_t& count, double& ms, double& bytes) {
    count = 0;
    ms = 0.0;
    bytes = 0.0;
    for (Launch& l : launches) {
      float t = 0.0f;
      if (cudaEventElapsedTime(&t, l.a, l.b) == cudaSuccess) {
        ++count;
        ms += t;
        bytes += l.bytes;
      } else {
        cudaGetLastError();
      }
    }
    release();
  }
  void release() {
    for (Launch& l : launches) {
      if (l.a) cudaEventDestroy(l.a);
      if (l.b) cudaEventDestroy(l.b);
    }
    launches.clear();
  }
  ~ProductClock() { release(); }
};

struct TcHeld {
  static constexpr uint64_t kSegChunks = 512;  // K-chunks (16,384 cells) per X^T work item
  static constexpr int kUnitScale = 14;        // |Omega|, |Q|, |V| <= 1: parts times 2^14
  uint64_t n = 0, g = 0, nnz = 0;
  ProductClock clock;
  // A product's algorithmic bytes, S (rows x K, nnz values) . D (K x l) read once and
  // the rows x l result written once: 8 nnz + 4 (n + 1) + 4 g l + 4 n l (f32 values and
  // u32 indices, row offsets, the dense operand and result in f32).
  double product_bytes(uint32_t l) const {
    return 8.0 * (double)nnz + 4.0 * (double)(n + 1) + 4.0 * (double)g * l + 4.0 * (double)n * l;
  }
  Blocked bx, bxt;
  DeviceBuffer<uint16_t> dt;   // 64 x dense_ld(n): Omega^T, the ones row or W^T
  DeviceBuffer<uint16_t> qt;   // 64 x dense_ld(g): Q^T or V^T
  int dt_scale = 0;
  double mean_norm = 0.0;      // |mu| (the gene means), for the bound on W's entries
  DeviceBuffer<int> error;     // set by a product whose bounded wait ran out
  int sm = 148;

  void build(const uint64_t* indptr, const uint32_t* col, const float* val, uint64_t n_rows,
             uint32_t n_genes, uint64_t nnz, int sm_count, cudaStream_t s, Trace& trace) {
    n = n_rows;
    g = n_genes;
    this->nnz = nnz;
    sm = sm_count;
    build_blocked(indptr, col, val, n, g, nnz, bx, s);
    trace.mark("blocked X");
    transpose_blocked(indptr, col, val, n, g, nnz, bx, bxt, s);
    trace.mark("blocked X^T");
    dt.alloc(64 * dense_ld(n), s);
    dt.zero();
    qt.alloc(64 * dense_ld(g), s);
    qt.zero();
    error.alloc(1, s);
    error.zero();
  }

  // Whether a product gave up waiting (reads the flag: synchronises the stream).
  void check(cudaStream_t s) {
    if (!error.ptr) return;
    int h = 0;
    KG_CUDA(cudaMemcpyAsync(&h, error.ptr, 4, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    if (h) fail(KG_ERR_TIMEOUT, "a tensor-core product gave up waiting on its pipeline");
  }

  // out (g x width column-major) = X^T Omega; omega_sums (width).
  void sketch(const uint64_t* cells, uint32_t width, uint64_t seed, double* out,
              double* omega_sums, cudaStream_t s) {
    const uint64_t ld = dense_ld(n);
    unsigned nb = blocks_for(ld / 2, 256);
    DeviceBuffer<double> bsum((uint64_t)nb * 64, s);
    omega_t_kernel<<<nb, 256, 0, s>>>(cells, n, width, seed, ld, kUnitScale, dt.ptr, bsum.ptr);
    KG_LAUNCH_CHECK();
    dt_scale = kUnitScale;
    sum_blocks_kernel<<<1, 1024, 0, s>>>(bsum.ptr, nb, width, omega_sums);
    KG_LAUNCH_CHECK();
    transposed(width, out, s);
  }

  // D^T = a row of ones (the stored values' gene sums, counts, squares).
  void ones_column() {
    const uint64_t ld = dense_ld(n);
    fill_rows_kernel<<<blocks_for(64 * ld, 256), 256, 0, dt.stream>>>(dt.ptr, n, ld);
    KG_LAUNCH_CHECK();
    dt_scale = 0;
  }

  // out (g x w column-major) = X^T W with W^T in dt (the stored values mapped by
  // value_mode first).
  void transposed(uint32_t w, double* out, cudaStream_t s, int value_mode = kValuePlain,
                  const double* row_means = nullptr) {
    uint64_t segs = (bxt.n_chunks + kSegChunks - 1) / kSegChunks;
    DeviceBuffer<double> partial(segs * g * 64, s);
    SpmmArgs a;
    a.value_mode = value_mode;
    a.row_means = row_means;
    a.s = &bxt;
    a.seg_chunks = kSegChunks;
    a.dt = dt.ptr;
    a.ld_t = dense_ld(n);
    a.dt_scale = dt_scale;
    a.out.mode = kOutPartial;
    a.out.partial = partial.ptr;
    a.sm_count = sm;
    a.error = error.ptr;
    clock.begin(s, product_bytes(w));
    spmm_tc(a, s);
    clock.end();
    reduce_segments_kernel<<<blocks_for(g * w, 256), 256, 0, s>>>(partial.ptr, (uint32_t)segs,
                                                                  (uint32_t)g, w, out);
    KG_LAUNCH_CHECK();
  }

  // Rows of X M - offsets for M = m (g x w column-major, orthonormal columns): as W^T into
  // dt (with the column sums into wsums) or as f32 rows into rows_f32.
  void rows(const double* m, uint32_t w, const double* offsets, double* wsums, float* rows_f32,
            cudaStream_t s) {
    const uint64_t ldq = dense_ld(g);
    split_t_kernel<<<blocks_for(64 * ldq / 2, 256), 256, 0, s>>>(m, (uint32_t)g, w, ldq,
                                                                 kUnitScale, qt.ptr);
    KG_LAUNCH_CHECK();
    uint64_t tiles = (n + 127) / 128;
    DeviceBuffer<double> colsum;
    SpmmArgs a;
    a.s = &bx;
    a.seg_chunks = bx.n_chunks;
    a.dt = qt.ptr;
    a.ld_t = ldq;
    a.dt_scale = kUnitScale;
    a.out.mode = kOutRows;
    a.out.width = w;
    a.out.offsets = offsets;
    if (wsums) {
      // |w_ij| = |(x_i - mu) . q_j| <= |x_i| + |mu| (unit columns q_j), with room to
      // spare for their rounding: the parts of W^T stay below 2^15.
      colsum.alloc(tiles * 64, s);
      a.out.t = dt.ptr;
      a.out.ld_t = dense_ld(n);
      a.out.t_scale = part_scale(2.0 * (bx.max_row_norm + mean_norm));
      a.out.colsum_partial = colsum.ptr;
    }
    a.out.rows_f32 = rows_f32;
    a.sm_count = sm;
    a.error = error.ptr;
    clock.begin(s, product_bytes(w));
    spmm_tc(a, s);
    clock.end();
    if (wsums) {
      dt_scale = a.out.t_scale;
      sum_blocks_kernel<<<1, 1024, 0, s>>>(colsum.ptr, tiles, w, wsums);
      KG_LAUNCH_CHECK();
    }
  }
};

}  // namespace kg

using namespace kg;

struct kg_pca {
  kg_ctx* ctx = nullptr;
  cudaStream_t stream = nullptr;
  cublasHandle_t cublas = nullptr;
  cusolverDnHandle_t cusolver = nullptr;
  uint32_t k = 0, stream_genes = 0, n_genes = 0, width = 0;
  uint64_t seed = 0;
  double target_sum = NAN;
  int log1p = 0;
  DeviceBuffer<uint32_t> gene_map, set_genes;
  // Held input (CSR over the PCA's genes).
  DeviceBuffer<uint64_t> indptr;
  DeviceBuffer<uint32_t> col;
  DeviceBuffer<float> val;
  DeviceBuffer<uint64_t> cells;
  uint64_t n_cells = 0, nnz = 0, next_cell = 0;
  // Set by the pack kernels when a pushed gene index is out of range (checked at run).
  DeviceBuffer<unsigned int> bad_index;
  // Results.
  bool ran = false;
  uint32_t passes_run = 0;
  DeviceBuffer<float> embedding, loadings;
  DeviceBuffer<double> means;
  std::vector<double> variance, variance_ratio;
  const char* products_engine = "";
  // The last run's sparse x dense products (kg_pca_run_stats).
  uint32_t product_launches = 0;
  double product_ms = 0.0, product_bytes = 0.0, run_ms = 0.0;

  ~kg_pca() {
    if (stream) cudaStreamSynchronize(stream);
    gene_map.reset();
    set_genes.reset();
    indptr.reset();
    col.reset();
    val.reset();
    cells.reset();
    embedding.reset();
    loadings.reset();
    means.reset();
    if (stream) cudaStreamSynchronize(stream);
    // The stream and handles go back to the context for the next session (a stream
    // with all three: they were made together and stay bound to each other).
    if (ctx && stream && cublas && cusolver) {
      std::lock_guard<std::mutex> lock(ctx->res_mu);
      ctx->free_res.push_back({stream, cublas, cusolver});
    } else {
      if (cusolver) cusolverDnDestroy(cusolver);
      if (cublas) cublasDestroy(cublas);
      if (stream) cudaStreamDestroy(stream);
    }
  }

  template <class T>
  void grow(DeviceBuffer<T>& buf, size_t used, size_t need) {
    if (need <= buf.count) return;
    size_t cap = std::max(need, buf.count + buf.count / 2);
    DeviceBuffer<T> bigger(cap, stream);
    if (used) KG_CUDA(cudaMemcpyAsync(bigger.ptr, buf.ptr, used * sizeof(T),
                                      cudaMemcpyDeviceToDevice, stream));
    buf = std::move(bigger);
  }

  void push(const uint64_t* h_indptr, const uint32_t* h_idx, const void* h_values,
            kg_dtype dtype, uint64_t n_rows, const uint64_t* h_cells, bool async);
  void run();
};

void kg_pca::push(const uint64_t* in_indptr, const uint32_t* in_idx, const void* in_values,
                  kg_dtype dtype, uint64_t n_rows, const uint64_t* in_cells, bool async) {
  if (ran) fail(KG_ERR_STATE, "kg_pca_push_block after kg_pca_run");
  if (dtype != KG_U32 && dtype != KG_F32) fail(KG_ERR_INVALID, "unknown dtype");
  if (n_rows == 0) return;
  cudaStream_t s = stream;
  Trace trace(s, "pca_push");
  // The block's first and last offsets: read in place from host memory; from device
  // memory through one copy.
  uint64_t ends[2];
  DeviceBuffer<uint64_t> hp, hc;
  if (is_device_pointer(in_indptr)) {
    KG_CUDA(cudaMemcpyAsync(&ends[0], in_indptr, 8, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaMemcpyAsync(&ends[1], in_indptr + n_rows, 8, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
  } else {
    ends[0] = in_indptr[0];
    ends[1] = in_indptr[n_rows];
  }
  if (ends[0] != 0) fail(KG_ERR_INVALID, "a block's indptr must start at 0");
  const uint64_t* d_indptr = device_view(in_indptr, n_rows + 1, hp, s);
  uint64_t bnnz = ends[1];
  DeviceBuffer<uint32_t> hi, hv;
  const uint32_t* d_idx = device_view(in_idx, bnnz, hi, s);
  const void* d_values = device_view((const uint32_t*)in_values, bnnz, hv, s);
  if (!bad_index.ptr) {
    bad_index.alloc(1, s);
    bad_index.zero();
  }
  if (!async) check_indices(d_idx, bnnz, stream_genes, s);
  trace.mark("checks");
  // Kept entries per row and the rows' normalize divisors, then the kept entries'
  // offsets after the held entries; the maps run inside write_kept.
  const bool normalize = !std::isnan(target_sum);
  DeviceBuffer<int> inexact;
  inexact_flag(d_values, dtype, bnnz, target_sum, inexact, s);
  DeviceBuffer<uint64_t> kept(n_rows + 1, s);
  DeviceBuffer<float> divisor;
  if (normalize) divisor.alloc(n_rows, s);
  kept.zero();
  unsigned threads = 256;
  if (dtype == KG_U32)
    count_kept_kernel<uint32_t><<<blocks_for(n_rows * 32, threads), threads, 0, s>>>(
        d_indptr, d_idx, (const uint32_t*)d_values, n_rows, gene_map.ptr, stream_genes,
        (float)target_sum, inexact.ptr, kept.ptr, divisor.ptr, bad_index.ptr);
  else
    count_kept_kernel<float><<<blocks_for(n_rows * 32, threads), threads, 0, s>>>(
        d_indptr, d_idx, (const float*)d_values, n_rows, gene_map.ptr, stream_genes,
        (float)target_sum, inexact.ptr, kept.ptr, divisor.ptr, bad_index.ptr);
  KG_LAUNCH_CHECK();
  size_t temp = 0;
  KG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, kept.ptr, kept.ptr, n_rows + 1, s));
  DeviceBuffer<unsigned char> scratch(temp, s);
  KG_CUDA(cub::DeviceScan::ExclusiveSum(scratch.ptr, temp, kept.ptr, kept.ptr, n_rows + 1, s));
  // Kept entries: every entry when every gene is kept (an out-of-range index makes the
  // run fail before the held input is used), else counted on the device.
  uint64_t added = bnnz;
  if (gene_map.ptr) {
    KG_CUDA(cudaMemcpyAsync(&added, kept.ptr + n_rows, 8, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
  }
  add_offset_kernel<<<blocks_for(n_rows + 1, 256), 256, 0, s>>>(kept.ptr, n_rows + 1, nnz);
  KG_LAUNCH_CHECK();
  trace.mark("kept counts");
  grow(indptr, n_cells + 1, n_cells + n_rows + 1);
  grow(col, nnz, nnz + added);
  grow(val, nnz, nnz + added);
  grow(cells, n_cells, n_cells + n_rows);
  trace.mark("held buffers");
  KG_CUDA(cudaMemcpyAsync(indptr.ptr + n_cells, kept.ptr, (n_rows + 1) * 8,
                          cudaMemcpyDeviceToDevice, s));
  if (dtype == KG_U32)
    write_kept_kernel<uint32_t><<<blocks_for(n_rows * 32, threads), threads, 0, s>>>(
        d_indptr, d_idx, (const uint32_t*)d_values, divisor.ptr, log1p, n_rows, gene_map.ptr,
        stream_genes, kept.ptr, col.ptr, val.ptr);
  else
    write_kept_kernel<float><<<blocks_for(n_rows * 32, threads), threads, 0, s>>>(
        d_indptr, d_idx, (const float*)d_values, divisor.ptr, log1p, n_rows, gene_map.ptr,
        stream_genes, kept.ptr, col.ptr, val.ptr);
  KG_LAUNCH_CHECK();
  if (in_cells) {
    const uint64_t* d_cells = device_view(in_cells, n_rows, hc, s);
    KG_CUDA(cudaMemcpyAsync(cells.ptr + n_cells, d_cells, n_rows * 8, cudaMemcpyDeviceToDevice, s));
    uint64_t last = 0;
    if (is_device_pointer(in_cells)) {
      KG_CUDA(cudaMemcpyAsync(&last, in_cells + n_rows - 1, 8, cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaStreamSynchronize(s));
    } else {
      last = in_cells[n_rows - 1];
    }
    next_cell = last + 1;
  } else {
    iota64_kernel<<<blocks_for(n_rows, 256), 256, 0, s>>>(cells.ptr + n_cells, n_rows, next_cell);
    KG_LAUNCH_CHECK();
    next_cell += n_rows;
  }
  n_cells += n_rows;
  nnz += added;
  // A synchronous push returns once the block is on the device (the caller may then
  // reuse its host arrays); an asynchronous one leaves the copies and kernels queued on
  // the session's stream (its host arrays stay in use until kg_pca_run returns).
  if (!async) KG_CUDA(cudaStreamSynchronize(s));
  trace.mark("held block");
}

namespace {

// Dense FP64 helpers over one session (column-major g x w matrices).
struct Dense {
  kg_pca* p;
  cudaStream_t s;
  uint32_t g;

  double fro_norm(const double* m, uint64_t count) {
    double out = 0.0;
    KG_CUBLAS(cublasDnrm2(p->cublas, (int)count, m, 1, &out));
    return out;
  }

  // pca_dense.rs:105-129: the directions `block` (g x w) adds to `basis` (g x m):
  // CGS twice, thin SVD, keep sigma > 1e-10 |block|_F. Returns the new block.
  DeviceBuffer<double> extend_basis(const double* basis, uint32_t m, const double* block,
                                    uint32_t w, uint32_t* keep_out) {
    *keep_out = 0;
    DeviceBuffer<double> none;
    if (w == 0) return none;
    double scale = fro_norm(block, (uint64_t)g * w);
    if (!(scale > 0.0)) {
      if (std::isnan(scale)) fail(KG_ERR_INVALID, "pca: the Krylov block is not finite");
      return none;
    }
    DeviceBuffer<double> rest((uint64_t)g * w, s);
    KG_CUDA(cudaMemcpyAsync(rest.ptr, block, rest.bytes(), cudaMemcpyDeviceToDevice, s));
    if (m > 0) {
      DeviceBuffer<double> proj((uint64_t)m * w, s);
      const double one = 1.0, zero = 0.0, minus = -1.0;
      for (int pass = 0; pass < 2; ++pass) {
        KG_CUBLAS(cublasDgemm(p->cublas, CUBLAS_OP_T, CUBLAS_OP_N, m, w, g, &one, basis, g,
                              rest.ptr, g, &zero, proj.ptr, m));
        KG_CUBLAS(cublasDgemm(p->cublas, CUBLAS_OP_N, CUBLAS_OP_N, g, w, m, &minus, basis, g,
                              proj.ptr, m, &one, rest.ptr, g));
      }
    }
    // Thin SVD in one kernel: QR + Jacobi on R for blocks of up to 64 columns (and
    // g >= w, always true here), one-sided Jacobi on the whole block beyond that.
    if (w > kJacobiMaxCols) fail(KG_ERR_INVALID, "pca: a Krylov block wider than 256 columns");
    DeviceBuffer<double> sv(w, s);
    DeviceBuffer<uint32_t> order(w, s);
    DeviceBuffer<int> info(1, s);
    DeviceBuffer<double> u;
    const bool qr = w <= kQrMaxCols;
    std::vector<double> h_sv(w);
    int h_info = 0;
    auto read_back = [&]() {
      KG_CUDA(cudaMemcpyAsync(h_sv.data(), sv.ptr, w * 8ull, cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaMemcpyAsync(&h_info, info.ptr, 4, cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaStreamSynchronize(s));
    };
    if (qr) {
      // Shifted CholeskyQR3 (rest = Q R: three Gram/Cholesky/triangular-solve rounds
      // across the GPU), the SVD of R in one CTA, U = Q U_R; Householder QR in one CTA
      // if a Cholesky pivot fails (a numerically rank-deficient block).
      u.alloc((uint64_t)g * w, s);
      DeviceBuffer<double> saved((uint64_t)g * w, s), gram((uint64_t)w * w, s),
          rt((uint64_t)w * w, s), rtot((uint64_t)w * w, s), ur((uint64_t)w * w, s);
      KG_CUDA(cudaMemcpyAsync(saved.ptr, rest.ptr, rest.bytes(), cudaMemcpyDeviceToDevice, s));
      info.zero();
      const double one = 1.0, zero = 0.0;
      const double shift = 11.0 * ((double)g * w + (double)w * (w + 1)) * 0x1p-53;
      for (int round = 0; round < 3; ++round) {
        KG_CUBLAS(cublasDgemm(p->cublas, CUBLAS_OP_T, CUBLAS_OP_N, w, w, g, &one, rest.ptr, g,
                              rest.ptr, g, &zero, gram.ptr, w));
        cholesky_step_kernel<<<1, 1024, 0, s>>>(gram.ptr, w, round == 0 ? shift : 0.0,
                                                round == 0, rt.ptr, rtot.ptr, info.ptr);
        KG_LAUNCH_CHECK();
        KG_CUBLAS(cublasDtrsm(p->cublas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N,
                              CUBLAS_DIAG_NON_UNIT, g, w, &one, rt.ptr, w, rest.ptr, g));
      }
      small_svd_kernel<<<1, 1024, 0, s>>>(rtot.ptr, w, sv.ptr, ur.ptr, info.ptr);
      KG_LAUNCH_CHECK();
      KG_CUBLAS(cublasDgemm(p->cublas, CUBLAS_OP_N, CUBLAS_OP_N, g, w, w, &one, rest.ptr, g,
                            ur.ptr, w, &zero, u.ptr, g));
      read_back();
      if (h_info != 0) {
        KG_CUDA(cudaMemcpyAsync(rest.ptr, saved.ptr, rest.bytes(), cudaMemcpyDeviceToDevice, s));
        info.zero();
        qr_svd_kernel<<<1, 1024, 0, s>>>(rest.ptr, g, w, sv.ptr, u.ptr, info.ptr);
        KG_LAUNCH_CHECK();
        read_back();
      }
    } else {
      jacobi_svd_kernel<<<1, 1024, 0, s>>>(rest.ptr, g, w, sv.ptr, order.ptr, info.ptr);
      KG_LAUNCH_CHECK();
      read_back();
    }
    if (h_info != 0)
      fail(KG_ERR_INVALID, "pca: orthonormalising a Krylov block did not converge");
    uint32_t keep = 0;
    while (keep < w && h_sv[keep] > kDropTolerance * scale) ++keep;
    *keep_out = keep;
    if (keep == 0) return none;
    DeviceBuffer<double> out((uint64_t)g * keep, s);
    if (qr) {
      KG_CUDA(cudaMemcpyAsync(out.ptr, u.ptr, out.bytes(), cudaMemcpyDeviceToDevice, s));
    } else {
      gather_unit_columns_kernel<<<blocks_for((uint64_t)g * keep, 256), 256, 0, s>>>(
          rest.ptr, g, keep, sv.ptr, order.ptr, out.ptr);
      KG_LAUNCH_CHECK();
    }
    return out;
  }

  void mean_dot(const double* m, const double* means, uint32_t w, double* out) {
    if (w == 0) return;
    mean_dot_kernel<<<w, 256, 0, s>>>(m, means, g, w, out);
    KG_LAUNCH_CHECK();
  }
};

}  // namespace

void kg_pca::run() {
  if (ran) fail(KG_ERR_STATE, "kg_pca_run called twice");
  kg_ctx* c = ctx;
  cudaStream_t s = stream;
  if (bad_index.ptr) {
    unsigned int bad = 0;
    KG_CUDA(cudaMemcpyAsync(&bad, bad_index.ptr, 4, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    if (bad)
      fail(KG_ERR_INVALID, "a pushed block holds a gene index at or past its " +
                               std::to_string(stream_genes) + " genes");
  }
  const uint64_t n = n_cells;
  const uint32_t g = n_genes;
  if (n < 2)
    fail(KG_ERR_INVALID, std::to_string(n) + " cells reach pca (it needs at least 2)");
  if (g == 0) fail(KG_ERR_INVALID, "pca: the gene set holds no gene");
  if (k > std::min<uint64_t>(n, g))
    fail(KG_ERR_INVALID, "pca: n_components " + std::to_string(k) + " is more than " +
                             std::to_string(std::min<uint64_t>(n, g)) +
                             " (the cells and genes reaching pca)");
  if (nnz >= (1ull << 32)) fail(KG_ERR_INVALID, "pca: more than 2^32 stored values");
  if (n >= (1ull << 32)) fail(KG_ERR_INVALID, "pca: more than 2^32 cells");
  const uint32_t l = width;
  c->total = n * kPasses;
  c->done = 0;

  Trace trace(s, "pca");
  // The products run on the tensor cores (fp16 hi/lo parts of both operands, about 2^-22
  // each; f32 sums of at most 512 terms flushed into f64) when the genes fit 16-bit
  // positions, the block one 64-column tile, the values span at most 2^30, and no gene's
  // mean dwarfs its spread (the rows are centred after the product, so the products'
  // relative error is scaled by |mean| / sd: at most 64, about 2^-16); else on the SIMT
  // pipes in f64 (kyto's arithmetic, any data).
  const char* pchoice = std::getenv("KYTO_GPU_PCA_PRODUCTS");
  bool tc = g <= 65535 && l <= 64 && k <= 64 && !(pchoice && std::string(pchoice) == "simt");
  means.alloc(g, s);
  std::vector<double> squares(g), h_means(g);
  std::vector<uint64_t> colptr(g + 1);
  TcHeld th;
  GeneMajor gm;
  auto check_means = [&]() {
    for (uint32_t i = 0; i < g; ++i)
      if (!std::isfinite(h_means[i]))
        fail(KG_ERR_INVALID, "pca: gene " + std::to_string(i) +
                                 " holds a value that is not finite (NaN or infinity)");
  };
  if (tc) {
    // Gene means (pass 0's sums, pca.rs:707-717), stored counts and centred sums of
    // squares over the stored values (the last pass's, pca.rs:664-676), as products
    // with a column of ones.
    th.build(indptr.ptr, col.ptr, val.ptr, n, g, nnz, c->sm_count, s, trace);
    trace.mark("operand buffers");
    DeviceBuffer<double> sums(g, s), cnt(g, s), sq(g, s);
    th.ones_column();
    th.transposed(1, sums.ptr, s, kValuePlain, nullptr);
    divide_kernel<<<blocks_for(g, 256), 256, 0, s>>>(sums.ptr, g, (double)n, means.ptr);
    KG_LAUNCH_CHECK();
    th.transposed(1, cnt.ptr, s, kValueOne, nullptr);
    th.transposed(1, sq.ptr, s, kValueCentredSquare, means.ptr);
    std::vector<double> h_cnt(g);
    KG_CUDA(cudaMemcpyAsync(h_means.data(), means.ptr, g * 8ull, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaMemcpyAsync(squares.data(), sq.ptr, g * 8ull, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaMemcpyAsync(h_cnt.data(), cnt.ptr, g * 8ull, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    check_means();
    th.check(s);
    double mn = 0.0;
    for (uint32_t i = 0; i < g; ++i) mn += h_means[i] * h_means[i];
    th.mean_norm = std::sqrt(mn);
    colptr[0] = 0;
    for (uint32_t i = 0; i < g; ++i) colptr[i + 1] = colptr[i] + (uint64_t)std::llround(h_cnt[i]);
    double worst_ratio = 0.0;
    for (uint32_t i = 0; i < g; ++i) {
      uint64_t stored = colptr[i + 1] - colptr[i];
      double var = (squares[i] + (double)(n - stored) * h_means[i] * h_means[i]) / (double)n;
      if (var > 0.0) worst_ratio = std::max(worst_ratio, h_means[i] * h_means[i] / var);
    }
    // The values' fp16 parts keep 22 bits of each value down to 2^-18 of the largest and
    // an absolute 2^-39 of it below: data spanning more than 2^30, or scaled out of f32's
    // comfortable range, goes to the f64 path.
    const bool range_ok = th.bx.min_abs == 0.0 || th.bx.max_abs / th.bx.min_abs <= 0x1p30;
    const bool scale_ok = th.bx.scale >= -100 && th.bx.scale <= 100;
    if (worst_ratio > 4096.0 || !range_ok || !scale_ok) {
      tc = false;
      th.clock.release();
      th = TcHeld();
    }
    trace.mark("gene statistics");
  }
  if (!tc) {
    // The gene-major twin of the held input (each gene's values in cell order), cut into
    // segments: the genes' exact f64 statistics and the SIMT products' operand.
    DeviceBuffer<uint32_t> row_of(nnz, s), iota(nnz, s);
    row_of_kernel<<<blocks_for(n * 32, 256), 256, 0, s>>>(indptr.ptr, n, row_of.ptr);
    KG_LAUNCH_CHECK();
    iota_fill(iota.ptr, nnz, s);
    DeviceBuffer<uint32_t> genes_sorted, perm;
    sort_by_gene<uint32_t>(col.ptr, iota.ptr, nnz, g, genes_sorted, perm, s);
    iota.reset();
    gm.colptr.alloc((uint64_t)g + 1, s);
    column_starts(genes_sorted.ptr, nnz, g, gm.colptr.ptr, s);
    genes_sorted.reset();
    gm.row.alloc(nnz, s);
    gm.val.alloc(nnz, s);
    if (nnz) {
      gather_csc_kernel<<<std::min<unsigned>(blocks_for(nnz, 256), 16384), 256, 0, s>>>(
          perm.ptr, row_of.ptr, val.ptr, nnz, gm.row.ptr, gm.val.ptr);
      KG_LAUNCH_CHECK();
    }
    gm.build_segments(g, nnz, s);
    trace.mark("gene-major twin");
    DeviceBuffer<double> ones(n, s), sums(g, s), sq(g, s);
    fill_kernel<<<blocks_for(n, 256), 256, 0, s>>>(ones.ptr, n, 1.0);
    KG_LAUNCH_CHECK();
    gm.transposed_product(ones.ptr, 1, g, sums.ptr, s);
    divide_kernel<<<blocks_for(g, 256), 256, 0, s>>>(sums.ptr, g, (double)n, means.ptr);
    KG_LAUNCH_CHECK();
    gm.centred_squares(means.ptr, g, sq.ptr, s);
    KG_CUDA(cudaMemcpyAsync(h_means.data(), means.ptr, g * 8ull, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaMemcpyAsync(squares.data(), sq.ptr, g * 8ull, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaMemcpyAsync(colptr.data(), gm.colptr.ptr, (g + 1) * 8ull, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    check_means();
    trace.mark("gene statistics");
  }
  products_engine = tc ? "tensor-core" : "simt";

  Dense dense{this, s, g};
  auto colsums = [&](const double* m, uint32_t w, uint32_t ld, double* out) {
    uint64_t rows_per = 2048;
    uint32_t nb = (uint32_t)((n + rows_per - 1) / rows_per);
    DeviceBuffer<double> part((uint64_t)nb * w, s);
    colsum_partial_kernel<<<nb, 64, 0, s>>>(m, n, w, ld, rows_per, part.ptr);
    KG_LAUNCH_CHECK();
    colsum_final_kernel<<<1, 64, 0, s>>>(part.ptr, nb, w, out);
    KG_LAUNCH_CHECK();
  };

  // ---- pass 0: sketch X^T Omega (pca.rs:588-622, end_pass pca.rs:707-749) ----
  DeviceBuffer<double> omega_sums(l, s), sketch1((uint64_t)g * l, s);
  if (tc) {
    th.sketch(cells.ptr, l, seed, sketch1.ptr, omega_sums.ptr, s);
  } else {
    DeviceBuffer<double> omega(n * l, s);
    omega_kernel<<<blocks_for(n, 128), 128, 0, s>>>(cells.ptr, n, l, seed, omega.ptr);
    KG_LAUNCH_CHECK();
    colsums(omega.ptr, l, l, omega_sums.ptr);
    gm.transposed_product(omega.ptr, l, g, sketch1.ptr, s);
  }
  subtract_outer_kernel<<<blocks_for((uint64_t)g * l, 256), 256, 0, s>>>(
      sketch1.ptr, means.ptr, omega_sums.ptr, g, l);
  KG_LAUNCH_CHECK();
  c->done += n;
  check_cancel(c);

  const uint32_t max_basis = (kPasses - 2) * l;
  DeviceBuffer<double> basis((uint64_t)g * max_basis, s), products((uint64_t)g * max_basis, s);
  uint32_t m = 0;  // basis columns
  uint32_t w = 0;
  trace.mark("sketch pass");
  DeviceBuffer<double> block = dense.extend_basis(basis.ptr, 0, sketch1.ptr, l, &w);
  trace.mark("extend basis");
  sketch1.reset();
  bool finished = false;
  std::vector<double> eigen;
  DeviceBuffer<double> loadings64, mean_projection;
  passes_run = 1;

  auto finish_basis = [&]() {
    // pca_dense.rs:141-174 (rayleigh_ritz) and pca.rs:848-862 (finish_basis).
    loadings64.alloc((uint64_t)g * k, s);
    uint32_t taken = std::min(k, m);
    eigen.assign(k, 0.0);
    if (m > 0) {
      DeviceBuffer<double> b((uint64_t)m * m, s), sym((uint64_t)m * m, s), evals(m, s);
      const double one = 1.0, zero = 0.0;
      KG_CUBLAS(cublasDgemm(cublas, CUBLAS_OP_T, CUBLAS_OP_N, m, m, g, &one, basis.ptr, g,
                            products.ptr, g, &zero, b.ptr, m));
      symmetrize_kernel<<<blocks_for((uint64_t)m * m, 256), 256, 0, s>>>(b.ptr, m, sym.ptr);
      KG_LAUNCH_CHECK();
      int lwork = 0;
      KG_CUSOLVER(cusolverDnDsyevd_bufferSize(cusolver, CUSOLVER_EIG_MODE_VECTOR,
                                              CUBLAS_FILL_MODE_LOWER, m, sym.ptr, m,
                                              evals.ptr, &lwork));
      DeviceBuffer<double> work(std::max(lwork, 1), s);
      DeviceBuffer<int> info(1, s);
      KG_CUSOLVER(cusolverDnDsyevd(cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                   m, sym.ptr, m, evals.ptr, work.ptr, lwork, info.ptr));
      std::vector<double> h_evals(m);
      int h_info = 0;
      KG_CUDA(cudaMemcpyAsync(h_evals.data(), evals.ptr, m * 8ull, cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaMemcpyAsync(&h_info, info.ptr, 4, cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaStreamSynchronize(s));
      if (h_info != 0)
        fail(KG_ERR_INVALID, "pca: the Rayleigh-Ritz eigendecomposition did not converge");
      for (uint32_t i = 0; i < taken; ++i) eigen[i] = std::max(h_evals[m - 1 - i], 0.0);
      DeviceBuffer<double> chosen((uint64_t)m * taken, s);
      pick_columns_kernel<<<blocks_for((uint64_t)m * taken, 256), 256, 0, s>>>(
          sym.ptr, m, taken, chosen.ptr);
      KG_LAUNCH_CHECK();
      KG_CUBLAS(cublasDgemm(cublas, CUBLAS_OP_N, CUBLAS_OP_N, g, taken, m, &one, basis.ptr, g,
                            chosen.ptr, m, &zero, loadings64.ptr, g));
    }
    if (taken < k) {
      DeviceBuffer<double> coeff(k, s), vec(g, s);
      complement_kernel<<<1, 256, 0, s>>>(loadings64.ptr, g, taken, k, coeff.ptr, vec.ptr);
      KG_LAUNCH_CHECK();
    }
    flip_signs_kernel<<<k, 256, 0, s>>>(loadings64.ptr, g);
    KG_LAUNCH_CHECK();
    mean_projection.alloc(k, s);
    dense.mean_dot(loadings64.ptr, means.ptr, k, mean_projection.ptr);
    finished = true;
    trace.mark("rayleigh-ritz");
  };

  if (w == 0) finish_basis();
  for (int pass = 1; pass < kPasses - 1 && !finished; ++pass) {
    check_cancel(c);
    // w = x Q - mu^T Q per row (pca.rs:623-645); C Q = X^T W - mu (sum w) (pca.rs:750-775).
    DeviceBuffer<double> block_means(w, s), wsums(w, s);
    dense.mean_dot(block.ptr, means.ptr, w, block_means.ptr);
    double* product = products.ptr + (uint64_t)m * g;
    if (tc) {
      th.rows(block.ptr, w, block_means.ptr, wsums.ptr, nullptr, s);
      th.transposed(w, product, s);
    } else {
      DeviceBuffer<double> block_rm((uint64_t)g * w, s), wrows(n * w, s);
      to_row_major_kernel<<<blocks_for((uint64_t)g * w, 256), 256, 0, s>>>(block.ptr, g, w,
                                                                            block_rm.ptr);
      KG_LAUNCH_CHECK();
      row_product(indptr.ptr, col.ptr, val.ptr, n, block_rm.ptr, block_means.ptr, w, wrows.ptr, s);
      colsums(wrows.ptr, w, w, wsums.ptr);
      gm.transposed_product(wrows.ptr, w, g, product, s);
    }
    trace.mark("product pass");
    subtract_outer_kernel<<<blocks_for((uint64_t)g * w, 256), 256, 0, s>>>(
        product, means.ptr, wsums.ptr, g, w);
    KG_LAUNCH_CHECK();
    KG_CUDA(cudaMemcpyAsync(basis.ptr + (uint64_t)m * g, block.ptr, (uint64_t)g * w * 8,
                            cudaMemcpyDeviceToDevice, s));
    m += w;
    ++passes_run;
    c->done += n;
    if (pass == kPasses - 2) {
      finish_basis();
    } else {
      trace.mark("basis bookkeeping");
      block = dense.extend_basis(basis.ptr, m, product, w, &w);
      trace.mark("extend basis");
      if (w == 0) finish_basis();
    }
  }
  check_cancel(c);

  // ---- last pass: rows (x - mu) V and the centred squares (pca.rs:649-677, 779-797) ----
  trace.mark("basis bookkeeping");
  embedding.alloc(n * k, s);
  if (tc) {
    th.rows(loadings64.ptr, k, mean_projection.ptr, nullptr, embedding.ptr, s);
  } else {
    DeviceBuffer<double> l_rm((uint64_t)g * k, s), rows(n * k, s);
    to_row_major_kernel<<<blocks_for((uint64_t)g * k, 256), 256, 0, s>>>(loadings64.ptr, g, k,
                                                                          l_rm.ptr);
    KG_LAUNCH_CHECK();
    row_product(indptr.ptr, col.ptr, val.ptr, n, l_rm.ptr, mean_projection.ptr, k, rows.ptr, s);
    to_f32_kernel<<<std::min<unsigned>(blocks_for(n * k, 256), 16384), 256, 0, s>>>(
        rows.ptr, n * k, embedding.ptr);
    KG_LAUNCH_CHECK();
  }
  trace.mark("embedding pass");
  loadings.alloc((uint64_t)stream_genes * k, s);
  loadings.zero();
  scatter_loadings_kernel<<<blocks_for((uint64_t)g * k, 256), 256, 0, s>>>(
      loadings64.ptr, g, k, set_genes.ptr, stream_genes, loadings.ptr);
  KG_LAUNCH_CHECK();
  wait_stream(c, s);
  if (tc) th.check(s);
  th.clock.collect(product_launches, product_ms, product_bytes);
  ++passes_run;
  c->done += n;
  double total = 0.0;
  for (uint32_t i = 0; i < g; ++i) {
    uint64_t stored = colptr[i + 1] - colptr[i];
    total += squares[i] + (double)(n - stored) * h_means[i] * h_means[i];
  }
  double total_variance = total / ((double)n - 1.0);
  bool constant = total_variance == 0.0;
  variance.assign(k, 0.0);
  variance_ratio.assign(k, 0.0);
  for (uint32_t i = 0; i < k; ++i) {
    variance[i] = constant ? 0.0 : eigen[i] / ((double)n - 1.0);
    variance_ratio[i] = variance[i] / total_variance;
  }
  ran = true;
}

namespace kg {

// A new session on ctx (kyto's PcaAccumulator::new, pca.rs:343-403): a pooled stream and
// solver handles, the gene map checked and uploaded.
kg_pca* make_session(kg_ctx* ctx, const kg_pca_params* params) {
  if (params->n_components == 0) fail(KG_ERR_INVALID, "pca: n_components must be at least 1");
  if (params->n_genes == 0) fail(KG_ERR_INVALID, "pca: blocks of 0 genes");
  use_device(ctx);
  auto* p = new kg_pca();
  try {
    p->ctx = ctx;
    {
      std::lock_guard<std::mutex> lock(ctx->res_mu);
      if (!ctx->free_res.empty()) {
        const kg_ctx::SessionRes r = ctx->free_res.back();
        ctx->free_res.pop_back();
        p->stream = r.stream;
        p->cublas = r.cublas;
        p->cusolver = r.cusolver;
      }
    }
    if (!p->stream) KG_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    if (!p->cublas) {
      KG_CUBLAS(cublasCreate(&p->cublas));
      KG_CUBLAS(cublasSetStream(p->cublas, p->stream));
    }
    if (!p->cusolver) {
      KG_CUSOLVER(cusolverDnCreate(&p->cusolver));
      KG_CUSOLVER(cusolverDnSetStream(p->cusolver, p->stream));
    }
    p->k = params->n_components;
    p->stream_genes = params->n_genes;
    p->seed = params->seed;
    p->target_sum = params->target_sum;
    p->log1p = params->log1p;
    if (params->gene_map) {
      std::vector<uint32_t> map(params->n_genes), set;
      KG_CUDA(cudaMemcpy(map.data(), params->gene_map, params->n_genes * 4ull,
                         cudaMemcpyDefault));
      uint32_t next = 0;
      for (uint32_t i = 0; i < params->n_genes; ++i) {
        if (map[i] == kNoGene) continue;
        if (map[i] != next)
          fail(KG_ERR_INVALID, "pca: gene_map must number the kept genes 0, 1, ... in order");
        set.push_back(i);
        ++next;
      }
      p->n_genes = next;
      p->gene_map.alloc(params->n_genes, p->stream);
      KG_CUDA(cudaMemcpyAsync(p->gene_map.ptr, map.data(), map.size() * 4, cudaMemcpyHostToDevice,
                              p->stream));
      p->set_genes.alloc(set.size(), p->stream);
      if (!set.empty())
        KG_CUDA(cudaMemcpyAsync(p->set_genes.ptr, set.data(), set.size() * 4,
                                cudaMemcpyHostToDevice, p->stream));
      KG_CUDA(cudaStreamSynchronize(p->stream));
    } else {
      p->n_genes = params->n_genes;
    }
    p->width = std::min<uint32_t>(p->k + kOversamples, p->n_genes);
    p->indptr.alloc(1, p->stream);
    p->indptr.zero();
  } catch (...) {
    delete p;
    throw;
  }
  return p;
}

}  // namespace kg

extern "C" {

kg_status kg_pca_knn_batch(kg_ctx* ctx, const kg_pca_params* params, uint32_t n_samples,
                           const kg_batch_sample* samples, uint32_t n_neighbors,
                           float* embedding, double* variance, uint64_t* indptr,
                           uint32_t* indices, float* distances, kg_batch_stats* stats) {
  return guarded([&] {
    if (!ctx || !params || !samples || !embedding || !indptr || !indices || !distances)
      fail(KG_ERR_INVALID, "kg_pca_knn_batch: NULL argument");
    if (n_samples == 0) fail(KG_ERR_INVALID, "kg_pca_knn_batch: no samples");
    const uint32_t kc = params->n_components;
    std::vector<uint64_t> first(n_samples + 1, 0);
    uint32_t k = 0, d = 0;
    for (uint32_t i = 0; i < n_samples; ++i) {
      const kg_batch_sample& b = samples[i];
      if (b.n_rows && (!b.indptr || !b.indices || !b.values))
        fail(KG_ERR_INVALID, "kg_pca_knn_batch: sample " + std::to_string(i) + ": NULL array");
      try {
        check_search_args(b.n_rows, kc, kc, n_neighbors, k, d);
      } catch (const Error& e) {
        fail(e.status, "sample " + std::to_string(i) + ": " + e.message);
      }
      first[i + 1] = first[i] + b.n_rows;
    }
    const uint64_t n = first[n_samples];
    use_device(ctx);
    cudaStream_t s = ctx->stream;
    DeviceBuffer<float> emb_all(n * kc, s);
    KG_CUDA(cudaStreamSynchronize(s));
    std::vector<double> var_all((size_t)n_samples * kc);
    // The samples' PCA: workers take the next sample, largest first, until none is left
    // (the largest samples do not start last and become the tail); each session has its
    // own stream, so the small samples' kernels run side by side. KYTO_GPU_BATCH_WORKERS
    // sets the worker count (default 8).
    const auto t0 = std::chrono::steady_clock::now();
    unsigned max_workers = 8;
    if (const char* w = std::getenv("KYTO_GPU_BATCH_WORKERS"))
      max_workers = (unsigned)std::max(1, std::min(64, std::atoi(w)));
    const unsigned workers = std::min<unsigned>(n_samples, max_workers);
    std::vector<uint32_t> order(n_samples);
    for (uint32_t i = 0; i < n_samples; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
      return samples[a].n_rows > samples[b].n_rows;
    });
    std::atomic<uint32_t> next{0};
    std::vector<std::exception_ptr> errors(workers);
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < workers; ++w) {
      pool.emplace_back([&, w] {
        try {
          KG_CUDA(cudaSetDevice(ctx->device));
          g_stage_pageable = true;
          for (;;) {
            const uint32_t at = next.fetch_add(1);
            if (at >= n_samples) break;
            const uint32_t i = order[at];
            check_cancel(ctx);
            std::unique_ptr<kg_pca> p(make_session(ctx, params));
            const kg_batch_sample& b = samples[i];
            p->push(b.indptr, b.indices, b.values, b.dtype, b.n_rows, nullptr, false);
            p->run();
            KG_CUDA(cudaMemcpyAsync(emb_all.ptr + first[i] * kc, p->embedding.ptr,
                                    b.n_rows * kc * 4ull, cudaMemcpyDeviceToDevice, p->stream));
            KG_CUDA(cudaStreamSynchronize(p->stream));
            std::memcpy(&var_all[(size_t)i * kc], p->variance.data(), kc * 8ull);
          }
        } catch (...) {
          errors[w] = std::current_exception();
          next.store(n_samples);
        }
      });
    }
    for (std::thread& t : pool) t.join();
    for (const std::exception_ptr& e : errors)
      if (e) std::rethrow_exception(e);
    const double pca_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    // Every sample's neighbours in one batched search.
    const auto t1 = std::chrono::steady_clock::now();
    kg_knn_stats ks{};
    knn_batch_run(ctx, emb_all.ptr, n, kc, d, k, first, indptr, indices, distances, &ks);
    KG_CUDA(cudaMemcpyAsync(embedding, emb_all.ptr, n * kc * 4ull, cudaMemcpyDefault, s));
    wait_stream(ctx, s);
    if (variance) std::memcpy(variance, var_all.data(), var_all.size() * 8);
    if (stats) {
      stats->pca_ms = pca_ms;
      stats->knn_ms = std::chrono::duration<double, std::milli>(
                          std::chrono::steady_clock::now() - t1).count();
      stats->workers = workers;
      stats->knn = ks;
    }
  });
}

kg_status kg_pca_begin(kg_ctx* ctx, const kg_pca_params* params, kg_pca** out) {
  return guarded([&] {
    if (!ctx || !params || !out) fail(KG_ERR_INVALID, "kg_pca_begin: NULL argument");
    *out = nullptr;
    *out = make_session(ctx, params);
  });
}

kg_status kg_pca_push_block(kg_pca* pca, const uint64_t* indptr, const uint32_t* indices,
                            const void* values, kg_dtype dtype, uint64_t n_rows,
                            const uint64_t* cells) {
  return guarded([&] {
    if (!pca || (n_rows && (!indptr || !indices || !values)))
      fail(KG_ERR_INVALID, "kg_pca_push_block: NULL argument");
    use_device(pca->ctx);
    pca->push(indptr, indices, values, dtype, n_rows, cells, false);
  });
}

kg_status kg_pca_push_block_async(kg_pca* pca, const uint64_t* indptr, const uint32_t* indices,
                                  const void* values, kg_dtype dtype, uint64_t n_rows,
                                  const uint64_t* cells) {
  return guarded([&] {
    if (!pca || (n_rows && (!indptr || !indices || !values)))
      fail(KG_ERR_INVALID, "kg_pca_push_block_async: NULL argument");
    use_device(pca->ctx);
    pca->push(indptr, indices, values, dtype, n_rows, cells, true);
  });
}

kg_status kg_pca_push_tiles(kg_pca* pca, const kg_tile_block* block) {
  return guarded([&] {
    if (!pca || !block) fail(KG_ERR_INVALID, "kg_pca_push_tiles: NULL argument");
    use_device(pca->ctx);
    if (pca->ran) fail(KG_ERR_STATE, "kg_pca_push_tiles after kg_pca_run");
    cudaStream_t s = pca->stream;
    const TileShape sh = tile_shape(block, s);
    const uint64_t rows = block->rows;
    DeviceBuffer<uint64_t> indptr(rows + 1, s), cells(rows, s);
    DeviceBuffer<uint32_t> indices(sh.nnz, s), values(sh.nnz, s);
    join_tiles(pca->ctx, s, block, sh, indptr.ptr, indices.ptr, values.ptr);
    // The rows' table positions b C + r (docs/format.md 4.1).
    iota64_kernel<<<blocks_for(rows, 256), 256, 0, s>>>(
        cells.ptr, rows, block->block * (uint64_t)block->cell_block_size);
    KG_LAUNCH_CHECK();
    pca->push(indptr.ptr, indices.ptr, values.ptr, block->dtype, rows, cells.ptr, false);
  });
}

kg_status kg_pca_run(kg_pca* pca) {
  return guarded([&] {
    if (!pca) fail(KG_ERR_INVALID, "kg_pca_run: NULL argument");
    use_device(pca->ctx);
    const auto t0 = std::chrono::steady_clock::now();
    pca->run();
    pca->run_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  });
}

kg_status kg_pca_run_stats(const kg_pca* pca, kg_pca_stats* out) {
  return guarded([&] {
    if (!pca || !out) fail(KG_ERR_INVALID, "kg_pca_run_stats: NULL argument");
    if (!pca->ran) fail(KG_ERR_STATE, "kg_pca_run_stats before kg_pca_run");
    out->product_launches = pca->product_launches;
    out->passes_run = pca->passes_run;
    out->product_ms = pca->product_ms;
    out->product_bytes = pca->product_bytes;
    out->run_ms = pca->run_ms;
  });
}

kg_status kg_diag_spmm(kg_ctx* ctx, const uint64_t* indptr, const uint32_t* indices,
                       const float* values, uint64_t n_rows, uint32_t n_cols,
                       int32_t transposed, int32_t value_mode, const double* row_means,
                       const double* dense, uint32_t width, double* out) {
  return guarded([&] {
    if (!ctx || !indptr || !out || (!dense && value_mode == kValuePlain))
      fail(KG_ERR_INVALID, "kg_diag_spmm: NULL argument");
    if (width == 0 || width > 64) fail(KG_ERR_INVALID, "kg_diag_spmm: width must be 1..64");
    if (value_mode < kValuePlain || value_mode > kValueOne)
      fail(KG_ERR_INVALID, "kg_diag_spmm: unknown value mode");
    if (n_cols > 65535) fail(KG_ERR_INVALID, "kg_diag_spmm: at most 65,535 columns");
    use_device(ctx);
    cudaStream_t s = ctx->stream;
    DeviceBuffer<uint64_t> hp;
    const uint64_t* d_ptr = device_view(indptr, n_rows + 1, hp, s);
    uint64_t nnz = 0;
    KG_CUDA(cudaMemcpyAsync(&nnz, d_ptr + n_rows, 8, cudaMemcpyDefault, s));
    KG_CUDA(cudaStreamSynchronize(s));
    DeviceBuffer<uint32_t> hi_idx;
    DeviceBuffer<float> hv;
    const uint32_t* d_idx = device_view(indices, nnz, hi_idx, s);
    const float* d_val = device_view(values, nnz, hv, s);
    Blocked bx, bxt;
    build_blocked(d_ptr, d_idx, d_val, n_rows, n_cols, nnz, bx, s);
    const Blocked* sp = &bx;
    if (transposed) {
      transpose_blocked(d_ptr, d_idx, d_val, n_rows, n_cols, nnz, bx, bxt, s);
      sp = &bxt;
    }
    const uint64_t rows = sp->rows, K = sp->K, ld = dense_ld(K);
    DeviceBuffer<double> hd;
    int dscale = 0;
    DeviceBuffer<uint16_t> dt(64 * ld, s);
    if (value_mode == kValuePlain) {
      std::vector<double> h((size_t)K * width);
      KG_CUDA(cudaMemcpyAsync(h.data(), dense, h.size() * 8, cudaMemcpyDefault, s));
      KG_CUDA(cudaStreamSynchronize(s));
      double mx = 0.0;
      for (double v : h) mx = std::max(mx, std::fabs(v));
      dscale = part_scale(mx);
      hd.alloc(h.size(), s);
      KG_CUDA(cudaMemcpyAsync(hd.ptr, h.data(), h.size() * 8, cudaMemcpyHostToDevice, s));
      split_t_kernel<<<blocks_for(64 * ld / 2, 256), 256, 0, s>>>(hd.ptr, (uint32_t)K, width, ld,
                                                                  dscale, dt.ptr);
      KG_LAUNCH_CHECK();
    } else {
      fill_rows_kernel<<<blocks_for(64 * ld, 256), 256, 0, s>>>(dt.ptr, K, ld);
      KG_LAUNCH_CHECK();
    }
    DeviceBuffer<double> hm;
    const double* d_means = nullptr;
    if (value_mode == kValueCentredSquare) {
      if (!row_means) fail(KG_ERR_INVALID, "kg_diag_spmm: centred squares need row_means");
      d_means = device_view(row_means, rows, hm, s);
    }
    constexpr uint64_t kSeg = 512;
    const uint64_t segs = (sp->n_chunks + kSeg - 1) / kSeg;
    DeviceBuffer<double> partial(std::max<uint64_t>(segs, 1) * rows * 64, s), res(rows * width, s);
    DeviceBuffer<int> err(1, s);
    err.zero();
    SpmmArgs a;
    a.s = sp;
    a.value_mode = value_mode;
    a.row_means = d_means;
    a.seg_chunks = kSeg;
    a.dt = dt.ptr;
    a.ld_t = ld;
    a.dt_scale = dscale;
    a.out.mode = kOutPartial;
    a.out.partial = partial.ptr;
    a.sm_count = ctx->sm_count;
    a.error = err.ptr;
    spmm_tc(a, s);
    reduce_segments_kernel<<<blocks_for(rows * width, 256), 256, 0, s>>>(
        partial.ptr, (uint32_t)segs, (uint32_t)rows, width, res.ptr);
    KG_LAUNCH_CHECK();
    KG_CUDA(cudaMemcpyAsync(out, res.ptr, rows * width * 8, cudaMemcpyDefault, s));
    wait_stream(ctx, s);
    int h_err = 0;  // read after the bounded wait: no copy outlives this frame
    KG_CUDA(cudaMemcpyAsync(&h_err, err.ptr, 4, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    if (h_err) fail(KG_ERR_TIMEOUT, "the tensor-core product gave up waiting on its pipeline");
  });
}

kg_status kg_diag_omega(kg_ctx* ctx, uint64_t seed, const uint64_t* cells, uint64_t n,
                        uint32_t width, double* out) {
  return guarded([&] {
    if (!ctx || !cells || !out) fail(KG_ERR_INVALID, "kg_diag_omega: NULL argument");
    if (width == 0 || width > 64) fail(KG_ERR_INVALID, "kg_diag_omega: width must be 1..64");
    if (n == 0) return;
    use_device(ctx);
    cudaStream_t s = ctx->stream;
    DeviceBuffer<uint64_t> hc;
    const uint64_t* d_cells = device_view(cells, n, hc, s);
    DeviceBuffer<double> omega(n * width, s);
    omega_kernel<<<blocks_for(n, 128), 128, 0, s>>>(d_cells, n, width, seed, omega.ptr);
    KG_LAUNCH_CHECK();
    KG_CUDA(cudaMemcpyAsync(out, omega.ptr, n * width * 8ull, cudaMemcpyDefault, s));
    wait_stream(ctx, s);
  });
}

kg_status kg_pca_results(kg_pca* pca, float* embedding, float* loadings, double* variance,
                         double* variance_ratio, double* means) {
  return guarded([&] {
    if (!pca) fail(KG_ERR_INVALID, "kg_pca_results: NULL argument");
    if (!pca->ran) fail(KG_ERR_STATE, "kg_pca_results before kg_pca_run");
    use_device(pca->ctx);
    cudaStream_t s = pca->stream;
    if (embedding)
      KG_CUDA(cudaMemcpyAsync(embedding, pca->embedding.ptr, pca->embedding.bytes(),
                              cudaMemcpyDefault, s));
    if (loadings)
      KG_CUDA(cudaMemcpyAsync(loadings, pca->loadings.ptr, pca->loadings.bytes(),
                              cudaMemcpyDefault, s));
    if (means)
      KG_CUDA(cudaMemcpyAsync(means, pca->means.ptr, pca->means.bytes(), cudaMemcpyDefault, s));
    wait_stream(pca->ctx, s);
    if (variance) std::memcpy(variance, pca->variance.data(), pca->k * 8ull);
    if (variance_ratio) std::memcpy(variance_ratio, pca->variance_ratio.data(), pca->k * 8ull);
  });
}

kg_status kg_pca_info(const kg_pca* pca, uint64_t* n_cells, uint32_t* n_pca_genes,
                      uint32_t* passes_run) {
  return guarded([&] {
    if (!pca) fail(KG_ERR_INVALID, "kg_pca_info: NULL argument");
    if (n_cells) *n_cells = pca->n_cells;
    if (n_pca_genes) *n_pca_genes = pca->n_genes;
    if (passes_run) *passes_run = pca->passes_run;
  });
}

}  // extern "C"

// DLPack's C ABI (the open DLPack standard, dlpack.h v0.8): the layouts a consumer reads,
// with the standard's names and field order (a consumer checks nothing but these bytes).
struct DLDevice {
  int32_t device_type;  // kDLCUDA = 2
  int32_t device_id;
};
struct DLDataType {
  uint8_t code;  // kDLFloat = 2
  uint8_t bits;
  uint16_t lanes;
};
struct DLTensor {
  void* data;
  DLDevice device;
  int32_t ndim;
  DLDataType dtype;
  int64_t* shape;
  int64_t* strides;
  uint64_t byte_offset;
};
struct DLManagedTensor {
  DLTensor dl_tensor;
  void* manager_ctx;
  void (*deleter)(DLManagedTensor* self);
};

namespace {

// One exported result: the managed tensor, its shape and the device its copy lives on.
struct DlpackExport {
  DLManagedTensor managed{};
  int64_t shape[2] = {0, 0};
  int device = 0;
};

std::atomic<int64_t> g_dlpack_live{0};

void dlpack_deleter(DLManagedTensor* t) {
  auto* e = static_cast<DlpackExport*>(t->manager_ctx);
  int prev = 0;
  const bool had = cudaGetDevice(&prev) == cudaSuccess;
  cudaSetDevice(e->device);
  if (t->dl_tensor.data) cudaFree(t->dl_tensor.data);
  if (had) cudaSetDevice(prev);
  delete e;
  g_dlpack_live.fetch_sub(1);
}

}  // namespace

extern "C" {

kg_status kg_pca_result_dlpack(kg_pca* pca, int32_t which, DLManagedTensor** out) {
  return guarded([&] {
    if (!pca || !out) fail(KG_ERR_INVALID, "kg_pca_result_dlpack: NULL argument");
    if (which != KG_RESULT_EMBEDDING && which != KG_RESULT_LOADINGS)
      fail(KG_ERR_INVALID, "kg_pca_result_dlpack: which must be KG_RESULT_EMBEDDING or "
                           "KG_RESULT_LOADINGS");
    if (!pca->ran) fail(KG_ERR_STATE, "kg_pca_result_dlpack before kg_pca_run");
    use_device(pca->ctx);
    const DeviceBuffer<float>& src = which == KG_RESULT_EMBEDDING ? pca->embedding : pca->loadings;
    auto e = std::make_unique<DlpackExport>();
    e->device = pca->ctx->device;
    e->shape[0] = (int64_t)(src.count / pca->k);
    e->shape[1] = (int64_t)pca->k;
    void* copy = nullptr;
    if (src.bytes()) KG_CUDA(cudaMalloc(&copy, src.bytes()));
    struct Guard {
      void* p;
      ~Guard() {
        if (p) cudaFree(p);
      }
    } guard{copy};
    if (src.bytes())
      KG_CUDA(cudaMemcpyAsync(copy, src.ptr, src.bytes(), cudaMemcpyDeviceToDevice, pca->stream));
    wait_stream(pca->ctx, pca->stream);
    DLTensor& t = e->managed.dl_tensor;
    t.data = copy;
    t.device = {2, e->device};
    t.ndim = 2;
    t.dtype = {2, 32, 1};
    t.shape = e->shape;
    t.strides = nullptr;
    t.byte_offset = 0;
    e->managed.manager_ctx = e.get();
    e->managed.deleter = dlpack_deleter;
    guard.p = nullptr;
    *out = &e->managed;
    e.release();
    g_dlpack_live.fetch_add(1);
  });
}

void kg_dlpack_free(DLManagedTensor* tensor) {
  if (tensor && tensor->deleter) tensor->deleter(tensor);
}

kg_status kg_diag_dlpack_live(int64_t* count) {
  return guarded([&] {
    if (!count) fail(KG_ERR_INVALID, "kg_diag_dlpack_live: NULL argument");
    *count = g_dlpack_live.load();
  });
}

kg_status kg_pca_embedding_device(const kg_pca* pca, const float** out) {
  return guarded([&] {
    if (!pca || !out) fail(KG_ERR_INVALID, "kg_pca_embedding_device: NULL argument");
    if (!pca->ran) fail(KG_ERR_STATE, "kg_pca_embedding_device before kg_pca_run");
    *out = pca->embedding.ptr;
  });
}

void kg_pca_free(kg_pca* pca) {
  if (!pca) return;
  cudaSetDevice(pca->ctx->device);
  delete pca;
}

}  // extern "C"
