// Test infrastructure, not product code: a CPU restatement of kyto's CPU algorithms for
// the PCA -> exact-kNN path, used only as the checker by the tests, by smoke() and as
// the CPU baseline leg of bench.py. The product (libkyto_gpu.so) never links or calls it.
//
// Built with -ffp-contract=off: kyto's Rust never fuses a*b+c, so neither may this file,
// or the f64 keys and sums would not carry kyto's bits.
//
// Citations are to datavil/kyto, paths within that project.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include <immintrin.h>
#include <omp.h>

namespace {

constexpr int kSumLanes = 8;  // crates/kyto-exec/src/kernels.rs:41

// crates/kyto-exec/src/kernels.rs:281-292 (combine_lanes): ((a0+a4)+(a2+a6))+((a1+a5)+(a3+a7)).
inline double combine_lanes(const double* lanes) {
  double h0 = lanes[0] + lanes[4];
  double h1 = lanes[1] + lanes[5];
  double h2 = lanes[2] + lanes[6];
  double h3 = lanes[3] + lanes[7];
  double q0 = h0 + h2;
  double q1 = h1 + h3;
  return q0 + q1;
}

// crates/kyto-exec/src/kernels.rs:420-448 (pair_sum, dot = false): component j's
// difference and square in f64 into lane j % 8, then the fixed tree.
inline double squared_distance(const float* q, const float* p, uint32_t width) {
  double lanes[kSumLanes] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (uint32_t j = 0; j < width; ++j) {
    double d = (double)q[j] - (double)p[j];
    lanes[j % kSumLanes] += d * d;
  }
  return combine_lanes(lanes);
}

// crates/kyto-exec/src/neighbors.rs:448-479 (Nearest::offer): the k smallest by (key, row).
struct Nearest {
  uint32_t k;
  std::vector<std::pair<double, uint32_t>> entries;
  explicit Nearest(uint32_t k_) : k(k_) { entries.reserve(k_ + 1); }
  static bool before(const std::pair<double, uint32_t>& e, double key, uint32_t index) {
    return e.first < key || (e.first == key && e.second < index);
  }
  void offer(double key, uint32_t index) {
    if (entries.size() == k) {
      if (before(entries.back(), key, index)) return;
      entries.pop_back();
    }
    size_t lo = 0, hi = entries.size();
    while (lo < hi) {
      size_t mid = (lo + hi) / 2;
      if (before(entries[mid], key, index)) lo = mid + 1; else hi = mid;
    }
    entries.insert(entries.begin() + lo, {key, index});
  }
};

inline float u32_or_f32(const void* values, int dtype, uint64_t i) {
  if (dtype == 0) return (float)((const uint32_t*)values)[i];
  return ((const float*)values)[i];
}

inline double u32_or_f32_wide(const void* values, int dtype, uint64_t i) {
  if (dtype == 0) return (double)((const uint32_t*)values)[i];
  return (double)((const float*)values)[i];
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------------
// normalize_total + log1p: crates/kyto-exec/src/elementwise.rs:149-199,241-269,
// crates/kyto-exec/src/kernels.rs:131-138,207-226,273-276, kernels/log1p.rs:49-75.
// dtype 0 = u32 counts, 1 = f32 values. target_sum NaN: no normalize_total.
// ---------------------------------------------------------------------------------
void ko_normalize_log1p(const uint64_t* indptr, const void* values, int dtype,
                        uint64_t n_rows, double target_sum, int do_log1p, float* out) {
  uint64_t nnz = indptr[n_rows];
  // cell_totals: a u32 count that is not exactly a float32 makes every value round first.
  bool exact = true;
  for (uint64_t i = 0; i < nnz && exact; ++i) {
    double wide = u32_or_f32_wide(values, dtype, i);
    exact = (double)(float)wide == wide;
  }
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t r = 0; r < (int64_t)n_rows; ++r) {
    uint64_t s = indptr[r], e = indptr[r + 1];
    float divisor = 1.0f;
    if (!std::isnan(target_sum)) {
      double lanes[kSumLanes] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (uint64_t i = s; i < e; ++i) {
        double v = exact ? u32_or_f32_wide(values, dtype, i)
                         : (double)u32_or_f32(values, dtype, i);
        lanes[(i - s) % kSumLanes] += v;
      }
      double total = combine_lanes(lanes);
      divisor = (float)total / (float)target_sum;  // elementwise.rs:262-269
      if (divisor == 0.0f) divisor = 1.0f;
    }
    for (uint64_t i = s; i < e; ++i) {
      float v = u32_or_f32(values, dtype, i);
      if (!std::isnan(target_sum)) v = v / divisor;
      if (do_log1p) v = (float)std::log1p((double)v);
      out[i] = v;
    }
  }
}

// ---------------------------------------------------------------------------------
// HVG (seurat) moments: crates/kyto-exec/src/hvg_pass.rs:157-219 over one leaf, cells in
// order: t = f32(expm1(f64(v))), sums += t, sums_of_squares += f64(t * t in f32),
// positives += (v > 0).
// ---------------------------------------------------------------------------------
void ko_hvg_moments(const uint64_t* indptr, const uint32_t* indices, const float* values,
                    uint64_t n_rows, uint32_t n_genes, double* sums, double* sums_sq,
                    uint64_t* positives) {
  std::fill(sums, sums + n_genes, 0.0);
  std::fill(sums_sq, sums_sq + n_genes, 0.0);
  std::fill(positives, positives + n_genes, 0);
  for (uint64_t r = 0; r < n_rows; ++r) {
    for (uint64_t i = indptr[r]; i < indptr[r + 1]; ++i) {
      uint32_t g = indices[i];
      float v32 = values[i];
      double v = (double)v32;
      if (v > 0.0) positives[g] += 1;
      float t = (float)std::expm1(v);
      sums[g] += (double)t;
      float sq = t * t;
      sums_sq[g] += (double)sq;
    }
  }
}

// ---------------------------------------------------------------------------------
// PCA folds over one leaf (all rows, cell order): crates/kyto-exec/src/pca.rs:499-679.
// gene_map: one entry per stream gene, its position among the PCA's genes or
// 0xFFFFFFFF to skip (pca.rs:352-372); NULL means every gene, in order.
// ---------------------------------------------------------------------------------

// pca.rs:936-950 (omega_row, mix).
static inline uint64_t mix(uint64_t v) {
  v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
  v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
  return v ^ (v >> 31);
}

void ko_omega_rows(uint64_t seed, const uint64_t* cells, uint64_t n, uint32_t width,
                   double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < (int64_t)n; ++r) {
    uint64_t state = mix(seed ^ mix(cells[r] + 0x9E3779B97F4A7C15ULL));
    for (uint32_t j = 0; j < width; ++j) {
      state += 0x9E3779B97F4A7C15ULL;
      out[(uint64_t)r * width + j] = (double)(mix(state) >> 11) * 0x1p-52 - 1.0;
    }
  }
}

static inline uint32_t position_of(const uint32_t* gene_map, uint32_t gene) {
  return gene_map ? gene_map[gene] : gene;
}

// The PCA genes cut into parts (pca.rs:879-905, gene_parts): positions [start, end)
// and the stream genes [stream_start, stream_end) that hold them. Each part's genes
// fold their rows in cell order, so the sums carry the same bits whatever the cut; kyto
// cuts at 256 genes (GENES_PER_PART, pca.rs:128), and this restatement cuts finer only
// while there are fewer parts than host threads (every part reads every row's
// projection, so finer parts cost traffic).
//
// The width-wide f64 loops below are compiled for AVX-512 and for the baseline target
// and picked at run time (target_clones): each element sees the same multiply and add
// in the same order either way, so the bits do not depend on the host.
struct GenePart {
  uint32_t start, end, stream_start, stream_end;
};

static std::vector<GenePart> gene_parts(const uint32_t* gene_map, uint32_t stream_genes,
                                        uint32_t n_genes) {
  std::vector<uint32_t> set_genes;  // position -> stream gene (positions rise with genes)
  if (gene_map) {
    set_genes.assign(n_genes, stream_genes);
    for (uint32_t g = 0; g < stream_genes; ++g)
      if (gene_map[g] != 0xFFFFFFFFu) set_genes[gene_map[g]] = g;
  }
  auto stream_at = [&](uint32_t position) -> uint32_t {
    if (position >= n_genes) return stream_genes;
    return gene_map ? set_genes[position] : position;
  };
  const uint32_t threads = (uint32_t)omp_get_max_threads();
  uint32_t size = 256;
  while (size > 16 && (n_genes + size - 1) / size < threads) size /= 2;
  std::vector<GenePart> parts;
  for (uint32_t start = 0; start < n_genes; start += size) {
    uint32_t end = std::min(n_genes, start + size);
    parts.push_back({start, end, stream_at(start), stream_at(end)});
  }
  return parts;
}

// y[j] += v * x[j] for j < n (separate multiply and add; the arrays do not overlap).
__attribute__((always_inline)) static inline void axpy(
    double* __restrict__ y, const double* __restrict__ x, double v, uint32_t n) {
  for (uint32_t j = 0; j < n; ++j) y[j] += v * x[j];
}

// Row r's stored entries of part `part`: one run of the row (its genes rise), found by
// binary search (pca.rs:527-537, part_row).
static inline void part_run(const uint64_t* indptr, const uint32_t* indices, uint64_t r,
                            const GenePart& part, uint64_t& lo, uint64_t& hi) {
  const uint32_t* first = indices + indptr[r];
  const uint32_t* last = indices + indptr[r + 1];
  const uint32_t* a = std::lower_bound(first, last, part.stream_start);
  const uint32_t* b = std::lower_bound(a, last, part.stream_end);
  lo = (uint64_t)(a - indices);
  hi = (uint64_t)(b - indices);
}

// Pass 0 (pca.rs:588-622): n_cells, gene sums, Omega column sums, sketch X^T Omega.
__attribute__((target_clones("avx512f", "default")))
void ko_pca_sketch(const uint64_t* indptr, const uint32_t* indices, const float* values,
                   uint64_t n_rows, const uint32_t* gene_map, uint32_t stream_genes,
                   uint32_t n_genes, const uint64_t* cells, uint64_t seed, uint32_t width,
                   double* sums, double* omega_sums, double* sketch) {
  std::vector<double> omega((size_t)n_rows * width);
  ko_omega_rows(seed, cells, n_rows, width, omega.data());
  std::fill(sums, sums + n_genes, 0.0);
  std::fill(omega_sums, omega_sums + width, 0.0);
  std::fill(sketch, sketch + (size_t)n_genes * width, 0.0);
  for (uint64_t r = 0; r < n_rows; ++r)
    for (uint32_t j = 0; j < width; ++j) omega_sums[j] += omega[r * width + j];
  const std::vector<GenePart> parts = gene_parts(gene_map, stream_genes, n_genes);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t pi = 0; pi < (int64_t)parts.size(); ++pi) {
    const GenePart& part = parts[pi];
    for (uint64_t r = 0; r < n_rows; ++r) {
      const double* om = &omega[r * width];
      uint64_t lo, hi;
      part_run(indptr, indices, r, part, lo, hi);
      for (uint64_t i = lo; i < hi; ++i) {
        uint32_t p = position_of(gene_map, indices[i]);
        if (p == 0xFFFFFFFFu) continue;
        double v = (double)values[i];
        sums[p] += v;
        axpy(&sketch[(size_t)p * width], om, v, width);
      }
    }
  }
}

// Each row's projection -offsets + sum value * matrix[gene], its values added in the
// row's gene order (pca.rs:548-586, `project`).
__attribute__((target_clones("avx512f", "default")))
void ko_pca_project(const uint64_t* indptr, const uint32_t* indices, const float* values,
                    uint64_t n_rows, const uint32_t* gene_map, const double* matrix,
                    const double* offsets, uint32_t width, double* out) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t r = 0; r < (int64_t)n_rows; ++r) {
    double* row = &out[(uint64_t)r * width];
    for (uint32_t j = 0; j < width; ++j) row[j] = -offsets[j];
    for (uint64_t i = indptr[r]; i < indptr[r + 1]; ++i) {
      uint32_t p = position_of(gene_map, indices[i]);
      if (p == 0xFFFFFFFFu) continue;
      axpy(row, &matrix[(size_t)p * width], (double)values[i], width);
    }
  }
}

// Passes 1..q (pca.rs:623-645): w = x Q - mu^T Q per row, sums of w, product X^T W.
__attribute__((target_clones("avx512f", "default")))
void ko_pca_product(const uint64_t* indptr, const uint32_t* indices, const float* values,
                    uint64_t n_rows, const uint32_t* gene_map, uint32_t stream_genes,
                    uint32_t n_genes, const double* block, const double* block_means,
                    uint32_t width, double* product, double* sums) {
  std::vector<double> projected((size_t)n_rows * width);
  ko_pca_project(indptr, indices, values, n_rows, gene_map, block, block_means, width,
                 projected.data());
  std::fill(sums, sums + width, 0.0);
  std::fill(product, product + (size_t)n_genes * width, 0.0);
  for (uint64_t r = 0; r < n_rows; ++r)
    for (uint32_t j = 0; j < width; ++j) sums[j] += projected[r * width + j];
  const std::vector<GenePart> parts = gene_parts(gene_map, stream_genes, n_genes);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t pi = 0; pi < (int64_t)parts.size(); ++pi) {
    const GenePart& part = parts[pi];
    for (uint64_t r = 0; r < n_rows; ++r) {
      const double* w = &projected[r * width];
      uint64_t lo, hi;
      part_run(indptr, indices, r, part, lo, hi);
      for (uint64_t i = lo; i < hi; ++i) {
        uint32_t p = position_of(gene_map, indices[i]);
        if (p == 0xFFFFFFFFu) continue;
        axpy(&product[(size_t)p * width], w, (double)values[i], width);
      }
    }
  }
}

// Last pass (pca.rs:649-677): rows (x - mu) V, centred squares and stored counts.
__attribute__((target_clones("avx512f", "default")))
void ko_pca_rows(const uint64_t* indptr, const uint32_t* indices, const float* values,
                 uint64_t n_rows, const uint32_t* gene_map, uint32_t stream_genes,
                 uint32_t n_genes, const double* loadings, const double* mean_projection,
                 uint32_t k, const double* means, double* rows, double* squares,
                 uint64_t* stored) {
  ko_pca_project(indptr, indices, values, n_rows, gene_map, loadings, mean_projection, k,
                 rows);
  std::fill(squares, squares + n_genes, 0.0);
  std::fill(stored, stored + n_genes, 0);
  const std::vector<GenePart> parts = gene_parts(gene_map, stream_genes, n_genes);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t pi = 0; pi < (int64_t)parts.size(); ++pi) {
    const GenePart& part = parts[pi];
    for (uint64_t r = 0; r < n_rows; ++r) {
      uint64_t lo, hi;
      part_run(indptr, indices, r, part, lo, hi);
      for (uint64_t i = lo; i < hi; ++i) {
        uint32_t p = position_of(gene_map, indices[i]);
        if (p == 0xFFFFFFFFu) continue;
        double c = (double)values[i] - means[p];
        squares[p] += c * c;
        stored[p] += 1;
      }
    }
  }
}

// ---------------------------------------------------------------------------------
// Exact kNN.
// ---------------------------------------------------------------------------------

// crates/kyto-exec/src/neighbors.rs:484-536 (brute_force): every row's k nearest other
// rows by (f64 key, row), ranked; self excluded by position.
void ko_knn_brute(const float* points, uint64_t n, uint32_t width, uint32_t k,
                  double* keys_out, uint32_t* rows_out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t q = 0; q < (int64_t)n; ++q) {
    Nearest found(k);
    const float* qp = &points[(uint64_t)q * width];
    for (uint64_t p = 0; p < n; ++p) {
      if (p == (uint64_t)q) continue;
      found.offer(squared_distance(qp, &points[p * width], width), (uint32_t)p);
    }
    for (uint32_t i = 0; i < k; ++i) {
      keys_out[(uint64_t)q * k + i] = found.entries[i].first;
      rows_out[(uint64_t)q * k + i] = found.entries[i].second;
    }
  }
}

// The f64 key of row q against row p (Space::keys, neighbors.rs:389-401).
double ko_key(const float* points, uint32_t width, uint64_t q, uint64_t p) {
  return squared_distance(&points[q * width], &points[p * width], width);
}

// crates/kyto-exec/src/neighbors_exact.rs:50-356: the CPU's filtered exact search (an
// f32 matrix-product filter with a proven slack, candidates re-ranked by f64 keys, rows
// that break an assumption searched against every row). Same result as ko_knn_brute.
//
// Split as kyto's is: `Prepared::new` (neighbors_exact.rs:98-160: the mean, centred f32
// rows, offsets and slacks, built once and in parallel here) and the per-block search
// (`search_block`, :162-356), so a timed sample of queries pays the setup once. The
// block products (kyto: `f32_products`, kernels/products.rs:21-112, a BLAS sgemm) are an
// AVX2 FMA register-blocked kernel over 128-query x 1,024-point tiles: the filter's keys
// are approximate by design (the slack covers any summation order and contraction), so
// only the exact f64 re-rank has to carry kyto's bits.

struct KnnPrepared {
  const float* points = nullptr;  // caller-owned, read by the exact keys
  uint64_t n = 0;
  uint32_t width = 0;
  bool brute = false;             // a row norm too large for f32 keys (neighbors_exact.rs:119)
  std::vector<float> rows;        // centred rows, n x width
  std::vector<float> offsets;     // fl32(|a~|^2)
  std::vector<double> slack;      // E_q
  uint64_t n_tiles = 0;
  uint32_t kpad = 0;              // width rounded up to 8
  // Point tiles of kPointRows rows as panels of 16 points: [tile][panel][j][16].
  std::vector<float> tiles;
};

constexpr uint64_t kQueryRows = 128, kPointRows = 1024, kCandidateLimit = 4096;
constexpr uint32_t kPanel = 16;

// keys[r][c] = (off_q[r] + off_p[c]) - 2 (q_r . p_c) for a block's query rows and a
// tile's columns, from the panel layout: R query rows x 16 columns per register block
// (AVX2: 6 x 2 ymm accumulators; AVX-512: 12 x 1 zmm, chosen at run time).
extern "C++" {
template <int R>
__attribute__((target("avx2,fma"))) static void tile_keys_avx2(const KnnPrepared& P,
                                                               const float* q, uint32_t rows,
                                                               const float* offq, uint64_t t,
                                                               float* keys) {
  const uint32_t w = P.width;
  const float* tile = &P.tiles[t * kPointRows * w];
  const float* offp = &P.offsets[t * kPointRows];
  const uint64_t cols = std::min<uint64_t>(kPointRows, P.n - t * kPointRows);
  const __m256 two = _mm256_set1_ps(2.0f);
  for (uint32_t r0 = 0; r0 < rows; r0 += R) {
    const float* qr[R];
    for (int r = 0; r < R; ++r) qr[r] = q + (uint64_t)std::min(r0 + r, rows - 1) * w;
    for (uint64_t c = 0; c < cols; c += kPanel) {
      const float* panel = tile + c * w;  // w x 16
      __m256 a[R][2];
      for (int r = 0; r < R; ++r) a[r][0] = a[r][1] = _mm256_setzero_ps();
      for (uint32_t j = 0; j < w; ++j) {
        const __m256 b0 = _mm256_loadu_ps(panel + j * kPanel);
        const __m256 b1 = _mm256_loadu_ps(panel + j * kPanel + 8);
        for (int r = 0; r < R; ++r) {
          const __m256 x = _mm256_broadcast_ss(qr[r] + j);
          a[r][0] = _mm256_fmadd_ps(x, b0, a[r][0]);
          a[r][1] = _mm256_fmadd_ps(x, b1, a[r][1]);
        }
      }
      const __m256 p0 = _mm256_loadu_ps(offp + c), p1 = _mm256_loadu_ps(offp + c + 8);
      for (int r = 0; r < R && r0 + r < rows; ++r) {
        const __m256 o = _mm256_set1_ps(offq[r0 + r]);
        float* kr = keys + (uint64_t)(r0 + r) * kPointRows + c;
        _mm256_storeu_ps(kr, _mm256_sub_ps(_mm256_add_ps(o, p0), _mm256_mul_ps(two, a[r][0])));
        _mm256_storeu_ps(kr + 8, _mm256_sub_ps(_mm256_add_ps(o, p1), _mm256_mul_ps(two, a[r][1])));
      }
    }
  }
}

template <int R>
__attribute__((target("avx512f"))) static void tile_keys_avx512(const KnnPrepared& P,
                                                                 const float* q, uint32_t rows,
                                                                 const float* offq, uint64_t t,
                                                                 float* keys) {
  const uint32_t w = P.width;
  const float* tile = &P.tiles[t * kPointRows * w];
  const float* offp = &P.offsets[t * kPointRows];
  const uint64_t cols = std::min<uint64_t>(kPointRows, P.n - t * kPointRows);
  const __m512 two = _mm512_set1_ps(2.0f);
  for (uint32_t r0 = 0; r0 < rows; r0 += R) {
    const float* qr[R];
    for (int r = 0; r < R; ++r) qr[r] = q + (uint64_t)std::min(r0 + r, rows - 1) * w;
    for (uint64_t c = 0; c < cols; c += 2 * kPanel) {
      const float* pa = tile + c * w;
      const float* pb = tile + (c + kPanel) * w;
      __m512 a[R][2];
      for (int r = 0; r < R; ++r) a[r][0] = a[r][1] = _mm512_setzero_ps();
      for (uint32_t j = 0; j < w; ++j) {
        const __m512 b0 = _mm512_loadu_ps(pa + j * kPanel);
        const __m512 b1 = _mm512_loadu_ps(pb + j * kPanel);
        for (int r = 0; r < R; ++r) {
          const __m512 x = _mm512_set1_ps(qr[r][j]);
          a[r][0] = _mm512_fmadd_ps(x, b0, a[r][0]);
          a[r][1] = _mm512_fmadd_ps(x, b1, a[r][1]);
        }
      }
      const __m512 p0 = _mm512_loadu_ps(offp + c), p1 = _mm512_loadu_ps(offp + c + kPanel);
      for (int r = 0; r < R && r0 + r < rows; ++r) {
        const __m512 o = _mm512_set1_ps(offq[r0 + r]);
        float* kr = keys + (uint64_t)(r0 + r) * kPointRows + c;
        _mm512_storeu_ps(kr, _mm512_sub_ps(_mm512_add_ps(o, p0), _mm512_mul_ps(two, a[r][0])));
        _mm512_storeu_ps(kr + kPanel,
                         _mm512_sub_ps(_mm512_add_ps(o, p1), _mm512_mul_ps(two, a[r][1])));
      }
    }
  }
}

static void tile_keys(const KnnPrepared& P, const float* q, uint32_t rows, const float* offq,
                      uint64_t t, float* keys) {
  static const bool avx512 = __builtin_cpu_supports("avx512f");
  if (avx512)
    tile_keys_avx512<12>(P, q, rows, offq, t, keys);
  else
    tile_keys_avx2<6>(P, q, rows, offq, t, keys);
}
}  // extern "C++"

// The first index in [c, cols) whose key is <= th (cols if none), 8 keys at a time.
__attribute__((target("avx2"))) static uint64_t next_at_most(const float* kr, uint64_t c,
                                                            uint64_t cols, float th) {
  const __m256 t = _mm256_set1_ps(th);
  for (; c + 8 <= cols; c += 8) {
    const int m = _mm256_movemask_ps(_mm256_cmp_ps(_mm256_loadu_ps(kr + c), t, _CMP_LE_OQ));
    if (m) return c + (uint64_t)__builtin_ctz((unsigned)m);
  }
  for (; c < cols; ++c)
    if (kr[c] <= th) return c;
  return cols;
}

void* ko_knn_prepare(const float* points, uint64_t n, uint32_t width) {
  auto* P = new KnnPrepared();
  P->points = points;
  P->n = n;
  P->width = width;
  const double u = 1.0 / 16777216.0;
  const double factor = 2.0 * ((double)width + 8.0) * u;
  const double underflow =
      4.0 * ((double)width + 8.0) * (double)std::numeric_limits<float>::min();
  // The mean in row order (neighbors_exact.rs:110-118): n x width adds, kept sequential
  // so the centred rows carry kyto's bits.
  std::vector<double> mean(width, 0.0);
  for (uint64_t r = 0; r < n; ++r)
    for (uint32_t j = 0; j < width; ++j) mean[j] += (double)points[r * width + j];
  for (uint32_t j = 0; j < width; ++j) mean[j] /= (double)n;
  P->rows.resize((size_t)n * width);
  std::vector<double> squares(n);
  double largest = 0.0;
#pragma omp parallel for schedule(static) reduction(max : largest)
  for (int64_t r = 0; r < (int64_t)n; ++r) {
    double s = 0.0;
    for (uint32_t j = 0; j < width; ++j) {
      float c = (float)((double)points[r * width + j] - mean[j]);
      P->rows[r * width + j] = c;
      s += (double)c * (double)c;
    }
    squares[r] = s;
    largest = std::max(largest, s);
  }
  largest = std::sqrt(largest);
  if (!std::isfinite(largest) || largest > 1e15) {
    P->brute = true;
    P->rows.clear();
    return P;
  }
  P->slack.resize(n);
  P->offsets.assign((n + kPointRows - 1) / kPointRows * kPointRows, 0.0f);
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < (int64_t)n; ++r) {
    double a = std::sqrt(squares[r]) + largest;
    P->slack[r] = factor * a * a + underflow;
    P->offsets[r] = (float)squares[r];
  }
  P->n_tiles = (n + kPointRows - 1) / kPointRows;
  P->tiles.assign((size_t)P->n_tiles * kPointRows * width, 0.0f);
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)n; ++p) {
    uint64_t t = p / kPointRows, c = p % kPointRows;
    float* panel = &P->tiles[(t * kPointRows + c / kPanel * kPanel) * width];
    for (uint32_t j = 0; j < width; ++j) panel[j * kPanel + c % kPanel] = P->rows[p * width + j];
  }
  return P;
}

void ko_knn_free(void* handle) { delete static_cast<KnnPrepared*>(handle); }

// The queries query_rows[0..count) (NULL: rows query_begin, query_begin + 1, ...) of a
// prepared search; output i is query i's k entries. Returns the rows that fell back to a
// full search. Blocks of kQueryRows consecutive queries share the tile products, as in
// kyto's search_block.
static uint64_t knn_search_impl(const KnnPrepared& P, uint32_t k, const uint64_t* query_rows,
                                uint64_t query_begin, uint64_t count, double* keys_out,
                                uint32_t* rows_out) {
  const uint64_t n = P.n;
  const uint32_t width = P.width;
  const float* points = P.points;
  if (P.brute) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < (int64_t)count; ++i) {
      const uint64_t q = query_rows ? query_rows[i] : query_begin + (uint64_t)i;
      Nearest found(k);
      for (uint64_t p = 0; p < n; ++p)
        if (p != q) found.offer(ko_key(points, width, q, p), (uint32_t)p);
      for (uint32_t j = 0; j < k; ++j) {
        keys_out[(uint64_t)i * k + j] = found.entries[j].first;
        rows_out[(uint64_t)i * k + j] = found.entries[j].second;
      }
    }
    return count;
  }
  uint64_t fallbacks = 0;
  uint64_t n_blocks = (count + kQueryRows - 1) / kQueryRows;
#pragma omp parallel reduction(+ : fallbacks)
  {
    std::vector<float> keys(kQueryRows * kPointRows);
    std::vector<float> qrows(kQueryRows * width), qoff(kQueryRows);
    std::vector<uint64_t> qid(kQueryRows);
    struct Query {
      std::vector<float> smallest;
      float threshold = std::numeric_limits<float>::infinity();
      std::vector<std::pair<float, uint32_t>> candidates;
      size_t compact_at = 64;
      bool overflowed = false;
    };
    std::vector<Query> states(kQueryRows);
#pragma omp for schedule(dynamic, 1)
    for (int64_t b = 0; b < (int64_t)n_blocks; ++b) {
      const uint64_t i0 = (uint64_t)b * kQueryRows;
      const uint32_t nq = (uint32_t)std::min<uint64_t>(kQueryRows, count - i0);
      for (uint64_t qi = 0; qi < nq; ++qi) {
        states[qi] = Query();
        states[qi].smallest.reserve(k + 1);
        qid[qi] = query_rows ? query_rows[i0 + qi] : query_begin + i0 + qi;
        std::memcpy(&qrows[qi * width], &P.rows[qid[qi] * width], width * sizeof(float));
        qoff[qi] = P.offsets[qid[qi]];
      }
      for (uint64_t t = 0; t < P.n_tiles; ++t) {
        uint64_t p0 = t * kPointRows, p1 = std::min(n, p0 + kPointRows);
        uint64_t cols = p1 - p0;
        tile_keys(P, qrows.data(), nq, qoff.data(), t, keys.data());
        for (uint64_t qi = 0; qi < nq; ++qi) {
          const float* kr = &keys[qi * kPointRows];
          Query& st = states[qi];
          if (st.overflowed) continue;
          uint64_t query = qid[qi];
          for (uint64_t c = next_at_most(kr, 0, cols, st.threshold); c < cols;
               c = next_at_most(kr, c + 1, cols, st.threshold)) {
            float key = kr[c];
            if (p0 + c == query) continue;
            // neighbors_exact.rs:216-255 (Query::offer).
            if (st.smallest.size() < k || key < st.smallest[k - 1]) {
              if (st.smallest.size() < k) st.smallest.push_back(key);
              size_t at = st.smallest.size() - 1;
              while (at > 0 && st.smallest[at - 1] > key) {
                st.smallest[at] = st.smallest[at - 1];
                --at;
              }
              st.smallest[at] = key;
              if (st.smallest.size() == k) {
                double v = (double)st.smallest[k - 1] + 2.0 * P.slack[query];
                float rounded = (float)v;
                if ((double)rounded < v) rounded = std::nextafter(rounded, INFINITY);
                st.threshold = rounded;
              }
            }
            if (key <= st.threshold) {
              st.candidates.push_back({key, (uint32_t)(p0 + c)});
              if (st.candidates.size() >= st.compact_at) {
                float th = st.threshold;
                size_t w = 0;
                for (auto& e : st.candidates)
                  if (e.first <= th) st.candidates[w++] = e;
                st.candidates.resize(w);
                if (w > kCandidateLimit) {
                  st.overflowed = true;
                  st.candidates.clear();
                  break;
                } else {
                  st.compact_at = std::max<size_t>(2 * w, 64);
                }
              }
            }
          }
        }
      }
      for (uint64_t qi = 0; qi < nq; ++qi) {
        uint64_t query = qid[qi];
        Query& st = states[qi];
        Nearest found(k);
        bool ok = !st.overflowed;
        if (ok) {
          for (auto& e : st.candidates) {
            if (e.first > st.threshold) continue;
            double exact = ko_key(points, width, query, e.second);
            if (std::fabs(exact - (double)e.first) > P.slack[query]) {
              ok = false;
              break;
            }
            found.offer(exact, e.second);
          }
          ok = ok && found.entries.size() == k;
        }
        if (!ok) {
          fallbacks += 1;
          found = Nearest(k);
          for (uint64_t p = 0; p < n; ++p)
            if (p != query) found.offer(ko_key(points, width, query, p), (uint32_t)p);
        }
        for (uint32_t i = 0; i < k; ++i) {
          keys_out[(i0 + qi) * k + i] = found.entries[i].first;
          rows_out[(i0 + qi) * k + i] = found.entries[i].second;
        }
      }
    }
  }
  return fallbacks;
}

// Queries [query_begin, query_end) of a prepared search; outputs indexed from
// query_begin. Returns the rows that fell back to a full search.
uint64_t ko_knn_search(const void* handle, uint32_t k, uint64_t query_begin,
                       uint64_t query_end, double* keys_out, uint32_t* rows_out) {
  return knn_search_impl(*static_cast<const KnnPrepared*>(handle), k, nullptr, query_begin,
                         query_end - query_begin, keys_out, rows_out);
}

// The queries rows[0..count) of a prepared search (any rows, in any order).
uint64_t ko_knn_search_rows(const void* handle, uint32_t k, const uint64_t* rows,
                            uint64_t count, double* keys_out, uint32_t* rows_out) {
  return knn_search_impl(*static_cast<const KnnPrepared*>(handle), k, rows, 0, count,
                         keys_out, rows_out);
}

uint64_t ko_knn_exact_range(const float* points, uint64_t n, uint32_t width, uint32_t k,
                            uint64_t query_begin, uint64_t query_end, double* keys_out,
                            uint32_t* rows_out) {
  void* h = ko_knn_prepare(points, n, width);
  uint64_t fb = ko_knn_search(h, k, query_begin, query_end, keys_out, rows_out);
  ko_knn_free(h);
  return fb;
}

uint64_t ko_knn_exact(const float* points, uint64_t n, uint32_t width, uint32_t k,
                      double* keys_out, uint32_t* rows_out) {
  return ko_knn_exact_range(points, n, width, k, 0, n, keys_out, rows_out);
}

int ko_max_threads(void) { return omp_get_max_threads(); }
void ko_set_threads(int n) { omp_set_num_threads(n); }

}  // extern "C"
