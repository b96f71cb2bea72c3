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

// Pass 0 (pca.rs:588-622): n_cells, gene sums, Omega column sums, sketch X^T Omega.
// Genes split over threads (pca.rs GENES_PER_PART): each gene's sums in cell order.
void ko_pca_sketch(const uint64_t* indptr, const uint32_t* indices, const float* values,
                   uint64_t n_rows, const uint32_t* gene_map, uint32_t n_genes,
                   const uint64_t* cells, uint64_t seed, uint32_t width, double* sums,
                   double* omega_sums, double* sketch) {
  std::vector<double> omega((size_t)n_rows * width);
  ko_omega_rows(seed, cells, n_rows, width, omega.data());
  std::fill(sums, sums + n_genes, 0.0);
  std::fill(omega_sums, omega_sums + width, 0.0);
  std::fill(sketch, sketch + (size_t)n_genes * width, 0.0);
  for (uint64_t r = 0; r < n_rows; ++r)
    for (uint32_t j = 0; j < width; ++j) omega_sums[j] += omega[r * width + j];
  int nt = omp_get_max_threads();
#pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    uint32_t g0 = (uint32_t)((uint64_t)n_genes * t / nt);
    uint32_t g1 = (uint32_t)((uint64_t)n_genes * (t + 1) / nt);
    for (uint64_t r = 0; r < n_rows; ++r) {
      const double* om = &omega[r * width];
      for (uint64_t i = indptr[r]; i < indptr[r + 1]; ++i) {
        uint32_t p = position_of(gene_map, indices[i]);
        if (p == 0xFFFFFFFFu || p < g0 || p >= g1) continue;
        double v = (double)values[i];
        sums[p] += v;
        double* target = &sketch[(size_t)p * width];
        for (uint32_t j = 0; j < width; ++j) target[j] += v * om[j];
      }
    }
  }
}

// Each row's projection -offsets + sum value * matrix[gene], its values added in the
// row's gene order (pca.rs:548-586, `project`).
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
      double v = (double)values[i];
      const double* m = &matrix[(size_t)p * width];
      for (uint32_t j = 0; j < width; ++j) row[j] += v * m[j];
    }
  }
}

// Passes 1..q (pca.rs:623-645): w = x Q - mu^T Q per row, sums of w, product X^T W.
void ko_pca_product(const uint64_t* indptr, const uint32_t* indices, const float* values,
                    uint64_t n_rows, const uint32_t* gene_map, uint32_t n_genes,
                    const double* block, const double* block_means, uint32_t width,
                    double* product, double* sums) {
  std::vector<double> projected((size_t)n_rows * width);
  ko_pca_project(indptr, indices, values, n_rows, gene_map, block, block_means, width,
                 projected.data());
  std::fill(sums, sums + width, 0.0);
  std::fill(product, product + (size_t)n_genes * width, 0.0);
  for (uint64_t r = 0; r < n_rows; ++r)
    for (uint32_t j = 0; j < width; ++j) sums[j] += projected[r * width + j];
  int nt = omp_get_max_threads();
#pragma omp parallel num_threads(nt)
  {
    int t = omp_get_thread_num();
    uint32_t g0 = (uint32_t)((uint64_t)n_genes * t / nt);
    uint32_t g1 = (uint32_t)((uint64_t)n_genes * (t + 1) / nt);
    for (uint64_t r = 0; r < n_rows; ++r) {
      const double* w = &projected[r * width];
      for (uint64_t i = indptr[r]; i < indptr[r + 1]; ++i) {
        uint32_t p = position_of(gene_map, indices[i]);
        if (p == 0xFFFFFFFFu || p < g0 || p >= g1) continue;
        double v = (double)values[i];
        double* target = &product[(size_t)p * width];
        for (uint32_t j = 0; j < width; ++j) target[j] += v * w[j];
      }
    }
  }
}

// Last pass (pca.rs:649-677): rows (x - mu) V, centred squares and stored counts.
void ko_pca_rows(const uint64_t* indptr, const uint32_t* indices, const float* values,
                 uint64_t n_rows, const uint32_t* gene_map, uint32_t n_genes,
                 const double* loadings, const double* mean_projection, uint32_t k,
                 const double* means, double* rows, double* squares, uint64_t* stored) {
  ko_pca_project(indptr, indices, values, n_rows, gene_map, loadings, mean_projection, k,
                 rows);
  std::fill(squares, squares + n_genes, 0.0);
  std::fill(stored, stored + n_genes, 0);
  for (uint64_t r = 0; r < n_rows; ++r) {
    for (uint64_t i = indptr[r]; i < indptr[r + 1]; ++i) {
      uint32_t p = position_of(gene_map, indices[i]);
      if (p == 0xFFFFFFFFu) continue;
      double c = (double)values[i] - means[p];
      squares[p] += c * c;
      stored[p] += 1;
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
// Timed as the CPU baseline. Returns the number of rows that fell back to a full search.
uint64_t ko_knn_exact_range(const float* points, uint64_t n, uint32_t width, uint32_t k,
                            uint64_t query_begin, uint64_t query_end, double* keys_out,
                            uint32_t* rows_out);

uint64_t ko_knn_exact(const float* points, uint64_t n, uint32_t width, uint32_t k,
                      double* keys_out, uint32_t* rows_out) {
  return ko_knn_exact_range(points, n, width, k, 0, n, keys_out, rows_out);
}

// Queries [query_begin, query_end) only (a timed sample of the CPU path); outputs are
// indexed from query_begin.
uint64_t ko_knn_exact_range(const float* points, uint64_t n, uint32_t width, uint32_t k,
                            uint64_t query_begin, uint64_t query_end, double* keys_out,
                            uint32_t* rows_out) {
  constexpr uint64_t kQueryRows = 128, kPointRows = 1024, kCandidateLimit = 4096;
  const double u = 1.0 / 16777216.0;
  const double factor = 2.0 * ((double)width + 8.0) * u;
  const double underflow =
      4.0 * ((double)width + 8.0) * (double)std::numeric_limits<float>::min();
  std::vector<double> mean(width, 0.0);
  for (uint64_t r = 0; r < n; ++r)
    for (uint32_t j = 0; j < width; ++j) mean[j] += (double)points[r * width + j];
  for (uint32_t j = 0; j < width; ++j) mean[j] /= (double)n;
  std::vector<float> rows((size_t)n * width);
  std::vector<double> squares(n);
  double largest = 0.0;
  for (uint64_t r = 0; r < n; ++r) {
    double s = 0.0;
    for (uint32_t j = 0; j < width; ++j) {
      float c = (float)((double)points[r * width + j] - mean[j]);
      rows[r * width + j] = c;
      s += (double)c * (double)c;
    }
    squares[r] = s;
    largest = std::max(largest, s);
  }
  largest = std::sqrt(largest);
  if (!std::isfinite(largest) || largest > 1e15) {
    if (query_begin != 0 || query_end != n) return (uint64_t)-1;
    ko_knn_brute(points, n, width, k, keys_out, rows_out);
    return n;
  }
  std::vector<double> slack(n);
  std::vector<float> offsets(n);
  for (uint64_t r = 0; r < n; ++r) {
    double a = std::sqrt(squares[r]) + largest;
    slack[r] = factor * a * a + underflow;
    offsets[r] = (float)squares[r];
  }
  // The point tiles transposed (width x kPointRows), so the product's inner loop runs
  // along points with contiguous loads.
  uint64_t n_tiles = (n + kPointRows - 1) / kPointRows;
  std::vector<float> tiles((size_t)n_tiles * kPointRows * width, 0.0f);
  for (uint64_t p = 0; p < n; ++p) {
    uint64_t t = p / kPointRows, c = p % kPointRows;
    for (uint32_t j = 0; j < width; ++j)
      tiles[(t * width + j) * kPointRows + c] = rows[p * width + j];
  }
  uint64_t fallbacks = 0;
  uint64_t n_queries = query_end - query_begin;
  uint64_t n_blocks = (n_queries + kQueryRows - 1) / kQueryRows;
#pragma omp parallel reduction(+ : fallbacks)
  {
    std::vector<float> keys(kQueryRows * kPointRows);
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
      uint64_t q0 = query_begin + (uint64_t)b * kQueryRows;
      uint64_t q1 = std::min(query_end, q0 + kQueryRows);
      for (uint64_t qi = 0; qi < q1 - q0; ++qi) {
        states[qi] = Query();
        states[qi].smallest.reserve(k + 1);
      }
      for (uint64_t t = 0; t < n_tiles; ++t) {
        uint64_t p0 = t * kPointRows, p1 = std::min(n, p0 + kPointRows);
        uint64_t cols = p1 - p0;
        const float* tile = &tiles[t * width * kPointRows];
        for (uint64_t qi = 0; qi < q1 - q0; ++qi) {
          float* kr = &keys[qi * kPointRows];
          const float* qrow = &rows[(q0 + qi) * width];
          for (uint64_t c = 0; c < kPointRows; ++c) kr[c] = 0.0f;
          for (uint32_t j = 0; j < width; ++j) {
            float a = qrow[j];
            const float* trow = &tile[(uint64_t)j * kPointRows];
            for (uint64_t c = 0; c < kPointRows; ++c) kr[c] += a * trow[c];
          }
          float off = offsets[q0 + qi];
          for (uint64_t c = 0; c < cols; ++c)
            kr[c] = (off + offsets[p0 + c]) - 2.0f * kr[c];
          Query& st = states[qi];
          uint64_t query = q0 + qi;
          for (uint64_t c = 0; c < cols; ++c) {
            float key = kr[c];
            if (!(key <= st.threshold) || p0 + c == query || st.overflowed) continue;
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
                double v = (double)st.smallest[k - 1] + 2.0 * slack[query];
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
                } else {
                  st.compact_at = std::max<size_t>(2 * w, 64);
                }
              }
            }
          }
        }
      }
      for (uint64_t qi = 0; qi < q1 - q0; ++qi) {
        uint64_t query = q0 + qi;
        Query& st = states[qi];
        Nearest found(k);
        bool ok = !st.overflowed;
        if (ok) {
          for (auto& e : st.candidates) {
            if (e.first > st.threshold) continue;
            double exact = ko_key(points, width, query, e.second);
            if (std::fabs(exact - (double)e.first) > slack[query]) {
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
          keys_out[(query - query_begin) * k + i] = found.entries[i].first;
          rows_out[(query - query_begin) * k + i] = found.entries[i].second;
        }
      }
    }
  }
  return fallbacks;
}

int ko_max_threads(void) { return omp_get_max_threads(); }
void ko_set_threads(int n) { omp_set_num_threads(n); }

}  // extern "C"
