// Learned-partition kNN: a BF16 MLP (kg_mlp.cuh) trained on the exact kNN graph of a
// sample of the rows proposes, for every row, the partitions to search; the search is
// the exact kNN's tensor-core filter and exact re-rank restricted to those partitions'
// points, and every row whose proposal is not confident enough is searched against
// every row. kyto has no learned partitioner: this form is this library's own.
//
//   1. sample: m evenly strided rows; their exact graph (the exact search itself);
//   2. partitions: k-means of the sample into P parts (kg_cluster.cuh);
//   3. training: the network starts as the parts' nearest-centre classifier (or from
//      random weights on request); soft targets = the parts of a row and of its k
//      neighbours, soft-target cross-entropy, Adam, `epochs` passes of seeded shuffles;
//   4. calibration: the softmax temperature whose confidence (the probed parts' summed
//      softmax) best predicts, by cross-entropy over the sample, the share of a row's
//      exact neighbours that live in the parts it probes;
//   5. index: the network's top-`probe` parts for every row (each row stored in its top
//      part) and its 32 most probable parts with their probabilities at that
//      temperature;
//   6. confidence: the rows in part order (a row's top three parts, most probable
//      first, so rows sharing their top part sit together and nearby rows nearer still)
//      form provisional blocks of 256 query slots; a row's confidence is its
//      probability in the parts its block probes (the union of its rows' top-`probe`
//      parts), and it falls back below the threshold;
//   7. search: query slots sorted by (fallback, part order); each block of 256 query
//      slots scans the tiles of the parts of the provisional blocks its confident rows
//      came from, then the exact re-rank; fallback rows are searched over every tile
//      with the filter's overflowed queries (the tiles split into ranges between copies
//      of those queries, so they spread over every SM).
#include <cuda_bf16.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "kg_cluster.cuh"
#include "kg_internal.cuh"
#include "kg_knn.cuh"
#include "kg_knn_tc.cuh"
#include "kg_mlp.cuh"

namespace kg {

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void strided_rows_kernel(const float* x, uint64_t n, uint32_t width, uint32_t d,
                                    uint64_t m, float* out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= m * d) return;
  const uint64_t r = i / d, j = i % d;
  const uint64_t row = r * n / m;
  out[r * d + j] = x[row * width + j];
}

// labels[i * L + 0] = part of row i, then the parts of its k neighbours (L = k + 1).
__global__ void target_labels_kernel(const uint32_t* part, const uint32_t* nbr, uint64_t m,
                                     uint32_t k, uint32_t* labels) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const uint32_t L = k + 1;
  labels[i * L] = part[i];
  for (uint32_t j = 0; j < k; ++j) labels[i * L + 1 + j] = part[nbr[i * k + j]];
}

__global__ void shuffle_keys_kernel(uint64_t m, uint64_t seed, uint32_t epoch,
                                    unsigned long long* key, uint32_t* idx) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  key[i] = mix64(seed * 0x9E3779B97F4A7C15ull + ((uint64_t)epoch << 40) + i);
  idx[i] = (uint32_t)i;
}

// The batch: rows order[b0 + r] of the sample and their labels.
__global__ void gather_batch_kernel(const float* xs, uint32_t d, const uint32_t* labels,
                                    uint32_t L, const uint32_t* order, uint64_t b0, uint32_t rows,
                                    float* xb, uint32_t* lb) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t w = d > L ? d : L;
  if (i >= (uint64_t)rows * w) return;
  const uint64_t r = i / w, j = i % w;
  const uint64_t src = order[b0 + r];
  if (j < d) xb[r * d + j] = xs[src * d + j];
  if (j < L) lb[r * L + j] = labels[src * L + j];
}

// A row's order key: its `levels` most probable parts, most probable first, pb bits
// each. Rows sharing their first part are one contiguous run, and inside it rows sharing
// their second (third) part sit together: nearby rows in nearby slots.
__device__ __forceinline__ unsigned long long part_key(const uint32_t* top, uint64_t r,
                                                       uint32_t probe, uint32_t levels,
                                                       uint32_t pb) {
  unsigned long long key = 0;
  for (uint32_t l = 0; l < levels; ++l) key = (key << pb) | top[r * probe + l];
  return key;
}

// key = (fallback, part key) for the query order (a fallback row: the part `parts`,
// lower levels 0); iota payload.
__global__ void query_key_kernel(const uint32_t* top, const float* conf, uint64_t n,
                                 uint32_t probe, uint32_t levels, uint32_t pb, float threshold,
                                 uint32_t parts, unsigned long long* key, uint32_t* iota,
                                 uint8_t* fallback) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  const bool fb = !(conf[r] >= threshold);
  fallback[r] = fb ? 1 : 0;
  key[r] = fb ? (unsigned long long)parts << (pb * (levels - 1))
              : part_key(top, r, probe, levels, pb);
  iota[r] = (uint32_t)r;
}

__global__ void point_key_kernel(const uint32_t* top, uint64_t n, uint32_t probe, uint32_t levels,
                                 uint32_t pb, unsigned long long* key, uint32_t* iota) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  key[r] = part_key(top, r, probe, levels, pb);
  iota[r] = (uint32_t)r;
}

__global__ void inverse_kernel(const uint32_t* perm, uint64_t n, uint32_t* inv) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) inv[perm[i]] = (uint32_t)i;
}

__global__ void full_slots_kernel(const uint32_t* qrows, const uint8_t* fallback, uint64_t n,
                                  uint8_t* q_full) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) q_full[i] = fallback[qrows[i]];
}

__global__ void compose_kernel(const uint32_t* qrows, const uint32_t* slot_of_row, uint64_t n,
                               uint32_t* q_point) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) q_point[i] = slot_of_row[qrows[i]];
}

// starts[c] = the first slot whose key's top part (key >> shift) is at least c.
__global__ void part_starts_kernel(const unsigned long long* sorted, uint64_t n, uint32_t parts,
                                   uint32_t shift, uint32_t* starts) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > parts) return;
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if ((sorted[mid] >> shift) < c) lo = mid + 1; else hi = mid;
  }
  starts[c] = (uint32_t)lo;
}

constexpr uint32_t kProbeThreads = 256;
constexpr uint32_t kMassParts = 32;  // parts per row whose probabilities the index keeps

// One CTA per block of query slots: the tiles of the union of the probed parts of its
// queries that do not fall back (a bitmap over tiles; a fallback row is searched over
// every tile apart from the blocks). Count pass (list NULL): the number of tiles into
// len[B]; fill pass: the tiles in increasing order at list + off[B].
__global__ void __launch_bounds__(kProbeThreads)
probe_tiles_kernel(const uint32_t* qrows, uint64_t n, const uint32_t* prov_of_row,
                   const uint32_t* prov_parts, uint32_t pwords, const uint8_t* fallback,
                   const uint32_t* part_start, uint32_t n_tiles, uint32_t block, uint64_t* len,
                   const uint64_t* off, uint32_t* list) {
  // Dynamic shared memory: n_tiles bits of tiles, then pwords words of parts.
  extern __shared__ uint32_t bits[];
  uint32_t* parts_bm = bits + (n_tiles + 31) / 32;
  __shared__ uint32_t word_base[kProbeThreads + 1];
  __shared__ uint32_t prov[kProbeThreads];
  const uint32_t words = (n_tiles + 31) / 32;
  for (uint32_t w = threadIdx.x; w < words; w += kProbeThreads) bits[w] = 0;
  for (uint32_t w = threadIdx.x; w < pwords; w += kProbeThreads) parts_bm[w] = 0;
  __syncthreads();
  // The parts of every provisional block a row of this block came from (a run of rows
  // from the same one contributes its bitmap once).
  const uint64_t q0 = blockIdx.x * (uint64_t)block;
  for (uint32_t i0 = 0; i0 < block; i0 += kProbeThreads) {
    const uint64_t q = q0 + i0 + threadIdx.x;
    uint32_t b = 0xFFFFFFFFu;
    if (i0 + threadIdx.x < block && q < n) {
      const uint32_t row = qrows[q];
      if (!fallback[row]) b = prov_of_row[row];
    }
    prov[threadIdx.x] = b;
    __syncthreads();
    if (b != 0xFFFFFFFFu && (threadIdx.x == 0 || prov[threadIdx.x - 1] != b))
      for (uint32_t w = 0; w < pwords; ++w) {
        const uint32_t v = prov_parts[(uint64_t)b * pwords + w];
        if (v) atomicOr(&parts_bm[w], v);
      }
    __syncthreads();
  }
  // The tiles of those parts.
  for (uint32_t pw = 0; pw < pwords; ++pw) {
    uint32_t v = parts_bm[pw];
    while (v) {
      const uint32_t part = pw * 32 + (uint32_t)(__ffs(v) - 1);
      v &= v - 1;
      const uint32_t a = part_start[part], e = part_start[part + 1];
      if (a == e) continue;
      for (uint32_t tile = (a >> 7) + threadIdx.x; tile <= (e - 1) >> 7; tile += kProbeThreads)
        atomicOr(&bits[tile >> 5], 1u << (tile & 31));
    }
  }
  __syncthreads();
  // Per thread a run of words, their popcounts scanned in thread order.
  const uint32_t per = (words + kProbeThreads - 1) / kProbeThreads;
  const uint32_t w0 = threadIdx.x * per, w1 = min(words, w0 + per);
  uint32_t c = 0;
  for (uint32_t w = w0; w < w1; ++w) c += __popc(bits[w]);
  word_base[threadIdx.x] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (uint32_t t = 0; t < kProbeThreads; ++t) {
      const uint32_t v = word_base[t];
      word_base[t] = acc;
      acc += v;
    }
    word_base[kProbeThreads] = acc;
  }
  __syncthreads();
  if (!list) {
    if (threadIdx.x == 0) len[blockIdx.x] = word_base[kProbeThreads];
    return;
  }
  uint64_t at = off[blockIdx.x] + word_base[threadIdx.x];
  for (uint32_t w = w0; w < w1; ++w) {
    uint32_t b = bits[w];
    while (b) {
      const int j = __ffs(b) - 1;
      b &= b - 1;
      list[at++] = w * 32 + j;
    }
  }
}

void sort_key_pairs(const unsigned long long* key, const uint32_t* val, uint64_t n, int bits,
                    DeviceBuffer<unsigned long long>& key_out, DeviceBuffer<uint32_t>& val_out,
                    cudaStream_t s) {
  key_out.alloc(n, s);
  val_out.alloc(n, s);
  size_t temp = 0;
  KG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, key, key_out.ptr, val, val_out.ptr,
                                          (int)n, 0, bits, s));
  DeviceBuffer<unsigned char> scratch(temp, s);
  KG_CUDA(cub::DeviceRadixSort::SortPairs(scratch.ptr, temp, key, key_out.ptr, val, val_out.ptr,
                                          (int)n, 0, bits, s));
}

// How many of a row's most probable parts order the rows (KYTO_GPU_LEARNED_LEVELS, 1-3;
// default 3).
uint32_t order_levels() {
  const char* e = std::getenv("KYTO_GPU_LEARNED_LEVELS");
  const int v = e ? std::atoi(e) : 3;
  return (uint32_t)std::min(3, std::max(1, v));
}

int bits_for_value(uint64_t v) {
  int b = 1;
  while (b < 32 && (1ull << b) <= v) ++b;
  return b;
}

// The network's top parts for n rows of x (chunks of 65,536 rows) and their confidence
// at each of n_temps temperatures (device array temps): conf[t * n + row].
void learned_probe(const Mlp& mlp, const float* x, uint64_t n, uint32_t width, uint32_t probe,
                   const float* temps, uint32_t n_temps, uint32_t* top, float* conf,
                   cudaStream_t s, uint32_t n_mass = 0, uint16_t* mass_part = nullptr,
                   float* mass_prob = nullptr, Trace* trace = nullptr) {
  const uint64_t chunk = 65536;
  MlpBatch b;
  b.alloc(mlp.sh, (uint32_t)std::min<uint64_t>(chunk, n), s);
  for (uint64_t r0 = 0; r0 < n; r0 += chunk) {
    const uint32_t rows = (uint32_t)std::min<uint64_t>(chunk, n - r0);
    b.rows = rows;
    mlp.forward(x + r0 * width, width, b, s);
    if (trace) trace->mark("index forward");
    top_parts(b.z3.ptr, rows, mlp.sh.parts, probe, top + r0 * probe, conf + r0, n, s, temps,
              n_temps, n_mass, mass_part ? mass_part + r0 * n_mass : nullptr,
              mass_prob ? mass_prob + r0 * n_mass : nullptr);
    if (trace) trace->mark("index top parts");
  }
}

// loss[t] = - sum over i of cov_i log p_ti + (1 - cov_i) log(1 - p_ti), p clamped to
// [1e-6, 1 - 1e-6], in f64: one CTA per temperature, each thread a fixed stride of rows,
// then a fixed tree (the same bits run to run).
__global__ void __launch_bounds__(256)
calibration_loss_kernel(const float* conf, const float* cov, uint64_t m, double* loss) {
  __shared__ double part[256];
  const uint32_t t = blockIdx.x;
  double acc = 0.0;
  for (uint64_t i = threadIdx.x; i < m; i += blockDim.x) {
    const double p = fmin(fmax((double)conf[t * m + i], 1e-6), 1.0 - 1e-6);
    const double c = (double)cov[i];
    acc -= c * log(p) + (1.0 - c) * log1p(-p);
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (uint32_t o = blockDim.x / 2; o; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss[t] = part[0];
}

// covered[i] = the share of sample row i's k graph neighbours that live in a part row i
// probes (a row lives in its top part): what the confidence should predict.
__global__ void covered_kernel(const uint32_t* top, uint32_t probe, const uint32_t* nbr,
                               uint64_t m, uint32_t k, float* covered) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  uint32_t hits = 0;
  for (uint32_t j = 0; j < k; ++j) {
    const uint32_t home = top[(uint64_t)nbr[i * k + j] * probe];
    bool in = false;
    for (uint32_t t = 0; t < probe; ++t) in |= top[i * probe + t] == home;
    hits += in ? 1u : 0u;
  }
  covered[i] = (float)hits / (float)k;
}

// Per provisional block (rows in top-part order, `block` slots a block): the parts its
// rows probe, as a bitmap of pwords words.
__global__ void block_parts_kernel(const uint32_t* rows, uint64_t n, const uint32_t* top,
                                   uint32_t probe, uint32_t block, uint32_t pwords,
                                   uint32_t* bitmap) {
  extern __shared__ uint32_t pb[];
  for (uint32_t w = threadIdx.x; w < pwords; w += blockDim.x) pb[w] = 0;
  __syncthreads();
  const uint64_t q0 = blockIdx.x * (uint64_t)block;
  for (uint32_t i = threadIdx.x; i < block; i += blockDim.x) {
    const uint64_t q = q0 + i;
    if (q >= n) break;
    const uint32_t row = rows[q];
    for (uint32_t t = 0; t < probe; ++t) {
      const uint32_t part = top[(uint64_t)row * probe + t];
      atomicOr(&pb[part >> 5], 1u << (part & 31));
    }
  }
  __syncthreads();
  for (uint32_t w = threadIdx.x; w < pwords; w += blockDim.x)
    bitmap[(uint64_t)blockIdx.x * pwords + w] = pb[w];
}

// Each row's confidence: its probability (over its n_mass most probable parts) in the
// parts its provisional block probes, which its search will probe (it is searched in at
// least those); and the row's provisional block.
__global__ void union_conf_kernel(const uint32_t* rows, uint64_t n, uint32_t block,
                                  const uint32_t* bitmap, uint32_t pwords,
                                  const uint16_t* mass_part, const float* mass_prob,
                                  uint32_t n_mass, uint32_t* prov_of_row, float* conf) {
  const uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const uint32_t row = rows[q];
  const uint64_t b = q / block;
  prov_of_row[row] = (uint32_t)b;
  const uint32_t* bm = bitmap + b * pwords;
  float c = 0.0f;
  for (uint32_t j = 0; j < n_mass; ++j) {
    const uint32_t part = mass_part[(uint64_t)row * n_mass + j];
    if ((bm[part >> 5] >> (part & 31)) & 1u) c += mass_prob[(uint64_t)row * n_mass + j];
  }
  conf[row] = c;
}

// The squared distance of each sample row to its cluster's centre (f64).
__global__ void sq_to_centre_kernel(const float* xs, uint64_t m, uint32_t d, const uint32_t* label,
                                    const double* centre, uint32_t ldc, double* out) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const double* c = centre + (uint64_t)label[i] * ldc;
  double s = 0.0;
  for (uint32_t j = 0; j < d; ++j) {
    const double v = (double)xs[i * d + j] - c[j];
    s += v * v;
  }
  out[i] = s;
}

// The temperatures the calibration tries (1: the network's own softmax).
constexpr float kTemps[] = {1.0f, 1.25f, 1.5f, 2.0f, 2.5f, 3.0f, 4.0f, 5.0f,
                            6.0f, 8.0f, 10.0f, 12.0f, 16.0f};
constexpr uint32_t kNumTemps = sizeof(kTemps) / sizeof(kTemps[0]);

}  // namespace

}  // namespace kg

using namespace kg;

extern "C" {

kg_status kg_learned_layout(uint32_t din, uint32_t hidden, uint32_t parts, uint64_t* offsets,
                            uint64_t* total) {
  return guarded([&] {
    if (!offsets || !total) fail(KG_ERR_INVALID, "kg_learned_layout: NULL argument");
    MlpShape sh;
    sh.din = din;
    sh.hidden = hidden;
    sh.parts = parts;
    sh.layout();
    for (int l = 0; l < 3; ++l) {
      offsets[2 * l] = sh.w_off[l];
      offsets[2 * l + 1] = sh.b_off[l];
    }
    *total = sh.total;
  });
}

kg_status kg_learned_gradients(kg_ctx* ctx, uint32_t din, uint32_t hidden, uint32_t parts,
                               const float* params, const float* x, uint32_t rows,
                               const uint32_t* labels, uint32_t n_labels, float* grads,
                               float* row_loss, float* logits) {
  return guarded([&] {
    if (!ctx || !params || !x || !labels || !grads || !row_loss)
      fail(KG_ERR_INVALID, "kg_learned_gradients: NULL argument");
    if (!din || !hidden || !parts || !rows || !n_labels)
      fail(KG_ERR_INVALID, "kg_learned_gradients: a zero size");
    use_device(ctx);
    cudaStream_t s = ctx->stream;
    Mlp mlp;
    mlp.init(din, hidden, parts, 0, s);
    mlp.set_params(params, s);
    DeviceBuffer<float> hx;
    const float* dx = device_view(x, (uint64_t)rows * din, hx, s);
    DeviceBuffer<uint32_t> hl;
    const uint32_t* dl = device_view(labels, (uint64_t)rows * n_labels, hl, s);
    MlpBatch b;
    b.alloc(mlp.sh, rows, s);
    mlp.forward(dx, din, b, s);
    mlp.backward(dl, n_labels, b, s);
    mlp.check(s);
    KG_CUDA(cudaMemcpyAsync(grads, mlp.grads.ptr, mlp.sh.total * 4, cudaMemcpyDefault, s));
    KG_CUDA(cudaMemcpyAsync(row_loss, b.row_loss.ptr, (uint64_t)rows * 4, cudaMemcpyDefault, s));
    if (logits)
      KG_CUDA(cudaMemcpyAsync(logits, b.z3.ptr, (uint64_t)rows * parts * 4, cudaMemcpyDefault, s));
    wait_stream(ctx, s);
  });
}

kg_status kg_knn_learned(kg_ctx* ctx, const float* embedding, uint64_t n, uint32_t width,
                         uint32_t n_components, uint32_t n_neighbors,
                         const kg_learned_params* params, uint64_t* indptr, uint32_t* indices,
                         float* distances, kg_learned_stats* stats) {
  return guarded([&] {
    if (!ctx || !embedding || !params || !indptr || !indices || !distances)
      fail(KG_ERR_INVALID, "kg_knn_learned: NULL argument");
    uint32_t k = 0, d = 0;
    check_search_args(n, width, n_components, n_neighbors, k, d);
    const kg_learned_params P = *params;
    if (P.n_parts < 2 || P.n_parts > 65536)
      fail(KG_ERR_INVALID, "kg_knn_learned: n_parts in 2..65536");
    if (P.n_probe < 1 || P.n_probe > P.n_parts || P.n_probe > 64)
      fail(KG_ERR_INVALID, "kg_knn_learned: n_probe in 1..min(64, n_parts)");
    if (P.hidden < 1 || P.batch < 1 || !(P.learning_rate > 0.0f))
      fail(KG_ERR_INVALID, "kg_knn_learned: hidden, batch and learning_rate must be positive");
    if (d + 3 > 64) fail(KG_ERR_INVALID, "kg_knn_learned: more than 61 components");
    use_device(ctx);
    cudaStream_t s = ctx->stream;
    ctx->total = n;
    ctx->done = 0;
    DeviceBuffer<float> hold;
    const float* x = device_view(embedding, n * width, hold, s);
    check_finite(x, n, width, d, s);
    Trace trace(s, "knn_learned");
    auto now = [] { return std::chrono::steady_clock::now(); };
    auto ms_since = [&](std::chrono::steady_clock::time_point t) {
      return std::chrono::duration<double, std::milli>(now() - t).count();
    };
    const uint32_t parts = P.n_parts, probe = P.n_probe, L = k + 1;

    // 1-3. The sample, its exact graph, its parts, the network.
    auto t_train = now();
    const uint64_t m = std::max<uint64_t>(std::min<uint64_t>(P.train_cells ? P.train_cells : n, n),
                                          std::min<uint64_t>(n, (uint64_t)n_neighbors + 1));
    DeviceBuffer<float> xs(m * d, s);
    strided_rows_kernel<<<blocks_for(m * d, 256), 256, 0, s>>>(x, n, width, d, m, xs.ptr);
    KG_LAUNCH_CHECK();
    KnnResult sg;
    knn_core(ctx, xs.ptr, m, d, d, k, nullptr, sg, trace);
    trace.mark("sample graph");
    Clusters cl;
    cluster_rows(xs.ptr, m, d, d, std::min<uint32_t>(parts, (uint32_t)m), 10, m, cl, s);
    DeviceBuffer<uint32_t> labels(m * L, s);
    target_labels_kernel<<<blocks_for(m, 256), 256, 0, s>>>(cl.label.ptr, sg.row.ptr, m, k,
                                                            labels.ptr);
    KG_LAUNCH_CHECK();
    trace.mark("sample parts");
    Mlp mlp;
    mlp.init(d, P.hidden, parts, P.seed, s);
    if (!(P.flags & KG_LEARNED_RANDOM_INIT) && P.hidden >= 2 * d) {
      // Start from the parts' own nearest-centre classifier, at the scale 1 / (mean
      // squared distance of a sample row to its centre), and let training move it
      // toward where the rows' neighbours live.
      DeviceBuffer<double> sq(m, s);
      sq_to_centre_kernel<<<blocks_for(m, 256), 256, 0, s>>>(xs.ptr, m, d, cl.label.ptr,
                                                             cl.centre.ptr, kClusterDim, sq.ptr);
      KG_LAUNCH_CHECK();
      std::vector<double> hsq(m);
      KG_CUDA(cudaMemcpyAsync(hsq.data(), sq.ptr, m * 8, cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaStreamSynchronize(s));
      double mean_sq = 0.0;
      for (double v : hsq) mean_sq += v;
      mean_sq /= (double)m;
      const float beta = mean_sq > 0.0 ? (float)(1.0 / mean_sq) : 1.0f;
      mlp.init_from_centres(cl.centre.ptr, cl.K, kClusterDim, beta, s);
    }
    const uint32_t batch = (uint32_t)std::min<uint64_t>(P.batch, m);
    MlpBatch b;
    b.alloc(mlp.sh, batch, s);
    DeviceBuffer<float> xb((uint64_t)batch * d, s);
    DeviceBuffer<uint32_t> lb((uint64_t)batch * L, s);
    DeviceBuffer<unsigned long long> skey(m, s), skey_sorted(m, s);
    DeviceBuffer<uint32_t> sidx(m, s), order(m, s);
    size_t temp = 0;
    KG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, skey.ptr, skey_sorted.ptr, sidx.ptr,
                                            order.ptr, (int)m, 0, 64, s));
    DeviceBuffer<unsigned char> scratch(temp, s);
    for (uint32_t e = 0; e < P.epochs; ++e) {
      check_cancel(ctx);
      shuffle_keys_kernel<<<blocks_for(m, 256), 256, 0, s>>>(m, P.seed, e, skey.ptr, sidx.ptr);
      KG_LAUNCH_CHECK();
      KG_CUDA(cub::DeviceRadixSort::SortPairs(scratch.ptr, temp, skey.ptr, skey_sorted.ptr,
                                              sidx.ptr, order.ptr, (int)m, 0, 64, s));
      for (uint64_t b0 = 0; b0 + batch <= m; b0 += batch) {
        const uint64_t w = std::max(d, L);
        gather_batch_kernel<<<blocks_for((uint64_t)batch * w, 256), 256, 0, s>>>(
            xs.ptr, d, labels.ptr, L, order.ptr, b0, batch, xb.ptr, lb.ptr);
        KG_LAUNCH_CHECK();
        mlp.forward(xb.ptr, d, b, s);
        mlp.backward(lb.ptr, L, b, s);
        mlp.adam(P.learning_rate, s);
      }
    }
    float final_loss = NAN;
    if (P.epochs) {
      std::vector<float> rl(batch);
      KG_CUDA(cudaMemcpyAsync(rl.data(), b.row_loss.ptr, batch * 4ull, cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaStreamSynchronize(s));
      double acc = 0.0;
      for (float v : rl) acc += v;
      final_loss = (float)(acc / batch);
    }
    KG_CUDA(cudaStreamSynchronize(s));
    mlp.check(s);
    const double train_ms = ms_since(t_train);
    trace.mark("training");

    // 4. Calibration: the temperature whose confidence best predicts (cross-entropy) the
    // share of a sample row's exact neighbours that live in the parts it probes.
    float temperature = 1.0f;
    DeviceBuffer<float> d_temps(kNumTemps, s);
    KG_CUDA(cudaMemcpyAsync(d_temps.ptr, kTemps, sizeof(kTemps), cudaMemcpyHostToDevice, s));
    {
      DeviceBuffer<uint32_t> stop(m * probe, s);
      DeviceBuffer<float> sconf(kNumTemps * m, s);
      learned_probe(mlp, xs.ptr, m, d, probe, d_temps.ptr, kNumTemps, stop.ptr, sconf.ptr, s);
      DeviceBuffer<float> cov(m, s);
      covered_kernel<<<blocks_for(m, 256), 256, 0, s>>>(stop.ptr, probe, sg.row.ptr, m, k,
                                                        cov.ptr);
      KG_LAUNCH_CHECK();
      DeviceBuffer<double> dloss(kNumTemps, s);
      calibration_loss_kernel<<<kNumTemps, 256, 0, s>>>(sconf.ptr, cov.ptr, m, dloss.ptr);
      KG_LAUNCH_CHECK();
      double hloss[kNumTemps];
      KG_CUDA(cudaMemcpyAsync(hloss, dloss.ptr, sizeof hloss, cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaStreamSynchronize(s));
      double best = INFINITY;
      for (uint32_t t = 0; t < kNumTemps; ++t) {
        if (hloss[t] < best) {
          best = hloss[t];
          temperature = kTemps[t];
        }
      }
    }
    trace.mark("calibration");

    // 5. Every row's parts.
    auto t_index = now();
    DeviceBuffer<uint32_t> top(n * probe, s);
    DeviceBuffer<float> conf(n, s);
    // Each row's most probable parts with their probabilities: the mass its search covers.
    const uint32_t n_mass = std::min<uint32_t>(kMassParts, parts);
    DeviceBuffer<uint16_t> mass_part(n * n_mass, s);
    DeviceBuffer<float> mass_prob(n * n_mass, s);
    KG_CUDA(cudaMemcpyAsync(d_temps.ptr, &temperature, 4, cudaMemcpyHostToDevice, s));
    trace.mark("index setup");
    learned_probe(mlp, x, n, width, probe, d_temps.ptr, 1, top.ptr, conf.ptr, s, n_mass,
                  mass_part.ptr, mass_prob.ptr, &trace);
    mlp.check(s);
    KG_CUDA(cudaStreamSynchronize(s));
    const double index_ms = ms_since(t_index);
    trace.mark("index");

    // 5. The restricted exact search.
    auto t_search = now();
    uint64_t fallback_rows = 0, scanned_tiles = 0;
    PlanBuilder plan = [&](const float*, uint64_t nn, uint32_t, uint32_t, double,
                           uint32_t qblock, ScanPlan& sp, Trace& tr) {
      DeviceBuffer<unsigned long long> key(nn, s), key_sorted;
      DeviceBuffer<uint32_t> iota(nn, s);
      DeviceBuffer<uint8_t> fallback(nn, s);
      // Points: by their first `levels` parts.
      const uint32_t pb = (uint32_t)bits_for_value(parts);
      const uint32_t levels = std::min<uint32_t>({order_levels(), probe, 64 / pb});
      const int key_bits = (int)(pb * levels);
      point_key_kernel<<<blocks_for(nn, 256), 256, 0, s>>>(top.ptr, nn, probe, levels, pb,
                                                           key.ptr, iota.ptr);
      KG_LAUNCH_CHECK();
      sort_key_pairs(key.ptr, iota.ptr, nn, key_bits, key_sorted, sp.prows, s);
      DeviceBuffer<uint32_t> part_start((uint64_t)parts + 1, s);
      part_starts_kernel<<<blocks_for((uint64_t)parts + 1, 256), 256, 0, s>>>(
          key_sorted.ptr, nn, parts, pb * (levels - 1), part_start.ptr);
      KG_LAUNCH_CHECK();
      DeviceBuffer<uint32_t> slot_of_row(nn, s);
      inverse_kernel<<<blocks_for(nn, 256), 256, 0, s>>>(sp.prows.ptr, nn, slot_of_row.ptr);
      KG_LAUNCH_CHECK();
      // Confidence: the rows in top-part order form provisional query blocks; a row's
      // confidence is its probability in the parts its provisional block probes, and its
      // final block will probe at least those (the union over its rows' provisional
      // blocks).
      const uint64_t n_prov = (nn + qblock - 1) / qblock;
      const uint32_t pwords = (parts + 31) / 32;
      DeviceBuffer<uint32_t> prov_parts(n_prov * pwords, s), prov_of_row(nn, s);
      DeviceBuffer<float> uconf(nn, s);
      block_parts_kernel<<<(unsigned)n_prov, 256, pwords * 4, s>>>(
          sp.prows.ptr, nn, top.ptr, probe, qblock, pwords, prov_parts.ptr);
      KG_LAUNCH_CHECK();
      union_conf_kernel<<<blocks_for(nn, 256), 256, 0, s>>>(sp.prows.ptr, nn, qblock,
                                                            prov_parts.ptr, pwords, mass_part.ptr,
                                                            mass_prob.ptr, n_mass,
                                                            prov_of_row.ptr, uconf.ptr);
      KG_LAUNCH_CHECK();
      // Queries: by (fallback, top part).
      query_key_kernel<<<blocks_for(nn, 256), 256, 0, s>>>(top.ptr, uconf.ptr, nn, probe, levels,
                                                           pb, P.confidence, parts, key.ptr,
                                                           iota.ptr, fallback.ptr);
      KG_LAUNCH_CHECK();
      sort_key_pairs(key.ptr, iota.ptr, nn, key_bits, key_sorted, sp.qrows, s);
      sp.q_point.alloc(nn, s);
      sp.q_full.alloc(nn, s);
      full_slots_kernel<<<blocks_for(nn, 256), 256, 0, s>>>(sp.qrows.ptr, fallback.ptr, nn,
                                                           sp.q_full.ptr);
      KG_LAUNCH_CHECK();
      compose_kernel<<<blocks_for(nn, 256), 256, 0, s>>>(sp.qrows.ptr, slot_of_row.ptr, nn,
                                                         sp.q_point.ptr);
      KG_LAUNCH_CHECK();
      // The blocks' tile lists (count, scan, fill).
      const uint64_t n_blocks = (nn + qblock - 1) / qblock;
      const uint32_t n_tiles = (uint32_t)((nn + 127) / 128);
      const size_t smem = (size_t)((n_tiles + 31) / 32 + pwords) * 4;
      if (smem > 200 * 1024)
        fail(KG_ERR_INVALID, "kg_knn_learned: too many rows for the tile bitmap");
      static std::once_flag attr;
      std::call_once(attr, [] {
        KG_CUDA(cudaFuncSetAttribute(probe_tiles_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
      });
      DeviceBuffer<uint64_t> len(n_blocks + 1, s);
      len.zero();
      probe_tiles_kernel<<<(unsigned)n_blocks, kProbeThreads, smem, s>>>(
          sp.qrows.ptr, nn, prov_of_row.ptr, prov_parts.ptr, pwords, fallback.ptr,
          part_start.ptr, n_tiles, qblock, len.ptr, nullptr, nullptr);
      KG_LAUNCH_CHECK();
      sp.list_off.alloc(n_blocks + 1, s);
      size_t t2 = 0;
      KG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t2, len.ptr, sp.list_off.ptr, n_blocks + 1, s));
      DeviceBuffer<unsigned char> sc2(t2, s);
      KG_CUDA(cub::DeviceScan::ExclusiveSum(sc2.ptr, t2, len.ptr, sp.list_off.ptr, n_blocks + 1, s));
      uint64_t total = 0;
      KG_CUDA(cudaMemcpyAsync(&total, sp.list_off.ptr + n_blocks, 8, cudaMemcpyDeviceToHost, s));
      std::vector<uint8_t> hf(nn);
      KG_CUDA(cudaMemcpyAsync(hf.data(), fallback.ptr, nn, cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaStreamSynchronize(s));
      fallback_rows = 0;
      for (uint8_t v : hf) fallback_rows += v;
      scanned_tiles = total;
      sp.list_tiles.alloc(std::max<uint64_t>(total, 1), s);
      probe_tiles_kernel<<<(unsigned)n_blocks, kProbeThreads, smem, s>>>(
          sp.qrows.ptr, nn, prov_of_row.ptr, prov_parts.ptr, pwords, fallback.ptr,
          part_start.ptr, n_tiles, qblock, len.ptr, sp.list_off.ptr, sp.list_tiles.ptr);
      KG_LAUNCH_CHECK();
      tr.mark("probe lists");
    };
    KnnResult r;
    knn_core(ctx, x, n, width, d, k, &plan, r, trace);
    write_graph(r, n, k, indptr, indices, distances, s);
    wait_stream(ctx, s);
    const double search_ms = ms_since(t_search);
    trace.mark("graph");
    ctx->done = n;
    if (stats) {
      stats->fallback_rows = fallback_rows;
      stats->scanned_tiles = scanned_tiles;
      stats->candidates = r.candidates;
      stats->rows_full = r.rows_full;
      stats->train_ms = train_ms;
      stats->index_ms = index_ms;
      stats->search_ms = search_ms;
      stats->final_loss = final_loss;
      stats->temperature = temperature;
      stats->tiles_computed = r.tiles_scanned;
    }
  });
}

}  // extern "C"
