// One cell block of kyto's tiled sparse layers (docs/format.md 4.1-4.3) joined into CSR
// rows on the device: kyto-store's decode_cell_block and its checks
// (crates/kyto-store/src/tile_decode.rs:74-196), which kyto runs on the host before
// kyto-exec rebuilds the rows once more for its GPU path (pca/gpu.rs:73-115).
//
// Three kernels, every one a pass over bytes (HBM-bound, no arithmetic to speak of):
//   1. tile_indptr_check_kernel: a thread per value of the block's indptr shard checks
//      kyto's four indptr rules (starts at 0, ends at the tile's nnz, never decreases,
//      flat over padding rows) and marks the tiles that break one;
//   2. tile_rows_kernel: a warp per row walks the row's segment in every tile whose
//      indptr passed (so every entry it reads lies inside that tile), checks that the
//      local indices strictly increase below the block width, and sums the row's length;
//   3. after a scan of the lengths, tile_join_kernel: a warp per row copies its segments
//      in gene-block order, adding each block's first gene to the local indices, unless
//      the checks found a problem (then it writes nothing).
// Every problem found becomes one 64-bit key ordered as kyto reports problems (gene
// block, then the check in kyto's order, then the row, then which of a row's two checks
// fails), and the smallest key wins (atomicMin). All three kernels are queued at once;
// the host reads the key once, after the join, and words a problem as kyto does
// (KG_ERR_CORRUPT, kyto's KY-E107). A call waits once (twice with host outputs, three
// times with device-resident tile_offsets).

#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <string>

#include "kg_tiles.cuh"

namespace kg {
namespace {

constexpr unsigned long long kNoProblem = ~0ull;
// The checks in kyto's order: check_tile_indptr's four, then check_tile_rows.
enum : uint64_t { kStart = 0, kEnd = 1, kDecrease = 2, kFlat = 3, kRow = 4 };
// Gene blocks a key can name (26 bits); the row takes 34 bits (C <= 2^32 - 1).
constexpr uint64_t kMaxGeneBlocks = 1ull << 26;

__host__ __device__ __forceinline__ unsigned long long problem_key(uint64_t g, uint64_t check,
                                                                   uint64_t row, uint64_t sub) {
  return (g << 38) | (check << 35) | (row << 1) | sub;
}

// A thread per value i of the shard (tile g = i / (C + 1), row r = i % (C + 1)).
__global__ void tile_indptr_check_kernel(const uint32_t* shard, uint32_t n_gb, uint64_t row_len,
                                         uint32_t rows, const uint64_t* start,
                                         unsigned long long* problem, uint32_t* tile_bad) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= (uint64_t)n_gb * row_len) return;
  const uint64_t g = i / row_len, r = i % row_len;
  const uint32_t v = shard[i];
  unsigned long long key = kNoProblem;
  if (r == 0 && v != 0) key = problem_key(g, kStart, 0, 0);
  if (r + 1 == row_len && (uint64_t)v != start[g + 1] - start[g])
    key = min(key, problem_key(g, kEnd, 0, 0));
  if (r + 1 < row_len && shard[i + 1] < v) key = min(key, problem_key(g, kDecrease, r, 0));
  if (r > rows && v != shard[g * row_len + rows]) key = min(key, problem_key(g, kFlat, 0, 0));
  if (key != kNoProblem) {
    atomicMin(problem, key);
    tile_bad[g] = 1;
  }
}

// A warp per row r < rows: the row's segments in the tiles whose indptr passed (their
// values run from 0 to the tile's nnz without decreasing, so [a, e) lies in the tile).
__global__ void tile_rows_kernel(const uint32_t* shard, uint32_t n_gb, uint64_t row_len,
                                 uint32_t rows, const uint64_t* start, const uint32_t* idx,
                                 uint64_t gene_block, uint64_t n_genes, const uint32_t* tile_bad,
                                 unsigned long long* problem, uint64_t* lengths) {
  const uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (r >= rows) return;
  uint64_t total = 0;
  for (uint32_t g = 0; g < n_gb; ++g) {
    if (tile_bad[g]) continue;
    const uint64_t a = shard[g * row_len + r], e = shard[g * row_len + r + 1];
    total += e - a;
    const uint32_t* t = idx + start[g];
    const uint64_t width = min(gene_block, n_genes - g * gene_block);
    bool wide = false, unsorted = false;
    for (uint64_t x = a + lane; x < e; x += 32) {
      const uint32_t v = t[x];
      wide |= v >= width;
      if (x > a) unsorted |= v <= t[x - 1];
    }
    const unsigned w = __ballot_sync(0xFFFFFFFFu, wide);
    const unsigned u = __ballot_sync(0xFFFFFFFFu, unsorted);
    if (lane == 0 && (w | u)) atomicMin(problem, problem_key(g, kRow, r, w ? 0 : 1));
  }
  if (lane == 0) lengths[r] = total;
}

// A warp per row r < rows: its segments in gene-block order, global gene indices, and
// its end offset. Writes nothing when the checks found a problem (the caller's outputs
// stay as they were): every thread reads the verdict, final once the checks ran before
// it on the stream.
__global__ void tile_join_kernel(const uint32_t* shard, uint32_t n_gb, uint64_t row_len,
                                 uint32_t rows, const uint64_t* start, const uint32_t* idx,
                                 const uint32_t* val, uint64_t gene_block,
                                 const unsigned long long* problem, const uint64_t* ends,
                                 uint64_t* out_ptr, uint32_t* out_idx, uint32_t* out_val) {
  const uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (r >= rows || *problem != kNoProblem) return;
  // ends[r] = the entries of rows 0..r (an inclusive scan of the row lengths).
  uint64_t dst = r ? ends[r - 1] : 0;
  if (lane == 0) {
    out_ptr[r + 1] = ends[r];
    if (r == 0) out_ptr[0] = 0;
  }
  for (uint32_t g = 0; g < n_gb; ++g) {
    const uint64_t a = shard[g * row_len + r], e = shard[g * row_len + r + 1];
    const uint64_t base = start[g];
    // g G + local < n_genes <= 2^32 - 1 (the checks passed).
    const uint32_t first_gene = (uint32_t)(g * gene_block);
    for (uint64_t x = a + lane; x < e; x += 32) {
      out_idx[dst + (x - a)] = first_gene + idx[base + x];
      out_val[dst + (x - a)] = val[base + x];
    }
    dst += e - a;
  }
}

template <class T>
T read_one(const T* p, cudaStream_t s) {
  T v{};
  KG_CUDA(cudaMemcpyAsync(&v, p, sizeof(T), cudaMemcpyDefault, s));
  KG_CUDA(cudaStreamSynchronize(s));
  return v;
}

}  // namespace

TileShape tile_shape(const kg_tile_block* tb, cudaStream_t s) {
  if (!tb || !tb->indptr || !tb->tile_offsets) fail(KG_ERR_INVALID, "tiles: NULL argument");
  if (tb->dtype != KG_U32 && tb->dtype != KG_F32) fail(KG_ERR_INVALID, "tiles: unknown dtype");
  const uint64_t c = tb->cell_block_size, gs = tb->gene_block_size;
  if (c == 0 || gs == 0) fail(KG_ERR_INVALID, "tiles: a tile size is 0");
  if (tb->rows == 0 || tb->rows > c || tb->rows > 0x7FFFFFFFu)
    fail(KG_ERR_INVALID, "tiles: rows must be 1..cell_block_size (" + std::to_string(tb->rows) +
                             " rows, cell_block_size " + std::to_string(c) + ")");
  if (tb->n_genes > 0xFFFFFFFFull) fail(KG_ERR_INVALID, "tiles: n_genes above 2^32 - 1");
  if ((unsigned __int128)c * gs > 0xFFFFFFFFull)
    fail(KG_ERR_INVALID, "tiles: cell_block_size * gene_block_size above 2^32 - 1");
  const uint64_t n_gb = (tb->n_genes + gs - 1) / gs;
  if (n_gb >= kMaxGeneBlocks) fail(KG_ERR_INVALID, "tiles: more than 2^26 gene blocks");
  TileShape sh;
  sh.n_gene_blocks = (uint32_t)n_gb;
  sh.start.resize(n_gb + 1);
  if (is_device_pointer(tb->tile_offsets)) {
    KG_CUDA(cudaMemcpyAsync(sh.start.data(), tb->tile_offsets, (n_gb + 1) * 8,
                            cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
  } else {
    std::memcpy(sh.start.data(), tb->tile_offsets, (n_gb + 1) * 8);
  }
  // check_tile_offsets (tile_decode.rs:29-66) over the block's slice.
  for (uint64_t g = 0; g < n_gb; ++g)
    if (sh.start[g + 1] < sh.start[g])
      fail(KG_ERR_CORRUPT, "the layer is corrupt: tile_offsets decreases after tile " +
                               std::to_string(tb->block * n_gb + g));
  sh.first = sh.start[0];
  for (auto& v : sh.start) v -= sh.first;
  sh.nnz = sh.start[n_gb];
  if (sh.nnz && (!tb->indices || !tb->data)) fail(KG_ERR_INVALID, "tiles: NULL entries");
  return sh;
}

void join_tiles(kg_ctx* ctx, cudaStream_t s, const kg_tile_block* tb, const TileShape& sh,
                uint64_t* d_indptr, uint32_t* d_indices, uint32_t* d_values) {
  const uint32_t n_gb = sh.n_gene_blocks, rows = tb->rows;
  const uint64_t row_len = (uint64_t)tb->cell_block_size + 1;
  DeviceBuffer<uint32_t> hs, hi, hv;
  const uint32_t* shard = device_view(tb->indptr, (size_t)n_gb * row_len, hs, s);
  const uint32_t* idx = device_view(tb->indices, sh.nnz, hi, s);
  const uint32_t* val = device_view(static_cast<const uint32_t*>(tb->data), sh.nnz, hv, s);
  DeviceBuffer<uint64_t> start(n_gb + 1, s), lengths(rows, s);
  KG_CUDA(cudaMemcpyAsync(start.ptr, sh.start.data(), (n_gb + 1) * 8ull, cudaMemcpyHostToDevice, s));
  DeviceBuffer<unsigned long long> problem(1, s);
  KG_CUDA(cudaMemsetAsync(problem.ptr, 0xFF, 8, s));
  DeviceBuffer<uint32_t> tile_bad(n_gb, s);
  tile_bad.zero();
  if (n_gb) {
    tile_indptr_check_kernel<<<blocks_for((uint64_t)n_gb * row_len, 256), 256, 0, s>>>(
        shard, n_gb, row_len, rows, start.ptr, problem.ptr, tile_bad.ptr);
    KG_LAUNCH_CHECK();
  }
  tile_rows_kernel<<<blocks_for((uint64_t)rows * 32, 256), 256, 0, s>>>(
      shard, n_gb, row_len, rows, start.ptr, idx, tb->gene_block_size, tb->n_genes, tile_bad.ptr,
      problem.ptr, lengths.ptr);
  KG_LAUNCH_CHECK();
  // The rows' ends and the join are queued before the verdict is read (one wait a call);
  // the join writes only when the checks passed.
  size_t temp = 0;
  KG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, temp, lengths.ptr, lengths.ptr, rows, s));
  DeviceBuffer<unsigned char> scratch(temp, s);
  KG_CUDA(cub::DeviceScan::InclusiveSum(scratch.ptr, temp, lengths.ptr, lengths.ptr, rows, s));
  tile_join_kernel<<<blocks_for((uint64_t)rows * 32, 256), 256, 0, s>>>(
      shard, n_gb, row_len, rows, start.ptr, idx, val, tb->gene_block_size, problem.ptr,
      lengths.ptr, d_indptr, d_indices, d_values);
  KG_LAUNCH_CHECK();
  unsigned long long key = kNoProblem;
  KG_CUDA(cudaMemcpyAsync(&key, problem.ptr, 8, cudaMemcpyDeviceToHost, s));
  wait_stream(ctx, s);
  if (key == kNoProblem) return;
  // kyto's wording (tile_decode.rs:129-196), the details read back from the inputs.
  const uint64_t g = key >> 38, check = (key >> 35) & 7u, r = (key >> 1) & ((1ull << 34) - 1);
  std::string what;
  if (check == kStart) {
    what = "indptr does not start at 0";
  } else if (check == kEnd) {
    const uint32_t end = read_one(shard + g * row_len + row_len - 1, s);
    what = "indptr ends at Some(" + std::to_string(end) + ") but tile_offsets gives " +
           std::to_string(sh.start[g + 1] - sh.start[g]) + " entries";
  } else if (check == kDecrease) {
    what = "indptr decreases after row " + std::to_string(r);
  } else if (check == kFlat) {
    what = "indptr is not flat after the last row " + std::to_string(rows);
  } else if (key & 1u) {
    what = "row " + std::to_string(r) + ": gene indices are not strictly increasing";
  } else {
    const uint64_t width = std::min(tb->gene_block_size, tb->n_genes - g * tb->gene_block_size);
    const uint32_t a = read_one(shard + g * row_len + r, s);
    const uint32_t e = read_one(shard + g * row_len + r + 1, s);
    std::vector<uint32_t> row(e - a);
    if (e > a) {
      KG_CUDA(cudaMemcpyAsync(row.data(), idx + sh.start[g] + a, (e - a) * 4ull,
                              cudaMemcpyDeviceToHost, s));
      KG_CUDA(cudaStreamSynchronize(s));
    }
    uint32_t local = 0;
    for (uint32_t v : row)
      if (v >= width) {
        local = v;
        break;
      }
    what = "row " + std::to_string(r) + ": local gene index " + std::to_string(local) +
           " is not below the block width " + std::to_string(width);
  }
  fail(KG_ERR_CORRUPT, "the layer is corrupt: tile (" + std::to_string(tb->block) + ", " +
                           std::to_string(g) + "): " + what);
}

}  // namespace kg

using namespace kg;

extern "C" {

kg_status kg_tiles_to_csr(kg_ctx* ctx, const kg_tile_block* block, uint64_t* indptr,
                          uint32_t* indices, void* values) {
  return guarded([&] {
    if (!ctx || !block || !indptr) fail(KG_ERR_INVALID, "kg_tiles_to_csr: NULL argument");
    use_device(ctx);
    cudaStream_t s = ctx->stream;
    const TileShape sh = tile_shape(block, s);
    if (sh.nnz && (!indices || !values)) fail(KG_ERR_INVALID, "kg_tiles_to_csr: NULL output");
    const uint64_t rows = block->rows;
    DeviceBuffer<uint64_t> op;
    DeviceBuffer<uint32_t> oi, ov;
    const bool dp = is_device_pointer(indptr), di = is_device_pointer(indices),
               dv = is_device_pointer(values);
    if (!dp) op.alloc(rows + 1, s);
    if (!di) oi.alloc(sh.nnz, s);
    if (!dv) ov.alloc(sh.nnz, s);
    uint64_t* d_ptr = dp ? indptr : op.ptr;
    uint32_t* d_idx = di ? indices : oi.ptr;
    uint32_t* d_val = dv ? static_cast<uint32_t*>(values) : ov.ptr;
    join_tiles(ctx, s, block, sh, d_ptr, d_idx, d_val);
    if (!dp) KG_CUDA(cudaMemcpyAsync(indptr, d_ptr, (rows + 1) * 8, cudaMemcpyDeviceToHost, s));
    if (!di && sh.nnz)
      KG_CUDA(cudaMemcpyAsync(indices, d_idx, sh.nnz * 4, cudaMemcpyDeviceToHost, s));
    if (!dv && sh.nnz)
      KG_CUDA(cudaMemcpyAsync(values, d_val, sh.nnz * 4, cudaMemcpyDeviceToHost, s));
    wait_stream(ctx, s);
  });
}

}  // extern "C"
