// The PCA's sparse x dense products on the 5th-generation tensor cores.
//
//   C (rows x 64) = S (rows x K, sparse, f32 values) . D (K x 64)
//
// S is the held input X (rows = cells, K = genes) for X Q and the embedding pass, or X^T
// (rows = genes, K = cells) for X^T W, the sketch and the gene statistics; both are kept
// in the bitmask block layout of kg_spmm_tc.cuh (128 rows x 32 columns per block). D
// comes as D^T (64 x K) in two tf32 parts (hi + lo), K-major f32. Each 128 x 32 block of
// S is expanded straight into tensor memory (one thread per row: its mask word and
// values become the row's 32 hi and 32 lo tf32 parts, stored into its TMEM lane) and
// multiplied by three TF32 MMAs that read A from TMEM and D^T from shared memory
// (hi.hi + hi.lo + lo.hi: the f32 operands to about 2^-21), accumulated in TMEM over at
// most kFlushChunks chunks and then added into f64 registers (no f32 sum runs over more
// than 512 terms). Shared memory carries only the loads (D^T tiles and blocks), so the
// MMAs' operand reads do not compete with the expansion for it.
//
// Per CTA (persistent, 320 threads) and per K-chunk of a work item (tile, K segment):
//   warp 8      loads: the chunk's D^T tiles (64 x 32, two parts, TMA) and the block (one
//               bulk copy) into one of kLoadStages stages; the next 32 blocks are
//               prefetched into L2 ahead of their copies;
//   warps 0-3   expand: thread r writes row r of the chunk's A tile (hi and lo parts)
//               into TMEM lane r of one of two A buffers;
//   warp 9      MMA: 12 tcgen05.mma (kind::tf32, A from TMEM, M=128 N=64 K=8) into one
//               of two TMEM accumulators;
//   warps 4-7   drain: TMEM -> f64 registers per flush group; at the end of the item the
//               rows (C - offsets, as tf32 parts of C^T, f32 rows and column sums) or the
//               segment's f64 partial.
// HBM sees each block once per product (its mask and values: 512 + 4 nnz bytes) and
// D^T about once per pass over it (L2 serves the other tiles of a segment).
#include <cudaTypedefs.h>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <mutex>

#include "kg_internal.cuh"
#include "kg_sm100.cuh"
#include "kg_spmm_tc.cuh"

namespace kg {

using namespace sm100;

namespace {

constexpr int kRows = 128;              // rows per tile (M)
constexpr int kChunk = 32;              // K per chunk (one 128-byte swizzle row of f32)
constexpr int kN = 64;                  // output columns (N)
constexpr int kLoadStages = 6;
constexpr int kFlushChunks = 16;        // K-chunks summed in f32 before the f64 flush
constexpr uint32_t kBBytes = kN * 128;  // 8 KB: 64 rows x 32 f32
constexpr uint32_t kMaskBytes = kRows * 4;
constexpr uint32_t kBlockMaxBytes = kMaskBytes + kRows * kChunk * 4;
constexpr int kProducerWarps = 4;
constexpr int kEpilogueWarps = 4;
constexpr int kSpThreads = (kProducerWarps + kEpilogueWarps + 2) * 32;
// TMEM columns: two 64-column f32 accumulators (0..127), then two A buffers of 64
// columns (hi parts in the first 32, lo parts in the next 32; lane = row of the tile).
constexpr uint32_t kTmemColsS = 256;
constexpr uint32_t kAccCols = 64, kABase = 128, kACols = 64;

struct LoadStage {
  uint8_t b_hi[kBBytes];
  uint8_t b_lo[kBBytes];
  uint8_t blk[(kBlockMaxBytes + 1023) / 1024 * 1024];  // mask words, then the values
};
// Swizzled tiles (TMA destinations, MMA operands) start on 1024-byte boundaries.
static_assert(sizeof(LoadStage) % 1024 == 0, "load stage size");

struct SpSmem {
  LoadStage st[kLoadStages];
  double colsum[2][kEpilogueWarps][kN];
  uint64_t ld_full[kLoadStages], ld_empty[kLoadStages];
  uint64_t a_full[2], a_empty[2];
  uint64_t cs_ready;
  uint64_t acc_full[2], acc_empty[2];
  uint64_t drained;
  uint32_t present[kLoadStages];
  uint32_t tmem_base;
  int abort;
};
constexpr size_t kSpSmemBytes = sizeof(SpSmem) + 1024;
static_assert(kSpSmemBytes <= 227 * 1024, "SpMM shared memory");
static_assert(offsetof(SpSmem, st) % 1024 == 0, "tile alignment");

__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// A 1D bulk copy global -> shared, counted in bytes on `bar` (16-byte aligned, size a
// multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Prefetch [src, src + bytes) into L2 (16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(reinterpret_cast<uint64_t>(src)),
               "r"(bytes)
               : "memory");
}

struct Geometry {
  uint32_t n_tiles, n_chunks, seg_chunks, n_segs;
  __device__ __forceinline__ uint64_t items() const { return (uint64_t)n_tiles * n_segs; }
  // Consecutive items share a K segment (its D^T tiles stay in L2 for the next tile).
  __device__ __forceinline__ void item(uint64_t w, uint32_t& tile, uint32_t& seg) const {
    tile = (uint32_t)(w % n_tiles);
    seg = (uint32_t)(w / n_tiles);
  }
  __device__ __forceinline__ uint32_t chunks(uint32_t seg) const {
    uint32_t c0 = seg * seg_chunks;
    return min(seg_chunks, n_chunks - c0);
  }
  __device__ __forceinline__ uint64_t first_block(uint32_t tile, uint32_t seg) const {
    return (uint64_t)tile * n_chunks + (uint64_t)seg * seg_chunks;
  }
};

__global__ void __launch_bounds__(kSpThreads, 1)
spmm_tc_kernel(const __grid_constant__ CUtensorMap tmap_hi,
               const __grid_constant__ CUtensorMap tmap_lo, const uint64_t* __restrict__ off,
               const uint8_t* __restrict__ data, uint64_t rows, Geometry geo, int value_mode,
               const double* __restrict__ row_means, SpmmOut out, int* error) {
  extern __shared__ uint8_t smem_raw[];
  // Aligned to 1024 bytes by an offset into the __shared__ array itself, so the compiler
  // keeps every access in the shared state space (no generic loads and stores).
  SpSmem& sm = *reinterpret_cast<SpSmem*>(smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u));
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint64_t n_items = geo.items();
  volatile int* abort = &sm.abort;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kLoadStages; ++s) {
      mbar_init(&sm.ld_full[s], 1);
      mbar_init(&sm.ld_empty[s], kProducerWarps + 1);  // the expanders and the MMA commit
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sm.a_full[b], kProducerWarps);
      mbar_init(&sm.a_empty[b], 1);
      mbar_init(&sm.acc_full[b], 1);
      mbar_init(&sm.acc_empty[b], kEpilogueWarps);
    }
    mbar_init(&sm.cs_ready, kEpilogueWarps);
    mbar_init(&sm.drained, 1);
    sm.abort = 0;
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(&sm.tmem_base, kTmemColsS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;

  if (warp < kProducerWarps) {
    // ----------------------------------------------------------- expand -------------
    const uint32_t r = threadIdx.x;  // the row of the tile this thread writes (0..127)
    uint64_t it = 0;
    bool ok = true;
    for (uint64_t w = blockIdx.x; w < n_items && ok; w += gridDim.x) {
      uint32_t tile, seg;
      geo.item(w, tile, seg);
      const uint32_t nc = geo.chunks(seg);
      float mean_r = 0.0f;
      if (value_mode == kValueCentredSquare) {
        const uint64_t row = (uint64_t)tile * kRows + r;
        mean_r = row < rows ? (float)row_means[row] : 0.0f;
      }
      for (uint32_t c = 0; c < nc; ++c, ++it) {
        const int ls = (int)(it % kLoadStages);
        const uint32_t lph = (uint32_t)((it / kLoadStages) & 1);
        const uint32_t ab = (uint32_t)(it & 1), aph = (uint32_t)((it >> 1) & 1);
        if (!mbar_wait(&sm.ld_full[ls], lph, abort) || !mbar_wait(&sm.a_empty[ab], aph ^ 1, abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const LoadStage& st = sm.st[ls];
        const bool present = sm.present[ls] != 0;
        const uint32_t* masks = reinterpret_cast<const uint32_t*>(st.blk);
        const float* vals = reinterpret_cast<const float*>(st.blk + kMaskBytes);
        // The row's first value: the stored values of the rows before it. The earlier
        // warps' rows: one warp-wide add of each lane's popcounts; the rows before it in
        // this warp: an exclusive scan of the row counts (at most 32, 6 bits) built from
        // one ballot per bit, popcounts of the lower lanes' bits, no dependent shuffles.
        uint32_t mword = 0, base = 0;
        if (present) {
          mword = masks[r];
          uint32_t before = 0;
          for (int q = 0; q < warp; ++q) before += __popc(masks[q * 32 + lane]);
          before = __reduce_add_sync(0xFFFFFFFFu, before);
          const uint32_t cnt = __popc(mword);
          const uint32_t lower = (1u << lane) - 1u;
          uint32_t excl = 0;
#pragma unroll
          for (int b = 0; b < 6; ++b)
            excl += (uint32_t)__popc(__ballot_sync(0xFFFFFFFFu, (cnt >> b) & 1u) & lower) << b;
          base = before + excl;
        }
        // Branch-free: every column's value is loaded from its would-be rank (the rank
        // of the next stored value for an empty cell: still inside the stage buffer,
        // which holds 4,224 values) and kept only where the mask bit is set, so all 32
        // loads issue back to back.
        float v[kChunk];
#pragma unroll
        for (int col = 0; col < kChunk; ++col) {
          const uint32_t below = col ? __popc(mword & ((1u << col) - 1u)) : 0u;
          const float x = vals[base + below];
          v[col] = ((mword >> col) & 1u) ? x : 0.0f;
        }
        if (value_mode == kValueCentredSquare) {
#pragma unroll
          for (int col = 0; col < kChunk; ++col) {
            const float d = v[col] - mean_r;
            v[col] = ((mword >> col) & 1u) ? d * d : 0.0f;
          }
        } else if (value_mode == kValueOne) {
#pragma unroll
          for (int col = 0; col < kChunk; ++col) v[col] = ((mword >> col) & 1u) ? 1.0f : 0.0f;
        }
        // Row r of the A tile (tf32 hi and lo parts) into TMEM lane r, where the MMA reads it.
        uint32_t hi[kChunk], lo[kChunk];
#pragma unroll
        for (int col = 0; col < kChunk; ++col) {
          const float h = tf32_round(v[col]);
          hi[col] = __float_as_uint(h);
          lo[col] = __float_as_uint(v[col] - h);
        }
        const uint32_t arow = tmem + (((uint32_t)warp * 32u) << 16) + kABase + ab * kACols;
        tmem_st_32(arow, hi);
        tmem_st_32(arow + 32u, lo);
        tmem_wait_st();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&sm.a_full[ab]);
          mbar_arrive(&sm.ld_empty[ls]);
        }
      }
    }
  } else if (warp < kProducerWarps + kEpilogueWarps) {
    // ----------------------------------------------------------- drain TMEM ---------
    const uint32_t quad = (uint32_t)warp & 3u;  // warps 4..7 -> TMEM lanes 32*quad..
    const uint32_t i = quad * 32u + lane;
    uint64_t fg = 0, item_no = 0;
    bool ok = true;
    for (uint64_t w = blockIdx.x; w < n_items && ok; w += gridDim.x, ++item_no) {
      uint32_t tile, seg;
      geo.item(w, tile, seg);
      const uint64_t row = (uint64_t)tile * kRows + i;
      double acc[kN];
#pragma unroll
      for (int j = 0; j < kN; ++j) acc[j] = 0.0;
      const uint32_t nc = geo.chunks(seg);
      const uint32_t groups = (nc + kFlushChunks - 1) / kFlushChunks;
      for (uint32_t gr = 0; gr < groups; ++gr, ++fg) {
        const uint32_t b = (uint32_t)(fg & 1), bph = (uint32_t)((fg >> 1) & 1);
        if (!mbar_wait(&sm.acc_full[b], bph, abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        __syncwarp();
        // One 32-column half at a time (fewer live registers beside the f64 sums).
#pragma unroll
        for (int hf = 0; hf < 2; ++hf) {
          uint32_t rr[32];
          tmem_ld_32(tmem + ((quad * 32u) << 16) + b * kAccCols + hf * 32u, rr);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 32; ++j) acc[hf * 32 + j] += (double)__uint_as_float(rr[j]);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.acc_empty[b]);
      }
      if (!ok) break;
      if (out.mode == kOutRows) {
        // C = S D - offsets: the next product's D^T (tf32 parts), the f32 rows, and this
        // tile's column sums (fixed tree: warp shuffles, then the 4 warps in order).
        const bool live = row < rows;
#pragma unroll
        for (int j = 0; j < kN; ++j) {
          double cval = live && j < (int)out.width ? acc[j] - out.offsets[j] : 0.0;
          float hi = tf32_round((float)cval);
          float lo = tf32_round((float)(cval - (double)hi));
          if (live && out.t_hi) {
            out.t_hi[(uint64_t)j * out.ld_t + row] = hi;
            out.t_lo[(uint64_t)j * out.ld_t + row] = lo;
          }
          if (live && out.rows_f32 && j < (int)out.width)
            out.rows_f32[row * (uint64_t)out.width + j] = (float)cval;
          if (out.colsum_partial) {
            double sv = (double)hi + (double)lo;
            for (int o = 16; o; o >>= 1) sv += __shfl_xor_sync(0xFFFFFFFFu, sv, o);
            if (lane == 0) sm.colsum[item_no & 1][quad][j] = sv;
          }
        }
        if (out.colsum_partial) {
          // The four warps' sums in a fixed order (double-buffered by item, so a warp
          // running one item ahead cannot overwrite what warp 4 still reads).
          __syncwarp();
          if (lane == 0) mbar_arrive(&sm.cs_ready);
          if (!mbar_wait(&sm.cs_ready, (uint32_t)(item_no & 1), abort)) break;
          if (quad == 0) {
            const double(*cs)[kN] = sm.colsum[item_no & 1];
            for (int j = lane; j < kN; j += 32) {
              double tsum = ((cs[0][j] + cs[1][j]) + cs[2][j]) + cs[3][j];
              out.colsum_partial[(uint64_t)tile * kN + j] = tsum;
            }
          }
        }
      } else if (row < rows) {
        double* dst = out.partial + ((uint64_t)seg * rows + row) * kN;
#pragma unroll
        for (int j = 0; j < kN; ++j) dst[j] = acc[j];
      }
    }
  } else if (warp == kProducerWarps + kEpilogueWarps) {
    // ----------------------------------------------------------- loads --------------
    // Lane 0 issues; the warp reads the item's block offsets 32 at a time ahead of it,
    // and each window's successor (or the next item's first window) is prefetched into
    // L2 while this one is copied.
    if (lane == 0) {
      prefetch_tmap(&tmap_hi);
      prefetch_tmap(&tmap_lo);
    }
    uint64_t it = 0;
    int issued_phase[kLoadStages];
    for (int s = 0; s < kLoadStages; ++s) issued_phase[s] = -1;
    bool ok = true;
    for (uint64_t w = blockIdx.x; w < n_items && ok; w += gridDim.x) {
      uint32_t tile, seg;
      geo.item(w, tile, seg);
      const uint32_t nc = geo.chunks(seg);
      const uint64_t b0 = geo.first_block(tile, seg);
      uint64_t win = 0, win_end = 0;
      for (uint32_t c = 0; c < nc; ++c, ++it) {
        const uint32_t at = c & 31u;
        if (at == 0) {
          // off[b0 + c + lane] and, in lane 0, off[b0 + c + 32] (indices <= nc: the
          // offsets array holds one entry past every block).
          win = c + lane <= nc ? off[b0 + c + lane] : 0;
          win_end = lane == 0 && c + 32 <= nc ? off[b0 + c + 32] : 0;
          if (lane == 0) {
            uint64_t p0 = 0, p1 = 0;
            if (c + 32 < nc) {
              p0 = win_end;
              p1 = off[b0 + min(c + 64, nc)];
            } else if (w + gridDim.x < n_items) {
              uint32_t t2, s2;
              geo.item(w + gridDim.x, t2, s2);
              const uint64_t nb0 = geo.first_block(t2, s2);
              p0 = off[nb0];
              p1 = off[nb0 + min(32u, geo.chunks(s2))];
            }
            for (uint64_t u = p0; u < p1; u += 4096) {  // 64 KB per prefetch
              const uint64_t units = p1 - u < 4096 ? p1 - u : 4096;
              bulk_prefetch_l2(data + u * 16, (uint32_t)(units * 16));
            }
          }
        }
        const uint64_t e0 = __shfl_sync(0xFFFFFFFFu, win, at);
        const uint64_t e1n = __shfl_sync(0xFFFFFFFFu, win, (at + 1) & 31u);
        const uint64_t e1w = __shfl_sync(0xFFFFFFFFu, win_end, 0);
        const uint64_t e1 = at == 31 ? e1w : e1n;
        if (lane == 0) {
          const int s = (int)(it % kLoadStages);
          const uint32_t ph = (uint32_t)((it / kLoadStages) & 1);
          if (!mbar_wait(&sm.ld_empty[s], ph ^ 1, abort)) {
            ok = false;
          } else {
            const uint32_t chunk = seg * geo.seg_chunks + c;
            const uint32_t bytes = (uint32_t)((e1 - e0) * 16);
            sm.present[s] = bytes ? 1u : 0u;
            mbar_arrive_expect_tx(&sm.ld_full[s], 2 * kBBytes + bytes);
            const int32_t x = (int32_t)(chunk * kChunk);
            tma_load_2d(sm.st[s].b_hi, &tmap_hi, &sm.ld_full[s], x, 0);
            tma_load_2d(sm.st[s].b_lo, &tmap_lo, &sm.ld_full[s], x, 0);
            if (bytes) bulk_load(sm.st[s].blk, data + e0 * 16, bytes, &sm.ld_full[s]);
            issued_phase[s] = (int)ph;
          }
        }
        ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
        if (!ok) break;
      }
    }
    if (lane == 0) {
      for (int s = 0; s < kLoadStages; ++s) {
        if (issued_phase[s] < 0) continue;
        for (uint32_t q = 0; q < kWaitPolls && !mbar_try_wait(&sm.ld_full[s], issued_phase[s]); ++q)
          ;
      }
    }
  } else {
    // ----------------------------------------------------------- MMA ----------------
    if (lane == 0) {
      const uint32_t idesc = idesc_f32acc(2u, kRows, kN);  // tf32 x tf32 -> f32
      uint64_t it = 0, fg = 0;
      bool ok = true;
      for (uint64_t w = blockIdx.x; w < n_items && ok; w += gridDim.x) {
        uint32_t tile, seg;
        geo.item(w, tile, seg);
        const uint32_t nc = geo.chunks(seg);
        for (uint32_t c = 0; c < nc && ok; ++c, ++it) {
          const uint32_t in_group = c % kFlushChunks;
          const uint32_t b = (uint32_t)(fg & 1), bph = (uint32_t)((fg >> 1) & 1);
          if (in_group == 0 && !mbar_wait(&sm.acc_empty[b], bph ^ 1, abort)) {
            ok = false;
            break;
          }
          const int ls = (int)(it % kLoadStages);
          const uint32_t lph = (uint32_t)((it / kLoadStages) & 1);
          const uint32_t ab = (uint32_t)(it & 1), aph = (uint32_t)((it >> 1) & 1);
          if (!mbar_wait(&sm.ld_full[ls], lph, abort) || !mbar_wait(&sm.a_full[ab], aph, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem + b * kAccCols;
          const uint32_t ah = tmem + kABase + ab * kACols, al = ah + 32u;
          const uint32_t bh = smem_addr(sm.st[ls].b_hi), bl = smem_addr(sm.st[ls].b_lo);
#pragma unroll
          for (int kk = 0; kk < kChunk / 8; ++kk) {
            const uint32_t o = kk * 32;  // 8 tf32 of K: 32 bytes of a B row, 8 A columns
            mma_tf32_ts(d, ah + kk * 8, desc_k_sw128(bh + o), idesc, (in_group | kk) != 0);
            mma_tf32_ts(d, ah + kk * 8, desc_k_sw128(bl + o), idesc, 1);
            mma_tf32_ts(d, al + kk * 8, desc_k_sw128(bh + o), idesc, 1);
          }
          mma_commit(&sm.ld_empty[ls]);
          mma_commit(&sm.a_empty[ab]);
          if (in_group == kFlushChunks - 1 || c == nc - 1) {
            mma_commit(&sm.acc_full[b]);
            ++fg;
          }
        }
      }
      mma_commit(&sm.drained);
      for (uint32_t q = 0; q < kWaitPolls && !mbar_try_wait(&sm.drained, 0); ++q)
        ;
    }
  }
  __syncwarp();
  __syncthreads();
  if (sm.abort && threadIdx.x == 0) atomicExch(error, 1);
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemColsS);
  }
}

// ------------------------------------------------------------------ builders -------

// The block of a stored value, and its row (in the tile) and column (in the chunk).
__device__ __forceinline__ void locate(uint64_t r, uint32_t c, bool transpose, uint32_t n_chunks,
                                       uint64_t& block, uint32_t& br, uint32_t& bc) {
  uint64_t orow = transpose ? c : r;  // row of the output layout
  uint64_t ocol = transpose ? r : c;
  block = (orow / kRows) * n_chunks + ocol / kChunk;
  br = (uint32_t)(orow % kRows);
  bc = (uint32_t)(ocol % kChunk);
}

// Stored values per block (warp per CSR row; lanes whose values share a block add once).
__global__ void blocked_count_kernel(const uint64_t* ptr, const uint32_t* col, uint64_t n_rows,
                                     bool transpose, uint32_t n_chunks, uint32_t* counts) {
  uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  if (r >= n_rows) return;
  for (uint64_t i0 = ptr[r]; i0 < ptr[r + 1]; i0 += 32) {
    uint64_t i = i0 + lane;
    bool in = i < ptr[r + 1];
    unsigned active = __ballot_sync(0xFFFFFFFFu, in);
    if (!in) continue;
    uint64_t block;
    uint32_t br, bc;
    locate(r, col[i], transpose, n_chunks, block, br, bc);
    unsigned same = __match_any_sync(active, block);
    if ((unsigned)__ffs(same) - 1 == lane) atomicAdd(&counts[block], (uint32_t)__popc(same));
  }
}

// A block's size in 16-byte units: 128 mask words and its values padded to 4 (none for
// an empty block).
__global__ void block_units_kernel(const uint32_t* counts, uint64_t n, uint64_t* units) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) units[i] = counts[i] ? kMaskBytes / 16 + ((uint64_t)counts[i] + 3) / 4 : 0;
  if (i == n) units[i] = 0;
}

// Mask bits: bit c of word r of a block marks the value at (row r, column c). Lanes that
// hit the same word OR their bits together first.
__global__ void blocked_mask_kernel(const uint64_t* ptr, const uint32_t* col, uint64_t n_rows,
                                    bool transpose, uint32_t n_chunks, const uint64_t* off,
                                    uint8_t* data) {
  uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  if (r >= n_rows) return;
  for (uint64_t i0 = ptr[r]; i0 < ptr[r + 1]; i0 += 32) {
    uint64_t i = i0 + lane;
    bool in = i < ptr[r + 1];
    unsigned active = __ballot_sync(0xFFFFFFFFu, in);
    if (!in) continue;
    uint64_t block;
    uint32_t br, bc;
    locate(r, col[i], transpose, n_chunks, block, br, bc);
    uint32_t* word = reinterpret_cast<uint32_t*>(data + off[block] * 16) + br;
    unsigned same = __match_any_sync(active, reinterpret_cast<uint64_t>(word));
    uint32_t bits = __reduce_or_sync(same, 1u << bc);
    if ((unsigned)__ffs(same) - 1 == lane) atomicOr(word, bits);
  }
}

// prefix[b * 128 + row]: the values of block b in the rows before `row` (warp per block).
__global__ void row_prefix_kernel(const uint64_t* off, const uint8_t* data, uint64_t n_blocks,
                                  uint16_t* prefix) {
  uint64_t b = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  if (b >= n_blocks || off[b + 1] == off[b]) return;
  const uint32_t* masks = reinterpret_cast<const uint32_t*>(data + off[b] * 16);
  uint32_t carry = 0;
  for (int q = 0; q < kRows / 32; ++q) {
    uint32_t v = __popc(masks[q * 32 + lane]);
    uint32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += t;
    }
    prefix[b * kRows + q * 32 + lane] = (uint16_t)(carry + incl - v);
    carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
  }
}

// Each value at its rank in its block (rows in order, columns in order inside a row).
__global__ void blocked_values_kernel(const uint64_t* ptr, const uint32_t* col, const float* val,
                                      uint64_t n_rows, bool transpose, uint32_t n_chunks,
                                      const uint64_t* off, const uint16_t* prefix,
                                      uint8_t* data) {
  uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  if (r >= n_rows) return;
  for (uint64_t i = ptr[r] + lane; i < ptr[r + 1]; i += 32) {
    uint64_t block;
    uint32_t br, bc;
    locate(r, col[i], transpose, n_chunks, block, br, bc);
    uint8_t* blk = data + off[block] * 16;
    const uint32_t word = reinterpret_cast<const uint32_t*>(blk)[br];
    const uint32_t rank = prefix[block * kRows + br] + __popc(word & ((1u << bc) - 1u));
    reinterpret_cast<float*>(blk + kMaskBytes)[rank] = val[i];
  }
}

// ---------------------------------------------------------------- the transpose --
//
// X^T's blocked layout from X's (no pass over the CSR, no atomics). Block (G, c) of X^T
// (genes 128 G.., cells 32 c..) holds the 32 cell rows 32 (c % 4).. of the four X blocks
// (tile c / 4, gene chunks 4 G ..4 G + 3), transposed: its gene row 32 i + j has bit l set
// where X block (c / 4, 4 G + i) has a value at cell row 32 (c % 4) + l, gene column j.
// One warp per X^T block; lane l reads cell row 32 (c % 4) + l of each source block.

// Source block i of X^T block (G, c), or ~0 past X's gene chunks.
__device__ __forceinline__ uint64_t transpose_source(uint32_t G, uint32_t c, int i,
                                                     uint32_t x_chunks) {
  const uint32_t chunk = 4 * G + (uint32_t)i;
  return chunk < x_chunks ? (uint64_t)(c / 4) * x_chunks + chunk : ~0ull;
}

__global__ void transpose_count_kernel(const uint64_t* x_off, const uint8_t* x_data,
                                       uint32_t x_chunks, uint32_t t_tiles, uint32_t t_chunks,
                                       uint32_t* counts) {
  const uint64_t b = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (b >= (uint64_t)t_tiles * t_chunks) return;
  const uint32_t G = (uint32_t)(b / t_chunks), c = (uint32_t)(b % t_chunks);
  uint32_t count = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint64_t src = transpose_source(G, c, i, x_chunks);
    if (src == ~0ull || x_off[src + 1] == x_off[src]) continue;
    const uint32_t* masks = reinterpret_cast<const uint32_t*>(x_data + x_off[src] * 16);
    count += __popc(masks[32 * (c % 4) + lane]);
  }
  for (int o = 16; o; o >>= 1) count += __shfl_xor_sync(0xFFFFFFFFu, count, o);
  if (lane == 0) counts[b] = count;
}

__global__ void transpose_fill_kernel(const uint64_t* x_off, const uint8_t* x_data,
                                      uint32_t x_chunks, uint32_t t_tiles, uint32_t t_chunks,
                                      const uint64_t* t_off, uint8_t* t_data) {
  const uint64_t b = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (b >= (uint64_t)t_tiles * t_chunks || t_off[b + 1] == t_off[b]) return;
  const uint32_t G = (uint32_t)(b / t_chunks), c = (uint32_t)(b % t_chunks);
  const uint32_t group = c % 4;  // the source blocks' cell rows 32 group..
  uint32_t src_mask[4], src_pre[4], mine[4];
  const float* src_vals[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    src_mask[i] = 0;
    src_pre[i] = 0;
    src_vals[i] = nullptr;
    const uint64_t src = transpose_source(G, c, i, x_chunks);
    if (src != ~0ull && x_off[src + 1] != x_off[src]) {
      const uint8_t* blk = x_data + x_off[src] * 16;
      const uint32_t* masks = reinterpret_cast<const uint32_t*>(blk);
      src_vals[i] = reinterpret_cast<const float*>(blk + kMaskBytes);
      src_mask[i] = masks[32 * group + lane];
      // Values of the source block before cell row 32 group + lane (rows in order).
      uint32_t base = 0;
      for (uint32_t q = 0; q < group; ++q) base += __popc(masks[32 * q + lane]);
      for (int o = 16; o; o >>= 1) base += __shfl_xor_sync(0xFFFFFFFFu, base, o);
      const uint32_t v = __popc(src_mask[i]);
      uint32_t incl = v;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += t;
      }
      src_pre[i] = base + incl - v;
    }
    // The 32 x 32 bit transpose: gene j's cell mask is the ballot of bit j.
    mine[i] = 0;
#pragma unroll 4
    for (int j = 0; j < 32; ++j) {
      const uint32_t t = __ballot_sync(0xFFFFFFFFu, (src_mask[i] >> j) & 1u);
      if ((int)lane == j) mine[i] = t;
    }
  }
  uint8_t* out = t_data + t_off[b] * 16;
  uint32_t* out_masks = reinterpret_cast<uint32_t*>(out);
  float* out_vals = reinterpret_cast<float*>(out + kMaskBytes);
  uint32_t carry = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    out_masks[32 * i + lane] = mine[i];
    // This gene row's first value: the values of the X^T rows before it.
    const uint32_t v = __popc(mine[i]);
    uint32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += t;
    }
    uint32_t at = carry + incl - v;
    carry += __shfl_sync(0xFFFFFFFFu, incl, 31);
    // Cells in order: cell l's value sits at its rank in source block i.
    const uint32_t below = (1u << lane) - 1u;  // gene columns before this lane's
    const float* sv = src_vals[i];
    const uint32_t mi = mine[i];
    for (int l = 0; l < 32; ++l) {
      const uint32_t pre = __shfl_sync(0xFFFFFFFFu, src_pre[i], l);
      const uint32_t m = __shfl_sync(0xFFFFFFFFu, src_mask[i], l);
      const uint32_t has = (mi >> l) & 1u;
      if (has) out_vals[at] = sv[pre + __popc(m & below)];
      at += has;
    }
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  if (!fn) fail(KG_ERR_DEVICE, "cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

// D^T part: 64 rows x K f32 (row stride ld floats), boxes of 64 rows x 32 columns.
CUtensorMap dt_map(const float* base, uint64_t K, uint64_t ld) {
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)kN};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
  cuuint32_t box[2] = {(cuuint32_t)kChunk, (cuuint32_t)kN};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    fail(KG_ERR_DEVICE, "cuTensorMapEncodeTiled (D^T) failed: " + std::to_string((int)r));
  return m;
}

}  // namespace

void build_blocked(const uint64_t* ptr, const uint32_t* col, const float* val, uint64_t n_rows,
                   uint64_t n_cols, uint64_t nnz, bool transpose, Blocked& out, cudaStream_t s) {
  out.rows = transpose ? n_cols : n_rows;
  out.K = transpose ? n_rows : n_cols;
  out.n_tiles = (uint32_t)((out.rows + kRows - 1) / kRows);
  out.n_chunks = (uint32_t)((out.K + kChunk - 1) / kChunk);
  const uint64_t nb = (uint64_t)out.n_tiles * out.n_chunks;
  DeviceBuffer<uint32_t> counts(nb, s);
  counts.zero();
  if (nnz) {
    blocked_count_kernel<<<blocks_for(n_rows * 32, 256), 256, 0, s>>>(
        ptr, col, n_rows, transpose, out.n_chunks, counts.ptr);
    KG_LAUNCH_CHECK();
  }
  out.off.alloc(nb + 1, s);
  block_units_kernel<<<blocks_for(nb + 1, 256), 256, 0, s>>>(counts.ptr, nb, out.off.ptr);
  KG_LAUNCH_CHECK();
  counts.reset();
  size_t temp = 0;
  KG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, out.off.ptr, out.off.ptr, nb + 1, s));
  DeviceBuffer<unsigned char> scratch(temp, s);
  KG_CUDA(cub::DeviceScan::ExclusiveSum(scratch.ptr, temp, out.off.ptr, out.off.ptr, nb + 1, s));
  uint64_t units = 0;
  KG_CUDA(cudaMemcpyAsync(&units, out.off.ptr + nb, 8, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  out.bytes = units * 16;
  out.data.alloc(std::max<uint64_t>(out.bytes, 16), s);
  out.data.zero();
  if (nnz) {
    blocked_mask_kernel<<<blocks_for(n_rows * 32, 256), 256, 0, s>>>(
        ptr, col, n_rows, transpose, out.n_chunks, out.off.ptr, out.data.ptr);
    KG_LAUNCH_CHECK();
    DeviceBuffer<uint16_t> prefix(nb * kRows, s);
    row_prefix_kernel<<<blocks_for(nb * 32, 256), 256, 0, s>>>(out.off.ptr, out.data.ptr, nb,
                                                               prefix.ptr);
    KG_LAUNCH_CHECK();
    blocked_values_kernel<<<blocks_for(n_rows * 32, 256), 256, 0, s>>>(
        ptr, col, val, n_rows, transpose, out.n_chunks, out.off.ptr, prefix.ptr, out.data.ptr);
    KG_LAUNCH_CHECK();
  }
}

void transpose_blocked(const Blocked& x, Blocked& out, cudaStream_t s) {
  out.rows = x.K;
  out.K = x.rows;
  out.n_tiles = (uint32_t)((out.rows + kRows - 1) / kRows);
  out.n_chunks = (uint32_t)((out.K + kChunk - 1) / kChunk);
  const uint64_t nb = (uint64_t)out.n_tiles * out.n_chunks;
  DeviceBuffer<uint32_t> counts(nb, s);
  transpose_count_kernel<<<blocks_for(nb * 32, 256), 256, 0, s>>>(
      x.off.ptr, x.data.ptr, x.n_chunks, out.n_tiles, out.n_chunks, counts.ptr);
  KG_LAUNCH_CHECK();
  out.off.alloc(nb + 1, s);
  block_units_kernel<<<blocks_for(nb + 1, 256), 256, 0, s>>>(counts.ptr, nb, out.off.ptr);
  KG_LAUNCH_CHECK();
  counts.reset();
  size_t temp = 0;
  KG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, out.off.ptr, out.off.ptr, nb + 1, s));
  DeviceBuffer<unsigned char> scratch(temp, s);
  KG_CUDA(cub::DeviceScan::ExclusiveSum(scratch.ptr, temp, out.off.ptr, out.off.ptr, nb + 1, s));
  uint64_t units = 0;
  KG_CUDA(cudaMemcpyAsync(&units, out.off.ptr + nb, 8, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  out.bytes = units * 16;
  out.data.alloc(std::max<uint64_t>(out.bytes, 16), s);
  // Padding past a block's values must read as zero (the expansion loads past the end).
  out.data.zero();
  transpose_fill_kernel<<<blocks_for(nb * 32, 256), 256, 0, s>>>(
      x.off.ptr, x.data.ptr, x.n_chunks, out.n_tiles, out.n_chunks, out.off.ptr, out.data.ptr);
  KG_LAUNCH_CHECK();
}

void spmm_tc(const SpmmArgs& a, cudaStream_t s) {
  const Blocked& b = *a.s;
  if (b.K == 0 || b.rows == 0) return;
  static std::once_flag attr;
  std::call_once(attr, [] {
    KG_CUDA(cudaFuncSetAttribute(spmm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSpSmemBytes));
  });
  if (a.ld_t % 4 != 0) fail(KG_ERR_INVALID, "spmm: D^T row stride must be a multiple of 4");
  Geometry geo;
  geo.n_tiles = b.n_tiles;
  geo.n_chunks = b.n_chunks;
  geo.seg_chunks = (uint32_t)std::min<uint64_t>(a.seg_chunks ? a.seg_chunks : b.n_chunks, b.n_chunks);
  geo.n_segs = (geo.n_chunks + geo.seg_chunks - 1) / geo.seg_chunks;
  if (a.out.mode == kOutRows && geo.n_segs != 1)
    fail(KG_ERR_INVALID, "spmm: row output needs one K segment");
  CUtensorMap mh = dt_map(a.dt_hi, b.K, a.ld_t), ml = dt_map(a.dt_lo, b.K, a.ld_t);
  DeviceBuffer<int> err(1, s);
  err.zero();
  uint64_t items = (uint64_t)geo.n_tiles * geo.n_segs;
  unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(items, (uint64_t)a.sm_count));
  spmm_tc_kernel<<<grid, kSpThreads, kSpSmemBytes, s>>>(mh, ml, b.off.ptr, b.data.ptr, b.rows,
                                                        geo, a.value_mode, a.row_means, a.out,
                                                        err.ptr);
  KG_LAUNCH_CHECK();
  int h = 0;
  KG_CUDA(cudaMemcpyAsync(&h, err.ptr, 4, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  if (h) fail(KG_ERR_TIMEOUT, "the tensor-core SpMM gave up waiting on its pipeline");
}

}  // namespace kg
