// The PCA's sparse x dense products on the 5th-generation tensor cores.
//
//   C (rows x 64) = S (rows x K, sparse) . D (K x 64)
//
// S is the held input X (rows = cells, K = genes) for X Q and the embedding pass, or X^T
// (rows = genes, K = cells) for X^T W, the sketch and the gene statistics; both are kept
// in the pair-entry layout of kg_spmm_tc.cuh (128 rows x 32 columns a block: a header of
// (mask, base) words per row quarter and column pair, then one 8-byte entry per row and
// pair holding the fp16 hi/lo parts of both columns' scaled values). D comes as D^T in the
// same two fp16 parts (the dense layout of kg_spmm_tc.cuh). Each 128 x 32 block of S is
// expanded straight into tensor memory as a 128 x 32 hi tile and a lo tile (a lane per
// row; a lane without an entry for a pair writes the absent value, so the loads have no
// branches), and multiplied by three kind::f16 MMAs per 16 K that read A from TMEM and
// D^T from shared memory (hi.hi + hi.lo + lo.hi: both operands to about 2^-22, as three
// tf32 products give, at twice their rate), accumulated in TMEM over at most
// kFlushChunks chunks and then added into f64 registers (no f32 sum runs over more than
// 512 terms); the scales come off in f64 at the end (powers of two, exact).
//
// Per CTA (persistent, 576 threads) and per K-chunk of a work item (tile, K segment):
//   warp 16     loads: the chunk's D^T tile (64 x (32 hi + 32 lo) fp16, one TMA box) and
//               the block (one bulk copy) into one of kLoadStages stages;
//   warps 0-7   expand: the 128 x 32 block in row quarters and column pairs, from the
//               block's header words and entries into TMEM lanes of one of kABufs A
//               buffers (16 hi and 16 lo words a row, two fp16 a word);
//   warp 17     MMA: 6 tcgen05.mma (kind::f16, A from TMEM, M=128 N=64 K=16) into one of
//               two TMEM accumulators;
//   warps 8-15  drain: TMEM -> f64 registers per flush group, 32 columns a warp; at the
//               end of the item the rows (C - offsets, as the next product's D^T, f32 rows
//               and column sums) or the segment's f64 partial.
// HBM sees each block once per product (512 header bytes and 8 bytes an entry) and D^T
// about once per pass over it (L2 serves the other tiles of a segment).
#include <cuda_fp16.h>
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
#include "kg_tma.cuh"

namespace kg {

using namespace sm100;

int part_scale(double bound) {
  if (!(bound > 0.0) || !std::isfinite(bound)) return 0;
  int e = 0;
  std::frexp(bound, &e);  // bound in [2^(e-1), 2^e)
  return 15 - e;
}

namespace {

constexpr int kRows = 128;              // rows per tile (M)
constexpr int kChunk = 32;              // K per chunk (a block's columns)
constexpr int kN = 64;                  // output columns (N)
constexpr int kLoadStages = 8;
constexpr int kFlushChunks = 16;        // K-chunks summed in f32 before the f64 flush
constexpr uint32_t kBBytes = kN * 128;  // 8 KB: 64 rows x (32 hi + 32 lo) fp16
constexpr uint32_t kHeaderBytes = 64 * 8;  // (mask, base) per row quarter and column pair
constexpr uint32_t kBlockMaxBytes = kHeaderBytes + kRows * (kChunk / 2) * 8;
constexpr uint32_t kAbsentHi = 0x8000u;  // fp16 -0: the high part of a column without a value
// Two expand warps per sub-partition (rows 32 q.. of a block, half of its column pairs
// each) and two drain warps (rows 32 q.., half of the 64 output columns each).
constexpr int kExpandWarps = 8;
constexpr int kDrainWarps = 8;
constexpr int kSpThreads = (kExpandWarps + kDrainWarps + 2) * 32;
constexpr int kABufs = 4;
// TMEM columns: two 64-column f32 accumulators (0..127), then kABufs A buffers of 32
// columns (16 words of hi parts, then 16 of lo parts; lane = row of the tile).
constexpr uint32_t kTmemColsS = 256;
constexpr uint32_t kAccCols = 64, kABase = 128, kACols = 32;
static_assert(kABase + kABufs * kACols <= kTmemColsS, "TMEM columns");

struct LoadStage {
  uint8_t b[kBBytes];
  uint8_t blk[(kBlockMaxBytes + 1023) / 1024 * 1024];  // header, then the entries
};
// The expansion may read one entry past a full block's last.
static_assert(sizeof(LoadStage::blk) >= kBlockMaxBytes + 8, "stage room past the entries");
// Swizzled tiles (TMA destinations, MMA operands) start on 1024-byte boundaries.
static_assert(sizeof(LoadStage) % 1024 == 0, "load stage size");

struct SpSmem {
  LoadStage st[kLoadStages];
  double colsum[2][4][kN];  // per item parity, per 32-row quarter of the tile
  uint64_t ld_full[kLoadStages], ld_empty[kLoadStages];
  uint64_t a_full[kABufs], a_empty[kABufs];
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


// The two fp16 parts of x (hi = fp16(x), lo = fp16(x - hi)) in one word, hi low.
__device__ __forceinline__ uint32_t split_pair(float x) {
  const __half hi = __float2half_rn(x);
  const __half lo = __float2half_rn(x - __half2float(hi));
  return (uint32_t)__half_as_ushort(hi) | ((uint32_t)__half_as_ushort(lo) << 16);
}

struct ValueMap;
__device__ __forceinline__ uint2 map_entry(uint2 e, const ValueMap& vm, float mean_r);

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

// How the expansion maps each stored value: the mode, and for centred squares the factor
// that undoes S's scale and the one that scales the squares.
struct ValueMap {
  int mode;
  float unscale, sq_scale;
};

// An entry's two columns mapped by the value mode: kValueOne gives 1 where a column holds
// a value, kValueCentredSquare (v - mean_r)^2 scaled; a column without a value gives 0.
__device__ __forceinline__ uint2 map_entry(uint2 e, const ValueMap& vm, float mean_r) {
  uint32_t hx = 0, lx = 0;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const uint32_t hi = (e.x >> (16 * k)) & 0xFFFFu, lo = (e.y >> (16 * k)) & 0xFFFFu;
    if (hi == kAbsentHi) continue;
    uint32_t w = 0x3C00u;  // fp16 1.0, low part 0
    if (vm.mode == kValueCentredSquare) {
      const float v = __half2float(__ushort_as_half((unsigned short)hi)) +
                      __half2float(__ushort_as_half((unsigned short)lo));
      const float d = v * vm.unscale - mean_r;
      w = split_pair(d * d * vm.sq_scale);
    }
    hx |= (w & 0xFFFFu) << (16 * k);
    lx |= (w >> 16) << (16 * k);
  }
  return make_uint2(hx, lx);
}

// One CTA per SM, 18 warps: the register file is split over the SM's four sub-partitions
// (five warps on two of them), so 96 registers a thread; each drain warp keeps 32 f64
// sums, and two expand warps per sub-partition hide each other's latency.
__global__ void __launch_bounds__(kSpThreads, 1)
spmm_tc_kernel(const __grid_constant__ CUtensorMap tmap_dt, const uint64_t* __restrict__ off,
               const uint8_t* __restrict__ data, uint64_t rows, Geometry geo, ValueMap vmap,
               const double* __restrict__ row_means, double out_scale, SpmmOut out,
               int* error) {
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
      mbar_init(&sm.ld_empty[s], kExpandWarps + 1);  // the expanders and the MMA commit
    }
    for (int b = 0; b < kABufs; ++b) {
      mbar_init(&sm.a_full[b], kExpandWarps);
      mbar_init(&sm.a_empty[b], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sm.acc_full[b], 1);
      mbar_init(&sm.acc_empty[b], kDrainWarps);
    }
    mbar_init(&sm.cs_ready, kDrainWarps);
    mbar_init(&sm.drained, 1);
    sm.abort = 0;
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(&sm.tmem_base, kTmemColsS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;

  if (warp < kExpandWarps) {
    // ----------------------------------------------------------- expand -------------
    const uint32_t q = (uint32_t)warp & 3u;   // rows 32 q .. 32 q + 31 of each block
    const int hh = warp >> 2;                 // column pairs 8 hh .. 8 hh + 7
    const uint32_t lt = (1u << lane) - 1u;    // the lanes (rows) before this one
    const uint32_t lb = 1u << lane;
    uint64_t it = 0;
    bool ok = true;
    for (uint64_t w = blockIdx.x; w < n_items && ok; w += gridDim.x) {
      uint32_t tile, seg;
      geo.item(w, tile, seg);
      const uint32_t nc = geo.chunks(seg);
      float mean_r = 0.0f;
      if (vmap.mode == kValueCentredSquare) {
        const uint64_t row = (uint64_t)tile * kRows + q * 32u + lane;
        mean_r = row < rows ? (float)row_means[row] : 0.0f;
      }
      for (uint32_t c = 0; c < nc; ++c, ++it) {
        const int ls = (int)(it % kLoadStages);
        const uint32_t lph = (uint32_t)((it / kLoadStages) & 1);
        const uint32_t ab = (uint32_t)(it % kABufs), aph = (uint32_t)((it / kABufs) & 1);
        if (!mbar_wait(&sm.ld_full[ls], lph, abort) || !mbar_wait(&sm.a_empty[ab], aph ^ 1, abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const LoadStage& st = sm.st[ls];
        // This quarter's 16 (mask, base) words, two pairs a 16-byte load, and the entries.
        const uint4* hdr = reinterpret_cast<const uint4*>(st.blk) + q * 8;
        const uint2* ent = reinterpret_cast<const uint2*>(st.blk + kHeaderBytes);
        const bool present = sm.present[ls] != 0;
        // Row (32 q + lane) of the A tiles: pair p's high-part word to column p, its
        // low-part word to column 16 + p (a row without an entry for the pair: zeros).
        const uint32_t arow = tmem + ((q * 32u) << 16) + kABase + ab * kACols;
        {
          uint32_t hw[8], lw[8];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            // Every lane loads (no divergence): a lane without an entry reads the next
            // lane's, or one past the block's last entry (inside the stage buffer), and
            // drops it.
            const uint4 m = present ? hdr[4 * hh + i] : make_uint4(0u, 0u, 0u, 0u);
            uint2 e0 = ent[m.y + __popc(m.x & lt)];
            uint2 e1 = ent[m.w + __popc(m.z & lt)];
            if (vmap.mode != kValuePlain) {
              e0 = map_entry(e0, vmap, mean_r);
              e1 = map_entry(e1, vmap, mean_r);
            }
            const bool h0 = (m.x & lb) != 0, h1 = (m.z & lb) != 0;
            hw[2 * i] = h0 ? e0.x : 0u;
            lw[2 * i] = h0 ? e0.y : 0u;
            hw[2 * i + 1] = h1 ? e1.x : 0u;
            lw[2 * i + 1] = h1 ? e1.y : 0u;
          }
          tmem_st_8(arow + 8u * hh, hw);
          tmem_st_8(arow + 16u + 8u * hh, lw);
        }
        tmem_wait_st();
        tc_fence_before();
        __syncwarp();  // every lane has read the stage
        if (lane == 0) {
          mbar_arrive(&sm.a_full[ab]);
          mbar_arrive(&sm.ld_empty[ls]);
        }
      }
    }
  } else if (warp < kExpandWarps + kDrainWarps) {
    // ----------------------------------------------------------- drain TMEM ---------
    const uint32_t quad = (uint32_t)warp & 3u;  // TMEM lanes 32 quad .. (rows of the tile)
    const uint32_t half = (uint32_t)(warp - kExpandWarps) >> 2;  // columns 32 half ..
    constexpr int kH = kN / 2;
    const uint32_t i = quad * 32u + lane;
    uint64_t fg = 0, item_no = 0;
    bool ok = true;
    for (uint64_t w = blockIdx.x; w < n_items && ok; w += gridDim.x, ++item_no) {
      uint32_t tile, seg;
      geo.item(w, tile, seg);
      const uint64_t row = (uint64_t)tile * kRows + i;
      double acc[kH];
#pragma unroll
      for (int j = 0; j < kH; ++j) acc[j] = 0.0;
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
#pragma unroll
        for (int hf = 0; hf < 2; ++hf) {
          uint32_t rr[16];
          tmem_ld_16(tmem + ((quad * 32u) << 16) + b * kAccCols + half * kH + hf * 16u, rr);
          tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 16; ++j) acc[hf * 16 + j] += (double)__uint_as_float(rr[j]);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.acc_empty[b]);
      }
      if (!ok) break;
      if (out.mode == kOutRows) {
        // C = S D - offsets: the next product's D^T (fp16 parts), the f32 rows, and this
        // tile's column sums (fixed tree: warp shuffles, then the 4 quarters in order).
        const bool live = row < rows;
        const double t_mul = ldexp(1.0, out.t_scale), t_inv = ldexp(1.0, -out.t_scale);
        uint16_t* t_row = out.t ? out.t + (row / 32) * 64 + (row % 32) : nullptr;
#pragma unroll
        for (int jj = 0; jj < kH; ++jj) {
          const int j = (int)half * kH + jj;
          const double cval =
              live && j < (int)out.width ? acc[jj] * out_scale - out.offsets[j] : 0.0;
          double seen = cval;
          if (out.t) {
            const double y = cval * t_mul;
            const __half hi = __double2half(y);
            const __half lo = __double2half(y - (double)__half2float(hi));
            seen = ((double)__half2float(hi) + (double)__half2float(lo)) * t_inv;
            if (live) {
              t_row[(uint64_t)j * out.ld_t] = __half_as_ushort(hi);
              t_row[(uint64_t)j * out.ld_t + 32] = __half_as_ushort(lo);
            }
          }
          if (live && out.rows_f32 && j < (int)out.width)
            out.rows_f32[row * (uint64_t)out.width + j] = (float)cval;
          if (out.colsum_partial) {
            double sv = seen;
            for (int o = 16; o; o >>= 1) sv += __shfl_xor_sync(0xFFFFFFFFu, sv, o);
            if (lane == 0) sm.colsum[item_no & 1][quad][j] = sv;
          }
        }
        if (out.colsum_partial) {
          // The four quarters' sums in a fixed order (double-buffered by item, so a warp
          // running one item ahead cannot overwrite what the quarter-0 warps still read).
          __syncwarp();
          if (lane == 0) mbar_arrive(&sm.cs_ready);
          if (!mbar_wait(&sm.cs_ready, (uint32_t)(item_no & 1), abort)) break;
          if (quad == 0) {
            const double(*cs)[kN] = sm.colsum[item_no & 1];
            const int j = (int)half * kH + lane;
            const double tsum = ((cs[0][j] + cs[1][j]) + cs[2][j]) + cs[3][j];
            out.colsum_partial[(uint64_t)tile * kN + j] = tsum;
          }
        }
      } else if (row < rows) {
        double* dst = out.partial + ((uint64_t)seg * rows + row) * kN + half * kH;
#pragma unroll
        for (int j = 0; j < kH; ++j) dst[j] = acc[j] * out_scale;
      }
    }
  } else if (warp == kExpandWarps + kDrainWarps) {
    // ----------------------------------------------------------- loads --------------
    // Lane 0 issues; the warp reads the item's block offsets 32 at a time ahead of it.
    // (Prefetching the next 32 blocks into L2 ahead of their copies made the products 9%
    // slower on the 1M benchmark: part of it was evicted before use and read twice.)
    if (lane == 0) prefetch_tmap(&tmap_dt);
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
            mbar_arrive_expect_tx(&sm.ld_full[s], kBBytes + bytes);
            tma_load_2d(sm.st[s].b, &tmap_dt, &sm.ld_full[s], (int32_t)(chunk * 64), 0);
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
      const uint32_t idesc = idesc_f32acc(0u, kRows, kN);  // f16 x f16 -> f32
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
          const uint32_t ab = (uint32_t)(it % kABufs), aph = (uint32_t)((it / kABufs) & 1);
          if (!mbar_wait(&sm.ld_full[ls], lph, abort) || !mbar_wait(&sm.a_full[ab], aph, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem + b * kAccCols;
          const uint32_t ah = tmem + kABase + ab * kACols, al = ah + 16u;
          const uint32_t bs = smem_addr(sm.st[ls].b);
#pragma unroll
          for (int kk = 0; kk < kChunk / 16; ++kk) {
            // 16 K: 8 A columns (pairs), 32 bytes of a B row; B's lo parts 64 bytes on.
            const uint32_t o = kk * 32;
            mma_f16_ts(d, ah + kk * 8, desc_k_sw128(bs + o), idesc, (in_group | kk) != 0);
            mma_f16_ts(d, ah + kk * 8, desc_k_sw128(bs + 64 + o), idesc, 1);
            mma_f16_ts(d, al + kk * 8, desc_k_sw128(bs + o), idesc, 1);
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

// Per row: the sum of squared values (f64) into the largest so far, and the largest and
// smallest nonzero |value| (non-negative doubles compare as their bit patterns).
__global__ void csr_stats_kernel(const uint64_t* ptr, const float* val, uint64_t n_rows,
                                 unsigned long long* max_sq, unsigned long long* max_abs,
                                 unsigned long long* min_abs) {
  uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  if (r >= n_rows) return;
  double sq = 0.0, hi = 0.0, lo = INFINITY;
  for (uint64_t i = ptr[r] + lane; i < ptr[r + 1]; i += 32) {
    const double v = fabs((double)val[i]);
    sq += v * v;
    hi = fmax(hi, v);
    if (v > 0.0) lo = fmin(lo, v);
    if (v != v) hi = v;  // a NaN dominates
  }
  for (int o = 16; o; o >>= 1) {
    sq += __shfl_xor_sync(0xFFFFFFFFu, sq, o);
    const double h2 = __shfl_xor_sync(0xFFFFFFFFu, hi, o);
    hi = (hi != hi) ? hi : ((h2 != h2) ? h2 : fmax(hi, h2));
    lo = fmin(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
  }
  if (lane == 0) {
    atomicMax(max_sq, (unsigned long long)__double_as_longlong(sq));
    atomicMax(max_abs, (unsigned long long)__double_as_longlong(hi));
    atomicMin(min_abs, (unsigned long long)__double_as_longlong(lo));
  }
}

// A value's two fp16 parts (hi in bits 0-15, lo in 16-31) of x = v * 2^scale; a stored
// -0 becomes +0 (-0 marks a column without a value).
__device__ __forceinline__ uint32_t stored_parts(float v, int scale) {
  const float x = ldexpf(v, scale);
  return split_pair(x == 0.0f ? 0.0f : x);
}

// An entry from its two columns' parts words (kAbsentHi for a column without a value).
__device__ __forceinline__ uint2 make_entry(uint32_t w0, uint32_t w1) {
  return make_uint2((w0 & 0xFFFFu) | (w1 << 16), (w0 >> 16) | (w1 & 0xFFFF0000u));
}

__device__ __forceinline__ uint64_t lower_bound_u32(const uint32_t* a, uint64_t lo, uint64_t hi,
                                                    uint32_t v) {
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// ----- X: layout rows = CSR rows.

// Header masks: a warp per (tile, row quarter) walks its 32 rows one after another, the
// lanes over each row's values (coalesced), setting the row's bit in the quarter's words
// held in shared memory (a window of kMaskWindow chunks at a time); then the words go out
// 16 per chunk. Within one row every write sets the same bit, so no atomics are needed.
constexpr uint32_t kMaskWindow = 128;  // K-chunks a pass (8 KB of words a warp)
constexpr int kMaskWarps = 4;

__global__ void __launch_bounds__(kMaskWarps * 32)
rows_mask_kernel(const uint64_t* ptr, const uint32_t* col, uint64_t n_rows, uint32_t n_tiles,
                 uint32_t n_chunks, uint32_t* masks) {
  __shared__ uint32_t words[kMaskWarps][kMaskWindow * 16];
  const unsigned lane = threadIdx.x & 31u, wi = threadIdx.x >> 5;
  const uint64_t wq = (uint64_t)blockIdx.x * kMaskWarps + wi;
  if (wq >= (uint64_t)n_tiles * 4) return;
  const uint64_t tile = wq / 4, q = wq % 4;
  uint32_t* w = words[wi];
  for (uint32_t c0 = 0; c0 < n_chunks; c0 += kMaskWindow) {
    const uint32_t nch = min(kMaskWindow, n_chunks - c0);
    for (uint32_t x = lane; x < nch * 16; x += 32) w[x] = 0;
    __syncwarp();
    const uint32_t g_lo = c0 * kChunk, g_hi = (c0 + nch) * kChunk;
    for (uint32_t j = 0; j < 32; ++j) {
      const uint64_t r = tile * kRows + q * 32 + j;
      if (r >= n_rows) break;
      uint64_t a = ptr[r], e = ptr[r + 1];
      if (c0 > 0) a = lower_bound_u32(col, a, e, g_lo);
      for (uint64_t i = a + lane; i < e; i += 32) {
        const uint32_t c = col[i];
        if (c >= g_hi) break;
        const uint32_t x = (c / kChunk - c0) * 16 + (c % kChunk) / 2;
        w[x] |= 1u << j;
      }
      __syncwarp();
    }
    for (uint32_t x = lane; x < nch * 16; x += 32)
      masks[(tile * n_chunks + c0 + x / 16) * 64 + q * 16 + x % 16] = w[x];
    __syncwarp();
  }
}

// Entries: a warp per CSR row, the lanes over its values; the lane holding a pair's first
// value writes the whole entry.
__global__ void rows_values_kernel(const uint64_t* ptr, const uint32_t* col, const float* val,
                                   uint64_t n_rows, uint32_t n_chunks, const uint32_t* masks,
                                   const uint16_t* bases, const uint64_t* off, int scale,
                                   uint8_t* data) {
  const uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (r >= n_rows) return;
  const uint64_t tile = r / kRows;
  const uint32_t q = (uint32_t)((r % kRows) / 32), bit = (uint32_t)(r % 32);
  const uint32_t below = (1u << bit) - 1u;
  const uint64_t a = ptr[r], end = ptr[r + 1];
  for (uint64_t i = a + lane; i < end; i += 32) {
    const uint32_t c = col[i];
    // The pair's odd column after its even one: written with it.
    if (c % 2 == 1 && i > a && col[i - 1] == c - 1) continue;
    uint32_t w0 = kAbsentHi, w1 = kAbsentHi;
    if (c % 2 == 0) {
      w0 = stored_parts(val[i], scale);
      if (i + 1 < end && col[i + 1] == c + 1) w1 = stored_parts(val[i + 1], scale);
    } else {
      w1 = stored_parts(val[i], scale);
    }
    const uint64_t b = tile * n_chunks + c / kChunk;
    const uint64_t h = b * 64 + q * 16 + (c % kChunk) / 2;
    const uint32_t e = bases[h] + __popc(masks[h] & below);
    reinterpret_cast<uint2*>(data + off[b] * 16 + kHeaderBytes)[e] = make_entry(w0, w1);
  }
}

// ----- X^T: layout rows = CSR columns (genes), layout columns = CSR rows (cells). A warp
// per pair of CSR rows (one column pair of the layout), lane = a group of 32 genes (one
// header word of one block), found in each row by binary search.

// Header masks: the word of (gene group, cell pair) = the genes of the group either cell
// holds; each word written once, no atomics.
__global__ void cols_mask_kernel(const uint64_t* ptr, const uint32_t* col, uint64_t n_rows,
                                 uint32_t n_cols, uint32_t n_chunks, uint32_t* masks) {
  const uint64_t pr = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t r0 = 2 * pr;
  if (r0 >= n_rows) return;
  const bool has1 = r0 + 1 < n_rows;
  const uint64_t a0 = ptr[r0], e0 = ptr[r0 + 1];
  const uint64_t a1 = has1 ? ptr[r0 + 1] : 0, e1 = has1 ? ptr[r0 + 2] : 0;
  const uint32_t groups = (n_cols + 31) / 32;
  const uint64_t kch = r0 / kChunk;
  const uint32_t p = (uint32_t)((r0 % kChunk) / 2);
  for (uint32_t gg = lane; gg < groups; gg += 32) {
    const uint32_t g0 = gg * 32;
    uint32_t bits = 0;
    for (uint64_t i = lower_bound_u32(col, a0, e0, g0); i < e0 && col[i] < g0 + 32; ++i)
      bits |= 1u << (col[i] - g0);
    for (uint64_t i = lower_bound_u32(col, a1, e1, g0); i < e1 && col[i] < g0 + 32; ++i)
      bits |= 1u << (col[i] - g0);
    if (bits) masks[((uint64_t)(gg / 4) * n_chunks + kch) * 64 + (gg % 4) * 16 + p] = bits;
  }
}

// Entries: per gene either cell holds, one whole entry (the two cells' parts), merged in
// gene order.
__global__ void cols_values_kernel(const uint64_t* ptr, const uint32_t* col, const float* val,
                                   uint64_t n_rows, uint32_t n_cols, uint32_t n_chunks,
                                   const uint32_t* masks, const uint16_t* bases,
                                   const uint64_t* off, int scale, uint8_t* data) {
  const uint64_t pr = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t r0 = 2 * pr;
  if (r0 >= n_rows) return;
  const bool has1 = r0 + 1 < n_rows;
  const uint64_t a0 = ptr[r0], e0 = ptr[r0 + 1];
  const uint64_t a1 = has1 ? ptr[r0 + 1] : 0, e1 = has1 ? ptr[r0 + 2] : 0;
  const uint32_t groups = (n_cols + 31) / 32;
  const uint64_t kch = r0 / kChunk;
  const uint32_t p = (uint32_t)((r0 % kChunk) / 2);
  for (uint32_t gg = lane; gg < groups; gg += 32) {
    const uint32_t g0 = gg * 32;
    uint64_t i = lower_bound_u32(col, a0, e0, g0), j = lower_bound_u32(col, a1, e1, g0);
    const uint32_t gi = i < e0 ? col[i] : 0xFFFFFFFFu, gj = j < e1 ? col[j] : 0xFFFFFFFFu;
    if (min(gi, gj) >= g0 + 32) continue;
    const uint64_t b = (uint64_t)(gg / 4) * n_chunks + kch;
    const uint64_t h = b * 64 + (gg % 4) * 16 + p;
    const uint32_t m = masks[h], base = bases[h];
    uint2* ent = reinterpret_cast<uint2*>(data + off[b] * 16 + kHeaderBytes);
    for (;;) {
      const uint32_t ci = i < e0 ? col[i] : 0xFFFFFFFFu, cj = j < e1 ? col[j] : 0xFFFFFFFFu;
      const uint32_t g = min(ci, cj);
      if (g >= g0 + 32) break;
      uint32_t w0 = kAbsentHi, w1 = kAbsentHi;
      if (ci == g) w0 = stored_parts(val[i++], scale);
      if (cj == g) w1 = stored_parts(val[j++], scale);
      ent[base + __popc(m & ((1u << (g - g0)) - 1u))] = make_entry(w0, w1);
    }
  }
}

// Per block (warp): each header word's base (the entries of the words before it) and the
// block's size in 16-byte units (0 for a block without entries).
__global__ void pair_base_kernel(const uint32_t* masks, uint64_t n_blocks, uint16_t* bases,
                                 uint64_t* units) {
  const uint64_t b = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (b > n_blocks) return;
  if (b == n_blocks) {
    if (lane == 0) units[b] = 0;
    return;
  }
  const uint32_t c0 = __popc(masks[b * 64 + 2 * lane]), c1 = __popc(masks[b * 64 + 2 * lane + 1]);
  uint32_t incl = c0 + c1;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if ((int)lane >= o) incl += t;
  }
  const uint32_t excl = incl - c0 - c1;
  bases[b * 64 + 2 * lane] = (uint16_t)excl;
  bases[b * 64 + 2 * lane + 1] = (uint16_t)(excl + c0);
  const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
  if (lane == 0) units[b] = total ? (kHeaderBytes + 8ull * total + 15) / 16 : 0;
}

// Per block (warp): the header (every entry is then written whole by the values kernel).
__global__ void pair_header_kernel(const uint32_t* masks, const uint16_t* bases,
                                   const uint64_t* off, uint64_t n_blocks, uint8_t* data) {
  const uint64_t b = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (b >= n_blocks || off[b + 1] == off[b]) return;
  uint2* blk = reinterpret_cast<uint2*>(data + off[b] * 16);
  for (uint32_t h = lane; h < 64; h += 32) blk[h] = make_uint2(masks[b * 64 + h], bases[b * 64 + h]);
}

// The layout (rows x K) of the CSR (n_rows x n_cols) or of its transpose.
void build_pairs(const uint64_t* ptr, const uint32_t* col, const float* val, uint64_t n_rows,
                 uint64_t nnz, bool transposed, Blocked& out, cudaStream_t s) {
  out.n_tiles = (uint32_t)((out.rows + kRows - 1) / kRows);
  out.n_chunks = (uint32_t)((out.K + kChunk - 1) / kChunk);
  const uint64_t nb = (uint64_t)out.n_tiles * out.n_chunks;
  DeviceBuffer<uint32_t> masks(nb * 64, s);
  masks.zero();
  // Warps: one per (tile, row quarter) of X, or one per pair of CSR rows for X^T.
  const uint64_t warps = transposed ? (n_rows + 1) / 2 : (uint64_t)out.n_tiles * 4;
  if (nnz) {
    if (transposed)
      cols_mask_kernel<<<blocks_for(warps * 32, 256), 256, 0, s>>>(ptr, col, n_rows,
                                                                   (uint32_t)out.rows,
                                                                   out.n_chunks, masks.ptr);
    else
      rows_mask_kernel<<<(unsigned)((warps + kMaskWarps - 1) / kMaskWarps), kMaskWarps * 32, 0,
                         s>>>(ptr, col, n_rows, out.n_tiles, out.n_chunks, masks.ptr);
    KG_LAUNCH_CHECK();
  }
  DeviceBuffer<uint16_t> bases(nb * 64, s);
  out.off.alloc(nb + 1, s);
  pair_base_kernel<<<blocks_for((nb + 1) * 32, 256), 256, 0, s>>>(masks.ptr, nb, bases.ptr,
                                                                  out.off.ptr);
  KG_LAUNCH_CHECK();
  size_t temp = 0;
  KG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, out.off.ptr, out.off.ptr, nb + 1, s));
  DeviceBuffer<unsigned char> scratch(temp, s);
  KG_CUDA(cub::DeviceScan::ExclusiveSum(scratch.ptr, temp, out.off.ptr, out.off.ptr, nb + 1, s));
  uint64_t units = 0;
  KG_CUDA(cudaMemcpyAsync(&units, out.off.ptr + nb, 8, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  out.bytes = units * 16;
  out.data.alloc(std::max<uint64_t>(out.bytes, 16), s);
  if (!units) return;
  pair_header_kernel<<<blocks_for(nb * 32, 256), 256, 0, s>>>(masks.ptr, bases.ptr, out.off.ptr,
                                                              nb, out.data.ptr);
  KG_LAUNCH_CHECK();
  if (transposed)
    cols_values_kernel<<<blocks_for(warps * 32, 256), 256, 0, s>>>(
        ptr, col, val, n_rows, (uint32_t)out.rows, out.n_chunks, masks.ptr, bases.ptr,
        out.off.ptr, out.scale, out.data.ptr);
  else
    rows_values_kernel<<<blocks_for(n_rows * 32, 256), 256, 0, s>>>(
        ptr, col, val, n_rows, out.n_chunks, masks.ptr, bases.ptr, out.off.ptr, out.scale,
        out.data.ptr);
  KG_LAUNCH_CHECK();
}

}  // namespace

void build_blocked(const uint64_t* ptr, const uint32_t* col, const float* val, uint64_t n_rows,
                   uint64_t n_cols, uint64_t nnz, Blocked& out, cudaStream_t s) {
  out.rows = n_rows;
  out.K = n_cols;
  // The values' range (the scale of their fp16 parts) and the largest row norm.
  DeviceBuffer<unsigned long long> st(3, s);
  const unsigned long long init[3] = {0ull, 0ull, 0x7FF0000000000000ull};  // 0, 0, +inf
  KG_CUDA(cudaMemcpyAsync(st.ptr, init, sizeof init, cudaMemcpyHostToDevice, s));
  if (nnz) {
    csr_stats_kernel<<<blocks_for(n_rows * 32, 256), 256, 0, s>>>(ptr, val, n_rows, st.ptr,
                                                                  st.ptr + 1, st.ptr + 2);
    KG_LAUNCH_CHECK();
  }
  unsigned long long h_st[3];
  KG_CUDA(cudaMemcpyAsync(h_st, st.ptr, sizeof h_st, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  double d[3];
  std::memcpy(d, h_st, sizeof d);
  out.max_row_norm = std::sqrt(d[0]);
  out.max_abs = d[1];
  out.min_abs = std::isinf(d[2]) ? 0.0 : d[2];
  out.scale = part_scale(out.max_abs);
  build_pairs(ptr, col, val, n_rows, nnz, false, out, s);
}

void transpose_blocked(const uint64_t* ptr, const uint32_t* col, const float* val,
                       uint64_t n_rows, uint64_t n_cols, uint64_t nnz, const Blocked& x,
                       Blocked& out, cudaStream_t s) {
  out.rows = n_cols;
  out.K = n_rows;
  out.scale = x.scale;
  out.max_abs = x.max_abs;
  out.min_abs = x.min_abs;
  out.max_row_norm = 0.0;  // not tracked for the transpose
  build_pairs(ptr, col, val, n_rows, nnz, true, out, s);
}

void spmm_tc(const SpmmArgs& a, cudaStream_t s) {
  const Blocked& b = *a.s;
  if (b.K == 0 || b.rows == 0) return;
  static std::once_flag attr;
  std::call_once(attr, [] {
    KG_CUDA(cudaFuncSetAttribute(spmm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSpSmemBytes));
  });
  if (a.ld_t != dense_ld(b.K)) fail(KG_ERR_INVALID, "spmm: D^T row length must be dense_ld(K)");
  if (a.out.mode == kOutRows && a.out.t && a.out.ld_t != dense_ld(b.rows))
    fail(KG_ERR_INVALID, "spmm: the output D^T row length must be dense_ld(rows)");
  if (!a.error) fail(KG_ERR_INVALID, "spmm: no error flag");
  Geometry geo;
  geo.n_tiles = b.n_tiles;
  geo.n_chunks = b.n_chunks;
  geo.seg_chunks = (uint32_t)std::min<uint64_t>(a.seg_chunks ? a.seg_chunks : b.n_chunks, b.n_chunks);
  geo.n_segs = (geo.n_chunks + geo.seg_chunks - 1) / geo.seg_chunks;
  if (a.out.mode == kOutRows && geo.n_segs != 1)
    fail(KG_ERR_INVALID, "spmm: row output needs one K segment");
  // S's stored values enter the MMA times 2^a_scale (the stored scale, 0 for the ones,
  // a square's own scale for the centred squares), D^T times 2^dt_scale.
  ValueMap vm;
  vm.mode = a.value_mode;
  vm.unscale = ldexpf(1.0f, -b.scale);
  int a_scale = b.scale;
  vm.sq_scale = 1.0f;
  if (a.value_mode == kValueOne) {
    a_scale = 0;
  } else if (a.value_mode == kValueCentredSquare) {
    // (v - mean)^2 <= (|v| + |mean|)^2 <= (2 max|v|)^2.
    a_scale = part_scale(4.0 * b.max_abs * b.max_abs);
    vm.sq_scale = ldexpf(1.0f, a_scale);
  }
  const double out_scale = std::ldexp(1.0, -(a_scale + a.dt_scale));
  CUtensorMap m = tma_map_2d_16bit(a.dt, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, a.ld_t, kN,
                                   a.ld_t * 2, 64, kN);
  uint64_t items = (uint64_t)geo.n_tiles * geo.n_segs;
  unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(items, (uint64_t)a.sm_count));
  spmm_tc_kernel<<<grid, kSpThreads, kSpSmemBytes, s>>>(m, b.off.ptr, b.data.ptr, b.rows, geo, vm,
                                                        a.row_means, out_scale, a.out, a.error);
  KG_LAUNCH_CHECK();
}

}  // namespace kg
