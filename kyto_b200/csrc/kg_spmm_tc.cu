// The PCA's sparse x dense products on the 5th-generation tensor cores.
//
//   C (rows x 64) = S (rows x K, sparse, f32 values) . D (K x 64)
//
// S is the held input X (rows = cells, K = genes) for X Q and the embedding pass, or X^T
// (rows = genes, K = cells) for X^T W, the sketch and the centred squares; both are kept
// in the blocked layout of kg_spmm_tc.cuh (128 rows x 32 columns per block). D comes as
// D^T (64 x K) in two tf32 parts (hi + lo), K-major f32. Each 128 x 32 tile of S is
// densified in shared memory and multiplied by three TF32 MMAs (hi.hi + hi.lo + lo.hi:
// the f32 operands to about 2^-21), accumulated in TMEM over at most kFlushChunks
// chunks and then added into f64 registers (no f32 sum runs over more than 512 terms).
//
// Per CTA (persistent, 320 threads) and per K-chunk of a work item (tile, K segment):
//   warp 8      TMA: the chunk's D^T tiles (64 x 32, two parts) and the block's entries
//               (one bulk copy of its indices, one of its values) into a stage;
//   warps 0-3   densify: zero the stage's 128 x 32 A tiles, then scatter the block's
//               entries into them (128-byte-swizzled K-major, the layout the MMA reads);
//   warp 9      MMA: 12 tcgen05.mma (kind::tf32, M=128 N=64 K=8) into one of two TMEM
//               accumulators;
//   warps 4-7   drain: TMEM -> f64 registers per flush group; at the end of the item the
//               rows (C - offsets, as tf32 parts of C^T, f32 rows and column sums) or the
//               segment's f64 partial.
// HBM sees each entry once per product (6 bytes) and D^T once per CTA pass (L2 serves
// the other tiles of a segment).
#include <cudaTypedefs.h>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
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
constexpr int kStagesS = 3;
constexpr int kFlushChunks = 16;        // K-chunks summed in f32 before the f64 flush
constexpr uint32_t kABytes = kRows * 128;  // 16 KB: 128 rows x 32 f32
constexpr uint32_t kBBytes = kN * 128;     // 8 KB: 64 rows x 32 f32
constexpr uint32_t kMaxEntries = kRows * kChunk;  // a full block (a multiple of 8)
constexpr int kProducerWarps = 4;
constexpr int kEpilogueWarps = 4;
constexpr int kSpThreads = (kProducerWarps + kEpilogueWarps + 2) * 32;
constexpr uint32_t kTmemColsS = 128;   // two 64-column f32 accumulators
constexpr uint16_t kPad = 0xFFFF;

struct Stage {
  uint8_t a_hi[kABytes];
  uint8_t a_lo[kABytes];
  uint8_t b_hi[kBBytes];
  uint8_t b_lo[kBBytes];
  float e_val[kMaxEntries];
  uint16_t e_idx[kMaxEntries];
};

struct SpSmem {
  Stage st[kStagesS];
  double colsum[2][kEpilogueWarps][kN];
  uint64_t load_full[kStagesS], a_ready[kStagesS], empty[kStagesS], zeroed[kStagesS];
  uint64_t cs_ready;
  uint64_t acc_full[2], acc_empty[2];
  uint64_t drained;
  uint32_t count[kStagesS];
  uint32_t tmem_base;
  int abort;
};
constexpr size_t kSpSmemBytes = sizeof(SpSmem) + 1024;

__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Byte offset of element kk (0..31) of row i in a 128-byte-swizzled K-major tile
// (8-row atoms of 1024 bytes; 16-byte chunk c of row i stored at chunk c ^ (i % 8)).
__device__ __forceinline__ uint32_t sw128_offset(uint32_t i, uint32_t kk) {
  return (i >> 3) * 1024u + (i & 7u) * 128u + ((((kk >> 2) ^ (i & 7u)) & 7u) << 4) +
         (kk & 3u) * 4u;
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
};

__global__ void __launch_bounds__(kSpThreads, 1)
spmm_tc_kernel(const __grid_constant__ CUtensorMap tmap_hi,
               const __grid_constant__ CUtensorMap tmap_lo, const uint64_t* __restrict__ off,
               const uint16_t* __restrict__ eidx, const float* __restrict__ evals,
               uint64_t rows, Geometry geo, int value_mode, const double* __restrict__ row_means,
               SpmmOut out, int* error) {
  extern __shared__ uint8_t smem_raw[];
  SpSmem& sm = *reinterpret_cast<SpSmem*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint64_t n_items = geo.items();
  volatile int* abort = &sm.abort;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStagesS; ++s) {
      mbar_init(&sm.load_full[s], 1);
      mbar_init(&sm.a_ready[s], kProducerWarps);
      mbar_init(&sm.empty[s], 1);
      mbar_init(&sm.zeroed[s], kProducerWarps);
    }
    mbar_init(&sm.cs_ready, kEpilogueWarps);
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sm.acc_full[b], 1);
      mbar_init(&sm.acc_empty[b], kEpilogueWarps);
    }
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
    // ----------------------------------------------------------- densify ------------
    const uint32_t t = threadIdx.x;  // 0..127
    uint64_t it = 0;
    bool ok = true;
    for (uint64_t w = blockIdx.x; w < n_items && ok; w += gridDim.x) {
      uint32_t tile, seg;
      geo.item(w, tile, seg);
      const uint32_t nc = geo.chunks(seg);
      for (uint32_t c = 0; c < nc; ++c, ++it) {
        const int s = (int)(it % kStagesS);
        const uint32_t ph = (uint32_t)((it / kStagesS) & 1);
        if (!mbar_wait(&sm.empty[s], ph ^ 1, abort)) {
          ok = false;
          break;
        }
        Stage& st = sm.st[s];
        // Zero the two A tiles: 32 KB, 16 stores of 16 bytes a thread.
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          reinterpret_cast<float4*>(st.a_hi)[q * 128 + t] = z;
          reinterpret_cast<float4*>(st.a_lo)[q * 128 + t] = z;
        }
        // Every producer warp's zeros land before any entry is scattered (bounded waits,
        // not a named barrier, so an aborted pipeline cannot strand a warp).
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.zeroed[s]);
        if (!mbar_wait(&sm.zeroed[s], ph, abort) || !mbar_wait(&sm.load_full[s], ph, abort)) {
          ok = false;
          break;
        }
        const uint32_t cnt = sm.count[s];
        for (uint32_t e = t; e < cnt; e += kProducerWarps * 32) {
          const uint16_t p = st.e_idx[e];
          if (p == kPad) continue;
          const uint32_t r = p >> 5, kk = p & 31u;
          float v = st.e_val[e];
          if (value_mode == kValueCentredSquare) {
            float d = v - (float)row_means[(uint64_t)tile * kRows + r];
            v = d * d;
          } else if (value_mode == kValueOne) {
            v = 1.0f;
          }
          const float h = tf32_round(v);
          const uint32_t o = sw128_offset(r, kk);
          *reinterpret_cast<float*>(st.a_hi + o) = h;
          *reinterpret_cast<float*>(st.a_lo + o) = v - h;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.a_ready[s]);
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
        uint32_t r0[32], r1[32];
        tmem_ld_32(tmem + ((quad * 32u) << 16) + b * 64u, r0);
        tmem_ld_32(tmem + ((quad * 32u) << 16) + b * 64u + 32u, r1);
        tmem_wait_ld();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.acc_empty[b]);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          acc[j] += (double)__uint_as_float(r0[j]);
          acc[32 + j] += (double)__uint_as_float(r1[j]);
        }
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
    // ----------------------------------------------------------- TMA ----------------
    if (lane == 0) {
      prefetch_tmap(&tmap_hi);
      prefetch_tmap(&tmap_lo);
      uint64_t it = 0;
      int issued_phase[kStagesS];
      for (int s = 0; s < kStagesS; ++s) issued_phase[s] = -1;
      bool ok = true;
      for (uint64_t w = blockIdx.x; w < n_items && ok; w += gridDim.x) {
        uint32_t tile, seg;
        geo.item(w, tile, seg);
        const uint32_t nc = geo.chunks(seg);
        for (uint32_t c = 0; c < nc; ++c, ++it) {
          const int s = (int)(it % kStagesS);
          const uint32_t ph = (uint32_t)((it / kStagesS) & 1);
          if (!mbar_wait(&sm.empty[s], ph ^ 1, abort)) {
            ok = false;
            break;
          }
          const uint32_t chunk = seg * geo.seg_chunks + c;
          const uint64_t b = (uint64_t)tile * geo.n_chunks + chunk;
          const uint64_t e0 = off[b];
          const uint32_t cnt = (uint32_t)(off[b + 1] - e0);
          sm.count[s] = cnt;
          mbar_arrive_expect_tx(&sm.load_full[s], 2 * kBBytes + cnt * 6u);
          const int32_t x = (int32_t)(chunk * kChunk);
          tma_load_2d(sm.st[s].b_hi, &tmap_hi, &sm.load_full[s], x, 0);
          tma_load_2d(sm.st[s].b_lo, &tmap_lo, &sm.load_full[s], x, 0);
          if (cnt) {
            bulk_load(sm.st[s].e_idx, eidx + e0, cnt * 2u, &sm.load_full[s]);
            bulk_load(sm.st[s].e_val, evals + e0, cnt * 4u, &sm.load_full[s]);
          }
          issued_phase[s] = (int)ph;
        }
      }
      for (int s = 0; s < kStagesS; ++s) {
        if (issued_phase[s] < 0) continue;
        for (uint32_t q = 0; q < kWaitPolls && !mbar_try_wait(&sm.load_full[s], issued_phase[s]); ++q)
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
          const int s = (int)(it % kStagesS);
          const uint32_t ph = (uint32_t)((it / kStagesS) & 1);
          if (!mbar_wait(&sm.load_full[s], ph, abort) || !mbar_wait(&sm.a_ready[s], ph, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t d = tmem + b * 64u;
          const uint32_t ah = smem_addr(sm.st[s].a_hi), al = smem_addr(sm.st[s].a_lo);
          const uint32_t bh = smem_addr(sm.st[s].b_hi), bl = smem_addr(sm.st[s].b_lo);
#pragma unroll
          for (int kk = 0; kk < kChunk / 8; ++kk) {
            const uint32_t o = kk * 32;
            mma_tf32(d, desc_k_sw128(ah + o), desc_k_sw128(bh + o), idesc, (in_group | kk) != 0);
            mma_tf32(d, desc_k_sw128(ah + o), desc_k_sw128(bl + o), idesc, 1);
            mma_tf32(d, desc_k_sw128(al + o), desc_k_sw128(bh + o), idesc, 1);
          }
          mma_commit(&sm.empty[s]);
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

// The block of each stored value, and its packed (row_in_tile << 5 | col_in_chunk).
__device__ __forceinline__ void locate(uint64_t r, uint32_t c, bool transpose, uint32_t n_chunks,
                                       uint64_t& block, uint16_t& packed) {
  uint64_t orow = transpose ? c : r;  // row of the output layout
  uint64_t ocol = transpose ? r : c;
  block = (orow / kRows) * n_chunks + ocol / kChunk;
  packed = (uint16_t)(((orow % kRows) << 5) | (ocol % kChunk));
}

// Entries per block (warp per CSR row; lanes whose entries share a block add once).
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
    uint16_t packed;
    uint32_t c = col[i];
    locate(r, c, transpose, n_chunks, block, packed);
    unsigned same = __match_any_sync(active, block);
    if ((unsigned)__ffs(same) - 1 == lane) atomicAdd(&counts[block], (uint32_t)__popc(same));
  }
}

__global__ void pad_counts_kernel(const uint32_t* counts, uint64_t n, uint64_t* padded) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) padded[i] = ((uint64_t)counts[i] + 7) & ~7ull;
  if (i == n) padded[i] = 0;
}

__global__ void blocked_fill_kernel(const uint64_t* ptr, const uint32_t* col, const float* val,
                                    uint64_t n_rows, bool transpose, uint32_t n_chunks,
                                    const uint64_t* off, uint32_t* cursor, uint16_t* out_idx,
                                    float* out_val) {
  uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  unsigned lane = threadIdx.x & 31u;
  if (r >= n_rows) return;
  for (uint64_t i0 = ptr[r]; i0 < ptr[r + 1]; i0 += 32) {
    uint64_t i = i0 + lane;
    bool in = i < ptr[r + 1];
    unsigned active = __ballot_sync(0xFFFFFFFFu, in);
    if (!in) continue;
    uint64_t block;
    uint16_t packed;
    locate(r, col[i], transpose, n_chunks, block, packed);
    unsigned same = __match_any_sync(active, block);
    unsigned leader = (unsigned)__ffs(same) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&cursor[block], (uint32_t)__popc(same));
    base = __shfl_sync(same, base, leader);
    uint64_t at = off[block] + base + __popc(same & ((1u << lane) - 1u));
    out_idx[at] = packed;
    out_val[at] = val[i];
  }
}

__global__ void fill_u16_kernel(uint16_t* p, uint64_t n, uint16_t v) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
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
  pad_counts_kernel<<<blocks_for(nb + 1, 256), 256, 0, s>>>(counts.ptr, nb, out.off.ptr);
  KG_LAUNCH_CHECK();
  size_t temp = 0;
  KG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, out.off.ptr, out.off.ptr, nb + 1, s));
  DeviceBuffer<unsigned char> scratch(temp, s);
  KG_CUDA(cub::DeviceScan::ExclusiveSum(scratch.ptr, temp, out.off.ptr, out.off.ptr, nb + 1, s));
  KG_CUDA(cudaMemcpyAsync(&out.nnz_padded, out.off.ptr + nb, 8, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  out.idx.alloc(std::max<uint64_t>(out.nnz_padded, 8), s);
  out.val.alloc(std::max<uint64_t>(out.nnz_padded, 8), s);
  fill_u16_kernel<<<std::min<unsigned>(blocks_for(out.idx.count, 256), 16384), 256, 0, s>>>(
      out.idx.ptr, out.idx.count, kPad);
  KG_LAUNCH_CHECK();
  out.val.zero();
  if (nnz) {
    counts.zero();  // reused as the per-block cursor
    blocked_fill_kernel<<<blocks_for(n_rows * 32, 256), 256, 0, s>>>(
        ptr, col, val, n_rows, transpose, out.n_chunks, out.off.ptr, counts.ptr, out.idx.ptr,
        out.val.ptr);
    KG_LAUNCH_CHECK();
  }
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
  spmm_tc_kernel<<<grid, kSpThreads, kSpSmemBytes, s>>>(mh, ml, b.off.ptr, b.idx.ptr, b.val.ptr,
                                                        b.rows, geo, a.value_mode, a.row_means,
                                                        a.out, err.ptr);
  KG_LAUNCH_CHECK();
  int h = 0;
  KG_CUDA(cudaMemcpyAsync(&h, err.ptr, 4, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  if (h) fail(KG_ERR_TIMEOUT, "the tensor-core SpMM gave up waiting on its pipeline");
}

}  // namespace kg
