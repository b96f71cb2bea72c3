// The PCA's sparse x dense products on the 5th-generation tensor cores.
//
//   C (rows x 64) = S (rows x K, CSR, f32 values) . D (K x 64)
//
// S is the held input X (rows = cells, K = genes) for X Q and the embedding pass, or
// its gene-major twin X^T (rows = genes, K = cells) for X^T W and the sketch. D comes in
// as D^T (64 x K) split into two tf32 parts, hi + lo, each a K-major f32 matrix.
// Products run as three TF32 MMAs per tile (hi.hi + hi.lo + lo.hi: the f32 input to
// about 2^-21), accumulated in TMEM over at most kFlushChunks K-chunks and then added
// into f64 registers (so no f32 sum runs over more than 512 terms).
//
// The sparse operand is densified on chip: per 32-column K-chunk, four producer warps
// (one thread per row of the 128-row tile) zero their row of the shared-memory tile and
// scatter the row's entries of that chunk into it (the 128-byte-swizzled K-major
// layout the MMA reads), while TMA brings D^T's matching 64 x 32 tiles. HBM is read
// once per product: the sparse values and indices, and D^T.
//
// CTA (persistent, 320 threads): warps 0-3 densify, warps 4-7 drain TMEM (thread =
// row = TMEM lane), warp 8 TMA, warp 9 MMA. Work items: (row tile, K segment).
#include <cudaTypedefs.h>

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
constexpr int kStagesS = 4;
constexpr int kFlushChunks = 16;        // K-chunks summed in f32 before the f64 flush
constexpr uint32_t kABytes = kRows * 128;  // 16 KB: 128 rows x 32 f32
constexpr uint32_t kBBytes = kN * 128;     // 8 KB: 64 rows x 32 f32
constexpr int kProducerWarps = 4;
constexpr int kEpilogueWarps = 4;
constexpr int kSpThreads = (kProducerWarps + kEpilogueWarps + 2) * 32;
constexpr uint32_t kTmemColsS = 128;   // two 64-column f32 accumulators

struct Stage {
  uint8_t a_hi[kABytes];
  uint8_t a_lo[kABytes];
  uint8_t b_hi[kBBytes];
  uint8_t b_lo[kBBytes];
};

struct SpSmem {
  Stage st[kStagesS];
  double colsum[kEpilogueWarps][kN];
  uint64_t full[kStagesS], empty[kStagesS];
  uint64_t acc_full[2], acc_empty[2];
  uint64_t drained;
  uint32_t tmem_base;
  int abort;
};
constexpr size_t kSpSmemBytes = sizeof(SpSmem) + 1024;

__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// The byte offset of element kk (0..31) of row i in a 128-byte-swizzled K-major tile
// (8-row atoms of 1024 bytes; 16-byte chunk c of row i stored at chunk c ^ (i % 8)).
__device__ __forceinline__ uint32_t sw128_offset(uint32_t i, uint32_t kk) {
  return (i >> 3) * 1024u + (i & 7u) * 128u + ((((kk >> 2) ^ (i & 7u)) & 7u) << 4) +
         (kk & 3u) * 4u;
}

struct WorkItem {
  uint32_t tile;   // row tile
  uint32_t seg;    // K segment
};

__device__ __forceinline__ WorkItem work_item(uint64_t w, uint32_t n_tiles) {
  // Consecutive items share a K segment (its D^T tiles stay in L2 for the next tile).
  return WorkItem{(uint32_t)(w % n_tiles), (uint32_t)(w / n_tiles)};
}

template <class ColT>
__global__ void __launch_bounds__(kSpThreads, 1)
spmm_tc_kernel(const __grid_constant__ CUtensorMap tmap_hi,
               const __grid_constant__ CUtensorMap tmap_lo, const uint64_t* __restrict__ ptr,
               const ColT* __restrict__ col, const float* __restrict__ val, uint64_t rows,
               uint64_t K, uint64_t seg_len, SpmmOut out, int* error) {
  extern __shared__ uint8_t smem_raw[];
  SpSmem& sm = *reinterpret_cast<SpSmem*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint32_t n_tiles = (uint32_t)((rows + kRows - 1) / kRows);
  const uint32_t n_segs = (uint32_t)((K + seg_len - 1) / seg_len);
  const uint64_t n_items = (uint64_t)n_tiles * n_segs;
  volatile int* abort = &sm.abort;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStagesS; ++s) {
      mbar_init(&sm.full[s], kProducerWarps + 1);
      mbar_init(&sm.empty[s], 1);
    }
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

  // Chunks of a work item and the flush groups they form.
  auto chunks_of = [&](const WorkItem& wi) -> uint32_t {
    uint64_t k0 = (uint64_t)wi.seg * seg_len;
    uint64_t k1 = min(K, k0 + seg_len);
    return (uint32_t)((k1 - k0 + kChunk - 1) / kChunk);
  };

  if (warp < kProducerWarps) {
    // ----------------------------------------------------------- densify ------------
    const uint32_t i = threadIdx.x;  // row within the tile
    uint64_t it = 0;
    bool ok = true;
    for (uint64_t w = blockIdx.x; w < n_items && ok; w += gridDim.x) {
      WorkItem wi = work_item(w, n_tiles);
      const uint64_t row = (uint64_t)wi.tile * kRows + i;
      const uint64_t k0 = (uint64_t)wi.seg * seg_len;
      const uint64_t k1 = min(K, k0 + seg_len);
      uint64_t cur = 0, end = 0;
      if (row < rows) {
        cur = ptr[row];
        end = ptr[row + 1];
        if (k0 > 0) {  // first entry at or after k0
          uint64_t lo = cur, hi = end;
          while (lo < hi) {
            uint64_t mid = (lo + hi) >> 1;
            if ((uint64_t)col[mid] < k0) lo = mid + 1; else hi = mid;
          }
          cur = lo;
        }
      }
      const uint32_t nc = chunks_of(wi);
      for (uint32_t c = 0; c < nc; ++c, ++it) {
        const int s = (int)(it % kStagesS);
        const uint32_t ph = (uint32_t)((it / kStagesS) & 1);
        if (!mbar_wait(&sm.empty[s], ph ^ 1, abort)) {
          ok = false;
          break;
        }
        uint8_t* ahi = sm.st[s].a_hi;
        uint8_t* alo = sm.st[s].a_lo;
        // Zero this thread's 128-byte row in both parts.
        const uint32_t rbase = (i >> 3) * 1024u + (i & 7u) * 128u;
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          *reinterpret_cast<float4*>(ahi + rbase + q * 16) = z;
          *reinterpret_cast<float4*>(alo + rbase + q * 16) = z;
        }
        const uint64_t cend = min(k1, k0 + (uint64_t)(c + 1) * kChunk);
        const uint64_t cbeg = k0 + (uint64_t)c * kChunk;
        while (cur < end) {
          uint64_t kcol = (uint64_t)col[cur];
          if (kcol >= cend) break;
          float v = val[cur];
          float h = tf32_round(v);
          float l = v - h;
          uint32_t off = sw128_offset(i, (uint32_t)(kcol - cbeg));
          *reinterpret_cast<float*>(ahi + off) = h;
          *reinterpret_cast<float*>(alo + off) = l;
          ++cur;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.full[s]);
      }
    }
  } else if (warp < kProducerWarps + kEpilogueWarps) {
    // ----------------------------------------------------------- drain TMEM ---------
    const uint32_t quad = (uint32_t)warp & 3u;  // warps 4..7 -> TMEM lanes 32*quad..
    const uint32_t i = quad * 32u + lane;
    uint64_t fg = 0;
    bool ok = true;
    for (uint64_t w = blockIdx.x; w < n_items && ok; w += gridDim.x) {
      WorkItem wi = work_item(w, n_tiles);
      const uint64_t row = (uint64_t)wi.tile * kRows + i;
      double acc[kN];
#pragma unroll
      for (int j = 0; j < kN; ++j) acc[j] = 0.0;
      const uint32_t nc = chunks_of(wi);
      const uint32_t groups = (nc + kFlushChunks - 1) / kFlushChunks;
      for (uint32_t gr = 0; gr < groups; ++gr, ++fg) {
        const uint32_t b = (uint32_t)(fg & 1), bph = (uint32_t)((fg >> 1) & 1);
        if (!mbar_wait(&sm.acc_full[b], bph, abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          __syncwarp();
          float v[32];
          tmem_load_32(tmem + ((quad * 32u) << 16) + b * 64u + h * 32u, v);
#pragma unroll
          for (int j = 0; j < 32; ++j) acc[h * 32 + j] += (double)v[j];
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.acc_empty[b]);
      }
      if (!ok) break;
      // The work item's rows.
      if (out.mode == kOutRows) {
        // C = S D - offsets: the next product's D^T (hi/lo), the f32 rows, and this
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
          double sv = (double)hi + (double)lo;
          if (out.colsum_partial) {
            for (int o = 16; o; o >>= 1) sv += __shfl_xor_sync(0xFFFFFFFFu, sv, o);
            if (lane == 0) sm.colsum[quad][j] = sv;
          }
        }
        if (out.colsum_partial) {
          asm volatile("bar.sync 1, %0;" ::"n"(kEpilogueWarps * 32));
          if (quad == 0) {
            for (int j = lane; j < kN; j += 32) {
              double t = ((sm.colsum[0][j] + sm.colsum[1][j]) + sm.colsum[2][j]) + sm.colsum[3][j];
              out.colsum_partial[(uint64_t)wi.tile * kN + j] = t;
            }
          }
          asm volatile("bar.sync 1, %0;" ::"n"(kEpilogueWarps * 32));
        }
      } else {
        // Partial sums of this K segment, f64, one row of 64 per row of S.
        if (row < rows) {
          double* dst = out.partial + ((uint64_t)wi.seg * rows + row) * kN;
#pragma unroll
          for (int j = 0; j < kN; ++j) dst[j] = acc[j];
        }
      }
    }
  } else if (warp == kProducerWarps + kEpilogueWarps) {
    // ----------------------------------------------------------- TMA (D^T) ----------
    if (lane == 0) {
      prefetch_tmap(&tmap_hi);
      prefetch_tmap(&tmap_lo);
      uint64_t it = 0;
      int issued_phase[kStagesS];
      for (int s = 0; s < kStagesS; ++s) issued_phase[s] = -1;
      bool ok = true;
      for (uint64_t w = blockIdx.x; w < n_items && ok; w += gridDim.x) {
        WorkItem wi = work_item(w, n_tiles);
        const uint64_t k0 = (uint64_t)wi.seg * seg_len;
        const uint32_t nc = chunks_of(wi);
        for (uint32_t c = 0; c < nc; ++c, ++it) {
          const int s = (int)(it % kStagesS);
          const uint32_t ph = (uint32_t)((it / kStagesS) & 1);
          if (!mbar_wait(&sm.empty[s], ph ^ 1, abort)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&sm.full[s], 2 * kBBytes);
          const int32_t x = (int32_t)(k0 + (uint64_t)c * kChunk);
          tma_load_2d(sm.st[s].b_hi, &tmap_hi, &sm.full[s], x, 0);
          tma_load_2d(sm.st[s].b_lo, &tmap_lo, &sm.full[s], x, 0);
          issued_phase[s] = (int)ph;
        }
      }
      for (int s = 0; s < kStagesS; ++s) {
        if (issued_phase[s] < 0) continue;
        for (uint32_t q = 0; q < kWaitPolls && !mbar_try_wait(&sm.full[s], issued_phase[s]); ++q)
          __nanosleep(64);
      }
    }
  } else {
    // ----------------------------------------------------------- MMA ----------------
    if (lane == 0) {
      const uint32_t idesc = idesc_f32acc(2u, kRows, kN);  // tf32 x tf32 -> f32
      uint64_t it = 0, fg = 0;
      bool ok = true;
      for (uint64_t w = blockIdx.x; w < n_items && ok; w += gridDim.x) {
        WorkItem wi = work_item(w, n_tiles);
        const uint32_t nc = chunks_of(wi);
        for (uint32_t c = 0; c < nc && ok; ++c, ++it) {
          const uint32_t in_group = c % kFlushChunks;
          const uint32_t b = (uint32_t)(fg & 1), bph = (uint32_t)((fg >> 1) & 1);
          if (in_group == 0 && !mbar_wait(&sm.acc_empty[b], bph ^ 1, abort)) {
            ok = false;
            break;
          }
          const int s = (int)(it % kStagesS);
          const uint32_t ph = (uint32_t)((it / kStagesS) & 1);
          if (!mbar_wait(&sm.full[s], ph, abort)) {
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
      for (uint32_t q = 0; q < kWaitPolls && !mbar_try_wait(&sm.drained, 0); ++q) __nanosleep(64);
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

template <class ColT>
void launch(const SpmmArgs& a, const ColT* col, cudaStream_t s) {
  static std::once_flag attr;
  std::call_once(attr, [] {
    KG_CUDA(cudaFuncSetAttribute(spmm_tc_kernel<ColT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kSpSmemBytes));
  });
  if (a.ld_t % 4 != 0) fail(KG_ERR_INVALID, "spmm: D^T row stride must be a multiple of 4");
  CUtensorMap mh = dt_map(a.dt_hi, a.K, a.ld_t), ml = dt_map(a.dt_lo, a.K, a.ld_t);
  DeviceBuffer<int> err(1, s);
  err.zero();
  uint64_t n_tiles = (a.rows + kRows - 1) / kRows;
  uint64_t n_segs = (a.K + a.seg_len - 1) / a.seg_len;
  uint64_t items = n_tiles * n_segs;
  unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(items, (uint64_t)a.sm_count));
  spmm_tc_kernel<ColT><<<grid, kSpThreads, kSpSmemBytes, s>>>(mh, ml, a.ptr, col, a.val, a.rows,
                                                              a.K, a.seg_len, a.out, err.ptr);
  KG_LAUNCH_CHECK();
  int h = 0;
  KG_CUDA(cudaMemcpyAsync(&h, err.ptr, 4, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  if (h) fail(KG_ERR_TIMEOUT, "the tensor-core SpMM gave up waiting on its pipeline");
}

}  // namespace

void spmm_tc(const SpmmArgs& a, cudaStream_t s) {
  if (a.K == 0 || a.rows == 0) return;
  if (a.seg_len % kChunk != 0) fail(KG_ERR_INVALID, "spmm: segment length not a multiple of 32");
  if (a.col16)
    launch<uint16_t>(a, a.col16, s);
  else
    launch<uint32_t>(a, a.col32, s);
}

}  // namespace kg
