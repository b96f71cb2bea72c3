// The exact-kNN candidate filter on the 5th-generation tensor cores (tcgen05, TMEM,
// TMA). It computes, for every (query, point) pair, an approximate key
//     A = |p|^2 - 2 q.p      (rows centred on the mean and scaled by a power of two)
// as ONE fp16 (or bf16) GEMM with f32 accumulation: the query operand is
// [-2 q, 1, 1, 1, 0...] and the point operand [p, h1, h2, h3, 0...] with h1+h2+h3 the
// point's squared norm split into three fp16 parts, so the norm is added by the tensor
// core and the epilogue reads finished keys straight from TMEM. The epilogue keeps
// kyto's filter state per query (neighbors_exact.rs:216-255): its k smallest keys and
// every point within twice the proven slack of the k-th, appended to the query's
// candidate slice. Candidates are then ranked by exact f64 keys (kg_knn.cu).
//
// Split operands (hi and lo fp16 parts of each component, two 64-wide sub-tiles per
// row) make the key three products, q_hi.p_hi + q_hi.p_lo + q_lo.p_hi, missing only
// q_lo.p_lo: the slack then comes from the f32 accumulation (about 2^-14 |q| R) rather
// than from fp16 rounding (2^-9 |q| R), which keeps the candidate sets near k where
// tight clusters sit far from the mean.
//
// CTA layout (one persistent CTA per SM, 320 threads):
//   warps 0-7  epilogue: thread t owns query t of the CTA's 256-query block (TMEM lane
//              32*(warp%4)+lane of accumulator warp/4);
//   warp 8     TMA producer: the block's two 128-query operand tiles, then 128-point
//              tiles through a ring of shared-memory stages;
//   warp 9     MMA issuer: per point tile, two M=128 N=128 K=64 products (one per
//              128-query half; three each with split operands) into one of two TMEM
//              accumulator buffers.
// TMEM: 2 buffers x (2 halves x 128 columns) = 512 columns, f32.
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "kg_internal.cuh"
#include "kg_knn.cuh"
#include "kg_knn_tc.cuh"
#include "kg_sm100.cuh"

namespace kg {

using namespace sm100;

constexpr int kTcQueries = (int)kTcQueryBlock;
constexpr int kTcPoints = 128;
constexpr int kTcK = 64;  // operand width (fp16 elements, one 128-byte swizzle row)
constexpr uint32_t kTileBytes = 128u * 128u;  // 128 rows x 64 fp16
constexpr int kEpiWarps = 8;
constexpr int kTcThreads = (kEpiWarps + 2) * 32;
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kEndOfBlock = 0xFFFFFFFFu;
constexpr uint32_t kNoBlock = 0xFFFFFFFFu;  // no query block left: the CTA's roles stop
enum : int { kAmSmem = kTcAmSmem, kAmTmem = kTcAmTmem, kAmHalf = kTcAmHalf };

// SUBS: 64-wide sub-tiles per operand row (1: fp16 or bf16; 2: split hi and lo). KR: the
// register top-k width (16, 32) or 0 (the k smallest in local memory, any k).
template <int KR, int SUBS>
struct TcShape {
  // Point-tile stages: eight where shared memory holds them (on the 1M benchmark
  // embedding, whose 128 MB point operand overflows L2, 166 ms against 168-178 ms with six
  // and 170 ms with seven).
  static constexpr int kStages = SUBS == 1 ? (KR == 32 ? 6 : 8) : (KR == 32 ? 2 : 3);
  static constexpr int kTopK = KR == 0 ? 1 : KR + 1;  // odd row stride: no bank conflicts
};

template <int KR, int SUBS>
struct TcSmem {
  static constexpr int kStages = TcShape<KR, SUBS>::kStages;
  uint8_t a[2][SUBS][kTileBytes];     // the query block's two 128-row halves
  uint8_t b[kStages][SUBS][kTileBytes];  // point tiles
  float scratch[kEpiWarps * 32][33];  // a thread's 32 keys when some may pass
  float topk[kEpiWarps * 32][TcShape<KR, SUBS>::kTopK];  // a thread's k smallest keys
  uint64_t full[kStages], empty[kStages];
  uint64_t tmem_full[4], tmem_empty[4];  // per accumulator slot (two to four in use)
  uint64_t a_full, a_empty, drained;
  uint32_t stage_tile[kStages];      // the point tile in a stage, or kEndOfBlock
  uint32_t acc_tile[4];              // the point tile in an accumulator slot, or kEndOfBlock
  uint32_t block_id[2];              // per block parity: the query block, or kNoBlock
  uint32_t acc_block[4];             // the query block of a slot's item
  // Per epilogue warp: the largest threshold + s^2 |q|^2 + slack of its live queries
  // (low word, f32 bits) in the query block of the high word. A value is used only by
  // that block's scan: an epilogue running behind (a short block before it) cannot
  // hand an older block's thresholds to the producer.
  unsigned long long u_pub[kEpiWarps];
  uint32_t tmem_base;
  int abort;
};
template <int KR, int SUBS>
constexpr size_t tc_smem_bytes() {
  return sizeof(TcSmem<KR, SUBS>) + 1024;  // + alignment slack
}
static_assert(tc_smem_bytes<32, 1>() <= 227 * 1024 && tc_smem_bytes<16, 1>() <= 227 * 1024 &&
                  tc_smem_bytes<0, 1>() <= 227 * 1024 && tc_smem_bytes<16, 2>() <= 227 * 1024 &&
                  tc_smem_bytes<32, 2>() <= 227 * 1024 && tc_smem_bytes<0, 2>() <= 227 * 1024,
              "filter shared memory");

__device__ __forceinline__ float round_up_f32d(double v) {
  float r = (float)v;
  if ((double)r < v) r = nextafterf(r, INFINITY);
  return r;
}

// The smallest of 32 keys held as f32 bits, by three-input minima (a tree, for
// independent instructions).
__device__ __forceinline__ float min3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
__device__ __forceinline__ float min_of_32(const uint32_t (&r)[32]) {
  float m[11];
#pragma unroll
  for (int i = 0; i < 10; ++i)
    m[i] = min3f(__uint_as_float(r[3 * i]), __uint_as_float(r[3 * i + 1]),
                 __uint_as_float(r[3 * i + 2]));
  m[10] = fminf(__uint_as_float(r[30]), __uint_as_float(r[31]));
  const float a = min3f(m[0], m[1], m[2]), b = min3f(m[3], m[4], m[5]);
  const float c = min3f(m[6], m[7], m[8]), d = fminf(m[9], m[10]);
  return fminf(min3f(a, b, c), d);
}

// Per-query filter state (kyto's Query, neighbors_exact.rs:196-255).
struct QueryState {
  float th;
  uint32_t n_small, count;
  bool overflowed;
};

constexpr uint32_t kCompactRound = 16;  // slice entries read per round of a compaction

// Compact the query's slice against its threshold (neighbors_exact.rs:236-252). It runs
// between tiles, when the slice may not hold another tile's keys (tc_make_room): entries
// above the threshold can never be neighbours and the re-rank skips any left in the
// slice, so compacting earlier would change nothing but the cost. Out of line, called
// where no tile's keys are live. The slice is read 16 entries a round, all loaded before
// any is written back (a write never passes the read position), so a round waits for its
// loads once instead of once an entry. The slice's base and cap are multiples of 16
// entries. More than half the slice kept: the query overflows.
__device__ __noinline__ void tc_compact(QueryState& st, float* ck, uint32_t* cr, uint32_t cap) {
  uint32_t kept = 0;
  for (uint32_t i = 0; i < st.count; i += kCompactRound) {
    float v[kCompactRound];
    uint32_t r[kCompactRound];
    if (i + kCompactRound <= st.count) {
#pragma unroll
      for (uint32_t j = 0; j < kCompactRound; j += 4) {
        const float4 a = *reinterpret_cast<const float4*>(ck + i + j);
        const uint4 b = *reinterpret_cast<const uint4*>(cr + i + j);
        v[j] = a.x, v[j + 1] = a.y, v[j + 2] = a.z, v[j + 3] = a.w;
        r[j] = b.x, r[j + 1] = b.y, r[j + 2] = b.z, r[j + 3] = b.w;
      }
    } else {
#pragma unroll
      for (uint32_t j = 0; j < kCompactRound; ++j) {
        const bool in = i + j < st.count;
        v[j] = in ? ck[i + j] : INFINITY;
        r[j] = in ? cr[i + j] : 0u;
      }
    }
#pragma unroll
    for (uint32_t j = 0; j < kCompactRound; ++j) {
      if (v[j] <= st.th) {
        ck[kept] = v[j];
        cr[kept] = r[j];
        ++kept;
      }
    }
  }
  st.count = kept;
  if (st.count > (cap >> 1)) st.overflowed = true;
}

// Every slice has room for a tile's keys at the start of each tile.
static_assert(kTcCap >= 2 * 128 && kTcRetrySplitCap >= 2 * 128 && kTcRetryCap >= 2 * 128,
              "a compacted slice keeps at most half its cap, and a tile appends 128 keys");

// Between tiles: compact the slice when another tile's keys might not fit.
__device__ __forceinline__ void tc_make_room(QueryState& st, float* ck, uint32_t* cr,
                                             uint32_t cap, uint32_t tile) {
  if (!st.overflowed && st.count > cap - tile) tc_compact(st, ck, cr, cap);
}

// Append candidate (key, p) (already <= st.th) to the query's slice, which has room for
// it (tc_make_room ran before the tile).
__device__ __forceinline__ void tc_append(QueryState& st, float key, uint32_t p, float* ck,
                                          uint32_t* cr) {
  ck[st.count] = key;
  cr[st.count] = p;
  ++st.count;
}

// Offer approximate key `key` of point `p` (already <= st.th) to the query's state: its
// k smallest keys in local memory (any k up to kMaxK).
__device__ __noinline__ void tc_offer(QueryState& st, float* smallest, uint32_t k,
                                      double slack2, float key, uint32_t p, float* ck,
                                      uint32_t* cr) {
  if (st.n_small < k || key < smallest[k - 1]) {
    if (st.n_small < k) ++st.n_small;
    uint32_t at = st.n_small - 1;
    while (at > 0 && smallest[at - 1] > key) {
      smallest[at] = smallest[at - 1];
      --at;
    }
    smallest[at] = key;
    if (st.n_small == k) st.th = round_up_f32d((double)smallest[k - 1] + slack2);
  }
  if (key <= st.th) tc_append(st, key, p, ck, cr);
}

// The points p0 .. p0 + 31 a query may take: bit j set when p0 + j lies in [lo, hi) and
// is not the query's own point slot.
__device__ __forceinline__ uint32_t tc_valid_bits(uint64_t p0, uint64_t self, uint64_t lo,
                                                  uint64_t hi) {
  uint32_t m = 0xFFFFFFFFu;
  if (p0 < lo || p0 + 32 > hi) {
    const uint32_t a = lo <= p0 ? 0u : (uint32_t)min(lo - p0, (uint64_t)32);
    const uint32_t b = hi <= p0 ? 0u : (uint32_t)min(hi - p0, (uint64_t)32);
    const uint32_t below_b = b >= 32 ? 0xFFFFFFFFu : (1u << b) - 1u;
    const uint32_t below_a = a >= 32 ? 0xFFFFFFFFu : (1u << a) - 1u;
    m = below_b & ~below_a;
  }
  if (self >= p0 && self < p0 + 32) m &= ~(1u << (uint32_t)(self - p0));
  return m;
}

// Offer the keys of one 32-point chunk selected by `mask` (bit j: point p0 + j, key
// keys[j]), in column order, to the query's state (k > 32: the k smallest in local
// memory, tc_offer); `mask` holds only points the query may take.
__device__ __forceinline__ void tc_offer_chunk(QueryState& st, float* smallest, uint32_t k,
                                               double slack2, const float* keys, uint32_t mask,
                                               uint64_t p0, float* ck, uint32_t* cr) {
  while (mask) {
    const int j = __ffs(mask) - 1;
    mask &= mask - 1;
    const float key = keys[j];
    if (key <= st.th) tc_offer(st, smallest, k, slack2, key, (uint32_t)(p0 + j), ck, cr);
  }
}

// Insert the keys of one 32-point chunk selected by `mask` (keys[j]) that fall below the
// query's k-th smallest, in column order. For k <= KR the query's k smallest keys live
// in the last k of KR slots (smallest[KR - k .. KR) in the thread's shared-memory slice,
// ascending, +inf past those seen; the first KR - k slots hold -inf), so the k-th
// smallest is always the last slot. They move into registers for the chunk: an
// insertion is 2 KR branch-free min/max (v[i] = max(v[i-1], min(v[i], key)) on the old
// values: the -inf slots stay -inf and the largest falls off the end). The threshold
// becomes the k-th + slack (one f32 add rounded up: never below the exact sum), and
// never rises (a bound from before, such as the first tile's, may be lower).
template <int KR>
__device__ __forceinline__ void tc_insert_chunk(float* smallest, float& kth, float& th,
                                                float sl2f, const float* keys, uint32_t mask) {
  float v[KR];
#pragma unroll
  for (int i = 0; i < KR; ++i) v[i] = smallest[i];
  bool changed = false;
  while (mask) {
    const int j = __ffs(mask) - 1;
    mask &= mask - 1;
    const float key = keys[j];
    if (key < kth) {
      float prev = v[0];
      v[0] = fminf(v[0], key);
#pragma unroll
      for (int i = 1; i < KR; ++i) {
        const float cur = v[i];
        v[i] = fmaxf(prev, fminf(cur, key));
        prev = cur;
      }
      kth = v[KR - 1];
      if (kth < INFINITY) th = fminf(th, __fadd_ru(kth, sl2f));
      changed = true;
    }
  }
  if (changed) {
#pragma unroll
    for (int i = 0; i < KR; ++i) smallest[i] = v[i];
  }
}

// The warp appends its lanes' selected keys of one chunk to their queries' slices: lane
// L's keys are rows[L][j] for the bits j of its mask (point p0 + j), and its query's slice
// starts at slot q0 + L. The warp writes one lane's keys at a time, a lane a key, in
// column order and contiguously from the lane's count (coalesced stores, no per-key
// loop). Every lane calls it; each lane's count grows by its keys. The slices have room
// (tc_make_room).
__device__ __forceinline__ void tc_warp_append(uint32_t mask, uint32_t& count,
                                               const float (*rows)[33], int lane, uint64_t q0,
                                               uint64_t p0, uint32_t cap, float* cand_key,
                                               uint32_t* cand_row) {
  uint32_t pend = __ballot_sync(0xFFFFFFFFu, mask != 0);
  while (pend) {
    const int L = __ffs(pend) - 1;
    pend &= pend - 1;
    const uint32_t m = __shfl_sync(0xFFFFFFFFu, mask, L);
    const uint32_t base = __shfl_sync(0xFFFFFFFFu, count, L);
    if ((m >> lane) & 1u) {
      const uint64_t at = (q0 + L) * cap + base + __popc(m & ((1u << lane) - 1u));
      cand_key[at] = rows[L][lane];
      cand_row[at] = (uint32_t)(p0 + lane);
    }
  }
  count += __popc(mask);
}

// KR: the register top-k width used on offers (k <= KR), or 0 for any k. SUBS: operand
// sub-tiles (1: one fp16/bf16 product; 2: split, three fp16 products). AM, where the
// query operand lives and how the accumulators are cut:
//   kAmSmem  A read from shared memory by every MMA; two accumulator slots of both
//            query halves (256 columns), each released by all eight epilogue warps;
//   kAmTmem  the query block's tiles copied into tensor memory once per block
//            (tcgen05.cp) and read there, so each MMA reads only its point tile from
//            shared memory (half the operand bytes at N = 128); three 128-column slots,
//            one query half each (a tile's two halves in consecutive slots), each
//            released by its half's four epilogue warps;
//   kAmHalf  A from shared memory, four 128-column half slots as with kAmTmem: the MMA
//            warp may run three half products ahead of the epilogue instead of two.
template <int KR, int SUBS, int AM>
__global__ void __launch_bounds__(kTcThreads, 1)
knn_filter_tc_kernel(const __grid_constant__ CUtensorMap tmap_q,
                     const __grid_constant__ CUtensorMap tmap_p, FilterScan scan, uint32_t k,
                     const float* __restrict__ slack2, uint32_t idesc, uint32_t cap,
                     float* cand_key, uint32_t* cand_row, uint32_t* cand_count,
                     float* threshold_out, int* error) {
  extern __shared__ uint8_t smem_raw[];
  // Aligned to 1024 bytes by an offset into the __shared__ array itself, so the compiler
  // keeps every access in the shared state space (no generic loads and stores).
  using Smem = TcSmem<KR, SUBS>;
  constexpr int kStages = Smem::kStages;
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u));
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const uint64_t n_q = scan.n_q, n_p = scan.n_p;
  const uint64_t n_qblocks = (n_q + kTcQueries - 1) / kTcQueries;
  const uint32_t n_tiles = (uint32_t)((n_p + kTcPoints - 1) / kTcPoints);
  volatile int* abort = &sm.abort;

  // TMEM columns with A in TMEM: the query halves' A operands (32 columns a 64-wide
  // sub-tile), then the three slots; with half slots and A in shared memory, four slots.
  constexpr bool TA = AM == kAmTmem;
  constexpr bool HS = AM != kAmSmem;
  constexpr uint32_t kHalfSlots = TA ? 3u : 4u;
  constexpr uint32_t kSlotBase = TA ? 64u * SUBS : 0u;
  static_assert(!HS || kSlotBase + kHalfSlots * 128 <= kTmemCols, "filter TMEM columns");
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], 1);
    }
    for (int b = 0; b < (HS ? (int)kHalfSlots : 2); ++b) {
      // Two arrivals: the MMA thread's own (releasing acc_tile) and the MMAs' commit.
      mbar_init(&sm.tmem_full[b], 2);
      mbar_init(&sm.tmem_empty[b], HS ? kEpiWarps / 2 : kEpiWarps);
    }
    mbar_init(&sm.a_full, 1);
    mbar_init(&sm.a_empty, 1);
    mbar_init(&sm.drained, 1);
    sm.abort = 0;
    for (int w = 0; w < kEpiWarps; ++w) sm.u_pub[w] = (unsigned long long)kNoBlock << 32;
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(&sm.tmem_base, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_base;
  volatile unsigned long long* u_pub = sm.u_pub;

  if (warp == kEpiWarps) {
    // ------------------------------------------------------------ TMA producer ----
    // Per query block: the two query tiles, then the block's point tiles in list order
    // (or every tile, from the block's own), then an end marker. With bounds, a tile
    // whose bound exceeds every query's threshold + s^2 |q|^2 is skipped (it holds no
    // neighbour: the thresholds only fall). Lane 0 issues; the warp reads the list 32
    // entries at a time ahead of it.
    if (lane == 0) {
      prefetch_tmap(&tmap_q);
      prefetch_tmap(&tmap_p);
    }
    uint64_t it = 0, loaded = 0;
    uint32_t bi = 0;
    int issued_phase[kStages];
    for (int s = 0; s < kStages; ++s) issued_phase[s] = -1;
    bool ok = true;
    // Query blocks: the CTA's first is its own index, the next ones come from a counter
    // shared by every CTA (blocks of very different list lengths then even out); the
    // block index goes to the MMA warp beside the query tiles, and kNoBlock when none is
    // left.
    for (;; ++bi) {
      uint64_t qb = 0;
      if (lane == 0) {
        ok = mbar_wait(&sm.a_empty, (bi & 1) ^ 1, abort);
        if (ok) {
          qb = bi == 0 ? (uint64_t)blockIdx.x
                       : (uint64_t)gridDim.x + atomicAdd(scan.block_counter, 1u);
          if (qb >= n_qblocks) {
            sm.block_id[bi & 1] = kNoBlock;
            mbar_arrive(&sm.a_full);
          } else {
            sm.block_id[bi & 1] = (uint32_t)qb;
            mbar_arrive_expect_tx(&sm.a_full, 2 * SUBS * kTileBytes);
            for (int h = 0; h < 2; ++h)
              for (int sub = 0; sub < SUBS; ++sub)
                tma_load_2d(sm.a[h][sub], &tmap_q, &sm.a_full, sub * kTcK,
                            (int32_t)(qb * kTcQueries + h * 128));
          }
        }
      }
      ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
      qb = __shfl_sync(0xFFFFFFFFu, qb, 0);
      if (!ok || qb >= n_qblocks) break;
      const uint64_t l0 = scan.list_off ? scan.list_off[qb] : qb * scan.list_stride;
      const uint64_t len = !scan.list_tiles ? n_tiles
                           : scan.list_off  ? scan.list_off[qb + 1] - l0
                                            : scan.list_stride;
      // The list is read 32 entries a window, the next window's loads issued a window
      // ahead (their latency hides behind 32 tiles).
      uint32_t win_tile = 0, nxt_tile = 0;
      float win_lb2 = 0.0f, nxt_lb2 = 0.0f;
      auto load_window = [&](uint64_t i0, uint32_t& t, float& b) {
        t = i0 + lane < len ? scan.list_tiles[l0 + i0 + lane] : 0u;
        b = (scan.list_lb2 && i0 + lane < len) ? scan.list_lb2[l0 + i0 + lane] : 0.0f;
      };
      if (scan.list_tiles) load_window(0, nxt_tile, nxt_lb2);
      for (uint64_t i = 0;; ++i) {
        const uint32_t at = (uint32_t)(i & 31);
        if (at == 0 && scan.list_tiles) {
          win_tile = nxt_tile;
          win_lb2 = nxt_lb2;
          if (i + 32 < len) load_window(i + 32, nxt_tile, nxt_lb2);
        }
        const uint32_t lt = __shfl_sync(0xFFFFFFFFu, win_tile, at);
        const float lb2 = __shfl_sync(0xFFFFFFFFu, win_lb2, at);
        if (i < len && scan.list_lb2) {
          // One lane reads the bounds (the epilogue may be writing them) and the warp
          // takes its value, so every lane makes the same choice.
          float u = 0.0f;
          if (lane == 0) {
            // All eight words loaded at once; a warp yet to publish for this block bounds
            // nothing.
            unsigned long long v[kEpiWarps];
#pragma unroll
            for (int w = 0; w < kEpiWarps; ++w) v[w] = u_pub[w];
            u = -INFINITY;
#pragma unroll
            for (int w = 0; w < kEpiWarps; ++w)
              u = (uint32_t)(v[w] >> 32) == (uint32_t)qb ? fmaxf(u, __uint_as_float((uint32_t)v[w]))
                                                         : INFINITY;
          }
          u = __shfl_sync(0xFFFFFFFFu, u, 0);
          if (lb2 > u) {
            // Ascending bounds: every later tile is skipped too (the thresholds only
            // fall), so the block's scan ends here.
            if (scan.list_sorted) i = len - 1;
            continue;
          }
        }
        bool end = false;
        if (lane == 0) {
          const int s = (int)(it % kStages);
          const uint32_t ph = (uint32_t)((it / kStages) & 1);
          if (!mbar_wait(&sm.empty[s], ph ^ 1, abort)) {
            ok = false;
          } else {
            end = i >= len;
            if (end) {
              sm.stage_tile[s] = kEndOfBlock;
              mbar_arrive(&sm.full[s]);
              issued_phase[s] = (int)ph;  // the stage's last phase: complete at once
            } else {
              // Without a list the scan starts at the query block's own tiles: with the
              // rows in a spatial order the nearest points come first.
              const uint32_t pt = scan.list_tiles
                                      ? lt
                                      : (uint32_t)((i + qb * (kTcQueries / kTcPoints)) % n_tiles);
              sm.stage_tile[s] = pt;
              mbar_arrive_expect_tx(&sm.full[s], SUBS * kTileBytes);
              for (int sub = 0; sub < SUBS; ++sub)
                tma_load_2d(sm.b[s][sub], &tmap_p, &sm.full[s], sub * kTcK,
                            (int32_t)(pt * kTcPoints));
              issued_phase[s] = (int)ph;
              ++loaded;
            }
          }
        }
        ok = __shfl_sync(0xFFFFFFFFu, ok, 0);
        end = __shfl_sync(0xFFFFFFFFu, end, 0);
        ++it;
        if (!ok || end) break;
      }
      if (!ok) break;
    }
    if (lane == 0 && scan.tiles_scanned) atomicAdd(scan.tiles_scanned, (unsigned long long)loaded);
    // Every load issued has landed before the CTA may leave (bounded, own loop).
    if (lane == 0) {
      for (int s = 0; s < kStages; ++s) {
        if (issued_phase[s] < 0) continue;
        for (uint32_t i = 0; i < kWaitPolls && !mbar_try_wait(&sm.full[s], issued_phase[s]); ++i)
          __nanosleep(64);
      }
    }
  } else if (warp == kEpiWarps + 1 && HS) {
    // ------------------------------------------------- MMA issuer (half slots) ------
    if (lane == 0) {
      uint64_t it = 0, item = 0;  // item: the slot sequence (two per tile, halves 0, 1)
      uint32_t bi = 0;
      bool ok = true;
      auto next_slot = [&](uint32_t& sl) -> bool {
        sl = (uint32_t)(item % kHalfSlots);
        return mbar_wait(&sm.tmem_empty[sl], (uint32_t)((item / kHalfSlots) & 1) ^ 1, abort);
      };
      auto marker = [&](uint32_t block) -> bool {
        for (int h = 0; h < 2; ++h) {
          uint32_t sl;
          if (!next_slot(sl)) return false;
          sm.acc_tile[sl] = kEndOfBlock;
          sm.acc_block[sl] = block;
          mbar_arrive(&sm.tmem_full[sl]);
          mbar_arrive(&sm.tmem_full[sl]);
          ++item;
        }
        return true;
      };
      for (;; ++bi) {
        if (!mbar_wait(&sm.a_full, bi & 1, abort)) break;
        tc_fence_after();
        const uint32_t qb = sm.block_id[bi & 1];
        if (qb == kNoBlock) {
          marker(kNoBlock);
          break;
        }
        if (TA) {
          // The block's query tiles into TMEM (after the previous block's MMAs, in issue
          // order); their shared memory goes back to the producer once the copies are
          // done.
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int sub = 0; sub < SUBS; ++sub) {
              const uint32_t asm_ = smem_addr(sm.a[h][sub]);
              const uint32_t at = tmem + (uint32_t)(h * 32 * SUBS + sub * 32);
#pragma unroll
              for (int kk = 0; kk < kTcK / 16; ++kk)
                tmem_cp_128x256b(at + kk * 8, desc_k_sw128(asm_ + kk * 32));
            }
          mma_commit(&sm.a_empty);
        }
        for (;; ++it) {
          const int s = (int)(it % kStages);
          const uint32_t ph = (uint32_t)((it / kStages) & 1);
          if (!mbar_wait(&sm.full[s], ph, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t pt = sm.stage_tile[s];
          if (pt == kEndOfBlock) {
            mbar_arrive(&sm.empty[s]);
            // A in shared memory: free once the block's MMAs are done.
            if (!TA) mma_commit(&sm.a_empty);
            ok = marker(qb);
            ++it;
            break;
          }
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            uint32_t sl;
            if (!next_slot(sl)) {
              ok = false;
              break;
            }
            tc_fence_after();
            sm.acc_tile[sl] = pt;
            sm.acc_block[sl] = qb;
            const uint32_t d = tmem + kSlotBase + sl * 128u;
            // Products (A sub-tile, B sub-tile): (0, 0) alone, or for split operands
            // (0, 0), (0, 1), (1, 0) (see below).
#pragma unroll
            for (int t = 0; t < (SUBS == 1 ? 1 : 3); ++t) {
              const int sa = t == 2 ? 1 : 0, sb = t == 1 ? 1 : 0;
              const uint32_t bsm = smem_addr(sm.b[s][sb]);
              if (TA) {
                const uint32_t a = tmem + (uint32_t)(h * 32 * SUBS + sa * 32);
#pragma unroll
                for (int kk = 0; kk < kTcK / 16; ++kk)
                  mma_f16_ts(d, a + kk * 8, desc_k_sw128(bsm + kk * 32), idesc, (t | kk) > 0);
              } else {
                const uint32_t asm_ = smem_addr(sm.a[h][sa]);
#pragma unroll
                for (int kk = 0; kk < kTcK / 16; ++kk)
                  mma_f16(d, desc_k_sw128(asm_ + kk * 32), desc_k_sw128(bsm + kk * 32), idesc,
                          (t | kk) > 0);
              }
            }
            if (h == 1) mma_commit(&sm.empty[s]);
            mbar_arrive(&sm.tmem_full[sl]);
            mma_commit(&sm.tmem_full[sl]);
            ++item;
          }
          if (!ok) break;
        }
        if (!ok) break;
      }
      // No product may still be running when TMEM is released.
      mma_commit(&sm.drained);
      for (uint32_t i = 0; i < kWaitPolls && !mbar_try_wait(&sm.drained, 0); ++i) __nanosleep(64);
    }
  } else if (warp == kEpiWarps + 1) {
    // ------------------------------------------------------------ MMA issuer ------
    if (lane == 0) {
      uint64_t it = 0;
      uint32_t bi = 0;
      bool ok = true;
      for (;; ++bi) {
        if (!mbar_wait(&sm.a_full, bi & 1, abort)) break;
        tc_fence_after();
        const uint32_t qb = sm.block_id[bi & 1];
        if (qb == kNoBlock) {
          // The end of the CTA's work goes to the epilogue through one accumulator.
          const uint32_t ab = (uint32_t)(it & 1), aph = (uint32_t)((it >> 1) & 1);
          if (!mbar_wait(&sm.tmem_empty[ab], aph ^ 1, abort)) break;
          sm.acc_tile[ab] = kEndOfBlock;
          sm.acc_block[ab] = kNoBlock;
          mbar_arrive(&sm.tmem_full[ab]);
          mbar_arrive(&sm.tmem_full[ab]);
          ++it;
          break;
        }
        for (;; ++it) {
          const int s = (int)(it % kStages);
          const uint32_t ph = (uint32_t)((it / kStages) & 1);
          const uint32_t ab = (uint32_t)(it & 1), aph = (uint32_t)((it >> 1) & 1);
          if (!mbar_wait(&sm.tmem_empty[ab], aph ^ 1, abort) ||
              !mbar_wait(&sm.full[s], ph, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t pt = sm.stage_tile[s];
          sm.acc_tile[ab] = pt;
          sm.acc_block[ab] = qb;
          if (pt == kEndOfBlock) {
            mbar_arrive(&sm.empty[s]);
            mbar_arrive(&sm.tmem_full[ab]);
            mbar_arrive(&sm.tmem_full[ab]);
            ++it;
            break;
          }
          const uint32_t d0 = tmem + ab * 256u, d1 = d0 + 128u;
          // Products (A sub-tile, B sub-tile): (0, 0) alone, or for split operands
          // [-2q_hi, 1, 1, 1 | -2q_lo] and [p_hi, h1, h2, h3 | p_lo] the pairs (0, 0),
          // (0, 1), (1, 0): q_hi.p_hi + norm, q_hi.p_lo, q_lo.p_hi (the norm columns meet
          // zeros in the other two).
#pragma unroll
          for (int t = 0; t < (SUBS == 1 ? 1 : 3); ++t) {
            const int sa = t == 2 ? 1 : 0, sb = t == 1 ? 1 : 0;
            const uint32_t bsm = smem_addr(sm.b[s][sb]);
            const uint32_t a0 = smem_addr(sm.a[0][sa]), a1 = smem_addr(sm.a[1][sa]);
#pragma unroll
            for (int kk = 0; kk < kTcK / 16; ++kk) {
              const uint64_t bd = desc_k_sw128(bsm + kk * 32);
              mma_f16(d0, desc_k_sw128(a0 + kk * 32), bd, idesc, (t | kk) > 0);
              mma_f16(d1, desc_k_sw128(a1 + kk * 32), bd, idesc, (t | kk) > 0);
            }
          }
          mma_commit(&sm.empty[s]);
          mbar_arrive(&sm.tmem_full[ab]);
          mma_commit(&sm.tmem_full[ab]);
        }
        if (!ok) break;
        mma_commit(&sm.a_empty);
      }
      // No product may still be running when TMEM is released.
      mma_commit(&sm.drained);
      for (uint32_t i = 0; i < kWaitPolls && !mbar_try_wait(&sm.drained, 0); ++i) __nanosleep(64);
    }
  } else {
    // ------------------------------------------------------------ epilogue --------
    // Per tile: the 128 keys come out of TMEM into registers and the accumulator is
    // released; a 32-key chunk whose minimum reaches the threshold (rare once it has
    // fallen) has its keys below the query's k-th smallest inserted by its lane and its
    // passing keys appended by the whole warp. The threshold, the k-th smallest and the
    // overflow flag stay in registers; after offers the warp publishes its largest
    // threshold + s^2 |q|^2 for the producer's bound checks, and a slice that might not
    // hold another tile's keys is compacted.
    const uint32_t half = (uint32_t)warp >> 2, quad = (uint32_t)warp & 3;
    // The warp's i-th item: with half slots, the half's slot sequence (items 2 i + half
    // of the MMA warp's, kHalfSlots slots of 128 columns); else the two shared slots,
    // this half's 128 columns of each.
    auto slot_of = [&](uint64_t i, uint32_t& sl, uint32_t& ph) {
      if (HS) {
        const uint64_t g = 2 * i + half;
        sl = (uint32_t)(g % kHalfSlots);
        ph = (uint32_t)((g / kHalfSlots) & 1);
      } else {
        sl = (uint32_t)(i & 1);
        ph = (uint32_t)((i >> 1) & 1);
      }
    };
    auto slot_cols = [&](uint32_t sl) -> uint32_t {
      return HS ? kSlotBase + sl * 128u : sl * 256u + half * 128u;
    };
    float* my = sm.scratch[threadIdx.x];
    float local_smallest[KR == 0 ? kMaxK : 1];
    float* smallest = KR == 0 ? local_smallest : sm.topk[threadIdx.x];
    uint64_t it = 0;
    uint32_t bi = 0;
    bool ok = true;
    for (;; ++bi) {
      // The block's first item names the block (or the end of the CTA's work).
      {
        uint32_t ab, aph;
        slot_of(it, ab, aph);
        if (!mbar_wait(&sm.tmem_full[ab], aph, abort)) break;
      }
      tc_fence_after();
      __syncwarp();
      uint32_t first_slot, first_ph;
      slot_of(it, first_slot, first_ph);
      const uint32_t qb32 = sm.acc_block[first_slot];
      if (qb32 == kNoBlock) {
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.tmem_empty[first_slot]);
        ++it;
        break;
      }
      const uint64_t qb = qb32;
      const uint64_t q = qb * kTcQueries + half * 128 + quad * 32 + lane;
      const bool active = q < n_q;
      const uint64_t self = active ? (scan.q_point ? scan.q_point[q] : q) : ~0ull;
      // The point slots the query may take (its own sample's, or every slot).
      uint64_t p_lo = 0, p_hi = n_p;
      if (active && scan.slot_sample) {
        const uint32_t smp = scan.slot_sample[q];
        p_lo = scan.sample_first[smp];
        p_hi = scan.sample_first[smp + 1];
      }
      const double s2qn2 = active && scan.qn2 ? scan.s2 * scan.qn2[q] : 0.0;
      QueryState st{INFINITY, 0, 0, false};
      if (KR > 0)
        for (int i = 0; i < KR; ++i) smallest[i] = i < KR - (int)k ? -INFINITY : INFINITY;
      float th = INFINITY, kth = INFINITY;  // kth: the k-th smallest key so far (k <= KR)
      bool live = active;  // not overflowed
      const double sl2 = active ? (double)slack2[q] : 0.0;
      // The doubled slack as an f32 (slack2 holds f32 values, so the conversion is exact).
      const float sl2f = (float)sl2;
      float* ck = cand_key + (active ? q : 0) * (uint64_t)cap;
      uint32_t* cr = cand_row + (active ? q : 0) * (uint64_t)cap;
      for (bool first = true;; ++it, first = false) {
        uint32_t ab, aph;
        slot_of(it, ab, aph);
        if (!first) {
          if (!mbar_wait(&sm.tmem_full[ab], aph, abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          __syncwarp();
        }
        const uint32_t pt = sm.acc_tile[ab];
        if (pt == kEndOfBlock) {
          __syncwarp();
          if (lane == 0) mbar_arrive(&sm.tmem_empty[ab]);
          ++it;
          break;
        }
        const uint32_t base = tmem + ((quad * 32u) << 16) + slot_cols(ab);
        // All 128 keys into registers with one wait; the accumulator goes back to the
        // MMA warp at once.
        uint32_t r[kTcPoints / 32][32];
#pragma unroll
        for (int c = 0; c < kTcPoints / 32; ++c) tmem_ld_32(base + c * 32u, r[c]);
        tmem_wait_ld();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&sm.tmem_empty[ab]);
        if (th == INFINITY && live) {
          // No threshold yet (the block's first tile): every key would be offered. The
          // tile's 128 keys in 16 groups of 8 have 16 minima at most M, so at least 16
          // keys, of which at most one is the query's own, lie at or below M: with every
          // point of the tile in the query's range and k (+1 when the query's own point is
          // in the tile) at most 16, the k-th smallest key of the scan is at most M, and
          // M + slack bounds every threshold the query will have. Only keys within it are
          // offered.
          const uint64_t t0 = (uint64_t)pt * kTcPoints;
          const uint32_t own = self >= t0 && self < t0 + kTcPoints ? 1u : 0u;
          if (t0 >= p_lo && t0 + kTcPoints <= p_hi && k + own <= 16u) {
            float m = -INFINITY;
#pragma unroll
            for (int c = 0; c < kTcPoints / 32; ++c)
#pragma unroll
              for (int g = 0; g < 4; ++g) {
                const uint32_t* e = &r[c][8 * g];
                const float a = min3f(__uint_as_float(e[0]), __uint_as_float(e[1]),
                                      __uint_as_float(e[2]));
                const float b = min3f(__uint_as_float(e[3]), __uint_as_float(e[4]),
                                      __uint_as_float(e[5]));
                m = fmaxf(m, min3f(a, b, fminf(__uint_as_float(e[6]), __uint_as_float(e[7]))));
              }
            th = __fadd_ru(m, (float)sl2);
          }
        }
        uint32_t hits = 0;
        float cmin[kTcPoints / 32];
#pragma unroll
        for (int c = 0; c < kTcPoints / 32; ++c) {
          cmin[c] = min_of_32(r[c]);
          hits |= (live && cmin[c] <= th ? 1u : 0u) << c;
        }
        const bool offered = __any_sync(0xFFFFFFFFu, hits != 0);
        if (offered) {
          // Chunk by chunk in column order: each lane with a key at most its threshold
          // copies the chunk's keys to its scratch row and selects the passing ones of
          // the points it may take; keys below its k-th smallest (rare once the threshold
          // has fallen) go into its k smallest one by one, the threshold falling with
          // them; then the warp appends every lane's selected keys. A key selected
          // against the threshold from before the chunk's insertions is kept even if the
          // threshold fell below it: the re-rank skips it.
#pragma unroll
          for (int c = 0; c < kTcPoints / 32; ++c) {
            const uint64_t p0 = (uint64_t)pt * kTcPoints + c * 32;
            uint32_t mask = 0;
            if (((hits >> c) & 1u) && live) {
#pragma unroll
              for (int j = 0; j < 32; ++j) {
                const float key = __uint_as_float(r[c][j]);
                my[j] = key;
                mask |= (key <= th ? 1u : 0u) << j;
              }
              mask &= tc_valid_bits(p0, self, p_lo, p_hi);
              if constexpr (KR > 0) {
                if (cmin[c] < kth) tc_insert_chunk<KR>(smallest, kth, th, sl2f, my, mask);
              } else {
                st.th = th;
                tc_offer_chunk(st, smallest, k, sl2, my, mask, p0, ck, cr);
                th = st.th;
              }
            }
            if constexpr (KR > 0) {
              __syncwarp();
              tc_warp_append(mask, st.count, &sm.scratch[warp * 32], lane, q - lane, p0, cap,
                             cand_key, cand_row);
              __syncwarp();
            }
          }
          if (live) {
            st.th = th;
            tc_make_room(st, ck, cr, cap, kTcPoints);
            live = !st.overflowed;
          }
        }
        if (offered && scan.list_lb2) {
          // A point is offered only if its key is at most th; its key is at least
          // s^2 (D - |q|^2) - slack, so no point farther than th + s^2 |q|^2 + slack
          // (scaled squared distance) can be. An overflowed query is searched in full
          // later: it no longer bounds the scan.
          const float u = active && live ? round_up_f32d((double)th + s2qn2 + sl2) : -INFINITY;
          float um = u;
          for (int o = 16; o; o >>= 1) um = fmaxf(um, __shfl_xor_sync(0xFFFFFFFFu, um, o));
          if (lane == 0) u_pub[warp] = ((unsigned long long)qb32 << 32) | __float_as_uint(um);
        }
      }
      if (active && ok) {
        cand_count[q] = st.overflowed ? kOverflow : st.count;
        threshold_out[q] = th;
      }
      if (!ok) break;
    }
  }
  __syncwarp();
  __syncthreads();
  if (sm.abort && threadIdx.x == 0) atomicExch(error, 1);
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kTmemCols);
  }
}

// ------------------------------------------------------------------ operands -------

// Rows centred (f64) and scaled by 2^e: the query operand [-2 q, 1, 1, 1, 0...] (with
// each query's centred squared norm, unscaled, f64, and its doubled slack in scaled
// units) or the point operand [p, h1, h2, h3, 0...] (fp16 or bf16). Slot r of the
// operand is row rows[r] of x (or row r).
template <class H>
__global__ void tc_operands_kernel(const float* x, uint64_t n, uint32_t width, uint32_t d,
                                   const uint32_t* rows, const double* mean, double scale,
                                   double u, double eta, const double* max_sq, bool query,
                                   H* out, double* qn2, float* slack2, double* slack_d) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  const float* xr = x + (uint64_t)(rows ? rows[r] : r) * width;
  double n2 = 0.0, n2s = 0.0;
  for (uint32_t j = 0; j < kTcK; ++j) {
    H v = H(0.0f);
    if (j < d) {
      double c = (double)xr[j] - mean[j];
      double cs = c * scale;
      n2 += c * c;
      n2s += cs * cs;
      const H b = H((float)cs);
      v = query ? H(-2.0f * (float)b) : b;  // -2b: exact, a power-of-two multiple
    }
    out[r * kTcK + j] = v;
  }
  if (!query) {
    // The squared norm in three parts (each rounded from what the previous left).
    double r1 = n2s;
    H h1 = H((float)r1);
    double r2 = r1 - (double)(float)h1;
    H h2 = H((float)r2);
    double r3 = r2 - (double)(float)h2;
    H h3 = H((float)r3);
    out[r * kTcK + d] = h1;
    out[r * kTcK + d + 1] = h2;
    out[r * kTcK + d + 2] = h3;
    return;
  }
  out[r * kTcK + d] = H(1.0f);
  out[r * kTcK + d + 1] = H(1.0f);
  out[r * kTcK + d + 2] = H(1.0f);
  qn2[r] = n2;
  // The bound of |A - s^2 (D - |q|^2)| (scaled units), D the exact squared distance:
  // quantisation 2(2u + u^2)|q||p| + 2 eta sqrt(d)(|q| + |p|) + 2 d eta^2, the norm's
  // three parts u^3 |p|^2 + 2 eta, the f32 accumulation gamma (2|q||p| + |p|^2) with
  // gamma = 2^-17 (64 terms, truncating adds), and f64 rounding of the exact key; |p|
  // bounded by the largest row norm R. Doubled, as kyto doubles its own.
  const double gamma = 0x1p-17, tiny = 0x1p-40;
  double qs = sqrt(n2s), rs = sqrt(*max_sq) * scale;
  double e = 2.0 * (2.0 * u + u * u) * qs * rs + 2.0 * eta * sqrt((double)d) * (qs + rs) +
             2.0 * d * eta * eta + 2.0 * u * u * u * rs * rs + 2.0 * eta +
             gamma * (2.02 * qs * rs + 1.02 * rs * rs) + tiny * (qs + rs) * (qs + rs);
  e *= 2.0;
  slack_d[r] = e / (scale * scale);
  slack2[r] = round_up_f32d(2.0 * e);
}

// The split operands, one warp per row (lane j: components j and j + 32): rows
// centred (f64) and scaled by 2^e, each component c as hi = fp16(c) and lo = fp16(c - hi).
// Query row [-2hi, 1, 1, 1, 0... | -2lo, 0...], point row [hi, h1, h2, h3, 0... | lo,
// 0...] (h1..h3 the scaled squared norm in three parts), 128 fp16 each; per query the
// centred squared norm (unscaled) and the slack.
__global__ void tc_split_operands_kernel(const float* x, uint64_t n, uint32_t width, uint32_t d,
                                         const uint32_t* rows, const double* mean, double scale,
                                         const double* max_sq, bool query, __half* out,
                                         double* qn2, float* slack2, double* slack_d) {
  const uint64_t r = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  if (r >= n) return;
  const float* xr = x + (uint64_t)(rows ? rows[r] : r) * width;
  double cs[2], n2 = 0.0, n2s = 0.0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t j = lane + 32u * h;
    cs[h] = 0.0;
    if (j < d) {
      const double c = (double)xr[j] - mean[j];
      cs[h] = c * scale;
      n2 += c * c;
      n2s += cs[h] * cs[h];
    }
  }
  for (int o = 16; o; o >>= 1) {
    n2 += __shfl_xor_sync(0xFFFFFFFFu, n2, o);
    n2s += __shfl_xor_sync(0xFFFFFFFFu, n2s, o);
  }
  // The squared norm in three parts (each rounded from what the previous left).
  const __half h1 = __float2half_rn((float)n2s);
  const double r2 = n2s - (double)__half2float(h1);
  const __half h2 = __float2half_rn((float)r2);
  const __half h3 = __float2half_rn((float)(r2 - (double)__half2float(h2)));
  __half* o = out + r * (2 * kTcK);
  const __half zero = __float2half_rn(0.0f), one = __float2half_rn(1.0f);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t j = lane + 32u * h;
    __half hi = zero, lo = zero, head = zero;
    if (j < d) {
      hi = __float2half_rn((float)cs[h]);
      lo = __float2half_rn((float)(cs[h] - (double)__half2float(hi)));
      if (query) {  // -2 hi, -2 lo: exact, a power-of-two multiple
        hi = __float2half_rn(-2.0f * __half2float(hi));
        lo = __float2half_rn(-2.0f * __half2float(lo));
      }
      head = hi;
    } else if (j < d + 3) {
      head = query ? one : (j == d ? h1 : j == d + 1 ? h2 : h3);
    }
    o[j] = head;
    o[kTcK + j] = lo;
  }
  if (!query || lane != 0) return;
  qn2[r] = n2;
  // The bound of |A - s^2 (D - |q|^2)| (scaled units): the dropped -2 lo.lo and the
  // components' residuals, 2((3u^2 + 5u^3)|q||p| + 2.01 eta sqrt(d)(|q| + |p|) + 10 d
  // eta^2) with u = 2^-11 (both roundings f64 -> f32 -> fp16) and eta = 2^-25 (fp16's
  // subnormal half-step); the norm's three parts u^3 |p|^2 + 2 eta; the f32
  // accumulation gamma (2|q||p| + |p|^2) with gamma = 2^-15 (three products of 64
  // terms in twelve K = 16 steps, truncating adds); and f64 rounding of the exact key;
  // |p| bounded by the largest row norm R. Doubled, as kyto doubles its own.
  const double u = 0x1p-11, eta = 0x1p-25, gamma = 0x1p-15, tiny = 0x1p-40;
  const double qs = sqrt(n2s), rs = sqrt(*max_sq) * scale, dd = (double)d;
  double e = 2.0 * (3.0 * u * u + 5.0 * u * u * u) * qs * rs +
             4.02 * eta * sqrt(dd) * (qs + rs) + 20.0 * dd * eta * eta +
             2.0 * u * u * u * rs * rs + 2.0 * eta + gamma * (2.02 * qs * rs + 1.02 * rs * rs) +
             tiny * (qs + rs) * (qs + rs);
  e *= 2.0;
  slack_d[r] = e / (scale * scale);
  slack2[r] = round_up_f32d(2.0 * e);
}

// The largest centred squared norm, f64.
__global__ void centred_norm_kernel(const float* x, uint64_t n, uint32_t width, uint32_t d,
                                    const double* mean, double* sq) {
  uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  double s = 0.0;
  for (uint32_t j = 0; j < d; ++j) {
    double c = (double)x[r * width + j] - mean[j];
    s += c * c;
  }
  sq[r] = s;
}

// ------------------------------------------------------------------ host -----------

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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

// A [rows x cols] 16-bit row-major matrix (cols a multiple of 64), boxes of 128 rows x
// 64 (one 128-byte swizzle row each), zero fill past the last row.
CUtensorMap tile_map(const void* base, uint64_t rows, bool bf16, uint32_t cols = kTcK) {
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  cuuint32_t box[2] = {(cuuint32_t)kTcK, 128};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(&m, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16,
                           2, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(KG_ERR_DEVICE, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return m;
}

}  // namespace

double tc_scale(const float* x, uint64_t n, uint32_t width, uint32_t d, const double* mean,
                double* max_sq, cudaStream_t s) {
  if (d + 3 > (uint32_t)kTcK) fail(KG_ERR_INVALID, "tensor-core filter: more than 61 components");
  DeviceBuffer<double> sq(n, s);
  centred_norm_kernel<<<blocks_for(n, 256), 256, 0, s>>>(x, n, width, d, mean, sq.ptr);
  KG_LAUNCH_CHECK();
  max_kernel_launch(sq.ptr, n, max_sq, s);
  double h_max = 0.0;
  KG_CUDA(cudaMemcpyAsync(&h_max, max_sq, 8, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  // Scale so that the largest centred row norm is at most 2^7: squared norms stay below
  // 2^14 (fp16's range) and -2q below 2^8.
  double scale = 1.0;
  if (h_max > 0.0 && std::isfinite(h_max)) {
    int e = 0;
    std::frexp(std::sqrt(h_max), &e);  // sqrt(h_max) < 2^e
    int shift = std::max(-1000, std::min(1000, 7 - e));
    scale = std::ldexp(1.0, shift);
  }
  return scale;
}

uint32_t filter_query_block(FilterKind) { return kTcQueryBlock; }

namespace {

template <int KR, int SUBS, int AM>
void launch_filter(unsigned grid, cudaStream_t s, const CUtensorMap& mq, const CUtensorMap& mp,
                   const FilterScan& scan, uint32_t k, const float* slack2, uint32_t idesc,
                   uint32_t cap, float* cand_key, uint32_t* cand_row, uint32_t* cand_count,
                   float* threshold, int* err) {
  static std::once_flag attr;
  std::call_once(attr, [] {
    KG_CUDA(cudaFuncSetAttribute(knn_filter_tc_kernel<KR, SUBS, AM>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tc_smem_bytes<KR, SUBS>()));
  });
  knn_filter_tc_kernel<KR, SUBS, AM><<<grid, kTcThreads, tc_smem_bytes<KR, SUBS>(), s>>>(
      mq, mp, scan, k, slack2, idesc, cap, cand_key, cand_row, cand_count, threshold, err);
}

// The filter's query operand and accumulator slots: KYTO_GPU_FILTER_A ("smem", "tmem"
// or "half") when set, else the scan's tuned mode, else shared memory (194 ms against
// 238 ms for "tmem" and 222 ms for "half" on the 1M benchmark search on a B200); all give
// the same keys.
int filter_a_mode(int tuned) {
  const char* v = std::getenv("KYTO_GPU_FILTER_A");
  if (v && std::string(v) == "tmem") return kAmTmem;
  if (v && std::string(v) == "half") return kAmHalf;
  if (v && std::string(v) == "smem") return kAmSmem;
  return tuned == kAmTmem || tuned == kAmHalf ? tuned : kAmSmem;
}

}  // namespace

void tc_filter(kg_ctx* ctx, cudaStream_t s, const float* x, uint32_t width, uint32_t d,
               const uint32_t* qrows, const uint32_t* prows, FilterScan scan,
               const double* mean, double scale, const double* max_sq, FilterKind kind,
               uint32_t k, uint32_t cap, float* cand_key, uint32_t* cand_row,
               uint32_t* cand_count, float* threshold, double* qn2, double* slack_d,
               Trace* trace, DeviceBuffer<uint16_t>* point_ops) {
  if (d + 3 > (uint32_t)kTcK) fail(KG_ERR_INVALID, "tensor-core filter: more than 61 components");
  const uint64_t n_q = scan.n_q, n_p = scan.n_p;
  const bool split = kind == FilterKind::Split, bf16 = kind == FilterKind::Bf16;
  const uint32_t width_op = split ? 2u * kTcK : (uint32_t)kTcK;
  // The point operands: built here, or the caller's from an earlier call on the same
  // points, kind, centre and scale (kept in *point_ops when given).
  DeviceBuffer<uint16_t> own;
  DeviceBuffer<uint16_t>& bp = point_ops ? *point_ops : own;
  const bool build_points = bp.count != n_p * width_op;
  if (build_points) bp.alloc(n_p * width_op, s);
  DeviceBuffer<uint16_t> aq(n_q * width_op, s);
  DeviceBuffer<float> slack2(n_q, s);
  if (split) {
    tc_split_operands_kernel<<<blocks_for(n_q * 32, 256), 256, 0, s>>>(
        x, n_q, width, d, qrows, mean, scale, max_sq, true, (__half*)aq.ptr, qn2, slack2.ptr,
        slack_d);
    if (build_points)
      tc_split_operands_kernel<<<blocks_for(n_p * 32, 256), 256, 0, s>>>(
          x, n_p, width, d, prows, mean, scale, max_sq, false, (__half*)bp.ptr, nullptr, nullptr,
          nullptr);
  } else {
    const double u = bf16 ? 0x1p-8 : 0x1p-11;
    const double eta = bf16 ? 0x1p-134 : 0x1p-25;
    if (bf16) {
      tc_operands_kernel<__nv_bfloat16><<<blocks_for(n_q, 128), 128, 0, s>>>(
          x, n_q, width, d, qrows, mean, scale, u, eta, max_sq, true, (__nv_bfloat16*)aq.ptr,
          qn2, slack2.ptr, slack_d);
      if (build_points)
        tc_operands_kernel<__nv_bfloat16><<<blocks_for(n_p, 128), 128, 0, s>>>(
            x, n_p, width, d, prows, mean, scale, u, eta, max_sq, false, (__nv_bfloat16*)bp.ptr,
            nullptr, nullptr, nullptr);
    } else {
      tc_operands_kernel<__half><<<blocks_for(n_q, 128), 128, 0, s>>>(
          x, n_q, width, d, qrows, mean, scale, u, eta, max_sq, true, (__half*)aq.ptr, qn2,
          slack2.ptr, slack_d);
      if (build_points)
        tc_operands_kernel<__half><<<blocks_for(n_p, 128), 128, 0, s>>>(
            x, n_p, width, d, prows, mean, scale, u, eta, max_sq, false, (__half*)bp.ptr, nullptr,
            nullptr, nullptr);
    }
  }
  KG_LAUNCH_CHECK();
  if (trace) trace->mark("filter operands");
  CUtensorMap mq = tile_map(aq.ptr, n_q, bf16, width_op), mp = tile_map(bp.ptr, n_p, bf16, width_op);
  DeviceBuffer<int> err(1, s);
  err.zero();
  DeviceBuffer<unsigned int> counter(1, s);
  counter.zero();
  scan.block_counter = counter.ptr;
  unsigned long long tiles_before = 0;
  if (trace_on() && scan.tiles_scanned)
    KG_CUDA(cudaMemcpyAsync(&tiles_before, scan.tiles_scanned, 8, cudaMemcpyDeviceToHost, s));
  scan.qn2 = qn2;
  scan.s2 = scale * scale;
  const uint64_t n_qblocks = (n_q + kTcQueries - 1) / kTcQueries;
  const unsigned grid = (unsigned)std::min<uint64_t>(n_qblocks, (uint64_t)ctx->sm_count);
  const uint32_t idesc = idesc_f32acc(bf16 ? 1u : 0u, 128, kTcPoints);
  const int kr = k <= 16 ? 16 : k <= 32 ? 32 : 0;
  auto pick = [&](auto am) {
    constexpr int AM = decltype(am)::value;
    return kr == 16 ? (split ? launch_filter<16, 2, AM> : launch_filter<16, 1, AM>)
           : kr == 32 ? (split ? launch_filter<32, 2, AM> : launch_filter<32, 1, AM>)
                      : (split ? launch_filter<0, 2, AM> : launch_filter<0, 1, AM>);
  };
  const int am = filter_a_mode(scan.a_mode);
  auto launch = am == kAmTmem   ? pick(std::integral_constant<int, kAmTmem>{})
                : am == kAmHalf ? pick(std::integral_constant<int, kAmHalf>{})
                                : pick(std::integral_constant<int, kAmSmem>{});
  launch(grid, s, mq, mp, scan, k, slack2.ptr, idesc, cap, cand_key, cand_row, cand_count,
         threshold, err.ptr);
  KG_LAUNCH_CHECK();
  if (trace) trace->mark("filter kernel");
  // The bounded host wait first: a copy into h_err must never outlive this frame.
  wait_stream(ctx, s);
  int h_err = 0;
  KG_CUDA(cudaMemcpyAsync(&h_err, err.ptr, 4, cudaMemcpyDeviceToHost, s));
  KG_CUDA(cudaStreamSynchronize(s));
  if (h_err) fail(KG_ERR_TIMEOUT, "the tensor-core kNN filter gave up waiting on its pipeline");
  if (trace_on() && scan.tiles_scanned) {
    unsigned long long h_tiles = 0;
    KG_CUDA(cudaMemcpyAsync(&h_tiles, scan.tiles_scanned, 8, cudaMemcpyDeviceToHost, s));
    KG_CUDA(cudaStreamSynchronize(s));
    h_tiles -= tiles_before;
    const double all = (double)n_qblocks * (double)((n_p + kTcPoints - 1) / kTcPoints);
    std::fprintf(stderr, "[kyto_gpu trace] filter %s: %llu block-tile products of %.0f (%.2f%%)%s\n",
                 split ? "split" : bf16 ? "bf16" : "fp16", h_tiles, all, 100.0 * h_tiles / all,
                 scan.list_lb2 ? ", with bounds" : "");
  }
}

}  // namespace kg
